"""ORACLE -- test infrastructure only.

MPI datatypes described from the MPI-3.1 standard (section 4.1), with no MPI
library involved.  Each ``OType`` knows its size, lb/ub, true bounds and can
expand its type map into the byte offsets that MPI_Pack visits, in order
(``byte_offsets``).  This is the independent check on the packed byte order
that the reference pins against "the system MPI_Pack" in
test/pack_unpack.cpp:62-97.

The same descriptions are lowered to the node array of ``typemap.c``
(``lower``) for large cases and for the timed CPU baseline.
"""
from __future__ import annotations

import numpy as np

ORDER_C = 56
ORDER_FORTRAN = 57


class OType:
    """One MPI datatype.  ``kind`` is the constructor name."""

    def __init__(self, kind, params, children, size, lb, ub, tlb, tub):
        self.kind = kind
        self.params = params
        self.children = children
        self.size = int(size)
        self.lb = int(lb)
        self.ub = int(ub)
        self.true_lb = int(tlb)
        self.true_ub = int(tub)

    @property
    def extent(self):
        return self.ub - self.lb

    # ---- type map -----------------------------------------------------
    def displacements(self):
        """(displacements, child) pairs: the ordered copies of children."""
        k, p = self.kind, self.params
        if k == "named":
            return []
        if k in ("dup", "resized"):
            return [(np.zeros(1, np.int64), self.children[0])]
        if k == "struct":
            out = []
            for bl, d, c in zip(p["bls"], p["displs"], self.children):
                out.append((d + c.extent * np.arange(bl, dtype=np.int64), c))
            return out
        c = self.children[0]
        e = c.extent
        if k == "contiguous":
            return [(e * np.arange(p["count"], dtype=np.int64), c)]
        if k in ("vector", "hvector"):
            stride = p["stride"] * e if k == "vector" else p["stride"]
            j = np.arange(p["count"], dtype=np.int64)[:, None] * stride
            kk = np.arange(p["bl"], dtype=np.int64)[None, :] * e
            return [((j + kk).ravel(), c)]
        if k in ("indexed", "hindexed", "indexed_block", "hindexed_block"):
            scale = e if k in ("indexed", "indexed_block") else 1
            parts = [
                d * scale + e * np.arange(bl, dtype=np.int64)
                for bl, d in zip(p["bls"], p["displs"])
            ]
            d = np.concatenate(parts) if parts else np.zeros(0, np.int64)
            return [(d, c)]
        if k == "subarray":
            sizes, subs, starts = p["sizes"], p["subsizes"], p["starts"]
            nd = len(sizes)
            # element stride of each dimension, in bytes
            strides = []
            for d in range(nd):
                s = e
                rng = range(d + 1, nd) if p["order"] == ORDER_C else range(0, d)
                for j in rng:
                    s *= sizes[j]
                strides.append(s)
            axes = [
                (starts[d] + np.arange(subs[d], dtype=np.int64)) * strides[d]
                for d in range(nd)
            ]
            # C order: last index fastest; Fortran: first index fastest
            order = range(nd) if p["order"] == ORDER_C else reversed(range(nd))
            disp = np.zeros(1, np.int64)
            for d in order:
                disp = (disp[:, None] + axes[d][None, :]).ravel()
            return [(disp, c)]
        raise ValueError(k)

    def byte_offsets(self):
        """Offsets (from the origin) of every byte MPI_Pack copies, in order."""
        if self.kind == "named":
            return np.arange(self.size, dtype=np.int64)
        parts = []
        for d, c in self.displacements():
            co = c.byte_offsets()
            parts.append((d[:, None] + co[None, :]).ravel())
        return np.concatenate(parts) if parts else np.zeros(0, np.int64)


def _bounds(pairs, size):
    lb = ub = tlb = tub = None
    for d, c in pairs:
        if len(d) == 0 or (c.size == 0 and c.extent == 0):
            continue
        lo, hi = int(d.min()), int(d.max())
        vals = (lo + c.lb, hi + c.ub, lo + c.true_lb, hi + c.true_ub)
        if lb is None:
            lb, ub, tlb, tub = vals
        else:
            lb, ub = min(lb, vals[0]), max(ub, vals[1])
            tlb, tub = min(tlb, vals[2]), max(tub, vals[3])
    if lb is None:
        return 0, 0, 0, 0
    return lb, ub, tlb, tub


def _make(kind, params, children):
    t = OType(kind, params, children, 0, 0, 0, 0, 0)
    pairs = t.displacements()
    t.size = sum(len(d) * c.size for d, c in pairs)
    t.lb, t.ub, t.true_lb, t.true_ub = _bounds(pairs, t.size)
    return t


def named(size):
    return OType("named", {"size": size}, [], size, 0, size, 0, size)


BYTE = named(1)
CHAR = named(1)
INT = named(4)
FLOAT = named(4)
DOUBLE = named(8)


def contiguous(count, old):
    return _make("contiguous", {"count": count}, [old])


def vector(count, bl, stride, old):
    return _make("vector", {"count": count, "bl": bl, "stride": stride}, [old])


def hvector(count, bl, stride, old):
    return _make("hvector", {"count": count, "bl": bl, "stride": stride}, [old])


def indexed(bls, displs, old):
    return _make("indexed", {"bls": list(bls), "displs": list(displs)}, [old])


def hindexed(bls, displs, old):
    return _make("hindexed", {"bls": list(bls), "displs": list(displs)}, [old])


def indexed_block(bl, displs, old):
    return _make(
        "indexed_block", {"bls": [bl] * len(displs), "displs": list(displs)}, [old]
    )


def hindexed_block(bl, displs, old):
    return _make(
        "hindexed_block", {"bls": [bl] * len(displs), "displs": list(displs)}, [old]
    )


def struct(bls, displs, types):
    return _make("struct", {"bls": list(bls), "displs": list(displs)}, list(types))


def subarray(sizes, subsizes, starts, order, old):
    p = {
        "sizes": list(sizes),
        "subsizes": list(subsizes),
        "starts": list(starts),
        "order": order,
    }
    t = _make("subarray", p, [old])
    # MPI-3.1 4.1.3: the subarray spans the full array, lb 0
    full = int(np.prod(sizes)) * old.extent
    t.lb, t.ub = 0, full
    return t


def resized(old, lb, extent):
    t = OType(
        "resized", {"lb": lb, "extent": extent}, [old], old.size, lb, lb + extent,
        old.true_lb, old.true_ub,
    )
    return t


def dup(old):
    return OType(
        "dup", {}, [old], old.size, old.lb, old.ub, old.true_lb, old.true_ub
    )


# ---- packing with the numpy expansion (small cases) ---------------------


def pack(t: OType, buf: np.ndarray, incount: int, origin: int = 0) -> np.ndarray:
    """MPI_Pack of ``incount`` objects whose origin is ``buf[origin]``."""
    offs = t.byte_offsets()
    allo = (np.arange(incount, dtype=np.int64) * t.extent)[:, None] + offs[None, :]
    return buf[origin + allo.ravel()].copy()


def unpack(t: OType, packed: np.ndarray, buf: np.ndarray, incount: int,
           origin: int = 0) -> None:
    """MPI_Unpack into ``buf`` in place (gap bytes untouched)."""
    offs = t.byte_offsets()
    allo = (np.arange(incount, dtype=np.int64) * t.extent)[:, None] + offs[None, :]
    buf[origin + allo.ravel()] = packed


# ---- lowering to the C walker's node array -------------------------------

NAMED, HVEC, HIND, STRUCT = 0, 1, 2, 3


class Lowered:
    """Node arrays for oracle/typemap.c (see the onode struct there)."""

    def __init__(self):
        self.nodes = []  # rows of 10 int64: kind,dense,child,count,bl,stride,size,lb,extent,aux
        self.bls = []
        self.displs = []
        self.kids = []

    def add(self, kind, dense, child, count, bl, stride, size, lb, extent, aux=0):
        self.nodes.append([kind, dense, child, count, bl, stride, size, lb, extent, aux])
        return len(self.nodes) - 1

    def node(self, i):
        r = self.nodes[i]
        return dict(dense=r[1], size=r[6], lb=r[7], extent=r[8])


def _hvec(L, count, bl, stride, child, extent=None, lb=None):
    c = L.node(child)
    dense = int(
        bool(c["dense"]) and count > 0 and bl > 0 and (count == 1 or stride == bl * c["size"])
    )
    size = count * bl * c["size"]
    if lb is None:
        lb = c["lb"] + min(0, (count - 1) * stride)
    if extent is None:
        extent = size if dense else 0
    return L.add(HVEC, dense, child, count, bl, stride, size, lb, extent)


def lower(t: OType, L: Lowered | None = None):
    """Lower ``t`` into ``L``; returns (L, root index)."""
    if L is None:
        L = Lowered()
    k, p = t.kind, t.params
    if k == "named":
        return L, L.add(NAMED, 1, 0, 1, 1, 0, t.size, 0, t.size)
    if k == "dup":
        return lower(t.children[0], L)
    if k == "struct":
        kids = [lower(c, L)[1] for c in t.children]
        aux = len(L.bls)
        L.bls += list(p["bls"])
        L.displs += list(p["displs"])
        L.kids += kids
        while len(L.kids) < len(L.bls):
            L.kids.append(0)
        return L, L.add(STRUCT, 0, 0, len(kids), 0, 0, t.size, t.true_lb, t.extent, aux)
    _, c = lower(t.children[0], L)
    ce = t.children[0].extent
    dense = 0
    if k == "contiguous":
        r = _hvec(L, 1, p["count"], 0, c, lb=t.true_lb)
    elif k == "vector":
        r = _hvec(L, p["count"], p["bl"], p["stride"] * ce, c, lb=t.true_lb)
    elif k == "hvector":
        r = _hvec(L, p["count"], p["bl"], p["stride"], c, lb=t.true_lb)
    elif k in ("indexed", "hindexed", "indexed_block", "hindexed_block"):
        scale = ce if k in ("indexed", "indexed_block") else 1
        aux = len(L.bls)
        L.bls += list(p["bls"])
        L.displs += [d * scale for d in p["displs"]]
        L.kids += [0] * len(p["bls"])
        r = L.add(HIND, 0, c, len(p["bls"]), 0, 0, t.size, t.true_lb, t.extent, aux)
    elif k == "subarray":
        sizes, subs, starts = p["sizes"], p["subsizes"], p["starts"]
        nd = len(sizes)
        strides, start = [], 0
        for d in range(nd):
            s = ce
            rng = range(d + 1, nd) if p["order"] == ORDER_C else range(0, d)
            for j in rng:
                s *= sizes[j]
            strides.append(s)
            start += starts[d] * s
        dims = range(nd) if p["order"] == ORDER_C else reversed(range(nd))
        dims = list(dims)  # slowest first
        inner = c
        for d in reversed(dims):
            inner = _hvec(L, subs[d], 1, strides[d], inner)
        aux = len(L.bls)
        L.bls.append(1)
        L.displs.append(start)
        L.kids.append(0)
        whole = all(a == b for a, b in zip(sizes, subs))
        dense = int(bool(L.node(inner)["dense"]) and whole)
        r = L.add(HIND, dense, inner, 1, 0, 0, t.size, t.true_lb, t.extent, aux)
    elif k == "resized":
        aux = len(L.bls)
        L.bls.append(1)
        L.displs.append(0)
        L.kids.append(0)
        cn = L.node(c)
        dense = int(bool(cn["dense"]) and t.lb == cn["lb"] and t.extent == cn["extent"])
        r = L.add(HIND, dense, c, 1, 0, 0, t.size, t.true_lb, t.extent, aux)
    else:
        raise ValueError(k)
    # the node's extent must be the MPI extent (parents step copies by it)
    L.nodes[r][8] = t.extent
    return L, r
