"""ORACLE -- test infrastructure only.

Restatement of the reference's canonicaliser and strided packers, so that
the tests can say what the reference would produce for a type:

* ``from_type``        types.cpp:42-354  (Type::from_mpi_datatype)
* ``stream_swap``      types.cpp:378-404
* ``stream_dense_fold`` types.cpp:409-449
* ``stream_elision2``  types.cpp:490-516
* ``stream_flatten``   types.cpp:529-563
* ``simplify``         types.cpp:567-614 (fixpoint of the four passes)
* ``to_strided_block`` types.cpp:654-715
* ``ref_pack``/``ref_unpack``: what Packer1D (packer_1d.cu:16-50),
  Packer2D (pack_kernels.cuh:64-120, packer_2d.cu:21-74) and Packer3D
  (pack_kernels.cuh:350-433, packer_3d.cu:80-115) write, for the StridedBlock
  chosen by plan_pack (types.cpp:619-646).

Where the reference departs from MPI type-map order these functions keep the
departure on purpose (``stream_swap`` reorders loops; Packer1D ignores the
type extent for incount > 1), because they describe the reference, not MPI.
"""
from __future__ import annotations

import copy

import numpy as np

from . import types as T


class Node:
    """Type tree node: kind is 'dense', 'stream' or 'empty'."""

    def __init__(self, kind, off=0, extent=0, stride=0, count=0, children=None):
        self.kind = kind
        self.off = off
        self.extent = extent  # DenseData extent, or the tree's type extent
        self.stride = stride
        self.count = count
        self.children = children or []
        self.type_extent = -1

    def data_eq(self, o):
        if self.kind != o.kind:
            return False
        if self.kind == "dense":
            return self.extent == o.extent  # DenseData::operator== (types.hpp)
        if self.kind == "stream":
            return (self.off, self.stride, self.count) == (o.off, o.stride, o.count) and bool(self.count)
        return True

    def __eq__(self, o):
        return self.data_eq(o) and len(self.children) == len(o.children) and all(
            a == b for a, b in zip(self.children, o.children)
        )


def empty():
    return Node("empty")


def from_type(t: T.OType) -> Node:
    """types.cpp:42-354."""
    k, p = t.kind, t.params
    if k == "named":
        n = Node("dense", off=0, extent=t.extent)
        n.type_extent = t.extent
        return n
    if k in ("vector", "hvector"):
        old = t.children[0]
        stride = old.extent * p["stride"] if k == "vector" else p["stride"]
        parent = Node("stream", off=0, count=p["count"], stride=stride)
        child = Node("stream", off=0, count=p["bl"], stride=old.extent)
        child.children = [from_type(old)]
        parent.children = [child]
        parent.type_extent = t.extent
        return parent
    if k == "contiguous":
        old = t.children[0]
        n = Node("stream", off=0, count=p["count"], stride=old.extent)
        n.children = [from_type(old)]
        n.type_extent = t.extent
        return n
    if k == "subarray":
        old = t.children[0]
        sizes, subs, starts = p["sizes"], p["subsizes"], p["starts"]
        nd = len(sizes)
        datas = []
        for i in range(nd):
            off = starts[i] * old.extent
            stride = old.extent
            rng = range(i + 1, nd) if p["order"] == T.ORDER_C else range(i - 1, -1, -1)
            for j in rng:
                stride *= sizes[j]
                off *= sizes[j]
            datas.append((off, stride, subs[i]))
        if p["order"] == T.ORDER_C:
            datas.reverse()
        child = from_type(old)
        for off, stride, cnt in datas:
            parent = Node("stream", off=off, stride=stride, count=cnt)
            parent.children = [child]
            child = parent
        child.type_extent = t.extent
        return child
    # indexed, hindexed, struct, resized, dup: the reference gives up
    return empty()


def stream_swap(n: Node) -> bool:
    if n.kind != "stream":
        return False
    c = n.children[0]
    if c.kind != "stream":
        return False
    changed = False
    if n.stride < c.stride:
        changed = True
        n.off, c.off = c.off, n.off
        n.stride, c.stride = c.stride, n.stride
        n.count, c.count = c.count, n.count
    changed |= stream_swap(c)
    return changed


def stream_dense_fold(n: Node) -> bool:
    changed = False
    for c in n.children:
        changed |= stream_dense_fold(c)
    if n.kind != "stream":
        return False
    c = n.children[0]
    if c.kind != "dense":
        return False
    if c.extent == n.stride:
        n.kind = "dense"
        n.extent = n.count * n.stride
        n.off = c.off + n.off
        n.children = list(c.children)
        n.stride = n.count = 0
        return True
    return changed


def stream_elision2(n: Node) -> bool:
    changed = False
    for c in n.children:
        changed |= stream_elision2(c)
    if n.kind != "stream":
        return False
    if n.count == 1:
        c = n.children[0]
        te = n.type_extent
        n.kind, n.off, n.extent = c.kind, c.off, c.extent
        n.stride, n.count, n.children = c.stride, c.count, list(c.children)
        n.type_extent = te
        return True
    return changed


def stream_flatten(n: Node) -> bool:
    changed = False
    for c in n.children:
        changed |= stream_flatten(c)
    if n.kind != "stream":
        return False
    c = n.children[0]
    if c.kind != "stream":
        return False
    if n.stride == c.count * c.stride:
        n.count *= c.count
        n.stride = c.stride
        n.off += c.off
        n.children = list(c.children)
        return True
    return changed


def simplify(t: Node) -> Node:
    s = copy.deepcopy(t)
    changed = True
    while changed:
        changed = False
        changed |= stream_swap(s)
        changed |= stream_dense_fold(s)
        changed |= stream_flatten(s)
        changed |= stream_elision2(s)
    return s


class StridedBlock:
    def __init__(self, start=0, extent=0, counts=None, strides=None):
        self.start = start
        self.extent = extent
        self.counts = counts or []
        self.strides = strides or []

    @property
    def ndims(self):
        return len(self.counts)

    def __eq__(self, o):  # StridedBlock::operator== ignores the extent
        return (self.start, self.counts, self.strides) == (o.start, o.counts, o.strides)

    def __repr__(self):
        return f"StridedBlock(start={self.start}, extent={self.extent}, counts={self.counts}, strides={self.strides})"


def to_strided_block(t: Node, type_extent: int) -> StridedBlock:
    """types.cpp:654-715."""
    if t.kind == "empty":
        return StridedBlock()
    chain, cur = [], t
    while True:
        chain.append(cur)
        if len(cur.children) == 1:
            cur = cur.children[0]
        elif not cur.children:
            break
        else:
            return StridedBlock()
    sb = StridedBlock(extent=type_extent)
    if chain[-1].kind != "dense":
        return StridedBlock()
    sb.start += chain[-1].off
    sb.counts.append(chain[-1].extent)
    sb.strides.append(1)
    for n in reversed(chain[:-1]):
        if n.kind != "stream":
            return StridedBlock()
        sb.start += n.off
        sb.counts.append(n.count)
        sb.strides.append(n.stride)
    return sb


def canonicalize(t: T.OType) -> StridedBlock:
    """traverse -> simplify -> to_strided_block, as MPI_Type_commit does
    (type_commit.cpp:164-166)."""
    return to_strided_block(simplify(from_type(t)), t.extent)


# ---- the reference packers --------------------------------------------------


def _view(buf: np.ndarray, base: int, shape, strides):
    return np.lib.stride_tricks.as_strided(
        buf[base:], shape=shape, strides=strides, writeable=True
    )


def ref_pack(sb: StridedBlock, buf: np.ndarray, incount: int,
             origin: int = 0) -> np.ndarray:
    """Bytes the reference packer writes for ``incount`` objects."""
    if sb.ndims == 1:
        # Packer1D copies incount*counts[0] contiguous bytes (packer_1d.cu:26-31)
        b = origin + sb.start
        return buf[b : b + incount * sb.counts[0]].copy()
    if sb.ndims == 2:
        shape = (incount, sb.counts[1], sb.counts[0])
        strides = (sb.extent, sb.strides[1], 1)
    elif sb.ndims == 3:
        shape = (incount, sb.counts[2], sb.counts[1], sb.counts[0])
        strides = (sb.extent, sb.strides[2], sb.strides[1], 1)
    else:
        raise ValueError("the reference has no packer for ndims=%d" % sb.ndims)
    return np.ascontiguousarray(_view(buf, origin + sb.start, shape, strides)).ravel()


def ref_unpack(sb: StridedBlock, packed: np.ndarray, buf: np.ndarray,
               incount: int, origin: int = 0) -> None:
    if sb.ndims == 1:
        b = origin + sb.start
        buf[b : b + incount * sb.counts[0]] = packed[: incount * sb.counts[0]]
        return
    if sb.ndims == 2:
        shape = (incount, sb.counts[1], sb.counts[0])
        strides = (sb.extent, sb.strides[1], 1)
    else:
        shape = (incount, sb.counts[2], sb.counts[1], sb.counts[0])
        strides = (sb.extent, sb.strides[2], sb.strides[1], 1)
    v = _view(buf, origin + sb.start, shape, strides)
    v[...] = packed.reshape(shape)
