"""Writes the golden fixtures in this directory.

Each fixture is a seeded case of the pack path: a type (described without
any MPI library), the seed and size of a random byte buffer, the object
count, and the packed bytes that MPI type-map order gives.  The packed bytes
come from the oracle's numpy type-map expansion (oracle/types.py), which
follows the MPI-3.1 type constructors.  Shapes: the 1024 x 64 B vector of the benchmark
(vector 1024 x 64 B, stride 512 B, truncated output is not stored -- only a
hash), the reference's test/pack_unpack.cpp shapes, and a Fortran-order
subarray.

Run from the repository root:  python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import numpy as np  # noqa: E402

from oracle import types as T  # noqa: E402


def named(size):
    return {"kind": "named", "size": size}


CASES = {
    "vector_2x3_stride4_count2": ({"kind": "vector", "count": 2, "bl": 3, "stride": 4, "child": named(1)}, 2),
    "subarray2d_byte_count2": ({"kind": "subarray", "sizes": [2, 4], "subsizes": [2, 3], "starts": [0, 0], "order": 56, "child": named(1)}, 2),
    "off_subarray_16cube_count2": ({"kind": "subarray", "sizes": [16, 16, 16], "subsizes": [2, 3, 4], "starts": [1, 1, 4], "order": 56, "child": named(1)}, 2),
    "v_hv_2x3x4_in_10cube_count2": ({"kind": "hvector", "count": 4, "bl": 1, "stride": 100, "child": {"kind": "vector", "count": 3, "bl": 2, "stride": 10, "child": named(1)}}, 2),
    "fortran_subarray_float": ({"kind": "subarray", "sizes": [7, 9, 5], "subsizes": [3, 4, 2], "starts": [1, 2, 3], "order": 57, "child": named(4)}, 3),
    "hv_by_cols_13_3_16_5_53": ({"kind": "hvector", "count": 3, "bl": 1, "stride": 16, "child": {"kind": "hvector", "count": 5, "bl": 1, "stride": 53, "child": {"kind": "contiguous", "count": 13, "child": named(1)}}}, 1),
    "resized_vector_double": ({"kind": "resized", "lb": 0, "extent": 200, "child": {"kind": "vector", "count": 3, "bl": 2, "stride": 5, "child": named(8)}}, 3),
}


def build(spec):
    k = spec["kind"]
    if k == "named":
        return T.named(spec["size"])
    c = build(spec["child"])
    if k == "vector":
        return T.vector(spec["count"], spec["bl"], spec["stride"], c)
    if k == "hvector":
        return T.hvector(spec["count"], spec["bl"], spec["stride"], c)
    if k == "contiguous":
        return T.contiguous(spec["count"], c)
    if k == "subarray":
        return T.subarray(spec["sizes"], spec["subsizes"], spec["starts"], spec["order"], c)
    if k == "resized":
        return T.resized(c, spec["lb"], spec["extent"])
    raise ValueError(k)


def main():
    for i, (name, (spec, incount)) in enumerate(CASES.items()):
        o = build(spec)
        lo = min(0, o.true_lb)
        hi = o.true_ub + (incount - 1) * o.extent
        nbytes = hi - lo + 32
        seed = 1000 + i
        buf = np.random.default_rng(seed).integers(0, 256, nbytes, dtype=np.uint8)
        packed = T.pack(o, buf, incount, origin=-lo)
        out = {
            "name": name, "type": spec, "incount": incount, "seed": seed,
            "buf_bytes": nbytes, "origin": -lo, "size": o.size, "extent": o.extent,
            "packed_hex": packed.tobytes().hex(),
            "sha256": hashlib.sha256(packed.tobytes()).hexdigest(),
        }
        with open(os.path.join(HERE, name + ".json"), "w") as f:
            json.dump(out, f, indent=1)
    print("wrote", len(CASES), "fixtures")


if __name__ == "__main__":
    main()
