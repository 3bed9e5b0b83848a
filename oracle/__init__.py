"""ORACLE -- test infrastructure only.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker.  The product
(``tempi_b200``) never imports, links or executes anything here.

Contents
--------
``oracle.types``     MPI-3.1 datatype descriptions built without any MPI
                     library, with an independent numpy type-map expansion.
``oracle.walker``    ctypes front end of ``typemap.c`` (C type-map walker,
                     multi-threaded; the timed CPU baseline).
``oracle.refcanon``  restatement of the reference canonicaliser
                     (src/internal/types.cpp) and of its strided packers
                     (include/pack_kernels.cuh, src/internal/packer_*.cu).
``oracle.interp``    restatement of the reference's perf-table interpolation
                     (src/internal/measure_system.cpp:181-299).
"""
