"""tempi_b200: B200-native interposed MPI derived-datatype pack/unpack.

The product is the C-ABI shared library ``csrc/libtempi_b200.so`` (declared
in ``include/tempi_b200.h``).  This package only loads it (``_lib``) and
mirrors its MPI surface for Python callers and tests (``mpi``), plus the
strided-block helpers in ``kernels``.
"""
from . import _lib  # noqa: F401

__all__ = ["_lib", "mpi"]
