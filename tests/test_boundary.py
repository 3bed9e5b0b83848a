"""The drop-in boundary on CPU: the library loads, exports what
include/tempi_b200.h declares, resolves the underlying MPI with
dlsym(RTLD_NEXT) from a real linked application, and routes host buffers to
the library exactly as the reference does (src/pack.cpp:51-55)."""
import os
import re
import subprocess
import sys

import numpy as np

from oracle import types as T
from tempi_b200 import _lib, mpi

from . import helpers as H

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "tempi_b200.h")


def header_symbols():
    text = open(HEADER).read()
    funcs = set(re.findall(r"^\s*(?:int|int64_t|const char \*|void \*)\s*(tempi_\w+)\(", text, re.M))
    mpis = set(re.findall(r"^\s+(MPI_\w+)\s+replaces", text, re.M))
    return funcs, mpis


def test_exports_every_declared_symbol():
    funcs, mpis = header_symbols()
    assert mpis == set(_lib.INTERPOSED)
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.TEMPI_SO],
                         capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = (funcs | mpis) - exported
    assert not missing, missing
    lib = _lib.tempi()
    for name in funcs | mpis:
        assert getattr(lib, name) is not None


def test_no_mpi_library_is_linked_in():
    out = subprocess.run(["readelf", "-d", _lib.TEMPI_SO], capture_output=True,
                         text=True, check=True).stdout
    assert "minimpi" not in out and "libmpi" not in out


def test_vector_1024x64_host_pack_goes_to_library_and_is_exact(mpi_init):
    """vector(1024,64,512,BYTE) on host buffers, through the
    interposed MPI_Pack, equals the oracle; unpack leaves 0xAA gaps alone."""
    t = H.make_2d_byte_vector(1024, 64, 512).commit()
    src = H.splitmix_bytes(512 * 1024, 0)
    out = np.zeros(65536, np.uint8)
    err, pos = mpi.Pack(src.ctypes.data, 1, t.h, out.ctypes.data, out.nbytes)
    assert (err, pos) == (0, 65536)
    assert out.tobytes() == T.pack(t.o, src, 1).tobytes()
    dst = np.full(512 * 1024, 0xAA, np.uint8)
    err, pos = mpi.Unpack(out.ctypes.data, out.nbytes, dst.ctypes.data, 1, t.h)
    assert (err, pos) == (0, 65536)
    exp = np.full_like(dst, 0xAA)
    T.unpack(t.o, out, exp, 1)
    assert dst.tobytes() == exp.tobytes()
    assert (dst.reshape(-1)[64:512] == 0xAA).all()


def test_host_pack_truncation(mpi_init):
    t = H.make_2d_byte_vector(4, 8, 16).commit()
    src = H.splitmix_bytes(64, 1)
    out = np.zeros(16, np.uint8)
    err, pos = mpi.Pack(src.ctypes.data, 1, t.h, out.ctypes.data, out.nbytes)
    assert err == mpi.ERR_TRUNCATE and pos == 0


def test_host_self_send_through_interposer(mpi_init):
    t = H.make_byte_v_hv((4, 3, 2), (8, 8, 8)).commit()
    src = H.splitmix_bytes(t.o.extent * 2, 5)
    dst = np.full_like(src, 0xAA)
    assert mpi.Send(src.ctypes.data, 2, t.h) == 0
    err, st = mpi.Recv(dst.ctypes.data, 2, t.h)
    assert err == 0 and mpi.Get_count(st, t.h) == 2
    exp = np.full_like(src, 0xAA)
    T.unpack(t.o, T.pack(t.o, src, 2), exp, 2)
    assert dst.tobytes() == exp.tobytes()
    # non-blocking host path
    dst2 = np.full_like(src, 0xAA)
    e1, rr = mpi.Irecv(dst2.ctypes.data, 2, t.h)
    e2, rs = mpi.Isend(src.ctypes.data, 2, t.h)
    assert (e1, e2) == (0, 0)
    assert mpi.Wait(rs)[0] == 0 and mpi.Wait(rr)[0] == 0
    assert dst2.tobytes() == exp.tobytes()


def test_underlying_library_matches_oracle_on_reference_shapes(mpi_init):
    """libminimpi (standing in for the system MPI) against the oracle, on
    every shape of test/pack_unpack.cpp."""
    for ty, count in H.reference_pack_cases():
        o = ty.o
        src = (np.arange(o.extent * count + 8) & 0xFF).astype(np.uint8)
        out = np.zeros(o.size * count, np.uint8)
        err, pos = mpi.Pack(src.ctypes.data, count, ty.h, out.ctypes.data, out.nbytes, library=True)
        assert err == 0 and pos == o.size * count
        assert out.tobytes() == T.pack(o, src, count).tobytes(), ty.name


def test_c_application_links_through_rtld_next(tmp_path):
    """An application linked -ltempi_b200 -lminimpi (in that order) gets the
    interposed MPI_Pack, which forwards host buffers to the library's."""
    src = os.path.join(ROOT, "tests", "c", "app_pack.c")
    exe = tmp_path / "app_pack"
    csrc = os.path.dirname(_lib.TEMPI_SO)
    subprocess.run(["gcc", "-O1", "-o", str(exe), src, "-I" + os.path.join(csrc, "minimpi"),
                    "-I" + os.path.join(ROOT, "include"), "-L" + csrc, "-ltempi_b200",
                    "-lminimpi", "-Wl,-rpath," + csrc], check=True)
    env = dict(os.environ)
    env.pop("TEMPI_LIBMPI", None)
    r = subprocess.run([str(exe)], capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK" in r.stdout


def test_env_disable_and_no_pack(tmp_path):
    """TEMPI_DISABLE / TEMPI_NO_TYPE_COMMIT are read at MPI_Init (any value,
    even empty, counts); with them set nothing is cached at commit.  MPI_Init
    itself caches MPI_BYTE, MPI_FLOAT and MPI_DOUBLE unless TEMPI is
    disabled (the reference's types_init)."""
    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "from tempi_b200 import mpi\n"
        "mpi.Init()\n"
        "from tempi_b200 import _lib\n"
        "t = mpi.Type_vector(4, 2, 8, mpi.BYTE); mpi.Type_commit(t)\n"
        "print(_lib.counter('cached_types'))\n" % ROOT
    )
    for var, want in (("TEMPI_DISABLE", "0"), ("TEMPI_NO_TYPE_COMMIT", "3"), ("UNSET_X", "4")):
        env = dict(os.environ, **{var: ""})
        r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                           env=env, timeout=120)
        assert r.returncode == 0, r.stderr
        assert r.stdout.strip() == want, (var, r.stdout)


def test_global_scope_binds_mpi_pack_to_the_interposer():
    """Loaded in link order, any later library's MPI_Pack reaches TEMPI,
    and TEMPI's dlsym(RTLD_NEXT) reaches the library's."""
    import ctypes

    _lib.tempi()

    class DlInfo(ctypes.Structure):
        _fields_ = [("fname", ctypes.c_char_p), ("fbase", ctypes.c_void_p),
                    ("sname", ctypes.c_char_p), ("saddr", ctypes.c_void_p)]

    libc = ctypes.CDLL(None)
    glob = ctypes.CDLL(None, mode=os.RTLD_NOW)
    for name in _lib.INTERPOSED:
        addr = ctypes.cast(getattr(glob, name), ctypes.c_void_p).value
        info = DlInfo()
        assert libc.dladdr(ctypes.c_void_p(addr), ctypes.byref(info))
        assert info.fname.decode().endswith("libtempi_b200.so"), name
