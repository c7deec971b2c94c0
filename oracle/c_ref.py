"""ctypes wrapper of oracle/c/libhkpsi_ref.so (C + OpenMP restatement of hk_psi_c16).

Test / CPU-baseline infrastructure only (see oracle/__init__.py).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from .hk_psi import ipoint_of

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "c", "libhkpsi_ref.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return SO


_blas = None


def openblas_path():
    """numpy's bundled OpenBLAS (64-bit integers, scipy_ prefixed symbols), or None."""
    import glob

    import numpy
    hits = glob.glob(os.path.join(os.path.dirname(numpy.__file__), "..", "numpy.libs", "*openblas64*.so*"))
    return hits[0] if hits else None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(SO):
            build()
        L = C.CDLL(SO)
        L.cpw_ref_hk_psi.restype = C.c_int
        L.cpw_ref_max_threads.restype = C.c_int
        L.cpw_ref_has_zgemm.restype = C.c_int
        L.cpw_ref_set_zgemm.argtypes = [C.c_void_p]
        _lib = L
    return _lib


def use_blas(on: bool = True) -> bool:
    """Projector ZGEMMs of the restatement in numpy's OpenBLAS (on) or in its own loops (off).
    Returns whether the optimised GEMM is in use."""
    global _blas
    L = lib()
    if not on:
        L.cpw_ref_set_zgemm(None)
        return False
    if _blas is None:
        path = openblas_path()
        if path is None:
            return False
        _blas = C.CDLL(path)
    fn = getattr(_blas, "scipy_cblas_zgemm64_", None)
    if fn is None:
        return False
    L.cpw_ref_set_zgemm(C.cast(fn, C.c_void_p))
    return bool(L.cpw_ref_has_zgemm())


def max_threads() -> int:
    return int(lib().cpw_ref_max_threads())


def hk_psi_c16(mtxd, neig, psi, ekpg, isort, vscr, kmscr, kgv, anlga, xnlkb, nthreads=0):
    """Same contract as oracle.hk_psi.hk_psi_c16, computed by the C restatement."""
    L = lib()
    ip, (kd1, kd2, kd3) = ipoint_of(mtxd, isort, kgv, kmscr)
    ip = np.ascontiguousarray(ip, dtype=np.int32)
    n1, n2, n3, ident = (int(v) for v in kmscr[3:7])
    psi = np.asfortranarray(psi, dtype=np.complex128)
    hpsi = np.zeros((mtxd, neig), dtype=np.complex128, order="F")
    v = np.ascontiguousarray(vscr[: ident * n2 * n3], dtype=np.float64)
    ek = np.ascontiguousarray(ekpg[:mtxd], dtype=np.float64)
    nanl = int(np.asarray(xnlkb).size)
    a = np.asfortranarray(anlga if nanl else np.zeros((max(mtxd, 1), 1)), dtype=np.complex128)
    x = np.ascontiguousarray(xnlkb if nanl else np.zeros(1), dtype=np.float64)
    vp = C.c_void_p
    st = L.cpw_ref_hk_psi(C.c_int(mtxd), C.c_int(neig), vp(psi.ctypes.data), C.c_int(psi.shape[0]),
                          vp(hpsi.ctypes.data), C.c_int(mtxd), vp(ip.ctypes.data), C.c_int(kd1), C.c_int(kd2),
                          C.c_int(kd3), C.c_int(n1), C.c_int(n2), C.c_int(n3), C.c_int(ident), vp(v.ctypes.data),
                          vp(ek.ctypes.data), vp(a.ctypes.data), C.c_int(a.shape[0]), vp(x.ctypes.data),
                          C.c_int(nanl), C.c_int(int(nthreads)))
    if st != 0:
        raise MemoryError("cpw_ref_hk_psi failed")
    return hpsi
