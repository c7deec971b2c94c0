"""ctypes binding of libcpwb200.so (the C ABI of include/cpw_b200.h).

The library is built in-tree by ``cpw2000_b200.build``. Loading fails loudly
when it is missing: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libcpwb200.so"

_lib = None

P = C.c_void_p
I = C.c_int
LL = C.c_longlong
IP = C.POINTER(C.c_int)
DP = C.POINTER(C.c_double)

# name -> (restype, argtypes); every symbol the header declares
SIGNATURES = {
    "cpw_b200_last_error": (C.c_char_p, []),
    "cpw_b200_version": (I, []),
    "cpw_b200_create": (I, [C.POINTER(P), I]),
    "cpw_b200_destroy": (I, [P]),
    "cpw_b200_stream": (P, [P]),
    "cpw_b200_synchronize": (I, [P]),
    "cpw_b200_set_precision": (I, [P, I]),
    "cpw_b200_set_slab_budget": (I, [P, LL]),
    "cpw_b200_set_wait_limits": (I, [P, LL, LL]),
    "cpw_b200_wait_selftest": (I, [P, LL, P]),
    "cpw_b200_set_projector_slices": (I, [P, I]),
    "cpw_b200_zgemm_i8": (I, [P, I, I, I, I, P, LL, P, LL, C.c_double, I, P, LL, I, P]),
    "cpw_b200_zgemm_i8_tri": (I, [P, I, I, I, I, P, LL, P, LL, C.c_double, I, P, LL, I, I, P]),
    "cpw_b200_timing_begin": (I, [P]),
    "cpw_b200_timing_end": (I, [P, DP, C.POINTER(C.c_longlong), I]),
    "cpw_b200_set_kpoint": (I, [P, I, IP, IP, I, DP, IP]),
    "cpw_b200_set_potential": (I, [P, DP, LL]),
    "cpw_b200_set_projectors": (I, [P, I, DP, I, DP]),
    "cpw_b200_set_projectors_device": (I, [P, I, P, I, P]),
    "cpw_b200_proj_nl_kb_device": (I, [P, DP, I, IP, DP, I, DP, IP, DP, DP, I, IP, I, DP, P, LL]),
    "cpw_b200_proj_nl_kb_der_device": (I, [P, I, DP, I, IP, DP, I, DP, IP, DP, DP, I, IP, I, DP, P, LL, LL, P, P]),
    "cpw_b200_hamilt_kb_device": (I, [P, I, DP, IP, DP, I, IP, DP, DP, IP, IP, IP, DP, DP, DP, IP, DP, DP, IP, I, DP,
                                      P, LL, I, I, I, I, I, I]),
    "cpw_b200_pot_local": (I, [P, DP, DP, DP, DP, DP, IP, I, I, IP, DP, DP, I, IP, I, I, I, I]),
    "cpw_b200_hk_psi_kin_device": (I, [P, I, P, LL, P, LL, I, I, P]),
    "cpw_b200_hk_psi_loc_c16_device": (I, [P, I, P, LL, P, LL, I, I, P]),
    "cpw_b200_set_potential_spin": (I, [P, DP, LL, I]),
    "cpw_b200_set_projectors_spin": (I, [P, I, DP, LL, DP]),
    "cpw_b200_hk_psi_spin_device": (I, [P, I, P, LL, P, LL, P]),
    "cpw_b200_hk_psi_spin_c16": (I, [IP, IP, DP, DP, IP, IP, IP, DP, IP, DP, IP, IP, DP, DP, IP, IP, IP, IP, IP, IP,
                                     IP]),
    "hk_psi_spin_c16_": (None, [IP, IP, DP, DP, IP, IP, IP, DP, IP, DP, IP, IP, DP, DP, IP, IP, IP, IP, IP, IP, IP]),
    "cpw_b200_hk_psi_device": (I, [P, I, P, LL, P, LL, P]),
    "cpw_b200_hk_psi_loc_device": (I, [P, I, P, LL, P, LL, P]),
    "cpw_b200_hk_psi_c16": (I, [IP, IP, DP, DP, IP, IP, IP, DP, IP, DP, IP, DP, DP, IP, IP, IP, IP, IP, IP]),
    "hk_psi_c16_": (None, [IP, IP, DP, DP, IP, IP, IP, DP, IP, DP, IP, DP, DP, IP, IP, IP, IP, IP, IP]),
    "cpw_b200_hk_psi_nl_c16": (I, [IP, IP, DP, DP, DP, DP, IP, IP, IP, IP, IP]),
    "hk_psi_nl_c16_": (None, [IP, IP, DP, DP, DP, DP, IP, IP, IP, IP, IP]),
    "cpw_b200_hk_psi_loc_noalloc": (I, [I, I, P, LL, P, LL, P, P, P, IP, P]),
    "cpw_b200_kbatch_create": (I, [P, I, IP, C.POINTER(IP), IP, I, C.POINTER(DP), IP, C.POINTER(P)]),
    "cpw_b200_kbatch_destroy": (I, [P]),
    "cpw_b200_kbatch_set_projectors": (I, [P, I, I, P, LL, DP]),
    "cpw_b200_kbatch_hk_psi_device": (I, [P, IP, C.POINTER(P), C.POINTER(LL), C.POINTER(P), C.POINTER(LL), P]),
    "cpw_b200_kbatch_synchronize": (I, [P]),
    "cpw_b200_kbatch_info": (I, [P, C.POINTER(LL), I]),
    "cpw_b200_density_device": (I, [P, I, P, LL, DP, P, P]),
    "cpw_b200_structure_grad_device": (I, [P, P, I, IP, DP, I, P, DP, P]),
    "cpw_b200_nl_grad_device": (I, [P, I, P, LL, DP, IP, I, DP, P]),
    "cpw_b200_stress_inputs_device": (I, [P, I, P, LL, DP, P, P, P]),
    "cpw_b200_ditsp_device": (I, [P, I, IP, I, I, C.c_double, IP, I, P, LL, P, DP, DP, I, DP, I,
                                  C.POINTER(C.c_longlong), P, DP, I]),
    "cpw_b200_ditsp_c16": (I, [IP, IP, IP, IP, DP, IP, IP, IP, IP, DP, DP, DP, DP, IP, DP, IP, IP, IP, DP, DP, IP,
                               DP, DP, IP, IP, IP, IP, IP, IP]),
    "ditsp_c16_": (None, [IP, IP, IP, IP, DP, IP, IP, IP, IP, DP, DP, DP, DP, IP, DP, IP, IP, IP, DP, DP, IP,
                          DP, DP, IP, IP, IP, IP, IP, IP]),
}


class CpwB200Error(RuntimeError):
    """A non-zero status from the C ABI; ``status`` holds the code."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"cpw_b200 status {status}: {msg}")
        self.status = status


def lib():
    """Load (once) and return the ctypes library; raises if it is not built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m cpw2000_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> int:
    if status != 0:
        msg = lib().cpw_b200_last_error().decode(errors="replace")
        raise CpwB200Error(status, msg)
    return status


def iptr(a):
    return a.ctypes.data_as(IP)


def dptr(a):
    return a.ctypes.data_as(DP)


def iref(v: int):
    return C.byref(C.c_int(int(v)))


def zptr(a):
    """Pointer to a complex128 array's data as double* (interleaved re, im)."""
    if a.dtype != "complex128":
        raise TypeError("expected complex128")
    return a.ctypes.data_as(DP)
