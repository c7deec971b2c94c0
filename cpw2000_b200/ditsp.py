"""Python mirror of cpw2000's block eigensolver ditsp_c16 over the C ABI.

``ditsp_c16`` takes the argument list of Src/ditsp/ditsp_c16.f90:20-27 with
host numpy arrays (Fortran order; psi/hpsi updated in place) and returns what
the Fortran routine returns through its arguments. ``eigensolve`` is the
device form on a ``hk_psi.Context`` with torch CUDA tensors.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import CpwB200Error, dptr, iptr, zptr
from .hk_psi import torch_stream_handle

NOT_CONVERGED = 5


def ditsp_c16(ipr, icmax, iguess, epspsi, lnewanl, neig, mtxd, mtxds, psi, hpsi, ekpg, isort, vscr, kmscr, ng,
              kgv, anlga, xnlkb, nanl, hamsm, hdiag, mxddim, mxdsml, mxdbnd, mxdgve, mxdscr, mxdanl):
    """Returns dict(ifail, ei, neig, lnewanl); psi, hpsi (complex128, Fortran) are updated in place."""
    L = _lib.lib()
    for a in (psi, hpsi):
        if not (isinstance(a, np.ndarray) and a.dtype == np.complex128 and a.flags.f_contiguous):
            raise TypeError("psi/hpsi must be Fortran-ordered complex128 arrays (updated in place)")
    kgv = np.asfortranarray(kgv, dtype=np.int32)
    isort = np.ascontiguousarray(isort, dtype=np.int32)
    ekpg = np.ascontiguousarray(ekpg, dtype=np.float64)
    vscr = np.ascontiguousarray(vscr, dtype=np.float64)
    kmscr = np.ascontiguousarray(kmscr, dtype=np.int32)
    anlga = np.asfortranarray(anlga if nanl > 0 else np.zeros((max(mxddim, 1), 1)), dtype=np.complex128)
    xnlkb = np.ascontiguousarray(xnlkb if nanl > 0 else np.zeros(1), dtype=np.float64)
    hamsm = np.asfortranarray(hamsm, dtype=np.complex128)
    hdiag = np.ascontiguousarray(hdiag, dtype=np.float64)
    ei = np.zeros(max(mxdbnd, 1))
    ifail = C.c_int(0)
    lnew = C.c_int(1 if lnewanl else 0)
    ne = C.c_int(int(neig))
    ri = _lib.iref
    st = L.cpw_b200_ditsp_c16(ri(ipr), C.byref(ifail), ri(icmax), ri(iguess), C.byref(C.c_double(epspsi)),
                              C.byref(lnew), C.byref(ne), ri(mtxd), ri(mtxds), zptr(psi), zptr(hpsi), dptr(ei),
                              dptr(ekpg), iptr(isort), dptr(vscr), iptr(kmscr), ri(ng), iptr(kgv), zptr(anlga),
                              dptr(xnlkb), ri(nanl), zptr(hamsm), dptr(hdiag), ri(mxddim), ri(mxdsml), ri(mxdbnd),
                              ri(mxdgve), ri(mxdscr), ri(mxdanl))
    if st not in (0, NOT_CONVERGED):
        raise CpwB200Error(st, L.cpw_b200_last_error().decode(errors="replace"))
    return dict(ifail=int(ifail.value), ei=ei[: ne.value].copy(), neig=int(ne.value), lnewanl=bool(lnew.value))


def eigensolve(ctx, psi, hpsi, neig, mtxds, hamsm, hdiag, epspsi=1e-5, icmax=40, iguess=0, stream=None, ipr=0,
               trace=False):
    """ditsp on device-resident column-major complex128 psi/hpsi (mxdbnd = psi.shape[1] columns).

    Returns dict(ifail, ei, neig, ihkpsum, converged[, trace]). With trace=True,
    ``trace`` is an (iterations, 4 + mxdbnd) array: elapsed s, xmax, nconv,
    H|psi> products and the Ritz values after every outer iteration.
    """
    L = _lib.lib()
    mxdbnd = int(psi.shape[1])
    hamsm = np.asfortranarray(hamsm, dtype=np.complex128)
    hdiag = np.ascontiguousarray(hdiag, dtype=np.float64)
    ei = np.zeros(mxdbnd)
    ifail = C.c_int(0)
    ne = C.c_int(int(neig))
    ih = C.c_longlong(0)
    s = stream if stream is not None else torch_stream_handle(psi.device)
    log = np.zeros((int(icmax), 4 + mxdbnd)) if trace else None
    st = L.cpw_b200_ditsp_device(ctx.handle, int(ipr), C.byref(ifail), int(icmax), int(iguess), float(epspsi), C.byref(ne),
                                 int(mtxds), C.c_void_p(psi.data_ptr()), ctx._ld(psi), C.c_void_p(hpsi.data_ptr()),
                                 dptr(ei), zptr(hamsm), int(hamsm.shape[0]), dptr(hdiag), mxdbnd, C.byref(ih),
                                 C.c_void_p(s), dptr(log) if trace else None, int(icmax) if trace else 0)
    if st not in (0, NOT_CONVERGED):
        raise CpwB200Error(st, L.cpw_b200_last_error().decode(errors="replace"))
    out = dict(ifail=int(ifail.value), ei=ei[: ne.value].copy(), neig=int(ne.value), ihkpsum=int(ih.value),
               converged=st == 0)
    if trace:
        used = int(np.count_nonzero(log[:, 0] > 0))
        out["trace"] = log[:used]
    return out
