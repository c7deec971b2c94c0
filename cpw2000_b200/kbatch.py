"""Batched H|psi> over the k-points of one crystal (cpw_b200_kbatch_* of the C ABI).

The reference applies H k-point by k-point (Src/cpw_lib/cpw_scf.f90:488 -> h_kb_dia
-> ditsp_c16 -> hk_psi_c16). ``KBatch`` holds the bases of many k-points of one
crystal (same FFT box and potential, each its own plane-wave count, kinetic
diagonal and KB projectors) and applies H_k psi_k to all of them in one call. The
first call with a given set of blocks autotunes the launch shape and captures the
call as a CUDA graph; later calls with the same blocks replay it.

Typical use::

    ctx = Context(0, precision=MIXED_TC).setup(inputs[0])    # box, potential
    kb = KBatch(ctx, inputs)                                  # every k-point
    kb.hk_psi(psis, hpsis)                                    # lists of (mtxd_k, nb_k) tensors
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, dptr, iptr
from .hk_psi import Context, torch_stream_handle

INFO = ("tuned", "chunk_bands", "b_grouping", "proj_splits", "tuned_call_us", "candidates", "graph_replays",
        "captures")


class KBatch:
    def __init__(self, ctx: Context, inputs: list[dict]):
        self._L = _lib.lib()
        self.ctx = ctx
        self.nk = len(inputs)
        self.mtxd = [int(d["mtxd"]) for d in inputs]
        kgv = np.asfortranarray(inputs[0]["kgv"], dtype=np.int32)
        kmscr = np.ascontiguousarray(inputs[0]["kmscr"], dtype=np.int32)
        self._keep = []
        isorts = [np.ascontiguousarray(d["isort"], dtype=np.int32) for d in inputs]
        ekpgs = [np.ascontiguousarray(d["ekpg"], dtype=np.float64) for d in inputs]
        self._keep += isorts + ekpgs
        m = (C.c_int * self.nk)(*self.mtxd)
        ip = (C.POINTER(C.c_int) * self.nk)(*[iptr(a) for a in isorts])
        dp = (C.POINTER(C.c_double) * self.nk)(*[dptr(a) for a in ekpgs])
        h = C.c_void_p()
        check(self._L.cpw_b200_kbatch_create(ctx.handle, self.nk, m, ip, iptr(kgv), int(kgv.shape[1]), dp,
                                             iptr(kmscr), C.byref(h)))
        self.handle = h
        for k, d in enumerate(inputs):
            self.set_projectors(k, d["anlga"], d["xnlkb"])

    def close(self):
        if getattr(self, "handle", None):
            self._L.cpw_b200_kbatch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_projectors(self, ik: int, anlga, xnlkb):
        a = np.asfortranarray(anlga, dtype=np.complex128)
        x = np.ascontiguousarray(xnlkb, dtype=np.float64)
        nanl = int(x.size)
        if nanl == 0:
            a = np.zeros((max(self.mtxd[ik], 1), 1), np.complex128, order="F")
            x = np.zeros(1)
        self._keep.append(a)
        check(self._L.cpw_b200_kbatch_set_projectors(self.handle, int(ik), nanl, C.c_void_p(a.ctypes.data),
                                                     int(a.shape[0]), dptr(x)))

    def hk_psi(self, psis, hpsis):
        """hpsi_k = H_k psi_k for every k on torch's current stream; psis/hpsis: lists of
        column-major complex128 CUDA tensors, block k of shape (mtxd_k, nb_k)."""
        if len(psis) != self.nk or len(hpsis) != self.nk:
            raise ValueError("one psi and one hpsi block per k-point")
        nb = (C.c_int * self.nk)()
        pp = (C.c_void_p * self.nk)()
        hp = (C.c_void_p * self.nk)()
        lp = (C.c_longlong * self.nk)()
        lh = (C.c_longlong * self.nk)()
        for k, (x, y) in enumerate(zip(psis, hpsis)):
            if x.shape != y.shape or x.shape[0] != self.mtxd[k]:
                raise ValueError(f"k-point {k}: blocks must be ({self.mtxd[k]}, nb)")
            if x.stride(0) != 1 or y.stride(0) != 1:
                raise ValueError("blocks must be column-major")
            nb[k] = int(x.shape[1])
            pp[k] = x.data_ptr()
            hp[k] = y.data_ptr()
            lp[k] = int(x.stride(1)) if x.shape[1] > 1 else self.mtxd[k]
            lh[k] = int(y.stride(1)) if y.shape[1] > 1 else self.mtxd[k]
        check(self._L.cpw_b200_kbatch_hk_psi_device(self.handle, nb, pp, lp, hp, lh,
                                                    C.c_void_p(torch_stream_handle(psis[0].device))))

    def synchronize(self):
        check(self._L.cpw_b200_kbatch_synchronize(self.handle))

    def info(self) -> dict:
        out = (C.c_longlong * 8)()
        check(self._L.cpw_b200_kbatch_info(self.handle, out, 8))
        return {n: int(out[i]) for i, n in enumerate(INFO)}
