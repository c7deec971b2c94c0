"""GPU small Hamiltonian of the start basis (cpw_b200_hamilt_kb_device, the device form of
Src/ALFA/hamilt_kb.f90) against the restatement oracle/hamilt.py (itself pinned on the CPU
against the operator's own matrix block): one star per G vector and G/-G pairs through the
conj flag, Gamma and k off Gamma, within 1e-12 of max|hamk|; the reference's argument checks.
"""
import ctypes as C

import numpy as np
import pytest

from cpw2000_b200 import _lib, configs
from cpw2000_b200 import hk_psi as H
from cpw2000_b200._lib import CpwB200Error
from oracle import hamilt as OH
from tests.test_oracle_hamilt import star_inputs

pytestmark = pytest.mark.gpu


def _device(ctx, w, d, mtxds, isort, kg, phase, conj, inds, kmax, indv, ek, sf, veff, torch, dev, ldh=None):
    L = _lib.lib()
    nt = len(w.species)
    ldh = ldh or mtxds
    out = torch.zeros((mtxds, ldh), dtype=torch.complex128, device=dev)
    nq = 4000
    vref = np.zeros((nq + 3, 4, 3, nt), order="F")
    nref = np.zeros((4, 3, nt), dtype=np.int32, order="F")
    for t in range(nt):
        for l in range(4):
            vref[:, l, 1, t] = d["vkb"][t, l, :nq + 3]
            nref[l, 1, t] = int(d["nkb"][t, l])
    ng = kg.shape[1]
    ns = int(np.max(inds))
    sfa = np.asfortranarray(sf[:, :ns], dtype=np.complex128)
    st = L.cpw_b200_hamilt_kb_device(
        ctx.handle, mtxds, _lib.dptr(np.ascontiguousarray(d["hdiag"])), _lib.iptr(np.ascontiguousarray(isort, np.int32)),
        _lib.dptr(np.ascontiguousarray(d["qmod"])), ng, _lib.iptr(np.asfortranarray(kg, np.int32)),
        _lib.zptr(np.ascontiguousarray(phase, np.complex128)), _lib.dptr(np.ascontiguousarray(conj, np.float64)),
        _lib.iptr(np.ascontiguousarray(inds, np.int32)), _lib.iptr(np.ascontiguousarray(kmax, np.int32)),
        _lib.iptr(np.ascontiguousarray(indv, np.int32)), _lib.dptr(np.ascontiguousarray(ek[:ns])), _lib.zptr(sfa),
        _lib.zptr(np.ascontiguousarray(veff[:ns], np.complex128)), _lib.iptr(np.full(nt, nq, np.int32)),
        _lib.dptr(np.full(nt, 0.01)), _lib.dptr(vref), _lib.iptr(nref), nt, _lib.dptr(np.asfortranarray(w.adot)),
        C.c_void_p(out.data_ptr()), ldh, nt, ng, ns, int(indv.size), nq, int(d["mtxd"]))
    _lib.check(st)
    torch.cuda.synchronize()
    return out.cpu().numpy().T[:mtxds, :mtxds]      # rows of the torch array are the columns of hamk


@pytest.mark.parametrize("ik,pair", [(0, False), (3, False), (5, True)])
def test_hamilt_kb_device_matches_restatement(cuda, ik, pair):
    import torch
    w = configs.si2_fcc()
    d = configs.kpoint_inputs(w, ik, with_hamsm=True)
    mtxds = d["mtxds"]
    isort, kg, phase, conj, inds, kmax, indv, ek, sf, veff = star_inputs(w, d, pair)
    nt = len(w.species)
    want = OH.hamilt_kb(mtxds, d["hdiag"], isort, d["qmod"], kg, phase, conj, inds, kmax, indv, ek, sf, veff,
                        np.full(nt, 4000), np.full(nt, 0.01), d["vkb"], d["nkb"], w.adot)
    ctx = H.Context(0)
    got = _device(ctx, w, d, mtxds, isort, kg, phase, conj, inds, kmax, indv, ek, sf, veff, torch, cuda)
    assert np.abs(got - want).max() < 1e-12 * np.abs(want).max()
    # and it is the block of the eigensolver's inputs
    assert np.abs(got - d["hamsm"][:mtxds, :mtxds]).max() < 1e-12 * np.abs(want).max()
    ctx.close()


def test_hamilt_kb_device_rejects_bad_star_index(cuda):
    import torch
    w = configs.si2_fcc()
    d = configs.kpoint_inputs(w, 0, with_hamsm=True)
    isort, kg, phase, conj, inds, kmax, indv, ek, sf, veff = star_inputs(w, d, False)
    inds = inds.copy()
    inds[3] = 0
    ctx = H.Context(0)
    with pytest.raises(CpwB200Error, match="inds"):
        _device(ctx, w, d, d["mtxds"], isort, kg, phase, conj, inds, kmax, indv, ek, sf, veff, torch, cuda)
    ctx.close()
