"""GPU: stress of the Hellmann-Feynman energy through the adjoint (cpw_b200_stress_inputs_device
+ density kernel + host contractions) against the restated reference routines and central
finite differences (Si2), and term by term against the numpy inputs on ZB64 (two species)."""
import numpy as np
import pytest

from cpw2000_b200 import configs
from cpw2000_b200 import forces as FF
from cpw2000_b200 import stress as ST
from oracle import stress as OS

pytestmark = pytest.mark.gpu


def _system(w, d, nb, seed, torch, dev):
    psi_h = configs.random_psi(d["mtxd"], nb, seed)
    psi = torch.from_numpy(np.ascontiguousarray(psi_h.T)).to(dev).t()
    return psi_h, FF.HFSystem(w, d, psi, np.full(nb, 2.0))


def test_stress_si2_vs_restatement_and_fd(cuda):
    import torch
    w = configs.si2_fcc()
    d = configs.kpoint_inputs(w, 1)
    psi_h, s = _system(w, d, 4, 21, torch, cuda)
    out = ST.stress(s)
    m = d["mtxd"]
    occ = s.occ
    rk = OS.strkin(d["rkpt"], m, d["isort"], d["kgv"], psi_h, occ)
    rl = OS.strhl(OS.rho_of(d, psi_h, occ), w.species, w.adot, w.box)
    rn = OS.strnlkb(d["rkpt"], m, d["isort"], d["kgv"], psi_h, occ, w.species, d["vkb"], d["nkb"], w.adot)
    for name, ref in (("kinetic", rk), ("local", rl), ("kb", rn)):
        assert np.abs(out[name] - ref).max() <= 1e-10 * np.abs(ref).max(), name
    fd = OS.fd_covariant_stress(d, w.species, w.adot, w.box, w.idpad, psi_h, occ)
    assert np.abs(out["total"] - fd).max() <= 1e-6 * np.abs(fd).max()
    # the autograd form returns dE/de
    e = torch.zeros((3, 3), dtype=torch.float64, requires_grad=True)
    E = ST.StrainEnergy.apply(e, s)
    E.backward()
    assert np.abs(e.grad.numpy() - out["dE_dstrain"]).max() <= 1e-12 * np.abs(out["dE_dstrain"]).max()


def test_stress_zb64_gpu_inputs(cuda):
    import torch
    w = configs.zb64_cubic()
    d = configs.kpoint_inputs(w, 0)
    nb = 8
    psi_h, s = _system(w, d, nb, 31, torch, cuda)
    out = ST.stress(s)
    m = d["mtxd"]
    occ = s.occ
    wG = np.sum(occ[None, :] * np.abs(psi_h[:m]) ** 2, axis=1)
    P = d["anlga"].conj().T @ psi_h[:m]
    Y = psi_h[:m] @ (occ[:, None] * P.conj().T * d["xnlkb"][None, :])
    cov = lambda S: ST.covariant(ST.strain_to_metric(S, w.adot), w.adot)
    Sn, _ = ST.kb_strain(Y, d, w.species, w.adot)
    rk = OS.strkin(d["rkpt"], m, d["isort"], d["kgv"], psi_h, occ)
    rl = OS.strhl(OS.rho_of(d, psi_h, occ), w.species, w.adot, w.box)
    assert np.abs(out["kinetic"] - rk).max() <= 1e-10 * np.abs(rk).max()
    assert np.abs(out["local"] - rl).max() <= 1e-9 * np.abs(rl).max()
    assert np.abs(out["kb"] - cov(Sn)).max() <= 1e-10 * np.abs(cov(Sn)).max()
