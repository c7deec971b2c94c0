"""CPU: the stress restatement (oracle/stress.py) against central finite differences of the
energy in the metric, and the library's host contractions (cpw2000_b200/stress.py, fed here
with numpy-computed w, Y and density) against the restatement, term by term."""
import numpy as np
import pytest

from cpw2000_b200 import configs
from cpw2000_b200 import stress as ST
from oracle import stress as OS


def _case(nb=3, seed=11, ik=1):
    w = configs.si2_fcc()
    d = configs.kpoint_inputs(w, ik)
    psi = configs.random_psi(d["mtxd"], nb, seed)
    return w, d, psi, np.full(nb, 2.0)


def _restated(w, d, psi, occ):
    m = d["mtxd"]
    rk = OS.strkin(d["rkpt"], m, d["isort"], d["kgv"], psi, occ)
    rl = OS.strhl(OS.rho_of(d, psi, occ), w.species, w.adot, w.box)
    rn = OS.strnlkb(d["rkpt"], m, d["isort"], d["kgv"], psi, occ, w.species, d["vkb"], d["nkb"], w.adot)
    return rk, rl, rn


def test_restated_stress_matches_finite_differences():
    w, d, psi, occ = _case()
    rk, rl, rn = _restated(w, d, psi, occ)
    fd = OS.fd_covariant_stress(d, w.species, w.adot, w.box, w.idpad, psi, occ)
    assert np.abs(rk + rl + rn - fd).max() <= 1e-6 * np.abs(fd).max()


@pytest.mark.parametrize("ik", [0, 3])
def test_host_contractions_match_restatement(ik):
    w, d, psi, occ = _case(nb=4, seed=5 + ik, ik=ik)
    m = d["mtxd"]
    wG = np.sum(occ[None, :] * np.abs(psi[:m]) ** 2, axis=1)
    P = d["anlga"].conj().T @ psi[:m]
    Y = psi[:m] @ (occ[:, None] * P.conj().T * d["xnlkb"][None, :])
    rho = OS.rho_of(d, psi, occ)
    cov = lambda S: ST.covariant(ST.strain_to_metric(S, w.adot), w.adot)
    Sl, _ = ST.local_strain(rho, w.species, w.adot, w.box)
    Sn, _ = ST.kb_strain(Y, d, w.species, w.adot)
    rk, rl, rn = _restated(w, d, psi, occ)
    for got, ref in ((cov(ST.kinetic_strain(wG, d, w.adot)), rk), (cov(Sl), rl), (cov(Sn), rn)):
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
