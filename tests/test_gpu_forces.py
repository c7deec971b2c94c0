"""GPU adjoint of H|psi>: density, dE/dV_loc and Hellmann-Feynman forces.

Checked against the oracle's restatements of charge_by_fft / for_str_nl_kb /
the local structure-factor force, and against central finite differences of
the GPU energy E(tau) with psi fixed. Tolerances: density 1e-12 relative;
forces 1e-8 Ha/bohr vs the oracle; finite differences (h = 1e-3 bohr) 1e-5 Ha/bohr.
"""
import numpy as np
import pytest
import torch

from cpw2000_b200 import configs, pseudo
from cpw2000_b200 import ditsp as E
from cpw2000_b200 import forces as FF
from cpw2000_b200 import hk_psi as H
from oracle import forces as OF

pytestmark = pytest.mark.gpu


def _system(w, ik, nb, seed, dev, normalise=True):
    d = configs.kpoint_inputs(w, ik)
    psi_h = configs.random_psi(d["mtxd"], nb, seed)
    if normalise:
        psi_h /= np.linalg.norm(psi_h, axis=0)[None, :]
    psi = torch.from_numpy(np.ascontiguousarray(psi_h.T)).to(dev).t()
    occ = np.linspace(2.0, 1.0, nb)
    return d, psi_h, FF.HFSystem(w, d, psi, occ)


def _oracle_forces(w, d, psi_h, occ):
    rho = OF.charge_by_fft(d["mtxd"], len(occ), psi_h, occ, d["isort"], d["kgv"], d["kmscr"])
    vgt = pseudo.local_form_factors_box(w.species, w.adot, w.box)
    return (OF.local_force(rho, w.species, vgt, d["kmscr"]) +
            OF.for_str_nl_kb_forces(d["rkpt"], d["mtxd"], d["isort"], d["kgv"], psi_h, occ, w.species, d["vkb"],
                                    d["nkb"], w.adot))


def test_density_matches_oracle(cuda):
    w = configs.si2_fcc()
    d, psi_h, s = _system(w, 3, 6, 1, cuda)
    rho = s.density().cpu().numpy()
    ref = OF.charge_by_fft(d["mtxd"], 6, psi_h, s.occ, d["isort"], d["kgv"], d["kmscr"])
    assert np.abs(rho - ref).max() < 1e-12 * ref.max()


@pytest.mark.parametrize("wname,ik", [("small", 1), ("si2", 2)])
def test_forces_match_oracle(cuda, wname, ik):
    w = configs.WORKLOADS[wname]()
    d, psi_h, s = _system(w, ik, 4, 2, cuda)
    e, f = FF.forces(s)
    ref = _oracle_forces(w, d, psi_h, s.occ)
    fc = FF.to_cartesian(f, w.adot)
    rc = FF.to_cartesian(ref, w.adot)
    assert np.abs(fc - rc).max() < 1e-8
    eo = OF.hf_energy(d["mtxd"], psi_h, s.occ, d["ekpg"], d["isort"], d["vscr"], d["kmscr"], d["kgv"], d["anlga"],
                      d["xnlkb"])
    assert abs(e - eo) < 1e-10 * abs(eo)


def test_forces_match_finite_differences(cuda):
    w = configs.small_test()
    d, psi_h, s = _system(w, 1, 3, 5, cuda)
    _, f = FF.forces(s)
    fc = FF.to_cartesian(f, w.adot)
    avec, _ = FF.adot_to_avec(w.adot)
    h = 1e-3                                       # bohr, Cartesian
    tau0 = s.tau0()
    for atom, j in ((0, 0), (1, 2), (2, 1)):
        dl = np.linalg.solve(avec, h * np.eye(3)[j])   # lattice displacement for a Cartesian step
        tp = tau0.clone()
        tm = tau0.clone()
        tp[atom] += torch.from_numpy(dl)
        tm[atom] -= torch.from_numpy(dl)
        ep = float(FF.energy(tp, s))
        em = float(FF.energy(tm, s))
        assert abs(-(ep - em) / (2 * h) - fc[atom, j]) < 1e-5


def test_dE_dvscr_is_density_over_n(cuda):
    w = configs.small_test()
    d, psi_h, s = _system(w, 0, 3, 6, cuda)
    tau = s.tau0()
    v = torch.from_numpy(d["vscr"].copy()).to(cuda).requires_grad_(True)
    e = FF.HFEnergy.apply(tau, v, s)
    e.backward()
    g = v.grad.cpu().numpy()
    n1, n2, n3 = w.box
    rng = np.random.default_rng(0)
    for _ in range(3):
        z, y, x = rng.integers(0, n3), rng.integers(0, n2), rng.integers(0, n1)
        k = (z * n2 + y) * (n1 + w.idpad) + x
        hv = 1e-3
        vp = d["vscr"].copy()
        vm = d["vscr"].copy()
        vp[k] += hv
        vm[k] -= hv
        fd = (float(FF.HFEnergy.apply(tau, torch.from_numpy(vp).to(cuda), s)) -
              float(FF.HFEnergy.apply(tau, torch.from_numpy(vm).to(cuda), s))) / (2 * hv)
        assert abs(fd - g[k]) < 1e-9 * max(1.0, abs(fd))


def test_zincblende64_forces_from_converged_states(cuda):
    """Config: ZB64 (two species, 192 force components), converged FP64 states."""
    w = configs.zb64_cubic()
    d = configs.kpoint_inputs(w, 0, with_hamsm=True)
    nb = 128                                         # occupied bands of the 160 solved
    ctx = H.Context(0).setup(d)
    ctx.set_slab_budget(4 << 30)
    P = torch.zeros((3 * 160, d["mtxd"]), dtype=torch.complex128, device=cuda).t()
    HP = torch.zeros_like(P)
    r = E.eigensolve(ctx, P, HP, 160, d["mtxds"], d["hamsm"], d["hdiag"], epspsi=1e-5, icmax=60)
    psi = P[:, :nb].contiguous() if False else torch.clone(P[:, :nb].t()).t()
    s = FF.HFSystem(w, d, psi, np.full(nb, 2.0))
    _, f = FF.forces(s)
    fc = FF.to_cartesian(f, w.adot)
    assert fc.shape == (64, 3)
    psi_h = psi.cpu().numpy()
    ref = FF.to_cartesian(_oracle_forces(w, d, psi_h, s.occ), w.adot)
    assert np.abs(fc - ref).max() < 1e-8
    avec, _ = FF.adot_to_avec(w.adot)
    h = 1e-3
    tau0 = s.tau0()
    for atom, j in ((5, 0), (40, 2)):
        dl = torch.from_numpy(np.linalg.solve(avec, h * np.eye(3)[j]))
        ep = float(FF.energy(tau0 + torch.nn.functional.one_hot(torch.tensor(atom), 64).double()[:, None] * dl, s))
        em = float(FF.energy(tau0 - torch.nn.functional.one_hot(torch.tensor(atom), 64).double()[:, None] * dl, s))
        assert abs(-(ep - em) / (2 * h) - fc[atom, j]) < 1e-5
    assert r["ei"][0] < r["ei"][-1]
