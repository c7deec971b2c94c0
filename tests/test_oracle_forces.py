"""CPU: the oracle's force restatements against central finite differences of
E(tau) = sum_n f_n <psi_n|H(tau)|psi_n> with psi fixed (exact for Hellmann-Feynman
forces), and the density against an explicit |psi(r)|^2 sum."""
import numpy as np
import pytest

from cpw2000_b200 import configs, pseudo
from oracle import forces as F


def _energy(w, d, psi, occ, rat_override):
    sp = [pseudo.Species(s.v0, s.sigma, s.ekb, s.sigma_kb, r) for s, r in zip(w.species, rat_override)]
    vscr, _ = pseudo.local_potential_box(sp, w.adot, w.box, w.idpad)
    anl, xnl = pseudo.proj_nl_kb(d["rkpt"], d["isort"], d["kgv"], sp, d["vkb"], d["nkb"], w.adot)
    return F.hf_energy(d["mtxd"], psi, occ, d["ekpg"], d["isort"], vscr, d["kmscr"], d["kgv"], anl, xnl)


def test_oracle_forces_match_finite_differences():
    w = configs.small_test()
    d = configs.kpoint_inputs(w, 1)
    nb = 3
    psi = configs.random_psi(d["mtxd"], nb, 4)
    psi /= np.linalg.norm(psi, axis=0)[None, :]
    occ = np.array([2.0, 2.0, 1.0])
    rho = F.charge_by_fft(d["mtxd"], nb, psi, occ, d["isort"], d["kgv"], d["kmscr"])
    vgt = pseudo.local_form_factors_box(w.species, w.adot, w.box)
    fl = F.local_force(rho, w.species, vgt, d["kmscr"])
    fn = F.for_str_nl_kb_forces(d["rkpt"], d["mtxd"], d["isort"], d["kgv"], psi, occ, w.species, d["vkb"],
                                d["nkb"], w.adot)
    ftot = fl + fn
    h = 1e-4
    rats = [s.rat.copy() for s in w.species]
    k = 0
    for t, s in enumerate(w.species):
        for a in range(s.natom):
            for j in range(3):
                rp = [r.copy() for r in rats]
                rm = [r.copy() for r in rats]
                rp[t][a, j] += h
                rm[t][a, j] -= h
                fd = -(_energy(w, d, psi, occ, rp) - _energy(w, d, psi, occ, rm)) / (2 * h)
                assert abs(fd - ftot[k, j]) < 1e-6 * max(1.0, abs(fd)), (t, a, j, fd, ftot[k, j])
            k += 1


def test_charge_by_fft_is_sum_of_squared_moduli():
    w = configs.small_test()
    d = configs.kpoint_inputs(w, 0)
    psi = configs.random_psi(d["mtxd"], 2, 8)
    rho = F.charge_by_fft(d["mtxd"], 2, psi, [1.0, 0.5], d["isort"], d["kgv"], d["kmscr"])
    n1, n2, n3 = w.box
    g = d["kgv"][:, d["isort"] - 1]
    x = np.arange(n1)[None, None, :] / n1
    y = np.arange(n2)[None, :, None] / n2
    z = np.arange(n3)[:, None, None] / n3
    ref = np.zeros((n3, n2, n1))
    for b, f in enumerate([1.0, 0.5]):
        v = np.zeros((n3, n2, n1), dtype=np.complex128)
        for i in range(d["mtxd"]):
            v += psi[i, b] * np.exp(2j * np.pi * (g[0, i] * x + g[1, i] * y + g[2, i] * z))
        ref += f * np.abs(v) ** 2
    assert np.abs(rho - ref).max() < 1e-10 * ref.max()
