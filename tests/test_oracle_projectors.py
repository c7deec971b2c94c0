"""CPU tests of the restated proj_nl_kb_der_c16 (oracle/projectors.py).

Pinned three ways: its projectors equal the restated proj_nl_kb_c16 (pseudo.proj_nl_kb)
to rounding; its first derivatives with respect to the k-point's lattice coordinates match
central finite differences of the projectors; its second derivatives match central finite
differences of its first derivatives. s, p, d and f channels of two atom types, a k-point
off Gamma (and the |k+G| = 0 branch at Gamma).
"""
import numpy as np
import pytest

from cpw2000_b200 import configs, pseudo
from oracle import projectors as OP


def _setup(ik):
    w = configs.WORKLOADS["si2"]()
    species = [pseudo.Species(v0=sp.v0, sigma=sp.sigma, ekb=(2.0, -1.5, 0.7, -0.3), sigma_kb=0.9, rat=sp.rat)
               for sp in w.species]
    species.append(pseudo.Species(v0=1.0, sigma=0.7, ekb=(0.0, 1.1), sigma_kb=0.8,
                                  rat=np.array([[0.3, 0.1, 0.2]])))
    d = configs.kpoint_inputs(w, ik)
    vkb, nkb = pseudo.kb_tables(species, 0.01, 4000, lmax=3)
    return w, species, d, vkb, nkb


def _der(w, species, d, vkb, nkb, rk, nder):
    nt = len(species)
    return OP.proj_nl_kb_der_c16(rk, d["isort"], d["kgv"], [sp.rat for sp in species], vkb, nkb,
                                 np.full(nt, 4000), np.full(nt, 0.01), w.adot, nder)


def test_projectors_equal_proj_nl_kb():
    w, species, d, vkb, nkb = _setup(2)
    a, x, _, _ = _der(w, species, d, vkb, nkb, d["rkpt"], 0)
    want, xw = pseudo.proj_nl_kb(d["rkpt"], d["isort"], d["kgv"], species, vkb, nkb, w.adot)
    assert a.shape == want.shape and a.shape[1] == 16 * 2 + 3
    assert np.abs(a - want).max() < 1e-13 * np.abs(want).max()
    assert np.array_equal(x, xw)


@pytest.mark.parametrize("ik", [2, 0])
def test_derivatives_match_finite_differences(ik):
    w, species, d, vkb, nkb = _setup(ik)
    rk = np.asarray(d["rkpt"], dtype=np.float64)
    a, _, da, d2a = _der(w, species, d, vkb, nkb, rk, 2)
    h = 1e-5
    scale1 = np.abs(da).max()
    scale2 = np.abs(d2a).max()
    # rows with |k+G| near a midpoint of the interpolation table (the derivative of the
    # piecewise interpolant jumps there) or near zero are left out of the comparison
    from cpw2000_b200.crystal import adot_to_avec
    _, bvec = adot_to_avec(w.adot)
    q = bvec @ (d["kgv"][:, d["isort"] - 1] + rk[:, None])
    xq = np.sqrt((q ** 2).sum(axis=0)) / 0.01
    frac = np.abs(xq - np.floor(xq) - 0.5)
    keep = (frac > 0.02) & (xq > 0.5)
    for n in range(3):
        e = np.zeros(3)
        e[n] = h
        ap, _, dap, _ = _der(w, species, d, vkb, nkb, rk + e, 1)
        am, _, dam, _ = _der(w, species, d, vkb, nkb, rk - e, 1)
        fd = (ap - am) / (2 * h)
        assert np.abs(fd - da[:, :, n])[keep].max() < 1e-6 * scale1
        fd2 = (dap - dam) / (2 * h)                       # (i, ind, j) = d/drk_n of da(:, :, j)
        assert np.abs(fd2 - d2a[:, :, :, n])[keep].max() < 1e-5 * scale2
    # symmetry of the second derivative
    assert np.abs(d2a - d2a.transpose(0, 1, 3, 2)).max() < 1e-12 * scale2
