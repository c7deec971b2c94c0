"""CPU tests of the oracle (restated reference algorithm) against known answers.

The reference ships no function-level golden vectors for hk_psi_c16 /
ditsp_c16, so the oracle is pinned here by analytic transforms, explicit dense
matrix elements, Hermiticity and dense-diagonalisation ground truth, plus the
committed fixtures in tests/golden (regression of the oracle itself).
"""
import json
import os

import numpy as np
import pytest

from cpw2000_b200 import configs, crystal
from oracle import ditsp as D
from oracle import fft as F
from oracle import hk_psi as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def small():
    w = configs.small_test()
    return w, configs.kpoint_inputs(w, 1, with_hamsm=True)


@pytest.fixture(scope="module")
def si2():
    w = configs.si2_fcc()
    return w, configs.kpoint_inputs(w, 0, with_hamsm=True)


def test_size_fft_matches_reference_table():
    # size_fft.f90: 2k+1 < 32 -> first of the primary list; else 2^(p-5) * secondary
    assert crystal.size_fft((15, 15, 15)) == (32, 32, 32)
    assert crystal.size_fft((19, 47, 71)) == (40, 96, 144)
    assert crystal.size_fft((0, 1, 2)) == (2, 4, 6)
    assert crystal.size_fft((36, 37, 40)) == (80, 80, 96)


@pytest.mark.parametrize("mode", [-1, 1])
def test_cfft_wf_single_plane_wave(mode):
    n1, n2, n3, nn1 = 24, 20, 18, 25
    kd = (3, 4, 2)
    m = (2, -3, 1)
    box = np.zeros(nn1 * n2 * n3, dtype=np.complex128)
    b3 = box.reshape(n3, n2, nn1)
    if mode == -1:
        b3[m[2] % n3, m[1] % n2, m[0] % n1] = 1.0
        F.cfft_wf_c16(box, nn1, n1, n2, n3, *kd, -1)
        x = np.arange(n1)[None, None, :] / n1
        y = np.arange(n2)[None, :, None] / n2
        z = np.arange(n3)[:, None, None] / n3
        ref = np.exp(2j * np.pi * (m[0] * x + m[1] * y + m[2] * z))
        assert np.abs(b3[:, :, :n1] - ref).max() < 1e-13
    else:
        x = np.arange(n1)[None, None, :] / n1
        y = np.arange(n2)[None, :, None] / n2
        z = np.arange(n3)[:, None, None] / n3
        b3[:, :, :n1] = np.exp(2j * np.pi * (m[0] * x + m[1] * y + m[2] * z))
        F.cfft_wf_c16(box, nn1, n1, n2, n3, *kd, 1)
        got = b3[m[2] % n3, m[1] % n2, m[0] % n1]
        assert abs(got - 1.0) < 1e-13
        # another kept frequency is zero
        assert abs(b3[0, 0, 0]) < 1e-13


def test_hk_psi_matches_dense_matrix(small):
    w, d = small
    m = d["mtxd"]
    psi = configs.random_psi(m, 5, 3)
    hp = O.hk_psi_c16(m, 5, psi, d["ekpg"], d["isort"], d["vscr"], d["kmscr"], d["kgv"], d["anlga"], d["xnlkb"])
    H = O.dense_h(m, d["ekpg"], d["isort"], d["vscr"], d["kmscr"], d["kgv"], d["anlga"], d["xnlkb"])
    assert np.abs(H - H.conj().T).max() < 1e-13
    assert np.abs(hp - H @ psi).max() < 1e-12 * np.abs(hp).max()


def test_hk_psi_single_plane_wave_elements(si2):
    """<G_i|H|G_j> from H applied to a unit vector equals ekpg + Vt(G_i-G_j) + KB term."""
    w, d = si2
    m = d["mtxd"]
    j = 7
    e = np.zeros((m, 1), dtype=np.complex128)
    e[j, 0] = 1.0
    hp = O.hk_psi_c16(m, 1, e, d["ekpg"], d["isort"], d["vscr"], d["kmscr"], d["kgv"], d["anlga"], d["xnlkb"])[:, 0]
    n1, n2, n3, ident = d["kmscr"][3:7]
    vb = d["vscr"].reshape(n3, n2, ident)[:, :, :n1].transpose(2, 1, 0)
    vt = np.fft.fftn(vb) / (n1 * n2 * n3)
    g = d["kgv"][:, d["isort"] - 1]
    dg = g - g[:, j:j + 1]
    ref = vt[dg[0] % n1, dg[1] % n2, dg[2] % n3]
    ref[j] += d["ekpg"][j]
    ref += (d["anlga"] * d["xnlkb"][None, :]) @ d["anlga"][j].conj()
    assert np.abs(hp - ref).max() < 1e-13


def test_hermiticity(si2):
    w, d = si2
    m = d["mtxd"]
    a = configs.random_psi(m, 2, 11)
    hp = O.hk_psi_c16(m, 2, a, d["ekpg"], d["isort"], d["vscr"], d["kmscr"], d["kgv"], d["anlga"], d["xnlkb"])
    lhs = np.vdot(a[:, 0], hp[:, 1])
    rhs = np.conj(np.vdot(a[:, 1], hp[:, 0]))
    assert abs(lhs - rhs) < 1e-10 * abs(lhs)


def test_wraparound_is_an_error(small):
    w, d = small
    km = d["kmscr"].copy()
    km[3:6] = (6, 6, 6)
    km[6] = 6
    with pytest.raises(ValueError):
        O.ipoint_of(d["mtxd"], d["isort"], d["kgv"], km)


def test_ran2_restart_is_deterministic():
    r = D.Ran2()
    s = [-1]
    a = [r(s) for _ in range(5)]
    r2 = D.Ran2()
    s2 = [-1]
    b = [r2(s2) for _ in range(5)]
    assert a == b
    assert all(0.0 < v < 1.0 for v in a)
    with open(os.path.join(GOLD, "ran2_seed_minus1.json")) as f:
        gold = json.load(f)
    r3 = D.Ran2()
    s3 = [-1]
    c = [r3(s3) for _ in range(len(gold["values"]))]
    assert c == gold["values"]


def test_grsch_loop_orthonormalises_and_drops_dependent():
    rng = np.random.default_rng(0)
    x = rng.standard_normal((200, 14)) + 1j * rng.standard_normal((200, 14))
    x[:, :3] = np.linalg.qr(x[:, :3])[0]              # the nconv columns are orthonormal on entry
    x[:, 9] = x[:, 2] * (0.3 - 0.1j) + x[:, 4]       # linearly dependent
    hx = x.copy()
    irow = D.grsch_loop(True, x, hx, 3, 14)
    assert irow[9] == 0 and irow.sum() == 13
    keep = np.nonzero(irow)[0]
    q = x[:, keep]
    assert np.abs(q[:, 3:].conj().T @ q[:, 3:] - np.eye(len(keep) - 3)).max() < 1e-12
    assert np.abs(x - hx).max() < 1e-12   # companion transformed identically


def test_ditsp_matches_dense_eigenvalues(si2):
    w, d = si2
    m = d["mtxd"]
    nb = 8
    hk = lambda X: O.hk_psi_c16(m, X.shape[1], X, d["ekpg"], d["isort"], d["vscr"], d["kmscr"], d["kgv"],
                                d["anlga"], d["xnlkb"])
    psi = np.zeros((m, 3 * nb), dtype=np.complex128, order="F")
    hpsi = np.zeros_like(psi)
    r = D.ditsp_c16(hk, nb, m, d["mtxds"], psi, hpsi, d["hamsm"], d["hdiag"], epspsi=1e-5, icmax=40,
                    mxdbnd=3 * nb)
    assert r["ifail"] == 0
    H = O.dense_h(m, d["ekpg"], d["isort"], d["vscr"], d["kmscr"], d["kgv"], d["anlga"], d["xnlkb"])
    ev = np.linalg.eigvalsh(H)
    assert np.abs(r["ei"] - ev[: r["neig"]]).max() < 1e-8
    assert D.ditsp_error(psi[:, :nb], hpsi[:, :nb]) < 1e-10


def test_ditsp_full_diagonalisation_path(small):
    w, d = small
    m = d["mtxd"]
    assert d["mtxds"] == m        # mtxd < 250: size_mtxds picks the full matrix
    psi = np.zeros((m, 6), dtype=np.complex128, order="F")
    hpsi = np.zeros_like(psi)
    r = D.ditsp_c16(None, 6, m, d["mtxds"], psi, hpsi, d["hamsm"], d["hdiag"], mxdbnd=6)
    H = O.dense_h(m, d["ekpg"], d["isort"], d["vscr"], d["kmscr"], d["kgv"], d["anlga"], d["xnlkb"])
    assert np.abs(r["ei"] - np.linalg.eigvalsh(H)[:6]).max() < 1e-12


def test_golden_hkpsi_fixture():
    """Regression: the oracle reproduces its committed small-case output."""
    z = np.load(os.path.join(GOLD, "hkpsi_small.npz"))
    w = configs.small_test()
    d = configs.kpoint_inputs(w, 1)
    assert d["mtxd"] == int(z["mtxd"])
    hp = O.hk_psi_c16(d["mtxd"], z["psi"].shape[1], z["psi"], d["ekpg"], d["isort"], d["vscr"], d["kmscr"],
                      d["kgv"], d["anlga"], d["xnlkb"])
    assert np.abs(hp - z["hpsi"]).max() < 1e-12 * np.abs(z["hpsi"]).max()


def test_potential_coefficients_reproduce_host_vscr():
    # the star arguments the pot_local tests give the device reproduce the host potential
    from cpw2000_b200 import configs as CF, pseudo as PS
    w = CF.WORKLOADS["si2"]()
    want, _ = PS.local_potential_box(w.species, w.adot, w.box, 2)
    kgv, vg = PS.local_potential_coefficients(w.species, w.adot, w.box)
    n1, n2, n3 = w.box
    box = np.zeros((n1, n2, n3), complex)
    box[kgv[0] % n1, kgv[1] % n2, kgv[2] % n3] = vg
    vr = np.fft.ifftn(box) * box.size
    got = np.zeros((n3, n2, n1 + 2))
    got[:, :, :n1] = vr.real.transpose(2, 1, 0)
    assert np.abs(got.ravel() - want).max() <= 1e-13 * np.abs(want).max()


def test_spin_restatement_components_and_hermiticity():
    # nsp = 1 acts on each component like hk_psi_c16; the nsp = 4 operator is Hermitian
    w = configs.WORKLOADS["si2"]()
    d = configs.kpoint_inputs(w, 0)
    m, nb = d["mtxd"], 2
    rng = np.random.default_rng(0)
    psi = rng.standard_normal((2 * m, nb)) + 1j * rng.standard_normal((2 * m, nb))
    none2, none = np.zeros((2 * m, 0), complex), np.zeros((m, 0), complex)
    h = O.hk_psi_spin_c16(m, nb, psi, d["ekpg"], d["isort"], d["vscr"][:, None], d["kmscr"], d["kgv"], 1, none2,
                          np.zeros(0))
    for c in range(2):
        hc = O.hk_psi_c16(m, nb, np.ascontiguousarray(psi[c::2]), d["ekpg"], d["isort"], d["vscr"], d["kmscr"],
                          d["kgv"], none, np.zeros(0))
        assert np.abs(h[c::2] - hc).max() <= 1e-12 * np.abs(hc).max()
    v4 = np.zeros((d["vscr"].size, 4))
    v4[:, 0] = d["vscr"]
    v4[:, 1:] = 0.3 * rng.standard_normal((d["vscr"].size, 3))
    a, b = psi[:, :1], psi[:, 1:]
    ha = O.hk_psi_spin_c16(m, 1, a, d["ekpg"], d["isort"], v4, d["kmscr"], d["kgv"], 4, none2, np.zeros(0))
    hb = O.hk_psi_spin_c16(m, 1, b, d["ekpg"], d["isort"], v4, d["kmscr"], d["kgv"], 4, none2, np.zeros(0))
    x, y = (b.conj() * ha).sum(), (hb.conj() * a).sum()
    assert abs(x - y) <= 1e-12 * abs(x)
