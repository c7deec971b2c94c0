"""CPU tests of the restated hamilt_kb (oracle/hamilt.py).

Pinned against the matrix of the H|psi> operator itself: on the start basis of a k-point the
small Hamiltonian from the star representation (one star per G vector, and again with G and
-G paired into one star through the conj flag) equals the block E^H H E the eigensolver's
inputs carry (pseudo.small_hamiltonian, built from the FFT-box potential and the projectors),
to rounding.
"""
import numpy as np
import pytest

from cpw2000_b200 import configs, pseudo
from cpw2000_b200.crystal import adot_to_bdot
from oracle import hamilt as OH


def star_inputs(w, d, pair_stars):
    """hamilt_kb's arguments for workload w, k-point inputs d: the box's G vectors (Nyquist
    planes left out) as the G list, one star per G or per (G, -G) pair."""
    kg, vg = pseudo.local_potential_coefficients(w.species, w.adot, w.box)
    kg = kg.astype(np.int64)
    ng = kg.shape[1]
    index = {tuple(kg[:, n]): n for n in range(ng)}
    # the basis in this G list
    gb = d["kgv"][:, d["isort"] - 1]
    isort = np.array([index[tuple(gb[:, i])] + 1 for i in range(gb.shape[1])])
    kmax = np.abs(kg).max(axis=1)
    imx, jmx, kmx = 2 * kmax + 1
    indv = np.zeros(imx * jmx * kmx, dtype=np.int64)
    for n in range(ng):
        kx, ky, kz = kg[:, n] + kmax + 1
        indv[((kx - 1) * jmx + ky - 1) * kmx + kz - 1] = n + 1
    _, bdot = adot_to_bdot(w.adot)
    ekg = 0.5 * np.einsum("in,ij,jn->n", kg, bdot, kg)
    sf = np.stack([np.exp(-2j * np.pi * (np.asarray(sp.rat) @ kg)).sum(axis=0) for sp in w.species])
    phase = np.ones(ng, dtype=np.complex128)
    conj = np.ones(ng)
    if not pair_stars:
        inds = np.arange(1, ng + 1)
        return isort, kg, phase, conj, inds, kmax, indv, ekg, sf, vg
    # stars {G, -G}: the member with the first nonzero component positive is the prototype
    inds = np.zeros(ng, dtype=np.int64)
    proto = []
    for n in range(ng):
        g = kg[:, n]
        nz = g[np.nonzero(g)[0][0]] if np.any(g) else 1
        if nz > 0 or not np.any(g):
            proto.append(n)
            inds[n] = len(proto)
    for n in range(ng):
        if inds[n] == 0:
            inds[n] = inds[index[tuple(-kg[:, n])]]
            conj[n] = -1.0
    proto = np.array(proto)
    return isort, kg, phase, conj, inds, kmax, indv, ekg[proto], sf[:, proto], vg[proto]


@pytest.mark.parametrize("ik,pair", [(0, False), (3, False), (5, True)])
def test_hamilt_kb_equals_operator_block(ik, pair):
    w = configs.si2_fcc()
    d = configs.kpoint_inputs(w, ik, with_hamsm=True)
    mtxds = d["mtxds"]
    assert mtxds < d["mtxd"]
    isort, kg, phase, conj, inds, kmax, indv, ek, sf, veff = star_inputs(w, d, pair)
    nt = len(w.species)
    hk = OH.hamilt_kb(mtxds, d["hdiag"], isort, d["qmod"], kg, phase, conj, inds, kmax, indv, ek, sf, veff,
                      np.full(nt, 4000), np.full(nt, 0.01), d["vkb"], d["nkb"], w.adot)
    ref = d["hamsm"][:mtxds, :mtxds]
    assert np.abs(hk - ref).max() < 1e-12 * np.abs(ref).max()
