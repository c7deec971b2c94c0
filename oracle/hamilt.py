"""The small dense Hamiltonian of the start basis, restated from the reference (CPU) -- test
infrastructure only (see oracle/__init__.py).

hamilt_kb -- Src/ALFA/hamilt_kb.f90:1-234: hamk(i, j) for the first mtxd plane waves of a
    k-point from the star representation of the potential: the diagonal hdiag, the local part
    veff(star of G_i - G_j) with the G vector's phase (conjugated when conj = -1), and the KB
    part through the Legendre addition theorem, sum_l vq_l(|k+G_i|) vq_l(|k+G_j|) nkb_l
    P_l(cos angle) times the structure factor of the star, per atom type.
"""
from __future__ import annotations

import math

import numpy as np

from cpw2000_b200.crystal import adot_to_bdot

EPS = float(np.float32(0.1e-8))      # hamilt_kb.f90:92, a default-real literal


def _vq(q, vtab, nq, delq, fac, l):
    """fac * v_l(q) * q^l with the quadratic interpolation of hamilt_kb.f90:172-198 (vtab indexed
    from q index -2)."""
    xn = q / delq
    n = np.maximum(np.floor(xn + 0.5).astype(np.int64), 0)          # nint, q >= 0
    ok = n < nq - 1
    nc = np.where(ok, n, 0)
    x = xn - nc
    v = vtab[nc + 2] * (1 + x) * (1 - x) + (vtab[nc + 3] * (1 + x) - vtab[nc + 1] * (1 - x)) * x / 2
    return np.where(ok, fac * v * q ** l, 0.0)


def hamilt_kb(mtxd, hdiag, isort, qmod, kgv, phase, conj, inds, kmax, indv, ek, sfact, veff, nqnl, delqnl, vkb,
              nkb, adot):
    """hamk (mtxd, mtxd) complex128.

    kgv (3, ng) int, phase (ng,) complex, conj (ng,) +-1, inds (ng,) 1-based stars, kmax (3,),
    indv (imx*jmx*kmx,) 1-based G index of each cube point (0 = none), ek (ns,), sfact
    (ntype, ns) complex, veff (ns,) complex, nqnl/delqnl (ntype,), vkb (ntype, 4, nq + 3) from
    q index -2, nkb (ntype, 4). Follows :123-234: lower triangle element by element (here all
    pairs i > j at once), then the Hermitian completion.
    """
    vcell, _ = adot_to_bdot(adot)
    fac = 1.0 / math.sqrt(vcell)
    imx, jmx, kmx = (2 * int(k) + 1 for k in kmax)
    isort = np.asarray(isort[:mtxd], dtype=np.int64) - 1
    q = np.asarray(qmod[:mtxd], dtype=np.float64)
    ii, jj = np.tril_indices(mtxd, -1)
    d = kgv[:, isort[ii]].astype(np.int64) - kgv[:, isort[jj]].astype(np.int64)
    kxd = d[0] + kmax[0] + 1
    kyd = d[1] + kmax[1] + 1
    kzd = d[2] + kmax[2] + 1
    inside = (kxd >= 1) & (kxd <= imx) & (kyd >= 1) & (kyd <= jmx) & (kzd >= 1) & (kzd <= kmx)
    cube = np.where(inside, ((kxd - 1) * jmx + kyd - 1) * kmx + kzd, 1) - 1
    kadd = np.where(inside, np.asarray(indv)[cube], 0)
    valid = kadd != 0
    ka = np.where(valid, kadd - 1, 0)
    st = np.asarray(inds)[ka] - 1
    ph = np.conj(np.asarray(phase)[ka])
    cj = np.asarray(conj)[ka] < 0
    h = np.asarray(veff)[st] * ph
    # the Legendre polynomials of the angle between k+G_i and k+G_j (:162-170)
    qi, qj = q[ii], q[jj]
    small = (qi > EPS) & (qj > EPS)
    gama = np.where(small, (qi * qi + qj * qj - 2 * np.asarray(ek)[st]) / np.where(small, qi * qj * 2, 1.0), 1.0)
    plg = [np.ones_like(gama), gama, (3 * gama * gama - 1) / 2, gama * (5 * gama * gama - 3) / 2]
    for nt in range(len(nqnl)):
        vnl = np.zeros_like(gama)
        for l in range(4):
            if nkb[nt, l] == 0:
                continue
            vqi = _vq(q, vkb[nt, l], nqnl[nt], delqnl[nt], fac, l)
            vnl += vqi[ii] * vqi[jj] * nkb[nt, l] * plg[l]
        h = h + vnl * np.asarray(sfact)[nt, st] * ph
    h = np.where(cj, np.conj(h), h)
    h = np.where(valid, h, 0.0)
    hamk = np.zeros((mtxd, mtxd), dtype=np.complex128)
    hamk[ii, jj] = h
    hamk = hamk + hamk.conj().T
    hamk[np.arange(mtxd), np.arange(mtxd)] = np.asarray(hdiag[:mtxd], dtype=np.float64)
    return hamk
