"""KB projectors and their k-point derivatives, restated from the reference (CPU) -- test
infrastructure only (see oracle/__init__.py).

proj_nl_kb_der_c16 -- Src/omp/proj_nl_kb_der_c16.f90:25-417: the projectors anlga of
    Src/omp/proj_nl_kb_c16.f90 with their first and second derivatives with respect to the
    k-point's lattice coordinates (nder = 0, 1, 2).
rylm_derivatives   -- the solid harmonics r^l sqrt(4 pi/(2l+1)) Y_lm of Src/numeric/ylm_rc.f90
    (real combinations, l <= 3) with their Cartesian gradient and Hessian, as ylm_rc returns
    them for nder = 1, 2. Each harmonic is a homogeneous polynomial of degree l; the table
    below lists its monomials x^a y^b z^c with their coefficients, and the derivatives are
    those of the polynomials.
"""
from __future__ import annotations

import math

import numpy as np

from cpw2000_b200.crystal import adot_to_avec, adot_to_bdot

PI = math.pi
EPS = 1.0e-8            # proj_nl_kb_der_c16.f90:121, below it |k+G| is treated as zero
LMAX = 3

_S3, _S58, _S15, _S38, _S154 = (math.sqrt(3.0), math.sqrt(5.0 / 8), math.sqrt(15.0), math.sqrt(3.0 / 8),
                                math.sqrt(15.0 / 4))
# (l, m) -> [(coefficient, (a, b, c)), ...] for x^a y^b z^c (same polynomials as ylm_rc.f90:82-106)
RYLM_MONOMIALS = {
    (0, 0): [(1.0, (0, 0, 0))],
    (1, -1): [(1.0, (0, 1, 0))],
    (1, 0): [(1.0, (0, 0, 1))],
    (1, 1): [(1.0, (1, 0, 0))],
    (2, -2): [(_S3, (1, 1, 0))],
    (2, -1): [(_S3, (0, 1, 1))],
    (2, 0): [(1.0, (0, 0, 2)), (-0.5, (2, 0, 0)), (-0.5, (0, 2, 0))],
    (2, 1): [(_S3, (1, 0, 1))],
    (2, 2): [(math.sqrt(0.75), (2, 0, 0)), (-math.sqrt(0.75), (0, 2, 0))],
    (3, -3): [(3 * _S58, (2, 1, 0)), (-_S58, (0, 3, 0))],
    (3, -2): [(_S15, (1, 1, 1))],
    (3, -1): [(4 * _S38, (0, 1, 2)), (-_S38, (2, 1, 0)), (-_S38, (0, 3, 0))],
    (3, 0): [(1.0, (0, 0, 3)), (-1.5, (2, 0, 1)), (-1.5, (0, 2, 1))],
    (3, 1): [(4 * _S38, (1, 0, 2)), (-_S38, (3, 0, 0)), (-_S38, (1, 2, 0))],
    (3, 2): [(_S154, (2, 0, 1)), (-_S154, (0, 2, 1))],
    (3, 3): [(-3 * _S58, (1, 2, 0)), (_S58, (3, 0, 0))],
}


def _pw(x, e):
    return np.ones_like(x) if e == 0 else x ** e


def rylm_derivatives(qcar: np.ndarray, l: int, m: int):
    """Value (n,), gradient (3, n) and Hessian (3, 3, n) of rylm(l, m) at the Cartesian points
    qcar (3, n)."""
    x = np.asarray(qcar, dtype=np.float64)
    n = x.shape[1]
    val = np.zeros(n)
    grad = np.zeros((3, n))
    hess = np.zeros((3, 3, n))
    for coef, e in RYLM_MONOMIALS[(l, m)]:
        val += coef * _pw(x[0], e[0]) * _pw(x[1], e[1]) * _pw(x[2], e[2])
        for i in range(3):
            if e[i] == 0:
                continue
            ei = list(e)
            ci = coef * ei[i]
            ei[i] -= 1
            grad[i] += ci * _pw(x[0], ei[0]) * _pw(x[1], ei[1]) * _pw(x[2], ei[2])
            for j in range(3):
                if ei[j] == 0:
                    continue
                ej = list(ei)
                cj = ci * ej[j]
                ej[j] -= 1
                hess[i, j] += cj * _pw(x[0], ej[0]) * _pw(x[1], ej[1]) * _pw(x[2], ej[2])
    return val, grad, hess


def proj_nl_kb_der_c16(rkpt, isort, kgv, species_rat, vkb, nkb, nqnl, delqnl, adot, nder):
    """anlga (mtxd, nanl), xnlkb (nanl,), danlgadrk (mtxd, nanl, 3), d2anlgadrk2 (mtxd, nanl, 3, 3).

    species_rat: list over types of (natom, 3) lattice coordinates; vkb (ntype, 4, nq + 3) the
    table vkb(-2:nq, l, 0, type) with index 0 at q index -2; nkb (ntype, 4) = nkb(l, 0, type);
    adot the metric (bvec and vcell as adot_to_avec / adot_to_bdot, :148-150); nder = 0, 1 or 2
    (derivatives above nder are returned as zeros). Follows proj_nl_kb_der_c16.f90:190-407 line by line: q = k + G in
    lattice and Cartesian coordinates, |q|, its derivatives dq/drk = bdot q / |q| and
    d2q/drk2 = bdot/|q| - dq dq^T/|q| (zero when |q| <= 1e-8), the solid harmonics and their
    derivatives converted to lattice coordinates with bvec, the phase e^{-2 pi i G.tau}, the
    quadratic interpolation of vkb at nint(|q|/delq) with its first and second derivatives, and
    the product rule for the projector (the |q| -> 0 branch of the second derivative).
    """
    _, bvec = adot_to_avec(adot)
    vcell, bdot = adot_to_bdot(adot)
    fac = 1.0 / math.sqrt(vcell)
    g = kgv[:, np.asarray(isort) - 1].astype(np.float64)
    qk = g + np.asarray(rkpt, dtype=np.float64)[:, None]
    qcar = bvec @ qk
    qi = np.sqrt((qcar ** 2).sum(axis=0))
    mtxd = g.shape[1]
    lqi = qi > EPS
    qs = np.where(lqi, qi, 1.0)
    dqi = np.where(lqi[None, :], (bdot @ qk) / qs[None, :], 0.0)                         # (3, n)
    d2qi = np.where(lqi[None, None, :], bdot[:, :, None] / qs[None, None, :]
                    - dqi[:, None, :] * dqi[None, :, :] / qs[None, None, :], 0.0)       # (3, 3, n)
    cols, dcols, d2cols, xnl = [], [], [], []
    for t, rat in enumerate(species_rat):
        st = np.exp(-2j * PI * (np.asarray(rat) @ g))                                  # (natom, n)
        xni = qi / delqnl[t]
        ni = np.floor(xni + 0.5).astype(np.int64)                                       # nint, qi >= 0
        ni = np.maximum(ni, 0)
        ok = ni < nqnl[t] - 1
        nic = np.where(ok, ni, 0)
        xi = xni - nic
        for l in range(LMAX + 1):
            if nkb[t, l] == 0:
                continue
            tab = vkb[t, l]
            v0, vp, vm = tab[nic + 2], tab[nic + 3], tab[nic + 1]
            vq0 = np.where(ok, fac * (v0 * (1 + xi) * (1 - xi) + 0.5 * (vp * (1 + xi) - vm * (1 - xi)) * xi), 0.0)
            dv = np.where(ok, fac * (-2 * xi * v0 + 0.5 * (vp * (1 + 2 * xi) - vm * (1 - 2 * xi))) / delqnl[t], 0.0)
            d2v = np.where(ok, fac * (-2 * v0 + vp + vm) / (delqnl[t] * delqnl[t]), 0.0)
            il = 1j ** l
            vqil, dvqil, d2vqil = vq0 * il, dv * il, d2v * il
            for m in range(-l, l + 1):
                ry, dryc, d2ryc = rylm_derivatives(qcar, l, m)
                dry = np.einsum("kn,kp->pn", dryc, bvec)                              # drylmdrk(n)
                d2ry = np.einsum("ij,ikp,kn->jnp", bvec, d2ryc, bvec)                   # d2rylmdrk2(j, n)
                for a in range(np.asarray(rat).shape[0]):
                    s = st[a]
                    cols.append(s * ry * vqil)
                    xnl.append(float(nkb[t, l]))
                    if nder > 0:
                        dcols.append(s[None, :] * (dry * vqil[None, :] + ry[None, :] * dvqil[None, :] * dqi))
                    if nder > 1:
                        gen = (d2ry * vqil + dry[None, :, :] * dvqil * dqi[:, None, :]
                               + dry[:, None, :] * dvqil * dqi[None, :, :]
                               + ry * d2vqil * dqi[None, :, :] * dqi[:, None, :] + ry * dvqil * d2qi)
                        small = d2ry * vqil + ry * d2vqil * bdot[:, :, None]
                        d2cols.append(s[None, None, :] * np.where(lqi[None, None, :], gen, small))
    nanl = len(cols)
    anlga = np.stack(cols, axis=1) if nanl else np.zeros((mtxd, 0), np.complex128)
    dan = np.zeros((mtxd, nanl, 3), np.complex128)
    d2an = np.zeros((mtxd, nanl, 3, 3), np.complex128)
    if nder > 0 and nanl:
        dan = np.stack(dcols, axis=1).transpose(2, 1, 0)                               # (n, nanl, 3)
    if nder > 1 and nanl:
        d2an = np.stack(d2cols, axis=0).transpose(3, 0, 1, 2)                          # (n, nanl, 3(j), 3(n))
    return anlga, np.array(xnl), dan, d2an
