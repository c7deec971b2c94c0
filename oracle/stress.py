"""Stress restated from the reference -- test infrastructure only.

Covariant lattice stress tensors (Hartree) of E = sum_n f_n <psi_n|H|psi_n> at fixed
wavefunctions, term by term as the reference computes them:

strkin  -- Src/ALFA/for_str_kinetic_stress.f90:95-120:
           strkin(k,j) = 2 pi^2 sum_G 2 sum_n f_n |psi(G,n)|^2 q_k q_j   (q = k+G, lattice coords)
strnlkb -- Src/ALFA/for_str_nl_kb.f90:196-376, stress part: per atom the strain variants
           anl(4+kl) = st (dflm(kl) vq + flm dvq dqi(kl)) of the projector, dhd = anl psi,
           strnlkb += enl adot - 8 pi^2 f xnlkb Re(dhd(4+kl) conj(dhd(1)))
strhl   -- Src/ALFA/for_str_local_stress.f90:73-112 with the local pseudopotential as the only
           potential (no Hartree, exchange-correlation or core terms in this energy):
           strhl = 8 pi^2 sum_G Re(dvql conj(den)) G G^T + (sum_G Re(vion conj(den))) adot,
           vion(G) = V(G) the box coefficients of the local potential, dvql = dV/d|G|^2,
           den(G) = (1/N) sum_r rho(r) e^{-iG.r}; the G = 0 term (the reference's ealpha) is
           part of the sum.

energy_at_metric gives E for a strained metric at fixed isort, kgv, atomic lattice
coordinates and coefficients, for central finite differences.
"""
from __future__ import annotations

import math

import numpy as np

from cpw2000_b200.crystal import adot_to_avec, adot_to_bdot
from cpw2000_b200.pseudo import _interp, local_potential_box, proj_nl_kb, rylm

from .forces import charge_by_fft
from .hk_psi import hk_psi_c16

PI = math.pi
PAIRS = [(0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (2, 0)]


def strkin(rkpt, mtxd, isort, kgv, psi, occ):
    g = kgv[:, np.asarray(isort[:mtxd]) - 1].astype(np.float64) + np.asarray(rkpt, dtype=np.float64)[:, None]
    z = 2 * np.sum(np.asarray(occ)[None, :] * np.abs(psi[:mtxd, : len(occ)]) ** 2, axis=1)
    return 2 * PI * PI * np.einsum("g,kg,jg->kj", z, g, g)


def _vint_dv(vtab, qi, delq, nq):
    xni = qi / delq
    ni = max(int(np.rint(xni)), 0)
    if ni >= nq - 1:
        return 0.0, 0.0
    xi = xni - ni
    v0, vp, vm = vtab[ni + 2], vtab[ni + 3], vtab[ni + 1]
    vint = v0 * (1 + xi) * (1 - xi) + 0.5 * (vp * (1 + xi) - vm * (1 - xi)) * xi
    dv = -2 * xi * v0 + (xi + 0.5) * vp + (xi - 0.5) * vm
    return vint, dv


def strnlkb(rkpt, mtxd, isort, kgv, psi, occ, species, vkb, nkb, adot, delq=0.01, nq=4000):
    avec, bvec = adot_to_avec(adot)
    vcell, bdot = adot_to_bdot(adot)
    vfac = 1.0 / math.sqrt(vcell)
    lmx = max((l for t in range(len(species)) for l in range(4) if nkb[t, l] != 0), default=0)
    R1 = rylm(np.eye(3), 1)[1]                       # d rylm_1m / d rc (constant)
    nb = len(occ)
    out = np.zeros((3, 3))
    for t, sp in enumerate(species):
        for a in range(sp.natom):
            rows = []                                # per projector: 7 rows (anl 1 and 5..10), plus xnl
            xnl = []
            anl = None
            for l in range(lmx + 1):
                if nkb[t, l] == 0:
                    continue
                for m in range(-l, l + 1):
                    xnl.append(float(nkb[t, l]))
            anl = np.zeros((len(xnl), 7, mtxd), dtype=np.complex128)
            for i in range(mtxd):
                qk = np.asarray(rkpt, dtype=np.float64) + kgv[:, isort[i] - 1]
                q2 = float(qk @ bdot @ qk)
                if q2 > 1e-20:
                    qi = math.sqrt(q2)
                    qinv = 1.0 / qi
                    dqi = np.array([-qk[p] * qk[r] * qinv for p, r in PAIRS])
                    qcar = (bvec @ qk) * qinv
                    dqcar = np.zeros((6, 3))
                    for kl, (p, r) in enumerate(PAIRS):
                        for c in range(3):
                            dqcar[kl, c] = (-avec[c, p] * qk[r] / (2 * PI) - dqi[kl] * qcar[c]) * qinv
                    ry = rylm(qcar[:, None], lmx)[:, :, 0]
                else:
                    qi = 0.0
                    dqi = np.zeros(6)
                    dqcar = np.zeros((6, 3))
                    ry = np.zeros((lmx + 1, 2 * lmx + 1))
                    ry[0, lmx] = 1.0
                st = np.exp(2j * PI * (kgv[:, isort[i] - 1] @ sp.rat[a]))
                ind = 0
                for l in range(lmx + 1):
                    if nkb[t, l] == 0:
                        continue
                    vint, dvdxi = _vint_dv(vkb[t, l], qi, delq, nq)
                    vq = vfac * vint * qi ** l
                    dvq = vfac * dvdxi * qi ** l / delq + (vfac * vint * l * qi ** (l - 1) if l > 0 else 0.0)
                    for m in range(-l, l + 1):
                        flm = ry[l, m + lmx]
                        anl[ind, 0, i] = st * flm * vq
                        for kl in range(6):
                            dflm = (R1[m + 1] @ dqcar[kl]) if l == 1 else 0.0
                            anl[ind, 1 + kl, i] = st * (dflm * vq + flm * dvq * dqi[kl])
                        ind += 1
            dhd = anl @ psi[:mtxd, :nb]                 # (nproj, 7, nb)
            for ip in range(len(xnl)):
                for n in range(nb):
                    enl = occ[n] * xnl[ip] * abs(dhd[ip, 0, n]) ** 2
                    fac = 8 * PI * PI * occ[n] * xnl[ip]
                    for kl, (p, r) in enumerate(PAIRS):
                        out[p, r] += enl * adot[p, r] - fac * float(np.real(dhd[ip, 1 + kl, n] * np.conj(dhd[ip, 0, n])))
    out[1, 0] = out[0, 1]
    out[2, 1] = out[1, 2]
    out[0, 2] = out[2, 0]
    return out


def strhl(rho, species, adot, box):
    """Local-pseudopotential stress from the mesh density rho (n3, n2, n1)."""
    n1, n2, n3 = box
    vcell, bdot = adot_to_bdot(adot)
    den = np.fft.fftn(rho) / (n1 * n2 * n3)            # axes (z, y, x)
    mz = np.fft.fftfreq(n3, 1.0 / n3)[:, None, None]
    my = np.fft.fftfreq(n2, 1.0 / n2)[None, :, None]
    mx = np.fft.fftfreq(n1, 1.0 / n1)[None, None, :]
    ms = [mx + 0 * my + 0 * mz, 0 * mx + my + 0 * mz, 0 * mx + 0 * my + mz]
    g2 = sum(bdot[i, j] * ms[i] * ms[j] for i in range(3) for j in range(3))
    vion = np.zeros((n3, n2, n1), dtype=np.complex128)
    dvql = np.zeros_like(vion)
    for sp in species:
        ff = -sp.v0 * (2 * PI * sp.sigma ** 2) ** 1.5 * np.exp(-0.5 * g2 * sp.sigma ** 2) / vcell
        sf = np.zeros_like(vion)
        for tau in sp.rat:
            sf += np.exp(-2j * PI * (mx * tau[0] + my * tau[1] + mz * tau[2]))
        vion += ff * sf
        dvql += (-0.5 * sp.sigma ** 2) * ff * sf
    for ax, n in ((2, n1), (1, n2), (0, n3)):
        if n % 2 == 0:
            sl = [slice(None)] * 3
            sl[ax] = n // 2
            vion[tuple(sl)] = 0
            dvql[tuple(sl)] = 0
    dvld = np.real(dvql * np.conj(den))
    out = np.zeros((3, 3))
    for i in range(3):
        for j in range(3):
            out[i, j] = 8 * PI * PI * float(np.sum(dvld * ms[i] * ms[j]))
    ssum = float(np.sum(np.real(vion * np.conj(den))))
    return out + ssum * np.asarray(adot)


def energy_at_metric(adot, d, species, box, idpad, psi, occ, delq=0.01, nq=4000):
    """E = sum_n f_n <psi_n|H(adot)|psi_n> with the basis (isort, kgv), the coefficients and the
    atoms' lattice coordinates of d held fixed."""
    mtxd = d["mtxd"]
    vcell, bdot = adot_to_bdot(adot)
    g = d["kgv"][:, np.asarray(d["isort"][:mtxd]) - 1].astype(np.float64) + np.asarray(d["rkpt"])[:, None]
    ekpg = 0.5 * np.einsum("in,ij,jn->n", g, bdot, g)
    vscr, _ = local_potential_box(species, adot, box, idpad)
    anlga, xnlkb = proj_nl_kb(d["rkpt"], d["isort"], d["kgv"], species, d["vkb"], d["nkb"], adot, delq, nq)
    nb = len(occ)
    hp = hk_psi_c16(mtxd, nb, psi, ekpg, d["isort"], vscr, d["kmscr"], d["kgv"], anlga, xnlkb)
    return float(np.sum(np.asarray(occ) * np.real(np.sum(psi[:mtxd, :nb].conj() * hp, axis=0))))


def fd_covariant_stress(d, species, adot, box, idpad, psi, occ, h=1e-4):
    """Central differences of E in the metric: -2 adot (dE/dadot) adot."""
    adot = np.asarray(adot, dtype=np.float64)
    G = np.zeros((3, 3))
    scale = np.sqrt(np.diag(adot).mean())
    for i in range(3):
        for j in range(i, 3):
            dA = np.zeros((3, 3))
            dA[i, j] += 1.0
            dA[j, i] += 1.0 if i != j else 0.0
            step = h * scale * scale
            ep = energy_at_metric(adot + step * dA, d, species, box, idpad, psi, occ)
            em = energy_at_metric(adot - step * dA, d, species, box, idpad, psi, occ)
            der = (ep - em) / (2 * step)          # = G_ii (i == j) or G_ij + G_ji = 2 G_ij
            G[i, j] = G[j, i] = der if i == j else der / 2
    return -2 * adot @ G @ adot


def rho_of(d, psi, occ):
    return charge_by_fft(d["mtxd"], len(occ), psi, occ, d["isort"], d["kgv"], d["kmscr"])
