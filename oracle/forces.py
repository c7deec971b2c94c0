"""Density and Hellmann-Feynman forces restated from the reference -- test infrastructure only.

charge_by_fft      -- Src/omp/charge_by_fft.f90:185-199 (mesh density, before the
                      transform to stars): rho(r) = sum_n occ_n |psi_n(r)|^2 with
                      psi_n(r) the unscaled backward pruned transform.
for_str_nl_kb      -- Src/ALFA/for_str_nl_kb.f90:169-398, force part: per atom the
                      projector variants anl(1) = st flm vq, anl(2..4) = -i st flm vq kgv_j
                      with st = e^{+2 pi i G.tau}; dhd = anl psi (zgemm 'n','n');
                      F_j = 2 pi sum_n 2 occ xnlkb Re(dhd(1+j) conj(dhd(1))).
local_force        -- the structure-factor force of Src/ALFA/for_str_local_force.f90:102-145,
                      F_aj = 2 pi sum_G Re[ i m_j e^{-2 pi i m.tau_a} v_t(G) conj(rho~(G)) ],
                      rho~ = (1/N) sum_r rho(r) e^{-iG.r}, over the G of the FFT box.
Forces are in lattice (covariant) components: F_j = -dE/dtau_j, tau in lattice
coordinates. hf_energy is E = sum_n occ_n <psi_n|H|psi_n> for fixed psi.
"""
from __future__ import annotations

import math

import numpy as np

from cpw2000_b200.crystal import adot_to_avec, adot_to_bdot
from cpw2000_b200.pseudo import rylm

from .fft import cfft_wf_c16
from .hk_psi import hk_psi_c16, ipoint_of

PI = math.pi


def charge_by_fft(mtxd, neig, psi, occ, isort, kgv, kmscr):
    """Mesh density, shape (n3, n2, n1)."""
    n1, n2, n3, ident = (int(v) for v in kmscr[3:7])
    ip, kd = ipoint_of(mtxd, isort, kgv, kmscr)
    ntot = ident * n2 * n3
    rho = np.zeros(ntot)
    chd = np.zeros(ntot, dtype=np.complex128)
    for j in range(neig):
        chd[:] = 0
        chd[ip] = psi[:mtxd, j]
        cfft_wf_c16(chd, ident, n1, n2, n3, *kd, -1)
        rho += occ[j] * (chd * chd.conj()).real
    return rho.reshape(n3, n2, ident)[:, :, :n1].copy()


def _interp_and_derivative(vtab, xq, nq):
    ni = np.maximum(np.rint(xq).astype(np.int64), 0)
    ok = ni < nq - 1
    nic = np.where(ok, ni, 0)
    xi = xq - nic
    v0, vp, vm = vtab[nic + 2], vtab[nic + 3], vtab[nic + 1]
    vint = v0 * (1 + xi) * (1 - xi) + 0.5 * (vp * (1 + xi) - vm * (1 - xi)) * xi
    dv = -2 * xi * v0 + (xi + 0.5) * vp + (xi - 0.5) * vm
    return np.where(ok, vint, 0.0), np.where(ok, dv, 0.0)


def for_str_nl_kb_forces(rkpt, mtxd, isort, kgv, psi, occ, species, vkb, nkb, adot, delq=0.01, nq=4000):
    """KB forces (natom_total, 3) in lattice components."""
    _, bvec = adot_to_avec(adot)
    vcell, bdot = adot_to_bdot(adot)
    vfac = 1.0 / math.sqrt(vcell)
    g = kgv[:, np.asarray(isort[:mtxd]) - 1].astype(np.float64)
    qk = g + np.asarray(rkpt, dtype=np.float64)[:, None]
    qi = np.sqrt(np.einsum("in,ij,jn->n", qk, bdot, qk))
    qcar = bvec @ qk
    lmx = max((l for t in range(len(species)) for l in range(4) if nkb[t, l] != 0), default=0)
    ry = rylm(qcar, lmx)                 # r^l sqrt(4pi/(2l+1)) Y_lm of k+G: flm * qi^l of the reference
    forces = []
    for t, sp in enumerate(species):
        for a in range(sp.natom):
            st = np.exp(2j * PI * (sp.rat[a] @ g))
            rows1, rows2 = [], []
            xnl = []
            for l in range(lmx + 1):
                if nkb[t, l] == 0:
                    continue
                vint, _ = _interp_and_derivative(vkb[t, l], qi / delq, nq)
                vq = vfac * vint
                for m in range(-l, l + 1):
                    base = st * ry[l, m + lmx] * vq
                    rows1.append(base)
                    rows2.append([-1j * base * g[j] for j in range(3)])
                    xnl.append(float(nkb[t, l]))
            if not rows1:
                forces.append(np.zeros(3))
                continue
            a1 = np.array(rows1)                        # (nproj, mtxd)
            d1 = a1 @ psi[:mtxd]                        # (nproj, neig)
            f = np.zeros(3)
            for j in range(3):
                dj = np.array([r[j] for r in rows2]) @ psi[:mtxd]
                f[j] = 2 * PI * np.sum(2 * np.asarray(occ)[None, :] * np.asarray(xnl)[:, None] *
                                       np.real(dj * np.conj(d1)))
            forces.append(f)
    return np.array(forces)


def local_force(rho, species, vgt, kmscr):
    """Local structure-factor forces (natom_total, 3), lattice components.

    rho: (n3, n2, n1) mesh density; vgt: (ntype, n3, n2, n1) form factors v_t(G)
    in FFT order.
    """
    n1, n2, n3 = (int(v) for v in kmscr[3:6])
    rt = np.fft.fftn(rho) / (n1 * n2 * n3)          # axes (z, y, x)
    mz = np.fft.fftfreq(n3, 1.0 / n3)[:, None, None]
    my = np.fft.fftfreq(n2, 1.0 / n2)[None, :, None]
    mx = np.fft.fftfreq(n1, 1.0 / n1)[None, None, :]
    out = []
    for t, sp in enumerate(species):
        for a in range(sp.natom):
            tau = sp.rat[a]
            ph = np.exp(-2j * PI * (mx * tau[0] + my * tau[1] + mz * tau[2]))
            w = ph * vgt[t] * np.conj(rt)
            out.append([2 * PI * np.sum(np.real(1j * m * w)) for m in (mx, my, mz)])
    return np.array(out)


def hf_energy(mtxd, psi, occ, ekpg, isort, vscr, kmscr, kgv, anlga, xnlkb):
    """E = sum_n occ_n <psi_n|H|psi_n> for fixed psi (FP64, oracle H|psi>)."""
    nb = len(occ)
    hp = hk_psi_c16(mtxd, nb, psi, ekpg, isort, vscr, kmscr, kgv, anlga, xnlkb)
    return float(np.sum(np.asarray(occ) * np.real(np.sum(psi[:mtxd, :nb].conj() * hp, axis=0))))
