"""H|psi> restated from the reference (CPU, FP64) -- test infrastructure only.

hk_psi_c16     -- Src/hk_psi/reference/hk_psi_c16.f90:28-241
hk_psi_nl_c16  -- Src/cpw_lib/hk_psi_nl_c16.f90:23-104
hk_psi_spin_c16 -- Src/hk_psi/reference/hk_psi_spin_c16.f90:1-316 (two-component spinors)
dense_h        -- explicit matrix of the same operator (ground truth)
"""
from __future__ import annotations

import numpy as np

from .fft import cfft_wf_c16


def ipoint_of(mtxd, isort, kgv, kmscr):
    """Box offsets of the basis (hk_psi_c16.f90:145-158) and the sphere extent.

    ipoint(i) = (k3*n2 + k2)*id + k1 (0-based here), negative components
    wrapped by n_j. Raises like the reference's stop (:161-172) when the
    basis would wrap around the box.
    """
    n1, n2, n3, ident = (int(v) for v in kmscr[3:7])
    g = kgv[:, np.asarray(isort[:mtxd]) - 1].astype(np.int64)
    kd1, kd2, kd3 = (int(np.abs(g[j]).max()) if mtxd > 0 else 0 for j in range(3))
    if kd1 > (n1 - 1) // 2 or kd2 > (n2 - 1) // 2 or kd3 > (n3 - 1) // 2:
        raise ValueError("hk_psi_c16: dimension of k index exceeds the box (wraparound)")
    k1 = np.where(g[0] < 0, g[0] + n1, g[0])
    k2 = np.where(g[1] < 0, g[1] + n2, g[1])
    k3 = np.where(g[2] < 0, g[2] + n3, g[2])
    return (k3 * n2 + k2) * ident + k1, (kd1, kd2, kd3)


def hk_psi_nl_c16(psi, hpsi, anlga, xnlkb, ladd=True):
    """Separable KB non-local part, hk_psi_nl_c16.f90:82-97.

    dhd = anlga^H psi (:82); dhd(i,:) *= xnlkb(i) (:87-91);
    hpsi = [hpsi if ladd else 0] + anlga dhd (:95).
    With no projectors (nanl = 0) the reference skips both products, the one
    that would zero hpsi included (the `if(nanl > 0)` of :78-98): hpsi is
    returned untouched whatever ladd is.
    """
    if anlga.shape[1] == 0:
        return hpsi
    dhd = anlga.conj().T @ psi
    dhd *= np.asarray(xnlkb)[:, None]
    if ladd:
        hpsi += anlga @ dhd
    else:
        hpsi[...] = anlga @ dhd
    return hpsi


def hk_psi_c16(mtxd, neig, psi, ekpg, isort, vscr, kmscr, kgv, anlga, xnlkb):
    """hpsi = (T + V_loc + V_NL) psi for neig bands, hk_psi_c16.f90:176-231.

    psi: (>= mtxd, >= neig) complex128. Returns hpsi (mtxd, neig).
    Per band: zero box, scatter psi into ipoint, backward pruned FFT, multiply
    by vscr, forward pruned FFT (scaled 1/N), gather, add ekpg*psi; then the
    non-local ZGEMMs for all bands at once.
    """
    n1, n2, n3, ident = (int(v) for v in kmscr[3:7])
    ntot = ident * n2 * n3
    ip, (kd1, kd2, kd3) = ipoint_of(mtxd, isort, kgv, kmscr)
    v = np.asarray(vscr[:ntot], dtype=np.float64)
    ek = np.asarray(ekpg[:mtxd], dtype=np.float64)
    hpsi = np.zeros((mtxd, neig), dtype=np.complex128)
    chd = np.zeros(ntot, dtype=np.complex128)
    for n in range(neig):
        chd[:] = 0
        chd[ip] = psi[:mtxd, n]
        cfft_wf_c16(chd, ident, n1, n2, n3, kd1, kd2, kd3, -1)
        chd *= v
        cfft_wf_c16(chd, ident, n1, n2, n3, kd1, kd2, kd3, 1)
        hpsi[:, n] = chd[ip] + ek * psi[:mtxd, n]
    hk_psi_nl_c16(psi[:mtxd, :neig], hpsi, anlga[:mtxd], xnlkb, ladd=True)
    return hpsi


def hk_psi_spin_c16(mtxd, neig, psi_sp, ekpg, isort, vscr_sp, kmscr, kgv, nsp, anlsp, xnlkbsp):
    """H|psi> of spinors, Src/hk_psi/reference/hk_psi_spin_c16.f90.

    psi_sp: (>= 2 mtxd, >= neig) complex128 with the up component of plane wave i at row 2i
    and the down component at 2i+1 (0-based). vscr_sp: (>= id n2 n3, nsp) real, the columns
    (1, sigma_z, sigma_x, sigma_y). Per spinor: both components to the box, backward pruned
    FFT, the local potential (nsp 1: V on both; 2: V1+V2 on up, V1-V2 on down; 4: the 2x2
    matrix [[V1+V2, V3-iV4], [V3+iV4, V1-V2]]), forward pruned FFT, gather, kinetic ekpg on
    both components; then the KB term with 2 mtxd rows and the spinor projectors anlsp.
    """
    if nsp not in (1, 2, 4):
        raise ValueError("hk_psi_spin_c16: nsp should be 1, 2 or 4")
    n1, n2, n3, ident = (int(v) for v in kmscr[3:7])
    ntot = ident * n2 * n3
    ip, (kd1, kd2, kd3) = ipoint_of(mtxd, isort, kgv, kmscr)
    v = np.asarray(vscr_sp, dtype=np.float64)[:ntot]
    ek = np.asarray(ekpg[:mtxd], dtype=np.float64)
    hpsi = np.zeros((2 * mtxd, neig), dtype=np.complex128)
    for n in range(neig):
        cp = np.zeros(ntot, dtype=np.complex128)
        cm = np.zeros(ntot, dtype=np.complex128)
        cp[ip] = psi_sp[0:2 * mtxd:2, n]
        cm[ip] = psi_sp[1:2 * mtxd:2, n]
        cfft_wf_c16(cp, ident, n1, n2, n3, kd1, kd2, kd3, -1)
        cfft_wf_c16(cm, ident, n1, n2, n3, kd1, kd2, kd3, -1)
        if nsp == 1:
            cp, cm = v[:, 0] * cp, v[:, 0] * cm
        elif nsp == 2:
            cp, cm = (v[:, 0] + v[:, 1]) * cp, (v[:, 0] - v[:, 1]) * cm
        else:
            tp = (v[:, 0] + v[:, 1]) * cp + (v[:, 2] - 1j * v[:, 3]) * cm
            tm = (v[:, 0] - v[:, 1]) * cm + (v[:, 2] + 1j * v[:, 3]) * cp
            cp, cm = tp, tm
        cfft_wf_c16(cp, ident, n1, n2, n3, kd1, kd2, kd3, 1)
        cfft_wf_c16(cm, ident, n1, n2, n3, kd1, kd2, kd3, 1)
        hpsi[0::2, n] = cp[ip] + ek * psi_sp[0:2 * mtxd:2, n]
        hpsi[1::2, n] = cm[ip] + ek * psi_sp[1:2 * mtxd:2, n]
    hk_psi_nl_c16(psi_sp[:2 * mtxd, :neig], hpsi, anlsp[:2 * mtxd], xnlkbsp, ladd=True)
    return hpsi


def hk_psi_loc(mtxd, neig, psi, isort, vscr, kmscr, kgv):
    """Local-potential part alone (Src/omp/hk_psi_loc_c16.f90, nsp = 1)."""
    zero_x = np.zeros((mtxd, 0), dtype=np.complex128)
    return hk_psi_c16(mtxd, neig, psi, np.zeros(mtxd), isort, vscr, kmscr, kgv, zero_x, np.zeros(0))


def dense_h(mtxd, ekpg, isort, vscr, kmscr, kgv, anlga, xnlkb):
    """The Hermitian matrix of the operator hk_psi_c16 applies, built entry by entry.

    H_ij = ekpg_i d_ij + Vt(G_i - G_j) + sum_a anlga_ia xnlkb_a conj(anlga_ja),
    with Vt(m) = (1/N) sum_r vscr(r) e^{-2 pi i m.r/n} on the box. Used as the
    dense ground truth for the eigensolver (zheevd on it).
    """
    n1, n2, n3, ident = (int(v) for v in kmscr[3:7])
    vb = np.asarray(vscr[: ident * n2 * n3]).reshape(n3, n2, ident)[:, :, :n1].transpose(2, 1, 0)
    vt = np.fft.fftn(vb) / (n1 * n2 * n3)
    g = kgv[:, np.asarray(isort[:mtxd]) - 1].astype(np.int64)
    h = vt[(g[0][:, None] - g[0][None, :]) % n1,
           (g[1][:, None] - g[1][None, :]) % n2,
           (g[2][:, None] - g[2][None, :]) % n3]
    h = h + np.diag(np.asarray(ekpg[:mtxd], dtype=np.float64))
    if anlga.shape[1]:
        x = anlga[:mtxd]
        h = h + (x * np.asarray(xnlkb)[None, :]) @ x.conj().T
    return h
