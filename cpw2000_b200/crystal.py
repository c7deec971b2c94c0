"""Host-side crystal and plane-wave basis set-up (the caller's side of H|psi>).

Everything here is cheap integer / FP64 book-keeping that the cpw2000 driver
does on the host before it calls ``hk_psi_c16`` or ``ditsp_c16``:

* lattice metric conversions   -- Src/crystal/adot_to_avec.f90, adot_to_bdot.f90
* G-space generation (stars)   -- Src/cpw/cpw_gspace.f90 (kgv ordered by length)
* FFT box sizes                -- Src/ALFA/size_fft.f90
* basis selection, ekpg, qmod  -- Src/ALFA/hamilt_struct.f90:87-153
* small-matrix size            -- Src/ALFA/size_mtxds.f90:62-96
* Monkhorst-Pack k-points reduced by the lattice point group

Arrays follow the reference's Fortran conventions where they cross the
boundary: ``kgv`` is (3, ng) integer, ``isort`` is 1-based into kgv columns,
vectors are columns of ``avec`` / ``bvec``.
"""
from __future__ import annotations

import itertools
import math

import numpy as np

PI = math.pi


def adot_to_avec(adot: np.ndarray):
    """Canonical (upper-triangular) lattice vectors and reciprocal vectors.

    Follows Src/crystal/adot_to_avec.f90: avec(:,j) is lattice vector j in a
    canonical orientation built by Cholesky factorisation of the metric, and
    bvec satisfies bvec^T avec = 2 pi I.
    """
    adot = np.asarray(adot, dtype=np.float64)
    avec = np.zeros((3, 3))
    a11 = adot[0, 0]
    if a11 < 1e-10:
        raise ValueError("adot_to_avec: avec(1,1) not positive")
    avec[0, 0] = math.sqrt(a11)
    avec[0, 1] = adot[0, 1] / avec[0, 0]
    a22 = adot[1, 1] - avec[0, 1] ** 2
    if a22 < 1e-10:
        raise ValueError("adot_to_avec: avec(2,2) not positive")
    avec[1, 1] = math.sqrt(a22)
    avec[0, 2] = adot[0, 2] / avec[0, 0]
    avec[1, 2] = (adot[1, 2] - avec[0, 1] * avec[0, 2]) / avec[1, 1]
    a33 = adot[2, 2] - avec[1, 2] ** 2 - avec[0, 2] ** 2
    if a33 < 1e-10:
        raise ValueError("adot_to_avec: avec(3,3) not positive")
    avec[2, 2] = math.sqrt(a33)
    bvec = 2 * PI * np.linalg.inv(avec).T
    return avec, bvec


def adot_to_bdot(adot: np.ndarray):
    """Cell volume and reciprocal metric bdot = (2 pi)^2 adot^-1.

    Src/crystal/adot_to_bdot.f90 (cofactor form; same quantity).
    """
    adot = np.asarray(adot, dtype=np.float64)
    det = float(np.linalg.det(adot))
    if det < 1e-10:
        raise ValueError("adot_to_bdot: cell volume squared not positive")
    bdot = (2 * PI) ** 2 * np.linalg.inv(adot)
    return math.sqrt(det), bdot


def size_fft(kmscr3) -> tuple[int, int, int]:
    """FFT sizes from the maximum G indices, Src/ALFA/size_fft.f90.

    For 2k+1 < 32 the size is the first of {2,4,6,8,10,12,16,18,20,24,32}
    that is >= 2k+1, otherwise the first of 2^(p-5)*{36,40,48,50,54,64} with
    p = int(log2(2k+1)).
    """
    prim = (2, 4, 6, 8, 10, 12, 16, 18, 20, 24, 32)
    sec = (36, 40, 48, 50, 54, 64)
    out = []
    for k in kmscr3:
        need = 2 * int(k) + 1
        if need < 32:
            n = prim[-1]
            for c in prim:
                n = c
                if need <= c:
                    break
        else:
            p = int(math.log(float(need)) / math.log(2.0))
            n = 0
            for c in sec:
                n = (2 ** (p - 5)) * c
                if need <= n:
                    break
        out.append(n)
    return tuple(out)


def gspace(adot: np.ndarray, gmax: float):
    """All G = m1 b1 + m2 b2 + m3 b3 with |G| <= gmax, sorted by length.

    Returns kgv (3, ng) int32, the analogue of the star-ordered kgv array
    (Src/cpw/cpw_gspace.f90). Ties in length are ordered by a stable sort of
    the generating index, which is deterministic.
    """
    _, bdot = adot_to_bdot(adot)
    # bound on |m_i|: |m_i| <= gmax * |a_i| / (2 pi)
    alen = np.sqrt(np.diag(adot))
    kmax = [int(math.floor(gmax * alen[i] / (2 * PI))) + 1 for i in range(3)]
    r = [np.arange(-k, k + 1) for k in kmax]
    m = np.stack(np.meshgrid(*r, indexing="ij"), axis=0).reshape(3, -1)
    g2 = np.einsum("in,ij,jn->n", m.astype(np.float64), bdot, m.astype(np.float64))
    keep = g2 <= gmax * gmax * (1 + 1e-12)
    m = m[:, keep]
    g2 = g2[keep]
    order = np.argsort(np.round(g2, 10), kind="stable")
    return np.ascontiguousarray(m[:, order].astype(np.int32))


def hamilt_struct(emax: float, rkpt, kgv: np.ndarray, adot: np.ndarray):
    """Basis selection for one k-point, Src/ALFA/hamilt_struct.f90:87-153.

    ekin(i) = 1/2 (k+G_i)^T bdot (k+G_i); the basis is the set of G with
    ekin <= emax, sorted by ekin (at k = 0 the star order of kgv is kept).
    Returns (mtxd, isort[1-based], qmod, ekpg).
    """
    _, bdot = adot_to_bdot(adot)
    rkpt = np.asarray(rkpt, dtype=np.float64)
    qk = kgv.astype(np.float64) + rkpt[:, None]
    ekin = 0.5 * np.einsum("in,ij,jn->n", qk, bdot, qk)
    xsum = float(rkpt @ bdot @ rkpt)
    if xsum < 0.1e-20:
        irow = np.arange(ekin.size)
    else:
        irow = np.argsort(ekin, kind="stable")
    sel = ekin[irow] <= emax
    mtxd = int(np.argmin(sel)) if not sel.all() else ekin.size
    if mtxd == ekin.size:
        raise ValueError("hamilt_struct: size of g-space equals the hamiltonian size")
    isort = irow[:mtxd].astype(np.int32) + 1
    ekpg = ekin[irow[:mtxd]].copy()
    qmod = np.sqrt(2 * ekpg)
    return mtxd, isort, qmod, ekpg


def size_mtxds(hdiag: np.ndarray, neig: int) -> int:
    """Small-matrix dimension, Src/ALFA/size_mtxds.f90:62-96."""
    mtxd = hdiag.size
    if mtxd < neig:
        raise ValueError("size_mtxds: matrix smaller than the number of states")
    if mtxd < 250 or 3 * neig + 20 >= mtxd:
        return mtxd
    href = abs(2 * hdiag[neig - 1] - hdiag[0]) + 1e-6
    for i in range(3 * neig + 20, mtxd):
        # Fortran i (1-based) -> hdiag(i) = hdiag[i-1], hdiag(i+1) = hdiag[i]
        if hdiag[i - 1] > href and (hdiag[i] - hdiag[i - 1]) > 1e-6:
            return i
    return mtxd


def kd_of_basis(kgv: np.ndarray, isort: np.ndarray):
    """Largest |k_j| over the basis (kd1, kd2, kd3), as hk_psi_c16.f90:145-158."""
    g = kgv[:, isort - 1]
    return tuple(int(np.abs(g[j]).max()) for j in range(3))


def point_group(adot: np.ndarray):
    """Integer 3x3 matrices S (lattice coordinates) with S^T adot S = adot."""
    adot = np.asarray(adot, dtype=np.float64)
    ops = []
    scale = np.abs(adot).max()
    for entries in itertools.product((-1, 0, 1), repeat=9):
        s = np.array(entries, dtype=np.int64).reshape(3, 3)
        if abs(round(np.linalg.det(s))) != 1:
            continue
        if np.allclose(s.T @ adot @ s, adot, atol=1e-8 * scale):
            ops.append(s)
    return ops


def monkhorst_pack(adot: np.ndarray, nk=(4, 4, 4), shift=(0.5, 0.5, 0.5)):
    """Shifted MP grid reduced by the lattice point group plus time reversal.

    Returns (rk (nk,3) lattice coordinates of reciprocal vectors, weights).
    k-points are expressed in the reciprocal basis; a real-space point
    operation S acts on them through S^-T.
    """
    ops = point_group(adot)
    rot = [np.linalg.inv(s).T for s in ops]
    pts = []
    for i, j, k in itertools.product(range(nk[0]), range(nk[1]), range(nk[2])):
        pts.append(((i + shift[0]) / nk[0], (j + shift[1]) / nk[1], (k + shift[2]) / nk[2]))
    pts = np.array(pts)
    pts = pts - np.round(pts)          # fold into (-1/2, 1/2]

    def key(v):
        w = v - np.floor(v + 1e-9)      # canonical representative in [0,1)
        return tuple(np.round(w * 1e6).astype(np.int64))

    seen = {}
    reps = []
    weights = []
    for p in pts:
        kk = key(p)
        if kk in seen:
            weights[seen[kk]] += 1
            continue
        idx = len(reps)
        reps.append(p)
        weights.append(1)
        for r in rot:
            for sgn in (1.0, -1.0):
                seen.setdefault(key(sgn * (r @ p)), idx)
    w = np.array(weights, dtype=np.float64)
    return np.array(reps), w / w.sum()
