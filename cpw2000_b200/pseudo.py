"""Synthetic pseudopotential inputs and the host-side Hamiltonian set-up.

The workloads use analytic Gaussian pseudopotentials in place of the
``*_POTKB_F.DAT`` tables, in exactly the array formats the reference consumes:

* ``vscr``  -- screened local potential on the FFT mesh, real, laid out as
  the reference's ``chd(id, n2, n3)`` box (Src/cpw_lib/pot_local.f90:104-186:
  V(G) placed on the box and transformed with e^{+iG.r}, no scaling).
* ``vkb(-2:nq, l)``, ``nkb(l)`` -- (1/q^l) times the Kleinman-Bylander
  projector on a uniform q grid with step ``delq``, sign of E_KB in ``nkb``
  (Src/omp/proj_nl_kb_c16.f90:226-240 interpolates it).
* ``anlga``, ``xnlkb`` -- projectors for one k-point, Src/omp/proj_nl_kb_c16.f90.
* ``hdiag`` -- Hamiltonian diagonal, Src/ALFA/hamilt_diag_kb.f90:89-127.
* ``hamsm`` -- the dense leading mtxds x mtxds block of H (what
  Src/ALFA/hamilt_kb.f90 builds from stars), here built exactly from the
  Fourier coefficients of ``vscr`` on the mesh, so that it is the same operator
  that H|psi> applies.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .crystal import adot_to_avec, adot_to_bdot

PI = math.pi


@dataclass
class Species:
    """One atomic species: Gaussian local potential and s/p KB projectors."""
    v0: float                    # depth of -v0 * exp(-r^2 / (2 sigma^2)) (Ha)
    sigma: float                 # width of the local Gaussian (bohr)
    ekb: tuple = (2.0, -1.5)     # E_KB per angular momentum l = 0, 1, ... (Ha)
    sigma_kb: float = 1.0        # width of r^l exp(-r^2/(2 s^2)) projectors
    rat: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))  # lattice coords

    @property
    def natom(self) -> int:
        return int(self.rat.shape[0])


def rylm(qcar: np.ndarray, lmax: int) -> np.ndarray:
    """Real solid harmonics r^l sqrt(4pi/(2l+1)) Y_lm, Src/numeric/ylm_rc.f90:82-106.

    qcar: (3, n) Cartesian vectors. Returns (lmax+1, 2*lmax+1, n) indexed
    [l, m + lmax].
    """
    x, y, z = qcar
    n = qcar.shape[1]
    out = np.zeros((lmax + 1, 2 * lmax + 1, n))
    c = lmax
    out[0, c] = 1.0
    if lmax > 0:
        out[1, c - 1] = y
        out[1, c + 0] = z
        out[1, c + 1] = x
    if lmax > 1:
        s3 = math.sqrt(3.0)
        out[2, c - 2] = s3 * x * y
        out[2, c - 1] = s3 * z * y
        out[2, c + 0] = 0.5 * (2 * z * z - x * x - y * y)
        out[2, c + 1] = s3 * z * x
        out[2, c + 2] = math.sqrt(0.75) * (x * x - y * y)
    if lmax > 2:
        out[3, c - 3] = math.sqrt(5.0 / 8) * (3 * x * x - y * y) * y
        out[3, c - 2] = math.sqrt(15.0) * z * x * y
        out[3, c - 1] = math.sqrt(3.0 / 8) * (4 * z * z - x * x - y * y) * y
        out[3, c + 0] = 0.5 * (2 * z * z - 3 * x * x - 3 * y * y) * z
        out[3, c + 1] = math.sqrt(3.0 / 8) * (4 * z * z - x * x - y * y) * x
        out[3, c + 2] = math.sqrt(15.0 / 4) * (x * x - y * y) * z
        out[3, c + 3] = -math.sqrt(5.0 / 8) * (3 * y * y - x * x) * x
    return out


def kb_radial(q: np.ndarray, l: int, ekb: float, s: float) -> np.ndarray:
    """(1/q^l) * KB projector of beta_l(r) = N_l r^l exp(-r^2/(2 s^2)).

    beta is normalised to 1 in real space and carries sqrt(|E_KB|); the
    angular factor sqrt((2l+1)/(4 pi)) converts rylm to Y_lm, so that
    anlga = e^{-iG.tau} rylm_lm(q) i^l vkb(q) / sqrt(vcell).
    """
    nl = math.sqrt(2.0 / (math.gamma(l + 1.5) * s ** (2 * l + 3)))
    amp = math.sqrt(abs(ekb)) * 4 * PI * nl * math.sqrt(PI / 2) * s ** (2 * l + 3)
    amp *= math.sqrt((2 * l + 1) / (4 * PI))
    return amp * np.exp(-0.5 * (q * s) ** 2)


def kb_tables(species: list[Species], delq: float = 0.01, nq: int = 4000, lmax: int = 1):
    """vkb(-2:nq, 0:3, type) (FP64) and nkb(0:3, type) (int), reference layout.

    Returned as numpy arrays vkb[ntype, 4, nq+3] (index n+2 is q = n*delq,
    negative indices by even extension) and nkb[ntype, 4].
    """
    ntype = len(species)
    vkb = np.zeros((ntype, 4, nq + 3))
    nkb = np.zeros((ntype, 4), dtype=np.int32)
    qn = np.abs(np.arange(-2, nq + 1)) * delq
    for t, sp in enumerate(species):
        for l in range(min(lmax, len(sp.ekb) - 1) + 1):
            e = sp.ekb[l]
            if e == 0.0:
                continue
            vkb[t, l] = kb_radial(qn, l, e, sp.sigma_kb)
            nkb[t, l] = 1 if e > 0 else -1
    return vkb, nkb


def nanl_of(species: list[Species], nkb: np.ndarray) -> int:
    """Number of projectors, sum over types of natom * sum_l (2l+1)."""
    return int(sum(sp.natom * sum(2 * l + 1 for l in range(4) if nkb[t, l] != 0)
                   for t, sp in enumerate(species)))


def _interp(vtab: np.ndarray, xq: np.ndarray, nq: int):
    """Quadratic interpolation used by proj_nl_kb_c16.f90:226-240."""
    ni = np.rint(xq).astype(np.int64)
    ni = np.maximum(ni, 0)
    ok = ni < nq - 1
    nic = np.where(ok, ni, 0)
    xi = xq - nic
    v0 = vtab[nic + 2]
    vp = vtab[nic + 3]
    vm = vtab[nic + 1]
    val = v0 * (1 + xi) * (1 - xi) + 0.5 * (vp * (1 + xi) - vm * (1 - xi)) * xi
    return np.where(ok, val, 0.0)


def proj_nl_kb(rkpt, isort, kgv, species, vkb, nkb, adot, delq=0.01, nq=4000):
    """KB projectors for one k-point, Src/omp/proj_nl_kb_c16.f90:23-275.

    anlga(i, ind) = e^{-2 pi i G_i . tau} * rylm_lm(k+G_i) * i^l * vkb_l(|k+G_i|)/sqrt(vcell)
    with projector order type -> l -> m -> atom (:170-184) and
    xnlkb(ind) = nkb(l, type) (:266). Returns (anlga (mtxd, nanl) complex128,
    xnlkb (nanl,) float64).
    """
    _, bvec = adot_to_avec(adot)
    vcell, _ = adot_to_bdot(adot)
    fac = 1.0 / math.sqrt(vcell)
    g = kgv[:, np.asarray(isort) - 1].astype(np.float64)
    qk = g + np.asarray(rkpt, dtype=np.float64)[:, None]
    qcar = bvec @ qk
    qi = np.sqrt((qcar ** 2).sum(axis=0))
    lmx = max((l for t in range(len(species)) for l in range(4) if nkb[t, l] != 0), default=0)
    ry = rylm(qcar, lmx)
    cols = []
    xnl = []
    for t, sp in enumerate(species):
        st = np.exp(-2j * PI * (sp.rat @ g))          # (natom, mtxd)
        for l in range(lmx + 1):
            if nkb[t, l] == 0:
                continue
            vq = fac * _interp(vkb[t, l], qi / delq, nq)
            vqil = vq * (1j ** l)
            for m in range(-l, l + 1):
                for a in range(sp.natom):
                    cols.append(st[a] * ry[l, m + lmx] * vqil)
                    xnl.append(float(nkb[t, l]))
    if not cols:
        return np.zeros((g.shape[1], 0), dtype=np.complex128), np.zeros(0)
    return np.ascontiguousarray(np.stack(cols, axis=1)), np.array(xnl)


def hamilt_diag_kb(qmod, ekpg, veffr1, species, vkb, nkb, adot, delq=0.01, nq=4000):
    """Diagonal of H, Src/ALFA/hamilt_diag_kb.f90:89-127.

    hdiag = ekpg + V(G=0) + sum_type natom * sum_l nkb * (fac vkb_l(q) q^l)^2.
    """
    vcell, _ = adot_to_bdot(adot)
    fac = 1.0 / math.sqrt(vcell)
    hd = np.asarray(ekpg, dtype=np.float64) + veffr1
    for t, sp in enumerate(species):
        acc = np.zeros_like(hd)
        for l in range(4):
            if nkb[t, l] == 0:
                continue
            vq = fac * _interp(vkb[t, l], qmod / delq, nq) * qmod ** l
            acc += vq * vq * nkb[t, l]
        hd = hd + acc * sp.natom
    return hd


def local_potential_box(species, adot, box, idpad: int = 0):
    """Real screened potential on the FFT box, vscr(id*n2*n3) in reference order.

    V(G) = (1/vcell) sum_atoms e^{-iG.tau} (-v0) (2 pi sigma^2)^{3/2} e^{-G^2 sigma^2/2}
    for every G on the box except the Nyquist planes (kept Hermitian), then
    vscr(r) = sum_G V(G) e^{+iG.r} (the reference's unscaled backward
    transform, pot_local.f90:137-186). Returns (vscr flat float64 of size
    id*n2*n3, veffr1 = V(G=0)).
    """
    n1, n2, n3 = box
    vcell, bdot = adot_to_bdot(adot)
    m = [np.fft.fftfreq(n, 1.0 / n).astype(np.int64) for n in (n1, n2, n3)]
    m1, m2, m3 = np.meshgrid(*m, indexing="ij")          # (n1, n2, n3)
    mm = np.stack([m1, m2, m3]).reshape(3, -1).astype(np.float64)
    g2 = np.einsum("in,ij,jn->n", mm, bdot, mm)
    vg = np.zeros(mm.shape[1], dtype=np.complex128)
    for sp in species:
        ff = -sp.v0 * (2 * PI * sp.sigma ** 2) ** 1.5 * np.exp(-0.5 * g2 * sp.sigma ** 2) / vcell
        # structure factor sum_a e^{-2 pi i m.rat_a}, separable in the three directions
        p1 = np.exp(-2j * PI * np.outer(sp.rat[:, 0], m[0]))          # (natom, n1)
        p2 = np.exp(-2j * PI * np.outer(sp.rat[:, 1], m[1]))
        p3 = np.exp(-2j * PI * np.outer(sp.rat[:, 2], m[2]))
        sf = np.empty((n1, n2, n3), dtype=np.complex128)
        for k in range(n3):
            sf[:, :, k] = (p1 * p3[:, k:k + 1]).T @ p2
        vg += ff * sf.reshape(-1)
    vg = vg.reshape(n1, n2, n3)
    for ax, n in enumerate((n1, n2, n3)):
        if n % 2 == 0:
            sl = [slice(None)] * 3
            sl[ax] = n // 2
            vg[tuple(sl)] = 0
    veffr1 = float(vg[0, 0, 0].real)
    vr = np.fft.ifftn(vg) * (n1 * n2 * n3)          # e^{+iG.r}, unscaled
    if np.abs(vr.imag).max() > 1e-9 * max(1.0, np.abs(vr.real).max()):
        raise RuntimeError("local_potential_box: potential is not real")
    ident = n1 + idpad
    box_arr = np.zeros((n3, n2, ident))
    box_arr[:, :, :n1] = vr.real.transpose(2, 1, 0)
    return box_arr.reshape(-1), veffr1


def local_potential_coefficients(species, adot, box):
    """V(G) of local_potential_box as a list of G vectors: (kgv (3, ng) int32 signed
    reciprocal-lattice coordinates, V (ng,) complex128), every G of the box except the Nyquist
    planes. With one star per G (inds = 1..ng, phase 1, conj +1) these are the veff, kgv,
    phase, conj and inds arguments of pot_local (Src/cpw_lib/pot_local.f90) that reproduce
    local_potential_box's vscr."""
    n1, n2, n3 = box
    vcell, bdot = adot_to_bdot(adot)
    m = [np.fft.fftfreq(n, 1.0 / n).astype(np.int64) for n in (n1, n2, n3)]
    m1, m2, m3 = np.meshgrid(*m, indexing="ij")
    keep = np.ones(m1.shape, dtype=bool)
    for mi, n in ((m1, n1), (m2, n2), (m3, n3)):
        if n % 2 == 0:
            keep &= mi != -(n // 2)
    g = np.stack([m1[keep], m2[keep], m3[keep]]).astype(np.float64)
    g2 = np.einsum("in,ij,jn->n", g, bdot, g)
    vg = np.zeros(g.shape[1], dtype=np.complex128)
    for sp in species:
        ff = -sp.v0 * (2 * PI * sp.sigma ** 2) ** 1.5 * np.exp(-0.5 * g2 * sp.sigma ** 2) / vcell
        vg += ff * np.exp(-2j * PI * (np.asarray(sp.rat) @ g)).sum(axis=0)
    return np.asfortranarray(g.astype(np.int32)), vg


def local_form_factors_box(species, adot, box):
    """Form factors v_t(G) of every species on the box, FFT order, shape (ntype, n3, n2, n1).

    The same coefficients local_potential_box places (Nyquist planes zero), so
    that V(G) = sum_a e^{-2 pi i m.tau_a} v_t(G) reproduces vscr.
    """
    n1, n2, n3 = box
    vcell, bdot = adot_to_bdot(adot)
    mz, my, mx = np.meshgrid(*[np.fft.fftfreq(n, 1.0 / n) for n in (n3, n2, n1)], indexing="ij")
    mm = np.stack([mx.ravel(), my.ravel(), mz.ravel()])
    g2 = np.einsum("in,ij,jn->n", mm, bdot, mm).reshape(n3, n2, n1)
    out = np.zeros((len(species), n3, n2, n1))
    for t, sp in enumerate(species):
        out[t] = -sp.v0 * (2 * PI * sp.sigma ** 2) ** 1.5 * np.exp(-0.5 * g2 * sp.sigma ** 2) / vcell
    for ax, n in ((3, n1), (2, n2), (1, n3)):
        if n % 2 == 0:
            sl = [slice(None)] * 4
            sl[ax] = n // 2
            out[tuple(sl)] = 0.0
    return out


def proj_atom_map(species, nkb):
    """0-based global atom index of each projector column (order type -> l -> m -> atom)."""
    out = []
    off = 0
    for t, sp in enumerate(species):
        for l in range(4):
            if nkb[t, l] == 0:
                continue
            for _m in range(2 * l + 1):
                out.extend(range(off, off + sp.natom))
        off += sp.natom
    return np.array(out, dtype=np.int32)


def potential_fourier(vscr, box, ident):
    """Fourier coefficients Vt(m) = (1/N) sum_r vscr(r) e^{-i 2pi m.r/n} on the box."""
    n1, n2, n3 = box
    v = np.asarray(vscr).reshape(n3, n2, ident)[:, :, :n1].transpose(2, 1, 0)
    return np.fft.fftn(v) / (n1 * n2 * n3)


def small_hamiltonian(mtxds, isort, kgv, ekpg, vscr, box, ident, anlga, xnlkb):
    """Leading mtxds x mtxds block of H (the ``hamsm`` input of ditsp_c16).

    H_ij = ekpg_i delta_ij + Vt(G_i - G_j) + sum_a anlga_ia xnlkb_a conj(anlga_ja),
    with Vt the mesh Fourier coefficients of vscr, i.e. exactly the matrix of
    the operator hk_psi_c16 applies (hamilt_kb.f90 builds the same block from
    the star representation of the potential).
    """
    n1, n2, n3 = box
    vt = potential_fourier(vscr, box, ident)
    g = kgv[:, np.asarray(isort[:mtxds]) - 1]
    d = g[:, :, None] - g[:, None, :]
    h = vt[d[0] % n1, d[1] % n2, d[2] % n3]
    h = h + np.diag(np.asarray(ekpg[:mtxds], dtype=np.float64))
    x = anlga[:mtxds]
    h = h + (x * xnlkb[None, :]) @ x.conj().T
    return np.asfortranarray(0.5 * (h + h.conj().T))
