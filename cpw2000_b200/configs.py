"""The five synthetic workloads (crystals, cut-offs, boxes, k-points, bands).

All inputs are seeded and built from analytic Gaussian pseudopotentials (no
pseudopotential files or datasets are involved). Geometry follows ideal
diamond / zincblende cells (the cells of the reference's
Structures/diamond_cubic_supercells inputs) with seeded Gaussian displacements.

``kpoint_inputs`` returns exactly the arrays ``hk_psi_c16`` / ``ditsp_c16``
take for one k-point.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import crystal, pseudo

DIAMOND_FCC = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0]], dtype=np.float64)


@dataclass
class Workload:
    name: str
    adot: np.ndarray
    species: list
    ecut: float                  # Ha; basis is 1/2 |k+G|^2 <= ecut
    box: tuple                   # (n1, n2, n3)
    kpoints: np.ndarray          # (nk, 3) reciprocal lattice coordinates
    nbands: int
    idpad: int = 0               # id = n1 + idpad (reference kmscr(7))
    extra: dict = field(default_factory=dict)

    @property
    def ident(self) -> int:
        return self.box[0] + self.idpad


def _cubic_supercell(a: float, ncell: int, seed: int, sigma: float, two_species=False):
    base_a = DIAMOND_FCC
    base_b = DIAMOND_FCC + 0.25
    shifts = np.array([(i, j, k) for i in range(ncell) for j in range(ncell) for k in range(ncell)], dtype=np.float64)
    pa = ((base_a[None, :, :] + shifts[:, None, :]) / ncell).reshape(-1, 3)
    pb = ((base_b[None, :, :] + shifts[:, None, :]) / ncell).reshape(-1, 3)
    rng = np.random.default_rng(seed)
    alat = a * ncell
    if sigma > 0:
        pa = pa + rng.normal(0.0, sigma, pa.shape) / alat
        pb = pb + rng.normal(0.0, sigma, pb.shape) / alat
    adot = np.eye(3) * alat * alat
    if two_species:
        return adot, [pa, pb]
    return adot, [np.concatenate([pa, pb])]


def si2_fcc() -> Workload:
    """Si diamond primitive cell, a=10.26, Ecut 16 Ha, 32^3, 10 k-points, 8 bands."""
    a = 10.26
    av = 0.5 * a * np.array([[0, 1, 1], [1, 0, 1], [1, 1, 0]], dtype=np.float64).T
    adot = av.T @ av
    sp = pseudo.Species(v0=4.0, sigma=0.8, ekb=(2.0, -1.5), sigma_kb=1.0,
                        rat=np.array([[0, 0, 0], [.25, .25, .25]], dtype=np.float64))
    rk, w = crystal.monkhorst_pack(adot, (4, 4, 4), (0.5, 0.5, 0.5))
    return Workload("si2_fcc_ecut16_box32", adot, [sp], 16.0, (32, 32, 32), rk, 8,
                    extra={"kweights": w})


def si64_cubic(seed: int = 64) -> Workload:
    """Si 64-atom cubic supercell a=20.52, sigma 0.02, Ecut 16, 96^3, Gamma, 160 bands."""
    adot, pos = _cubic_supercell(10.26, 2, seed, 0.02)
    sp = pseudo.Species(v0=4.0, sigma=0.8, ekb=(2.0, -1.5), sigma_kb=1.0, rat=pos[0])
    return Workload("si64_cubic_ecut16_box96", adot, [sp], 16.0, (96, 96, 96),
                    np.zeros((1, 3)), 160)


def si8_cubic_kbatch(seed: int = 8, nk: int = 64) -> Workload:
    """Si 8-atom cubic cell a=10.26, Ecut 20, 40^3, 64 random k, 40 bands."""
    adot, pos = _cubic_supercell(10.26, 1, seed, 0.0)
    sp = pseudo.Species(v0=4.0, sigma=0.8, ekb=(2.0, -1.5), sigma_kb=1.0, rat=pos[0])
    rng = np.random.default_rng(seed)
    rk = rng.uniform(-0.5, 0.5, (nk, 3))
    return Workload("si8_cubic_ecut20_box40_k64", adot, [sp], 20.0, (40, 40, 40), rk, 40)


def zb64_cubic(seed: int = 164) -> Workload:
    """Zincblende 64-atom cubic a=21.0, two species, sigma 0.05, Ecut 16, 96^3, 160 bands."""
    adot, pos = _cubic_supercell(10.5, 2, seed, 0.05, two_species=True)
    cat = pseudo.Species(v0=4.5, sigma=0.9, ekb=(2.0, -1.5), sigma_kb=1.0, rat=pos[0])
    ani = pseudo.Species(v0=3.5, sigma=0.7, ekb=(2.0, -1.5), sigma_kb=1.0, rat=pos[1])
    return Workload("zb64_cubic_ecut16_box96", adot, [cat, ani], 16.0, (96, 96, 96),
                    np.zeros((1, 3)), 160)


def si216_cubic(seed: int = 216) -> Workload:
    """Si 216-atom cubic a=30.78, sigma 0.03, Ecut 16, 144^3, Gamma + 3 random k, 480 bands."""
    adot, pos = _cubic_supercell(10.26, 3, seed, 0.03)
    sp = pseudo.Species(v0=4.0, sigma=0.8, ekb=(2.0, -1.5), sigma_kb=1.0, rat=pos[0])
    rng = np.random.default_rng(seed)
    rk = np.concatenate([np.zeros((1, 3)), rng.uniform(-0.5, 0.5, (3, 3))])
    return Workload("si216_cubic_ecut16_box144", adot, [sp], 16.0, (144, 144, 144), rk, 480)


def small_test(seed: int = 5, box=(24, 20, 18), ecut=4.0) -> Workload:
    """A small non-cubic cell with a non-cubic box, for fast parity tests."""
    av = np.array([[7.1, 0.0, 0.0], [1.3, 6.4, 0.0], [0.7, 0.9, 5.8]]).T
    adot = av.T @ av
    rng = np.random.default_rng(seed)
    sp1 = pseudo.Species(v0=3.0, sigma=0.9, ekb=(2.0, -1.5), sigma_kb=0.9, rat=rng.uniform(0, 1, (2, 3)))
    sp2 = pseudo.Species(v0=2.0, sigma=0.7, ekb=(1.0, 0.8), sigma_kb=0.8, rat=rng.uniform(0, 1, (1, 3)))
    rk = np.array([[0.0, 0.0, 0.0], [0.13, -0.27, 0.31]])
    return Workload("small_triclinic", adot, [sp1, sp2], ecut, tuple(box), rk, 6, idpad=1)


WORKLOADS = {
    "si2": si2_fcc,
    "si64": si64_cubic,
    "si8k": si8_cubic_kbatch,
    "zb64": zb64_cubic,
    "si216": si216_cubic,
    "small": small_test,
}


def kpoint_inputs(w: Workload, ik: int = 0, nbands: int | None = None, delq=0.01, nq=4000,
                  with_hamsm: bool = False):
    """Every array hk_psi_c16 / ditsp_c16 takes for k-point ik of workload w.

    Returns a dict with: mtxd, isort (1-based int32), kgv (3, ng) int32, ng,
    ekpg, qmod, vscr (flat id*n2*n3), kmscr (7 ints), anlga (mtxd, nanl)
    complex128, xnlkb, nanl, hdiag, veffr1, and (optionally) mtxds + hamsm.
    """
    rk = np.asarray(w.kpoints[ik], dtype=np.float64)
    gmax = math.sqrt(2 * w.ecut)
    _, bvec = crystal.adot_to_avec(w.adot)
    kcar = float(np.linalg.norm(bvec @ rk))
    kgv = crystal.gspace(w.adot, gmax + kcar + 1.0)
    mtxd, isort, qmod, ekpg = crystal.hamilt_struct(w.ecut, rk, kgv, w.adot)
    kd = crystal.kd_of_basis(kgv, isort)
    n1, n2, n3 = w.box
    if kd[0] > (n1 - 1) // 2 or kd[1] > (n2 - 1) // 2 or kd[2] > (n3 - 1) // 2:
        raise ValueError(f"box {w.box} too small for basis extent {kd}")
    vscr, veffr1 = pseudo.local_potential_box(w.species, w.adot, w.box, w.idpad)
    vkb, nkb = pseudo.kb_tables(w.species, delq, nq)
    anlga, xnlkb = pseudo.proj_nl_kb(rk, isort, kgv, w.species, vkb, nkb, w.adot, delq, nq)
    hdiag = pseudo.hamilt_diag_kb(qmod, ekpg, veffr1, w.species, vkb, nkb, w.adot, delq, nq)
    # kmscr(1:3): extent of the potential's G-space on the mesh; size_fft of it
    # reproduces the box for every size the reference's size_fft can return.
    kmscr = np.array([(n1 - 1) // 2, (n2 - 1) // 2, (n3 - 1) // 2, n1, n2, n3, n1 + w.idpad],
                     dtype=np.int32)
    out = dict(mtxd=mtxd, isort=isort, kgv=kgv, ng=int(kgv.shape[1]), ekpg=ekpg, qmod=qmod,
               vscr=vscr, kmscr=kmscr, anlga=np.asfortranarray(anlga), xnlkb=xnlkb,
               nanl=int(xnlkb.size), hdiag=hdiag, veffr1=veffr1, rkpt=rk,
               nbands=w.nbands if nbands is None else nbands, vkb=vkb, nkb=nkb)
    if with_hamsm:
        mtxds = crystal.size_mtxds(hdiag, out["nbands"])
        out["mtxds"] = mtxds
        out["hamsm"] = pseudo.small_hamiltonian(mtxds, isort, kgv, ekpg, vscr, w.box, w.ident,
                                                anlga, xnlkb)
    return out


def random_psi(mtxd: int, nb: int, seed: int = 0, ld: int | None = None) -> np.ndarray:
    """Seeded complex128 normal wavefunctions, Fortran order (ld, nb)."""
    rng = np.random.default_rng(seed)
    ld = mtxd if ld is None else ld
    psi = np.zeros((ld, nb), dtype=np.complex128, order="F")
    psi[:mtxd] = rng.standard_normal((mtxd, nb)) + 1j * rng.standard_normal((mtxd, nb))
    return psi
