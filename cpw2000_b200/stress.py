"""Hellmann-Feynman stress: the strain derivative of E = sum_n f_n <psi_n|H|psi_n>.

At fixed plane-wave coefficients and fixed lattice coordinates of the atoms, a
symmetric Cartesian strain e (lattice vectors a -> (1 + e) a) changes the k+G
vectors to (1 - e) q, the cell volume to (1 + tr e) vcell, and with them

    kinetic   E_kin = sum_G w(G) |q|^2 / 2,              w(G) = sum_n f_n |c_n(G)|^2
    local     E_loc = sum_G Re conj(rho~(G)) V(G),       V(G) = sum_t S_t(G) v_t(|G|^2) / vcell
    KB        E_nl  = sum_a Re sum_G conj(X_a(G)) Y_a(G), X_a = vcell^-1/2 S_a(G) h_lm(q),
                                                          Y = psi diag(f) P^H diag(xnlkb)

so that S_ij = dE/de_ij is

    kinetic   - sum_G w q_i q_j
    local     - delta_ij E_loc - 2 sum_G Re conj(rho~) W(G) G_i G_j,   W = sum_t S_t dv_t/d|G|^2 / vcell
    KB        - delta_ij E_nl + 2 Re sum_a sum_G vcell^-1/2 conj(S_a dh_lm/de_ij) Y_a

with d|q|/de_ij = -q_i q_j / |q| and d q_c/de_ij = -(delta_ci q_j + delta_cj q_i) / 2 in h.
The GPU supplies w and Y (cpw_b200_stress_inputs_device) and rho (the density kernel);
the derivatives of the set-up quantities (form factors, projector radial tables and
solid harmonics) are host arithmetic, as their set-up is.

Reported as the reference does (Src/ALFA/for_str_kinetic_stress.f90,
for_str_local_stress.f90, for_str_nl_kb.f90:364-376): the covariant lattice tensor
sigma = -2 adot (dE/dadot) adot, with dE/dadot = (1/2) avec^-1 S avec^-T the derivative
with respect to the real-space metric.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _lib, pseudo
from .crystal import adot_to_avec, adot_to_bdot

PI = math.pi


def strain_to_metric(S: np.ndarray, adot) -> np.ndarray:
    """dE/dadot from the Cartesian strain derivative S = dE/de (e symmetric)."""
    avec, _ = adot_to_avec(adot)
    ai = np.linalg.inv(avec)
    return 0.5 * ai @ S @ ai.T


def covariant(dedadot: np.ndarray, adot) -> np.ndarray:
    """The reference's covariant stress tensor -2 adot (dE/dadot) adot."""
    adot = np.asarray(adot, dtype=np.float64)
    return -2.0 * adot @ dedadot @ adot


def interp_with_derivative(vtab: np.ndarray, xq: np.ndarray, nq: int):
    """The quadratic interpolation of proj_nl_kb_c16.f90:226-240 and its derivative in xq."""
    ni = np.maximum(np.rint(xq).astype(np.int64), 0)
    ok = ni < nq - 1
    nic = np.where(ok, ni, 0)
    xi = xq - nic
    v0, vp, vm = vtab[nic + 2], vtab[nic + 3], vtab[nic + 1]
    val = v0 * (1 + xi) * (1 - xi) + 0.5 * (vp * (1 + xi) - vm * (1 - xi)) * xi
    der = -2 * xi * v0 + (xi + 0.5) * vp + (xi - 0.5) * vm
    return np.where(ok, val, 0.0), np.where(ok, der, 0.0)


def box_potential(species, adot, box):
    """V(G) and W(G) = sum_t S_t(G) dv_t/d|G|^2 / vcell on the box, arrays (n3, n2, n1) in FFT
    order with the Nyquist planes zero (as pseudo.local_potential_box places them), and the
    Cartesian G vectors (3, n3, n2, n1)."""
    n1, n2, n3 = box
    vcell, _ = adot_to_bdot(adot)
    _, bvec = adot_to_avec(adot)
    m = [np.fft.fftfreq(n, 1.0 / n) for n in (n1, n2, n3)]
    M3, M2, M1 = np.meshgrid(m[2], m[1], m[0], indexing="ij")
    gc = np.einsum("ij,jabc->iabc", bvec, np.stack([M1, M2, M3]))
    g2 = (gc ** 2).sum(axis=0)
    V = np.zeros((n3, n2, n1), dtype=np.complex128)
    W = np.zeros_like(V)
    for sp in species:
        f = -sp.v0 * (2 * PI * sp.sigma ** 2) ** 1.5 * np.exp(-0.5 * g2 * sp.sigma ** 2) / vcell
        p1 = np.exp(-2j * PI * np.outer(sp.rat[:, 0], m[0]))          # (natom, n1)
        p2 = np.exp(-2j * PI * np.outer(sp.rat[:, 1], m[1]))
        p3 = np.exp(-2j * PI * np.outer(sp.rat[:, 2], m[2]))
        sf = np.empty((n3, n2, n1), dtype=np.complex128)
        for k in range(n3):
            sf[k] = (p2 * p3[:, k:k + 1]).T @ p1
        V += f * sf
        W += (-0.5 * sp.sigma ** 2) * f * sf
    for ax, n in ((2, n1), (1, n2), (0, n3)):
        if n % 2 == 0:
            sl = [slice(None)] * 3
            sl[ax] = n // 2
            V[tuple(sl)] = 0
            W[tuple(sl)] = 0
    return V, W, gc


def kinetic_strain(w: np.ndarray, inputs: dict, adot) -> np.ndarray:
    _, bvec = adot_to_avec(adot)
    g = inputs["kgv"][:, np.asarray(inputs["isort"][: inputs["mtxd"]]) - 1].astype(np.float64)
    qc = bvec @ (g + np.asarray(inputs["rkpt"], dtype=np.float64)[:, None])
    return -np.einsum("g,ig,jg->ij", np.asarray(w), qc, qc)


def local_strain(rho_r: np.ndarray, species, adot, box):
    """(S_loc, E_loc) from the mesh density rho(r) (n3, n2, n1) = sum_n f_n |psi_n(r)|^2."""
    n1, n2, n3 = box
    rt = np.fft.fftn(rho_r) / (n1 * n2 * n3)
    V, W, gc = box_potential(species, adot, box)
    eloc = float(np.real(np.conj(rt) * V).sum())
    a = np.real(np.conj(rt) * W)
    S = -eloc * np.eye(3) - 2.0 * np.einsum("abc,iabc,jabc->ij", a, gc, gc)
    return S, eloc


def kb_strain(Y: np.ndarray, inputs: dict, species, adot, delq=0.01, nq=4000):
    """(S_nl, E_nl) from Y = psi diag(f) P^H diag(xnlkb) (mtxd x nanl)."""
    vcell, _ = adot_to_bdot(adot)
    _, bvec = adot_to_avec(adot)
    fac = 1.0 / math.sqrt(vcell)
    vkb, nkb = inputs["vkb"], inputs["nkb"]
    isort = np.asarray(inputs["isort"][: inputs["mtxd"]]) - 1
    g = inputs["kgv"][:, isort].astype(np.float64)
    qc = bvec @ (g + np.asarray(inputs["rkpt"], dtype=np.float64)[:, None])
    qi = np.sqrt((qc ** 2).sum(axis=0))
    qsafe = np.where(qi > 1e-12, qi, 1.0)
    lmx = max((l for t in range(len(species)) for l in range(4) if nkb[t, l] != 0), default=0)
    ry = pseudo.rylm(qc, lmx)
    # linear solid harmonics l = 1: rylm_1m(q) = R[m] . q
    R = pseudo.rylm(np.eye(3), 1)[1] if lmx >= 1 else None              # (3 m, 3 c)
    pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (2, 0)]
    dqn = np.stack([-qc[i] * qc[j] / qsafe for i, j in pairs])         # d|q|/de_ij (6, mtxd)
    dqn[:, qi <= 1e-12] = 0.0
    S6 = np.zeros(6)
    enl = 0.0
    col = 0
    X = inputs["anlga"]
    for t, sp in enumerate(species):
        st_conj = np.exp(2j * PI * (sp.rat @ g))                         # conj(e^{-2 pi i G.tau}) (natom, mtxd)
        for l in range(lmx + 1):
            if nkb[t, l] == 0:
                continue
            vint, dv = interp_with_derivative(vkb[t, l], qi / delq, nq)
            dvdq = dv / delq
            il = 1j ** l
            for m in range(-l, l + 1):
                cols = slice(col, col + sp.natom)
                Ya = Y[:, cols]                                           # (mtxd, natom)
                enl += float(np.real(np.sum(np.conj(X[:, cols]) * Ya)))
                Z = np.einsum("ag,ga->g", st_conj, Ya)                    # sum over atoms
                h_r = ry[l, m + lmx]
                for kk, (i, j) in enumerate(pairs):
                    dh = h_r * dvdq * dqn[kk]
                    if l == 1:
                        dh = dh - 0.5 * (R[m + 1, i] * qc[j] + R[m + 1, j] * qc[i]) * vint
                    S6[kk] += 2.0 * fac * float(np.real(np.sum(np.conj(il * dh) * Z)))
                col += sp.natom
    S = np.zeros((3, 3))
    for kk, (i, j) in enumerate(pairs):
        S[i, j] = S[j, i] = S6[kk]
    return S - enl * np.eye(3), enl


def stress_inputs(ctx, psi, occ):
    """(w (mtxd,), Y (mtxd, nanl)) on the GPU for the context's k-point, psi (mtxd, nb) CUDA tensor."""
    from .hk_psi import torch_stream_handle
    L = _lib.lib()
    if psi.stride(0) != 1:
        raise ValueError("psi must be column-major")
    m, nb = psi.shape
    occ = np.ascontiguousarray(occ, dtype=np.float64)
    w = torch.empty(m, dtype=torch.float64, device=psi.device)
    Y = torch.empty((max(ctx.nanl, 1), m), dtype=torch.complex128, device=psi.device).t()
    from .hk_psi import Context
    ld = Context._ld(psi)
    _lib.check(L.cpw_b200_stress_inputs_device(ctx.handle, int(nb), C.c_void_p(psi.data_ptr()), ld,
                                               occ.ctypes.data_as(_lib.DP), C.c_void_p(w.data_ptr()),
                                               C.c_void_p(Y.data_ptr()),
                                               C.c_void_p(torch_stream_handle(psi.device))))
    return w.cpu().numpy(), Y.cpu().numpy()[:, : ctx.nanl]


def stress(system, delq=0.01, nq=4000) -> dict:
    """Stress of a forces.HFSystem (one k-point, fixed wavefunctions): per term and total,
    covariant lattice tensors (Hartree) as the reference reports them, plus dE/dadot and the
    Cartesian strain derivative dE/de."""
    w_l = system.w
    d = system.d
    adot = w_l.adot
    psi = system.psi
    system.ctx.set_projectors(d["anlga"], d["xnlkb"])
    wG, Y = stress_inputs(system.ctx, psi, system.occ)
    rho = system.density().cpu().numpy()
    S_kin = kinetic_strain(wG, d, adot)
    S_loc, eloc = local_strain(rho, w_l.species, adot, system.box)
    S_nl, enl = kb_strain(Y, d, w_l.species, adot, delq, nq)
    out = {}
    total = np.zeros((3, 3))
    for name, S in (("kinetic", S_kin), ("local", S_loc), ("kb", S_nl)):
        dm = strain_to_metric(S, adot)
        out[name] = covariant(dm, adot)
        total = total + S
    out["dE_dstrain"] = total
    out["dE_dadot"] = strain_to_metric(total, adot)
    out["total"] = covariant(out["dE_dadot"], adot)
    out["e_local"] = eloc
    out["e_kb"] = enl
    return out


class StrainEnergy(torch.autograd.Function):
    """E(e) at fixed wavefunctions for a symmetric Cartesian strain e (3 x 3 tensor, evaluated at
    e = 0): forward returns the energy, backward the stress dE/de from the GPU adjoint."""

    @staticmethod
    def forward(ctx, e, system):
        ctx.system = system
        system.ctx.set_potential(system.d["vscr"])
        system.ctx.set_projectors(system.d["anlga"], system.d["xnlkb"])
        return torch.tensor(system.energy_now(), dtype=torch.float64)

    @staticmethod
    def backward(ctx, g):
        S = stress(ctx.system)["dE_dstrain"]
        return g * torch.from_numpy(S), None
