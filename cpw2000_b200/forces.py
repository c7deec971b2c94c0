"""Hellmann-Feynman energy, forces and dE/dV_loc behind torch.autograd.

For fixed wavefunctions psi (one k-point, device-resident) and occupations f:

    E(tau) = sum_n f_n <psi_n| T + V_loc[vscr(tau)] + V_KB[tau] |psi_n>

``LocalPotential.apply(tau, system)`` builds vscr(tau) (the screened potential
on the FFT box, reference layout); its backward contracts the incoming dE/dvscr
with the structure-factor derivative on the GPU (cpw_b200_structure_grad_device).
``HFEnergy.apply(tau, vscr, system)`` evaluates E with the library's H|psi>;
its backward returns dE/dvscr = rho(r)/N from the GPU density
(cpw_b200_density_device, the mesh density of Src/omp/charge_by_fft.f90) and
the KB term of dE/dtau from the projector derivatives
(cpw_b200_nl_grad_device, Src/ALFA/for_str_nl_kb.f90). Composed,
``energy(tau, system)`` has tau.grad = dE/dtau, and forces = -dE/dtau.

tau is (natom, 3) float64 in lattice coordinates, atoms ordered by species as
the workload lists them; ``to_cartesian`` converts covariant lattice
derivatives to Cartesian Ha/bohr. The density recomputes psi(r) band chunk by
band chunk (nothing real-space is stored across calls).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib, pseudo
from .crystal import adot_to_avec
from .hk_psi import FP64, Context, torch_stream_handle


class HFSystem:
    """Fixed wavefunctions and the parameters H depends on (one k-point)."""

    def __init__(self, workload, inputs: dict, psi, occ, device: int = 0, precision: int = FP64):
        self.w = workload
        self.d = inputs
        self.psi = psi                        # (mtxd, nb) column-major complex128 CUDA tensor
        self.occ = np.ascontiguousarray(occ, dtype=np.float64)
        self.nb = int(len(self.occ))
        self.dev = psi.device
        self.ctx = Context(device, precision=precision)
        self.ctx.set_kpoint(inputs["mtxd"], inputs["isort"], inputs["kgv"], inputs["ekpg"], inputs["kmscr"])
        n1, n2, n3 = (int(v) for v in inputs["kmscr"][3:6])
        self.box = (n1, n2, n3)
        self.ident = int(inputs["kmscr"][6])
        self.natom = sum(sp.natom for sp in workload.species)
        self.atom_type = np.concatenate([np.full(sp.natom, t, dtype=np.int32)
                                         for t, sp in enumerate(workload.species)])
        self.proj_atom = pseudo.proj_atom_map(workload.species, inputs["nkb"])
        vgt = pseudo.local_form_factors_box(workload.species, workload.adot, self.box)
        self.vgt = torch.from_numpy(np.ascontiguousarray(vgt)).to(self.dev)

    def tau0(self) -> torch.Tensor:
        return torch.from_numpy(np.concatenate([sp.rat for sp in self.w.species]).astype(np.float64))

    def species_at(self, tau: np.ndarray):
        out, k = [], 0
        for sp in self.w.species:
            out.append(pseudo.Species(sp.v0, sp.sigma, sp.ekb, sp.sigma_kb, tau[k:k + sp.natom].copy()))
            k += sp.natom
        return out

    # ---- library calls ----
    def density(self) -> torch.Tensor:
        """rho(r) = sum_n f_n |psi_n(r)|^2, (n3, n2, n1) float64 on the device."""
        n1, n2, n3 = self.box
        rho = torch.empty((n3, n2, n1), dtype=torch.float64, device=self.dev)
        L = _lib.lib()
        _lib.check(L.cpw_b200_density_device(self.ctx.handle, self.nb, C.c_void_p(self.psi.data_ptr()),
                                             Context._ld(self.psi), _lib.dptr(self.occ), C.c_void_p(rho.data_ptr()),
                                             C.c_void_p(torch_stream_handle(self.dev))))
        return rho

    def structure_grad(self, g_box: torch.Tensor, tau: np.ndarray) -> np.ndarray:
        g = g_box.contiguous()
        out = np.zeros((self.natom, 3))
        t = np.ascontiguousarray(tau, dtype=np.float64)
        L = _lib.lib()
        _lib.check(L.cpw_b200_structure_grad_device(self.ctx.handle, C.c_void_p(g.data_ptr()), self.natom,
                                                    _lib.iptr(self.atom_type), _lib.dptr(t), len(self.w.species),
                                                    C.c_void_p(self.vgt.data_ptr()), _lib.dptr(out),
                                                    C.c_void_p(torch_stream_handle(self.dev))))
        return out

    def nl_grad(self) -> np.ndarray:
        out = np.zeros((self.natom, 3))
        L = _lib.lib()
        _lib.check(L.cpw_b200_nl_grad_device(self.ctx.handle, self.nb, C.c_void_p(self.psi.data_ptr()),
                                             Context._ld(self.psi), _lib.dptr(self.occ), _lib.iptr(self.proj_atom),
                                             self.natom, _lib.dptr(out), C.c_void_p(torch_stream_handle(self.dev))))
        return out

    def energy_now(self) -> float:
        hp = torch.empty((self.nb, self.psi.shape[0]), dtype=torch.complex128, device=self.dev).t()
        self.ctx.hk_psi(self.psi, hp)
        e = torch.real(torch.sum(torch.conj(self.psi) * hp, dim=0))
        return float(torch.sum(torch.from_numpy(self.occ).to(self.dev) * e).item())


class LocalPotential(torch.autograd.Function):
    """vscr(tau) on the FFT box (reference layout id*n2*n3)."""

    @staticmethod
    def forward(ctx, tau, system: HFSystem):
        species = system.species_at(tau.detach().cpu().numpy())
        vscr, _ = pseudo.local_potential_box(species, system.w.adot, system.box, system.w.idpad)
        ctx.system = system
        ctx.save_for_backward(tau)
        return torch.from_numpy(vscr).to(system.dev)

    @staticmethod
    def backward(ctx, g):
        (tau,) = ctx.saved_tensors
        s = ctx.system
        n1, n2, n3 = s.box
        gbox = g.reshape(n3, n2, s.ident)[:, :, :n1]
        d = s.structure_grad(gbox, tau.detach().cpu().numpy())
        return torch.from_numpy(d).to(tau), None


class HFEnergy(torch.autograd.Function):
    """E = sum_n f_n <psi_n|H(tau, vscr)|psi_n> for the system's fixed psi."""

    @staticmethod
    def forward(ctx, tau, vscr, system: HFSystem):
        species = system.species_at(tau.detach().cpu().numpy())
        system.ctx.set_potential(vscr.detach().cpu().numpy())
        d = system.d
        anl, xnl = pseudo.proj_nl_kb(d["rkpt"], d["isort"], d["kgv"], species, d["vkb"], d["nkb"], system.w.adot)
        system.ctx.set_projectors(anl, xnl)
        ctx.system = system
        ctx.tau_dtype = tau.dtype
        return torch.tensor(system.energy_now(), dtype=torch.float64)

    @staticmethod
    def backward(ctx, gE):
        s = ctx.system
        n1, n2, n3 = s.box
        rho = s.density()
        gv = torch.zeros((n3, n2, s.ident), dtype=torch.float64, device=s.dev)
        gv[:, :, :n1] = rho / float(n1 * n2 * n3)
        gt = torch.from_numpy(s.nl_grad())
        ge = float(gE)
        return gt * ge, gv.reshape(-1) * ge, None


def energy(tau: torch.Tensor, system: HFSystem) -> torch.Tensor:
    """E(tau) with local and KB terms both differentiable in tau."""
    return HFEnergy.apply(tau, LocalPotential.apply(tau, system), system)


def forces(system: HFSystem, tau: torch.Tensor | None = None):
    """(E, F) with F = -dE/dtau in lattice components (natom, 3)."""
    t = (system.tau0() if tau is None else tau.detach().clone()).requires_grad_(True)
    e = energy(t, system)
    e.backward()
    return float(e.item()), -t.grad.numpy().copy()


def to_cartesian(f_lattice: np.ndarray, adot) -> np.ndarray:
    """Covariant lattice components -dE/dtau_j -> Cartesian Ha/bohr in the canonical orientation."""
    avec, _ = adot_to_avec(adot)
    return np.asarray(f_lattice) @ np.linalg.inv(avec)
