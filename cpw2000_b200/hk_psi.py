"""Python mirror of cpw2000's H|psi> interface over the C ABI.

``hk_psi_c16`` / ``hk_psi_nl_c16`` take the reference's argument lists
(Src/hk_psi/reference/hk_psi_c16.f90:28-32, Src/cpw_lib/hk_psi_nl_c16.f90:23-24)
with numpy arrays in Fortran order and host memory, like the Fortran callers.
``Context`` is the device-resident form used by the eigensolver and the
benchmarks: per-k-point inputs are uploaded once, H|psi> runs on torch CUDA
tensors (torch supplies the device memory and streams; the compute is the
library's CUDA kernels).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib, crystal, pseudo
from ._lib import check, dptr, iptr, zptr

FP64 = 0
MIXED = 1
MIXED_TC = 2


def _as_f(a, dtype):
    a = np.asarray(a)
    if a.dtype != dtype or not (a.flags.f_contiguous or a.ndim == 1):
        a = np.asfortranarray(a, dtype=dtype)
    return a


def hk_psi_c16(mtxd, neig, psi, hpsi, lnewanl, ng, kgv, ekpg, isort, vscr, kmscr, anlga, xnlkb, nanl,
               mxddim, mxdbnd, mxdanl, mxdgve, mxdscr):
    """hpsi(:mtxd, :neig) = H psi, as hk_psi_c16 (psi, hpsi: complex128 (mxddim, mxdbnd)).

    ``hpsi`` must be a Fortran-ordered complex128 array; it is written in place
    and also returned, with ``lnewanl`` as the library left it (the library only
    reads the flag: a set flag forces the projectors to be re-uploaded, and
    unchanged flags are checked against the projectors' content). Errors raise
    ``CpwB200Error`` (the reference stops the program).
    """
    L = _lib.lib()
    psi = _as_f(psi, np.complex128)
    if not (isinstance(hpsi, np.ndarray) and hpsi.dtype == np.complex128 and hpsi.flags.f_contiguous):
        raise TypeError("hpsi must be a Fortran-ordered complex128 numpy array (written in place)")
    if psi.shape[0] < mxddim or hpsi.shape[0] < mxddim:
        raise ValueError("psi/hpsi leading dimension smaller than mxddim")
    kgv = _as_f(kgv, np.int32)
    isort = _as_f(isort, np.int32)
    ekpg = _as_f(ekpg, np.float64)
    vscr = _as_f(vscr, np.float64)
    kmscr = _as_f(kmscr, np.int32)
    anlga = _as_f(anlga, np.complex128) if nanl > 0 else np.zeros((max(mxddim, 1), 1), np.complex128, order="F")
    xnlkb = _as_f(xnlkb, np.float64) if nanl > 0 else np.zeros(1)
    lnew = C.c_int(1 if lnewanl else 0)
    ri = _lib.iref
    st = L.cpw_b200_hk_psi_c16(ri(mtxd), ri(neig), zptr(psi), zptr(hpsi),
                               C.byref(lnew), ri(ng), iptr(kgv), dptr(ekpg), iptr(isort), dptr(vscr), iptr(kmscr),
                               zptr(anlga), dptr(xnlkb), ri(nanl), ri(mxddim), ri(mxdbnd),
                               ri(mxdanl), ri(mxdgve), ri(mxdscr))
    check(st)
    return hpsi, bool(lnew.value)


def hk_psi_nl_c16(mtxd, neig, psi, hpsi, anlga, xnlkb, nanl, ladd, mxddim, mxdbnd, mxdanl):
    """hpsi = [hpsi if ladd] + anlga diag(xnlkb) anlga^H psi, as hk_psi_nl_c16 (in place)."""
    L = _lib.lib()
    psi = _as_f(psi, np.complex128)
    if not (isinstance(hpsi, np.ndarray) and hpsi.dtype == np.complex128 and hpsi.flags.f_contiguous):
        raise TypeError("hpsi must be a Fortran-ordered complex128 numpy array (updated in place)")
    anlga = _as_f(anlga, np.complex128) if nanl > 0 else np.zeros((max(mxddim, 1), 1), np.complex128, order="F")
    xnlkb = _as_f(xnlkb, np.float64) if nanl > 0 else np.zeros(1)
    ri = _lib.iref
    check(L.cpw_b200_hk_psi_nl_c16(ri(mtxd), ri(neig), zptr(psi), zptr(hpsi),
                                   zptr(anlga), dptr(xnlkb), ri(nanl), ri(1 if ladd else 0),
                                   ri(mxddim), ri(mxdbnd), ri(mxdanl)))
    return hpsi


def _kb_arrays(rkpt, species, vkb, nkb, adot, delq, nq):
    """The arguments of proj_nl_kb_c16 / proj_nl_kb_der_c16 in the reference layouts: natom(ntype),
    rat(3, mxdatm, ntype), vkb(-2:nq, 0:3, -1:1, ntype) and nkb(0:3, -1:1, ntype) (spin-orbit
    channel 0 filled), nanl, an xnlkb buffer, rkpt, adot, nqnl(ntype), delqnl(ntype)."""
    ntype = len(species)
    natom = np.array([sp.natom for sp in species], dtype=np.int32)
    mxdatm = max(1, int(natom.max()) if ntype else 1)
    rat = np.zeros((3, mxdatm, max(ntype, 1)), order="F")
    for t, sp in enumerate(species):
        if sp.natom:
            rat[:, :sp.natom, t] = np.asarray(sp.rat, dtype=np.float64).T
    vkb = np.asarray(vkb, dtype=np.float64)
    vref = np.zeros((nq + 3, 4, 3, max(ntype, 1)), order="F")
    nref = np.zeros((4, 3, max(ntype, 1)), dtype=np.int32, order="F")
    for t in range(ntype):
        for l in range(4):
            vref[:, l, 1, t] = vkb[t, l, :nq + 3]
            nref[l, 1, t] = int(nkb[t, l])
    nanl = pseudo.nanl_of(species, np.asarray(nkb))
    xnl = np.zeros(max(nanl, 1))
    rk = np.ascontiguousarray(rkpt, dtype=np.float64)
    ad = np.asfortranarray(adot, dtype=np.float64)
    nqa = np.full(max(ntype, 1), nq, dtype=np.int32)
    dqa = np.full(max(ntype, 1), delq, dtype=np.float64)
    return ntype, natom, rat, mxdatm, vref, nref, nanl, xnl, rk, ad, nqa, dqa


class Context:
    """One k-point's device state; H|psi> on device-resident complex128 torch tensors."""

    def __init__(self, device: int = 0, precision: int = FP64):
        self._L = _lib.lib()
        h = C.c_void_p()
        check(self._L.cpw_b200_create(C.byref(h), int(device)))
        self.handle = h
        self.device = device
        self.mtxd = 0
        self.nanl = 0
        if precision != FP64:
            self.set_precision(precision)

    def close(self):
        if self.handle:
            self._L.cpw_b200_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream_ptr(self) -> int:
        return int(self._L.cpw_b200_stream(self.handle) or 0)

    def set_precision(self, mode: int):
        check(self._L.cpw_b200_set_precision(self.handle, int(mode)))

    def synchronize(self):
        """Wait for the device; raises if a bounded device-side wait gave up."""
        check(self._L.cpw_b200_synchronize(self.handle))

    def set_wait_limits(self, mbarrier_ns: int = -1, grid_polls: int = -1):
        """Limits of the bounded device waits (negative: the defaults, 2 s and 2^24 polls)."""
        check(self._L.cpw_b200_set_wait_limits(self.handle, int(mbarrier_ns), int(grid_polls)))

    def set_projector_slices(self, slices: int):
        """Projector products on the int8 tensor cores with that many slices (0: the form's default)."""
        check(self._L.cpw_b200_set_projector_slices(self.handle, int(slices)))

    def set_slab_budget(self, nbytes: int):
        check(self._L.cpw_b200_set_slab_budget(self.handle, int(nbytes)))

    STAGES = ("inv_xy", "z_vloc", "fwd_xy", "nl_proj", "nl_expand", "eig", "s6", "s7")

    def timing_begin(self):
        check(self._L.cpw_b200_timing_begin(self.handle))

    def timing_end(self) -> dict:
        """Per-stage {name: (total_ms, launches)} since timing_begin (synchronises)."""
        ms = (C.c_double * 8)()
        nl = (C.c_longlong * 8)()
        check(self._L.cpw_b200_timing_end(self.handle, ms, nl, 8))
        return {n: (float(ms[i]), int(nl[i])) for i, n in enumerate(self.STAGES)}

    def set_kpoint(self, mtxd, isort, kgv, ekpg, kmscr):
        isort = np.ascontiguousarray(isort, dtype=np.int32)
        kgv = np.asfortranarray(kgv, dtype=np.int32)
        ekpg = np.ascontiguousarray(ekpg, dtype=np.float64)
        kmscr = np.ascontiguousarray(kmscr, dtype=np.int32)
        check(self._L.cpw_b200_set_kpoint(self.handle, int(mtxd), iptr(isort), iptr(kgv), int(kgv.shape[1]),
                                          dptr(ekpg), iptr(kmscr)))
        self.mtxd = int(mtxd)

    def set_potential(self, vscr):
        v = np.ascontiguousarray(vscr, dtype=np.float64)
        check(self._L.cpw_b200_set_potential(self.handle, dptr(v), int(v.size)))

    def set_projectors(self, anlga, xnlkb):
        a = np.asfortranarray(anlga, dtype=np.complex128)
        x = np.ascontiguousarray(xnlkb, dtype=np.float64)
        nanl = int(x.size)
        if nanl == 0:
            a = np.zeros((max(self.mtxd, 1), 1), np.complex128, order="F")
            x = np.zeros(1)
        check(self._L.cpw_b200_set_projectors(self.handle, nanl, zptr(a), int(a.shape[0]),
                                              dptr(x)))
        self.nanl = nanl

    def proj_nl_kb(self, rkpt, species, vkb, nkb, adot, delq: float = 0.01, nq: int = 4000, anlga_out=None):
        """Build the KB projectors of the current k-point on the device and install them
        (cpw_b200_proj_nl_kb_device, the device form of Src/omp/proj_nl_kb_c16.f90).

        species: list of pseudo.Species (natom, rat); vkb[ntype, 4, nq+3] and nkb[ntype, 4] as
        returned by pseudo.kb_tables; adot the real-space metric. The tables are passed in the
        reference layouts vkb(-2:nq, 0:3, -1:1, ntype) and nkb(0:3, -1:1, ntype) (spin-orbit
        channel 0). anlga_out: optional complex128 CUDA tensor (mtxd, nanl) column-major that
        receives a copy. Returns xnlkb (numpy)."""
        ntype, natom, rat, mxdatm, vref, nref, nanl, xnl, rk, ad, nqa, dqa = _kb_arrays(rkpt, species, vkb, nkb, adot,
                                                                                    delq, nq)
        out_ptr, ld = None, 0
        if anlga_out is not None:
            if anlga_out.stride(0) != 1:
                raise ValueError("anlga_out must be column-major")
            out_ptr = C.c_void_p(anlga_out.data_ptr())
            ld = int(anlga_out.stride(1)) if anlga_out.shape[1] > 1 else self.mtxd
        check(self._L.cpw_b200_proj_nl_kb_device(self.handle, dptr(rk), ntype, iptr(natom), dptr(rat), mxdatm,
                                                 dptr(ad), iptr(nqa), dptr(dqa), dptr(vref), nq, iptr(nref), nanl,
                                                 dptr(xnl), out_ptr, ld))
        self.nanl = nanl
        return xnl[:nanl]

    def proj_nl_kb_der(self, rkpt, species, vkb, nkb, adot, nder: int = 2, delq: float = 0.01, nq: int = 4000):
        """Projectors of the current k-point and their derivatives with respect to the k-point's
        lattice coordinates on the device (cpw_b200_proj_nl_kb_der_device, the device form of
        Src/omp/proj_nl_kb_der_c16.f90). Returns (anlga (mtxd, nanl), danlgadrk (mtxd, nanl, 3) or
        None, d2anlgadrk2 (mtxd, nanl, 3, 3) or None) as complex128 CUDA tensors in the reference
        layouts (Fortran order), and xnlkb (numpy). The context's projectors are not changed."""
        import torch
        ntype, natom, rat, mxdatm, vref, nref, nanl, xnl, rk, ad, nqa, dqa = _kb_arrays(rkpt, species, vkb, nkb, adot,
                                                                                    delq, nq)
        m = self.mtxd
        dev = torch.device("cuda", self.device)
        # Fortran-order buffers: a flat tensor viewed with the reference's strides
        a = torch.zeros(max(m * nanl, 1), dtype=torch.complex128, device=dev)
        da = torch.zeros(max(m * nanl * 3, 1) if nder > 0 else 1, dtype=torch.complex128, device=dev)
        d2a = torch.zeros(max(m * nanl * 9, 1) if nder > 1 else 1, dtype=torch.complex128, device=dev)
        check(self._L.cpw_b200_proj_nl_kb_der_device(
            self.handle, int(nder), dptr(rk), ntype, iptr(natom), dptr(rat), mxdatm, dptr(ad), iptr(nqa), dptr(dqa),
            dptr(vref), nq, iptr(nref), nanl, dptr(xnl), C.c_void_p(a.data_ptr()), max(m, 1), max(nanl, 1),
            C.c_void_p(da.data_ptr()) if nder > 0 else None, C.c_void_p(d2a.data_ptr()) if nder > 1 else None))
        torch.cuda.synchronize(dev)
        A = a[: m * nanl].as_strided((m, nanl), (1, m))
        DA = da[: m * nanl * 3].as_strided((m, nanl, 3), (1, m, m * nanl)) if nder > 0 else None
        D2A = d2a[: m * nanl * 9].as_strided((m, nanl, 3, 3), (1, m, m * nanl, 3 * m * nanl)) if nder > 1 else None
        return A, DA, D2A, xnl[:nanl]

    def pot_local(self, veff, kgv, inds, phase=None, conj=None, kmscr=(0, 0, 0), idshift: int = 0,
                  install: bool = True, want_vscr: bool = True):
        """Screened potential on the mesh from its values per star (cpw_b200_pot_local, the
        device form of Src/cpw_lib/pot_local.f90). veff (ns,) complex; kgv (3, ng) int;
        inds (ng,) 1-based stars; phase (ng,) complex (default 1); conj (ng,) +-1 (default +1);
        kmscr(1:3) the extent of G on the mesh. install: also make it this context's potential.
        Returns dict(vscr, vmax, vmin, cmax, kmscr)."""
        veff = np.ascontiguousarray(veff, dtype=np.complex128)
        kgv = np.asfortranarray(kgv, dtype=np.int32)
        ng = int(kgv.shape[1])
        inds = np.ascontiguousarray(inds, dtype=np.int32)
        phase = np.ones(ng, np.complex128) if phase is None else np.ascontiguousarray(phase, dtype=np.complex128)
        conj = np.ones(ng) if conj is None else np.ascontiguousarray(conj, dtype=np.float64)
        km = np.zeros(7, dtype=np.int32)
        km[:3] = np.asarray(kmscr, dtype=np.int32)[:3]
        ns = int(veff.size)
        # the mesh is size_fft(kmscr); the library checks it and sets kmscr(4:7)
        n1, n2, n3 = crystal.size_fft(km[:3])
        mxdscr = max((n1 + idshift) * n2 * n3, 4 * max(n1 * n2, n1 * n3, n2 * n3))
        vscr = np.zeros(mxdscr) if want_vscr else None
        vmax, vmin, cmax = C.c_double(), C.c_double(), C.c_double()
        check(self._L.cpw_b200_pot_local(self.handle, dptr(vscr) if want_vscr else None, C.byref(vmax),
                                         C.byref(vmin), C.byref(cmax), zptr(veff), iptr(km), int(idshift), ng,
                                         iptr(kgv), zptr(phase), dptr(conj), ns, iptr(inds), mxdscr, ng,
                                         max(ns, 1), 1 if install else 0))
        n1, n2, n3, ident = (int(x) for x in km[3:7])
        return dict(vscr=vscr[:ident * n2 * n3] if want_vscr else None, vmax=vmax.value, vmin=vmin.value,
                    cmax=cmax.value, kmscr=km)

    def hk_psi_kin(self, psi, hpsi, ladd: bool = False, nspin: int = 1):
        """hpsi (+)= ekpg psi (Src/omp/hk_psi_kin_c16.f90) on column-major CUDA tensors."""
        check(self._L.cpw_b200_hk_psi_kin_device(self.handle, int(psi.shape[1]), C.c_void_p(psi.data_ptr()),
                                                 self._ld(psi), C.c_void_p(hpsi.data_ptr()), self._ld(hpsi),
                                                 1 if ladd else 0, int(nspin),
                                                 C.c_void_p(torch_stream_handle(psi.device))))

    def hk_psi_loc(self, psi, hpsi, ladd: bool = False, nspin: int = 1):
        """hpsi (+)= V_loc psi (Src/omp/hk_psi_loc_c16.f90), nspin 1 or 2 (interleaved spinors)."""
        check(self._L.cpw_b200_hk_psi_loc_c16_device(self.handle, int(psi.shape[1]), C.c_void_p(psi.data_ptr()),
                                                     self._ld(psi), C.c_void_p(hpsi.data_ptr()), self._ld(hpsi),
                                                     1 if ladd else 0, int(nspin),
                                                     C.c_void_p(torch_stream_handle(psi.device))))

    def set_potential_spin(self, vscr_sp, nsp: int):
        """vscr_sp: (mxdscr, nsp) real, columns (1, sigma_z, sigma_x, sigma_y) of the box."""
        v = np.asfortranarray(vscr_sp, dtype=np.float64)
        check(self._L.cpw_b200_set_potential_spin(self.handle, dptr(v), int(v.shape[0]), int(nsp)))

    def set_projectors_spin(self, anlsp, xnlkbsp):
        """Spinor KB projectors anlsp (2*mtxd, nanlsp) complex128 and xnlkbsp (nanlsp,)."""
        a = np.asfortranarray(anlsp, dtype=np.complex128)
        x = np.ascontiguousarray(xnlkbsp, dtype=np.float64)
        if x.size == 0:
            a = np.zeros((max(2 * self.mtxd, 1), 1), np.complex128, order="F")
            x = np.zeros(1)
            n = 0
        else:
            n = int(x.size)
        check(self._L.cpw_b200_set_projectors_spin(self.handle, n, zptr(a), int(a.shape[0]), dptr(x)))

    def hk_psi_spin(self, psi_sp, hpsi_sp):
        """hpsi_sp = H psi_sp for column-major complex128 CUDA tensors (2*mtxd, nb), rows
        interleaved (up, down) per plane wave, on torch's current stream."""
        check(self._L.cpw_b200_hk_psi_spin_device(self.handle, int(psi_sp.shape[1]), C.c_void_p(psi_sp.data_ptr()),
                                                  self._ld(psi_sp), C.c_void_p(hpsi_sp.data_ptr()),
                                                  self._ld(hpsi_sp), C.c_void_p(torch_stream_handle(psi_sp.device))))

    def setup(self, inputs: dict):
        """Upload one k-point from a dict as returned by configs.kpoint_inputs."""
        self.set_kpoint(inputs["mtxd"], inputs["isort"], inputs["kgv"], inputs["ekpg"], inputs["kmscr"])
        self.set_potential(inputs["vscr"])
        self.set_projectors(inputs["anlga"], inputs["xnlkb"])
        return self

    @staticmethod
    def _ld(t) -> int:
        # column-major (mtxd, nb) stored as torch (nb, ld) row-major or a Fortran view
        if t.dim() != 2:
            raise ValueError("expected a 2-D complex128 tensor")
        if t.stride(0) == 1:
            return int(t.stride(1))
        raise ValueError("tensor must be column-major (use .t() of a contiguous (nb, ld) tensor)")

    def hk_psi(self, psi, hpsi, neig=None, stream=None, local_only=False):
        """hpsi[:, :neig] = H psi[:, :neig] for column-major complex128 CUDA tensors (mtxd rows)."""
        import torch
        if psi.dtype != torch.complex128 or hpsi.dtype != torch.complex128:
            raise TypeError("psi/hpsi must be complex128")
        if not (psi.is_cuda and hpsi.is_cuda):
            raise TypeError("psi/hpsi must be CUDA tensors")
        nb = psi.shape[1] if neig is None else int(neig)
        s = stream if stream is not None else torch_stream_handle(psi.device)
        fn = self._L.cpw_b200_hk_psi_loc_device if local_only else self._L.cpw_b200_hk_psi_device
        check(fn(self.handle, nb, C.c_void_p(psi.data_ptr()), self._ld(psi), C.c_void_p(hpsi.data_ptr()),
                 self._ld(hpsi), C.c_void_p(s)))
        return hpsi


def torch_stream_handle(device=None) -> int:
    """cudaStream_t of torch's current stream; the legacy default stream (handle 0)
    is passed as cudaStreamLegacy, because a null stream means "the context's
    own stream" to the C ABI."""
    import torch
    h = int(torch.cuda.current_stream(device).cuda_stream)
    return h if h != 0 else CUDA_STREAM_LEGACY


CUDA_STREAM_LEGACY = 0x1


def colmajor(t):
    """A (rows, cols) column-major view of a contiguous (cols, rows) tensor."""
    return t.t()
