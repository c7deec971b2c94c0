"""GPU H|psi> of two-component spinors (hk_psi_spin_c16) against the CPU restatement.

Every potential form (nsp = 1: one potential on both components; 2: V1 +- V2; 4: the 2x2
matrix [[V1+V2, V3-iV4], [V3+iV4, V1-V2]] coupling the components), FP64 within 1e-12 and the
FP32 local part within 2e-5 of max|H psi|, through the device API and through the drop-in with
the reference's leading dimensions, k-points off Gamma included.
"""
import ctypes as C

import numpy as np
import pytest

from cpw2000_b200 import configs
from cpw2000_b200 import hk_psi as H
from cpw2000_b200._lib import CpwB200Error, check, dptr, iptr, iref, lib, zptr
from oracle import hk_psi as O

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-5


def relerr(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def spin_inputs(wname, ik, nsp, nanl=6, seed=0):
    w = configs.WORKLOADS[wname]()
    d = configs.kpoint_inputs(w, ik)
    rng = np.random.default_rng(seed)
    nv = d["vscr"].size
    vsp = np.zeros((nv, nsp), order="F")
    vsp[:, 0] = d["vscr"]
    for j in range(1, nsp):
        vsp[:, j] = 0.3 * rng.standard_normal(nv)
    m = d["mtxd"]
    anl = (rng.standard_normal((2 * m, nanl)) + 1j * rng.standard_normal((2 * m, nanl))) / np.sqrt(m)
    xnl = np.where(rng.random(nanl) < 0.5, -1.0, 1.0)
    return d, vsp, np.asfortranarray(anl), xnl


def oracle(d, psi, nb, vsp, nsp, anl, xnl):
    return O.hk_psi_spin_c16(d["mtxd"], nb, psi, d["ekpg"], d["isort"], vsp, d["kmscr"], d["kgv"], nsp, anl, xnl)


@pytest.mark.parametrize("nsp", [1, 2, 4])
@pytest.mark.parametrize("prec,tol", [(H.FP64, TOL64), (H.MIXED, TOL32)])
@pytest.mark.parametrize("wname,ik,nb", [("si2", 0, 5), ("si2", 3, 3)])
def test_device_spin_matches_oracle(cuda, nsp, prec, tol, wname, ik, nb):
    import torch
    d, vsp, anl, xnl = spin_inputs(wname, ik, nsp, seed=nsp)
    m = d["mtxd"]
    rng = np.random.default_rng(10 + nsp)
    psi = (rng.standard_normal((2 * m, nb)) + 1j * rng.standard_normal((2 * m, nb)))
    ctx = H.Context(0, precision=prec)
    ctx.set_kpoint(m, d["isort"], d["kgv"], d["ekpg"], d["kmscr"])
    ctx.set_potential_spin(vsp, nsp)
    ctx.set_projectors_spin(anl, xnl)
    x = torch.from_numpy(np.ascontiguousarray(psi.T)).to(cuda).t()
    y = torch.zeros((nb, 2 * m), dtype=torch.complex128, device=cuda).t()
    ctx.hk_psi_spin(x, y)
    torch.cuda.synchronize()
    assert relerr(y.cpu().numpy(), oracle(d, psi, nb, vsp, nsp, anl, xnl)) < tol


@pytest.mark.parametrize("nsp", [2, 4])
def test_dropin_spin_with_leading_dimensions(cuda, nsp):
    d, vsp, anl, xnl = spin_inputs("si2", 1, nsp, seed=7)
    m, nb = d["mtxd"], 4
    mxddim, mxdbnd, mxdasp = m + 5, nb + 2, xnl.size + 1
    rng = np.random.default_rng(3)
    psi = np.zeros((2 * mxddim, mxdbnd), np.complex128, order="F")
    psi[:2 * m, :nb] = rng.standard_normal((2 * m, nb)) + 1j * rng.standard_normal((2 * m, nb))
    hpsi = np.zeros_like(psi)
    anlp = np.zeros((2 * mxddim, mxdasp), np.complex128, order="F")
    anlp[:2 * m, :xnl.size] = anl
    xnlp = np.zeros(mxdasp)
    xnlp[:xnl.size] = xnl
    mxdscr = vsp.shape[0]
    kgv = np.asfortranarray(d["kgv"], dtype=np.int32)
    isort = np.ascontiguousarray(d["isort"], dtype=np.int32)
    kmscr = np.ascontiguousarray(d["kmscr"], dtype=np.int32)
    ekpg = np.ascontiguousarray(d["ekpg"])
    L = lib()
    want = oracle(d, psi, nb, vsp, nsp, anl, xnl)
    for call in range(2):      # the second call reuses the cached k-point, potential and projectors
        lnew = C.c_int(1 if call == 0 else 0)
        check(L.cpw_b200_hk_psi_spin_c16(iref(m), iref(nb), zptr(psi), zptr(hpsi), C.byref(lnew), iref(d["ng"]),
                                         iptr(kgv), dptr(ekpg), iptr(isort), dptr(vsp), iptr(kmscr), iref(nsp),
                                         zptr(anlp), dptr(xnlp), iref(xnl.size), iref(mxddim), iref(mxdbnd),
                                         iref(mxdasp), iref(d["ng"]), iref(mxdscr), iref(4)))
        assert lnew.value == (1 if call == 0 else 0)      # the library never writes lnewanl
        assert relerr(hpsi[:2 * m, :nb], want) < TOL64
    # projectors changed without the flag: picked up by the content check
    anlp2 = np.asfortranarray(anlp * 0.5)
    want2 = oracle(d, psi, nb, vsp, nsp, anl * 0.5, xnl)
    lnew = C.c_int(0)
    check(L.cpw_b200_hk_psi_spin_c16(iref(m), iref(nb), zptr(psi), zptr(hpsi), C.byref(lnew), iref(d["ng"]),
                                     iptr(kgv), dptr(ekpg), iptr(isort), dptr(vsp), iptr(kmscr), iref(nsp),
                                     zptr(anlp2), dptr(xnlp), iref(xnl.size), iref(mxddim), iref(mxdbnd),
                                     iref(mxdasp), iref(d["ng"]), iref(mxdscr), iref(4)))
    assert relerr(hpsi[:2 * m, :nb], want2) < TOL64


def test_dropin_spin_rejects_bad_nsp(cuda):
    d, vsp, anl, xnl = spin_inputs("si2", 0, 1)
    m = d["mtxd"]
    psi = np.zeros((2 * m, 1), np.complex128, order="F")
    L = lib()
    lnew = C.c_int(1)
    with pytest.raises(CpwB200Error, match="nsp"):
        check(L.cpw_b200_hk_psi_spin_c16(iref(m), iref(1), zptr(psi), zptr(psi), C.byref(lnew), iref(d["ng"]),
                                         iptr(np.asfortranarray(d["kgv"], dtype=np.int32)),
                                         dptr(np.ascontiguousarray(d["ekpg"])),
                                         iptr(np.ascontiguousarray(d["isort"], dtype=np.int32)), dptr(vsp),
                                         iptr(np.ascontiguousarray(d["kmscr"], dtype=np.int32)), iref(3), zptr(anl),
                                         dptr(xnl), iref(xnl.size), iref(m), iref(1), iref(xnl.size), iref(d["ng"]),
                                         iref(vsp.shape[0]), iref(4)))


@pytest.mark.parametrize("nspin", [1, 2])
@pytest.mark.parametrize("ladd", [False, True])
def test_split_kinetic_and_local_operators(cuda, nspin, ladd):
    # hk_psi_kin_c16 and hk_psi_loc_c16 on device blocks: T psi and V_loc psi, added or stored
    import torch
    nsp = 2 if nspin == 2 else 1
    d, vsp, anl, xnl = spin_inputs("si2", 2, nsp, seed=11)
    m, nb = d["mtxd"], 3
    rows = nspin * m
    rng = np.random.default_rng(4)
    psi = rng.standard_normal((rows, nb)) + 1j * rng.standard_normal((rows, nb))
    h0 = rng.standard_normal((rows, nb)) + 1j * rng.standard_normal((rows, nb))
    ctx = H.Context(0)
    ctx.set_kpoint(m, d["isort"], d["kgv"], d["ekpg"], d["kmscr"])
    ctx.set_potential(d["vscr"])
    ctx.set_potential_spin(vsp, nsp)
    x = torch.from_numpy(np.ascontiguousarray(psi.T)).to(cuda).t()
    base = h0 if ladd else np.zeros_like(h0)
    ek = np.repeat(np.asarray(d["ekpg"][:m]), nspin)
    want_kin = base + ek[:, None] * psi
    none = np.zeros((rows, 0), complex)
    if nspin == 1:
        want_loc = base + O.hk_psi_loc(m, nb, psi, d["isort"], d["vscr"], d["kmscr"], d["kgv"])
    else:
        want_loc = base + O.hk_psi_spin_c16(m, nb, psi, np.zeros(m), d["isort"], vsp, d["kmscr"], d["kgv"], nsp,
                                            none, np.zeros(0))
    for op, want in ((ctx.hk_psi_kin, want_kin), (ctx.hk_psi_loc, want_loc)):
        y = torch.from_numpy(np.ascontiguousarray(h0.T)).to(cuda).t()
        op(x, y, ladd=ladd, nspin=nspin)
        torch.cuda.synchronize()
        assert relerr(y.cpu().numpy(), want) < TOL64


@pytest.mark.parametrize("nsp", [2, 4])
def test_device_spin_box96(cuda, nsp):
    # the compile-time 96^3 kernels on the component views (nsp 2) and the spinor z stage (nsp 4)
    import torch
    d, vsp, anl, xnl = spin_inputs("si64", 0, nsp, nanl=8, seed=20 + nsp)
    m, nb = d["mtxd"], 3
    rng = np.random.default_rng(30 + nsp)
    psi = rng.standard_normal((2 * m, nb)) + 1j * rng.standard_normal((2 * m, nb))
    ctx = H.Context(0)
    ctx.set_kpoint(m, d["isort"], d["kgv"], d["ekpg"], d["kmscr"])
    ctx.set_potential_spin(vsp, nsp)
    ctx.set_projectors_spin(anl, xnl)
    x = torch.from_numpy(np.ascontiguousarray(psi.T)).to(cuda).t()
    y = torch.zeros((nb, 2 * m), dtype=torch.complex128, device=cuda).t()
    ctx.hk_psi_spin(x, y)
    torch.cuda.synchronize()
    assert relerr(y.cpu().numpy(), oracle(d, psi, nb, vsp, nsp, anl, xnl)) < TOL64
