"""GPU test of the allocation-free local H|psi> entry point (collected last).

cpw_b200_hk_psi_loc_noalloc serves callers that cannot call cudaMalloc (a
caller-owned pool or fixed device budget, host codes that own every device
buffer): it takes only caller-owned device buffers and keeps its work space
in a fixed device array of the library. This test calls it through the C ABI
twice in a row, on two different k-points (different boxes and basis sizes,
so the shared array is reused with new contents), the second time with the
kinetic diagonal ekpg, and checks each result against the existing entry
points (cpw_b200_hk_psi_loc_device, plus cpw_b200_hk_psi_kin_device for the
kinetic term) and against the oracle's local (+ kinetic) operator, within the
FP64 tolerance of the other H|psi> tests. It runs alone or after the others.
"""
import ctypes as C

import numpy as np
import pytest

from cpw2000_b200 import _lib, configs
from cpw2000_b200 import hk_psi as H
from oracle import hk_psi as O

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


def _case(torch, dev, wname, ik, nb, seed):
    w = configs.WORKLOADS[wname]()
    d = configs.kpoint_inputs(w, ik)
    m = d["mtxd"]
    psi_h = configs.random_psi(m, nb, seed)
    psi = torch.from_numpy(np.ascontiguousarray(psi_h.T)).to(dev).t()
    kgvb = torch.from_numpy(np.ascontiguousarray(d["kgv"][:, d["isort"] - 1].T)).to(dev)   # (mtxd, 3) = kgvb(3, mtxd)
    vscr = torch.from_numpy(np.ascontiguousarray(d["vscr"])).to(dev)
    return d, psi, kgvb, vscr


def _existing(d, psi, torch, dev, kinetic):
    ctx = H.Context(0).setup(d)
    out = torch.zeros((psi.shape[1], psi.shape[0]), dtype=torch.complex128, device=dev).t()
    ctx.hk_psi(psi, out, local_only=True)
    if kinetic:
        ctx.hk_psi_kin(psi, out, ladd=True)
    torch.cuda.synchronize()
    res = out.cpu().numpy()
    ctx.close()
    return res


def _noalloc(d, psi, kgvb, vscr, ekpg, torch, dev):
    L = _lib.lib()
    m, nb = psi.shape
    out = torch.full((nb, m), complex(3.0, -3.0), dtype=torch.complex128, device=dev).t()
    kmscr = np.ascontiguousarray(d["kmscr"], dtype=np.int32)
    stream = H.torch_stream_handle(dev)
    st = L.cpw_b200_hk_psi_loc_noalloc(m, nb, C.c_void_p(psi.data_ptr()), int(psi.stride(1)),
                                       C.c_void_p(out.data_ptr()), int(out.stride(1)), C.c_void_p(kgvb.data_ptr()),
                                       C.c_void_p(ekpg.data_ptr()) if ekpg is not None else None,
                                       C.c_void_p(vscr.data_ptr()), _lib.iptr(kmscr), C.c_void_p(stream))
    _lib.check(st)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _oracle(d, psi_h, kinetic):
    m, nb = psi_h.shape
    ref = O.hk_psi_loc(m, nb, psi_h, d["isort"], d["vscr"], d["kmscr"], d["kgv"])
    if kinetic:
        ref = ref + np.asarray(d["ekpg"])[:m, None] * psi_h
    return ref


def test_noalloc_matches_existing_entry_point_on_two_calls(cuda):
    import torch
    # a 32^3 box without the kinetic term, then a 24x20x18 box with id = 25 and ekpg
    cases = [("si2", 2, 7, 31, False), ("small", 1, 5, 32, True)]
    for wname, ik, nb, seed, kinetic in cases:
        d, psi, kgvb, vscr = _case(torch, cuda, wname, ik, nb, seed)
        ekpg = torch.from_numpy(np.ascontiguousarray(d["ekpg"], dtype=np.float64)).to(cuda) if kinetic else None
        ref = _existing(d, psi, torch, cuda, kinetic)
        got = _noalloc(d, psi, kgvb, vscr, ekpg, torch, cuda)
        err = float(np.abs(got - ref).max() / np.abs(ref).max())
        assert err < TOL64, f"{wname} k{ik}: relative difference {err:.3e} to the existing entry point"
        want = _oracle(d, psi.cpu().numpy(), kinetic)
        err = float(np.abs(got - want).max() / np.abs(want).max())
        assert err < TOL64, f"{wname} k{ik}: relative difference {err:.3e} to the oracle"


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    import torch
    d, psi, kgvb, vscr = _case(torch, cuda, "si2", 0, 1, 3)
    km = np.ascontiguousarray(d["kmscr"], dtype=np.int32).copy()
    km[3:7] = (256, 256, 160, 256)            # the repacked potential alone (84 MB) exceeds the array
    L = _lib.lib()
    out = torch.zeros((1, d["mtxd"]), dtype=torch.complex128, device=cuda).t()
    st = L.cpw_b200_hk_psi_loc_noalloc(d["mtxd"], 1, C.c_void_p(psi.data_ptr()), int(psi.stride(1)),
                                       C.c_void_p(out.data_ptr()), int(out.stride(1)), C.c_void_p(kgvb.data_ptr()),
                                       None, C.c_void_p(vscr.data_ptr()), _lib.iptr(km), None)
    assert st == 1
    assert "maximum" in L.cpw_b200_last_error().decode()
