"""GPU parity of H|psi> (C ABI -> sm_100a kernels) against the CPU oracle.

FP64 path: relative error <= 1e-12 of max|H psi| (rounding only; the GPU
pruned FFT and numpy's FFT differ in operation order). Mixed path (FP32
FFT/V_loc): relative error <= 2e-5.
"""
import numpy as np
import pytest

from cpw2000_b200 import configs
from cpw2000_b200 import hk_psi as H
from cpw2000_b200._lib import CpwB200Error
from oracle import hk_psi as O

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-5


def oracle_hpsi(d, psi, nb):
    return O.hk_psi_c16(d["mtxd"], nb, psi, d["ekpg"], d["isort"], d["vscr"], d["kmscr"], d["kgv"], d["anlga"],
                        d["xnlkb"])


def to_dev(a, torch, dev):
    # column-major complex128 (rows, cols) on the device
    return torch.from_numpy(np.ascontiguousarray(a.T)).to(dev).t()


def run_device(ctx, psi, torch, dev, local_only=False):
    m, nb = psi.shape
    x = to_dev(psi, torch, dev)
    y = torch.zeros((nb, m), dtype=torch.complex128, device=dev).t()
    ctx.hk_psi(x, y, local_only=local_only)
    torch.cuda.synchronize()
    return y.cpu().numpy()


def relerr(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("wname,ik,nb", [("small", 0, 3), ("small", 1, 6), ("si2", 0, 8), ("si2", 3, 5),
                                         ("si2", 9, 1)])
def test_device_fp64_matches_oracle(cuda, wname, ik, nb):
    import torch
    w = configs.WORKLOADS[wname]()
    d = configs.kpoint_inputs(w, ik)
    ctx = H.Context(0).setup(d)
    psi = configs.random_psi(d["mtxd"], nb, 100 + ik)
    got = run_device(ctx, psi, torch, cuda)
    assert relerr(got, oracle_hpsi(d, psi, nb)) < TOL64


def test_device_fp64_si64_box96(cuda):
    import torch
    w = configs.si64_cubic()
    d = configs.kpoint_inputs(w, 0)
    ctx = H.Context(0).setup(d)
    psi = configs.random_psi(d["mtxd"], 6, 7)
    got = run_device(ctx, psi, torch, cuda)
    assert relerr(got, oracle_hpsi(d, psi, 6)) < TOL64


@pytest.mark.parametrize("prec,tol", [(0, TOL64), (1, TOL32), (2, TOL32)])
def test_device_box40_kpoint_batch_cell(cuda, prec, tol):
    import torch
    w = configs.si8_cubic_kbatch()
    d = configs.kpoint_inputs(w, 3)
    ctx = H.Context(0, precision=prec).setup(d)
    psi = configs.random_psi(d["mtxd"], 5, 13)
    got = run_device(ctx, psi, torch, cuda)
    assert relerr(got, oracle_hpsi(d, psi, 5)) < tol


@pytest.mark.parametrize("prec,tol", [(0, TOL64), (1, TOL32), (2, TOL32)])
def test_device_box144_si216(cuda, prec, tol):
    import torch
    w = configs.si216_cubic()
    d = configs.kpoint_inputs(w, 1)
    ctx = H.Context(0, precision=prec).setup(d)
    psi = configs.random_psi(d["mtxd"], 2, 17)
    got = run_device(ctx, psi, torch, cuda)
    assert relerr(got, oracle_hpsi(d, psi, 2)) < tol


def test_local_only_matches_oracle(cuda):
    import torch
    w = configs.si2_fcc()
    d = configs.kpoint_inputs(w, 2)
    ctx = H.Context(0).setup(d)
    psi = configs.random_psi(d["mtxd"], 4, 5)
    got = run_device(ctx, psi, torch, cuda, local_only=True)
    ref = O.hk_psi_loc(d["mtxd"], 4, psi, d["isort"], d["vscr"], d["kmscr"], d["kgv"])
    assert relerr(got, ref) < TOL64


def test_band_chunking_is_invisible(cuda):
    import torch
    w = configs.si2_fcc()
    d = configs.kpoint_inputs(w, 1)
    ctx = H.Context(0).setup(d)
    psi = configs.random_psi(d["mtxd"], 7, 9)
    a = run_device(ctx, psi, torch, cuda)
    ctx.set_slab_budget(1)          # one band per chunk
    b = run_device(ctx, psi, torch, cuda)
    assert np.array_equal(a, b)


def test_mixed_precision_local_within_fp32_tolerance(cuda):
    import torch
    w = configs.si2_fcc()
    d = configs.kpoint_inputs(w, 0)
    ctx = H.Context(0, precision=H.MIXED).setup(d)
    psi = configs.random_psi(d["mtxd"], 8, 3)
    got = run_device(ctx, psi, torch, cuda)
    assert relerr(got, oracle_hpsi(d, psi, 8)) < TOL32


def test_dropin_host_arrays_with_leading_dimensions(cuda):
    w = configs.small_test()
    d = configs.kpoint_inputs(w, 1)
    m, nb = d["mtxd"], 4
    mxddim, mxdbnd = m + 5, nb + 2
    psi = configs.random_psi(m, mxdbnd, 44, ld=mxddim)
    hpsi = np.full((mxddim, mxdbnd), 7.0 + 7.0j, dtype=np.complex128, order="F")
    anl = np.zeros((mxddim, d["nanl"] + 1), dtype=np.complex128, order="F")
    anl[:m, : d["nanl"]] = d["anlga"]
    xnl = np.zeros(d["nanl"] + 1)
    xnl[: d["nanl"]] = d["xnlkb"]
    kgv = np.asfortranarray(d["kgv"])
    out, lnew = H.hk_psi_c16(m, nb, psi, hpsi, True, d["ng"], kgv, d["ekpg"], d["isort"], d["vscr"], d["kmscr"],
                             anl, xnl, d["nanl"], mxddim, mxdbnd, d["nanl"] + 1, d["ng"], d["vscr"].size)
    assert lnew is True            # only read by the library
    ref = oracle_hpsi(d, psi[:m], nb)
    assert relerr(hpsi[:m, :nb], ref) < TOL64
    assert np.all(hpsi[m:, :] == 7.0 + 7.0j) and np.all(hpsi[:, nb:] == 7.0 + 7.0j)
    # a changed potential is picked up without any flag
    v2 = d["vscr"] * 0.5
    H.hk_psi_c16(m, nb, psi, hpsi, False, d["ng"], kgv, d["ekpg"], d["isort"], v2, d["kmscr"], anl, xnl,
                 d["nanl"], mxddim, mxdbnd, d["nanl"] + 1, d["ng"], v2.size)
    ref2 = O.hk_psi_c16(m, nb, psi[:m], d["ekpg"], d["isort"], v2, d["kmscr"], d["kgv"], d["anlga"], d["xnlkb"])
    assert relerr(hpsi[:m, :nb], ref2) < TOL64
    # and so are changed projectors without lnewanl, and a changed xnlkb alone
    anl2 = np.asfortranarray(anl * (0.75 - 0.25j))
    H.hk_psi_c16(m, nb, psi, hpsi, False, d["ng"], kgv, d["ekpg"], d["isort"], v2, d["kmscr"], anl2, xnl,
                 d["nanl"], mxddim, mxdbnd, d["nanl"] + 1, d["ng"], v2.size)
    ref3 = O.hk_psi_c16(m, nb, psi[:m], d["ekpg"], d["isort"], v2, d["kmscr"], d["kgv"], anl2[:m, : d["nanl"]],
                        d["xnlkb"])
    assert relerr(hpsi[:m, :nb], ref3) < TOL64
    xnl2 = xnl.copy()
    xnl2[0] = -xnl2[0]
    H.hk_psi_c16(m, nb, psi, hpsi, False, d["ng"], kgv, d["ekpg"], d["isort"], v2, d["kmscr"], anl2, xnl2,
                 d["nanl"], mxddim, mxdbnd, d["nanl"] + 1, d["ng"], v2.size)
    ref4 = O.hk_psi_c16(m, nb, psi[:m], d["ekpg"], d["isort"], v2, d["kmscr"], d["kgv"], anl2[:m, : d["nanl"]],
                        xnl2[: d["nanl"]])
    assert relerr(hpsi[:m, :nb], ref4) < TOL64
    # and so is another k-point
    d1 = configs.kpoint_inputs(w, 0)
    m1 = d1["mtxd"]
    psi1 = configs.random_psi(m1, nb, 45, ld=mxddim)
    anl1 = np.zeros((mxddim, d1["nanl"]), dtype=np.complex128, order="F")
    anl1[:m1] = d1["anlga"]
    H.hk_psi_c16(m1, nb, psi1, hpsi, True, d1["ng"], np.asfortranarray(d1["kgv"]), d1["ekpg"], d1["isort"],
                 d1["vscr"], d1["kmscr"], anl1, d1["xnlkb"], d1["nanl"], mxddim, mxdbnd, d1["nanl"], d1["ng"],
                 d1["vscr"].size)
    assert relerr(hpsi[:m1, :nb], oracle_hpsi(d1, psi1[:m1], nb)) < TOL64


@pytest.mark.parametrize("ladd", [True, False])
def test_dropin_nl_matches_oracle(cuda, ladd):
    w = configs.si2_fcc()
    d = configs.kpoint_inputs(w, 4)
    m, nb = d["mtxd"], 3
    psi = configs.random_psi(m, nb, 8)
    h0 = configs.random_psi(m, nb, 9)
    hpsi = np.asfortranarray(h0.copy())
    H.hk_psi_nl_c16(m, nb, psi, hpsi, d["anlga"], d["xnlkb"], d["nanl"], ladd, m, nb, d["nanl"])
    ref = O.hk_psi_nl_c16(psi, h0.copy(), d["anlga"], d["xnlkb"], ladd=ladd)
    assert relerr(hpsi, ref) < TOL64


@pytest.mark.parametrize("ladd", [True, False])
def test_dropin_nl_without_projectors_leaves_hpsi(cuda, ladd):
    # nanl = 0: hk_psi_nl_c16.f90:78-98 runs neither product, so hpsi keeps its input values even
    # when ladd is false (the zeroing lives in the skipped zgemm's beta)
    w = configs.si2_fcc()
    d = configs.kpoint_inputs(w, 4)
    m, nb = d["mtxd"], 3
    psi = configs.random_psi(m, nb, 8)
    h0 = configs.random_psi(m, nb, 9)
    hpsi = np.asfortranarray(h0.copy())
    H.hk_psi_nl_c16(m, nb, psi, hpsi, np.zeros((m, 0), np.complex128), np.zeros(0), 0, ladd, m, nb, 1)
    assert np.array_equal(hpsi, h0)
    ref = O.hk_psi_nl_c16(psi, h0.copy(), np.zeros((m, 0), np.complex128), np.zeros(0), ladd=ladd)
    assert np.array_equal(ref, h0)


def test_wraparound_box_is_rejected(cuda):
    w = configs.small_test()
    d = configs.kpoint_inputs(w, 0)
    ctx = H.Context(0)
    km = d["kmscr"].copy()
    km[3:7] = (6, 6, 6, 6)
    with pytest.raises(CpwB200Error) as e:
        ctx.set_kpoint(d["mtxd"], d["isort"], d["kgv"], d["ekpg"], km)
    assert e.value.status == 2


def test_unsupported_box_is_rejected(cuda):
    w = configs.small_test()
    d = configs.kpoint_inputs(w, 0)
    ctx = H.Context(0)
    km = d["kmscr"].copy()
    km[3:7] = (49, 49, 49, 49)      # 7 x 7: radix 7 is not supported
    with pytest.raises(CpwB200Error) as e:
        ctx.set_kpoint(d["mtxd"], d["isort"], d["kgv"], d["ekpg"], km)
    assert e.value.status == 3


def test_mixed_projector_products_on_tensor_cores(cuda):
    """Split-TF32 tcgen05 projector GEMMs (opt-in MIXED_TC form) against the FP64 cuBLAS path, Si64 (256 KB
    projectors, K = 53,058 reals split over CTAs): the non-local term agrees to 1.5e-6 of its size
    (FP32 accumulation in tensor memory; eigenvalue accuracy is checked in test_gpu_ditsp)."""
    import torch
    w = configs.si64_cubic()
    d = configs.kpoint_inputs(w, 0)
    nb = 160
    psi = torch.from_numpy(np.ascontiguousarray(configs.random_psi(d["mtxd"], nb, 3).T)).to(cuda).t()
    out = {}
    for prec in (H.FP64, H.MIXED_TC):
        ctx = H.Context(0, precision=prec).setup(d)
        full = torch.zeros((nb, d["mtxd"]), dtype=torch.complex128, device=cuda).t()
        loc = torch.zeros_like(full)
        ctx.hk_psi(psi, full)
        ctx.hk_psi(psi, loc, local_only=True)
        torch.cuda.synchronize()
        ctx.synchronize()
        kin = torch.from_numpy(d["ekpg"]).to(cuda)[:, None] * psi
        out[prec] = (full - loc - kin).cpu().numpy()       # the projector term
    ref = out[H.FP64]
    assert relerr(out[H.MIXED_TC], ref) < 1.5e-6


@pytest.mark.parametrize("wname,nb", [("si2_fcc", 3), ("small_test", 5), ("si8_cubic_kbatch", 17), ("si8_cubic_kbatch", 130)])
def test_mixed_tc_edge_shapes(cuda, wname, nb):
    """Tensor-core projector path on shapes with partial 128-row tiles, K not a multiple of 32
    (2 nanl = 16 and 64), band counts below 16 and just above 128: the projector term agrees with
    the FP64 path to 1e-7 of its size, the full H|psi> with the oracle to the FP32 tolerance."""
    import torch
    w = getattr(configs, wname)()
    d = configs.kpoint_inputs(w, 1 if wname == "si8_cubic_kbatch" else 0)
    psi = configs.random_psi(d["mtxd"], nb, 29)
    nl = {}
    for prec in (H.FP64, H.MIXED_TC):
        ctx = H.Context(0, precision=prec).setup(d)
        full = run_device(ctx, psi, torch, cuda)
        loc = run_device(ctx, psi, torch, cuda, local_only=True)
        ctx.synchronize()
        nl[prec] = full - loc
        if prec == H.MIXED_TC:
            assert relerr(full, oracle_hpsi(d, psi, nb)) < TOL32
    assert relerr(nl[H.MIXED_TC], nl[H.FP64]) < 1e-7


@pytest.mark.parametrize("pinned", [False, True])
def test_dropin_pipelined_band_chunks(cuda, pinned):
    """Drop-in hk_psi_c16 with 70 bands (five 16-band chunks, the last partial): the pipelined
    host transfers give the oracle's result; with page-locked host arrays the copies overlap."""
    import torch
    w = configs.si2_fcc()
    d = configs.kpoint_inputs(w, 2)
    m, nb = d["mtxd"], 70
    mxddim, mxdbnd = m + 3, nb + 1
    psi = configs.random_psi(m, mxdbnd, 71, ld=mxddim)
    hpsi = np.full((mxddim, mxdbnd), 5.0 - 5.0j, dtype=np.complex128, order="F")
    if pinned:
        tp = torch.from_numpy(psi.ravel(order="F").view(np.float64)).pin_memory()
        th = torch.from_numpy(hpsi.ravel(order="F").view(np.float64)).pin_memory()
        psi = tp.numpy().view(np.complex128).reshape((mxddim, mxdbnd), order="F")
        hpsi = th.numpy().view(np.complex128).reshape((mxddim, mxdbnd), order="F")
    anl = np.asfortranarray(np.vstack([d["anlga"], np.zeros((3, d["nanl"]), np.complex128)]))
    H.hk_psi_c16(m, nb, psi, hpsi, True, d["ng"], np.asfortranarray(d["kgv"]), d["ekpg"], d["isort"], d["vscr"],
                 d["kmscr"], anl, d["xnlkb"], d["nanl"], mxddim, mxdbnd, d["nanl"], d["ng"], d["vscr"].size)
    assert relerr(hpsi[:m, :nb], oracle_hpsi(d, psi[:m], nb)) < TOL64
    assert np.all(hpsi[m:, :] == 5.0 - 5.0j) and np.all(hpsi[:, nb:] == 5.0 - 5.0j)


@pytest.mark.parametrize("wname,ik,nb", [("si2", 3, 7), ("small", 1, 5)])
def test_projector_products_on_int8_tensor_cores(cuda, wname, ik, nb):
    # FP64 context with 7-slice int8 projector products: within the FP64 tolerance of the
    # oracle; MIXED_TC with 4 slices: within the FP32 local-part tolerance
    import torch
    w = configs.WORKLOADS[wname]()
    d = configs.kpoint_inputs(w, ik)
    psi = configs.random_psi(d["mtxd"], nb, 300 + ik)
    ref = oracle_hpsi(d, psi, nb)
    ctx = H.Context(0).setup(d)
    ctx.set_projector_slices(7)
    assert relerr(run_device(ctx, psi, torch, cuda), ref) < TOL64
    ctx.set_projector_slices(0)
    assert relerr(run_device(ctx, psi, torch, cuda), ref) < TOL64
    ctx.close()
    ctx = H.Context(0, precision=H.MIXED_TC).setup(d)
    ctx.set_projector_slices(4)
    assert relerr(run_device(ctx, psi, torch, cuda), ref) < TOL32
    ctx.close()


def test_int8_projector_term_si64(cuda):
    # the projector term alone on the Si64 cell (256 projectors, 26,529 plane waves), 7, 5 and 4
    # slices against FP64: 1e-12, 1e-8 and 1e-6 of its maximum (each slice carries 7 more bits)
    import torch
    w = configs.si64_cubic()
    d = configs.kpoint_inputs(w, 0)
    nb = 24
    psi = configs.random_psi(d["mtxd"], nb, 31)
    want = O.hk_psi_nl_c16(psi, np.zeros_like(psi), d["anlga"], d["xnlkb"], ladd=True)
    for slices, tol in ((7, 1e-12), (5, 1e-8), (4, 1e-6)):
        ctx = H.Context(0).setup(d)
        ctx.set_projector_slices(slices)
        full = run_device(ctx, psi, torch, cuda)
        ctx.set_projector_slices(0)
        ctx.close()
        ctx = H.Context(0).setup(d)
        loc = run_device(ctx, psi, torch, cuda, local_only=True)
        kin = np.asarray(d["ekpg"])[:, None] * psi
        ctx.close()
        got = full - loc - kin
        assert relerr(got, want) < tol, (slices, relerr(got, want))
