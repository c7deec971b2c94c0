"""Failure detection on the GPU without a fault: bounded device waits that run out.

Every wait of the library's kernels on another party is bounded; when the limit
runs out the kernel records the failure and returns, the host reports
CPW_B200_TIMEOUT, and the context stays usable. Nothing here faults, traps or
hangs the GPU:

1. mbarrier wait (tensor-core GEMM roles): cpw_b200_wait_selftest runs the
   GEMMs' bounded wait on an mbarrier that nothing arrives at, with a 1 ms
   limit. cpw_b200_synchronize then returns CPW_B200_TIMEOUT, the next one 0,
   and a MIXED_TC H|psi> on the same context still matches the oracle.
2. grid barrier (the eigensolver's cooperative Gram-Schmidt kernel): with its
   poll limit set to 0, a CTA that reaches a grid barrier before the others
   gives up at its first poll, so the eigensolver call returns
   CPW_B200_TIMEOUT; with the default limit restored the same context solves
   to the dense eigenvalues.
"""
import numpy as np
import pytest

from cpw2000_b200 import _lib, configs
from cpw2000_b200 import ditsp as E
from cpw2000_b200 import hk_psi as H
from cpw2000_b200._lib import CpwB200Error
from oracle import hk_psi as O

pytestmark = pytest.mark.gpu

TIMEOUT = -4


def test_mbarrier_wait_runs_out_and_context_recovers(cuda):
    import torch
    w = configs.si2_fcc()
    d = configs.kpoint_inputs(w, 1)
    ctx = H.Context(0, precision=H.MIXED_TC).setup(d)
    L = _lib.lib()
    assert L.cpw_b200_wait_selftest(ctx.handle, 1_000_000, None) == 0
    assert L.cpw_b200_synchronize(ctx.handle) == TIMEOUT
    assert "gave up" in L.cpw_b200_last_error().decode()
    assert L.cpw_b200_synchronize(ctx.handle) == 0          # the flag is cleared once reported
    m, nb = d["mtxd"], 5
    psi_h = configs.random_psi(m, nb, 71)
    psi = torch.from_numpy(np.ascontiguousarray(psi_h.T)).to(cuda).t()
    out = torch.zeros((nb, m), dtype=torch.complex128, device=cuda).t()
    ctx.hk_psi(psi, out)
    ctx.synchronize()
    ref = O.hk_psi_c16(m, nb, psi_h, d["ekpg"], d["isort"], d["vscr"], d["kmscr"], d["kgv"], d["anlga"], d["xnlkb"])
    assert np.abs(out.cpu().numpy() - ref).max() / np.abs(ref).max() < 2e-5
    ctx.close()


def test_selftest_rejects_limits_above_two_seconds(cuda):
    ctx = H.Context(0)
    L = _lib.lib()
    assert L.cpw_b200_wait_selftest(ctx.handle, 3_000_000_000, None) == 1
    ctx.close()


def test_grid_barrier_wait_runs_out_and_context_recovers(cuda):
    import torch
    w = configs.si2_fcc()
    d = configs.kpoint_inputs(w, 0, with_hamsm=True)
    nb = 8
    ctx = H.Context(0).setup(d)            # FP64: the reference's modified Gram-Schmidt on the device
    m = d["mtxd"]

    def solve():
        psi = torch.zeros((3 * nb, m), dtype=torch.complex128, device=cuda).t()
        hpsi = torch.zeros_like(psi)
        return E.eigensolve(ctx, psi, hpsi, nb, d["mtxds"], d["hamsm"], d["hdiag"], epspsi=1e-5)

    ctx.set_wait_limits(grid_polls=0)
    with pytest.raises(CpwB200Error) as ei:
        solve()
    assert ei.value.status == TIMEOUT and "grid barrier" in str(ei.value)
    ctx.set_wait_limits()                   # defaults again
    r = solve()
    assert r["converged"]
    dense = np.linalg.eigvalsh(O.dense_h(m, d["ekpg"], d["isort"], d["vscr"], d["kmscr"], d["kgv"], d["anlga"],
                                         d["xnlkb"]))
    assert np.abs(r["ei"] - dense[: r["neig"]]).max() < 1e-8
    ctx.close()
