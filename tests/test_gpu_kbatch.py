"""GPU: batched H|psi> over k-points (cpw_b200_kbatch_*) against per-k-point contexts.

Workload: the Si8 cubic cell at Ecut 20 Ha (40^3 box) with seeded random k-points,
uneven plane-wave counts per k and uneven band counts per k (including 1 band).
The batch uses the union of the k-points' spheres for its kept planes, so its FP64
result agrees with the single-k path to rounding (1e-12); the mixed forms agree
with FP64 to the FP32 tolerance. Calls after the first replay a captured CUDA
graph: the replay must read the current contents of the blocks.
"""
import numpy as np
import pytest

from cpw2000_b200 import configs
from cpw2000_b200 import hk_psi as H
from cpw2000_b200.kbatch import KBatch
from oracle import hk_psi as O

pytestmark = pytest.mark.gpu

NBS = [40, 37, 40, 12, 1, 25]


def _inputs():
    w = configs.si8_cubic_kbatch()
    return [configs.kpoint_inputs(w, ik) for ik in range(len(NBS))]


def _blocks(inputs, torch, dev, seed):
    out = []
    for k, (d, nb) in enumerate(zip(inputs, NBS)):
        psi = configs.random_psi(d["mtxd"], nb, seed + k)
        out.append(torch.from_numpy(np.ascontiguousarray(psi.T)).to(dev).t())
    return out


def _single(d, psi, prec, torch, dev):
    ctx = H.Context(0, precision=prec).setup(d)
    y = torch.zeros_like(psi)
    ctx.hk_psi(psi, y)
    torch.cuda.synchronize()
    ctx.synchronize()
    ctx.close()
    return y.cpu().numpy()


def relerr(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("prec,tol", [(H.FP64, 1e-12), (H.MIXED, 2e-5), (H.MIXED_TC, 2e-5)])
def test_kbatch_matches_single_kpoint(cuda, prec, tol):
    import torch
    inputs = _inputs()
    assert len({d["mtxd"] for d in inputs}) > 1          # uneven plane-wave counts
    ctx = H.Context(0, precision=prec).setup(inputs[0])
    kb = KBatch(ctx, inputs)
    psis = _blocks(inputs, torch, cuda, 100)
    hps = [torch.zeros_like(x) for x in psis]
    kb.hk_psi(psis, hps)
    torch.cuda.synchronize()
    kb.synchronize()
    for k, d in enumerate(inputs):
        ref = _single(d, psis[k], H.FP64, torch, cuda)
        assert relerr(hps[k].cpu().numpy(), ref) < tol, k
    # one k-point against the oracle as well
    got0 = hps[3].cpu().numpy()
    ora = O.hk_psi_c16(inputs[3]["mtxd"], NBS[3], psis[3].cpu().numpy(), inputs[3]["ekpg"], inputs[3]["isort"],
                       inputs[3]["vscr"], inputs[3]["kmscr"], inputs[3]["kgv"], inputs[3]["anlga"],
                       inputs[3]["xnlkb"])
    assert relerr(got0, ora) < max(tol, 1e-12)
    info = kb.info()
    assert info["tuned"] == 1 and info["captures"] == 1 and info["candidates"] >= 3
    kb.close()
    ctx.close()


def test_kbatch_graph_replay_reads_current_data(cuda):
    import torch
    inputs = _inputs()
    ctx = H.Context(0, precision=H.FP64).setup(inputs[0])
    kb = KBatch(ctx, inputs)
    psis = _blocks(inputs, torch, cuda, 200)
    hps = [torch.zeros_like(x) for x in psis]
    kb.hk_psi(psis, hps)                       # tunes, runs, captures
    new = _blocks(inputs, torch, cuda, 300)
    for x, y in zip(psis, new):
        x.copy_(y)                             # same arrays, new contents
    for y in hps:
        y.zero_()
    kb.hk_psi(psis, hps)                       # graph replay
    kb.hk_psi(psis, hps)
    torch.cuda.synchronize()
    kb.synchronize()
    for k, d in enumerate(inputs):
        assert relerr(hps[k].cpu().numpy(), _single(d, psis[k], H.FP64, torch, cuda)) < 1e-12
    info = kb.info()
    assert info["graph_replays"] == 2 and info["captures"] == 1
    # other arrays: a new capture
    hps2 = [torch.zeros_like(x) for x in psis]
    kb.hk_psi(psis, hps2)
    torch.cuda.synchronize()
    assert kb.info()["captures"] == 2
    for a, b in zip(hps, hps2):
        assert torch.equal(a, b)
    kb.close()
    ctx.close()
