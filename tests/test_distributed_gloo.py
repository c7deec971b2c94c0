"""CPU, world size 2 over gloo: the k-point sharded reduction of the multi-GPU path.

Each rank evaluates the oracle's KB forces (Src/ALFA/for_str_nl_kb.f90 restated) for its
round-robin share of the Si2 fcc k-points with k-dependent wavefunctions; the all-reduced
weighted sum must equal the serial sum over all k-points, and max_over_ranks must return
the largest rank value."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from cpw2000_b200 import distributed as D

pytestmark = pytest.mark.timeout(300)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _per_k_forces(k):
    from cpw2000_b200 import configs
    from oracle import forces as OF
    w = configs.si2_fcc()
    d = configs.kpoint_inputs(w, k)
    psi = configs.random_psi(d["mtxd"], 4, 1000 + k)
    occ = np.full(4, 2.0)
    return OF.for_str_nl_kb_forces(d["rkpt"], d["mtxd"], d["isort"], d["kgv"], psi, occ, w.species, d["vkb"],
                                   d["nkb"], w.adot)


def _worker(rank, world, port, nk, weights, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        total = D.weighted_kpoint_sum(_per_k_forces, weights, nk, rank, world)
        tmax = D.max_over_ranks(float(rank + 1))
        out[rank] = (total, tmax)
    finally:
        dist.destroy_process_group()


def test_kpoint_shard_round_robin():
    shards = [D.kpoint_shard(10, r, 3) for r in range(3)]
    assert shards == [[0, 3, 6, 9], [1, 4, 7], [2, 5, 8]]
    assert sorted(sum(shards, [])) == list(range(10))


def test_sharded_force_sum_world2():
    nk = 4
    weights = np.array([0.1, 0.2, 0.3, 0.4])
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, nk, weights, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(240)
            assert p.exitcode == 0
        res = dict(out)
    serial = sum(weights[k] * _per_k_forces(k) for k in range(nk))
    for r in range(2):
        total, tmax = res[r]
        assert np.abs(total - serial).max() <= 1e-13 * max(1.0, np.abs(serial).max())
        assert tmax == 2.0
