"""Eigensolver over the k-points of one crystal, several k-points in flight on one GPU.

The reference loops over k-points serially (Src/cpw_lib/cpw_scf.f90:488 -> h_kb_dia ->
ditsp_c16), each k-point's solve a chain of small dependent steps (H|psi> of a few dozen
bands, block Gram-Schmidt, a small zheevd) that leaves most of a B200 idle when the basis is
a few thousand plane waves. Here ``workers`` host threads each own a context (its own CUDA
stream, cuBLAS and cuSOLVER handles, device buffers) and take k-points from a shared queue;
the solves of different k-points are independent, so their kernels overlap on the GPU while
every k-point runs exactly the single-k-point eigensolver (results identical to a serial run).
The ctypes calls release the GIL for their whole duration.
"""
from __future__ import annotations

import os
import queue
import threading
import time

import numpy as np

from . import ditsp as E
from .hk_psi import FP64, Context


def eigensolve_kpoints(inputs: list[dict], nbands: int, workers: int = 8, precision: int = FP64, epspsi=1e-5,
                       icmax=60, device: int = 0, seed: int = 0, mxdbnd: int | None = None, trace: bool = False,
                       keep: int = 0, slab_budget: int = 0, env: dict | None = None, ipr: int = 0,
                       priorities: list[int] | None = None):
    """Run ditsp for every k-point dict of ``inputs`` (configs.kpoint_inputs(..., with_hamsm=True)).

    Returns (results, seconds): results[k] = dict(ei, neig, ihkpsum, converged) in input order,
    seconds the wall time of the whole set (inputs already on the host, contexts created inside).
    icmax: outer iterations at most, one count for every k-point or a sequence with one per input.
    mxdbnd: columns of psi/hpsi (default nbands; the reference's array dimension, which bounds
    the iterative block). trace: also the per-iteration trace of each k-point (eigensolve's), with
    times from the common start of the set. keep: the first ``keep`` columns of each k-point's
    converged psi are returned (device tensors, ``psi``). slab_budget: FFT slab bytes per context.
    env: environment variables set while the set runs (the eigensolver reads its switches then).
    ipr: the eigensolver's print level (2: per-phase wall times of every k-point).
    priorities: CUDA stream priority of each k-point's solve (lower = scheduled first, within the
    device's range, e.g. -5 .. 0); k-points are also taken from the queue in that order. An SCF
    code can rank k-points by the outer iterations their previous solve took, so that the longest
    solve is not held back by the others (longest-processing-time-first).
    """
    import torch
    dev = torch.device("cuda", device)
    todo: queue.Queue = queue.Queue()
    order = sorted(range(len(inputs)), key=lambda k: priorities[k]) if priorities else range(len(inputs))
    for k in order:
        todo.put(k)
    results: list = [None] * len(inputs)
    errors: list = []
    nw = max(1, min(int(workers), len(inputs)))
    mxdbnd = int(mxdbnd or nbands)
    icmaxes = [int(v) for v in icmax] if hasattr(icmax, "__len__") else [int(icmax)] * len(inputs)
    if len(icmaxes) != len(inputs):
        raise ValueError("icmax: one count per k-point expected")
    saved = {k: os.environ.get(k) for k in (env or {})}
    os.environ.update(env or {})
    ctxs = [Context(device, precision=precision) for _ in range(nw)]
    if slab_budget:
        for c in ctxs:
            c.set_slab_budget(slab_budget)
    # size every context's basis buffers for the largest k-point before the clock starts
    big = max(range(len(inputs)), key=lambda k: inputs[k]["mtxd"])
    for c in ctxs:
        c.setup(inputs[big])
    torch.cuda.synchronize(dev)

    def work(ctx: Context):
        streams: dict = {}
        try:
            while True:
                try:
                    k = todo.get_nowait()
                except queue.Empty:
                    return
                pr = int(priorities[k]) if priorities else 0
                if pr not in streams:
                    streams[pr] = torch.cuda.Stream(device=dev, priority=pr)
                stream = streams[pr]
                d = inputs[k]
                ctx.setup(d)
                with torch.cuda.stream(stream):
                    psi = torch.zeros((mxdbnd, d["mtxd"]), dtype=torch.complex128, device=dev).t()
                    hpsi = torch.zeros_like(psi)
                    t_k = time.perf_counter() - t0
                    r = E.eigensolve(ctx, psi, hpsi, nbands, d["mtxds"], d["hamsm"], d["hdiag"], epspsi=epspsi,
                                     icmax=icmaxes[k], stream=stream.cuda_stream, trace=trace, ipr=ipr)
                stream.synchronize()
                if trace:
                    r["trace"][:, 0] += t_k          # times from the start of the set
                if keep:
                    r["psi"] = psi[:, :keep].clone()
                del psi, hpsi
                results[k] = r
        except Exception as exc:            # reported to the caller after the join
            errors.append(exc)

    t0 = time.perf_counter()
    threads = [threading.Thread(target=work, args=(c,)) for c in ctxs]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    torch.cuda.synchronize(dev)
    seconds = time.perf_counter() - t0
    for c in ctxs:
        c.close()
    for k, v in saved.items():
        if v is None:
            os.environ.pop(k, None)
        else:
            os.environ[k] = v
    if errors:
        raise errors[0]
    return results, seconds
