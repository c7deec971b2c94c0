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

import queue
import threading
import time

import numpy as np

from . import ditsp as E
from .hk_psi import FP64, Context


def eigensolve_kpoints(inputs: list[dict], nbands: int, workers: int = 8, precision: int = FP64, epspsi=1e-5,
                       icmax=60, device: int = 0, seed: int = 0):
    """Run ditsp for every k-point dict of ``inputs`` (configs.kpoint_inputs(..., with_hamsm=True)).

    Returns (results, seconds): results[k] = dict(ei, neig, ihkpsum, converged) in input order,
    seconds the wall time of the whole set (inputs already on the host, contexts created inside).
    """
    import torch
    dev = torch.device("cuda", device)
    todo: queue.Queue = queue.Queue()
    for k in range(len(inputs)):
        todo.put(k)
    results: list = [None] * len(inputs)
    errors: list = []
    nw = max(1, min(int(workers), len(inputs)))
    ctxs = [Context(device, precision=precision) for _ in range(nw)]
    # size every context's basis buffers for the largest k-point before the clock starts
    big = max(range(len(inputs)), key=lambda k: inputs[k]["mtxd"])
    for c in ctxs:
        c.setup(inputs[big])
    torch.cuda.synchronize(dev)

    def work(ctx: Context):
        stream = torch.cuda.Stream(device=dev)
        try:
            while True:
                try:
                    k = todo.get_nowait()
                except queue.Empty:
                    return
                d = inputs[k]
                ctx.setup(d)
                with torch.cuda.stream(stream):
                    psi = torch.zeros((nbands, d["mtxd"]), dtype=torch.complex128, device=dev).t()
                    hpsi = torch.zeros_like(psi)
                    r = E.eigensolve(ctx, psi, hpsi, nbands, d["mtxds"], d["hamsm"], d["hdiag"], epspsi=epspsi,
                                     icmax=icmax, stream=stream.cuda_stream)
                stream.synchronize()
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
    if errors:
        raise errors[0]
    return results, seconds
