"""Benchmark of the H|psi> drop-in and the eigensolver on the Si216 workload (one JSON line on rank 0).

Workload (the configuration the headline metric is quoted on): Si 216-atom
cubic supercell, a = 30.78 bohr, seeded 0.03 bohr displacements, Ecut 16 Ha
(88,951 plane waves at Gamma), 144^3 FFT box, 864 KB projectors, 480 bands.
A step is one H|psi> application to all 480 bands at Gamma (one hk_psi_c16 call).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--eig 0|1] [--eig-repeats R] [--eig-kpoints NK]

value: bands/s of the FP64 drop-in with inputs resident in HBM, summed over
ranks (replicas, one per GPU), device-timed with CUDA events; psi + hpsi
(1.37 GB) exceed L2, so no flush between steps. e2e: the same metric through
the reference-facing C ABI (cpw_b200_hk_psi_c16) on pinned host arrays, the H2D
copy of psi and the D2H copy of hpsi inside the timed region. time_to_eigvals:
the eigensolver (ditsp_c16 restated) on Gamma and the 3 random k-points of the
workload, FP64 drop-in vs the mixed form, to 1e-6 Ha (both) and 1e-8 Ha (FP64),
median of R repeats, then adjoint forces of both converged sets at Gamma (on by default on
one GPU; --gpus N > 1 runs the H|psi> replicas only unless --eig 1 is given).
--impl reference times the CPU restatement of the reference's hk_psi_c16
(C + OpenMP, all host threads) on the same workload, a sample of bands per step.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from cpw2000_b200 import configs  # noqa: E402

METRIC = "H|psi> bands/s"
NB = 480
WORKLOAD = "si216"
NB64 = 160


def workload_desc(d):
    return {"workload": "si216_cubic_ecut16_box144: Si216 cubic a=30.78, sigma 0.03, Ecut 16 Ha, Gamma, "
                        f"mtxd {d['mtxd']}, box 144^3, {d['nanl']} KB projectors, {NB} bands",
            "bands": NB, "mtxd": int(d["mtxd"]), "box": [int(v) for v in d["kmscr"][3:6]], "nanl": int(d["nanl"]),
            "l2": "not flushed: inputs larger than L2 (psi + hpsi 1.37 GB > 126 MB)"}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), float(j.get("bf16_tflops", 0.0)), "measured"
    return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def gemm_text(blas: bool) -> str:
    if blas:
        return ("in numpy's bundled OpenBLAS zgemm, like the reference's default build, which links an "
                "optimised external BLAS")
    return "as plain OpenMP loops, like the reference built with its vendored netlib BLAS"


def cpu_reference_rate(d, nbands: int, nthreads: int = 0, repeats: int = 1):
    """bands/s of the C + OpenMP restatement of hk_psi_c16 on a sample of bands."""
    from oracle import c_ref
    psi = configs.random_psi(d["mtxd"], nbands, 1234)
    args = (d["mtxd"], nbands, psi, d["ekpg"], d["isort"], d["vscr"], d["kmscr"], d["kgv"], d["anlga"], d["xnlkb"])
    c_ref.hk_psi_c16(*args[:1], 1, psi[:, :1], *args[3:], nthreads=nthreads)     # warm (plans, pages)
    times = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        c_ref.hk_psi_c16(*args, nthreads=nthreads)
        times.append(time.perf_counter() - t0)
    return nbands / min(times), (nthreads or c_ref.max_threads())


def first_within(trace, ref, nocc, tol):
    """0-based outer iteration at which the lowest nocc Ritz values of an eigensolver trace (rows:
    elapsed s, xmax, nconv, H|psi> products, eigenvalues...) are all within tol of ref, or None."""
    err = np.abs(trace[:, 4:4 + nocc] - ref[None, :]).max(axis=1)
    ok = np.nonzero(err <= tol)[0]
    return int(ok[0]) if len(ok) else None


def stop_iterations(results, refs, nocc, tol, icmax, margin=5):
    """Per k-point outer-iteration limit of a later repeat: `margin` iterations past the one at which
    the first repeat met the tolerance (all its iterations when it never did), at most icmax."""
    per_k = []
    for r, ref in zip(results, refs):
        i = first_within(r["trace"], ref, nocc, tol)
        per_k.append(min(icmax, (i + 1 if i is not None else r["trace"].shape[0]) + margin))
    return per_k


def longest_first_priorities(per_k):
    """CUDA stream priorities (lower runs first) ranking k-points by their iteration counts: the
    longest solve gets -(n-1), the shortest 0; ties keep input order."""
    rank = sorted(range(len(per_k)), key=lambda k: -per_k[k])
    prio = [0] * len(per_k)
    for pos, k in enumerate(rank):
        prio[k] = -(len(per_k) - 1 - pos)
    return prio


def set_time(results, refs, nocc, tol):
    """(seconds, iterations per k-point, H|psi> band products) until every k-point met the tolerance:
    the latest k-point's time (traces hold times from the start of the set), or (None, None, None)
    if one never did."""
    ts, its, hk = [], [], 0
    for r, ref in zip(results, refs):
        i = first_within(r["trace"], ref, nocc, tol)
        if i is None:
            return None, None, None
        ts.append(float(r["trace"][i, 0]))
        its.append(i + 1)
        hk += int(r["trace"][i, 3])
    return max(ts), its, hk


def time_to_eigvals(w, inputs, local, repeats=3, workers=4, icmax=300, nocc=None, budget_s=480.0,
                    prioritise=False):
    """Eigensolver (ditsp_c16 restated) on the k-points of the Si216 workload, FP64 drop-in vs mixed.

    Each repeat solves every k-point of ``inputs`` (Gamma + 3 random k) from the start basis
    (iguess 0, epspsi 1e-5, psi/hpsi with 3*480 columns), ``workers`` k-points in flight on
    their own contexts (cpw2000_b200.kpoints). Reference values: the FP64 path's converged Ritz
    values of each k-point (first repeat). Time to eigenvalues of a form at a tolerance = the
    time from the start of the set until every k-point's lowest nocc (occupied) Ritz values are
    within the tolerance of the reference values (the latest of the k-points' first such outer
    iteration). Reported as the median over repeats with the spread, at 1e-6 Ha for both forms
    and 1e-8 Ha for FP64. The first repeat runs icmax outer iterations (its last values are the
    reference); later repeats stop each k-point 5 outer iterations after the one at which its
    Ritz values met the form's tolerance in the first repeat (1e-8 Ha for FP64, 1e-6 Ha for the
    mixed form), and start only while the eigensolver sets stay within budget_s seconds (the
    number of repeats done is reported). Forces: adjoint (Hellmann-Feynman) forces at Gamma from
    each form's converged occupied wavefunctions; their largest difference in Ha/bohr.
    """
    import torch

    from cpw2000_b200 import forces as FF
    from cpw2000_b200 import hk_psi as H
    from cpw2000_b200 import kpoints
    natom = sum(sp.natom for sp in w.species)
    nocc = nocc or 2 * natom
    forms = (("fp64", H.FP64), ("mixed_tc", H.MIXED_TC))
    runs = {name: [] for name, _ in forms}
    keep = {}
    icmax_rep = {name: icmax for name, _ in forms}
    prio_rep = {name: None for name, _ in forms}
    t_start = time.perf_counter()
    refs = None
    for rep in range(repeats):
        t_rep = time.perf_counter()
        for name, prec in forms:
            res, secs = kpoints.eigensolve_kpoints(inputs, NB, workers=workers, precision=prec, epspsi=1e-5,
                                                   icmax=icmax_rep[name], device=local, mxdbnd=3 * NB, trace=True,
                                                   keep=nocc if rep == 0 else 0, slab_budget=2 << 30,
                                                   priorities=prio_rep[name])
            if rep == 0:
                keep[name] = res[0].pop("psi")
                for r in res[1:]:
                    r.pop("psi", None)
            runs[name].append((res, secs))
            torch.cuda.empty_cache()
        if rep == 0:
            refs = [r["trace"][-1, 4:4 + nocc] for r in runs["fp64"][0][0]]
            # later repeats stop every k-point 5 outer iterations after the one at which its own
            # Ritz values met the form's tolerance in the first repeat (a converged k-point does
            # not keep running beside the others)
            for name, _ in forms:
                tol = 1e-8 if name == "fp64" else 1e-6
                icmax_rep[name] = stop_iterations(runs[name][0][0], refs, nocc, tol, icmax)
                if prioritise:
                    # longest solve first: stream priority by the first repeat's iteration counts
                    prio_rep[name] = longest_first_priorities(icmax_rep[name])
        dt = time.perf_counter() - t_rep
        if time.perf_counter() - t_start + 0.8 * dt > budget_s:
            break

    out = {"kpoints": [[float(x) for x in w.kpoints[k]] for k in range(len(inputs))],
           "mtxd": [int(d["mtxd"]) for d in inputs], "occupied": nocc, "repeats": len(runs["fp64"]),
           "repeats_asked": repeats, "kpoints_in_flight": workers, "icmax_first": icmax,
           "icmax_later": icmax_rep, "stream_priorities_later": prio_rep}
    for name, _ in forms:
        tols = (1e-6, 1e-8) if name == "fp64" else (1e-6,)
        entry = {}
        for tol in tols:
            vals = [set_time(res, refs, nocc, tol) for res, _ in runs[name]]
            times = [v[0] for v in vals if v[0] is not None]
            key = f"{tol:.0e}".replace("e-0", "e-")
            entry[f"seconds_to_{key}_ha"] = statistics.median(times) if len(times) == len(vals) else None
            entry[f"seconds_to_{key}_ha_all"] = [v[0] for v in vals]
            entry[f"iterations_to_{key}_ha"] = vals[0][1]
            entry[f"hpsi_band_products_to_{key}_ha"] = vals[0][2]
        res0 = runs[name][0][0]
        entry["converged"] = [bool(r["converged"]) for r in res0]
        entry["outer_iterations"] = [int(r["trace"].shape[0]) for r in res0]
        entry["set_wall_s"] = [float(sec) for _, sec in runs[name]]
        entry["max_err_ha_at_end"] = float(max(np.abs(r["trace"][-1, 4:4 + nocc] - ref).max()
                                               for r, ref in zip(res0, refs)))
        out[name] = entry
    a, b = out["fp64"]["seconds_to_1e-6_ha"], out["mixed_tc"]["seconds_to_1e-6_ha"]
    out["speedup_mixed_tc_vs_fp64_at_1e-6"] = a / b if a and b else None
    a8 = out["fp64"]["seconds_to_1e-8_ha"]
    out["speedup_mixed_tc_1e-6_vs_fp64_1e-8"] = a8 / b if a8 and b else None
    d0 = inputs[0]
    fc = {}
    for name in keep:
        sysm = FF.HFSystem(w, d0, keep[name], np.full(nocc, 2.0), device=local)
        _, f = FF.forces(sysm)
        fc[name] = FF.to_cartesian(f, w.adot)
        sysm.ctx.close()
    out["force_max_abs_diff_ha_bohr"] = float(np.abs(fc["mixed_tc"] - fc["fp64"]).max())
    out["force_max_abs_ha_bohr"] = float(np.abs(fc["fp64"]).max())
    out["definition"] = (f"time from the start of the k-point set until the lowest {nocc} Ritz values of every "
                         "k-point are within the tolerance of the FP64 path's converged values; epspsi 1e-5; "
                         "start basis from the small matrix (iguess 0); median over repeats (the first runs every "
                         "k-point to icmax_first outer iterations, later ones stop each k-point 5 iterations after "
                         "its Ritz values met the tolerance in the first); forces at Gamma")
    return out


def kpoint_eig(local, nk=16, nb=40, workers=8):
    """Eigensolver over nk k-points of the Si8 cell (Ecut 20 Ha, 40^3, ~4,610 PW, 40 bands):
    one context after another vs `workers` contexts in flight on host threads
    (cpw2000_b200.kpoints); the Ritz values of both runs must agree."""
    from cpw2000_b200 import kpoints
    w = configs.si8_cubic_kbatch(nk=nk)
    inputs = [configs.kpoint_inputs(w, k, nbands=nb, with_hamsm=True) for k in range(nk)]
    kpoints.eigensolve_kpoints(inputs[:2], nb, workers=2, device=local)          # warm-up
    serial, t1 = kpoints.eigensolve_kpoints(inputs, nb, workers=1, device=local)
    conc, tn = kpoints.eigensolve_kpoints(inputs, nb, workers=workers, device=local)
    diff = max(float(np.abs(a["ei"] - b["ei"]).max()) for a, b in zip(serial, conc))
    return {"workload": f"si8 cubic, Ecut 20 Ha, 40^3 box, {nk} random k-points, {nb} bands, epspsi 1e-5, icmax 60, FP64",
            "serial_s": t1, "concurrent_s": tn, "workers": workers, "speedup": t1 / tn,
            "kpoints_per_s": nk / tn, "max_ritz_diff_vs_serial": diff,
            "converged": int(sum(r["converged"] for r in conc))}


def kbatch_throughput(local, steps, warmup, nk=64):
    """Batched H|psi> over the 64 random k-points of the Si8 cubic cell (Ecut 20 Ha, 40^3 box,
    ~4,600 plane waves per k, 40 bands per k): one batched call (autotuned, replayed from a
    CUDA graph) per step, against the same work as one H|psi> call per k-point on per-k
    contexts. Inputs (188 MB of psi and as much hpsi) exceed L2, so no flush between steps."""
    import torch

    from cpw2000_b200 import hk_psi as H
    from cpw2000_b200.kbatch import KBatch
    dev = torch.device("cuda", local)
    w = configs.si8_cubic_kbatch()
    inputs = [configs.kpoint_inputs(w, ik) for ik in range(nk)]
    nbk = 40
    psis = [torch.from_numpy(np.ascontiguousarray(configs.random_psi(d["mtxd"], nbk, 500 + k).T)).to(dev).t()
            for k, d in enumerate(inputs)]
    hps = [torch.empty_like(x) for x in psis]
    out = {"workload": f"si8 cubic, Ecut 20 Ha, 40^3 box, {nk} random k-points, {nbk} bands per k",
           "mtxd_min": min(d["mtxd"] for d in inputs), "mtxd_max": max(d["mtxd"] for d in inputs)}

    def timeit(fn):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(steps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / steps

    for name, prec in (("fp64", H.FP64), ("mixed_tc", H.MIXED_TC)):
        ctx = H.Context(local, precision=prec).setup(inputs[0])
        kb = KBatch(ctx, inputs)
        kb.hk_psi(psis, hps)                  # autotune + capture
        ms_b = timeit(lambda: kb.hk_psi(psis, hps))
        kb.synchronize()
        info = kb.info()
        ctxs = [H.Context(local, precision=prec).setup(d) for d in inputs]

        def seq():
            for c, x, y in zip(ctxs, psis, hps):
                c.hk_psi(x, y)
        ms_s = timeit(seq)
        for c in ctxs:
            c.close()
        kb.close()
        ctx.close()
        out[name] = {"batched_bands_per_s": nk * nbk / (ms_b / 1e3), "batched_ms": ms_b,
                     "per_k_loop_bands_per_s": nk * nbk / (ms_s / 1e3), "per_k_loop_ms": ms_s,
                     "speedup_batched_vs_loop": ms_s / ms_b, "tuning": info}
    return out


def run_eig_study(args, local):
    """Eigensolver to convergence on one workload, FP64 drop-in vs the mixed form, then adjoint forces.

    Prints one JSON line: per variant the iteration trace summary; time-to-eigvals of the mixed form =
    elapsed time at the first outer iteration whose lowest nocc (occupied) Ritz values are all within
    1e-6 Ha of the converged FP64 values (FP64: within 1e-8 Ha of its own converged values); and the
    largest difference between the adjoint forces of the two converged wavefunction sets.
    """
    import torch

    from cpw2000_b200 import crystal
    from cpw2000_b200 import ditsp as E
    from cpw2000_b200 import forces as FF
    from cpw2000_b200 import hk_psi as H
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    w = {"si216": configs.si216_cubic, "si64": configs.si64_cubic, "zb64": configs.zb64_cubic}[args.workload]()
    nb = {"si216": 480, "si64": 160, "zb64": 160}[args.workload]
    t0 = time.time()
    d = configs.kpoint_inputs(w, 0, with_hamsm=True)
    natom = sum(sp.natom for sp in w.species)
    nocc = 2 * natom
    out = {"mode": "eig", "workload": args.workload, "mtxd": d["mtxd"], "nanl": d["nanl"], "bands": nb,
           "occupied": nocc, "epspsi": args.epspsi, "icmax": args.icmax, "setup_s": time.time() - t0}
    known = {"fp64": (H.FP64, {}), "fp64_cholqr": (H.FP64, {"CPW_B200_ORTHO": "cholqr"}),
             "mixed": (H.MIXED, {}), "mixed_tc": (H.MIXED_TC, {})}
    names = ["fp64"] + [v for v in args.variants.split(",") if v and v != "fp64"]
    if args.with_cholqr and "fp64_cholqr" not in names:
        names.insert(1, "fp64_cholqr")
    variants = [(n, known[n][0], known[n][1]) for n in names]
    traces, psis = {}, {}
    for name, prec, env in variants:
        os.environ.pop("CPW_B200_ORTHO", None)
        os.environ.update(env)
        ctx = H.Context(local, precision=prec).setup(d)
        ctx.set_slab_budget(4 << 30)
        P = torch.zeros((3 * nb, d["mtxd"]), dtype=torch.complex128, device=dev).t()
        HP = torch.zeros_like(P)
        torch.cuda.synchronize()
        icmax = args.icmax_ref if (name == "fp64" and args.icmax_ref) else args.icmax
        r = E.eigensolve(ctx, P, HP, nb, d["mtxds"], d["hamsm"], d["hdiag"], epspsi=args.epspsi, icmax=icmax,
                         trace=True, ipr=args.ipr)
        ctx.close()
        traces[name] = r["trace"]
        if args.save_traces:
            os.makedirs(args.save_traces, exist_ok=True)
            np.save(os.path.join(args.save_traces, f"trace_{args.workload}_{name}.npy"), r["trace"])
        psis[name] = P[:, :nocc].clone()
        out[name] = {"converged": bool(r["converged"]), "outer_iterations": int(r["trace"].shape[0]),
                     "seconds_total": float(r["trace"][-1, 0]), "hpsi_band_products": int(r["ihkpsum"]),
                     "xmax_end": float(r["trace"][-1, 1])}
        del P, HP
        torch.cuda.empty_cache()
    os.environ.pop("CPW_B200_ORTHO", None)
    ref = traces["fp64"][-1, 4:4 + nocc]
    for name, _, _ in variants:
        tol = 1e-8 if name.startswith("fp64") else 1e-6
        err = np.abs(traces[name][:, 4:4 + nocc] - ref[None, :]).max(axis=1)
        ok = np.nonzero(err <= tol)[0]
        k = int(ok[0]) if len(ok) else None
        out[name].update({"tolerance_ha": tol, "seconds_to_tolerance": float(traces[name][k, 0]) if k is not None
                          else None, "iterations_to_tolerance": k + 1 if k is not None else None,
                          "max_err_ha_at_end": float(err[-1])})
    for name in [v[0] for v in variants[1:]]:
        a, b = out["fp64"]["seconds_to_tolerance"], out[name]["seconds_to_tolerance"]
        if a and b:
            out[f"speedup_{name}_vs_fp64"] = a / b
    # adjoint forces (FP64 adjoint) from the converged occupied wavefunctions of each variant
    fcart = {}
    for name in psis:
        s = FF.HFSystem(w, d, psis[name], np.full(nocc, 2.0), device=local)
        _, f = FF.forces(s)
        fcart[name] = FF.to_cartesian(f, w.adot)
        s.ctx.close()
    for name in fcart:
        if name != "fp64":
            out[name]["force_max_abs_diff_ha_bohr_vs_fp64"] = float(np.abs(fcart[name] - fcart["fp64"]).max())
    out["force_max_abs_ha_bohr"] = float(np.abs(fcart["fp64"]).max())
    out["definition"] = (f"time to the lowest {nocc} Ritz values within the tolerance of the FP64 path's converged "
                         f"values; epspsi {args.epspsi}; start basis from the {d['mtxds']}x{d['mtxds']} small "
                         "matrix (iguess 0); forces: Hellmann-Feynman via the adjoint, occupation 2 per band")
    print(json.dumps(out), flush=True)


REF_SAMPLE = 24     # bands per step of the CPU arms (of the 480 of the workload)


def run_reference(args, rank):
    """CPU restatement of hk_psi_c16 on the same workload and config as our arm; every step is
    one call on a sample of REF_SAMPLE bands (the whole 480-band step takes the CPU ~a minute)."""
    if rank != 0:
        return
    w = configs.si216_cubic()
    d = configs.kpoint_inputs(w, 0)
    from oracle import c_ref
    c_ref.lib()
    blas = c_ref.use_blas(True)
    nthreads = c_ref.max_threads()
    sample = REF_SAMPLE
    for _ in range(args.warmup):
        cpu_reference_rate(d, sample, nthreads)
    rates = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        r, _ = cpu_reference_rate(d, sample, nthreads)
        rates.append(r)
    wall = time.perf_counter() - t0
    value = statistics.median(rates)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "bands/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sample / value,
            "ms_per_full_step_est": 1e3 * NB / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Gaussian pseudopotentials, random complex128 wavefunctions)",
            "config": {**workload_desc(d), "parallelism": "single GPU",
                       "precision": "fp64 drop-in (FP64 pruned FFT, FP64 projector products)"},
            "cpu_baseline": {"value": value, "unit": "bands/s", "cores": nthreads, "kind": "port",
                             "sample": f"{sample} of {NB} bands per step (median over steps), C+OpenMP restatement "
                                       f"of hk_psi_c16 (own pruned FFT; projector products {gemm_text(blas)}), "
                                       f"{nthreads} threads"},
            "e2e": {"value": value, "unit": "bands/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": wall}
    print(json.dumps(line), flush=True)


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1 and args.impl == "ours":
        import datetime

        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def per_band_bytes(d, elem):
    """Algorithmic bytes per band of the three local kernels (elem: bytes of a complex box value)."""
    from cpw2000_b200 import crystal
    kd = crystal.kd_of_basis(d["kgv"], d["isort"])
    nz = 2 * kd[2] + 1
    n1, n2, n3 = (int(v) for v in d["kmscr"][3:6])
    plane = n1 * n2
    m = d["mtxd"]
    return {"inv_xy": 16 * m + nz * plane * elem,          # psi in (complex128), kept planes out
            "z_vloc": 2 * nz * plane * elem,                 # kept planes in and out (+ V once per launch)
            "fwd_xy": nz * plane * elem + 2 * 16 * m}        # kept planes in, psi in, hpsi out


def roofline_of(stages, steps, nb, d, elem, v_bytes, hbm, peak_kind, traffic_per_band=None):
    """Roofline entry of the dominant local kernel from the live stage timers (CUDA events on the
    launching stream): algorithmic bytes per launch / average launch duration."""
    ours = {k: stages[k] for k in ("inv_xy", "z_vloc", "fwd_xy") if stages[k][1]}
    dom = max(ours, key=lambda k: ours[k][0])
    tot_ms, launches = ours[dom]
    bands_per_launch = nb * steps / max(launches, 1)
    alg = per_band_bytes(d, elem)[dom] * bands_per_launch + (v_bytes if dom == "z_vloc" else 0)
    avg_s = tot_ms / max(launches, 1) / 1e3
    achieved = alg / avg_s / 1e9
    traffic = None
    if traffic_per_band and dom in traffic_per_band:
        traffic = traffic_per_band[dom] * bands_per_launch
    return {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm, "peak_kind": peak_kind, "traffic": traffic, "alg_bytes_per_launch": alg,
            "avg_launch_ms": avg_s * 1e3, "bands_per_launch": bands_per_launch}


def load_traffic(name):
    """Per-band DRAM bytes of the local kernels from a committed ncu summary (profiles/), or None."""
    path = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(path):
        return None
    with open(path) as f:
        tj = json.load(f)
    return {k: v["bytes_per_band"] for k, v in tj.items() if isinstance(v, dict) and "bytes_per_band" in v}


def run_ours(args, world, rank, local, dist):
    import torch

    from cpw2000_b200 import _lib
    from cpw2000_b200 import hk_psi as H

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    w = configs.si216_cubic()
    nk = max(1, min(args.eig_kpoints, len(w.kpoints)))
    inputs = [configs.kpoint_inputs(w, k, with_hamsm=True) for k in range(nk if args.eig else 1)]
    d = inputs[0]
    m = d["mtxd"]
    psi_h = configs.random_psi(m, NB, 2024 + rank)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def timed(ctx, psi, hpsi, steps, warmup):
        for _ in range(warmup):
            ctx.hk_psi(psi, hpsi)
        barrier()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        ctx.timing_begin()
        for a, b in evs:
            a.record()
            ctx.hk_psi(psi, hpsi)
            b.record()
        barrier()
        stages = ctx.timing_end()
        ms = sum(a.elapsed_time(b) for a, b in evs) / steps
        return ms, stages

    hbm, _, peak_kind = measured_peaks()
    psi = torch.from_numpy(np.ascontiguousarray(psi_h.T)).to(dev).t()
    hpsi = torch.empty((NB, m), dtype=torch.complex128, device=dev).t()
    results = {}
    sampler = ClockSampler(local)
    sampler.start()
    hpsi64 = None
    i8_rel = None
    for prec_name, prec, slices in (("fp64", H.FP64, 0), ("mixed", H.MIXED, 0), ("mixed_tc", H.MIXED_TC, 0),
                                    ("fp64_i8", H.FP64, 7)):
        ctx = H.Context(local, precision=prec).setup(d)
        ctx.set_slab_budget(8 << 30)
        if slices:
            ctx.set_projector_slices(slices)
        ms, stages = timed(ctx, psi, hpsi, args.steps, args.warmup)
        ctx.synchronize()
        results[prec_name] = (max_over_ranks(ms), stages)
        if prec_name == "fp64":
            hpsi64 = hpsi.clone()
        elif prec_name == "fp64_i8":
            i8_rel = float((hpsi - hpsi64).abs().max() / hpsi64.abs().max())
        ctx.close()
    del hpsi64
    clocks = sampler.stop()

    # e2e through the reference-facing C ABI with pinned host arrays
    psi_pin = torch.from_numpy(np.asfortranarray(psi_h).ravel(order="F").view(np.float64)).pin_memory()
    hpsi_pin = torch.empty_like(psi_pin).pin_memory()
    kgv = np.asfortranarray(d["kgv"], dtype=np.int32)
    isort = np.ascontiguousarray(d["isort"], dtype=np.int32)
    ekpg = np.ascontiguousarray(d["ekpg"])
    vscr = np.ascontiguousarray(d["vscr"])
    kmscr = np.ascontiguousarray(d["kmscr"], dtype=np.int32)
    anlga = np.asfortranarray(d["anlga"])
    xnlkb = np.ascontiguousarray(d["xnlkb"])
    L = _lib.lib()
    import ctypes as C
    DP = C.POINTER(C.c_double)
    pp = C.cast(C.c_void_p(psi_pin.data_ptr()), DP)
    hp = C.cast(C.c_void_p(hpsi_pin.data_ptr()), DP)
    ri = _lib.iref

    def dropin(lnew):
        lv = C.c_int(lnew)
        st = L.cpw_b200_hk_psi_c16(ri(m), ri(NB), pp, hp, C.byref(lv), ri(d["ng"]), _lib.iptr(kgv),
                                   _lib.dptr(ekpg), _lib.iptr(isort), _lib.dptr(vscr), _lib.iptr(kmscr),
                                   _lib.zptr(anlga), _lib.dptr(xnlkb), ri(d["nanl"]), ri(m), ri(NB),
                                   ri(d["nanl"]), ri(d["ng"]), ri(vscr.size))
        _lib.check(st)

    dropin(1)
    for _ in range(args.warmup):
        dropin(0)
    barrier()
    t_e2e = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        dropin(0)
        t_e2e.append(time.perf_counter() - t0)
    barrier()
    e2e_ms = max_over_ranks(1e3 * sum(t_e2e) / len(t_e2e))
    # the drop-in's result against the device path (same operator, same inputs)
    ref_dev = torch.empty_like(hpsi)
    ctx = H.Context(local).setup(d)
    ctx.set_slab_budget(8 << 30)
    ctx.hk_psi(psi, ref_dev)
    ctx.synchronize()
    ctx.close()
    got = torch.from_numpy(hpsi_pin.numpy().view(np.complex128).reshape((NB, m))).to(dev).t()
    e2e_rel = float((got - ref_dev).abs().max() / ref_dev.abs().max())
    del psi_pin, hpsi_pin, got, ref_dev

    ms64, st64 = results["fp64"]
    msmx, stmx = results["mixed"]
    mstc, sttc = results["mixed_tc"]
    value = world * NB / (ms64 / 1e3)
    n1, n2, n3 = (int(v) for v in d["kmscr"][3:6])
    roof64 = roofline_of(st64, args.steps, NB, d, 16, n1 * n2 * n3 * 8, hbm, peak_kind,
                         load_traffic("traffic_si216_fp64.json"))
    rooftc = roofline_of(sttc, args.steps, NB, d, 8, n1 * n2 * n3 * 4, hbm, peak_kind,
                         load_traffic("traffic_si216_mixed_tc.json"))
    total_stage_ms = sum(v[0] for v in st64.values())
    line = {
        "metric": METRIC, "value": value, "unit": "bands/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms64, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Gaussian pseudopotentials, random complex128 wavefunctions)",
        "config": {**workload_desc(d), "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "precision": "fp64 drop-in (FP64 pruned FFT, FP64 projector products)"},
        "e2e": {"value": world * NB / (e2e_ms / 1e3), "unit": "bands/s", "h2d_bytes_per_step": 16 * m * NB,
                "d2h_bytes_per_step": 16 * m * NB, "ms_per_step": e2e_ms,
                "path": "cpw_b200_hk_psi_c16 (drop-in C ABI) on pinned host arrays; inputs compared by content "
                        "on the host every call", "max_rel_diff_vs_device_path": e2e_rel},
        "roofline": roof64,
        "stages_fp64": {k: {"ms_per_step": v[0] / args.steps, "launches": v[1],
                            "share": v[0] / total_stage_ms if total_stage_ms else None}
                        for k, v in st64.items() if v[1]},
        "mixed": {"value": world * NB / (msmx / 1e3), "ms_per_step": msmx,
                  "speedup_vs_fp64": ms64 / msmx,
                  "precision": "FP32 pruned FFT + V_loc, FP64 projector GEMMs",
                  "stages": {k: v[0] / args.steps for k, v in stmx.items() if v[1]}},
        "mixed_tc": {"value": world * NB / (mstc / 1e3), "ms_per_step": mstc,
                     "speedup_vs_fp64": ms64 / mstc,
                     "precision": "FP32 pruned FFT + V_loc, split-TF32 tcgen05 projector GEMMs "
                                  "(hi.hi + hi.lo + lo.hi, FP64 drain of short FP32 chains)",
                     "stages": {k: v[0] / args.steps for k, v in sttc.items() if v[1]},
                     "roofline": rooftc},
        "fp64_i8_projectors": {
            "value": world * NB / (results["fp64_i8"][0] / 1e3), "ms_per_step": results["fp64_i8"][0],
            "speedup_vs_fp64": ms64 / results["fp64_i8"][0], "max_rel_diff_vs_fp64": i8_rel,
            "precision": "FP64 pruned FFT + V_loc, projector products in the FP64-accurate int8 tensor-core "
                         "Ozaki GEMM (7 slices; cpw_b200_set_projector_slices)",
            "stages": {k: v[0] / args.steps for k, v in results["fp64_i8"][1].items() if v[1]}},
        "gpu_launches": int(sum(v[1] for k, v in st64.items() if k in ("inv_xy", "z_vloc", "fwd_xy"))),
        "library_launches": {"cublas_zgemm": int(st64["nl_proj"][1] + st64["nl_expand"][1])},
        "clocks": clocks,
    }
    line["si64"] = si64_throughput(local, max(3, args.steps // 2), 3)
    line["kbatch"] = kbatch_throughput(local, max(3, args.steps // 2), 2)
    if args.eig:
        line["time_to_eigvals"] = time_to_eigvals(w, inputs, local, repeats=args.eig_repeats,
                                                  workers=min(args.eig_workers, len(inputs)),
                                                  budget_s=args.eig_budget)
    if rank == 0 and world == 1:
        from oracle import c_ref
        blas = c_ref.use_blas(True)
        rate, cores = cpu_reference_rate(d, REF_SAMPLE, repeats=2)
        line["cpu_baseline"] = {"value": rate, "unit": "bands/s", "cores": cores, "kind": "port",
                                "sample": f"{REF_SAMPLE} of {NB} bands, best of 2, C+OpenMP restatement of "
                                          f"hk_psi_c16 (own pruned FFT; projector products {gemm_text(blas)}), "
                                          f"{cores} threads"}
    if rank == 0:
        print(json.dumps(line), flush=True)


def si64_throughput(local, steps, warmup):
    """H|psi> of the Si64 workload (the 64-atom cubic cell: 26,529 PW, 96^3, 256 projectors, 160 bands): FP64 and
    MIXED_TC bands/s, device-resident, L2 flushed (256 MiB memset) before each timed step."""
    import torch

    from cpw2000_b200 import hk_psi as H
    dev = torch.device("cuda", local)
    d = configs.kpoint_inputs(configs.si64_cubic(), 0)
    psi = torch.from_numpy(np.ascontiguousarray(configs.random_psi(d["mtxd"], NB64, 2024).T)).to(dev).t()
    hpsi = torch.empty_like(psi)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    out = {"workload": f"si64 cubic, Ecut 16 Ha, Gamma, mtxd {d['mtxd']}, 96^3, {d['nanl']} projectors, "
                       f"{NB64} bands"}
    for name, prec in (("fp64", H.FP64), ("mixed_tc", H.MIXED_TC)):
        ctx = H.Context(local, precision=prec).setup(d)
        ctx.set_slab_budget(4 << 30)
        for _ in range(warmup):
            ctx.hk_psi(psi, hpsi)
        torch.cuda.synchronize()
        ts = []
        for _ in range(steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            ctx.hk_psi(psi, hpsi)
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        ctx.close()
        ms = statistics.median(ts)
        out[name] = {"bands_per_s": NB64 / (ms / 1e3), "ms_per_step": ms}
    return out


def run_gemm(args, local):
    """The eigensolver's basis-product shapes on the int8 tensor cores (cpw_b200_zgemm_i8, 7 slices)
    against cuBLAS ZGEMM (torch complex128 matmul): median ms of --steps calls after --warmup."""
    import ctypes as C

    import torch

    from cpw2000_b200 import _lib
    from cpw2000_b200 import hk_psi as H
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ctx = H.Context(local)
    L = _lib.lib()
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    st = stream.cuda_stream
    shapes = [("C", 1000, 180, 88951), ("N", 88951, 180, 1000), ("C", 180, 180, 88951), ("N", 88951, 490, 1160),
              ("C", 864, 480, 88951), ("N", 88951, 480, 864)]
    out = {"mode": "gemm", "slices": args.slices, "shapes": []}
    chosen = [shapes[args.shape_index]] if args.shape_index >= 0 else shapes[: args.nshapes]
    for ta, m, n, k in chosen:
        a = torch.randn((k, m) if ta == "C" else (m, k), dtype=torch.complex128, device=dev)
        a = a.t().contiguous().t()                   # column-major
        b = torch.randn((k, n), dtype=torch.complex128, device=dev).t().contiguous().t()
        c = torch.zeros((n, m), dtype=torch.complex128, device=dev).t()
        lda = a.shape[0]

        def ours():
            _lib.check(L.cpw_b200_zgemm_i8(ctx.handle, ord(ta), m, n, k, C.c_void_p(a.data_ptr()), lda,
                                           C.c_void_p(b.data_ptr()), k, 1.0, 0, C.c_void_p(c.data_ptr()), m,
                                           args.slices, C.c_void_p(st)))

        def theirs():
            return (a.conj().t() if ta == "C" else a) @ b

        res = {}
        for name, fn in (("i8", ours), ("cublas", theirs)):
            for _ in range(args.warmup):
                fn()
            torch.cuda.synchronize()
            ts = []
            for _ in range(args.steps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                fn()
                e1.record()
                torch.cuda.synchronize()
                ts.append(e0.elapsed_time(e1))
            ms = statistics.median(ts)
            res[name] = {"ms": ms, "tflops_complex": 8.0 * m * n * k / (ms / 1e3) / 1e12}
        ctx.synchronize()
        ref = theirs()
        res["rel_err"] = float((c - ref).abs().max() / ref.abs().max())
        out["shapes"].append({"op": ta, "m": m, "n": n, "k": k, **res})
        del a, b, c, ref
        torch.cuda.empty_cache()
    # the subspace eigensolve size of the Si216 Ritz steps: torch.linalg.eigh (cuSOLVER) for reference
    n = 1160
    x = torch.randn((n, n), dtype=torch.complex128, device=dev)
    hm = x + x.conj().t()
    for _ in range(2):
        torch.linalg.eigh(hm)
    torch.cuda.synchronize()
    ts = []
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.linalg.eigh(hm)
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    out["eigh_1160_ms"] = statistics.median(ts)
    ctx.close()
    print(json.dumps(out), flush=True)


def run_tte(args, local):
    """time_to_eigvals alone (the bench line's key of that name), for studies of the eigensolver."""
    import torch
    torch.cuda.set_device(local)
    w = configs.si216_cubic()
    nk = max(1, min(args.eig_kpoints, len(w.kpoints)))
    inputs = [configs.kpoint_inputs(w, k, with_hamsm=True) for k in range(nk)]
    out = time_to_eigvals(w, inputs, local, repeats=args.eig_repeats, workers=min(args.eig_workers, nk),
                          budget_s=args.eig_budget, prioritise=bool(args.eig_priorities))
    print(json.dumps({"mode": "tte", **out}), flush=True)


def run_kset(args, local):
    """The eigensolver on the first --eig-kpoints k-points of the Si216 workload, --eig-workers in
    flight, --icmax outer iterations, in the --precision form, with --env KEY=VALUE switches set
    while it runs (--ipr 2 prints every k-point's phase times): the set's wall time and H|psi>
    products. Studies of the eigensolver's switches under several k-points in flight."""
    import torch

    from cpw2000_b200 import hk_psi as H
    from cpw2000_b200 import kpoints
    torch.cuda.set_device(local)
    w = configs.si216_cubic()
    nk = max(1, min(args.eig_kpoints, len(w.kpoints)))
    inputs = [configs.kpoint_inputs(w, k, with_hamsm=True) for k in range(nk)]
    env = dict(kv.split("=", 1) for kv in args.env)
    prec = {"fp64": H.FP64, "mixed": H.MIXED, "mixed_tc": H.MIXED_TC}[args.precision]
    res, sec = kpoints.eigensolve_kpoints(inputs, NB, workers=min(args.eig_workers, nk), precision=prec,
                                          icmax=args.icmax, device=local, mxdbnd=3 * NB, slab_budget=2 << 30,
                                          env=env, ipr=args.ipr)
    print(json.dumps({"mode": "kset", "precision": args.precision, "kpoints": nk, "in_flight": args.eig_workers,
                      "icmax": args.icmax, "env": env, "seconds": sec,
                      "hpsi_band_products": [int(r["ihkpsum"]) for r in res]}), flush=True)


def run_eig_profile(args, local):
    """One eigensolver run on the Si216 Gamma point in one precision form (--precision), --icmax
    outer iterations, for ncu launch lists of the eigensolver's kernels."""
    import torch

    from cpw2000_b200 import ditsp as E
    from cpw2000_b200 import hk_psi as H
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    d = configs.kpoint_inputs(configs.si216_cubic(), 0, with_hamsm=True)
    nb = 480
    prec = {"fp64": H.FP64, "mixed": H.MIXED, "mixed_tc": H.MIXED_TC}[args.precision]
    ctx = H.Context(local, precision=prec).setup(d)
    ctx.set_slab_budget(8 << 30)
    P = torch.zeros((3 * nb, d["mtxd"]), dtype=torch.complex128, device=dev).t()
    HP = torch.zeros_like(P)
    t0 = time.perf_counter()
    r = E.eigensolve(ctx, P, HP, nb, d["mtxds"], d["hamsm"], d["hdiag"], epspsi=1e-5, icmax=args.icmax,
                     ipr=args.ipr)
    torch.cuda.synchronize()
    print(json.dumps({"mode": "eigprof", "precision": args.precision, "icmax": args.icmax,
                      "seconds": time.perf_counter() - t0, "ihkpsum": r["ihkpsum"]}), flush=True)
    ctx.close()


def run_profile(args, local):
    """Device path only, for ncu: --bands bands of the --pworkload workload (Si216 or Si64, Gamma),
    --steps + --warmup calls."""
    import torch

    from cpw2000_b200 import hk_psi as H
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    w = {"si216": configs.si216_cubic, "si64": configs.si64_cubic}[args.pworkload]()
    d = configs.kpoint_inputs(w, 0)
    nb = args.bands
    psi = torch.from_numpy(np.ascontiguousarray(configs.random_psi(d["mtxd"], nb, 5).T)).to(dev).t()
    hpsi = torch.empty((nb, d["mtxd"]), dtype=torch.complex128, device=dev).t()
    ctx = H.Context(local, precision={"fp64": H.FP64, "mixed": H.MIXED, "mixed_tc": H.MIXED_TC}[args.precision]).setup(d)
    ctx.set_slab_budget(8 << 30)
    if args.nl_slices:
        ctx.set_projector_slices(args.nl_slices)
    for _ in range(args.warmup + args.steps):
        ctx.hk_psi(psi, hpsi)
    torch.cuda.synchronize()
    print(json.dumps({"mode": "profile", "bands": nb, "precision": args.precision, "calls": args.warmup + args.steps}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--mode", choices=["bench", "profile", "eig", "gemm", "eigprof", "tte", "kset"], default="bench")
    ap.add_argument("--env", action="append", default=[], help="kset mode: KEY=VALUE switch (repeatable)")
    ap.add_argument("--slices", type=int, default=7, help="gemm mode: int8 slices")
    ap.add_argument("--nshapes", type=int, default=6, help="gemm mode: how many of the shapes")
    ap.add_argument("--shape-index", type=int, default=-1, help="gemm mode: this one shape only (0-5)")
    ap.add_argument("--workload", choices=["si216", "si64", "zb64"], default="si216", help="eig mode workload")
    ap.add_argument("--icmax", type=int, default=200, help="eig mode: outer iterations at most")
    ap.add_argument("--epspsi", type=float, default=1e-5, help="eig mode: residual tolerance")
    ap.add_argument("--with-cholqr", action="store_true", help="eig mode: also FP64 with Cholesky QR")
    ap.add_argument("--variants", default="mixed_tc", help="eig mode: comma list of fp64_cholqr, mixed, mixed_tc "
                    "(fp64 always runs first as the reference)")
    ap.add_argument("--icmax-ref", type=int, default=0, help="eig mode: outer iterations of the FP64 reference run "
                    "(default: --icmax)")
    ap.add_argument("--ipr", type=int, default=0, help="eig mode: eigensolver print level (2: phase timers)")
    ap.add_argument("--save-traces", default="", help="eig mode: directory for the iteration traces (.npy)")
    ap.add_argument("--bands", type=int, default=NB, help="profile mode: bands per call")
    ap.add_argument("--pworkload", choices=["si216", "si64"], default="si216", help="profile mode workload")
    ap.add_argument("--nl-slices", type=int, default=0, help="profile mode: int8 projector slices (0: form default)")
    ap.add_argument("--precision", choices=["fp64", "mixed", "mixed_tc"], default="fp64", help="profile mode precision")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--eig", type=int, default=None, help="also measure time-to-eigvals (1) or not (0); default 1 on "
                    "one GPU, 0 on several (the replicas' H|psi> scaling run stays short)")
    ap.add_argument("--eig-repeats", type=int, default=3, help="repeats of the time-to-eigvals sets (median)")
    ap.add_argument("--eig-kpoints", type=int, default=4, help="k-points of the Si216 workload solved (Gamma first)")
    ap.add_argument("--eig-workers", type=int, default=4, help="k-points in flight during the eigensolver sets")
    ap.add_argument("--eig-budget", type=float, default=560.0, help="seconds the eigensolver repeats may take")
    ap.add_argument("--eig-priorities", type=int, default=0, help="later eigensolver repeats: stream priority by the "
                    "first repeat's per-k iteration counts (1) or equal priorities (0)")
    args = ap.parse_args()
    world, rank, local, dist = dist_setup(args)
    if args.eig is None:
        args.eig = 1 if world == 1 else 0
    try:
        if args.mode == "profile":
            run_profile(args, local)
        elif args.mode == "eig":
            run_eig_study(args, local)
        elif args.mode == "gemm":
            run_gemm(args, local)
        elif args.mode == "eigprof":
            run_eig_profile(args, local)
        elif args.mode == "tte":
            run_tte(args, local)
        elif args.mode == "kset":
            run_kset(args, local)
        elif args.impl == "reference":
            run_reference(args, rank)
        else:
            run_ours(args, world, rank, local, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
