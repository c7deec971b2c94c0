"""CPU tests of the bench's measurement rules (bench.py), on synthetic data.

* Time to eigenvalues: the first outer iteration whose lowest occupied Ritz values are all within
  the tolerance; a set's time is its latest k-point; a k-point that never gets there voids the set.
* Later repeats stop each k-point 5 iterations past its own first repeat's success, capped at icmax.
* The longest-first stream priorities rank k-points by those counts.
* The roofline entry divides the dominant local kernel's algorithmic bytes per launch by its
  average launch time. The algorithmic bytes are ψ, the kept planes of the slab and Hψ; the V
  tile is counted once per launch of kernel B.
"""
import numpy as np
import pytest

import bench


def _trace(times, errs, nocc=3, e0=(-1.0, -0.5, 0.25), hk_per_it=100):
    # rows: elapsed s, xmax, nconv, H|psi> products, eigenvalues (nocc of them, offset by err)
    t = np.zeros((len(times), 4 + nocc))
    t[:, 0] = times
    t[:, 3] = hk_per_it * (np.arange(len(times)) + 1)
    t[:, 4:] = np.asarray(e0)[None, :] + np.asarray(errs)[:, None]
    return t


def test_first_within_and_set_time():
    ref = np.array([-1.0, -0.5, 0.25])
    a = {"trace": _trace([1.0, 2.0, 3.0, 4.0], [1e-3, 5e-6, 5e-7, 1e-9])}
    b = {"trace": _trace([1.5, 2.5, 3.5, 4.5], [1e-2, 1e-4, 2e-6, 1e-8])}
    assert bench.first_within(a["trace"], ref, 3, 1e-6) == 2
    assert bench.first_within(b["trace"], ref, 3, 1e-6) == 3
    assert bench.first_within(b["trace"], ref, 3, 1e-10) is None
    secs, its, hk = bench.set_time([a, b], [ref, ref], 3, 1e-6)
    assert secs == 4.5 and its == [3, 4] and hk == 300 + 400
    assert bench.set_time([a, b], [ref, ref], 3, 1e-10) == (None, None, None)


def test_only_the_occupied_values_count():
    ref = np.array([-1.0, -0.5])
    t = _trace([1.0, 2.0], [1e-9, 1e-9])
    t[:, 6] = 99.0            # an unoccupied Ritz value far off
    assert bench.first_within(t, ref, 2, 1e-6) == 0


def test_stop_iterations_and_priorities():
    ref = np.array([-1.0, -0.5, 0.25])
    fast = {"trace": _trace(np.arange(1, 11), [1e-3] * 2 + [1e-9] * 8)}          # met at iteration 3
    slow = {"trace": _trace(np.arange(1, 11), [1e-3] * 7 + [1e-9] * 3)}          # met at iteration 8
    never = {"trace": _trace(np.arange(1, 11), [1e-3] * 10)}
    per_k = bench.stop_iterations([fast, slow, never], [ref] * 3, 3, 1e-6, icmax=12)
    assert per_k == [3 + 5, min(12, 8 + 5), 12]     # the margin past the success, capped at icmax
    assert bench.longest_first_priorities([8, 12, 12, 3]) == [-1, -3, -2, 0]


def test_roofline_of_counts_algorithmic_bytes():
    d = {"mtxd": 1000, "kmscr": np.array([0, 0, 0, 8, 8, 8, 9]),
         "kgv": np.array([[0, 1, -1, 0, 0, 0, 0], [0, 0, 0, 1, -1, 0, 0], [0, 0, 0, 0, 0, 2, -2]]),
         "isort": np.arange(1, 8)}
    pb = bench.per_band_bytes(d, 16)
    nz, plane = 5, 64                               # kept z-planes 2 * kd3 + 1 with kd3 = 2
    assert pb["z_vloc"] == 2 * nz * plane * 16
    assert pb["inv_xy"] == 16 * 1000 + nz * plane * 16
    assert pb["fwd_xy"] == nz * plane * 16 + 2 * 16 * 1000
    # kernel B dominant: 2 steps of 40 bands in 4 launches of 20 bands, 1 ms each
    stages = {"inv_xy": (1.0, 4), "z_vloc": (4.0, 4), "fwd_xy": (2.0, 4)}
    r = bench.roofline_of(stages, 2, 40, d, 16, 512 * 8, 6538.0, "measured", {"z_vloc": 12345})
    alg = pb["z_vloc"] * 20 + 512 * 8
    assert r["kernel"] == "z_vloc" and r["bands_per_launch"] == 20
    assert r["alg_bytes_per_launch"] == alg
    assert r["achieved"] == pytest.approx(alg / 1e-3 / 1e9)
    assert r["frac"] == pytest.approx(r["achieved"] / 6538.0)
    assert r["traffic"] == 12345 * 20


def test_time_to_eigvals_bookkeeping_with_fake_solves(monkeypatch):
    # the whole time-to-eigenvalues procedure on the CPU, with the eigensolver and the forces
    # replaced by fakes: the error falls by 10 decades in 10 + 5k iterations for FP64 and in 6 + 3k
    # for the mixed form, down to a 1e-7 floor; later repeats must receive the per-k stop counts
    from types import SimpleNamespace

    from cpw2000_b200 import forces as FF
    from cpw2000_b200 import hk_psi as H
    from cpw2000_b200 import kpoints

    nocc = 2
    exact = np.array([-1.0, 0.5])
    calls = []

    def fake_solve(inputs, nbands, workers, precision, icmax, keep=0, priorities=None, **kw):
        calls.append((precision, icmax if np.isscalar(icmax) else list(icmax), priorities))
        res = []
        for k, _ in enumerate(inputs):
            n = icmax if np.isscalar(icmax) else icmax[k]
            slow = 10 + 5 * k if precision == H.FP64 else 6 + 3 * k
            it = np.arange(n)
            err = np.maximum(0.5 * 10.0 ** (-(it + 1) * 10.0 / slow), 0.0 if precision == H.FP64 else 1e-7)
            tr = np.zeros((n, 4 + 8))
            tr[:, 0] = 0.1 * (it + 1) * (2.0 if precision == H.FP64 else 1.0)
            tr[:, 3] = 50 * (it + 1)
            tr[:, 4:4 + nocc] = exact[None, :] + err[:, None]
            r = {"trace": tr, "converged": False}
            if keep:
                r["psi"] = np.zeros((4, keep))
            res.append(r)
        return res, float(tr[-1, 0])

    class FakeSystem:
        def __init__(self, w, d, psi, occ, device=0):
            self.ctx = SimpleNamespace(close=lambda: None)

    monkeypatch.setattr(kpoints, "eigensolve_kpoints", fake_solve)
    monkeypatch.setattr(FF, "HFSystem", FakeSystem)
    monkeypatch.setattr(FF, "forces", lambda s: (0.0, np.zeros((1, 3))))
    monkeypatch.setattr(FF, "to_cartesian", lambda f, adot: np.array([[0.1, 0.0, 0.0]]))
    w = SimpleNamespace(species=[SimpleNamespace(natom=1)], kpoints=[(0, 0, 0), (0.1, 0, 0)], adot=np.eye(3))
    inputs = [{"mtxd": 10}, {"mtxd": 11}]
    out = bench.time_to_eigvals(w, inputs, 0, repeats=3, workers=2, icmax=40, nocc=nocc, budget_s=1e9,
                                prioritise=True)
    assert out["repeats"] == 3
    # FP64 at 1e-8 within 8 iterations of k0 (slow 10) and 12 of k1 (slow 15): stop at 13 and 17
    assert out["icmax_later"]["fp64"] == [8 + 5, 12 + 5]
    assert out["stream_priorities_later"]["fp64"] == [0, -1]
    assert calls[2] == (H.FP64, [13, 17], [0, -1])
    # the mixed form reaches 1e-6 but not 1e-8 (floor 1e-7)
    assert out["mixed_tc"]["iterations_to_1e-6_ha"] == [4, 6]
    assert out["fp64"]["iterations_to_1e-6_ha"] == [6, 9]
    # times: FP64 0.2 s per iteration, mixed 0.1 s; the set time is the slower k-point's
    assert out["fp64"]["seconds_to_1e-6_ha"] == pytest.approx(1.8)
    assert out["mixed_tc"]["seconds_to_1e-6_ha"] == pytest.approx(0.6)
    assert out["speedup_mixed_tc_vs_fp64_at_1e-6"] == pytest.approx(3.0)
    assert out["force_max_abs_diff_ha_bohr"] == 0.0
