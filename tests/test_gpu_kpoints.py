"""k-points of one crystal solved concurrently (cpw2000_b200.kpoints): every k-point's Ritz
values equal those of the serial single-context run (each solve is the same deterministic
eigensolver on its own context and stream), in input order."""
import numpy as np
import pytest

from cpw2000_b200 import configs, kpoints

pytestmark = pytest.mark.gpu


def test_concurrent_kpoints_match_serial(cuda):
    w = configs.si8_cubic_kbatch(nk=6)
    inputs = [configs.kpoint_inputs(w, k, nbands=24, with_hamsm=True) for k in range(6)]
    serial, _ = kpoints.eigensolve_kpoints(inputs, 24, workers=1, icmax=30)
    conc, _ = kpoints.eigensolve_kpoints(inputs, 24, workers=4, icmax=30)
    for a, b in zip(serial, conc):
        assert a["neig"] == b["neig"] and a["ihkpsum"] == b["ihkpsum"]
        assert np.abs(a["ei"] - b["ei"]).max() <= 1e-12
    # distinct k-points give distinct spectra: the results are not mixed up
    assert np.abs(serial[0]["ei"][:8] - serial[1]["ei"][:8]).max() > 1e-6


def test_prioritised_kpoints_match_serial(cuda):
    # stream priorities and queue order change only when each solve runs, not what it computes;
    # per-k iteration limits apply to their own k-point
    w = configs.si8_cubic_kbatch(nk=4)
    inputs = [configs.kpoint_inputs(w, k, nbands=24, with_hamsm=True) for k in range(4)]
    serial, _ = kpoints.eigensolve_kpoints(inputs, 24, workers=1, icmax=[30, 25, 30, 25])
    prio, _ = kpoints.eigensolve_kpoints(inputs, 24, workers=2, icmax=[30, 25, 30, 25], priorities=[0, -3, -1, -2])
    for a, b in zip(serial, prio):
        assert a["neig"] == b["neig"] and a["ihkpsum"] == b["ihkpsum"]
        assert np.abs(a["ei"] - b["ei"]).max() <= 1e-12
    with pytest.raises(ValueError):
        kpoints.eigensolve_kpoints(inputs, 24, workers=1, icmax=[30, 25])
