"""CPU test: the C + OpenMP restatement of hk_psi_c16 (oracle/c/hkpsi_ref.c, the CPU
baseline of the bench) against the numpy restatement (oracle/hk_psi.py).

Both restate Src/hk_psi/reference/hk_psi_c16.f90:28-241; they differ only in FFT
algorithm and summation order, so they agree to rounding (<= 1e-12 of max|H psi|),
on the Si2 fcc cell (32^3 box) and on a triclinic cell with a non-cubic box
(24 x 20 x 18, leading dimension id = 25), with 1 and with several threads, with the
projector products in its own loops and in numpy's bundled OpenBLAS zgemm.
"""
import numpy as np
import pytest

from cpw2000_b200 import configs
from oracle import c_ref
from oracle import hk_psi as O

TOL64 = 1e-12


def _both(wname, ik, nb, seed, nthreads):
    w = configs.WORKLOADS[wname]()
    d = configs.kpoint_inputs(w, ik)
    m = d["mtxd"]
    psi = configs.random_psi(m, nb, seed)
    args = (m, nb, psi, d["ekpg"], d["isort"], d["vscr"], d["kmscr"], d["kgv"], d["anlga"], d["xnlkb"])
    return O.hk_psi_c16(*args), c_ref.hk_psi_c16(*args, nthreads=nthreads), d


@pytest.mark.parametrize("wname,ik,nb,nthreads", [("si2", 0, 4, 1), ("si2", 3, 5, 4), ("small", 1, 3, 1),
                                                  ("small", 0, 6, 3)])
def test_c_restatement_matches_numpy_oracle(wname, ik, nb, nthreads):
    ref, got, d = _both(wname, ik, nb, 40 + ik, nthreads)
    err = float(np.abs(got - ref).max() / np.abs(ref).max())
    assert err < TOL64, f"{wname} k{ik}: relative difference {err:.3e}"


def test_c_restatement_box_is_not_cubic():
    # the second case really exercises id > n1 and unequal n1, n2, n3
    d = configs.kpoint_inputs(configs.WORKLOADS["small"](), 1)
    n1, n2, n3, ident = (int(v) for v in d["kmscr"][3:7])
    assert len({n1, n2, n3}) == 3 and ident > n1


@pytest.mark.parametrize("wname,ik,nb", [("si2", 2, 5), ("small", 1, 4)])
def test_c_restatement_with_optimised_blas(wname, ik, nb):
    if not c_ref.use_blas(True):
        pytest.skip("numpy ships no 64-bit-integer OpenBLAS here")
    try:
        ref, got, _ = _both(wname, ik, nb, 70 + ik, 2)
    finally:
        c_ref.use_blas(False)
    err = float(np.abs(got - ref).max() / np.abs(ref).max())
    assert err < TOL64, f"{wname} k{ik}: relative difference {err:.3e}"
