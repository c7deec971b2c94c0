"""The gfortran-mangled drop-ins driven from compiled C, as a Fortran caller drives them.

tests/harness/dropin_harness.c is built with gcc against libcpwb200.so and run
as a child process. It passes lnewanl from read-only memory (gfortran's literal
.TRUE. at Src/ALFA/berry_derivative.f90:229 lives in read-only storage), so a
library that wrote the flag would crash the child with SIGSEGV. Between its
two hk_psi_c16_ calls it changes anlga in place and passes lnewanl .FALSE.:
the second result must follow the new projectors (the library compares them
by content). ditsp_c16_ then solves with the changed projectors. Every result
is checked against the oracle: H|psi> to 1e-12 of max|H psi|, eigenvalues to
1e-8 Ha of the dense ground truth.
"""
import os
import subprocess

import numpy as np
import pytest

from cpw2000_b200 import configs
from oracle import hk_psi as O

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
PKG = os.path.join(ROOT, "cpw2000_b200")
SRC = os.path.join(HERE, "harness", "dropin_harness.c")


def build_harness(outdir):
    exe = os.path.join(outdir, "dropin_harness")
    subprocess.run(["gcc", "-O1", "-std=c11", "-Wall", "-o", exe, SRC, "-L" + PKG, "-lcpwb200",
                    "-Wl,-rpath," + PKG], check=True, capture_output=True, text=True)
    return exe


def test_harness_builds_and_links(tmp_path):
    # CPU: the harness compiles and every mangled symbol it calls resolves in the library
    exe = build_harness(str(tmp_path))
    assert os.path.exists(exe)


def _write_inputs(dirn, d, psi, anl1, anl2, mxdsml, mxdbnd, neig):
    m, nb = psi.shape
    with open(os.path.join(dirn, "dims.txt"), "w") as f:
        f.write(f"{m} {nb} {d['ng']} {d['nanl']} {d['mtxds']} {neig} {mxdsml} {mxdbnd}\n")
        f.write(" ".join(str(int(v)) for v in d["kmscr"]) + "\n")
    hamsm = np.zeros((mxdsml, mxdsml), np.complex128, order="F")
    hamsm[: d["mtxds"], : d["mtxds"]] = d["hamsm"][: d["mtxds"], : d["mtxds"]]
    arrays = {"kgv.bin": np.asfortranarray(d["kgv"], dtype=np.int32),
              "isort.bin": np.asarray(d["isort"], dtype=np.int32),
              "ekpg.bin": np.asarray(d["ekpg"], dtype=np.float64),
              "vscr.bin": np.asarray(d["vscr"], dtype=np.float64),
              "anl1.bin": np.asfortranarray(anl1), "anl2.bin": np.asfortranarray(anl2),
              "xnl.bin": np.asarray(d["xnlkb"], dtype=np.float64), "psi.bin": np.asfortranarray(psi),
              "hamsm.bin": hamsm, "hdiag.bin": np.asarray(d["hdiag"], dtype=np.float64)}
    for name, a in arrays.items():
        with open(os.path.join(dirn, name), "wb") as f:
            f.write(a.tobytes(order="F"))


@pytest.mark.gpu
def test_mangled_dropins_read_only_lnewanl_and_changed_projectors(cuda, tmp_path):
    w = configs.si2_fcc()
    d = configs.kpoint_inputs(w, 2, with_hamsm=True)
    m, nb, neig = d["mtxd"], 5, 8
    psi = configs.random_psi(m, nb, 61)
    anl1 = np.asfortranarray(d["anlga"])
    anl2 = np.asfortranarray(d["anlga"] * (0.6 + 0.3j))
    mxdsml, mxdbnd = max(d["mtxds"], 3 * neig), 3 * neig
    dirn = str(tmp_path)
    _write_inputs(dirn, d, psi, anl1, anl2, mxdsml, mxdbnd, neig)
    exe = build_harness(dirn)
    r = subprocess.run([exe, dirn], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, f"harness failed (rc {r.returncode}): {r.stdout[-2000:]} {r.stderr[-2000:]}"
    assert "harness ok: lnewanl flags 1 0" in r.stdout

    def rd(name, shape):
        return np.fromfile(os.path.join(dirn, name), dtype=np.complex128).reshape(shape, order="F")

    ref1 = O.hk_psi_c16(m, nb, psi, d["ekpg"], d["isort"], d["vscr"], d["kmscr"], d["kgv"], anl1, d["xnlkb"])
    ref2 = O.hk_psi_c16(m, nb, psi, d["ekpg"], d["isort"], d["vscr"], d["kmscr"], d["kgv"], anl2, d["xnlkb"])
    for got, ref in ((rd("hpsi1.bin", (m, nb)), ref1), (rd("hpsi2.bin", (m, nb)), ref2)):
        assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-12
    ifail, ne = (int(v) for v in open(os.path.join(dirn, "ditsp.txt")).read().split())
    assert ifail == 0 and ne >= neig
    ei = np.fromfile(os.path.join(dirn, "ei.bin"), dtype=np.float64)
    dense = np.linalg.eigvalsh(O.dense_h(m, d["ekpg"], d["isort"], d["vscr"], d["kmscr"], d["kgv"], anl2,
                                         d["xnlkb"]))
    assert np.abs(ei[:ne] - dense[:ne]).max() < 1e-8
