"""GPU test: the drop-in entry points' form chosen by environment.

hk_psi_c16_ and the other drop-ins take no context argument. A host code that links them in
place of the reference routines selects their precision form (CPW_B200_DROPIN_PRECISION) and
int8 projector products (CPW_B200_DROPIN_PROJECTOR_SLICES) when the library creates the drop-in
context. Each case runs in a fresh process, because that context lives for the whole process. The
results are checked against the oracle: FP64 with 7-slice int8 projector products within the FP64
tolerance (1e-12 of max|H psi|), MIXED_TC within the mixed tolerance (2e-5), and an unknown form
is refused with a message.
"""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import numpy as np
from cpw2000_b200 import configs
from cpw2000_b200 import hk_psi as H
from cpw2000_b200._lib import CpwB200Error
from oracle import hk_psi as O
d = configs.kpoint_inputs(configs.si2_fcc(), 3)
m, nb = d["mtxd"], 5
psi = configs.random_psi(m, nb, 61)
hpsi = np.zeros((m, nb), dtype=np.complex128, order="F")
try:
    H.hk_psi_c16(m, nb, psi, hpsi, True, d["ng"], np.asfortranarray(d["kgv"]), d["ekpg"], d["isort"], d["vscr"],
                 d["kmscr"], d["anlga"], d["xnlkb"], d["nanl"], m, nb, d["nanl"], d["ng"], d["vscr"].size)
except CpwB200Error as e:
    print("ERROR", e)
    raise SystemExit(0)
ref = O.hk_psi_c16(m, nb, psi, d["ekpg"], d["isort"], d["vscr"], d["kmscr"], d["kgv"], d["anlga"], d["xnlkb"])
print("RELERR", float(np.abs(hpsi - ref).max() / np.abs(ref).max()))
"""


def _child(env_extra):
    env = dict(os.environ)
    env.pop("CPW_B200_DROPIN_PRECISION", None)
    env.pop("CPW_B200_DROPIN_PROJECTOR_SLICES", None)
    env.update(env_extra)
    r = subprocess.run([sys.executable, "-c", CHILD], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return r.stdout.strip().splitlines()[-1]


@pytest.mark.parametrize("env,tol", [({"CPW_B200_DROPIN_PROJECTOR_SLICES": "7"}, 1e-12),
                                     ({"CPW_B200_DROPIN_PRECISION": "mixed_tc"}, 2e-5),
                                     ({"CPW_B200_DROPIN_PRECISION": "fp64"}, 1e-12)])
def test_dropin_form_from_environment(cuda, env, tol):
    out = _child(env)
    assert out.startswith("RELERR"), out
    assert float(out.split()[1]) < tol, out


def test_dropin_unknown_form_refused(cuda):
    out = _child({"CPW_B200_DROPIN_PRECISION": "fp16"})
    assert out.startswith("ERROR") and "CPW_B200_DROPIN_PRECISION" in out, out
