"""Generate the committed fixtures of tests/golden from the oracle.

Run from the repository root:  python tests/golden/make_golden.py
The fixtures are regression vectors of the oracle on seeded synthetic inputs
(the reference has no function-level golden vectors to copy).
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from cpw2000_b200 import configs  # noqa: E402
from oracle import ditsp as D  # noqa: E402
from oracle import hk_psi as O  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    r = D.Ran2()
    s = [-1]
    vals = [r(s) for _ in range(16)]
    with open(os.path.join(HERE, "ran2_seed_minus1.json"), "w") as f:
        json.dump({"seed": -1, "values": vals}, f, indent=1)
    w = configs.small_test()
    d = configs.kpoint_inputs(w, 1)
    psi = configs.random_psi(d["mtxd"], 4, 21)
    hp = O.hk_psi_c16(d["mtxd"], 4, psi, d["ekpg"], d["isort"], d["vscr"], d["kmscr"], d["kgv"], d["anlga"],
                      d["xnlkb"])
    np.savez_compressed(os.path.join(HERE, "hkpsi_small.npz"), mtxd=d["mtxd"], psi=psi, hpsi=hp)


if __name__ == "__main__":
    main()
