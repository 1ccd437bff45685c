"""Generates tests/golden/*.npz from the reference's own CoupLB headers.

Run in a checkout where the reference sources exist (oracle/_ref built by
`make -C oracle ref`):

    python tests/golden/make_golden.py

Every case is a seeded small problem; the inputs are regenerated from the same
seeds by tests/cases.py, so a fixture stores only the outputs of the
reference build (oracle/_ref/libcouplb_ref.so, no FMA contraction).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle.bindings import available  # noqa: E402
import cases  # noqa: E402


def main():
    if not available("ref"):
        sys.exit("oracle/_ref/libcouplb_ref.so is not built (make -C oracle ref)")
    for name, case in cases.LB_CASES.items():
        out = cases.run_lb_case_oracle(case, kind="ref")
        np.savez_compressed(os.path.join(HERE, f"lb_{name}.npz"), **out)
        print("wrote", name, {k: v.shape for k, v in out.items()})
    for name, case in cases.IBM_CASES.items():
        out = cases.run_ibm_case_oracle(case, kind="ref")
        np.savez_compressed(os.path.join(HERE, f"ibm_{name}.npz"), **out)
        print("wrote", name, {k: v.shape for k, v in out.items()})
    for name, case in cases.FIX_CASES.items():
        out = cases.run_fix_case(case, engine="ref")
        np.savez_compressed(os.path.join(HERE, f"fix_{name}.npz"), **out)
        print("wrote", name, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
