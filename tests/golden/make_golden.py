"""Generate the golden fixtures of tests/golden/ from the reference itself.

Runs the reference's own step (oracle/_ref/libref_fp{64,32}.so, built from the
reference sources by oracle/build_ref.py) on the seeded `tiny` organoid
(64x64 grid, 3 cells, zone_size 17) for 5 steps and stores the state after
step 1 and step 5, the areas, centroids and the per-cell velocity of step 5.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from multicellular_phase_field_active_gel_organoids_b200.params import CONFIGS  # noqa: E402
from oracle import refrun  # noqa: E402

STEPS = 5


def main():
    cfg = CONFIGS["tiny"]()
    for prec, dtype in (("fp64", np.float64), ("fp32", np.float32)):
        res = refrun.run_reference(cfg.params(), cfg.initial_state(dtype), STEPS, precision=prec,
                                   snapshots=[1], velocity=(prec == "fp64"))
        s1 = res["snapshots"][1]
        out = {"phi": res["phi"], "rho": res["rho"], "lum": res["lum"], "ECM": res["ECM"], "s": res["s"],
               "xc": res["xc"], "yc": res["yc"], "phi_1": s1["phi"], "rho_1": s1["rho"], "s_1": s1["s"],
               "steps": np.array(STEPS)}
        if res["velocity"] is not None:
            out["vx"], out["vy"] = res["velocity"]
        path = os.path.join(HERE, f"tiny_ref_{prec}.npz")
        np.savez_compressed(path, **out)
        print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()
