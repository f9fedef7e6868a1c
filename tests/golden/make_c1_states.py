"""Oracle trajectory of the 64-icosphere scene (scene configuration 1: 64 level-2 icospheres
over a ground box, 300 steps), for the GPU trajectory test: the step counters of every step
(Newton, Krylov and line-search iterations, culled and active contact counts, energy) and the
states, the warm start and the contact flags after steps 100, 200 and 300.

Run from the repository root:  python tests/golden/make_c1_states.py
Writes tests/golden/c1_trajectory.npz."""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from abd_warp_b200 import scenes  # noqa: E402

STEPS = 300
KEEP = (100, 200, 300)
INFO = ("newton_iters", "linear_iters", "ls_trials", "n_pt", "n_ee", "n_vg", "n_ij", "n_active", "energy", "alpha",
        "toi")


def main():
    bodies, prm, _ = scenes.make_config(1)
    o = oracle.Oracle(scenes.flatten_bodies(bodies), prm)
    out = {k: [] for k in INFO}
    t0 = time.time()
    for s in range(1, STEPS + 1):
        info = o.step()
        for k in INFO:
            out[k].append(info[k])
        if s in KEEP:
            st = o.get_state()
            for k in ("A0", "p0", "Adot", "pdot", "dq"):
                out[f"s{s}_{k}"] = st[k]
            out[f"s{s}_highlight"] = o.highlight()
            print(f"step {s} ({time.time() - t0:.0f} s): {info}", flush=True)
    arrays = {k: np.asarray(v) for k, v in out.items()}
    arrays["keep"] = np.array(KEEP)
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "c1_trajectory.npz"), **arrays)


if __name__ == "__main__":
    main()
