"""Oracle states of the 1024-body pile (scene configuration 2) at steps 0, 75, 150 and 225 of
its 300-step trajectory, for the CPU reference arm of bench.py, which times oracle steps from
each of them (a step's cost grows as the pile settles into contact).

Run from the repository root:  python tests/golden/make_c2_states.py
Writes tests/golden/c2_states.npz (A0, p0, Adot, pdot and the dq warm start per state)."""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from abd_warp_b200 import scenes  # noqa: E402

STEPS = (0, 75, 150, 225)


def main():
    bodies, prm, _ = scenes.make_config(2)
    o = oracle.Oracle(scenes.flatten_bodies(bodies), prm)
    out = {"steps": np.array(STEPS)}
    t0 = time.time()
    for s in range(max(STEPS) + 1):
        if s in STEPS:
            st = o.get_state()
            for k in ("A0", "p0", "Adot", "pdot", "dq"):
                out[f"s{s}_{k}"] = st[k]
            print(f"state at step {s} ({time.time() - t0:.0f} s)", flush=True)
        if s < max(STEPS):
            o.step()
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "c2_states.npz"), **out)


if __name__ == "__main__":
    main()
