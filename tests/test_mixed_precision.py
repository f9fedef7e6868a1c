"""Mixed precision (FP32 PCG inside FP64 iterative refinement), in the oracle.

The refinement converges when cond(H) eps_FP32 < 1.  The step's systems meet that until
bodies touch; then the barrier Hessian pushes cond(H) to ~1e10 and the FP32 inner solves stop
reducing the residual.  These tests pin both halves of that measurement, which is why the CUDA
library accepts FP64 only (precision 1 is rejected at creation)."""
import dataclasses

import numpy as np

import oracle
from abd_warp_b200 import scenes


def _run(bodies, prm, precision, nsteps):
    o = oracle.Oracle(scenes.flatten_bodies(bodies), dataclasses.replace(prm, precision=precision))
    infos = [o.step() for _ in range(nsteps)]
    return o.get_state(), infos


def test_mixed_matches_fp64_before_contact():
    bodies, prm, _ = scenes.make_config(0)
    ref, ri = _run(bodies, prm, 0, 2)
    got, gi = _run(bodies, prm, 1, 2)
    assert all(i["n_active"] == 0 for i in gi)
    assert all(i["refine_iters"] > 0 for i in gi)  # the FP32 solves ran
    err = np.abs(got["p0"] - ref["p0"]).max() / np.abs(ref["p0"]).max()
    assert err <= 1e-9, err


def test_mixed_diverges_in_contact():
    bodies, prm, _ = scenes.make_config(1)
    ref, _ = _run(bodies, prm, 0, 6)
    got, gi = _run(bodies, prm, 1, 6)
    assert any(i["n_active"] > 0 for i in gi)
    err = np.abs(got["p0"] - ref["p0"]).max() / np.abs(ref["p0"]).max()
    energy = gi[-1]["energy"]
    assert err > 1e-3 or not np.isfinite(energy), (err, energy)
