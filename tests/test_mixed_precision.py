"""Mixed precision, in the oracle: two designs, both measured, neither viable on contact systems.

* precision 2, FP32 PCG inside FP64 iterative refinement: converges while cond(H) eps_FP32 < 1,
  which the step's systems meet until bodies touch; then the barrier Hessian pushes cond(H) to
  ~1e10 and the FP32 inner solves stop reducing the residual.
* precision 1, FP64 flexible PCG with an FP32 preconditioner (the contact clusters' systems
  rounded to FP32 and inverted in FP32, applied in FP32): the Krylov iteration stays FP64, so
  FP32 rounding could only cost iterations -- but a contact cluster's system has a condition
  number far above 1 / eps_FP32, its FP32 inverse is no longer positive definite, b.M^-1 b
  comes out non-positive and the solve returns no step: the bodies freeze at first contact.

These tests pin both measurements, which is why the CUDA library accepts FP64 only."""
import dataclasses

import numpy as np

import oracle
from abd_warp_b200 import scenes


def _run(bodies, prm, precision, nsteps):
    o = oracle.Oracle(scenes.flatten_bodies(bodies), dataclasses.replace(prm, precision=precision))
    infos = [o.step() for _ in range(nsteps)]
    return o.get_state(), infos


def test_refinement_matches_fp64_before_contact():
    bodies, prm, _ = scenes.make_config(0)
    ref, ri = _run(bodies, prm, 0, 2)
    got, gi = _run(bodies, prm, 2, 2)
    assert all(i["n_active"] == 0 for i in gi)
    assert all(i["refine_iters"] > 0 for i in gi)  # the FP32 solves ran
    err = np.abs(got["p0"] - ref["p0"]).max() / np.abs(ref["p0"]).max()
    assert err <= 1e-9, err


def test_refinement_diverges_in_contact():
    bodies, prm, _ = scenes.make_config(1)
    ref, _ = _run(bodies, prm, 0, 6)
    got, gi = _run(bodies, prm, 2, 6)
    assert any(i["n_active"] > 0 for i in gi)
    err = np.abs(got["p0"] - ref["p0"]).max() / np.abs(ref["p0"]).max()
    energy = gi[-1]["energy"]
    assert err > 1e-3 or not np.isfinite(energy), (err, energy)


def test_fp32_preconditioner_before_contact():
    """Free fall (no contact): the FP64 flexible PCG with the FP32 preconditioner converges
    to the FP64 tolerance, in more iterations, and the step matches FP64 to 1e-9."""
    bodies, prm, _ = scenes.make_config(1)
    ref, ri = _run(bodies, prm, 0, 2)
    got, gi = _run(bodies, prm, 1, 2)
    assert all(i["n_active"] == 0 for i in gi)
    assert sum(i["linear_iters"] for i in gi) > sum(i["linear_iters"] for i in ri) > 0
    err = np.abs(got["p0"] - ref["p0"]).max() / np.abs(ref["p0"]).max()
    assert err <= 1e-9, err


def test_fp32_preconditioner_freezes_in_contact():
    """From the first contact on (step 3 of the 64-sphere scene), the FP32 inverse of the
    contact cluster is indefinite: the solves take no iteration, return dq = 0, and the state
    stops moving while the FP64 step goes on."""
    bodies, prm, _ = scenes.make_config(1)
    ref, ri = _run(bodies, prm, 0, 8)
    got, gi = _run(bodies, prm, 1, 8)
    assert gi[2]["n_active"] > 0
    assert all(i["linear_iters"] == 0 for i in gi[4:])
    assert len({i["energy"] for i in gi[5:]}) == 1  # frozen
    err = np.abs(got["p0"] - ref["p0"]).max() / np.abs(ref["p0"]).max()
    assert err > 1e-4, err
