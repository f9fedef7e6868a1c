"""Failure paths of the step, with the failures made on the host (no GPU fault): a
non-finite state, a Krylov solve capped below what it needs, and the status word that
reports them (abd_take_status), through the C ABI.

* A NaN velocity: the Newton system of the body is non-finite, the body kernel raises the
  NaN status bit and abd_step returns ABD_ERR_DEVICE after finishing the step (the kernels'
  loops are bounded by the tree sizes, the Krylov iteration cap and the line search's trial
  count, so a NaN ends them like any other value).
* cg_max_iter = 1 on a contact-rich state: the step completes (the reference's truncated
  Newton carries on with an inexact direction) and reports solver non-convergence in its
  status; the bit is not raised again once taken."""
import dataclasses
import os

import numpy as np
import pytest

from abd_warp_b200 import _lib, scenes
from abd_warp_b200.params import SimParams

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _sim(bodies, prm):
    from abd_warp_b200.simulator import AffineBodySimulator
    return AffineBodySimulator(bodies=bodies, params=prm, device="cuda:0")


def test_nan_state_raises_the_nan_status():
    prm = SimParams()
    bodies = [scenes._body("cube:0.5", (0.0, 2.0, 0.0), v=(0.3, 0.0, 0.0))]
    sim = _sim(bodies, prm)
    try:
        assert sim.step()["status"] == 0
        sim.states.pdot[0, 0] = float("nan")
        with pytest.raises(_lib.AbdError) as e:
            sim.step()
        assert "device-side error" in str(e.value)
        assert sim.take_status() == 0  # the step took its bits into the step info
        # a finite state again: the next step is clean
        sim.reset()
        info = sim.step()
        assert info["status"] == 0 and np.isfinite(sim.states.p0.cpu().numpy()).all()
    finally:
        sim.close()


def test_nan_status_in_step_info():
    """The step info's status carries the NaN bit (read through the C ABI directly)."""
    import ctypes

    prm = SimParams()
    bodies = [scenes._body("cube:0.5", (0.0, 2.0, 0.0))]
    sim = _sim(bodies, prm)
    try:
        sim.states.pdot[0, 1] = float("nan")
        info = _lib.StepInfo()
        rc = sim._L.abd_step(sim._h, ctypes.byref(sim._cstates()), None, ctypes.byref(info))
        assert rc == _lib.ABD_ERR_DEVICE
        assert info.status & _lib.ST_NAN
    finally:
        sim.close()


def test_krylov_cap_reports_nonconvergence():
    z = np.load(os.path.join(GOLDEN, "c1_trajectory.npz"))
    bodies, prm, _ = scenes.make_config(1)
    capped = dataclasses.replace(prm, cg_max_iter=1)
    sim = _sim(bodies, capped)
    try:
        import torch
        for k in ("A0", "p0", "Adot", "pdot"):
            getattr(sim.states, k).copy_(torch.as_tensor(z[f"s200_{k}"]))
        sim.states.A.copy_(sim.states.A0)
        sim.states.p.copy_(sim.states.p0)
        sim.dq = torch.as_tensor(z["s200_dq"])
        info = sim.step()
        assert info["status"] & _lib.ST_SOLVER_NOCONV, info
        assert info["linear_iters"] <= info["newton_iters"]  # one iteration per solve at most
        assert sim.take_status() == 0  # taken by the step
        # the uncapped solver converges on the same state
        sim.set_params(prm)
        for k in ("A0", "p0", "Adot", "pdot"):
            getattr(sim.states, k).copy_(torch.as_tensor(z[f"s200_{k}"]))
        sim.states.A.copy_(sim.states.A0)
        sim.states.p.copy_(sim.states.p0)
        sim.dq = torch.as_tensor(z["s200_dq"])
        assert sim.step()["status"] == 0
    finally:
        sim.close()
