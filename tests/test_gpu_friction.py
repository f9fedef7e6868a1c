"""Lagged IPC friction in the GPU step (SimParams.friction_mu > 0, with the full contact
model), through the C ABI, against the oracle's step in the same per-contact arithmetic (the
full-model header's friction_lag / friction_gh and point-to-body map), bit for bit.

Friction is not in the reference.  At a step's start every contact within dhat fixes its
closest-point weights, a tangent basis and its normal force; the step adds the friction
potential of those contacts to the energy of every evaluation, their terms to the pair
assembly, and keeps their body pairs in the pair lists for the whole step."""
import dataclasses

import numpy as np
import pytest

import oracle
from abd_warp_b200 import scenes
from abd_warp_b200.params import SimParams

pytestmark = pytest.mark.gpu

FIELDS = ("A0", "p0", "Adot", "pdot")
COUNTERS = ("newton_iters", "linear_iters", "ls_trials", "n_pt", "n_ee", "n_vg", "n_ij", "n_active")


def _sliding_cube(newton_loop):
    prm = SimParams()
    prm.max_iter, prm.tol = 100, 1e-12  # converged steps
    prm = dataclasses.replace(prm, ipc_full=1, friction_mu=0.5, friction_epsv=1e-3, newton_loop=newton_loop)
    bodies = [scenes.ground_box(), scenes._body("cube:0.3", (0.0, 0.15 + 1.2 * prm.dhat, 0.0), v=(1.0, 0.0, 0.0))]
    return bodies, prm


def _run(bodies, prm, nsteps):
    from abd_warp_b200.simulator import AffineBodySimulator
    o = oracle.Oracle(scenes.flatten_bodies(bodies), prm)
    sim = AffineBodySimulator(bodies=bodies, params=prm)
    active, hist = 0, []
    try:
        for s in range(nsteps):
            ri, gi = o.step(), sim.step()
            assert gi["status"] == 0, (s, gi)
            for k in COUNTERS:
                assert gi[k] == ri[k], (s, k, gi, ri)
            assert gi["energy"] == ri["energy"], s
            ost = o.get_state()
            for k in FIELDS:
                np.testing.assert_array_equal(getattr(sim.states, k).cpu().numpy(), ost[k], err_msg=f"{s} {k}")
            np.testing.assert_array_equal(sim.dq.cpu().numpy(), ost["dq"], err_msg=f"{s} dq")
            np.testing.assert_array_equal(np.asarray(sim.highlight), o.highlight(), err_msg=f"{s} highlight")
            active += ri["n_active"]
            hist.append(ost)
    finally:
        sim.close()
    return active, hist


@pytest.mark.parametrize("newton_loop", [0, 1], ids=["device", "host"])
def test_friction_sliding_cube(newton_loop):
    """A 0.3 m cube sliding on the ground box at 1 m/s with mu = 0.5: bit for bit with the
    oracle for 30 steps, and it decelerates at mu g once the landing's normal force is lagged."""
    bodies, prm = _sliding_cube(newton_loop)
    active, hist = _run(bodies, prm, 30)
    assert active > 0
    g = -prm.gravity
    v = [h["pdot"][1, 0] for h in hist]
    for k in range(3, 12):  # steps k + 1 = 4 .. 12, well before it stops
        assert v[k] == pytest.approx(1.0 - prm.friction_mu * g * k * prm.dt, abs=1e-3)


def test_friction_pile():
    """Eight bodies falling onto the ground box and onto each other with mu = 0.3: 40 steps
    bit for bit (friction between free bodies and with the fixed ground)."""
    bodies, prm = scenes.small_pile(2, 2, seed=7)
    prm = dataclasses.replace(prm, ipc_full=1, friction_mu=0.3, friction_epsv=1e-3)
    active, _ = _run(bodies, prm, 40)
    assert active > 0


def test_friction_needs_the_full_model():
    """Friction without the full contact model, with a negative coefficient or a non-positive
    slip velocity is refused at creation and by set_params."""
    from abd_warp_b200 import _lib
    from abd_warp_b200.simulator import AffineBodySimulator
    bodies, prm = _sliding_cube(0)
    for bad in (dict(ipc_full=0), dict(friction_mu=-0.1), dict(friction_epsv=0.0)):
        with pytest.raises(_lib.AbdError):
            AffineBodySimulator(bodies=bodies, params=dataclasses.replace(prm, **bad))
    sim = AffineBodySimulator(bodies=bodies, params=prm)
    try:
        with pytest.raises(_lib.AbdError):
            sim.set_params(dataclasses.replace(prm, ipc_full=0))
    finally:
        sim.close()


def test_friction_energy_and_gradient_hessian_apis():
    """After friction steps the energy pass and the GH pass of the API carry the last step's
    lagged friction contacts, as the oracle's: energies at two DOF sets and the assembled
    gradient and blocks at the current DOFs, bit for bit."""
    import torch
    from abd_warp_b200.simulator import AffineBodySimulator
    bodies, prm = _sliding_cube(0)
    o = oracle.Oracle(scenes.flatten_bodies(bodies), prm)
    sim = AffineBodySimulator(bodies=bodies, params=prm)
    try:
        for _ in range(8):
            o.step()
            sim.step()
        st = o.get_state()
        cu = lambda v: torch.as_tensor(v, device="cuda")
        for shift in (0.0, 2e-4):
            A, p = st["A0"], st["p0"] + np.array([shift, 0.0, 0.0])
            assert sim.compute_energy(cu(A), cu(p)) == o.energy(A, p), shift
        ref = o.gh(st["A0"], st["p0"])
        got = sim.gradient_hessian(cu(st["A0"]), cu(st["p0"]))
        assert got["n_active"] == ref["n_active"] > 0
        for k in ("g", "diag", "off", "ij"):
            np.testing.assert_array_equal(got[k].cpu().numpy(), ref[k], err_msg=k)
    finally:
        sim.close()
