"""GPU tests not yet run on a GPU: parity at the full size of the benchmark workload, and edge
cases (a single free body with no pairs, a scene of fixed bodies only).

Full size: the 1024-body pile (scene
configuration 2, 332,808 vertices) stepped on the GPU along its trajectory, against the
oracle's states at steps 75, 150 and 225 (tests/golden/c2_states.npz, made by
tests/golden/make_c2_states.py), bit for bit, and three steps from the stored state at step
225 against fresh oracle steps.

Marked ``gpu_full`` (not ``gpu``): they run when selected with ``-m gpu_full`` (the full-size
tests take about a minute of host time for the oracle steps)."""
import os

import numpy as np
import pytest

import oracle
from abd_warp_b200 import scenes
from abd_warp_b200.simulator import AffineBodySimulator

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "c2_states.npz")
FIELDS = ("A0", "p0", "Adot", "pdot")


def _state(sim):
    return {k: getattr(sim.states, k).cpu().numpy() for k in FIELDS} | {"dq": sim.dq.cpu().numpy()}


@pytest.mark.gpu_full
def test_pile1024_trajectory_matches_the_oracle_states():
    z = np.load(GOLDEN)
    bodies, prm, _ = scenes.make_config(2)
    sim = AffineBodySimulator(bodies=bodies, params=prm, device="cuda:0")
    try:
        for s in range(226):
            if s in (75, 150, 225):
                got = _state(sim)
                for k in (*FIELDS, "dq"):
                    ref = z[f"s{s}_{k}"]
                    assert np.array_equal(got[k].reshape(ref.shape), ref), (s, k)
            if s < 225:
                assert sim.step()["status"] == 0, s
    finally:
        sim.close()


@pytest.mark.gpu_full
def test_pile1024_steps_from_a_stored_state():
    import torch

    z = np.load(GOLDEN)
    bodies, prm, _ = scenes.make_config(2)
    flat = scenes.flatten_bodies(bodies)
    o = oracle.Oracle(flat, prm)
    o.set_state(*(z[f"s225_{k}"] for k in FIELDS), dq=z["s225_dq"])
    sim = AffineBodySimulator(bodies=bodies, params=prm, device="cuda:0")
    try:
        for k in FIELDS:
            getattr(sim.states, k).copy_(torch.as_tensor(z[f"s225_{k}"]).reshape(getattr(sim.states, k).shape))
        sim.states.A.copy_(sim.states.A0)
        sim.states.p.copy_(sim.states.p0)
        sim.dq = torch.as_tensor(z["s225_dq"], device="cuda:0")
        for _ in range(3):
            ref = o.step()
            got = sim.step()
            assert got["status"] == 0, got
            for key in ("newton_iters", "linear_iters", "ls_trials", "n_pt", "n_ee", "n_vg", "n_ij", "n_active"):
                assert got[key] == ref[key], (key, got, ref)
            assert got["energy"] == ref["energy"]
            st = o.get_state()
            mine = _state(sim)
            for k in FIELDS:
                assert np.array_equal(mine[k].reshape(st[k].shape), st[k]), k
    finally:
        sim.close()


def _oracle_and_gpu(bodies, prm):
    o = oracle.Oracle(scenes.flatten_bodies(bodies), prm)
    sim = AffineBodySimulator(bodies=bodies, params=prm, device="cuda:0")
    return o, sim


@pytest.mark.gpu_full
def test_single_free_body_falls_as_implicit_euler():
    """One free cube and nothing else: no pairs at all.  Ten steps equal the oracle bit for
    bit and the closed form of implicit Euler, p_y(k) = p_y(0) + g dt^2 k (k + 1) / 2."""
    from abd_warp_b200.params import SimParams

    prm = SimParams()
    bodies = [scenes._body("cube:0.5", (0.0, 2.0, 0.0), v=(0.3, 0.0, 0.0))]
    o, sim = _oracle_and_gpu(bodies, prm)
    try:
        for k in range(1, 11):
            ref, got = o.step(), sim.step()
            assert got["status"] == 0 and got["n_ij"] == 0 and got["newton_iters"] == ref["newton_iters"]
            st = o.get_state()
            for key in FIELDS:
                assert np.array_equal(getattr(sim.states, key).cpu().numpy(), st[key]), (k, key)
            y = sim.states.p0.cpu().numpy()[0, 1]
            assert y == pytest.approx(2.0 + prm.gravity * prm.dt ** 2 * k * (k + 1) / 2, abs=1e-12)
    finally:
        sim.close()


@pytest.mark.gpu_full
def test_only_fixed_bodies():
    """A scene whose bodies are all fixed: a step moves nothing and reports no device status."""
    from abd_warp_b200.params import SimParams

    prm = SimParams()
    bodies = [scenes.ground_box(), scenes._body("cube:0.5", (0.0, 2.0, 0.0), fixed=True)]
    o, sim = _oracle_and_gpu(bodies, prm)
    try:
        p0 = sim.states.p0.cpu().numpy().copy()
        ref, got = o.step(), sim.step()
        assert got["status"] == 0 and got["newton_iters"] == ref["newton_iters"]
        assert np.array_equal(sim.states.p0.cpu().numpy(), p0)
        assert np.array_equal(sim.states.pdot.cpu().numpy(), np.zeros_like(p0))
    finally:
        sim.close()
