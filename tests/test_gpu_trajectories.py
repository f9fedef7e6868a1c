"""GPU trajectories against the oracle at the benchmark's sizes, bit for bit, through the C ABI
(via the Python mirror of the reference's simulator API).

* The 1024-body pile (scene configuration 2, 332,808 vertices; the benchmarked workload): its
  trajectory against the oracle's states at steps 75, 150 and 225
  (tests/golden/c2_states.npz, made by tests/golden/make_c2_states.py), and three steps from
  the stored state at step 225 against fresh oracle steps, with the contact flags.
* The 64-icosphere scene (configuration 1): all 300 steps against the oracle's step counters
  and its states after steps 100, 200 and 300 (tests/golden/c1_trajectory.npz, made by
  tests/golden/make_c1_states.py).  The spheres land on the ground box and on each other, so
  the contact sets are non-empty from about step 20 on.
* Injected capacity shortfalls (``SimParams.min_capacity``): every list of the simulator starts
  with 16 entries and the breadth-first traversal frontier holds 16 nodes, so each pass runs its
  grow-and-rerun paths and the traversal's depth-first fallback; the steps still equal the
  oracle's bit for bit.  Lists started above the contact scan's one-CTA scatter bound take the
  separate scatter kernel, with the same result.
* Edge cases: a single free body with no pairs (implicit-Euler free fall in closed form), and a
  scene of fixed bodies only."""
import os

import numpy as np
import pytest

import oracle
from abd_warp_b200 import scenes
from abd_warp_b200.simulator import AffineBodySimulator

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIELDS = ("A0", "p0", "Adot", "pdot")
COUNTERS = ("newton_iters", "linear_iters", "ls_trials", "n_pt", "n_ee", "n_vg", "n_ij", "n_active")


def _state(sim):
    return {k: getattr(sim.states, k).cpu().numpy() for k in FIELDS} | {"dq": sim.dq.cpu().numpy()}


def _start_from(sim, st):
    import torch
    for k in FIELDS:
        getattr(sim.states, k).copy_(torch.as_tensor(st[k]).reshape(getattr(sim.states, k).shape))
    sim.states.A.copy_(sim.states.A0)
    sim.states.p.copy_(sim.states.p0)
    sim.dq = torch.as_tensor(st["dq"], device=sim.device)


def _steps_against_oracle(bodies, prm, st, nsteps, sim_prm=None):
    """nsteps steps from state st on the GPU (parameters sim_prm, default prm) and on the
    oracle: counters, energy, states and contact flags equal after every step."""
    o = oracle.Oracle(scenes.flatten_bodies(bodies), prm)
    o.set_state(*(st[k] for k in FIELDS), dq=st["dq"])
    sim = AffineBodySimulator(bodies=bodies, params=sim_prm or prm, device="cuda:0")
    try:
        _start_from(sim, st)
        for s in range(nsteps):
            ref = o.step()
            got = sim.step()
            assert got["status"] == 0, (s, got)
            for key in COUNTERS:
                assert got[key] == ref[key], (s, key, got, ref)
            assert got["energy"] == ref["energy"], s
            ost = o.get_state()
            mine = _state(sim)
            for k in (*FIELDS, "dq"):
                assert np.array_equal(mine[k].reshape(ost[k].shape), ost[k]), (s, k)
            np.testing.assert_array_equal(sim.highlight, o.highlight(), err_msg=f"step {s} highlight")
        return sim.take_status()
    finally:
        sim.close()


def test_pile1024_trajectory_matches_the_oracle_states():
    z = np.load(os.path.join(GOLDEN, "c2_states.npz"))
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


def test_pile1024_steps_from_a_stored_state():
    z = np.load(os.path.join(GOLDEN, "c2_states.npz"))
    bodies, prm, _ = scenes.make_config(2)
    st = {k: z[f"s225_{k}"] for k in (*FIELDS, "dq")}
    _steps_against_oracle(bodies, prm, st, 3)


def test_pile64_full_trajectory():
    """All 300 steps of the 64-icosphere scene: every step's counters and energy equal the
    oracle's, and the states and contact flags after steps 100, 200 and 300."""
    z = np.load(os.path.join(GOLDEN, "c1_trajectory.npz"))
    bodies, prm, nsteps = scenes.make_config(1)
    assert nsteps == len(z["newton_iters"])
    sim = AffineBodySimulator(bodies=bodies, params=prm, device="cuda:0")
    try:
        for s in range(1, nsteps + 1):
            got = sim.step()
            assert got["status"] == 0, (s, got)
            for key in (*COUNTERS, "energy", "alpha", "toi"):
                assert got[key] == z[key][s - 1], (s, key, got[key], z[key][s - 1])
            if s in z["keep"]:
                mine = _state(sim)
                for k in (*FIELDS, "dq"):
                    ref = z[f"s{s}_{k}"]
                    assert np.array_equal(mine[k].reshape(ref.shape), ref), (s, k)
                np.testing.assert_array_equal(sim.highlight, z[f"s{s}_highlight"], err_msg=f"step {s}")
                assert z[f"s{s}_highlight"].any() and got["n_active"] > 0
    finally:
        sim.close()


@pytest.mark.parametrize("scene", ["pile64_step200", "pile1024_step225"])
def test_injected_capacity_shortfalls(scene):
    """Lists that start with 16 entries and a 16-node traversal frontier: every pass overflows,
    grows and reruns, and the traversals fall back to depth-first walks; the steps are still the
    oracle's, bit for bit."""
    import dataclasses
    if scene == "pile64_step200":
        z = np.load(os.path.join(GOLDEN, "c1_trajectory.npz"))
        bodies, prm, _ = scenes.make_config(1)
        st = {k: z[f"s200_{k}"] for k in (*FIELDS, "dq")}
    else:
        z = np.load(os.path.join(GOLDEN, "c2_states.npz"))
        bodies, prm, _ = scenes.make_config(2)
        st = {k: z[f"s225_{k}"] for k in (*FIELDS, "dq")}
    tiny = dataclasses.replace(prm, min_capacity=16)
    assert _steps_against_oracle(bodies, prm, st, 3, sim_prm=tiny) == 0


def test_contact_lists_beyond_the_scan_scatter():
    """Lists that start with 20,000 entries, more than the 16,384 contacts the contact scan's
    CTA scatters itself: the GH passes group their contacts with the one-thread-per-contact
    scatter kernel, and the steps are still the oracle's, bit for bit."""
    import dataclasses
    z = np.load(os.path.join(GOLDEN, "c1_trajectory.npz"))
    bodies, prm, _ = scenes.make_config(1)
    st = {k: z[f"s200_{k}"] for k in (*FIELDS, "dq")}
    large = dataclasses.replace(prm, min_capacity=20000)
    assert _steps_against_oracle(bodies, prm, st, 3, sim_prm=large) == 0


def _oracle_and_gpu(bodies, prm):
    o = oracle.Oracle(scenes.flatten_bodies(bodies), prm)
    sim = AffineBodySimulator(bodies=bodies, params=prm, device="cuda:0")
    return o, sim


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
        assert not sim.highlight.any()
    finally:
        sim.close()


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
