"""The full IPC contact model in the GPU step (SimParams.ipc_full = 1), through the C ABI,
against the oracle's full mode in the same per-contact arithmetic (the model's header with the
shared logarithm; the oracle's own forward-mode restatement agrees with it to 1e-9,
tests/test_ipc_full.py), bit for bit.

The full model classifies every candidate's closest feature pair (point-triangle, -edge,
-point; edge-edge, point-edge, point-point), puts the barrier on that pair's squared distance
with the edge-edge mollifier, projects each contact's exact local Hessian onto the PSD cone,
and counts CCD roots on the closed triangle or segments.  The reference's model (the library's
default) evaluates interior pairs only (ipcsk/energy.py:20-22, 46-48; ccd.py:44-54)."""
import dataclasses
import os

import numpy as np
import pytest

import oracle
from abd_warp_b200 import scenes

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIELDS = ("A0", "p0", "Adot", "pdot")
COUNTERS = ("newton_iters", "linear_iters", "ls_trials", "n_pt", "n_ee", "n_vg", "n_ij", "n_active")


def _full(prm):
    return dataclasses.replace(prm, ipc_full=1)


def _pair(bodies, prm, st=None):
    from abd_warp_b200.simulator import AffineBodySimulator
    import torch
    o = oracle.Oracle(scenes.flatten_bodies(bodies), prm)
    sim = AffineBodySimulator(bodies=bodies, params=prm)
    if st is not None:
        o.set_state(*(st[k] for k in FIELDS), dq=st["dq"])
        for k in FIELDS:
            getattr(sim.states, k).copy_(torch.as_tensor(st[k]).reshape(getattr(sim.states, k).shape))
        sim.states.A.copy_(sim.states.A0)
        sim.states.p.copy_(sim.states.p0)
        sim.dq = torch.as_tensor(st["dq"], device=sim.device)
    return o, sim


def _c1(step):
    z = np.load(os.path.join(GOLDEN, "c1_trajectory.npz"))
    return {k: z[f"s{step}_{k}"] for k in (*FIELDS, "dq")}


@pytest.mark.parametrize("scene", ["c1_step200", "pile_step30"])
def test_full_model_passes(scene):
    """Gradient and Hessian blocks, energies and the CCD bound of one state, bit for bit."""
    import torch
    if scene == "c1_step200":
        bodies, prm, _ = scenes.make_config(1)
        prm = _full(prm)
        st = _c1(200)
    else:
        bodies, prm = scenes.small_pile(2, 2, seed=7)
        prm = _full(prm)
        o0 = oracle.Oracle(scenes.flatten_bodies(bodies), prm)
        for _ in range(30):
            o0.step()
        st = o0.get_state()
    o, sim = _pair(bodies, prm, st)
    try:
        A = st["A0"] + prm.dt * st["Adot"]
        p = st["p0"] + prm.dt * st["pdot"]
        cu = lambda v: torch.as_tensor(v, device="cuda")
        ref = o.gh(A, p)
        got = sim.gradient_hessian(cu(A), cu(p))
        assert got["n_active"] == ref["n_active"] > 0
        for k in ("g", "diag", "off", "ij"):
            np.testing.assert_array_equal(got[k].cpu().numpy(), ref[k], err_msg=k)
        for a in (0.0, 0.5, 1.0):
            Ak, pk = st["A0"] + a * prm.dt * st["Adot"], st["p0"] + a * prm.dt * st["pdot"]
            assert sim.compute_energy(cu(Ak), cu(pk)) == o.energy(Ak, pk), a
        A1, p1 = A + 5 * prm.dt * st["Adot"], p + 5 * prm.dt * st["pdot"] + np.array([0.0, -0.01, 0.0])
        assert sim.ccd(cu(A), cu(p), cu(A1), cu(p1)) == o.ccd(A, p, A1, p1)
    finally:
        sim.close()


@pytest.mark.parametrize("case,nsteps", [("c0", 60), ("pile", 60), ("c1_step200", 5)])
def test_full_model_steps(case, nsteps):
    """Whole steps with the full model, bit for bit: counters, energy, states, warm start."""
    st = None
    if case == "c0":
        bodies, prm, _ = scenes.make_config(0)
    elif case == "pile":
        bodies, prm = scenes.small_pile(2, 2, seed=7)
    else:
        bodies, prm, _ = scenes.make_config(1)
        st = _c1(200)
    prm = _full(prm)
    o, sim = _pair(bodies, prm, st)
    active = 0
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
            active += ri["n_active"]
        assert active > 0
    finally:
        sim.close()
