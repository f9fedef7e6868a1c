"""GPU parity: libabd_b200.so (through the C ABI, via the Python mirror) against the CPU
oracle on the same seeded scenes and states.

Bar: bit for bit.  Vertex transforms, culled pair sets (compared as sorted sets), the
assembled gradient and Hessian blocks, energies, times of impact, linear solves and whole
time steps (positions, velocities and the iteration counts of Newton, the Krylov solver and
the line search) are identical.  Both sides compute every term with the same operation
order (no FMA contraction), sum every reduction exactly with a single rounding, and use
the same IEEE-exact logarithm, so the order in which the GPU's threads deliver the terms
does not reach the result."""
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


def _c1_state(step):
    """The oracle's state of the 64-icosphere scene after `step` steps (golden fixture)."""
    import os
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "c1_trajectory.npz"))
    return {k: z[f"s{step}_{k}"] for k in ("A0", "p0", "Adot", "pdot", "dq")}


SCENES = {
    "c0_contact": lambda: (scenes.make_config(0)[0], SimParams(), 3),
    "pile_ground": lambda: (scenes.small_pile(2, 2, seed=7)[0], SimParams(), 30),
    "c1_start": lambda: (scenes.make_config(1)[0], SimParams(), 0),
    # 64 icospheres piled on the ground box after 200 steps: 600 PT / 2361 EE culled pairs
    "c1_contact": lambda: (scenes.make_config(1)[0], SimParams(), _c1_state(200)),
    "pile_plane": lambda: (*scenes.small_pile(2, 2, seed=7, plane=True), 30),
}


@pytest.fixture(scope="module", params=sorted(SCENES))
def scene_state(request):
    bodies, prm, steps = SCENES[request.param]()
    if isinstance(steps, dict):
        o, st = oracle.Oracle(scenes.flatten_bodies(bodies), prm), steps
    else:
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
    if name != "c1_start":  # the 64 spheres start more than dhat apart
        assert len(ref["pt"]) + len(ref["ee"]) + len(ref["vg"]) > 0


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
    np.testing.assert_array_equal(got["g"].cpu().numpy(), ref["g"])
    np.testing.assert_array_equal(got["diag"].cpu().numpy(), ref["diag"])
    np.testing.assert_array_equal(got["ij"].cpu().numpy(), ref["ij"])
    np.testing.assert_array_equal(got["off"].cpu().numpy(), ref["off"])
    # per-body contact flags of this pass (the reference's sim.highlight, abd.py:238)
    np.testing.assert_array_equal(sim.highlight, o.highlight())
    if name in ("pile_ground", "c1_contact"):
        assert ref["n_active"] > 0  # the bodies rest on the ground and on each other
        assert o.highlight().any()


def test_energy(scene_state):
    name, bodies, prm, o, st, sim = scene_state
    import torch
    for a in (0.0, 0.5, 1.0):
        Ak = st["A0"] + a * prm.dt * st["Adot"]
        pk = st["p0"] + a * prm.dt * st["pdot"]
        e_ref = o.energy(Ak, pk)
        e = sim.compute_energy(torch.as_tensor(Ak, device="cuda"), torch.as_tensor(pk, device="cuda"))
        assert e == e_ref, (a, e, e_ref)


def test_energies_along(scene_state):
    """The step's batched line-search energies: one culling pass over the segment from (A, p)
    to (A, p) - dq, then every trial re-evaluated from those candidates with the culling
    predicate applied at the trial's DOFs.  Each energy equals the oracle's energy pass at the
    same DOFs bit for bit, and the library's own energy pass too; 20 step lengths take two
    batches."""
    name, bodies, prm, o, st, sim = scene_state
    import torch
    n = len(bodies)
    fixed = np.array([bool(b.fixed) for b in bodies])
    dq = np.zeros((n, 12))
    dq[:, :3] = -3 * prm.dt * st["pdot"] + np.array([0.0, 0.02, 0.0])
    dq[:, 3:] = -3 * prm.dt * st["Adot"].reshape(n, 9)
    dq[fixed] = 0.0
    alphas = [2.0 ** -k for k in range(18)] + [0.0, 0.7]
    A, p = st["A0"], st["p0"]
    sim.dq = torch.as_tensor(dq)
    try:
        got = sim.energies_along(alphas, torch.as_tensor(A, device="cuda"), torch.as_tensor(p, device="cuda"))
        for al, e in zip(alphas, got):
            Ak = A - dq[:, 3:].reshape(n, 3, 3) * al
            pk = p - dq[:, :3] * al
            assert e == o.energy(Ak, pk), (name, al, e, o.energy(Ak, pk))
            assert e == sim.compute_energy(torch.as_tensor(Ak, device="cuda"), torch.as_tensor(pk, device="cuda"))
    finally:
        sim.dq = torch.as_tensor(st["dq"])


def test_ccd(scene_state):
    name, bodies, prm, o, st, sim = scene_state
    import torch
    for scale in (1.0, 5.0):
        A1 = st["A0"] + scale * prm.dt * st["Adot"]
        p1 = st["p0"] + scale * prm.dt * st["pdot"] + np.array([0, -scale * 0.01, 0])
        a_ref, raw_ref = o.ccd(st["A0"], st["p0"], A1, p1)
        cu = lambda v: torch.as_tensor(v, device="cuda")
        a, raw = sim.ccd(cu(st["A0"]), cu(st["p0"]), cu(A1), cu(p1))
        assert raw == raw_ref and a == a_ref, (scale, raw, raw_ref)


@pytest.mark.parametrize("solver", [0, 1])
def test_solve(scene_state, solver):
    """Same system, same contact clusters, exact dot products and the same SpMV and
    preconditioner order: identical iterates, so the same solution and iteration count."""
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
        assert it == it_ref
        np.testing.assert_array_equal(dq.cpu().numpy(), dq_ref)
    finally:
        sim.set_params(prm0)
        o.set_params(prm0)


def _steps_match_the_oracle(bodies, prm, nsteps, loop):
    """nsteps whole steps on the GPU (device or host Newton loop) and on the oracle, bit for
    bit at every step; the trajectory goes through contact."""
    import dataclasses
    o = oracle.Oracle(scenes.flatten_bodies(bodies), prm)
    sim = _sim(bodies, dataclasses.replace(prm, newton_loop=0 if loop == "device" else 1))
    active = 0
    try:
        for s in range(nsteps):
            ri = o.step()
            gi = sim.step()
            assert gi["status"] == 0, (s, gi)
            for k in ("newton_iters", "linear_iters", "ls_trials", "n_active", "n_pt", "n_ee", "n_vg", "n_ij"):
                assert gi[k] == ri[k], (s, k, gi, ri)
            assert gi["energy"] == ri["energy"], (s, gi["energy"], ri["energy"])
            st = o.get_state()
            for k in ("A0", "p0", "Adot", "pdot"):
                np.testing.assert_array_equal(getattr(sim.states, k).cpu().numpy(), st[k], err_msg=f"step {s} {k}")
            np.testing.assert_array_equal(sim.dq.cpu().numpy(), st["dq"], err_msg=f"step {s} dq")
            active += ri["n_active"]
        np.testing.assert_array_equal(sim.x_view.cpu().numpy(), st["x_view"])
        assert active > 0  # the trajectory went through contact
    finally:
        sim.close()


@pytest.mark.parametrize("loop", ["device", "host"])
@pytest.mark.parametrize("case,nsteps", [("c0", 200), ("pile", 60), ("plane", 60)])
def test_step_parity(case, nsteps, loop):
    """Whole time steps against the oracle, bit for bit: positions, velocities, the dq warm
    start and every iteration count, at every step (c0: the two-cube configuration for its
    200 steps; pile: 8 bodies on the ground box, 60 steps through landing and contact;
    plane: the same bodies landing on the vertex-ground plane), with the Newton iterations
    run as a device loop (the default) and driven from the host."""
    if case == "c0":
        bodies, prm, _ = scenes.make_config(0)
    else:
        bodies, prm = scenes.small_pile(2, 2, seed=7, plane=case == "plane")
    _steps_match_the_oracle(bodies, prm, nsteps, loop)


@pytest.mark.parametrize("loop", ["device", "host"])
def test_step_parity_bicgstab(loop):
    """The pile's 60 steps with the reference's solver, right-preconditioned BiCGSTAB
    (solver = 0), against the oracle's BiCGSTAB steps, bit for bit at every step (the Krylov
    iterations end inside the kernel that completes their last dot products)."""
    import dataclasses
    bodies, prm = scenes.small_pile(2, 2, seed=7)
    _steps_match_the_oracle(bodies, dataclasses.replace(prm, solver=0), 60, loop)


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


def test_step_after_state_change():
    """Steps reuse the last CCD pass's candidates for their first GH pass only when they start
    from the DOFs the previous step ended with: after the states are set to another point of the
    trajectory, the steps still agree with the oracle bit for bit."""
    import torch
    bodies, prm = scenes.small_pile(2, 2, seed=7)
    o = oracle.Oracle(scenes.flatten_bodies(bodies), prm)
    states = []
    for _ in range(30):
        o.step()
        states.append(o.get_state())
    sim = _sim(bodies, prm)
    try:
        for _ in range(25):
            sim.step()
        # back to the oracle's state after step 12, then five steps
        st = states[11]
        _set_state(sim, st)
        o.set_state(st["A0"], st["p0"], st["Adot"], st["pdot"], st["dq"])
        for s in range(5):
            ri = o.step()
            gi = sim.step()
            for k in ("newton_iters", "linear_iters", "ls_trials", "n_active", "n_pt", "n_ee"):
                assert gi[k] == ri[k], (s, k, gi, ri)
            ref = o.get_state()
            for k in ("A0", "p0", "Adot", "pdot"):
                np.testing.assert_array_equal(getattr(sim.states, k).cpu().numpy(), ref[k], err_msg=f"step {s} {k}")
    finally:
        sim.close()
