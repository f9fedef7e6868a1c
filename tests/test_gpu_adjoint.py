"""The GPU adjoint of the time step (abd_adjoint_step, through the C ABI; the autograd
Function of abd_warp_b200/adjoint.py) on the differentiable configuration: 16 level-2
icospheres resting on the ground box with in-plane velocities, loss ||com_1(T) - target||^2.

The derivative exists where the steps converge, so the forward runs with the barrier stiffness
lowered to 1e3 and Newton to g.g < 1e-22 (60 iterations at most); at the default stiffness
1e6 the reference's Newton stops at its cap in contact steps and the forward map is not
differentiable in practice.

* Against the oracle's adjoint (oracle/adjoint_ref.py, exact reference-model Hessians, dense
  solves) on the same trajectory, which the GPU reproduces bit for bit: 5 steps, to 1e-6.
* Against central differences (h = 1e-6) of the GPU's own forward: 10 steps with checkpoints
  every 4 (so the backward recomputes three segments), and the configuration's 100 steps with
  checkpoints every 10, to 1e-4 (the bar of the differentiable configuration)."""
import numpy as np
import pytest

import oracle
from oracle import adjoint_ref as AJ
from abd_warp_b200 import scenes

pytestmark = pytest.mark.gpu

BODY = 1
H = 1e-6


def _setup():
    bodies, prm, _ = scenes.make_config(4)
    prm.kappa, prm.tol, prm.max_iter = 1e3, 1e-22, 60
    flat = scenes.flatten_bodies(bodies)
    target = np.asarray(flat["p"][BODY]) + np.array([0.3, 0.0, -0.2])
    return bodies, prm, flat, target


def _init(sim):
    import torch
    s = sim.states
    return [getattr(s, k).clone().requires_grad_(True) for k in ("A0", "p0", "Adot", "pdot")]


def _loss(p_T, target):
    import torch
    d = p_T[BODY] - torch.as_tensor(target, device=p_T.device)
    return (d * d).sum()


def _gpu_grads(sim, target, steps, checkpoint):
    from abd_warp_b200.adjoint import trajectory
    sim.reset()
    x = _init(sim)
    out = trajectory(sim, *x, steps=steps, checkpoint=checkpoint)
    L = _loss(out[1], target)
    L.backward()
    return float(L.item()), [v.grad.detach().cpu().numpy() for v in x]


def _gpu_loss(sim, target, steps, field, idx, dv):
    import torch
    from abd_warp_b200.adjoint import trajectory
    sim.reset()
    x = _init(sim)
    with torch.no_grad():
        k = ("A0", "p0", "Adot", "pdot").index(field)
        x[k][idx] += dv
        out = trajectory(sim, *[v.detach() for v in x], steps=steps, checkpoint=steps)
        return float(_loss(out[1], target).item())


def test_adjoint_matches_the_oracle_adjoint():
    from abd_warp_b200.simulator import AffineBodySimulator
    bodies, prm, flat, target = _setup()
    sim = AffineBodySimulator(bodies=bodies, params=prm)
    try:
        L, (gA0, gp0, gAd, gpd) = _gpu_grads(sim, target, steps=5, checkpoint=2)
        o = oracle.Oracle(flat, prm)
        states, infos = AJ.forward(o, 5)
        assert max(i["n_active"] for i in infos) > 10
        Lr, gp = AJ.com_loss(states, BODY, target)
        assert L == Lr  # the GPU trajectory is the oracle's, bit for bit
        qb = np.zeros((o.n, 12))
        qb[BODY, :3] = gp
        gq0, gqd0 = AJ.backward(o, flat, prm, states, qb, model="reference")
        n = o.n
        ref = {"p0": gq0[:, :3], "A0": gq0[:, 3:].reshape(n, 3, 3), "pdot": gqd0[:, :3],
               "Adot": gqd0[:, 3:].reshape(n, 3, 3)}
        got = {"p0": gp0, "A0": gA0, "pdot": gpd, "Adot": gAd}
        for k in ref:
            scale = np.abs(ref[k]).max()
            assert np.abs(got[k] - ref[k]).max() <= 1e-6 * scale, (k, np.abs(got[k] - ref[k]).max(), scale)
    finally:
        sim.close()


@pytest.mark.parametrize("steps,checkpoint", [(10, 4), (100, 10)])
def test_adjoint_matches_central_differences(steps, checkpoint):
    from abd_warp_b200.simulator import AffineBodySimulator
    bodies, prm, flat, target = _setup()
    sim = AffineBodySimulator(bodies=bodies, params=prm)
    try:
        _, grads = _gpu_grads(sim, target, steps, checkpoint)
        g = dict(zip(("A0", "p0", "Adot", "pdot"), grads))
        checks = [("pdot", (BODY, 0)), ("pdot", (BODY, 2)), ("p0", (BODY, 0)), ("A0", (BODY, 0, 1)),
                  ("pdot", (2, 0))]
        for field, idx in checks:
            lp = _gpu_loss(sim, target, steps, field, idx, +H)
            lm = _gpu_loss(sim, target, steps, field, idx, -H)
            fd = (lp - lm) / (2 * H)
            ad = g[field][idx]
            assert abs(ad - fd) <= 1e-4 * abs(fd), (steps, field, idx, ad, fd)
    finally:
        sim.close()
