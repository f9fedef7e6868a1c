"""The oracle's adjoint of a trajectory (oracle/adjoint_ref.py: implicit function theorem per
step with the exact, unprojected Hessian of the full contact model) against central
differences of the oracle's own forward steps.  The checker for a GPU adjoint; CPU only.

Scene: configuration 4 (16 icospheres resting on the ground box, in-plane velocities), loss
||com_1(T) - target||^2.  The forward must converge for the derivative of its result to
exist: the barrier stiffness is lowered to 1e3 and Newton runs to g.g < 1e-22 (60 iterations
at most).  At the default stiffness 1e6, Newton stops at its iteration cap in contact steps,
and the differences of the forward map are noise."""
import numpy as np
import pytest

import oracle
from oracle import adjoint_ref as AJ
from abd_warp_b200 import scenes

BODY = 1
H = 1e-6


def _setup(kappa=1e3):
    bodies, prm, _ = scenes.make_config(4)
    prm.kappa, prm.tol, prm.max_iter = kappa, 1e-22, 60
    flat = scenes.flatten_bodies(bodies)
    target = np.asarray(flat["p"][BODY]) + np.array([0.3, 0.0, -0.2])
    return flat, prm, target


def _run(flat, prm, steps, mod=None, full=True):
    o = oracle.Oracle(flat, prm)
    o.set_ipc_full(full)
    if mod is not None:
        st = o.get_state()
        mod(st)
        o.set_state(st["A0"], st["p0"], st["Adot"], st["pdot"], st["dq"])
    states, infos = AJ.forward(o, steps)
    return o, states, infos


def _check(steps, tol, model="full"):
    flat, prm, target = _setup()
    o, states, infos = _run(flat, prm, steps, full=model == "full")
    _, gp = AJ.com_loss(states, BODY, target)
    qb = np.zeros((o.n, 12))
    qb[BODY, :3] = gp
    gq0, gqd0 = AJ.backward(o, flat, prm, states, qb, model=model)
    params = [("pdot", (BODY, 0), gqd0[BODY, 0]), ("pdot", (BODY, 2), gqd0[BODY, 2]),
              ("p0", (BODY, 0), gq0[BODY, 0]), ("A0", (BODY, 0, 1), gq0[BODY, 3 + 1])]
    for field, idx, ad in params:
        def mod(sign):
            def f(st):
                st[field][idx] += sign * H
            return f
        lp = AJ.com_loss(_run(flat, prm, steps, mod(+1), full=model == "full")[1], BODY, target)[0]
        lm = AJ.com_loss(_run(flat, prm, steps, mod(-1), full=model == "full")[1], BODY, target)[0]
        fd = (lp - lm) / (2 * H)
        assert abs(ad - fd) <= tol * abs(fd), (field, idx, ad, fd)
    return infos


def test_adjoint_contact_free_step():
    infos = _check(steps=1, tol=1e-7)
    assert infos[0]["n_active"] == 0


def test_adjoint_through_contact():
    infos = _check(steps=5, tol=1e-4)
    assert min(i["n_active"] for i in infos[1:]) > 10  # four steps in resting contact


def test_full_hessian_needs_the_full_model():
    flat, prm, _ = _setup()
    o = oracle.Oracle(flat, prm)
    st = o.get_state()
    with pytest.raises(RuntimeError):
        o.full_hessian(st["A0"], st["p0"])


def test_adjoint_reference_model_through_contact():
    """The reference's contact model (the library's default, which the GPU adjoint
    differentiates): its exact Hessian (interior contacts with every second-derivative term)
    gives gradients within 1e-4 of central differences over five steps in contact."""
    infos = _check(steps=5, tol=1e-4, model="reference")
    assert min(i["n_active"] for i in infos[1:]) > 10
