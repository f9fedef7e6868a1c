"""Adjoint of a trajectory of implicit steps on the CPU oracle, by the implicit function
theorem, for checking a GPU adjoint.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, never by the product path.

A converged step solves grad_q E(q; q~) = 0 with q~ = q_t + dt qdot_t (+ dt^2 g for p), and E
depends on q~ only through the inertia term 1/2 (q - q~)^T M (q - q~).  So
dq_{t+1} / dq~ = H^-1 M, with H the exact Hessian of E at q_{t+1}: inertia, orthogonality
and the unprojected contact Hessians of the full contact model.  The projected Hessian that
Newton uses does not enter.  With qdot_{t+1} = (q_{t+1} - q_t) / dt, the adjoints
(qb, qdb) of (q_{t+1}, qdot_{t+1}) go back one step as
    a = qb + qdb / dt,   lambda = H^-1 a,   qb_t = M lambda - qdb / dt,   qdb_t = dt M lambda.
DOFs per body: [p, A row 0, row 1, row 2] (12).  Fixed bodies carry no adjoint.

The reference has no adjoint.  This is the differentiable-simulation form of the library
(checkpointed forward, transposed Hessian solve per step), restated for the oracle: every
state is kept, since the scenes it checks are small.
"""
from __future__ import annotations

import numpy as np


def dofs(A, p):
    """[n, 12] DOF vectors from A [n, 3, 3] (row k = a_k) and p [n, 3]."""
    n = len(p)
    return np.concatenate([np.asarray(p).reshape(n, 3), np.asarray(A).reshape(n, 9)], axis=1)


def forward(o, steps):
    """States before every step and after the last: [S_0, ..., S_steps]."""
    states = [o.get_state()]
    infos = []
    for _ in range(steps):
        infos.append(o.step())
        states.append(o.get_state())
    return states, infos


def com_loss(states, body, target):
    """||p_body(T) - target||^2 (the body frame's origin is its centre of mass)."""
    d = states[-1]["p0"][body] - target
    return float(d @ d), 2.0 * d


def backward(o, flat, prm, states, qb_T, model="full", qdb_T=None):
    """dL/dq_0 and dL/dqdot_0 ([n, 12] each) from the adjoints qb_T (and qdb_T) of the final
    DOFs (and velocities); model: the contact model of the forward ("full" or "reference")."""
    n = o.n
    dt = prm.dt
    free = np.repeat(np.asarray(flat["fixed"]) == 0, 12)
    Mdiag = np.concatenate([np.repeat(np.asarray(flat["mass"])[:, None], 3, axis=1),
                            np.repeat(np.asarray(flat["I0"])[:, None], 9, axis=1)], axis=1).ravel()
    qb = np.asarray(qb_T, dtype=np.float64).reshape(n * 12).copy()
    qdb = np.zeros(n * 12) if qdb_T is None else np.asarray(qdb_T, dtype=np.float64).reshape(n * 12).copy()
    for t in range(len(states) - 2, -1, -1):
        S = states[t + 1]
        H = o.full_hessian(S["A0"], S["p0"], model=model)
        a = qb + qdb / dt
        lam = np.zeros(n * 12)
        lam[free] = np.linalg.solve(H[np.ix_(free, free)], a[free])
        tb = Mdiag * lam
        qb, qdb = tb - qdb / dt, dt * tb
        qb[~free] = 0.0
        qdb[~free] = 0.0
    return qb.reshape(n, 12), qdb.reshape(n, 12)
