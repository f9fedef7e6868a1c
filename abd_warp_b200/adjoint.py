"""Differentiable trajectories: ``torch.autograd`` through K implicit time steps.

The reference has no backward (abd/hl_entry.py:4 sets ``enable_backward = False``).  Here
:func:`trajectory` runs K steps of :meth:`AffineBodySimulator.step` inside a
``torch.autograd.Function`` whose backward is the hand-written adjoint of the step
(``abd_adjoint_step`` in libabd_b200.so):

* **Forward**: the K steps from the given initial states, keeping a checkpoint (states and the
  warm-started dq) every ``checkpoint`` steps; returns the final states.
* **Backward**: segment by segment from the last, the segment's steps are recomputed from its
  checkpoint (the step is deterministic, so they are the forward's bit for bit), then the
  adjoint runs back through them.  Per step, with q_{t+1} the converged DOFs,
  a = qb + qdb / dt, H lambda = a (H: the exact, unprojected Hessian of the step's energy at
  q_{t+1}, solved on the GPU by BiCGSTAB), qb_t = M lambda - qdb / dt, qdb_t = dt M lambda.

The derivative is the implicit-function derivative of converged steps: run the forward with a
Newton tolerance the steps reach (``SimParams.tol``) and a cap (``max_iter``) that does not cut
them short.  DOFs per body are [p, A row 0, row 1, row 2]; fixed bodies carry no gradient.
"""
from __future__ import annotations

import ctypes

from . import _lib

FIELDS = ("A0", "p0", "Adot", "pdot")


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _dofs(A, p):
    """[n, 12] from A [n, 3, 3] (row k = a_k) and p [n, 3]."""
    n = p.shape[0]
    import torch
    return torch.cat([p.reshape(n, 3), A.reshape(n, 9)], dim=1).contiguous()


def _split(q):
    """(A [n, 3, 3], p [n, 3]) from [n, 12]."""
    n = q.shape[0]
    return q[:, 3:].reshape(n, 3, 3), q[:, :3].reshape(n, 3)


def _load(sim, A0, p0, Adot, pdot, dq):
    s = sim.states
    s.A0.copy_(A0)
    s.p0.copy_(p0)
    s.Adot.copy_(Adot)
    s.pdot.copy_(pdot)
    s.A.copy_(s.A0)
    s.p.copy_(s.p0)
    sim.dq = dq


def _save(sim):
    s = sim.states
    return tuple(getattr(s, k).clone() for k in FIELDS) + (sim.dq.clone(),)


def adjoint_step(sim, A, p, qb, qdb):
    """One step back: (qb_t, qdb_t) [n, 12] from the adjoints (qb, qdb) [n, 12] of the DOFs and
    velocities after a step that converged at (A, p); also the Krylov iterations."""
    import torch
    qb = qb.contiguous()
    qdb = qdb.contiguous()
    qb_out = torch.empty_like(qb)
    qdb_out = torch.empty_like(qdb)
    it = ctypes.c_int(0)
    cst = sim._cstates()
    _lib.check(sim._L.abd_adjoint_step(sim._h, ctypes.byref(cst), _ptr(A.contiguous()), _ptr(p.contiguous()),
                                       _ptr(qb), _ptr(qdb), _ptr(qb_out), _ptr(qdb_out), ctypes.byref(it)),
               "abd_adjoint_step")
    return qb_out, qdb_out, it.value


class _Trajectory:
    """Namespace of the autograd Function (built lazily: torch is imported on first use)."""
    fn = None


def _function():
    if _Trajectory.fn is not None:
        return _Trajectory.fn
    import torch

    class Trajectory(torch.autograd.Function):
        @staticmethod
        def forward(ctx, sim, steps, checkpoint, A0, p0, Adot, pdot):
            dq0 = torch.zeros((sim.n_bodies, 12), dtype=torch.float64, device=sim.device)
            _load(sim, A0, p0, Adot, pdot, dq0)
            ckpts = {}
            infos = []
            for t in range(steps):
                if t % checkpoint == 0:
                    ckpts[t] = _save(sim)
                infos.append(sim.step())
            ctx.sim, ctx.steps, ctx.checkpoint, ctx.ckpts = sim, steps, checkpoint, ckpts
            ctx.infos = infos
            s = sim.states
            return tuple(getattr(s, k).clone() for k in FIELDS)

        @staticmethod
        def backward(ctx, gA, gp, gAd, gpd):
            sim, steps, cp = ctx.sim, ctx.steps, ctx.checkpoint
            n = sim.n_bodies
            zeros = lambda shape: torch.zeros(shape, dtype=torch.float64, device=sim.device)
            gA = zeros((n, 3, 3)) if gA is None else gA
            gp = zeros((n, 3)) if gp is None else gp
            gAd = zeros((n, 3, 3)) if gAd is None else gAd
            gpd = zeros((n, 3)) if gpd is None else gpd
            qb = _dofs(gA, gp)
            qdb = _dofs(gAd, gpd)
            iters = 0
            starts = sorted(ctx.ckpts)
            for c in reversed(starts):
                end = min(c + cp, steps)
                _load(sim, *ctx.ckpts[c])
                after = []  # the converged DOFs of the segment's steps
                for _ in range(c, end):
                    sim.step()
                    after.append((sim.states.A0.clone(), sim.states.p0.clone()))
                for A, p in reversed(after):
                    qb, qdb, it = adjoint_step(sim, A, p, qb, qdb)
                    iters += it
            ctx.adjoint_iters = iters
            A_b, p_b = _split(qb)
            Ad_b, pd_b = _split(qdb)
            return None, None, None, A_b, p_b, Ad_b, pd_b

    _Trajectory.fn = Trajectory
    return Trajectory


def trajectory(sim, A0, p0, Adot, pdot, steps: int, checkpoint: int = 10):
    """The states (A0, p0, Adot, pdot) after ``steps`` steps from the given initial states, as
    torch tensors on the simulator's device, differentiable with respect to the initial ones
    through the step's adjoint (checkpoints every ``checkpoint`` steps).  The simulator's states
    are overwritten."""
    return _function().apply(sim, int(steps), int(checkpoint), A0, p0, Adot, pdot)
