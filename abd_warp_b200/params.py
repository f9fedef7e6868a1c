"""Simulation parameters.

The reference reads its physics constants from module globals (const_params.py:24-44)
and ignores the values in ``AffineBodySimulator.simulator_args`` (abd.py:107-121).
Here every constant is a field of :class:`SimParams`, passed by value to the CUDA
library and to the oracle, so one object fixes the physics of a run.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field, asdict

SOLVER_BICGSTAB = 0
SOLVER_PCG = 1

PRECISION_FP64 = 0
PRECISION_MIXED = 1


@dataclass
class SimParams:
    dt: float = 0.01                 # const_params.py:24
    dhat: float = 1e-3               # barrier distance; d2hat = dhat^2 (const_params.py:33-34)
    kappa: float = 1e6               # barrier stiffness (const_params.py:35)
    stiffness: float = 1e7           # orthogonality stiffness (const_params.py:27)
    gravity: float = -9.8            # y component (const_params.py:32)
    tol: float = 1e-6                # Newton stop: g.g < tol (abd.py:265-268)
    c1: float = 1e-4                 # Armijo constant (const_params.py:28)
    alpha_min: float = 1e-3          # line-search floor (const_params.py:29)
    ls_noise_floor: float = 1e-12    # also accept a trial when |E1 - E0| <= floor |E0|: below the
                                     # energies' rounding error the Armijo test is noise
    max_iter: int = 10               # Newton iteration cap: the value step() reads (const_params.py:25
                                     # via abd.py:1); simulator_args' 100 (abd.py:114) is never used
    armijo_sign: int = -1            # -1: E1 < E0 - c1 a dq.g ; +1: reference form abd.py:156
    ground_enabled: bool = False     # vertex-ground plane contact (culling.py:54-82)
    ground: float = -0.5             # plane height (const_params.py:36)
    psd_ee: bool = False             # contact_psd 0 only: clamp EE eigenvalues too (ee_ipc.py:33-36)
    contact_psd: int = 1             # 1: PSD-project the barrier Hessian (mu_k = B' lam_k, clamped);
                                     # 0: reference form, clamp lam_k then scale by B' < 0
                                     #    (pt_ipc.py:166, 266-269)
    enable_pt: bool = True           # const_params.py:41-43
    enable_ee: bool = True
    enable_vg: bool = True
    solver: int = SOLVER_PCG         # the reference calls bicgstab (abd.py:244); the projected
                                     # Hessian is SPD, so CG is the default
    precond: int = 1                 # 1: contact-cluster block Jacobi; 0: per-body 12x12 blocks
    cluster_max: int = 12            # bodies per preconditioner cluster
    cg_tol: float = 1e-10            # stop when r^T M^-1 r <= cg_tol^2 b^T M^-1 b
    cg_max_iter: int = 2000
    precision: int = PRECISION_FP64  # the CUDA library accepts FP64 only; the oracle also runs
                                     # PRECISION_MIXED (FP32 PCG inside FP64 refinement), which
                                     # diverges once bodies touch (cond(H) ~ 1e10 > 1 / eps_FP32)
    refine_tol: float = 1e-4         # oracle mixed precision: the FP32 inner solve's relative tolerance
    newton_loop: int = 0             # 0: the step's Newton iterations run as a device loop (one graph
                                     # launch per step); 1: the host drives them (same results)
    ipc_full: int = 0                # 1: the full IPC contact model (closest-feature types, edge-edge
                                     # mollifier, per-contact PSD projection, inclusive CCD); 0: the
                                     # reference's interior-only model
    min_capacity: int = 0            # > 0: every list of the simulator starts this small and the
                                     # traversal frontier holds at most this many nodes (tests force
                                     # the grow-and-rerun paths and the depth-first fallback with it)
    friction_mu: float = 0.0         # lagged IPC friction (not in the reference; needs ipc_full = 1):
                                     # the Coulomb coefficient, 0 = off
    friction_epsv: float = 1e-3      # its static-friction slip velocity (eps = friction_epsv dt)

    @property
    def d2hat(self) -> float:
        return self.dhat * self.dhat

    def to_c(self) -> "CParams":
        c = CParams()
        c.dt = self.dt
        c.dhat = self.dhat
        c.d2hat = self.d2hat
        c.kappa = self.kappa
        c.stiffness = self.stiffness
        c.gravity = self.gravity
        c.tol = self.tol
        c.c1 = self.c1
        c.alpha_min = self.alpha_min
        c.ground = self.ground
        c.cg_tol = self.cg_tol
        c.refine_tol = self.refine_tol
        c.ls_noise_floor = self.ls_noise_floor
        c.max_iter = self.max_iter
        c.armijo_sign = self.armijo_sign
        c.ground_enabled = int(self.ground_enabled)
        c.psd_ee = int(self.psd_ee)
        c.enable_pt = int(self.enable_pt)
        c.enable_ee = int(self.enable_ee)
        c.enable_vg = int(self.enable_vg)
        c.solver = self.solver
        c.cg_max_iter = self.cg_max_iter
        c.precision = self.precision
        c.contact_psd = self.contact_psd
        c.precond = self.precond
        c.cluster_max = self.cluster_max
        c.min_capacity = self.min_capacity
        c.newton_loop = self.newton_loop
        c.ipc_full = self.ipc_full
        c.friction_mu = self.friction_mu
        c.friction_epsv = self.friction_epsv
        return c

    def as_dict(self):
        return asdict(self)


class CParams(ctypes.Structure):
    """Mirror of ``abd_params`` in include/abd_b200.h (and of the oracle's copy)."""
    _fields_ = [
        ("dt", ctypes.c_double), ("dhat", ctypes.c_double), ("d2hat", ctypes.c_double),
        ("kappa", ctypes.c_double), ("stiffness", ctypes.c_double), ("gravity", ctypes.c_double),
        ("tol", ctypes.c_double), ("c1", ctypes.c_double), ("alpha_min", ctypes.c_double),
        ("ground", ctypes.c_double), ("cg_tol", ctypes.c_double), ("refine_tol", ctypes.c_double),
        ("ls_noise_floor", ctypes.c_double),
        ("max_iter", ctypes.c_int), ("armijo_sign", ctypes.c_int), ("ground_enabled", ctypes.c_int),
        ("psd_ee", ctypes.c_int), ("enable_pt", ctypes.c_int), ("enable_ee", ctypes.c_int),
        ("enable_vg", ctypes.c_int), ("solver", ctypes.c_int), ("cg_max_iter", ctypes.c_int),
        ("precision", ctypes.c_int), ("contact_psd", ctypes.c_int), ("precond", ctypes.c_int),
        ("cluster_max", ctypes.c_int), ("min_capacity", ctypes.c_int), ("newton_loop", ctypes.c_int),
        ("ipc_full", ctypes.c_int), ("friction_mu", ctypes.c_double), ("friction_epsv", ctypes.c_double),
    ]
