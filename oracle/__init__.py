"""ctypes wrapper of the CPU FP64 oracle (oracle/abd_oracle.cpp).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline as the checker.  The product (abd_warp_b200) never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libabd_oracle.so")
_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.POINTER
        d, i, v = ctypes.c_double, ctypes.c_int, ctypes.c_void_p
        L.orc_create.restype = v
        L.orc_create.argtypes = [i] + [v] * 10
        L.orc_destroy.argtypes = [v]
        L.orc_get_highlight.argtypes = [v, v]
        L.orc_set_params.argtypes = [v, v]
        L.orc_set_threads.argtypes = [i]
        L.orc_max_threads.restype = i
        L.orc_set_state.argtypes = [v] * 6
        L.orc_get_state.argtypes = [v] * 7
        L.orc_step.argtypes = [v, v]
        L.orc_step.restype = i
        L.orc_transform.argtypes = [v] * 4
        L.orc_collision_set.argtypes = [v, i, v, v, v, v, v, v, i, v]
        L.orc_gh.argtypes = [v, v, v, v, v, v, v, i, v]
        L.orc_gh.restype = i
        L.orc_energy.argtypes = [v, v, v]
        L.orc_energy.restype = d
        L.orc_ccd.argtypes = [v] * 6
        L.orc_ccd.restype = d
        L.orc_contact_gh.argtypes = [i, v, v, v, v, v, v, v, v]
        L.orc_contact_gh.restype = i
        L.orc_contact_terms.argtypes = [i, v, v, v, v]
        L.orc_contact_terms.restype = i
        L.orc_log.argtypes = [d]
        L.orc_log.restype = d
        L.orc_exact_sum.argtypes = [v, ctypes.c_long]
        L.orc_exact_sum.restype = d
        L.orc_inertia_energy_sum.argtypes = [i, v] + [v] * 9
        L.orc_inertia_energy_sum.restype = d
        L.orc_contact_energy.argtypes = [i, v, v]
        L.orc_contact_energy.restype = d
        L.orc_collision_time.argtypes = [i, v, v]
        L.orc_collision_time.restype = d
        L.orc_set_ipc_full.argtypes = [v, i]
        L.orc_full_terms.argtypes = [i, v, v, v, i, v, v, v, v]
        L.orc_full_terms.restype = i
        L.orc_set_friction.argtypes = [v, d, d]
        L.orc_friction_contact.argtypes = [i, v, v, v, d, d, v, v, v, v, v, v]
        L.orc_friction_contact.restype = i
        L.orc_full_hessian.argtypes = [v, v, v, v, i]
        L.orc_full_hessian.restype = i
        L.orc_cubic_roots.argtypes = [v, d, d, v]
        L.orc_cubic_roots.restype = i
        L.orc_solve.argtypes = [v, v]
        L.orc_solve.restype = i
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class OrcInfo(ctypes.Structure):
    _fields_ = [("newton_iters", ctypes.c_int), ("linear_iters", ctypes.c_int), ("ls_trials", ctypes.c_int),
                ("n_pt", ctypes.c_int), ("n_ee", ctypes.c_int), ("n_vg", ctypes.c_int), ("n_ij", ctypes.c_int),
                ("n_active", ctypes.c_int), ("alpha", ctypes.c_double), ("toi", ctypes.c_double),
                ("energy", ctypes.c_double), ("refine_iters", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def _c64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _c32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class Oracle:
    """One scene on the CPU oracle.  ``flat`` comes from
    ``abd_warp_b200.scenes.flatten_bodies``; ``prm`` is a ``SimParams``."""

    def __init__(self, flat: dict, prm):
        L = lib()
        self.flat = flat
        self.n = flat["n"]
        self.V = int(flat["voff"][-1])
        self._keep = [_c32(flat["voff"]), _c32(flat["toff"]), _c32(flat["eoff"]), _c64(flat["x0"]),
                      _c32(flat["tris"]), _c32(flat["edges"]), _c64(flat["mass"]), _c64(flat["I0"]),
                      _c32(flat["fixed"])]
        self._prm = prm.to_c()
        self.h = L.orc_create(self.n, *[_p(a) for a in self._keep], ctypes.byref(self._prm))
        self.set_state(flat["A"], flat["p"], flat["Adot"], flat["pdot"])

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_destroy(self.h)
            self.h = None

    def set_params(self, prm):
        self._prm = prm.to_c()
        lib().orc_set_params(self.h, ctypes.byref(self._prm))

    def set_ipc_full(self, on: bool, independent: bool = False):
        """The full IPC contact model (closest-feature types, edge-edge mollifier, inclusive
        CCD) instead of the reference's interior-only model.  Per contact, the CUDA library's
        arithmetic (its header, so that steps compare bit for bit) or, with independent, the
        oracle's own forward-mode restatement.  SimParams.ipc_full = 1 also selects the first."""
        lib().orc_set_ipc_full(self.h, (2 if independent else 1) if on else 0)

    def set_friction(self, mu: float, eps_v: float = 1e-3):
        """Lagged friction (coefficient mu, slip velocity eps_v) on the full contact model's
        contacts; 0 turns it off."""
        lib().orc_set_friction(self.h, float(mu), float(eps_v))

    def full_hessian(self, A, p, model="full"):
        """Exact, unprojected Hessian of the step's energy at (A, p): dense [12n, 12n], DOFs
        [p, A rows] per body, fixed bodies' rows zero.  model "full": the full contact model
        (needs set_ipc_full(True)); "reference": the reference's interior PT / EE contacts with
        their complete second derivatives."""
        A, p = _c64(A), _c64(p)
        H = np.zeros((12 * self.n, 12 * self.n))
        if lib().orc_full_hessian(self.h, _p(A), _p(p), _p(H), 1 if model == "full" else 0) < 0:
            raise RuntimeError("full_hessian needs set_ipc_full(True)")
        return H

    def set_state(self, A0, p0, Adot, pdot, dq=None):
        A0, p0, Adot, pdot = _c64(A0), _c64(p0), _c64(Adot), _c64(pdot)
        dqa = _c64(dq) if dq is not None else None
        lib().orc_set_state(self.h, _p(A0), _p(p0), _p(Adot), _p(pdot), _p(dqa) if dqa is not None else None)

    def get_state(self):
        n = self.n
        A0, p0 = np.zeros((n, 3, 3)), np.zeros((n, 3))
        Adot, pdot = np.zeros((n, 3, 3)), np.zeros((n, 3))
        dq = np.zeros((n, 12))
        xv = np.zeros((self.V, 3))
        lib().orc_get_state(self.h, _p(A0), _p(p0), _p(Adot), _p(pdot), _p(dq), _p(xv))
        return {"A0": A0, "p0": p0, "Adot": Adot, "pdot": pdot, "dq": dq, "x_view": xv}

    def highlight(self):
        """Per-body contact flags of the last assembly (bool [n])."""
        out = np.zeros(self.n, dtype=np.int32)
        lib().orc_get_highlight(self.h, _p(out))
        return out.astype(bool)

    def step(self):
        info = OrcInfo()
        lib().orc_step(self.h, ctypes.byref(info))
        return info.as_dict()

    def transform(self, A, p):
        A, p = _c64(A), _c64(p)
        x = np.zeros((self.V, 3))
        lib().orc_transform(self.h, _p(A), _p(p), _p(x))
        return x

    def collision_set(self, y0, y1=None, cap=1 << 22):
        """Static (y1 None) or swept culling lists: dict of ij [m,2], pt [k,5], ee [k,5],
        vg [k,2] (body, global vertex)."""
        y0 = _c64(y0)
        y1a = _c64(y1) if y1 is not None else y0
        counts = np.zeros(4, dtype=np.int32)
        bufs = [np.zeros((cap, 2), np.int32), np.zeros((cap, 5), np.int32), np.zeros((cap, 5), np.int32),
                np.zeros((cap, 2), np.int32)]
        lib().orc_collision_set(self.h, 0 if y1 is None else 1, _p(y0), _p(y1a), *[_p(b) for b in bufs], cap,
                                _p(counts))
        if counts.max() > cap:
            return self.collision_set(y0, y1, cap=int(counts.max()))
        return {"ij": bufs[0][:counts[0]].copy(), "pt": bufs[1][:counts[1]].copy(),
                "ee": bufs[2][:counts[2]].copy(), "vg": bufs[3][:counts[3]].copy()}

    def gh(self, A, p, cap=1 << 16):
        A, p = _c64(A), _c64(p)
        n = self.n
        g = np.zeros((n, 12))
        diag = np.zeros((n, 12, 12))
        off = np.zeros((cap, 12, 12))
        ij = np.zeros((cap, 2), np.int32)
        na = ctypes.c_int(0)
        m = lib().orc_gh(self.h, _p(A), _p(p), _p(g), _p(diag), _p(off), _p(ij), cap, ctypes.byref(na))
        if m > cap:
            return self.gh(A, p, cap=m)
        return {"g": g, "diag": diag, "off": off[:m].copy(), "ij": ij[:m].copy(), "n_active": na.value}

    def energy(self, Ak, pk):
        Ak, pk = _c64(Ak), _c64(pk)
        return lib().orc_energy(self.h, _p(Ak), _p(pk))

    def ccd(self, A, p, A1, p1):
        A, p, A1, p1 = _c64(A), _c64(p), _c64(A1), _c64(p1)
        raw = ctypes.c_double(0)
        t = lib().orc_ccd(self.h, _p(A), _p(p), _p(A1), _p(p1), ctypes.byref(raw))
        return t, raw.value

    def solve(self, dq0):
        dq = _c64(dq0).copy()
        it = lib().orc_solve(self.h, _p(dq))
        return dq, it


def contact_gh(type_, x4, r4, prm):
    """Per-pair PT (type 0) / EE (type 1) terms: (active, d2, g24, Hi, Hj, Hij)."""
    x4, r4 = _c64(x4), _c64(r4)
    c = prm.to_c()
    d2 = ctypes.c_double(0)
    g = np.zeros(24)
    Hi, Hj, Hij = np.zeros((12, 12)), np.zeros((12, 12)), np.zeros((12, 12))
    a = lib().orc_contact_gh(type_, _p(x4), _p(r4), ctypes.byref(c), ctypes.byref(d2), _p(g), _p(Hi), _p(Hj),
                             _p(Hij))
    return bool(a), d2.value, g, Hi, Hj, Hij


def contact_terms(type_, x4, r4, prm):
    """Rank-one form of the pair terms: (active, H_IJ, H_II, H_JJ, g24)."""
    x4, r4 = _c64(x4), _c64(r4)
    c = prm.to_c()
    out = np.zeros(456)
    a = lib().orc_contact_terms(type_, _p(x4), _p(r4), ctypes.byref(c), _p(out))
    return bool(a), out[:144].reshape(12, 12), out[144:288].reshape(12, 12), out[288:432].reshape(12, 12), out[432:]


def full_terms(kind, x4, r4, prm, swap=0):
    """Full-model pair terms of one candidate: (active, E, d2, type, H_IJ, H_II, H_JJ, g24)."""
    x4, r4 = _c64(x4), _c64(r4)
    c = prm.to_c()
    out = np.zeros(456)
    E, d2, ty = ctypes.c_double(0), ctypes.c_double(0), ctypes.c_int(0)
    a = lib().orc_full_terms(kind, _p(x4), _p(r4), ctypes.byref(c), swap, _p(out), ctypes.byref(E), ctypes.byref(d2),
                             ctypes.byref(ty))
    return (bool(a), E.value, d2.value, ty.value, out[:144].reshape(12, 12), out[144:288].reshape(12, 12),
            out[288:432].reshape(12, 12), out[432:])


def friction_contact(kind, xt4, r4, prm, mu, eps, x4):
    """One candidate's lagged friction, fixed at xt4 and evaluated at x4:
    (active, D, g (12), H (12x12), weights (4), lambda)."""
    xt4, r4, x4 = _c64(xt4), _c64(r4), _c64(x4)
    c = prm.to_c()
    D, lam = ctypes.c_double(0), ctypes.c_double(0)
    g, H, w = np.zeros(12), np.zeros((12, 12)), np.zeros(4)
    a = lib().orc_friction_contact(kind, _p(xt4), _p(r4), ctypes.byref(c), mu, eps, _p(x4), ctypes.byref(D), _p(g),
                                   _p(H), _p(w), ctypes.byref(lam))
    return bool(a), D.value, g, H, w, lam.value


def abd_log(x: float) -> float:
    """The logarithm shared bit for bit with the CUDA product."""
    return lib().orc_log(float(x))


def exact_sum(values) -> float:
    v = _c64(np.ravel(values))
    return lib().orc_exact_sum(_p(v), len(v))


def inertia_energy_sum(prm, Ak, pk, A0, p0, Adot, pdot, mass, I0, fixed):
    """Exact sum of the bodies' inertia + orthogonality energies (fixed bodies: none)."""
    arrs = [_c64(a) for a in (Ak, pk, A0, p0, Adot, pdot, mass, I0)]
    fx = _c32(fixed)
    c = prm.to_c()
    return lib().orc_inertia_energy_sum(len(fx), ctypes.byref(c), *[_p(a) for a in arrs], _p(fx))


def contact_energy(type_, x4, prm):
    x4 = _c64(x4)
    c = prm.to_c()
    return lib().orc_contact_energy(type_, _p(x4), ctypes.byref(c))


def collision_time(type_, P0, P1):
    P0, P1 = _c64(P0), _c64(P1)
    return lib().orc_collision_time(type_, _p(P0), _p(P1))


def cubic_roots(coef, x0, x1):
    coef = _c64(coef)
    roots = np.zeros(3)
    n = lib().orc_cubic_roots(_p(coef), x0, x1, _p(roots))
    return n, roots


def set_threads(t: int):
    lib().orc_set_threads(int(t))


def max_threads() -> int:
    return lib().orc_max_threads()
