"""ctypes binding of libabd_b200.so (C ABI declared in include/abd_b200.h).

The library is built in-tree by ``abd_warp_b200/build.py``.  There is no fallback: if it is
missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

from .params import CParams

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libabd_b200.so")

ABD_OK = 0
ABD_ERR_CUDA, ABD_ERR_INVALID, ABD_ERR_OVERFLOW, ABD_ERR_DEVICE = 1, 2, 3, 4  # include/abd_b200.h
STATUS_NAMES = {1: "pt_overflow", 2: "ee_overflow", 4: "pair_overflow", 8: "stack_overflow",
                16: "solver_not_converged", 32: "nan", 64: "vg_overflow", 128: "active_pair_overflow",
                256: "contact_overflow", 512: "ccd_overflow", 1024: "ls_candidate_overflow",
                2048: "line_search_needs_more_trials", 4096: "friction_contact_overflow"}
ST_STACK_OVERFLOW, ST_SOLVER_NOCONV, ST_NAN = 8, 16, 32

c_int, c_double, c_void_p, c_longlong = ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_longlong


class SceneDesc(ctypes.Structure):
    _fields_ = [("n_bodies", c_int), ("vert_off", c_void_p), ("tri_off", c_void_p), ("edge_off", c_void_p),
                ("x0", c_void_p), ("tris", c_void_p), ("edges", c_void_p), ("mass", c_void_p), ("I0", c_void_p),
                ("fixed", c_void_p)]


class States(ctypes.Structure):
    _fields_ = [(k, c_void_p) for k in ("A", "p", "Ak", "pk", "Adot", "pdot", "A0", "p0")]


class StepInfo(ctypes.Structure):
    _fields_ = [("newton_iters", c_int), ("linear_iters", c_int), ("ls_trials", c_int), ("n_pt", c_int),
                ("n_ee", c_int), ("n_vg", c_int), ("n_ij", c_int), ("n_active", c_int), ("alpha", c_double),
                ("toi", c_double), ("energy", c_double), ("status", c_int), ("refine_iters", c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class AbdError(RuntimeError):
    pass


_lib = None


def load():
    """Load libabd_b200.so (raises if it is absent: there is no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise AbdError(f"{LIB_PATH} is missing; build it with `python -m abd_warp_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    P = c_void_p
    sig = {
        "abd_sim_create": ([P, P, P, P], c_int),
        "abd_sim_destroy": ([P], c_int),
        "abd_sim_set_params": ([P, P], c_int),
        "abd_sim_set_stream": ([P, P], c_int),
        "abd_sim_reset": ([P], c_int),
        "abd_sim_get_dq": ([P, P], c_int),
        "abd_sim_set_dq": ([P, P], c_int),
        "abd_sim_get_g": ([P, P], c_int),
        "abd_sim_sizes": ([P, P, P, P, P], c_int),
        "abd_step": ([P, P, P, P], c_int),
        "abd_update_mesh_vertex": ([P, P, P, P], c_int),
        "abd_collision_set": ([P, P, P, P], c_int),
        "abd_collision_set_dofs": ([P, P, P, P, P, P], c_int),
        "abd_export_lists": ([P, P, P, P, P, c_int], c_int),
        "abd_ipc_gh": ([P, P, P, P, P], c_int),
        "abd_export_system": ([P, P, P, P, P, c_int, P], c_int),
        "abd_solve": ([P, P, P], c_int),
        "abd_compute_energy": ([P, P, P, P, P], c_int),
        "abd_ccd": ([P, P, P, P, P, P, P], c_int),
        "abd_energies_along": ([P, P, P, P, P, c_int, P], c_int),
        "abd_get_highlight": ([P, P], c_int),
        "abd_adjoint_step": ([P, P, P, P, P, P, P, P, P], c_int),
        "abd_batch_create": ([c_int, P, P, P], c_int),
        "abd_batch_destroy": ([P], c_int),
        "abd_batch_step": ([P, P, P, P], c_int),
        "abd_take_status": ([P, P], c_int),
        "abd_status_string": ([c_int], ctypes.c_char_p),
        "abd_error_detail": ([], ctypes.c_char_p),
        "abd_launch_count": ([P], c_longlong),
        "abd_profile": ([P, c_int], c_int),
        "abd_profile_read": ([P, P, P, P], c_int),
        "abd_fp64_peak": ([P], c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def exported_symbols():
    """Names of the C ABI entry points this binding expects (all must resolve)."""
    load()
    return ["abd_sim_create", "abd_sim_destroy", "abd_sim_set_params", "abd_sim_set_stream", "abd_sim_reset",
            "abd_sim_get_dq", "abd_sim_set_dq", "abd_sim_get_g", "abd_sim_sizes", "abd_step", "abd_update_mesh_vertex",
            "abd_collision_set", "abd_collision_set_dofs", "abd_export_lists", "abd_ipc_gh", "abd_export_system", "abd_solve",
            "abd_compute_energy", "abd_ccd", "abd_energies_along", "abd_get_highlight", "abd_adjoint_step", "abd_batch_create", "abd_batch_destroy", "abd_batch_step", "abd_take_status", "abd_status_string", "abd_error_detail", "abd_launch_count",
            "abd_profile", "abd_profile_read", "abd_fp64_peak"]


def check(rc: int, what: str = ""):
    if rc != ABD_OK:
        L = load()
        msg = L.abd_status_string(rc).decode()
        if rc == ABD_ERR_CUDA:
            msg += f" [{L.abd_error_detail().decode()}]"
        raise AbdError(f"{what}: {msg} (code {rc})")


def params_ptr(prm) -> CParams:
    return prm.to_c()
