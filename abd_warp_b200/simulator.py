"""``AffineBodySimulator``: the reference's simulator API (abd/abd.py:16-333) on the B200
library.

Construction mirrors ``AffineBodySimulator(config_file)`` / ``BaseSimulator.__init__``
(abd/abd.py:21-95, simulator/base.py:31-45): the config JSON names a scene JSON whose
``objects`` become :class:`AffineMesh` bodies, and its ``simulator_args`` keys (frame range,
``save_sequence``, output folder, verbosity; simulator/base.py:17-28) become attributes.
Unlike the reference, the physics keys of the config (``dt, dhat, kappa, stiffness, tol,
max_iter`` and any other :class:`SimParams` field) are honoured (the reference ignores them,
abd/abd.py:107-121).  Scenes can also be passed directly as a list of bodies.

Headless trajectory export replaces the reference's viewer loop (abd/abd.py:364-416) and its
``export_frame`` stub (simulator/base.py:70-75): ``run()`` steps the frames
``[frame_in, frame_out)`` and, with ``save_sequence``, writes each frame's vertex positions to
``output_seq_folder/frame_NNNN.npz`` (read back by :func:`load_trajectory`).

All arrays live on one CUDA device as float64 torch tensors.  ``step()`` runs the whole
Newton time step inside libabd_b200.so; the stage methods (``collision_set``,
``compute_energy``, ``ccd``, ``gradient_hessian``, ``solve``) expose the pieces for testing.
"""
from __future__ import annotations

import ctypes
import json
import os

import numpy as np

from . import _lib
from .affine_body import AffineMesh, Scene, WarpMesh, affine_body_states_empty
from .params import SimParams
from .scenes import flatten_bodies


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


class AffineBodySimulator:
    """One scene of affine bodies on the GPU.

    Attributes (as in the reference): ``scene``, ``n_bodies``, ``states``
    (:class:`AffineBodyStates`), ``meshes`` (list of :class:`WarpMesh` views), ``highlight``
    (numpy bool per body), plus ``g`` / ``dq`` properties, ``params`` and ``last_info``.
    """

    @classmethod
    def simulator_args(cls):
        """Frame-loop arguments and their defaults, overridden by the config file's keys
        (simulator/base.py:17-28)."""
        return {
            "frame_in": 0,
            "frame_out": 100,
            "save_sequence": False,
            "input_seq_folder": "bgeo/",
            "output_seq_folder": "bgeo/",
            "verbose": 0,
        }

    def __init__(self, config_file: str | None = None, bodies=None, params: SimParams | None = None,
                 device: str = "cuda", mesh_map: dict | None = None):
        import torch
        self.torch = torch
        self.params = params if params is not None else SimParams()
        config = {}
        if config_file is not None:
            with open(config_file) as f:
                config = json.load(f)
            for k, v in config.items():
                if hasattr(self.params, k) and not k.startswith("_"):
                    setattr(self.params, k, v)
        for k, v in self.simulator_args().items():
            setattr(self, k, config.get(k, v))
        if config_file is not None:
            here = os.path.dirname(os.path.abspath(config_file))
            for k in ("input_seq_folder", "output_seq_folder"):
                if k in config and not os.path.isabs(getattr(self, k)):
                    setattr(self, k, os.path.join(here, getattr(self, k)))
            scene_file = config["scene"]
            if not os.path.isabs(scene_file):
                scene_file = os.path.join(here, scene_file)
            mesh_map = {**config.get("mesh_map", {}), **(mesh_map or {})}
            self.scene = Scene(AffineMesh, scene_config_file=scene_file, mesh_map=mesh_map)
        else:
            if bodies is None:
                raise ValueError("pass config_file or bodies")
            self.scene = Scene(AffineMesh, objects=list(bodies))
        bodies = self.scene.kinetic_objects
        self.n_bodies = n = len(bodies)
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise _lib.AbdError("AffineBodySimulator runs on a CUDA device only")
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.flat = flat = flatten_bodies(bodies)
        self.n_verts = int(flat["voff"][-1])
        L = _lib.load()
        dev = self.device
        f64 = dict(dtype=torch.float64, device=dev)
        self.states = affine_body_states_empty(n, dev)
        self.states.mass.copy_(torch.as_tensor(flat["mass"]))
        self.states.I0.copy_(torch.as_tensor(flat["I0"]))
        self.x0 = torch.as_tensor(flat["x0"], **f64)
        self.x = torch.zeros_like(self.x0)
        self.xk = torch.zeros_like(self.x0)
        self.x_view = torch.zeros_like(self.x0)
        self.meshes = []
        for i, b in enumerate(bodies):
            v0, v1 = int(flat["voff"][i]), int(flat["voff"][i + 1])
            self.meshes.append(WarpMesh(
                id=i, x0=self.x0[v0:v1], x=self.x[v0:v1], xk=self.xk[v0:v1], x_view=self.x_view[v0:v1],
                triangles=torch.as_tensor(b.F, dtype=torch.int32, device=dev),
                edges=torch.as_tensor(b.edges, dtype=torch.int32, device=dev)))
        self.last_info = None
        # C ABI scene description (host arrays are copied by abd_sim_create)
        self._host = {k: np.ascontiguousarray(flat[k], dtype=np.int32 if k in ("voff", "toff", "eoff", "tris", "edges", "fixed") else np.float64)
                      for k in ("voff", "toff", "eoff", "x0", "tris", "edges", "mass", "I0", "fixed")}
        hp = {k: v.ctypes.data_as(ctypes.c_void_p) for k, v in self._host.items()}
        desc = _lib.SceneDesc(n, hp["voff"], hp["toff"], hp["eoff"], hp["x0"], hp["tris"], hp["edges"],
                              hp["mass"], hp["I0"], hp["fixed"])
        self._cprm = self.params.to_c()
        h = ctypes.c_void_p()
        torch.cuda.set_device(dev)
        stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
        _lib.check(L.abd_sim_create(ctypes.byref(desc), ctypes.byref(self._cprm), stream, ctypes.byref(h)),
                   "abd_sim_create")
        self._h = h
        self._L = L
        self.reset()

    # ------------------------------------------------------------------ lifecycle
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self.torch.cuda.synchronize(self.device)
            self._L.abd_sim_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, params: SimParams):
        self.params = params
        self._cprm = params.to_c()
        _lib.check(self._L.abd_sim_set_params(self._h, ctypes.byref(self._cprm)), "abd_sim_set_params")

    def _cstates(self):
        s = self.states
        return _lib.States(*[_ptr(t) for t in (s.A, s.p, s.Ak, s.pk, s.Adot, s.pdot, s.A0, s.p0)])

    def gather(self, field):
        """Stack a per-body field of the scene objects (simulator/base.py:78-79)."""
        return np.array([getattr(ko, field) for ko in self.scene.kinetic_objects])

    def reset(self):
        """Initial states from the scene, dq = 0, meshes at their initial pose
        (abd/abd.py:97-104)."""
        t = self.torch
        s = self.states
        s.A0.copy_(t.as_tensor(self.gather("A")))
        s.p0.copy_(t.as_tensor(self.gather("p")))
        s.pdot.copy_(t.as_tensor(self.gather("pdot")))
        s.Adot.copy_(t.as_tensor(self.gather("Adot")))
        s.A.copy_(s.A0)
        s.p.copy_(s.p0)
        s.Ak.copy_(s.A0)
        s.pk.copy_(s.p0)
        _lib.check(self._L.abd_sim_reset(self._h), "abd_sim_reset")
        self.update_mesh_vertex("x")
        self.xk.copy_(self.x)
        self.x_view.copy_(self.x)

    # ------------------------------------------------------------------ the time step
    def step(self, frame: int = 1):
        """One implicit time step (abd/abd.py:212-276); updates ``states`` in place and
        ``x_view`` to the new positions."""
        info = _lib.StepInfo()
        cst = self._cstates()
        _lib.check(self._L.abd_step(self._h, ctypes.byref(cst), _ptr(self.x_view), ctypes.byref(info)), "abd_step")
        self.last_info = info.as_dict()
        return self.last_info

    # ------------------------------------------------------------------ frames
    def export_frame(self, frame: int, folder: str | None = None):
        """Write the current ``x_view`` (vertex positions of the last completed step) and the
        bodies' DOFs to ``folder/frame_NNNN.npz`` (default ``output_seq_folder``); returns the
        path.  Headless stand-in for the reference's bgeo export (simulator/base.py:70-75)."""
        folder = self.output_seq_folder if folder is None else folder
        os.makedirs(folder, exist_ok=True)
        path = os.path.join(folder, f"frame_{frame:04d}.npz")
        s = self.states
        np.savez(path, frame=np.int64(frame), x=self.x_view.cpu().numpy(), A=s.A0.cpu().numpy(),
                 p=s.p0.cpu().numpy(), vert_off=self.flat["voff"])
        return path

    def run(self, frame_in: int | None = None, frame_out: int | None = None, save_sequence: bool | None = None):
        """Step the frames [frame_in, frame_out) (defaults from the config), exporting each
        frame's positions when ``save_sequence``; returns the per-step infos.  This replaces
        the viewer's callback loop (abd/abd.py:364-416), which calls ``step(frame)`` once per
        frame."""
        f0 = self.frame_in if frame_in is None else frame_in
        f1 = self.frame_out if frame_out is None else frame_out
        save = self.save_sequence if save_sequence is None else save_sequence
        infos = []
        for frame in range(f0, f1):
            infos.append(self.step(frame))
            if save:
                self.export_frame(frame)
            if self.verbose:
                print(f"frame {frame}: {infos[-1]}")
        return infos

    # ------------------------------------------------------------------ stages
    def update_mesh_vertex(self, field: str = "x"):
        """``x = p + sum_k r_k a_k`` into ``x`` / ``xk`` / ``x_view`` from (A, p) / (Ak, pk) /
        (A0, p0) (abd/abd.py:305-324).  Returns the per-axis minimum."""
        s = self.states
        A, p = {"x": (s.A, s.p), "xk": (s.Ak, s.pk), "x_view": (s.A0, s.p0)}[field]
        out = getattr(self, field)
        _lib.check(self._L.abd_update_mesh_vertex(self._h, _ptr(A), _ptr(p), _ptr(out)), "abd_update_mesh_vertex")
        return out.min(dim=0).values

    def transform(self, A, p):
        out = self.torch.empty_like(self.x0)
        _lib.check(self._L.abd_update_mesh_vertex(self._h, _ptr(A.contiguous()), _ptr(p.contiguous()), _ptr(out)),
                   "abd_update_mesh_vertex")
        return out

    def _lists(self, y0, y1, dofs=None):
        t = self.torch
        counts = (ctypes.c_int * 4)()
        if dofs is None:
            _lib.check(self._L.abd_collision_set(self._h, _ptr(y0), _ptr(y1) if y1 is not None else None, counts),
                       "abd_collision_set")
        else:
            A, p, A1, p1 = (None if v is None else _ptr(v.contiguous()) for v in dofs)
            _lib.check(self._L.abd_collision_set_dofs(self._h, A, p, A1, p1, counts), "abd_collision_set_dofs")
        cap = max(1, max(counts))
        i32 = dict(dtype=t.int32, device=self.device)
        ij, pt, ee, vg = (t.zeros((cap, 2), **i32), t.zeros((cap, 5), **i32), t.zeros((cap, 5), **i32),
                          t.zeros((cap, 2), **i32))
        _lib.check(self._L.abd_export_lists(self._h, _ptr(ij), _ptr(pt), _ptr(ee), _ptr(vg), cap), "abd_export_lists")
        return ij[:counts[0]], pt[:counts[1]], ee[:counts[2]], vg[:counts[3]]

    def collision_set(self, y=None):
        """Culling on positions ``y`` (default ``xk``): ``(ij, ee, pt, vg)`` as the reference
        returns them (abd/abd.py:187-207); pt/ee rows are (I, J, pair, prim of I, prim of J)."""
        y = self.xk if y is None else y
        ij, pt, ee, vg = self._lists(y.contiguous(), None)
        return ij, ee, pt, vg

    def trajectory_intersection_set(self, y0=None, y1=None):
        """Culling on the swept boxes x -> xk: ``(ij, pt, ee, vg)`` (abd/abd.py:170-185)."""
        y0 = self.x if y0 is None else y0
        y1 = self.xk if y1 is None else y1
        ij, pt, ee, vg = self._lists(y0.contiguous(), y1.contiguous())
        return ij, pt, ee, vg

    def collision_set_dofs(self, A, p, A1=None, p1=None):
        """Culling at DOFs as the time step runs it: positions ``transform(A, p)`` (swept to
        ``transform(A1, p1)`` when given) land in ``x`` / ``xk``; returns ``(ij, pt, ee, vg)``."""
        return self._lists(None, None, (A, p, A1, p1))

    def gradient_hessian(self, A=None, p=None):
        """Assemble g and the block system at DOFs (A, p) (default the current ones):
        returns dict(g [n,12], diag [n,12,12], off [m,12,12], ij [m,2], n_active)."""
        t = self.torch
        s = self.states
        A = s.A if A is None else A.contiguous()
        p = s.p if p is None else p.contiguous()
        na = ctypes.c_int(0)
        cst = self._cstates()
        _lib.check(self._L.abd_ipc_gh(self._h, ctypes.byref(cst), _ptr(A), _ptr(p), ctypes.byref(na)), "abd_ipc_gh")
        n = self.n_bodies
        npairs = ctypes.c_int(0)
        g = t.zeros((n, 12), dtype=t.float64, device=self.device)
        diag = t.zeros((n, 12, 12), dtype=t.float64, device=self.device)
        _lib.check(self._L.abd_export_system(self._h, _ptr(g), _ptr(diag), None, None, 0, ctypes.byref(npairs)),
                   "abd_export_system")
        m = npairs.value
        off = t.zeros((max(m, 1), 12, 12), dtype=t.float64, device=self.device)
        ij = t.zeros((max(m, 1), 2), dtype=t.int32, device=self.device)
        _lib.check(self._L.abd_export_system(self._h, None, None, _ptr(off), _ptr(ij), m, ctypes.byref(npairs)),
                   "abd_export_system")
        return {"g": g, "diag": diag, "off": off[:m], "ij": ij[:m], "n_active": na.value}

    def solve(self, dq0=None):
        """Solve the last assembled system H dq = g, warm-started from dq0 (default: the
        simulator's dq).  Returns (dq, iterations)."""
        t = self.torch
        dq = (self.dq if dq0 is None else dq0).contiguous().clone()
        it = ctypes.c_int(0)
        _lib.check(self._L.abd_solve(self._h, _ptr(dq), ctypes.byref(it)), "abd_solve")
        return dq, it.value

    def compute_energy(self, Ak=None, pk=None):
        """Total energy at trial DOFs (default Ak, pk) (abd/abd.py:133-141)."""
        s = self.states
        Ak = s.Ak if Ak is None else Ak.contiguous()
        pk = s.pk if pk is None else pk.contiguous()
        E = ctypes.c_double(0)
        cst = self._cstates()
        _lib.check(self._L.abd_compute_energy(self._h, ctypes.byref(cst), _ptr(Ak), _ptr(pk), ctypes.byref(E)),
                   "abd_compute_energy")
        return E.value

    def ccd(self, A, p, A1, p1):
        """Step bound between two DOF sets (abd/abd.py:278-303): (alpha, raw toi)."""
        a = ctypes.c_double(0)
        raw = ctypes.c_double(0)
        _lib.check(self._L.abd_ccd(self._h, _ptr(A.contiguous()), _ptr(p.contiguous()), _ptr(A1.contiguous()),
                                   _ptr(p1.contiguous()), ctypes.byref(a), ctypes.byref(raw)), "abd_ccd")
        return a.value, raw.value

    def energies_along(self, alphas, A=None, p=None):
        """Energies at (A, p) - alpha dq for step lengths 0 <= alpha <= 1 along the current dq
        (default A, p: the states' iterate), as the step's line search evaluates its trials:
        one culling pass over the whole segment, then the trials in batches.  Each value is
        bitwise compute_energy at the same DOFs.  Ak, pk receive (A, p) - dq."""
        s = self.states
        A = s.A if A is None else A.contiguous()
        p = s.p if p is None else p.contiguous()
        al = (ctypes.c_double * max(1, len(alphas)))(*[float(a) for a in alphas])
        E = (ctypes.c_double * max(1, len(alphas)))()
        cst = self._cstates()
        _lib.check(self._L.abd_energies_along(self._h, ctypes.byref(cst), _ptr(A), _ptr(p), al, len(alphas), E),
                   "abd_energies_along")
        return [E[k] for k in range(len(alphas))]

    # ------------------------------------------------------------------ contact flags
    @property
    def highlight(self):
        """Per-body contact flags of the last gradient / Hessian pass (the last step's last
        Newton iteration), numpy bool [n]: the reference's ``sim.highlight``, which the step
        sets from its contact pass (abd/abd.py:238) and the viewer colours bodies by
        (abd/abd.py:412-413).  A body is flagged when it takes part in an active PT, EE or
        vertex-ground contact.  Read from the device on access."""
        t = self.torch
        out = t.zeros(self.n_bodies, dtype=t.int32, device=self.device)
        _lib.check(self._L.abd_get_highlight(self._h, _ptr(out)), "abd_get_highlight")
        return out.cpu().numpy().astype(bool)

    def take_status(self) -> int:
        """Device status bits accumulated since the last call (and cleared); see
        ``_lib.STATUS_NAMES``."""
        st = ctypes.c_int(0)
        _lib.check(self._L.abd_take_status(self._h, ctypes.byref(st)), "abd_take_status")
        return st.value

    # ------------------------------------------------------------------ dq / g
    @property
    def dq(self):
        """The warm-started Newton step (reference ``sim.dq``), [n, 12] float64."""
        t = self.torch
        out = t.empty((self.n_bodies, 12), dtype=t.float64, device=self.device)
        _lib.check(self._L.abd_sim_get_dq(self._h, _ptr(out)), "abd_sim_get_dq")
        return out

    @dq.setter
    def dq(self, value):
        t = self.torch
        v = value.to(self.device, t.float64).contiguous()
        _lib.check(self._L.abd_sim_set_dq(self._h, _ptr(v)), "abd_sim_set_dq")

    @property
    def g(self):
        """The last assembled gradient (reference ``sim.g``), [n, 12] float64."""
        t = self.torch
        out = t.empty((self.n_bodies, 12), dtype=t.float64, device=self.device)
        _lib.check(self._L.abd_sim_get_g(self._h, _ptr(out)), "abd_sim_get_g")
        return out

    def profile(self, mode: int = 1):
        """Start (reset) or stop (0) the timing of the step's CCD-pass narrow kernel (which also
        collects the line-search candidates); mode 2 also counts the data it moves (algorithmic
        bytes), which slows the kernel down."""
        _lib.check(self._L.abd_profile(self._h, int(mode)), "abd_profile")

    def profile_read(self):
        """(kernel ms, launches, algorithmic bytes) accumulated since profile()."""
        ms, n, b = ctypes.c_double(0), ctypes.c_longlong(0), ctypes.c_double(0)
        _lib.check(self._L.abd_profile_read(self._h, ctypes.byref(ms), ctypes.byref(n), ctypes.byref(b)),
                   "abd_profile_read")
        return ms.value, n.value, b.value

    def launch_count(self) -> int:
        return int(self._L.abd_launch_count(self._h))


def load_trajectory(folder: str):
    """Frames written by :meth:`AffineBodySimulator.export_frame`, in frame order: a dict of
    ``frames`` [F], ``x`` [F, V, 3], ``A`` [F, n, 3, 3], ``p`` [F, n, 3] and ``vert_off``."""
    names = sorted(f for f in os.listdir(folder) if f.startswith("frame_") and f.endswith(".npz"))
    if not names:
        raise FileNotFoundError(f"no frame_*.npz in {folder}")
    data = [np.load(os.path.join(folder, f)) for f in names]
    return {"frames": np.array([int(d["frame"]) for d in data]), "x": np.stack([d["x"] for d in data]),
            "A": np.stack([d["A"] for d in data]), "p": np.stack([d["p"] for d in data]),
            "vert_off": data[0]["vert_off"]}
