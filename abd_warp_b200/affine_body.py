"""Data model: per-body meshes and the structure-of-arrays body state.

Mirrors the reference's ``AffineBodyStates`` (affine_body.py:7-21),
``affine_body_states_empty`` (affine_body.py:24-40), ``WarpMesh`` (affine_body.py:42-51)
and ``AffineMesh`` (affine_body.py:54-97).

Convention (one for the whole package): the degrees of freedom of a body are ``p`` and the
three rows ``a_k`` of ``A``; a rest vertex ``r`` maps to ``x = p + r_0 a_0 + r_1 a_1 + r_2 a_2``,
i.e. ``x = A^T r + p`` as in the simulator (abd.py:31, abd.py:313-316).  The reference's
``AffineMesh.assign_to`` uses ``A r + p`` (affine_body.py:79); it only agrees because every
reference scene has ``A = I``.  Here ``assign_to`` uses the simulator's convention.
"""
from __future__ import annotations

import json
import os
from dataclasses import dataclass

import numpy as np

from .meshes import box_mesh, cube_mesh, icosphere_mesh, mass_properties, unique_edges

DEFAULT_DENSITY = 1000.0


def _read_obj(path: str):
    V, F = [], []
    with open(path) as f:
        for line in f:
            s = line.split()
            if not s:
                continue
            if s[0] == "v":
                V.append([float(t) for t in s[1:4]])
            elif s[0] == "f":
                idx = [int(t.split("/")[0]) - 1 for t in s[1:]]
                for k in range(1, len(idx) - 1):
                    F.append([idx[0], idx[k], idx[k + 1]])
    return np.asarray(V, dtype=np.float64), np.asarray(F, dtype=np.int32)


def mesh_from_spec(spec: str, folder: str = "", mesh_map: dict | None = None):
    """Procedural mesh names stand in for the reference's asset files
    (simulator/mesh.py:37-55): ``cube[:edge]``, ``box:sx,sy,sz``,
    ``icosphere:level[:radius]``, or a path to an ``.obj`` file.  ``mesh_map`` renames asset
    files that have no reader here (the reference's ``.bgeo`` / ``.usd`` assets) to one of
    those, e.g. ``{"box.bgeo": "cube:1.0"}``."""
    if mesh_map and spec in mesh_map:
        return mesh_from_spec(mesh_map[spec], folder)
    kind = spec.split(":")[0]
    if kind == "cube":
        parts = spec.split(":")
        return cube_mesh(float(parts[1]) if len(parts) > 1 else 1.0)
    if kind == "box":
        parts = spec.split(":")
        if len(parts) == 1:
            return cube_mesh(1.0)
        sx, sy, sz = (float(t) for t in parts[1].split(","))
        return box_mesh(sx, sy, sz)
    if kind == "icosphere":
        parts = spec.split(":")
        level = int(parts[1]) if len(parts) > 1 else 2
        radius = float(parts[2]) if len(parts) > 2 else 1.0
        return icosphere_mesh(level, radius)
    if spec.endswith(".obj"):
        return _read_obj(os.path.join(folder, spec))
    raise ValueError(f"unsupported mesh '{spec}': bgeo/usd readers are not available; "
                     "use cube / box / icosphere or an .obj file, or map the name with mesh_map")


class AffineMesh:
    """I/O-side description of one affine body (affine_body.py:54-97).

    Fields: ``V`` (rest vertices, centred at the centre of mass), ``F``, ``edges``,
    ``A``, ``p``, ``Adot``, ``pdot``, ``mass``, ``I0`` and ``fixed`` (Dirichlet body;
    the reference has no fixed bodies).
    """

    @classmethod
    def states_default(cls):
        return {
            "A": np.identity(3),
            "p": np.zeros(3),
            "Adot": np.zeros((3, 3)),
            "pdot": np.zeros(3),
        }

    def __init__(self, obj_json: dict, density: float = DEFAULT_DENSITY, mesh_map: dict | None = None):
        spec = obj_json.get("file", "cube")
        V, F = mesh_from_spec(spec, obj_json.get("folder", ""), mesh_map)
        mass, com, I0 = mass_properties(V, F, density)
        self.V = np.ascontiguousarray(V - com, dtype=np.float64)
        self.F = np.ascontiguousarray(F, dtype=np.int32)
        self.edges = unique_edges(self.F)
        for key, value in self.states_default().items():
            setattr(self, key, np.array(obj_json.get(key, value), dtype=np.float64))
        self.mass = float(obj_json.get("mass", mass))
        self.I0 = float(obj_json.get("I0", I0))
        self.fixed = bool(obj_json.get("fixed", False))
        self.name = spec

    def vertices_world(self):
        """``x = A^T r + p`` for every rest vertex (abd.py:313-316)."""
        return self.V @ self.A + self.p.reshape(1, 3)

    def assign_to(self, ab: "WarpMesh"):
        """Write rest shape and current positions into a device mesh view
        (affine_body.py:73-82, with the simulator's ``A^T r + p`` convention)."""
        import torch
        x = torch.as_tensor(self.vertices_world(), dtype=torch.float64)
        ab.x0.copy_(torch.as_tensor(self.V))
        ab.x.copy_(x)
        ab.xk.copy_(x)
        ab.x_view.copy_(x)


@dataclass
class WarpMesh:
    """Per-body device view (affine_body.py:42-51): rows of the simulator's concatenated
    vertex buffers, plus the body's local triangle and edge indices."""
    id: int
    x0: "object"
    x: "object"
    xk: "object"
    x_view: "object"
    triangles: "object"
    edges: "object"


@dataclass
class AffineBodyStates:
    """Structure of arrays of body states (affine_body.py:7-21), float64 torch tensors:
    ``A, Ak, Adot, A0`` are ``[n, 3, 3]`` (row k = DOF a_k), ``p, pk, pdot, p0`` are ``[n, 3]``,
    ``mass, I0`` are ``[n]``."""
    A: "object"
    p: "object"
    Ak: "object"
    pk: "object"
    Adot: "object"
    pdot: "object"
    A0: "object"
    p0: "object"
    mass: "object"
    I0: "object"


def affine_body_states_empty(n_bodies: int, device="cuda") -> AffineBodyStates:
    """Zero-initialised states (affine_body.py:24-40), with the per-body ``mass`` and
    ``I0`` arrays allocated (the reference declares but never allocates them)."""
    import torch
    z3 = lambda: torch.zeros((n_bodies, 3, 3), dtype=torch.float64, device=device)
    z1 = lambda: torch.zeros((n_bodies, 3), dtype=torch.float64, device=device)
    return AffineBodyStates(A=z3(), p=z1(), Ak=z3(), pk=z1(), Adot=z3(), pdot=z1(),
                            A0=z3(), p0=z1(),
                            mass=torch.zeros(n_bodies, dtype=torch.float64, device=device),
                            I0=torch.zeros(n_bodies, dtype=torch.float64, device=device))


class Scene:
    """JSON scene -> list of :class:`AffineMesh` (simulator/scene.py:52-60)."""

    def __init__(self, member_type=AffineMesh, scene_config_file: str | None = None,
                 objects: list | None = None, density: float = DEFAULT_DENSITY, mesh_map: dict | None = None):
        self.kinetic_objects = []
        if objects is None:
            with open(scene_config_file) as f:
                objects = json.load(f)["objects"]
        for obj in objects:
            self.kinetic_objects.append(obj if isinstance(obj, AffineMesh)
                                        else member_type(obj, density=density, mesh_map=mesh_map))
