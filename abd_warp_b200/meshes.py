"""Procedural triangle meshes and their rigid mass properties.

The reference loads meshes from bgeo/USD/OBJ files (simulator/mesh.py:37-55) and
derives the edge list with ``igl.edges`` (affine_body.py:71).  Neither the readers'
dependencies nor the ``assets/`` folder exist here, so meshes are generated
procedurally.  The edge list is defined by :func:`unique_edges` (sorted, unique,
undirected), and every consumer (the CUDA path, the oracle and the tests) uses the
same arrays, so primitive indices agree everywhere.
"""
from __future__ import annotations

from functools import lru_cache

import numpy as np


def unique_edges(F: np.ndarray) -> np.ndarray:
    """Unique undirected edges of a triangle list, as sorted (min, max) pairs in
    lexicographic order.  Stands in for ``igl.edges(F)`` (affine_body.py:71)."""
    F = np.asarray(F, dtype=np.int64)
    e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]], axis=0)
    e = np.sort(e, axis=1)
    e = np.unique(e, axis=0)
    return e.astype(np.int32)


def box_mesh(sx: float, sy: float, sz: float):
    """Axis-aligned box centred at the origin: 8 vertices, 12 outward triangles."""
    hx, hy, hz = 0.5 * sx, 0.5 * sy, 0.5 * sz
    V = np.array([
        [-hx, -hy, -hz], [hx, -hy, -hz], [hx, hy, -hz], [-hx, hy, -hz],
        [-hx, -hy, hz], [hx, -hy, hz], [hx, hy, hz], [-hx, hy, hz],
    ], dtype=np.float64)
    F = np.array([
        [0, 2, 1], [0, 3, 2],      # -z
        [4, 5, 6], [4, 6, 7],      # +z
        [0, 1, 5], [0, 5, 4],      # -y
        [3, 7, 6], [3, 6, 2],      # +y
        [0, 4, 7], [0, 7, 3],      # -x
        [1, 2, 6], [1, 6, 5],      # +x
    ], dtype=np.int32)
    return V, F


def cube_mesh(edge: float = 1.0):
    return box_mesh(edge, edge, edge)


def icosphere_mesh(level: int, radius: float = 1.0):
    """Icosahedron subdivided ``level`` times, vertices projected to ``radius``.

    level 2: 162 vertices / 320 triangles / 480 edges; level 3: 642 / 1280 / 1920.
    """
    V, F = _unit_icosphere(level)
    return V * radius, F.copy()


@lru_cache(maxsize=None)
def _unit_icosphere(level: int):
    t = (1.0 + 5.0 ** 0.5) / 2.0
    V = [[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0],
         [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
         [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]]
    F = [[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
         [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
         [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
         [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]]
    V = [list(np.asarray(v, dtype=np.float64) / np.linalg.norm(v)) for v in V]
    for _ in range(level):
        cache = {}

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                m = (np.asarray(V[a]) + np.asarray(V[b])) * 0.5
                m = m / np.linalg.norm(m)
                cache[key] = len(V)
                V.append(list(m))
            return cache[key]

        F2 = []
        for a, b, c in F:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            F2 += [[a, ab, ca], [b, bc, ab], [c, ca, bc], [ab, bc, ca]]
        F = F2
    V = np.asarray(V, dtype=np.float64)
    V.setflags(write=False)
    return V, np.asarray(F, dtype=np.int32)


def mass_properties(V: np.ndarray, F: np.ndarray, density: float):
    """Mass, centre of mass and the isotropic second moment of a closed mesh.

    Returns ``(mass, com, I0)`` with ``I0 = density * trace(int r r^T dV) / 3`` about the
    centre of mass: the per-axis second moment that the affine-body mass matrix
    ``diag(m, I0, I0, I0)`` uses (orthogonal_energy.py:34-41, with per-body values in
    place of the reference's global constants, const_params.py:38-39).
    """
    a = V[F[:, 0]]
    b = V[F[:, 1]]
    c = V[F[:, 2]]
    det = np.einsum("ij,ij->i", a, np.cross(b, c))      # 6 x signed tet volume
    vol = det.sum() / 6.0
    com = (det[:, None] * (a + b + c)).sum(axis=0) / (24.0 * vol)
    s = a + b + c
    # int x x^T over tet (0,a,b,c) = det/120 (aa^T + bb^T + cc^T + ss^T)
    cov = (np.einsum("i,ij,ik->jk", det, a, a) + np.einsum("i,ij,ik->jk", det, b, b)
           + np.einsum("i,ij,ik->jk", det, c, c) + np.einsum("i,ij,ik->jk", det, s, s)) / 120.0
    cov_c = cov - vol * np.outer(com, com)
    mass = density * vol
    I0 = density * np.trace(cov_c) / 3.0
    return float(mass), com, float(I0)
