"""Seeded synthetic scenes for the five benchmark configurations (configuration 3, the
batched workload, is a list of scenes: ``config3``).

The reference publishes no benchmark scenes and its assets are absent, so every scene
is generated procedurally with ``numpy.random.default_rng(seed)`` (seed = config index
unless given).  Bodies are returned as :class:`AffineMesh` objects; the ground, where
present, is a fixed box body ``20 x 0.2 x 20`` whose top face is at ``y = 0``, placed
first (body 0).
"""
from __future__ import annotations

import numpy as np

from .affine_body import AffineMesh
from .params import SimParams


def random_rotation(rng) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def _body(spec, p, R=None, v=None, fixed=False):
    """``R`` maps rest to world (x = R r + p); the DOF matrix is ``A = R^T``."""
    obj = {"file": spec, "p": list(map(float, p))}
    if R is not None:
        obj["A"] = R.T.tolist()
    if v is not None:
        obj["pdot"] = list(map(float, v))
    if fixed:
        obj["fixed"] = True
    return AffineMesh(obj)


def ground_box():
    return _body("box:20,0.2,20", (0.0, -0.1, 0.0), fixed=True)


def config0(seed: int = 0):
    """Two unit cubes: A fixed at the origin, B at +1.2 y with a random rotation
    (rejection-sampled until its lowest vertex is above y = 0.5 + dhat) and velocity
    (0, -2, 0).  200 steps, no ground."""
    prm = SimParams()
    rng = np.random.default_rng(seed)
    a = _body("cube:1.0", (0, 0, 0), fixed=True)
    while True:
        R = random_rotation(rng)
        b = _body("cube:1.0", (0, 1.2, 0), R=R, v=(0, -2, 0))
        if b.vertices_world()[:, 1].min() > 0.5 + prm.dhat:
            break
    return [a, b], prm, 200


def _grid_jitter(rng, centers, radius, jitter, gap):
    while True:
        c = centers + rng.uniform(-jitter, jitter, size=centers.shape)
        d = np.linalg.norm(c[:, None, :] - c[None, :, :], axis=-1)
        np.fill_diagonal(d, np.inf)
        if d.min() > 2 * radius + gap:
            return c


def config1(seed: int = 1):
    """64 level-2 icospheres (r = 0.25) on a 4x4x4 grid (spacing 0.6, jitter
    U(-0.05, 0.05)) above the ground box, random rotations, velocities N(0, 0.5^2).
    300 steps."""
    prm = SimParams()
    rng = np.random.default_rng(seed)
    r, sp, jit = 0.25, 0.6, 0.05
    y0 = r + 2 * prm.dhat + jit
    cs = np.array([[(i - 1.5) * sp, y0 + j * sp, (k - 1.5) * sp]
                   for j in range(4) for i in range(4) for k in range(4)])
    cs = _grid_jitter(rng, cs, r, jit, 2 * prm.dhat)
    bodies = [ground_box()]
    for c in cs:
        bodies.append(_body(f"icosphere:2:{r}", c, R=random_rotation(rng),
                            v=rng.normal(0.0, 0.5, size=3)))
    return bodies, prm, 300


def config2(seed: int = 2):
    """1024-body pile: 512 cubes (edge U(0.15, 0.4)) and 512 level-3 icospheres
    (r U(0.1, 0.3)) on a 16x4x16 grid with spacing 0.8, random rotations, velocities
    N(0, 1), dropping onto the ground box.  300 steps."""
    prm = SimParams()
    rng = np.random.default_rng(seed)
    sp = 0.8
    y0 = 0.35 + 2 * prm.dhat + 0.01
    kinds = rng.permutation(np.array([0] * 512 + [1] * 512))
    bodies = [ground_box()]
    idx = 0
    for j in range(4):
        for i in range(16):
            for k in range(16):
                c = ((i - 7.5) * sp, y0 + j * sp, (k - 7.5) * sp)
                R = random_rotation(rng)
                v = rng.normal(0.0, 1.0, size=3)
                if kinds[idx] == 0:
                    spec = f"cube:{rng.uniform(0.15, 0.4)}"
                else:
                    spec = f"icosphere:3:{rng.uniform(0.1, 0.3)}"
                bodies.append(_body(spec, c, R=R, v=v))
                idx += 1
    return bodies, prm, 300


def config4(seed: int = 4):
    """16 level-2 icospheres (r = 0.2) resting on the ground box at random in-plane
    positions in a 4 x 4 m region, velocities N(0, 1) in x and z.  100 steps."""
    prm = SimParams()
    rng = np.random.default_rng(seed)
    r = 0.2
    while True:
        xz = rng.uniform(-2.0 + r, 2.0 - r, size=(16, 2))
        d = np.linalg.norm(xz[:, None] - xz[None], axis=-1)
        np.fill_diagonal(d, np.inf)
        if d.min() > 2 * r + 4 * prm.dhat:
            break
    bodies = [ground_box()]
    for (x, z) in xz:
        v = rng.normal(0.0, 1.0, size=3)
        v[1] = 0.0
        bodies.append(_body(f"icosphere:2:{r}", (x, r + 2 * prm.dhat, z),
                            R=random_rotation(rng), v=v))
    return bodies, prm, 100


def config3(seed: int = 3, n_scenes: int = 512):
    """The batched workload: ``n_scenes`` independent scenes, each with U{2..48} bodies over
    its own ground box.  Bodies are cubes (edge U(0.15, 0.4)) or level-2 icospheres
    (r U(0.1, 0.3)), half and half at random, with random rotations and velocities
    N(0, 0.5^2).  They are placed without overlap (rejection on bounding spheres with a gap of
    2 dhat) in a 3 x 3 x 3 m box on the ground.  100 steps.  Returns
    ``(list of body lists, prm, steps)``; each body list is one scene, ground box first."""
    prm = SimParams()
    rng = np.random.default_rng(seed)
    gap = 2 * prm.dhat
    out = []
    for _ in range(n_scenes):
        nb = int(rng.integers(2, 49))
        bodies = [ground_box()]
        placed = []
        while len(placed) < nb:
            if rng.random() < 0.5:
                e = float(rng.uniform(0.15, 0.4))
                spec, rad = f"cube:{e}", 0.5 * np.sqrt(3.0) * e
            else:
                r = float(rng.uniform(0.1, 0.3))
                spec, rad = f"icosphere:2:{r}", r
            c = rng.uniform([-1.5 + rad, rad + gap, -1.5 + rad], [1.5 - rad, 3.0 - rad, 1.5 - rad])
            if all(np.linalg.norm(c - c2) > rad + r2 + gap for c2, r2 in placed):
                placed.append((c, rad))
                bodies.append(_body(spec, c, R=random_rotation(rng), v=rng.normal(0.0, 0.5, size=3)))
        out.append(bodies)
    return out, prm, 100


CONFIGS = {0: config0, 1: config1, 2: config2, 4: config4}


def make_config(index: int, seed: int | None = None):
    fn = CONFIGS[index]
    return fn() if seed is None else fn(seed)


def small_pile(n_side: int = 2, layers: int = 2, seed: int = 7, level: int = 1,
               radius: float = 0.2, plane: bool = False):
    """A small mixed pile for fast parity tests: cubes and icospheres on a grid above
    the ground box, or, with plane, above the vertex-ground plane y = 0 (no ground body)."""
    prm = SimParams()
    rng = np.random.default_rng(seed)
    bodies = [] if plane else [ground_box()]
    if plane:
        prm.ground_enabled = True
        prm.ground = 0.0
    sp = 2.2 * radius + 0.05
    y0 = radius * 1.8 + 2 * prm.dhat
    t = 0
    for j in range(layers):
        for i in range(n_side):
            for k in range(n_side):
                c = ((i - (n_side - 1) / 2) * sp, y0 + j * sp, (k - (n_side - 1) / 2) * sp)
                spec = f"cube:{1.4 * radius}" if t % 2 == 0 else f"icosphere:{level}:{radius}"
                bodies.append(_body(spec, c, R=random_rotation(rng),
                                    v=rng.normal(0.0, 0.5, size=3)))
                t += 1
    return bodies, prm


def flatten_bodies(bodies):
    """Concatenate per-body meshes into the flat arrays both the CUDA library and the
    oracle take: per-body vertex / triangle / edge offsets, rest positions, triangles and
    edges with GLOBAL vertex indices, mass, I0, fixed flags and the initial states."""
    n = len(bodies)
    nv = np.array([b.V.shape[0] for b in bodies], dtype=np.int64)
    nt = np.array([b.F.shape[0] for b in bodies], dtype=np.int64)
    ne = np.array([b.edges.shape[0] for b in bodies], dtype=np.int64)
    voff = np.concatenate([[0], np.cumsum(nv)]).astype(np.int32)
    toff = np.concatenate([[0], np.cumsum(nt)]).astype(np.int32)
    eoff = np.concatenate([[0], np.cumsum(ne)]).astype(np.int32)
    x0 = np.concatenate([b.V for b in bodies], axis=0).astype(np.float64)
    tris = np.concatenate([b.F + voff[i] for i, b in enumerate(bodies)], axis=0).astype(np.int32)
    edges = np.concatenate([b.edges + voff[i] for i, b in enumerate(bodies)], axis=0).astype(np.int32)
    return {
        "n": n, "voff": voff, "toff": toff, "eoff": eoff,
        "x0": np.ascontiguousarray(x0), "tris": np.ascontiguousarray(tris),
        "edges": np.ascontiguousarray(edges),
        "mass": np.array([b.mass for b in bodies], dtype=np.float64),
        "I0": np.array([b.I0 for b in bodies], dtype=np.float64),
        "fixed": np.array([1 if b.fixed else 0 for b in bodies], dtype=np.int32),
        "A": np.stack([b.A for b in bodies]).astype(np.float64),
        "p": np.stack([b.p for b in bodies]).astype(np.float64),
        "Adot": np.stack([b.Adot for b in bodies]).astype(np.float64),
        "pdot": np.stack([b.pdot for b in bodies]).astype(np.float64),
    }
