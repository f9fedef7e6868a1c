"""NumPy restatement of the full IPC contact model: closest-feature classification of a
point-triangle (PT) or edge-edge (EE) pair, the log barrier on the squared distance of the
classified feature pair, and the edge-edge mollifier.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, never by the product path.  It checks the
host build of the CUDA model (``abd_warp_b200/csrc/abd_ipc_full.cuh``) with arithmetic of its
own: barycentric coordinates from sub-triangle areas instead of normal equations, distances
from explicit closest points, derivatives by central differences.

The reference has no such model.  Its contact energy and CCD evaluate only the interior
cases (point over the triangle's interior, crossing edge interiors: ipcsk/energy.py:20-22,
46-48; ccd.py:44-54), so a contact at an edge or a vertex is missed.  The model restated
here follows Li et al., "Incremental Potential Contact" (SIGGRAPH 2020).  Parity against the
reference is pinned only where the reference defines a value: on interior, non-parallel
contacts the energy and gradient must equal the reference model's (``oracle.contact_gh``).
The other feature pairs are pinned by brute-force sampling of the closest points and by
central differences.
"""
from __future__ import annotations

import numpy as np

# closest-feature types (triangle edges E0 = t0t1, E1 = t1t2, E2 = t2t0)
PT_P_T, PT_P_E0, PT_P_E1, PT_P_E2, PT_P_V0, PT_P_V1, PT_P_V2 = range(7)
EE_EA_EB, EE_EA0_EB, EE_EA1_EB, EE_EA_EB0, EE_EA_EB1, EE_EA0_EB0, EE_EA0_EB1, EE_EA1_EB0, EE_EA1_EB1 = range(9)


def _seg_closest(p, a, b):
    """Clamped parameter s of the point of segment [a, b] nearest p, and the squared distance."""
    e = b - a
    ee = float(e @ e)
    s = 0.0 if ee == 0.0 else float(np.clip((p - a) @ e / ee, 0.0, 1.0))
    c = a + s * e
    return s, float((p - c) @ (p - c))


def pt_closest(p, t0, t1, t2):
    """(type, squared distance, closest point of the triangle) of a point and a triangle."""
    n = np.cross(t1 - t0, t2 - t0)
    nn = float(n @ n)
    if nn > 0.0:
        q = p - ((p - t0) @ n) / nn * n  # projection onto the plane
        u = np.cross(t1 - q, t2 - q) @ n / nn
        v = np.cross(t2 - q, t0 - q) @ n / nn
        w = np.cross(t0 - q, t1 - q) @ n / nn
        if u >= 0.0 and v >= 0.0 and w >= 0.0:
            return PT_P_T, float(((p - t0) @ n) ** 2 / nn), q
    tv = (t0, t1, t2)
    best = None
    for k in range(3):
        s, d2 = _seg_closest(p, tv[k], tv[(k + 1) % 3])
        if best is None or d2 < best[2]:
            best = (k, s, d2)
    k, s, d2 = best
    a, b = tv[k], tv[(k + 1) % 3]
    q = a + s * (b - a)
    if s <= 0.0:
        return PT_P_V0 + k, d2, a
    if s >= 1.0:
        return PT_P_V0 + (k + 1) % 3, d2, b
    return PT_P_E0 + k, d2, q


def ee_closest(a0, a1, b0, b1):
    """(type, squared distance, closest point of edge a, closest point of edge b)."""
    u, v = a1 - a0, b1 - b0
    M = np.array([[u @ u, -(u @ v)], [u @ v, -(v @ v)]])
    if abs(np.linalg.det(M)) > 0.0:
        s, t = np.linalg.solve(M, np.array([-(u @ (a0 - b0)), -(v @ (a0 - b0))]))
        if 0.0 < s < 1.0 and 0.0 < t < 1.0:
            pa, pb = a0 + s * u, b0 + t * v
            return EE_EA_EB, float((pa - pb) @ (pa - pb)), pa, pb
    cand = [_seg_closest(a0, b0, b1), _seg_closest(a1, b0, b1), _seg_closest(b0, a0, a1), _seg_closest(b1, a0, a1)]
    k = min(range(4), key=lambda m: (cand[m][1], m))
    s, d2 = cand[k]
    pa = (a0, a1, a0 + s * u, a0 + s * u)[k]
    pb = (b0 + s * v, b0 + s * v, b0, b1)[k]
    if s <= 0.0:
        return (EE_EA0_EB0, EE_EA1_EB0, EE_EA0_EB0, EE_EA0_EB1)[k], d2, pa, pb
    if s >= 1.0:
        return (EE_EA0_EB1, EE_EA1_EB1, EE_EA1_EB0, EE_EA1_EB1)[k], d2, pa, pb
    return (EE_EA0_EB, EE_EA1_EB, EE_EA_EB0, EE_EA_EB1)[k], d2, pa, pb


def classify(kind, x12):
    """(type, squared distance) of a pair: kind 0 PT (point, triangle), 1 EE (edge a, edge b)."""
    x = np.asarray(x12, dtype=np.float64).reshape(4, 3)
    r = pt_closest(*x) if kind == 0 else ee_closest(*x)
    return r[0], r[1]


def separation(kind, x12):
    """The closest points of the two groups (point or edge a; triangle or edge b)."""
    x = np.asarray(x12, dtype=np.float64).reshape(4, 3)
    if kind == 0:
        return x[0], pt_closest(*x)[2]
    r = ee_closest(*x)
    return r[2], r[3]


def _d2_point_line(p, a, b):
    c = np.cross(a - p, b - p)
    e = b - a
    return (c @ c) / (e @ e)


def typed_d2(kind, type_, x12):
    """Squared distance of the given feature pair (the type's formula, no classification)."""
    x = np.asarray(x12, dtype=np.float64).reshape(4, 3)
    if kind == 0:
        p, t0, t1, t2 = x
        if type_ == PT_P_T:
            n = np.cross(t1 - t0, t2 - t0)
            return ((p - t0) @ n) ** 2 / (n @ n)
        if type_ <= PT_P_E2:
            a, b = ((t0, t1), (t1, t2), (t2, t0))[type_ - PT_P_E0]
            return _d2_point_line(p, a, b)
        q = (t0, t1, t2)[type_ - PT_P_V0]
        return (p - q) @ (p - q)
    a0, a1, b0, b1 = x
    if type_ == EE_EA_EB:
        n = np.cross(a1 - a0, b1 - b0)
        return ((b0 - a0) @ n) ** 2 / (n @ n)
    pe = {EE_EA0_EB: (a0, b0, b1), EE_EA1_EB: (a1, b0, b1), EE_EA_EB0: (b0, a0, a1), EE_EA_EB1: (b1, a0, a1)}
    if type_ in pe:
        return _d2_point_line(*pe[type_])
    pp = {EE_EA0_EB0: (a0, b0), EE_EA0_EB1: (a0, b1), EE_EA1_EB0: (a1, b0), EE_EA1_EB1: (a1, b1)}[type_]
    return (pp[0] - pp[1]) @ (pp[0] - pp[1])


def eps_x(r12):
    r = np.asarray(r12, dtype=np.float64).reshape(4, 3)
    return 1e-3 * float((r[1] - r[0]) @ (r[1] - r[0])) * float((r[3] - r[2]) @ (r[3] - r[2]))


def mollifier(x12, ex):
    x = np.asarray(x12, dtype=np.float64).reshape(4, 3)
    n = np.cross(x[1] - x[0], x[3] - x[2])
    c = float(n @ n)
    if c >= ex:
        return 1.0
    q = c / ex
    return (2.0 - q) * q


def barrier(d, dh, kappa):
    if d >= dh:
        return 0.0
    s = d / dh
    return -kappa * (s - 1.0) ** 2 * np.log(s)


def energy(kind, x12, r12, dh, kappa, type_=None):
    """Contact energy; with ``type_`` the feature pair is fixed (no classification)."""
    if type_ is None:
        type_, _ = classify(kind, x12)
    d2 = typed_d2(kind, type_, x12)
    if not d2 < dh:
        return 0.0
    e = barrier(d2, dh, kappa)
    return e * mollifier(x12, eps_x(r12)) if kind == 1 else e


def fd_gradient_hessian(kind, x12, r12, dh, kappa, h, type_):
    """Central differences of ``energy`` at a fixed feature pair: gradient (12), Hessian (12x12)."""
    x = np.asarray(x12, dtype=np.float64).ravel()
    f = lambda y: energy(kind, y, r12, dh, kappa, type_)
    g = np.zeros(12)
    H = np.zeros((12, 12))
    I = np.eye(12) * h
    for i in range(12):
        g[i] = (f(x + I[i]) - f(x - I[i])) / (2 * h)
        for j in range(i, 12):
            H[i, j] = H[j, i] = (f(x + I[i] + I[j]) - f(x + I[i] - I[j]) - f(x - I[i] + I[j]) + f(x - I[i] - I[j])) / (
                4 * h * h)
    return g, H


def project_psd(H):
    w, V = np.linalg.eigh(0.5 * (H + H.T))
    return (V * np.maximum(w, 0.0)) @ V.T


def to_affine(gx, Hx, r12, nI):
    """Point-coordinate gradient / Hessian to the two bodies' affine DOFs [p, A rows]:
    x_a = p_a + sum_k r_k A_ka, so d x / d q = [I3, r_0 I3, r_1 I3, r_2 I3] per point."""
    r = np.asarray(r12, dtype=np.float64).reshape(4, 3)
    J = np.zeros((12, 24))
    for v in range(4):
        off = 0 if v < nI else 12
        w = np.concatenate([[1.0], r[v]])
        for m in range(4):
            J[3 * v:3 * v + 3, off + 3 * m:off + 3 * m + 3] = w[m] * np.eye(3)
    g24 = J.T @ np.asarray(gx).ravel()
    H24 = J.T @ np.asarray(Hx).reshape(12, 12) @ J
    return g24, H24[:12, :12], H24[12:, 12:], H24[:12, 12:]


def sample_d2(kind, x12, n=400):
    """Brute-force minimum squared distance over a grid of the two primitives' parameters."""
    x = np.asarray(x12, dtype=np.float64).reshape(4, 3)
    s = np.linspace(0.0, 1.0, n)
    if kind == 0:
        p, t0, t1, t2 = x
        B, G = np.meshgrid(s, s, indexing="ij")
        keep = B + G <= 1.0
        pts = t0 + B[keep, None] * (t1 - t0) + G[keep, None] * (t2 - t0)
        d = pts - p
    else:
        a0, a1, b0, b1 = x
        S, T = np.meshgrid(s, s, indexing="ij")
        d = (a0 + S.ravel()[:, None] * (a1 - a0)) - (b0 + T.ravel()[:, None] * (b1 - b0))
    return float(np.min(np.einsum("ij,ij->i", d, d)))


# ---------------------------------------------------------------------------------------
# lagged friction (Li et al. 2020, section 5)
# ---------------------------------------------------------------------------------------
def closest_weights(kind, x12):
    """Weights w (4) with sum_v w_v x_v = c_a - c_b, the closest points of the pair's two groups
    (+ on the first group, - on the second), from this module's own closest points."""
    x = np.asarray(x12, dtype=np.float64).reshape(4, 3)
    ca, cb = separation(kind, x)
    w = np.zeros(4)
    if kind == 0:
        w[0] = 1.0
        t0, t1, t2 = x[1:]
        # barycentric coordinates of cb in the triangle (least squares on its plane)
        M = np.stack([t1 - t0, t2 - t0], axis=1)
        s, t = np.linalg.lstsq(M, cb - t0, rcond=None)[0]
        w[1:] = -np.array([1.0 - s - t, s, t])
        return w
    a0, a1, b0, b1 = x
    s = float(np.clip(np.linalg.lstsq((a1 - a0)[:, None], ca - a0, rcond=None)[0][0], 0.0, 1.0))
    t = float(np.clip(np.linalg.lstsq((b1 - b0)[:, None], cb - b0, rcond=None)[0][0], 0.0, 1.0))
    return np.array([1.0 - s, s, -(1.0 - t), -t])


def friction_f0(y, eps):
    return y if y >= eps else -y ** 3 / (3 * eps * eps) + y * y / eps + eps / 3.0


def friction_potential(w, P, lam, x12, xt12, mu, eps):
    """D(x) = mu lambda f0(|P^T sum_v w_v (x_v - xt_v)|)."""
    d = np.asarray(w) @ (np.asarray(x12).reshape(4, 3) - np.asarray(xt12).reshape(4, 3))
    u = np.asarray(P).reshape(3, 2).T @ d
    return mu * lam * friction_f0(float(np.linalg.norm(u)), eps)


def normal_force(kind, x12, r12, dh, kappa, h=1e-7):
    """lambda = -dE/dd at the pair's distance, E = m b(d^2) (central difference in d)."""
    _, d2 = classify(kind, x12)
    d = np.sqrt(d2)
    m = mollifier(x12, eps_x(r12)) if kind == 1 else 1.0
    return -m * (barrier((d + h) ** 2, dh, kappa) - barrier((d - h) ** 2, dh, kappa)) / (2 * h)
