"""NumPy restatement of the reference's per-primitive contact math, barrier, CCD cubic and
inertia terms.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()`` and the
golden-fixture script, never by the product path.  It is the second, independent CPU
restatement that cross-checks the C++ oracle (oracle/abd_oracle.cpp), and it follows the
reference line by line, including its matrix formulation (``np.kron`` Jacobians,
``Q diag(lambda) Q^-1`` reconstruction).

Parity pins: the reference cannot be imported here (Warp and the ``abdtk`` module are
absent), so this module is pinned by the reference's own known-answer checks:
the 4-point fixture of abd/hl_entry.py:8-13 with the eigensystem reconstruction identities
(hl_entry.py:115-147), the distance identity (psd/hl.py:253-265), constructed-root cubics
(cubic_roots.py:225-269) and the inside-triangle negatives (test_distance.py:35-81).
"""
from __future__ import annotations

import math

import numpy as np


# ---------------------------------------------------------------------------------------
# distance geometry: psd/vf.py, psd/ee.py, psd/hl.py
# ---------------------------------------------------------------------------------------
def _solve22(e0, e1, e2):
    """[beta, gamma] = inverse([[e0.e0, e0.e1],[e0.e1, e1.e1]]) @ [e0.e2, e1.e2]
    (psd/vf.py:11-18 and psd/ee.py:124-130)."""
    a = np.dot(e0, e0)
    b = np.dot(e0, e1)
    d = np.dot(e1, e1)
    det = a * d - b * b
    inv = np.array([[d, -b], [-b, a]]) * (1.0 / det)
    rhs = np.array([np.dot(e0, e2), np.dot(e1, e2)])
    bg = inv @ rhs
    return bg[0], bg[1]


def C_vf(x0, x1, x2, x3):
    """Point-triangle c-coordinates (psd/vf.py:22-41)."""
    e0 = x1 - x2
    e1 = x3 - x2
    e2 = x0 - x2
    alpha = np.dot(e0, e1) / np.dot(e0, e0)
    e1perp = e1 - alpha * e0
    beta, gamma = _solve22(e0, e1, e2)
    e2perp = e2 - beta * e0 - gamma * e1
    return e0, e1perp, e2perp


def C_ee(x0, x1, x2, x3):
    """Edge-edge c-coordinates (psd/ee.py:5-31)."""
    e0 = x1 - x0
    e1 = x3 - x2
    e2 = x2 - x0
    alpha = np.dot(e0, e1) / np.dot(e0, e0)
    e1perp = e1 - alpha * e0
    beta, gamma = _solve22(e0, e1, e2)
    e2perp = e2 - beta * e0 - gamma * e1
    return e0, e1perp, e2perp


def beta_gamma_pt(x0, x1, x2, x3):
    return _solve22(x1 - x2, x3 - x2, x0 - x2)


def beta_gamma_ee(x0, x1, x2, x3):
    return _solve22(x1 - x0, x3 - x2, x2 - x0)


def verify_root_pt(x0, x1, x2, x3):
    """Interior test of the point projection (ccd.py:44-48)."""
    b, g = beta_gamma_pt(x0, x1, x2, x3)
    return (0.0 < b < 1.0) and (0.0 < g < 1.0) and (0.0 < b + g < 1.0)


def verify_root_ee(x0, x1, x2, x3):
    """Interior test of the closest points of two edges (ccd.py:50-54)."""
    b, g = beta_gamma_ee(x0, x1, x2, x3)
    return (0.0 < b < 1.0) and (0.0 < -g < 1.0)


def dcvfdx_s(x0, x1, x2, x3):
    """3x4 dc/dx of the point-triangle map with alpha, beta, gamma frozen (psd/vf.py:43-71)."""
    e0 = x1 - x2
    e1 = x3 - x2
    alpha = np.dot(e0, e1) / np.dot(e0, e0)
    beta, gamma = beta_gamma_pt(x0, x1, x2, x3)
    D = np.zeros((3, 4))
    D[0, 1] = 1.0
    D[0, 2] = -1.0
    D[1, 1] = -alpha
    D[1, 2] = alpha - 1.0
    D[1, 3] = 1.0
    D[2, 0] = 1.0
    D[2, 1] = -beta
    D[2, 2] = beta + gamma - 1.0
    D[2, 3] = -gamma
    return D


def dceedx_s(x0, x1, x2, x3):
    """3x4 dc/dx of the edge-edge map (psd/ee.py:134-163)."""
    e0 = x1 - x0
    e1 = x3 - x2
    al = np.dot(e0, e1) / np.dot(e0, e0)
    bet, gam = beta_gamma_ee(x0, x1, x2, x3)
    return np.array([[-1.0, 1.0, 0.0, 0.0],
                     [al, -al, -1.0, 1.0],
                     [bet - 1.0, -bet, gam + 1.0, -gam]])


def signed_distance(e0p, e1p, e2p):
    """psd/hl.py:15-17"""
    n = np.cross(e0p, e1p)
    return np.dot(e2p, n) / np.linalg.norm(n)


def gl(l, e2o):
    """Gradient of the signed distance in c-space (psd/hl.py:36-39)."""
    z = np.zeros(3)
    return z, z, e2o * l / np.dot(e2o, e2o)


def Hl(e0o, e1o, e2o):
    """Hessian blocks of the signed distance in c-space (psd/hl.py:19-34)."""
    l = signed_distance(e0o, e1o, e2o)
    l02 = -l * np.outer(e2o, e0o) / (np.dot(e2o, e2o) * np.dot(e0o, e0o))
    l12 = -l * np.outer(e2o, e1o) / (np.dot(e2o, e2o) * np.dot(e1o, e1o))
    e0u = e0o / np.linalg.norm(e0o)
    e1u = e1o / np.linalg.norm(e1o)
    block = np.eye(3) - np.outer(e0u, e0u) - np.outer(e1u, e1u)
    l00 = -l * block / np.dot(e0o, e0o)
    l11 = -l * block / np.dot(e1o, e1o)
    return l00, l11, l02, l12


def d2Psi(e0p, e1p, e2p):
    """9x9 Hessian of l^2 in c-space, 2 l Hl + 2 gl gl^T (psd/hl.py:57-70)."""
    l = signed_distance(e0p, e1p, e2p)
    H00, H11, H02, H12 = Hl(e0p, e1p, e2p)
    g0, g1, g2 = gl(l, e2p)
    G = [g0, g1, g2]
    Hb = [[2 * l * H00, None, 2 * l * H02], [None, 2 * l * H11, 2 * l * H12],
          [2 * l * H02.T, 2 * l * H12.T, None]]
    out = np.zeros((9, 9))
    for i in range(3):
        for j in range(3):
            blk = 2.0 * np.outer(G[i], G[j])
            if Hb[i][j] is not None:
                blk = blk + Hb[i][j]
            out[3 * i:3 * i + 3, 3 * j:3 * j + 3] = blk
    return out


def eig_Hl(e0p, e1p, e2p):
    """Analytic eigensystem of 2 l Hl (psd/hl.py:155-195) plus the fifth pair
    (2 l gl, lambda = 2) added by the contact terms (pt_ipc.py:275-280).

    Returns ``(Q, lam)``: Q is 9x5 with eigenvectors as columns, lam has 5 entries
    (unclamped)."""
    l = signed_distance(e0p, e1p, e2p)
    e0pn = np.dot(e0p, e0p)
    e1pn = np.dot(e1p, e1p)
    e2pn = np.dot(e2p, e2p)
    f12 = math.sqrt(1.0 + 4.0 * (e1pn / e2pn))
    f02 = math.sqrt(1.0 + 4.0 * (e0pn / e2pn))
    lam0 = -l / (2.0 * e1pn) * (1.0 + f12)
    lam1 = -l / (2.0 * e1pn) * (1.0 - f12)
    lam2 = -l / (2.0 * e0pn) * (1.0 + f02)
    lam3 = -l / (2.0 * e0pn) * (1.0 - f02)
    om = [lam / (lam - l / e2pn) for lam in (lam0, lam1, lam2, lam3)]
    z = np.zeros(3)
    q = [np.concatenate([z, e2p, om[0] * e1p]), np.concatenate([z, e2p, om[1] * e1p]),
         np.concatenate([e2p, z, om[2] * e0p]), np.concatenate([e2p, z, om[3] * e0p])]
    _, _, g2 = gl(l, e2p)
    q.append(np.concatenate([z, z, g2 * 2.0 * l]))
    lam = np.array([lam0 * 2.0 * l, lam1 * 2.0 * l, lam2 * 2.0 * l, lam3 * 2.0 * l, 2.0])
    return np.stack(q, axis=1), lam


def QLQinv(Q, lam):
    """Q diag(lam) Q^-1 with Q^-1 = diag(1/|q_i|^2) Q^T (pt_ipc.py:225-231)."""
    QTQ = Q.T @ Q
    diag_inv = np.diag(np.array([1.0 / QTQ[i, i] for i in range(Q.shape[1])]))
    return Q @ np.diag(lam) @ (diag_inv @ Q.T)


# ---------------------------------------------------------------------------------------
# barrier: ipcsk/barrier.py
# ---------------------------------------------------------------------------------------
def barrier(d, d2hat, kappa):
    if d < d2hat:
        s = d / d2hat
        return kappa * -((s - 1.0) ** 2.0) * math.log(s)
    return 0.0


def barrier_derivative(d, d2hat, kappa):
    if d < d2hat:
        return kappa * (d2hat - d) * (2.0 * math.log(d / d2hat) + (d - d2hat) / d) / (d2hat * d2hat)
    return 0.0


def barrier_derivative2(d, d2hat, kappa):
    if d < d2hat:
        return -kappa * (2.0 * math.log(d / d2hat) + (d - d2hat) / d
                         + (d - d2hat) * (2.0 / d + d2hat / (d * d))) / (d2hat * d2hat)
    return 0.0


# ---------------------------------------------------------------------------------------
# per-pair gradient / Hessian: ipcsk/pt_ipc.py:111-247, ipcsk/ee_ipc.py:381-475
# ---------------------------------------------------------------------------------------
def _kron3(M):
    return np.kron(M, np.eye(3))


def _project(Q, lam, d2, d2hat, kappa, clamp, contact_psd):
    """c-space Hessian of the barrier.  contact_psd 0: the reference form
    (clamp lam_k if ``clamp``, then B' Hc + B'' q4 q4^T, pt_ipc.py:166); contact_psd 1: the
    eigenvalues of that matrix on the eigenvectors q_k clamped at zero."""
    Bp = barrier_derivative(d2, d2hat, kappa)
    Bpp = barrier_derivative2(d2, d2hat, kappa)
    lam = lam.copy()
    if contact_psd == 1:
        mu = Bp * lam
        mu[4] = Bp * 2.0 + Bpp * np.dot(Q[:, 4], Q[:, 4])
        return QLQinv(Q, np.maximum(mu, 0.0)), Bp, None
    if clamp:
        lam[:4] = np.maximum(lam[:4], 0.0)
    return QLQinv(Q, lam), Bp, Bpp


def pt_term(x, r, d2hat, kappa, contact_psd=1):
    """One point-triangle pair.  ``x``: 4x3 current (point, t0, t1, t2), ``r``: 4x3 rest.

    Returns ``None`` when inactive, else ``(d2, g24, Hi, Hj, Hij)`` in body DOF order
    ``[p, a0, a1, a2]`` x xyz."""
    x0, x1, x2, x3 = x
    valid = verify_root_pt(x0, x1, x2, x3)
    e0p, e1p, e2p = C_vf(x0, x1, x2, x3)
    l = signed_distance(e0p, e1p, e2p)
    d2 = l * l
    if not (d2 < d2hat and valid):
        return None
    Q, lam = eig_Hl(e0p, e1p, e2p)
    D = dcvfdx_s(x0, x1, x2, x3)
    g12 = _kron3(D.T) @ Q[:, 4]                        # extract_g, pt_ipc.py:194-200
    Hc, Bp, Bpp = _project(Q, lam, d2, d2hat, kappa, True, contact_psd)   # pt_ipc.py:266-269
    Hpt = _kron3(D).T @ Hc @ _kron3(D)                 # dcTHldc, pt_ipc.py:233-235
    Hipc = Hpt if Bpp is None else Hpt * Bp + np.outer(g12, g12) * Bpp   # pt_ipc.py:166
    Jp = np.array([1.0, *r[0]])
    Jt = np.array([[1.0, *r[1]], [1.0, *r[2]], [1.0, *r[3]]])
    gp = np.kron(Jp.reshape(1, 4).T, np.eye(3)) @ g12[:3]
    gt = np.kron(Jt.T, np.eye(3)) @ g12[3:]
    g = np.concatenate([gp, gt]) * Bp
    Jpk = np.kron(Jp.reshape(1, 4), np.eye(3))
    Jtk = np.kron(Jt, np.eye(3))
    Hi = Jpk.T @ Hipc[:3, :3] @ Jpk
    Hj = Jtk.T @ Hipc[3:, 3:] @ Jtk
    Hij = Jpk.T @ Hipc[:3, 3:] @ Jtk
    return d2, g, Hi, Hj, Hij


def ee_term(x, r, d2hat, kappa, psd_ee=False, contact_psd=1):
    """One edge-edge pair.  ``x``: 4x3 current (ei0, ei1, ej0, ej1), ``r``: 4x3 rest."""
    x0, x1, x2, x3 = x
    valid = verify_root_ee(x0, x1, x2, x3)
    e0p, e1p, e2p = C_ee(x0, x1, x2, x3)
    d2 = np.dot(e2p, e2p)
    if not (d2 < d2hat and valid):
        return None
    Q, lam = eig_Hl(e0p, e1p, e2p)
    D = dceedx_s(x0, x1, x2, x3)
    g12 = _kron3(D.T) @ Q[:, 4]
    Hc, Bp, Bpp = _project(Q, lam, d2, d2hat, kappa, psd_ee, contact_psd)  # ee_ipc.py:33-36
    Hee = _kron3(D).T @ Hc @ _kron3(D)
    Hipc = Hee if Bpp is None else Hee * Bp + np.outer(g12, g12) * Bpp   # ee_ipc.py:416
    Jei = np.array([[1.0, *r[0]], [1.0, *r[1]]])
    Jej = np.array([[1.0, *r[2]], [1.0, *r[3]]])
    gi = np.kron(Jei.T, np.eye(3)) @ g12[:6]
    gj = np.kron(Jej.T, np.eye(3)) @ g12[6:]
    g = np.concatenate([gi, gj]) * Bp
    Jik = np.kron(Jei, np.eye(3))
    Jjk = np.kron(Jej, np.eye(3))
    Hi = Jik.T @ Hipc[:6, :6] @ Jik
    Hj = Jjk.T @ Hipc[6:, 6:] @ Jjk
    Hij = Jik.T @ Hipc[:6, 6:] @ Jjk
    return d2, g, Hi, Hj, Hij


def vg_term(x, r, ground, d2hat, kappa):
    """Vertex-ground term (ipcsk/vg_ipc.py:4-34): returns (g12, H12) for the body."""
    d = x[1] - ground
    d2bdb2 = barrier_derivative2(d * d, d2hat, kappa)
    dbdd = barrier_derivative(d * d, d2hat, kappa)
    theta = np.array([1.0, r[0], r[1], r[2]])
    g = np.zeros(12)
    H = np.zeros((12, 12))
    for ii in range(4):
        g[3 * ii + 1] = d * 2.0 * theta[ii] * dbdd
        for jj in range(4):
            H[3 * ii + 1, 3 * jj + 1] = theta[ii] * theta[jj] * d2bdb2 * 4.0 * d * d
    return g, H


def pt_energy(x, d2hat, kappa):
    """ipcsk/energy.py:36-48"""
    x0, x1, x2, x3 = x
    cond = verify_root_pt(x0, x1, x2, x3)
    _, _, e2p = C_vf(x0, x1, x2, x3)
    d2 = np.dot(e2p, e2p)
    return barrier(d2, d2hat, kappa) if cond else 0.0


def ee_energy(x, d2hat, kappa):
    """ipcsk/energy.py:9-22"""
    x0, x1, x2, x3 = x
    cond = verify_root_ee(x0, x1, x2, x3)
    e0p, e1p, e2p = C_ee(x0, x1, x2, x3)
    d = signed_distance(e0p, e1p, e2p)
    return barrier(d * d, d2hat, kappa) if cond else 0.0


# ---------------------------------------------------------------------------------------
# CCD: cubic_roots.py:6-193, ccd.py:56-195
# ---------------------------------------------------------------------------------------
X_ERROR = 1e-10


def evaluate(coef, x):
    return coef[0] + x * (coef[1] + x * (coef[2] + x * coef[3]))


def _multi_sign(a, b):
    return -a if b < 0.0 else a


def _diff_sign(y0, yr):
    return y0 * yr < 0.0


def deflate(coef, root):
    d = [0.0, 0.0, 0.0]
    d[2] = coef[3]
    for i in range(2, 0, -1):
        d[i - 1] = coef[i] + root * d[i]
    return d


def find_closed(coef, deriv, x0, x1, y0, y1):
    xr = (x0 + x1) / 2.0
    yr = evaluate(coef, xr)
    xb0, xb1 = x0, x1
    if x1 - x0 <= X_ERROR * 2.0:
        return xr
    while True:
        if _diff_sign(y0, yr):
            xb1 = xr
        else:
            xb0 = xr
        dy = evaluate(deriv, xr)
        dx = _div(yr, dy)
        xn = xr - dx
        if xn > xb0 and xn < xb1:
            step = abs(xr - xn)
            xr = xn
            if step > X_ERROR:
                yr = evaluate(coef, xr)
            else:
                break
        else:
            xr = (xb0 + xb1) / 2.0
            yr = evaluate(coef, xr)
            if xb0 == xr or xb1 == xr or xb1 - xb0 <= 2.0 * X_ERROR:
                break
    return xr


def quadratic_roots(coef, x0, x1):
    roots = [0.0, 0.0]
    c, b, a = coef[0], coef[1], coef[2]
    delta = b * b - 4.0 * a * c
    ret = 0
    if delta > 0.0:
        d = math.sqrt(delta)
        q = -(b + _multi_sign(d, b)) * 0.5
        rv0 = _div(q, a)
        rv1 = _div(c, q)
        xa, xb = min(rv0, rv1), max(rv0, rv1)
        if x0 <= xa <= x1:
            roots[ret] = xa
            ret += 1
        if x0 <= xb <= x1:
            roots[ret] = xb
            ret += 1
    elif delta < 0.0:
        ret = 0
    else:
        r0 = _div(-0.5 * b, a)
        roots[0] = r0
        if x0 <= r0 <= x1:
            ret = 1
    return ret, roots


def _div(a, b):
    """IEEE division (numpy semantics) without Python's ZeroDivisionError."""
    with np.errstate(all="ignore"):
        return float(np.float64(a) / np.float64(b))


def _fmin(a, b):
    return a if a < b else b


def _fmax(a, b):
    return a if a > b else b


def cubic_roots(coef, x0, x1):
    """Roots of coef[0] + coef[1] x + coef[2] x^2 + coef[3] x^3 on [x0, x1]
    (cubic_roots.py:95-193).  Returns (count, [r0, r1, r2])."""
    roots = [0.0, 0.0, 0.0]
    y0 = evaluate(coef, x0)
    y1 = evaluate(coef, x1)
    a = coef[3] * 3.0
    b_2 = coef[2]
    c = coef[1]
    deriv = [c, 2.0 * b_2, a, 0.0]
    delta_4 = b_2 * b_2 - a * c
    if delta_4 > 0.0:
        d_2 = math.sqrt(delta_4)
        q = -(b_2 + _multi_sign(d_2, b_2))
        rv0 = _div(q, a)
        rv1 = _div(c, q)
        xa, xb = _fmin(rv0, rv1), _fmax(rv0, rv1)
        if _diff_sign(y0, y1):
            if xa >= x1 or xb <= x0 or (xa <= x0 and xb >= x1):
                roots[0] = find_closed(coef, deriv, x0, x1, y0, y1)
                return 1, roots
        else:
            if xa >= x1 or xb <= x0 or (xa <= x0 and xb >= x1):
                return 0, roots
        if xa > x0:
            ya = evaluate(coef, xa)
            if _diff_sign(y0, ya):
                roots[0] = find_closed(coef, deriv, x0, xa, y0, ya)
                if _diff_sign(ya, y1) or (xb < x1 and _diff_sign(ya, evaluate(coef, xb))):
                    dp = deflate(coef, roots[0])
                    r, qr = quadratic_roots(dp, xa, x1)
                    roots[1], roots[2] = qr[0], qr[1]
                    return r + 1, roots
                return 1, roots
            if xb < x1:
                yb = evaluate(coef, xb)
                if _diff_sign(ya, yb):
                    roots[0] = find_closed(coef, deriv, xa, xb, ya, yb)
                    if _diff_sign(yb, y1):
                        dp = deflate(coef, roots[0])
                        r, qr = quadratic_roots(dp, xb, x1)
                        roots[1], roots[2] = qr[0], qr[1]
                        return r + 1, roots
                    return 1, roots
                if _diff_sign(yb, y1):
                    roots[0] = find_closed(coef, deriv, xb, x1, yb, y1)
                    return 1, roots
            elif _diff_sign(ya, y1):
                roots[0] = find_closed(coef, deriv, xa, x1, ya, y1)
                return 1, roots
        else:
            yb = evaluate(coef, xb)
            if _diff_sign(y0, yb):
                roots[0] = find_closed(coef, deriv, x0, xb, y0, yb)
                if _diff_sign(yb, y1):
                    dp = deflate(coef, roots[0])
                    r, qr = quadratic_roots(dp, xb, x1)
                    roots[1], roots[2] = qr[0], qr[1]
                    return r + 1, roots
                return 1, roots
            if _diff_sign(yb, y1):
                roots[0] = find_closed(coef, deriv, xb, x1, yb, y1)
                return 1, roots
        return 0, roots
    if _diff_sign(y0, y1):
        roots[0] = find_closed(coef, deriv, x0, x1, y0, y1)
        return 1, roots
    return 0, roots


def cubic_binomial(a, b):
    """prod_i (b_i + t a_i) as coefficients in t (ccd.py:122-129)."""
    return np.array([b[0] * b[1] * b[2],
                     a[0] * b[1] * b[2] + b[0] * b[1] * a[2] + b[0] * a[1] * b[2],
                     a[0] * a[1] * b[2] + a[0] * b[1] * a[2] + b[0] * a[1] * a[2],
                     a[0] * a[1] * a[2]])


def det_polynomial(a, b):
    """Leibniz expansion of det(b + t a) for 3x3 a, b (ccd.py:82-119)."""
    pos = np.zeros(4)
    neg = np.zeros(4)
    terms_pos = [((0, 0), (1, 1), (2, 2)), ((0, 1), (1, 2), (2, 0)), ((0, 2), (1, 0), (2, 1))]
    terms_neg = [((0, 0), (1, 2), (2, 1)), ((0, 1), (1, 0), (2, 2)), ((0, 2), (1, 1), (2, 0))]
    for t in terms_pos:
        pos = pos + cubic_binomial([a[i] for i in t], [b[i] for i in t])
    for t in terms_neg:
        neg = neg + cubic_binomial([a[i] for i in t], [b[i] for i in t])
    return pos - neg


def _cols(p, q, r):
    """wp.mat33(v0, v1, v2) places the vectors as columns."""
    return np.stack([p, q, r], axis=1)


def coplanarity_cubic(P0, P1):
    """build_and_solve_4_points_coplanar's polynomial (ccd.py:56-79).  ``P0``/``P1``:
    4x3 positions at t=0 / t=1."""
    p0a, p1a, p2a, p3a = P1
    p0b, p1b, p2b, p3b = P0
    a = [_cols(p1a, p2a, p3a), _cols(p0a, p2a, p3a), _cols(p0a, p1a, p3a), _cols(p0a, p1a, p2a)]
    b = [_cols(p1b, p2b, p3b), _cols(p0b, p2b, p3b), _cols(p0b, p1b, p3b), _cols(p0b, p1b, p2b)]
    a = [a[k] - b[k] for k in range(4)]
    return (det_polynomial(a[0], b[0]) - det_polynomial(a[1], b[1])
            + det_polynomial(a[2], b[2]) - det_polynomial(a[3], b[3]))


def _collision_time(P0, P1, verify):
    coef = coplanarity_cubic(P0, P1)
    n, roots = cubic_roots(coef, 0.0, 1.0)
    root = 1.0
    ok = False
    for i in range(n):
        root = roots[i]
        Pt = P0 * (1.0 - root) + P1 * root  # wp.lerp(a, b, t) = a (1 - t) + b t
        ok = verify(*Pt)
        if ok:
            break
    return root if ok else 1.0


def pt_collision_time(P0, P1):
    """ccd.py:133-156"""
    return _collision_time(np.asarray(P0, float), np.asarray(P1, float), verify_root_pt)


def ee_collision_time(P0, P1):
    """ccd.py:158-186"""
    return _collision_time(np.asarray(P0, float), np.asarray(P1, float), verify_root_ee)


def vg_collision_time(y0, y1, ground):
    """ccd.py:188-195"""
    d1 = y1 - ground
    if d1 < 0:
        d0 = y0 - ground
        return d0 / (d0 - d1)
    return 1.0


# ---------------------------------------------------------------------------------------
# inertia + orthogonality: orthogonal_energy.py
# ---------------------------------------------------------------------------------------
def inertia_terms(A, p, A0, p0, Adot, pdot, Ak, pk, mass, I0, dt, gravity, stiffness):
    """Energy at (Ak, pk); gradient (12) and Hessian (12x12) at (A, p)
    (orthogonal_energy.py:24-135)."""
    At = A0 + dt * Adot
    pt = p0 + dt * pdot + dt * dt * np.array([0.0, gravity, 0.0])
    eo = 0.0
    for i in range(3):
        for j in range(3):
            t = np.dot(Ak[i], Ak[j]) - (1.0 if i == j else 0.0)
            eo += t * t
    eo *= stiffness
    dq = [pk - pt, Ak[0] - At[0], Ak[1] - At[1], Ak[2] - At[2]]
    nm = np.dot(dq[0], dq[0]) * mass + (np.dot(dq[1], dq[1]) + np.dot(dq[2], dq[2])
                                          + np.dot(dq[3], dq[3])) * I0
    E = eo * dt * dt + 0.5 * nm
    g = np.zeros(12)
    for ii in range(1, 4):
        i = ii - 1
        gr = -A[i].copy()
        for j in range(3):
            gr = gr + np.dot(A[i], A[j]) * A[j]
        g[3 * ii:3 * ii + 3] = dt * dt * (gr * 4.0 * stiffness)
    Mq = [(p - pt) * mass, (A[0] - At[0]) * I0, (A[1] - At[1]) * I0, (A[2] - At[2]) * I0]
    for k in range(4):
        g[3 * k:3 * k + 3] += Mq[k]
    H = np.zeros((12, 12))
    for ii in range(4):
        for jj in range(4):
            m = 0.0 if ii != jj else (mass if ii == 0 else I0)
            dh = np.diag([m, m, m])
            if ii > 0 and jj > 0:
                i, j = ii - 1, jj - 1
                if i == j:
                    h = np.zeros((3, 3))
                    for k in range(3):
                        h = h + np.outer(A[k], A[k])
                    h = h + (np.outer(A[i], A[i]) + np.diag([np.dot(A[i], A[i]) - 1.0] * 3))
                else:
                    h = np.outer(A[j], A[i]) + np.diag([np.dot(A[j], A[i])] * 3)
                dh = dh + h * 4.0 * stiffness * dt * dt
            H[3 * ii:3 * ii + 3, 3 * jj:3 * jj + 3] = dh
    return E, g, H


FIXTURE = np.array([[0.4360, 0.0259, 0.5497],
                    [0.4353, 0.4204, 0.3303],
                    [0.2046, 0.6193, 0.2997],
                    [0.2668, 0.6211, 0.5291]])
"""Fixed 4-point fixture of abd/hl_entry.py:8-13 (= abd/ipc.py:98-103)."""
