"""Known-answer tests of the CPU restatements (oracle/np_ref.py, oracle/abd_oracle.cpp)
against the reference's own checks and the committed golden fixture."""
import os

import numpy as np
import pytest

import oracle
from oracle import np_ref as R
from abd_warp_b200.params import SimParams

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "contact_fixture.npz")


@pytest.mark.parametrize("C", [R.C_vf, R.C_ee])
def test_fixture_eigensystem_reconstruction(C):
    """hl_entry.py:115-147: Q Lambda Q^-1 equals 2 l Hl + 2 gl gl^T on the fixed fixture."""
    e0, e1, e2 = C(*R.FIXTURE)
    Q, lam = R.eig_Hl(e0, e1, e2)
    H = R.d2Psi(e0, e1, e2)
    assert np.abs(R.QLQinv(Q, lam) - H).max() <= 1e-12 * np.abs(H).max()
    G = Q.T @ Q
    assert np.abs(G - np.diag(np.diag(G))).max() <= 1e-12 * np.abs(G).max()


@pytest.mark.parametrize("C", [R.C_vf, R.C_ee])
def test_distance_identity(C):
    """psd/hl.py:253-265: l^2 equals |e2_perp|^2."""
    rng = np.random.default_rng(1)
    for _ in range(50):
        e0, e1, e2 = C(*rng.normal(size=(4, 3)))
        l = R.signed_distance(e0, e1, e2)
        assert abs(l * l - e2 @ e2) <= 1e-12 * (e2 @ e2)


@pytest.mark.parametrize("typ", [0, 1])
def test_gradient_matches_finite_differences(typ):
    """The c-space gradient mapped by the frozen dc/dx is the exact gradient of d^2."""
    C, D = (R.C_vf, R.dcvfdx_s) if typ == 0 else (R.C_ee, R.dceedx_s)
    rng = np.random.default_rng(2 + typ)
    for _ in range(5):
        X = rng.normal(size=(4, 3))
        e0, e1, e2 = C(*X)
        Q, _ = R.eig_Hl(e0, e1, e2)
        g = np.kron(D(*X).T, np.eye(3)) @ Q[:, 4]
        f = lambda Y: float(np.dot(C(*Y)[2], C(*Y)[2]))
        fd = np.zeros(12)
        for i in range(12):
            Xp, Xm = X.ravel().copy(), X.ravel().copy()
            Xp[i] += 1e-6
            Xm[i] -= 1e-6
            fd[i] = (f(Xp.reshape(4, 3)) - f(Xm.reshape(4, 3))) / 2e-6
        assert np.abs(fd - g).max() <= 1e-6 * np.abs(g).max()


def test_golden_restatement_regression():
    d = np.load(GOLDEN)
    for typ, C in ((0, R.C_vf), (1, R.C_ee)):
        name = "pt" if typ == 0 else "ee"
        for i, x in enumerate(d["x"]):
            Q, lam = R.eig_Hl(*C(*x))
            np.testing.assert_allclose(lam, d[f"{name}_lam"][i], rtol=1e-12, atol=0)


@pytest.mark.parametrize("mode", [0, 1])
def test_oracle_per_pair_matches_golden(mode):
    d = np.load(GOLDEN)
    prm = SimParams(dhat=1.0, kappa=1.0, contact_psd=mode)
    n_act = 0
    for typ in (0, 1):
        name = "pt" if typ == 0 else "ee"
        for i in range(len(d["x"])):
            a, d2, g, Hi, Hj, Hij = oracle.contact_gh(typ, d["x"][i], d["r"][i], prm)
            gold_g = d[f"{name}_g_mode{mode}"][i]
            assert a == (not np.isnan(gold_g).any())
            if not a:
                continue
            n_act += 1
            gH = d[f"{name}_H_mode{mode}"][i]
            for got, ref in ((g, gold_g), (Hi, gH[0]), (Hj, gH[1]), (Hij, gH[2])):
                assert np.abs(got - ref).max() <= 1e-12 * max(np.abs(ref).max(), 1e-300)
            e = oracle.contact_energy(typ, d["x"][i], prm)
            assert e == pytest.approx(d[f"{name}_energy"][i], rel=1e-12, abs=1e-300)
    assert n_act >= 8


@pytest.mark.parametrize("mode", [0, 1])
def test_oracle_per_pair_matches_numpy_random(mode):
    prm = SimParams(dhat=1.0, kappa=1.0, contact_psd=mode)
    rng = np.random.default_rng(11)
    for _ in range(200):
        X, r = rng.normal(size=(4, 3)), rng.normal(size=(4, 3))
        for typ, term in ((0, R.pt_term), (1, R.ee_term)):
            a, d2, g, Hi, Hj, Hij = oracle.contact_gh(typ, X, r, prm)
            ref = term(X, r, prm.d2hat, prm.kappa, contact_psd=mode)
            assert a == (ref is not None)
            if a:
                for got, want in zip((g, Hi, Hj, Hij), ref[1:]):
                    assert np.abs(got - want).max() <= 1e-12 * max(np.abs(want).max(), 1e-300)


def _three_root_cubics(n, bound, rng):
    """cubic_roots.py:225-246: a0 (x-a)(x-b)(x-c) with a <= b <= c in [0, bound)."""
    out = []
    for _ in range(n):
        abc = np.sort(rng.random(3) * bound)
        a, b, c = abc
        a0 = rng.random() * bound + 0.1
        out.append((np.array([-a * b * c, a * b + a * c + b * c, -a - b - c, 1.0]) * a0, abc))
    return out


def test_cubic_roots_constructed():
    rng = np.random.default_rng(5)
    for coef, abc in _three_root_cubics(200, 5.0, rng):
        if np.min(np.diff(abc)) < 1e-3:
            continue
        n, roots = oracle.cubic_roots(coef, -5.0, 5.0)
        n2, roots2 = R.cubic_roots(coef, -5.0, 5.0)
        assert n == n2 == 3
        np.testing.assert_array_equal(roots, np.array(roots2))
        np.testing.assert_allclose(np.sort(roots), abc, rtol=0, atol=1e-7)


def test_quadratic_and_deflate():
    """cubic_roots.py:248-279: constructed 2-root quadratics; deflation by a known root."""
    rng = np.random.default_rng(6)
    for _ in range(100):
        ab = np.sort(rng.random(2) * 5.0)
        a0 = rng.random() * 5 + 0.1
        n, r = R.quadratic_roots([ab[0] * ab[1] * a0, -(ab[0] + ab[1]) * a0, a0], -5.0, 5.0)
        assert n == 2
        np.testing.assert_allclose(r, ab, atol=1e-9)
    coef = np.array([-6.0, 11.0, -6.0, 1.0])
    n, r = R.quadratic_roots(R.deflate(coef, 1.0), -5.0, 5.0)
    assert n == 2 and np.allclose(r, [2.0, 3.0])


def test_inside_triangle_negatives():
    """test_distance.py:35-81: points above reflected barycentric coordinates are outside.
    (The reference seeds every sample identically; each sample here has its own seed.)"""
    for s in range(1000):
        rng = np.random.default_rng(114514 + s)
        e0, e1 = rng.random(3), rng.random(3)
        b_, g_ = rng.random(), 0.0
        g_ = rng.random() * (1.0 - b_)
        beta, gamma = 1.0 - g_, 1.0 - b_
        n = np.cross(e0, e1)
        t0 = np.zeros(3)
        p = n * rng.random() + t0 + beta * e0 + gamma * e1
        assert not R.verify_root_pt(p, t0 + e0, t0, t0 + e1)


@pytest.mark.parametrize("typ", [0, 1])
def test_collision_time_known_crossing(typ):
    rng = np.random.default_rng(9 + typ)
    for _ in range(50):
        t_hit = rng.uniform(0.1, 0.9)
        if typ == 0:
            tri = rng.normal(size=(3, 3))
            b, c = 0.25, 0.3
            n = np.cross(tri[1] - tri[0], tri[2] - tri[0])
            n /= np.linalg.norm(n)
            q = tri[0] + b * (tri[1] - tri[0]) + c * (tri[2] - tri[0])
            p0, p1 = q + n * t_hit, q - n * (1.0 - t_hit)
            P0 = np.stack([p0, tri[1], tri[0], tri[2]])
            P1 = np.stack([p1, tri[1], tri[0], tri[2]])
        else:
            a0, a1 = np.array([-1.0, 0, 0]), np.array([1.0, 0, 0])
            b0, b1 = np.array([0.1, -1.0, 0]), np.array([0.1, 1.0, 0])
            up = np.array([0, 0, 1.0])
            P0 = np.stack([a0, a1, b0 + up * t_hit, b1 + up * t_hit])
            P1 = np.stack([a0, a1, b0 - up * (1 - t_hit), b1 - up * (1 - t_hit)])
        t = oracle.collision_time(typ, P0, P1)
        t2 = (R.pt_collision_time if typ == 0 else R.ee_collision_time)(P0, P1)
        assert t == pytest.approx(t_hit, abs=1e-8)
        assert t == t2


def test_oracle_free_fall_matches_implicit_euler():
    """orthogonal_energy.py:190-238: inertia-only body; implicit Euler under gravity is exact
    for the quadratic energy: v1 = v0 + g dt, x1 = x0 + v1 dt."""
    from abd_warp_b200 import scenes
    b = scenes._body("cube:0.5", (0.0, 2.0, 0.0), v=(0.3, 0.0, -0.2))
    prm = SimParams()
    o = oracle.Oracle(scenes.flatten_bodies([b]), prm)
    p, v = np.array([0.0, 2.0, 0.0]), np.array([0.3, 0.0, -0.2])
    for _ in range(20):
        info = o.step()
        v = v + np.array([0, prm.gravity, 0]) * prm.dt
        p = p + v * prm.dt
        assert info["newton_iters"] <= 3
    st = o.get_state()
    np.testing.assert_allclose(st["p0"][0], p, rtol=0, atol=1e-10)
    np.testing.assert_allclose(st["A0"][0], np.eye(3), atol=1e-12)
