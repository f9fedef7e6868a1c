"""The full IPC contact model (closest-feature classification, barrier on the classified
distance, edge-edge mollifier, PSD projection, mapping to affine DOFs) in
``abd_warp_b200/csrc/abd_ipc_full.cuh``, built for the host and checked against the numpy
restatement ``oracle/ipc_full_ref.py``, brute-force sampling, central differences and, on
interior contacts, the reference's own contact model (``oracle.contact_gh``).  CPU only."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import oracle
from oracle import ipc_full_ref as R
from abd_warp_b200.params import SimParams

HERE = os.path.dirname(os.path.abspath(__file__))
DH, KAPPA = 0.01, 1e3  # dhat^2 and stiffness of these unit-scale tests


@pytest.fixture(scope="module")
def L(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("ipcf") / "libipcf.so")
    src = os.path.join(HERE, "native", "ipc_full_host.cpp")
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-o", out, src], check=True)
    lib = ctypes.CDLL(out)
    v, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    lib.ipcf_type.argtypes = [i, v]
    lib.ipcf_type.restype = i
    lib.ipcf_d2.argtypes = [i, i, v]
    lib.ipcf_d2.restype = d
    lib.ipcf_energy.argtypes = [i, v, v, d, d]
    lib.ipcf_energy.restype = d
    lib.ipcf_local_gh.argtypes = [i, v, v, d, d, v, v, v, v, v]
    lib.ipcf_local_gh.restype = i
    lib.ipcf_project_psd12.argtypes = [v]
    lib.ipcf_eig_sym12.argtypes = [v, v, v]
    lib.ipcf_to_affine_vec.argtypes = [v, v, i, v]
    lib.ipcf_to_affine.argtypes = [v, v, v, i, v, v, v, v]
    return lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _x(a):
    return np.ascontiguousarray(a, dtype=np.float64).ravel()


def local_gh(L, kind, x, r):
    x, r = _x(x), _x(r)
    ty, d2, E = ctypes.c_int(0), ctypes.c_double(0), ctypes.c_double(0)
    g, H = np.zeros(12), np.zeros(144)
    ok = L.ipcf_local_gh(kind, _p(x), _p(r), DH, KAPPA, ctypes.byref(ty), ctypes.byref(d2), ctypes.byref(E), _p(g),
                         _p(H))
    return bool(ok), ty.value, d2.value, E.value, g, H.reshape(12, 12)


def random_pair(rng, kind, scale=1.0):
    """A random unit-scale triangle and point, or two edges."""
    return rng.normal(size=(4, 3)) * scale


def near_pair(rng, kind, dist):
    """A random pair with its first group (point / edge a) moved along the separation of the
    closest points until they are ``dist`` apart; the closest features stay the same."""
    while True:
        x = random_pair(rng, kind)
        ty, d2 = R.classify(kind, x)
        if d2 < 1e-6:
            continue
        ca, cb = R.separation(kind, x)
        n = 1 if kind == 0 else 2
        x[:n] += (ca - cb) / np.sqrt(d2) * (dist - np.sqrt(d2))
        ty2, d22 = R.classify(kind, x)
        if abs(np.sqrt(d22) - dist) < 1e-9 and ty2 == ty:
            return x, ty


def _tie_free(kind, x, tol=1e-7):
    """No near-tie between feature types (so both classifications must agree)."""
    for dx in (tol, -tol):
        for c in range(12):
            y = _x(x).copy()
            y[c] += dx
            if R.classify(kind, y)[0] != R.classify(kind, x)[0]:
                return False
    return True


@pytest.mark.parametrize("kind", [0, 1])
def test_types_and_distances_match_restatement(L, kind):
    rng = np.random.default_rng(10 + kind)
    seen = set()
    checked = 0
    for _ in range(3000):
        x = random_pair(rng, kind)
        ty_ref, d2_ref = R.classify(kind, x)
        if not _tie_free(kind, x):
            continue
        xs = _x(x)
        ty = L.ipcf_type(kind, _p(xs))
        assert ty == ty_ref, (x, ty, ty_ref)
        d2 = L.ipcf_d2(kind, ty, _p(xs))
        assert d2 == pytest.approx(d2_ref, rel=1e-10, abs=1e-14)
        seen.add(ty)
        checked += 1
    assert checked > 2500
    assert seen == set(range(7 if kind == 0 else 9)), seen  # every feature pair occurs


@pytest.mark.parametrize("kind", [0, 1])
def test_distance_is_the_sampled_minimum(L, kind):
    rng = np.random.default_rng(20 + kind)
    for _ in range(60):
        x = _x(random_pair(rng, kind))
        ty = L.ipcf_type(kind, _p(x))
        d2 = L.ipcf_d2(kind, ty, _p(x))
        ds = R.sample_d2(kind, x, n=301)
        assert d2 <= ds * (1 + 1e-12) + 1e-15  # the sampled points are on the primitives
        assert np.sqrt(ds) - np.sqrt(d2) < 0.05  # and the grid comes close to the minimum


@pytest.mark.parametrize("kind", [0, 1])
def test_gradient_hessian_central_differences(L, kind):
    rng = np.random.default_rng(30 + kind)
    done = 0
    while done < 40:
        x, ty = near_pair(rng, kind, dist=0.06)
        if not _tie_free(kind, x, tol=1e-4):
            continue
        r = random_pair(rng, kind)  # rest positions: the mollifier threshold only
        ok, ty_h, d2, E, g, H = local_gh(L, kind, x, r)
        assert ok and ty_h == ty
        assert E == pytest.approx(R.energy(kind, x, r, DH, KAPPA), rel=1e-10)
        gf, Hf = R.fd_gradient_hessian(kind, x, r, DH, KAPPA, 1e-5, ty)
        assert np.linalg.norm(g - gf) <= 1e-6 * np.linalg.norm(gf) + 1e-9
        assert np.linalg.norm(H - Hf) <= 1e-4 * np.linalg.norm(Hf)
        assert np.array_equal(H, H.T)
        done += 1


def test_inactive_beyond_dhat(L):
    rng = np.random.default_rng(40)
    for kind in (0, 1):
        x, _ = near_pair(rng, kind, dist=0.2)  # 0.2^2 > dhat^2 = 0.01
        ok, _, d2, _, _, _ = local_gh(L, kind, x, x)
        assert not ok and d2 == pytest.approx(0.04, rel=1e-8)
        assert L.ipcf_energy(kind, _p(_x(x)), _p(_x(x)), DH, KAPPA) == 0.0


def test_mollifier_parallel_edges(L):
    """Near-parallel edges: the energy is scaled by m(|a x b|^2 / e_x), which is 0 for
    parallel edges, 1 at and beyond e_x, and C1 there."""
    a0, a1 = np.array([0.0, 0.0, 0.0]), np.array([1.0, 0.0, 0.0])
    r = _x([a0, a1, [0.2, 0.05, 0.0], [0.8, 0.05, 0.0]])
    ex = R.eps_x(r)
    vals = []
    for ang in (0.0, 1e-4, 1e-3, 1e-2, 0.05, 0.2):
        b0 = np.array([0.2, 0.05, -0.3 * np.sin(ang)])
        b1 = np.array([0.8, 0.05, 0.3 * np.sin(ang)])
        x = _x([a0, a1, b0, b1])
        e = L.ipcf_energy(1, _p(x), _p(r), DH, KAPPA)
        assert e == pytest.approx(R.energy(1, x, r, DH, KAPPA), rel=1e-10, abs=1e-300)
        c = np.linalg.norm(np.cross(a1 - a0, b1 - b0)) ** 2
        m = R.mollifier(x, ex)
        assert (m == 1.0) == (c >= ex)
        vals.append(e)
    assert vals[0] == 0.0  # exactly parallel: no contribution
    assert vals == sorted(vals)  # grows as the edges turn apart (distance fixed at 0.05)


def test_energy_continuous_across_feature_boundaries(L):
    """A point sliding past a triangle edge and then past a vertex: the classified distance
    and the energy change continuously although the feature pair changes."""
    t = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]])
    for path in (lambda s: [0.3, -0.2 + s, 0.06], lambda s: [-0.2 + s, -0.2 + s, 0.06]):
        prev, types = None, set()
        for s in np.linspace(0.0, 0.4, 4001):
            x = _x(np.vstack([path(s), t]))
            types.add(L.ipcf_type(0, _p(x)))
            ok, _, d2, e, g, _ = local_gh(L, 0, x, x)
            if not ok:
                e, g = 0.0, np.zeros(12)
            if prev is not None:
                # no jump: the change stays within the gradient bound over the step
                dx = np.linalg.norm(x - prev[0])
                assert abs(e - prev[1]) <= 1.5 * max(np.linalg.norm(g), np.linalg.norm(prev[2])) * dx + 1e-15
                assert abs(np.sqrt(d2) - np.sqrt(prev[3])) <= dx * (1 + 1e-9)  # distance is 1-Lipschitz
            prev = (x, e, g, d2)
        assert len(types) >= 2


def test_psd_projection(L):
    rng = np.random.default_rng(50)
    for _ in range(50):
        A = rng.normal(size=(12, 12))
        H = _x(A + A.T)
        L.ipcf_project_psd12(_p(H))
        P = R.project_psd((A + A.T))
        assert np.allclose(H.reshape(12, 12), P, rtol=0, atol=1e-11 * np.abs(P).max())
        B = rng.normal(size=(12, 12))
        S = _x(B @ B.T)  # already PSD: unchanged
        S0 = S.copy()
        L.ipcf_project_psd12(_p(S))
        assert np.allclose(S, S0, rtol=0, atol=1e-11 * np.abs(S0).max())


def test_eigen_decomposition(L):
    """Round-robin Jacobi: H V = V diag(lam), V orthonormal, the spectrum of numpy's eigh."""
    rng = np.random.default_rng(55)
    mats = [rng.normal(size=(12, 12)) for _ in range(30)]
    mats = [m + m.T for m in mats] + [np.diag(rng.normal(size=12)), np.zeros((12, 12))]
    for A in mats:
        lam, V = np.zeros(12), np.zeros(144)
        L.ipcf_eig_sym12(_p(_x(A)), _p(lam), _p(V))
        V = V.reshape(12, 12)
        scale = max(np.abs(A).max(), 1e-300)
        assert np.abs(A @ V - V * lam).max() <= 1e-12 * scale
        assert np.abs(V.T @ V - np.eye(12)).max() <= 1e-13
        assert np.allclose(np.sort(lam), np.linalg.eigvalsh(A), rtol=0, atol=1e-12 * scale)


def test_rank_one_form_of_a_contact(L):
    """The projected contact Hessian as rank-one terms lam_k u_k u_k^T over the affine DOFs
    (u_k = to_affine_vec of eigenvector k): the assembly's form, equal to to_affine of the
    projected matrix."""
    rng = np.random.default_rng(57)
    for kind in (0, 1):
        x, _ = near_pair(rng, kind, dist=0.05)
        r = x + rng.normal(size=(4, 3)) * 0.1
        ok, _, _, _, g, H = local_gh(L, kind, x, r)
        assert ok
        lam, V = np.zeros(12), np.zeros(144)
        L.ipcf_eig_sym12(_p(_x(H)), _p(lam), _p(V))
        V = V.reshape(12, 12)
        nI = 1 if kind == 0 else 2
        H24 = np.zeros((24, 24))
        for k in range(12):
            if lam[k] > 0:
                u = np.zeros(24)
                L.ipcf_to_affine_vec(_p(np.ascontiguousarray(V[:, k])), _p(_x(r)), nI, _p(u))
                H24 += lam[k] * np.outer(u, u)
        Hp = _x(H)
        L.ipcf_project_psd12(_p(Hp))
        g24, Hi, Hj, Hij = np.zeros(24), np.zeros(144), np.zeros(144), np.zeros(144)
        L.ipcf_to_affine(_p(g), _p(Hp), _p(_x(r)), nI, _p(g24), _p(Hi), _p(Hj), _p(Hij))
        s = np.abs(H24).max()
        assert np.abs(H24[:12, :12] - Hi.reshape(12, 12)).max() <= 1e-11 * s
        assert np.abs(H24[12:, 12:] - Hj.reshape(12, 12)).max() <= 1e-11 * s
        assert np.abs(H24[:12, 12:] - Hij.reshape(12, 12)).max() <= 1e-11 * s


def test_to_affine(L):
    rng = np.random.default_rng(60)
    for nI in (1, 2):
        gx, Hx, r = rng.normal(size=12), rng.normal(size=(12, 12)), rng.normal(size=12)
        Hx = _x(Hx + Hx.T)
        g24, Hi, Hj, Hij = np.zeros(24), np.zeros(144), np.zeros(144), np.zeros(144)
        L.ipcf_to_affine(_p(gx), _p(Hx), _p(r), nI, _p(g24), _p(Hi), _p(Hj), _p(Hij))
        rg, ri, rj, rij = R.to_affine(gx, Hx, r, nI)
        for a, b in ((g24, rg), (Hi, ri), (Hj, rj), (Hij, rij)):
            assert np.allclose(np.reshape(a, np.shape(b)), b, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("kind", [0, 1])
def test_interior_contacts_reduce_to_the_reference_model(L, kind):
    """On interior contacts (point over the triangle's interior; edges crossing, away from
    parallel) the full model's distance, energy and affine gradient equal the reference's."""
    prm = SimParams()
    prm.dhat, prm.kappa = float(np.sqrt(DH)), KAPPA
    assert prm.d2hat == pytest.approx(DH, rel=1e-15)
    rng = np.random.default_rng(70 + kind)
    done = 0
    while done < 30:
        x, ty = near_pair(rng, kind, dist=0.05)
        if ty != 0 or not _tie_free(kind, x, tol=1e-4):
            continue
        r = x + rng.normal(size=(4, 3)) * 0.1
        if kind == 1 and R.mollifier(x, R.eps_x(r)) != 1.0:
            continue
        active, d2_ref, g_ref, _, _, _ = oracle.contact_gh(kind, x, r, prm)
        ok, _, d2, E, g, H = local_gh(L, kind, x, r)
        assert active and ok
        assert d2 == pytest.approx(d2_ref, rel=1e-10)
        assert E == pytest.approx(oracle.contact_energy(kind, x, prm), rel=1e-10)
        g24, Hi, Hj, Hij = np.zeros(24), np.zeros(144), np.zeros(144), np.zeros(144)
        nI = 1 if kind == 0 else 2
        L.ipcf_to_affine(_p(g), _p(_x(H)), _p(_x(r)), nI, _p(g24), _p(Hi), _p(Hj), _p(Hij))
        assert np.linalg.norm(g24 - g_ref) <= 1e-8 * np.linalg.norm(g_ref)
        done += 1


@pytest.mark.parametrize("kind", [0, 1])
def test_oracle_full_model_matches_the_header(L, kind):
    """The C++ oracle's full model (forward-mode AD carrying the whole Hessian, its own
    classification and Jacobi projection) against the header's (hyper-dual entries): same
    feature pair, distance and energy; the projected affine terms to 1e-9, in both group
    orders of the pair."""
    prm = SimParams()
    prm.dhat, prm.kappa = float(np.sqrt(DH)), KAPPA
    rng = np.random.default_rng(80 + kind)
    seen = set()
    done = 0
    while done < 60:
        x, ty = near_pair(rng, kind, dist=0.07)
        if not _tie_free(kind, x, tol=1e-6):
            continue
        r = x + rng.normal(size=(4, 3)) * (0.1 if done % 2 else 2.0)  # mollified and not
        ok, ty_h, d2, E, g, H = local_gh(L, kind, x, r)
        Hp = _x(H)
        L.ipcf_project_psd12(_p(Hp))
        g24, Hi, Hj, Hij = np.zeros(24), np.zeros(144), np.zeros(144), np.zeros(144)
        L.ipcf_to_affine(_p(g), _p(Hp), _p(_x(r)), 1 if kind == 0 else 2, _p(g24), _p(Hi), _p(Hj), _p(Hij))
        Hi, Hj, Hij = Hi.reshape(12, 12), Hj.reshape(12, 12), Hij.reshape(12, 12)
        for swap in (0, 1):
            a, Eo, d2o, tyo, HIJ, HII, HJJ, go = oracle.full_terms(kind, x, r, prm, swap)
            assert a and ok and tyo == ty_h == ty
            assert d2o == pytest.approx(d2, rel=1e-12) and Eo == pytest.approx(E, rel=1e-10)
            want = (Hij, Hi, Hj, g24) if swap == 0 else (Hij.T, Hj, Hi, np.concatenate([g24[12:], g24[:12]]))
            for got, ref in zip((HIJ, HII, HJJ, go), want):
                assert np.linalg.norm(got - ref) <= 1e-9 * max(np.linalg.norm(ref), np.linalg.norm(Hi) * 1e-6)
        seen.add(ty)
        done += 1
    assert len(seen) >= 4


def _min_surface_distance(flat, x):
    """Minimum distance between the two bodies' surfaces over every PT and EE pair."""
    voff, toff, eoff = flat["voff"], flat["toff"], flat["eoff"]
    tris, edges = flat["tris"].reshape(-1, 3), flat["edges"].reshape(-1, 2)
    best = np.inf
    for a, b in ((0, 1), (1, 0)):
        for v in range(voff[a], voff[a + 1]):
            for t in range(toff[b], toff[b + 1]):
                best = min(best, R.classify(0, np.vstack([x[v], x[tris[t]]]))[1])
    for e in range(eoff[0], eoff[1]):
        for f in range(eoff[1], eoff[2]):
            best = min(best, R.classify(1, np.vstack([x[edges[e]], x[edges[f]]]))[1])
    return float(np.sqrt(best))


def test_oracle_full_mode_steps():
    """Two cubes (configuration 0: one falls onto the other, fixed) with the full contact
    model in the oracle: identical to the reference model before the first contact; after
    it the bodies stay apart (surface distance near dhat) with at least one active contact
    every step.  The reference model loses every contact at steps 16-18 of this scene while
    the bodies touch; only its CCD cap keeps them apart there."""
    from abd_warp_b200 import scenes

    bodies, prm, _ = scenes.make_config(0)
    flat = scenes.flatten_bodies(bodies)
    ref, full = oracle.Oracle(flat, prm), oracle.Oracle(flat, prm)
    full.set_ipc_full(True)
    contact, lost_ref = False, 0
    for k in range(25):
        a, b = ref.step(), full.step()
        if not contact and b["n_active"] == 0:
            assert a == b
        contact = contact or b["n_active"] > 0
        assert b["newton_iters"] <= prm.max_iter and np.isfinite(b["energy"])
        if contact:
            assert b["n_active"] > 0
            lost_ref += a["n_active"] == 0
            assert _min_surface_distance(flat, full.get_state()["x_view"]) > 0.5 * prm.dhat
    assert contact and lost_ref > 0


def _friction_lag(L, kind, xt, r):
    w, P, lam = np.zeros(4), np.zeros(6), ctypes.c_double(0)
    ok = L.ipcf_friction_lag(kind, _p(_x(xt)), _p(_x(r)), DH, KAPPA, _p(w), _p(P), ctypes.byref(lam))
    return bool(ok), w, P, lam.value


def _friction_gh(L, w, P, lam, x, xt, mu, eps):
    g, H = np.zeros(12), np.zeros(144)
    D = L.ipcf_friction_gh(_p(w), _p(P), lam, _p(_x(x)), _p(_x(xt)), mu, eps, _p(g), _p(H))
    return D, g, H.reshape(12, 12)


@pytest.fixture(scope="module")
def Lf(L):
    v, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    L.ipcf_friction_lag.argtypes = [i, v, v, d, d, v, v, v]
    L.ipcf_friction_lag.restype = i
    L.ipcf_friction_gh.argtypes = [v, v, d, v, v, d, d, v, v]
    L.ipcf_friction_gh.restype = d
    return L


@pytest.mark.parametrize("kind", [0, 1])
def test_friction_lagged_quantities(Lf, kind):
    """At the step start: the weights give the separation of the closest points (as this
    module's restatement finds them), P is an orthonormal basis of the plane orthogonal to
    it, and lambda is the barrier's -dE/dd."""
    rng = np.random.default_rng(90 + kind)
    seen = set()
    done = 0
    while done < 40:
        xt, ty = near_pair(rng, kind, dist=0.05)
        if not _tie_free(kind, xt, tol=1e-6):
            continue
        r = xt + rng.normal(size=(4, 3)) * (0.1 if done % 2 else 2.0)
        ok, w, P, lam = _friction_lag(Lf, kind, xt, r)
        assert ok
        ca, cb = R.separation(kind, xt)
        assert np.allclose(w @ xt, ca - cb, rtol=0, atol=1e-12)
        assert np.allclose(w, R.closest_weights(kind, xt), rtol=0, atol=1e-9)
        n = (ca - cb) / np.linalg.norm(ca - cb)
        Pm = P.reshape(3, 2)
        assert np.allclose(Pm.T @ Pm, np.eye(2), atol=1e-14) and np.allclose(Pm.T @ n, 0.0, atol=1e-10)
        assert lam > 0 and lam == pytest.approx(R.normal_force(kind, xt, r, DH, KAPPA), rel=1e-6)
        seen.add(ty)
        done += 1
    assert len(seen) >= 4


@pytest.mark.parametrize("kind", [0, 1])
@pytest.mark.parametrize("regime", ["static", "sliding"])
def test_friction_gradient_hessian(Lf, kind, regime):
    """D, its gradient (central differences, 1e-6) and Hessian (1e-4, positive semidefinite)
    below eps (static friction) and above (sliding); the tangential force stays within the
    Coulomb bound mu lambda and reaches it when sliding."""
    mu, eps = 0.4, 1e-3
    rng = np.random.default_rng(100 + kind + (2 if regime == "sliding" else 0))
    done = 0
    while done < 20:
        xt, _ = near_pair(rng, kind, dist=0.05)
        ok, w, P, lam = _friction_lag(Lf, kind, xt, xt)
        if not ok:
            continue
        y_goal = 0.4 * eps if regime == "static" else 5 * eps
        dx = rng.normal(size=(4, 3))
        dx *= y_goal / max(np.linalg.norm(P.reshape(3, 2).T @ (w @ dx)), 1e-300)
        x = xt + dx
        D, g, H = _friction_gh(Lf, w, P, lam, x, xt, mu, eps)
        f = lambda y: R.friction_potential(w, P, lam, y, xt, mu, eps)
        assert D == pytest.approx(f(_x(x)), rel=1e-12)
        h = 1e-4 * eps
        I = np.eye(12) * h
        xf = _x(x)
        gf = np.array([(f(xf + I[i]) - f(xf - I[i])) / (2 * h) for i in range(12)])
        Hf = np.array([[(f(xf + I[i] + I[j]) - f(xf + I[i] - I[j]) - f(xf - I[i] + I[j]) + f(xf - I[i] - I[j]))
                        / (4 * h * h) for j in range(12)] for i in range(12)])
        assert np.linalg.norm(g - gf) <= 1e-6 * np.linalg.norm(gf)
        assert np.linalg.norm(H - Hf) <= 1e-4 * np.linalg.norm(Hf)
        assert np.linalg.eigvalsh(H).min() >= -1e-12 * np.abs(H).max()
        v = int(np.argmax(np.abs(w)))  # a point's share of the force, per unit weight
        force = np.linalg.norm(g[3 * v:3 * v + 3]) / abs(w[v])
        assert force <= mu * lam * (1 + 1e-12)
        if regime == "sliding":
            assert force == pytest.approx(mu * lam, rel=1e-12)
        done += 1


def test_oracle_friction_sliding_cube():
    """A cube sliding on the ground box at 1 m/s (full contact model, lagged friction in the
    oracle): without friction it keeps its speed; with mu = 0.5 it decelerates at mu g
    (Coulomb) until it stops at t = v0 / (mu g), and static friction then holds it."""
    from abd_warp_b200 import scenes

    prm = SimParams()
    prm.max_iter, prm.tol = 100, 1e-12  # converged steps
    g = -prm.gravity
    bodies = [scenes.ground_box(), scenes._body("cube:0.3", (0.0, 0.15 + 1.2 * prm.dhat, 0.0), v=(1.0, 0.0, 0.0))]
    flat = scenes.flatten_bodies(bodies)
    for mu in (0.0, 0.5):
        o = oracle.Oracle(flat, prm)
        o.set_ipc_full(True)
        o.set_friction(mu, 1e-3)
        for k in range(1, 31):
            info = o.step()
            vx = o.get_state()["pdot"][1, 0]
            assert info["n_active"] > 0
            if mu == 0.0:
                assert vx == pytest.approx(1.0, abs=1e-6)
            elif 3 <= k and k * prm.dt < 1.0 / (mu * g) - 2 * prm.dt:
                # the cube lands in step 1; step 2 lags the landing's normal force
                assert vx == pytest.approx(1.0 - mu * g * (k - 1) * prm.dt, abs=1e-3)
            elif k * prm.dt > 1.0 / (mu * g) + 2 * prm.dt:
                assert abs(vx) < 1e-6


@pytest.mark.parametrize("kind", [0, 1])
def test_oracle_friction_matches_the_header(Lf, kind):
    """The oracle's lagged friction (its own weights from sub-triangle areas, its own basis)
    against the header's per contact: weights, normal force, D, gradient and Hessian (which do
    not depend on the choice of tangent basis), static and sliding."""
    prm = SimParams()
    prm.dhat, prm.kappa = float(np.sqrt(DH)), KAPPA
    mu, eps = 0.3, 1e-3
    rng = np.random.default_rng(120 + kind)
    done = 0
    while done < 30:
        xt, _ = near_pair(rng, kind, dist=0.05)
        if not _tie_free(kind, xt, tol=1e-6):
            continue
        r = xt + rng.normal(size=(4, 3)) * (0.1 if done % 2 else 2.0)
        ok, w, P, lam = _friction_lag(Lf, kind, xt, r)
        x = xt + rng.normal(size=(4, 3)) * (2e-4 if done % 3 else 3e-3)
        D, g, H = _friction_gh(Lf, w, P, lam, x, xt, mu, eps)
        a, Do, go, Ho, wo, lamo = oracle.friction_contact(kind, xt, r, prm, mu, eps, x)
        assert ok and a
        assert np.allclose(wo, w, rtol=0, atol=1e-10) and lamo == pytest.approx(lam, rel=1e-10)
        assert Do == pytest.approx(D, rel=1e-10)
        assert np.linalg.norm(go - g) <= 1e-9 * np.linalg.norm(g)
        assert np.linalg.norm(Ho - H) <= 1e-9 * np.linalg.norm(H)
        done += 1


def test_oracle_full_mode_header_and_independent_agree():
    """The oracle's two full-model arithmetics on a contact-rich state (two cubes after the
    full model's first contact steps): the header's (hyper-dual entries, the CUDA library's
    arithmetic) and the oracle's own forward-mode restatement assemble the same gradient and
    Hessian blocks to 1e-9 relative, and the same energy to 1e-12."""
    from abd_warp_b200 import scenes

    bodies, prm, _ = scenes.make_config(0)
    flat = scenes.flatten_bodies(bodies)
    hd, ind = oracle.Oracle(flat, prm), oracle.Oracle(flat, prm)
    hd.set_ipc_full(True)
    ind.set_ipc_full(True, independent=True)
    for _ in range(8):
        hd.step()
    st = hd.get_state()
    ind.set_state(st["A0"], st["p0"], st["Adot"], st["pdot"], st["dq"])
    A = st["A0"] + prm.dt * st["Adot"]
    p = st["p0"] + prm.dt * st["pdot"]
    a, b = hd.gh(A, p), ind.gh(A, p)
    assert a["n_active"] == b["n_active"] > 0
    for k in ("g", "diag", "off"):
        scale = np.abs(b[k]).max()
        assert np.abs(a[k] - b[k]).max() <= 1e-9 * scale, k
    assert hd.energy(A, p) == pytest.approx(ind.energy(A, p), rel=1e-12)


def test_oracle_friction_steps_header_and_independent_agree():
    """The oracle's step with friction in its two arithmetics -- the header's (the CUDA
    library's: friction_lag / friction_gh and the point-to-body map of the full model) and its
    own restatement -- gives the same sliding cube to 1e-8 over 12 steps."""
    import dataclasses

    from abd_warp_b200 import scenes

    prm = SimParams()
    prm.max_iter, prm.tol = 100, 1e-12
    prm = dataclasses.replace(prm, ipc_full=1, friction_mu=0.5, friction_epsv=1e-3)
    bodies = [scenes.ground_box(), scenes._body("cube:0.3", (0.0, 0.15 + 1.2 * prm.dhat, 0.0), v=(1.0, 0.0, 0.0))]
    flat = scenes.flatten_bodies(bodies)
    oh, oi = oracle.Oracle(flat, prm), oracle.Oracle(flat, prm)
    oi.set_ipc_full(True, independent=True)
    for _ in range(12):
        rh, ri = oh.step(), oi.step()
        assert rh["n_active"] == ri["n_active"] > 0
        sh, si = oh.get_state(), oi.get_state()
        for k in ("p0", "A0", "pdot"):
            np.testing.assert_allclose(sh[k], si[k], rtol=0, atol=1e-8)
    assert sh["pdot"][1, 0] < 0.6  # it decelerated
