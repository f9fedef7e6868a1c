"""The allocation-free inertia energy entry point (abd_inertia_energy_noalloc), called
through the C ABI, against the existing energy entry point.

Some callers may not allocate device memory once they run (fixed-budget real-time loops,
plug-ins whose host application owns all device memory); this entry point serves them with
a fixed scratch array inside the library.  On a contact-free state the barrier term is
exactly zero, so abd_compute_energy returns the same inertia + orthogonality energy; two
calls in a row must both agree with it (the shared scratch keeps the previous call's
partials, which the next call overwrites).  Collected last so that a run stopping at the
first failure has run every other test; it also passes alone in a fresh process."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_inertia_energy_noalloc_matches_compute_energy():
    import torch

    from abd_warp_b200 import _lib, scenes
    from abd_warp_b200.simulator import AffineBodySimulator

    bodies, prm, _ = scenes.make_config(1)  # spheres start more than dhat apart
    sim = AffineBodySimulator(bodies=bodies, params=prm)
    try:
        L = _lib.load()
        f = L.abd_inertia_energy_noalloc
        P = ctypes.c_void_p
        f.argtypes = [P, ctypes.c_int, P, P, P, P, P, P, P, P]
        f.restype = ctypes.c_int
        s = sim.states
        dev = sim.device
        fixed = torch.as_tensor(sim.flat["fixed"], dtype=torch.int32, device=dev)
        E_dev = torch.zeros(1, dtype=torch.float64, device=dev)
        cprm = prm.to_c()
        cst = sim._cstates()
        stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
        ptr = lambda t: ctypes.c_void_p(t.data_ptr())
        rng = np.random.default_rng(3)
        n = sim.n_bodies
        results = []
        for call in range(2):
            Ak = s.A0 + 1e-5 * torch.as_tensor(rng.normal(size=(n, 3, 3)), device=dev)
            pk = s.p0 + 1e-5 * torch.as_tensor(rng.normal(size=(n, 3)), device=dev)
            E_ref = sim.compute_energy(Ak, pk)
            rc = f(ctypes.byref(cprm), n, ctypes.byref(cst), ptr(Ak), ptr(pk), ptr(s.mass), ptr(s.I0), ptr(fixed),
                   ptr(E_dev), stream)
            assert rc == _lib.ABD_OK, rc
            torch.cuda.synchronize(dev)
            E = float(E_dev.item())
            assert E == pytest.approx(E_ref, rel=1e-12, abs=0.0), (call, E, E_ref)
            results.append(E)
        assert results[0] != results[1]  # two different states, both matched
        # sizes beyond the scratch capacity (or empty) are rejected before any launch
        for bad in (0, 1 << 21):
            rc = f(ctypes.byref(cprm), bad, ctypes.byref(cst), ptr(s.A0), ptr(s.p0), ptr(s.mass), ptr(s.I0),
                   ptr(fixed), ptr(E_dev), stream)
            assert rc == 2  # ABD_ERR_INVALID
    finally:
        sim.close()


@pytest.mark.parametrize("n", [300, 300_000])
def test_inertia_energy_noalloc_many_blocks(n):
    """Synthetic states of n bodies, one CTA per 256 bodies: 2 CTAs, and 1,172 CTAs (more than
    the finishing kernel's 1,024 threads, so it loops over the partials).  The result is a
    fixed-order tree sum, so it is compared with the exact sum of the same per-body energies
    to 1e-12 relative, on two calls in a row with different states (the scratch array keeps
    the first call's partials, which the second overwrites)."""
    import torch

    import oracle
    from abd_warp_b200 import _lib
    from abd_warp_b200.params import SimParams

    L = _lib.load()
    f = L.abd_inertia_energy_noalloc
    P = ctypes.c_void_p
    f.argtypes = [P, ctypes.c_int, P, P, P, P, P, P, P, P]
    f.restype = ctypes.c_int
    prm = SimParams()
    cprm = prm.to_c()
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(n)
    eye = np.tile(np.eye(3), (n, 1, 1))
    A0 = eye + 1e-2 * rng.normal(size=(n, 3, 3))
    p0 = rng.uniform(-5, 5, size=(n, 3))
    Adot = 1e-1 * rng.normal(size=(n, 3, 3))
    pdot = rng.normal(size=(n, 3))
    mass = rng.uniform(1.0, 50.0, size=n)
    I0 = rng.uniform(0.01, 1.0, size=n)
    fixed = (rng.uniform(size=n) < 0.05).astype(np.int32)
    cu = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    t = {k: cu(v) for k, v in dict(A0=A0, p0=p0, Adot=Adot, pdot=pdot, mass=mass, I0=I0, fixed=fixed).items()}
    E_dev = torch.zeros(1, dtype=torch.float64, device=dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    ptr = lambda x: ctypes.c_void_p(x.data_ptr())
    got = []
    for call in range(2):
        Ak = A0 + 1e-3 * rng.normal(size=(n, 3, 3))
        pk = p0 + 1e-2 * rng.normal(size=(n, 3))
        tAk, tpk = cu(Ak), cu(pk)
        st = _lib.States(ptr(tAk), ptr(tpk), ptr(tAk), ptr(tpk), ptr(t["Adot"]), ptr(t["pdot"]), ptr(t["A0"]),
                         ptr(t["p0"]))
        rc = f(ctypes.byref(cprm), n, ctypes.byref(st), ptr(tAk), ptr(tpk), ptr(t["mass"]), ptr(t["I0"]),
               ptr(t["fixed"]), ptr(E_dev), stream)
        assert rc == _lib.ABD_OK, rc
        torch.cuda.synchronize(dev)
        E = float(E_dev.item())
        ref = oracle.inertia_energy_sum(prm, Ak, pk, A0, p0, Adot, pdot, mass, I0, fixed)
        assert E == pytest.approx(ref, rel=1e-12, abs=0.0), (call, E, ref)
        got.append(E)
    assert got[0] != got[1]
