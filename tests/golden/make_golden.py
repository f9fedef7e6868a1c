"""Generate tests/golden/contact_fixture.npz from the NumPy restatement (oracle/np_ref.py).

Inputs: the reference's fixed 4-point array (abd/hl_entry.py:8-13 = abd/ipc.py:98-103) used
as a point-triangle and an edge-edge configuration, plus seeded random configurations.  The
barrier is evaluated with d2hat = 1 and kappa = 1 so the fixture's pairs are active.
Outputs: d^2, eigenvalues, the 9x9 c-space Hessian reconstruction, per-pair gradients and
12x12 body blocks in both eigenvalue modes, and contact energies.
Run: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import np_ref as R  # noqa: E402


def main():
    rng = np.random.default_rng(20240601)
    # the fixture, 3 unconstrained random configurations, and 12 constructed ones whose
    # projection is interior for both the PT and the EE reading (test_distance.py:17-33)
    X = [R.FIXTURE.copy()] + [rng.normal(size=(4, 3)) for _ in range(3)]
    for _ in range(12):
        t0 = rng.normal(size=3)
        e0, e1 = rng.normal(size=3), rng.normal(size=3)
        b = rng.uniform(0.1, 0.6)
        c = rng.uniform(0.1, 0.9) * (1.0 - b)
        n = np.cross(e0, e1)
        h = rng.uniform(0.05, 0.5) * rng.choice([-1.0, 1.0])
        p = t0 + b * e0 + c * e1 + h * n / np.linalg.norm(n)
        X.append(np.stack([p, t0 + e0, t0, t0 + e1]))
    Rr = [R.FIXTURE.copy()] + [rng.normal(size=(4, 3)) for _ in range(15)]
    out = {"x": np.stack(X), "r": np.stack(Rr)}
    d2hat, kappa = 1.0, 1.0
    for typ, C, term in ((0, R.C_vf, R.pt_term), (1, R.C_ee, R.ee_term)):
        name = "pt" if typ == 0 else "ee"
        lam, recon, act = [], [], []
        g = {m: [] for m in (0, 1)}
        H = {m: [] for m in (0, 1)}
        en = []
        for x, r in zip(X, Rr):
            e0, e1, e2 = C(*x)
            Q, lm = R.eig_Hl(e0, e1, e2)
            lam.append(lm)
            recon.append(R.QLQinv(Q, lm))
            for m in (0, 1):
                res = term(x, r, d2hat, kappa, contact_psd=m)
                if res is None:
                    g[m].append(np.full(24, np.nan))
                    H[m].append(np.full((3, 12, 12), np.nan))
                else:
                    g[m].append(res[1])
                    H[m].append(np.stack(res[2:]))
            act.append(term(x, r, d2hat, kappa) is not None)
            en.append(R.pt_energy(x, d2hat, kappa) if typ == 0 else R.ee_energy(x, d2hat, kappa))
        out[f"{name}_lam"] = np.stack(lam)
        out[f"{name}_recon"] = np.stack(recon)
        out[f"{name}_active"] = np.array(act)
        out[f"{name}_energy"] = np.array(en)
        for m in (0, 1):
            out[f"{name}_g_mode{m}"] = np.stack(g[m])
            out[f"{name}_H_mode{m}"] = np.stack(H[m])
    np.savez_compressed(os.path.join(HERE, "contact_fixture.npz"), **out)


if __name__ == "__main__":
    main()
