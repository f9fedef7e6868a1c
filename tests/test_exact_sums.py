"""The oracle's reproducible arithmetic, on the CPU: exact summation, the shared logarithm
and the rank-one form of the contact terms.

The CUDA product and the oracle sum every reduction of the step exactly and round once, and
compute the barrier's logarithm from IEEE-exact operations; with those two pieces, whole
time steps agree bit for bit (tests/test_gpu_parity.py).  Here each piece is pinned on its
own: the exact sum against math.fsum (the correctly rounded sum), the logarithm against
math.log within 1 ulp, and the rank-one contact terms against the reference's matrix form
(contact_gh, itself pinned to the golden fixtures) within 1e-12."""
import math

import numpy as np
import pytest

import oracle
from abd_warp_b200.params import SimParams


def _ulps(a, b):
    return abs(a - b) / math.ulp(b) if b != 0 else abs(a)


def test_exact_sum_is_the_correctly_rounded_sum():
    rng = np.random.default_rng(5)
    for trial in range(200):
        n = int(rng.integers(1, 400))
        mag = 10.0 ** rng.uniform(-40, 30, size=n)
        v = rng.choice([-1.0, 1.0], size=n) * mag * rng.random(n)
        if trial % 3 == 0:  # heavy cancellation
            v = np.concatenate([v, -v[: n // 2] * (1 + 1e-15)])
        assert oracle.exact_sum(v) == math.fsum(v)
        assert oracle.exact_sum(rng.permutation(v)) == oracle.exact_sum(v)


def test_exact_sum_edge_cases():
    assert oracle.exact_sum([]) == 0.0
    assert oracle.exact_sum([1e300 * 0.0]) == 0.0
    assert oracle.exact_sum([2.0 ** -1074]) == 0.0  # below the grid: dropped
    assert math.isnan(oracle.exact_sum([1.0, float("nan")]))
    assert oracle.exact_sum([1.0, float("inf")]) == float("inf")
    assert math.isnan(oracle.exact_sum([float("inf"), float("-inf")]))
    assert oracle.exact_sum([2.0 ** 120]) == 2.0 ** 120
    assert math.isnan(oracle.exact_sum([2.0 ** 130]))  # out of range is reported, not wrapped
    # ties round to even
    assert oracle.exact_sum([1.0, 2.0 ** -53]) == 1.0
    assert oracle.exact_sum([1.0 + 2.0 ** -52, 2.0 ** -53]) == 1.0 + 2.0 ** -51
    assert oracle.exact_sum([1.0, 2.0 ** -53, 2.0 ** -150]) == 1.0 + 2.0 ** -52


def test_shared_log_accuracy():
    rng = np.random.default_rng(9)
    xs = np.concatenate([10.0 ** rng.uniform(-300, 300, 3000), 1.0 + rng.normal(size=2000) * 1e-3,
                         rng.uniform(0.5, 2.0, 2000), [1.0, 2.0, 0.5, 1e-6, 1e-12, 5e-324, 1.7e308]])
    worst = max(_ulps(oracle.abd_log(float(x)), math.log(x)) for x in xs if x != 1.0)
    assert worst <= 1.0, worst
    assert oracle.abd_log(1.0) == 0.0
    assert oracle.abd_log(0.0) == float("-inf")
    assert math.isnan(oracle.abd_log(-1.0))


@pytest.mark.parametrize("mode", [0, 1])
def test_rank_one_terms_match_matrix_form(mode):
    prm = SimParams(dhat=1.0, kappa=1.0, contact_psd=mode)
    rng = np.random.default_rng(13)
    n_act = 0
    for _ in range(300):
        X, r = rng.normal(size=(4, 3)), rng.normal(size=(4, 3))
        for typ in (0, 1):
            a, d2, g, Hi, Hj, Hij = oracle.contact_gh(typ, X, r, prm)
            b, Tij, Tii, Tjj, tg = oracle.contact_terms(typ, X, r, prm)
            assert a == b
            if not a:
                continue
            n_act += 1
            scale = max(np.abs(Hi).max(), np.abs(Hj).max(), np.abs(Hij).max())
            for got, want in ((Tii, Hi), (Tjj, Hj), (Tij, Hij)):
                assert np.abs(got - want).max() <= 1e-11 * scale
            assert np.abs(tg - g).max() <= 1e-11 * max(np.abs(g).max(), 1e-300)
    assert n_act > 50
