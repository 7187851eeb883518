"""The CPU oracle itself: Philox known-answer vectors, the deterministic
elementary functions, the Poisson sampler's distribution, and exact moments
of first-order networks (CPU only)."""

import math

import numpy as np
import pytest
from scipy import stats

from py_stoch_b200 import networks
from py_stoch_b200.model import Model


def test_philox_known_answers(oracle_mod):
    for ctr, key, want in oracle_mod.PHILOX_KAT:
        want = np.array(want, np.uint32)
        np.testing.assert_array_equal(oracle_mod.philox_np([ctr], [key])[0],
                                      want)
        np.testing.assert_array_equal(oracle_mod.philox_c([ctr], [key])[0],
                                      want)
    rng = np.random.default_rng(0)
    c = rng.integers(0, 2**32, (500, 4), dtype=np.uint64).astype(np.uint32)
    k = rng.integers(0, 2**32, (500, 2), dtype=np.uint64).astype(np.uint32)
    np.testing.assert_array_equal(oracle_mod.philox_np(c, k),
                                  oracle_mod.philox_c(c, k))


def test_elementary_functions_accuracy(oracle_mod):
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.uniform(2**-53, 1, 100000),
                        np.exp(rng.uniform(-700, 700, 100000))])
    ulp = np.abs(oracle_mod.math(x, 0) - np.log(x)) / np.spacing(
        np.abs(np.log(x)) + 1e-300)
    assert ulp.max() <= 3
    y = -rng.uniform(0, 700, 100000)
    e = oracle_mod.math(y, 1)
    assert (np.abs(e - np.exp(y)) / np.spacing(np.exp(y))).max() <= 2
    k = np.arange(0, 3000, dtype=np.float64)
    lf = oracle_mod.math(k, 2)
    ref = np.array([math.lgamma(v + 1) for v in k])
    assert np.abs(lf - ref).max() < 1e-9


@pytest.mark.parametrize('lam', [0.3, 4.0, 9.99, 10.0, 37.5, 1000.0, 2.5e6])
def test_poisson_sampler_distribution(oracle_mod, lam):
    n = 200000
    k = oracle_mod.poisson(np.full(n, lam, np.float32), seed=int(lam * 7) + 1)
    assert (k >= 0).all()
    lam32 = float(np.float32(lam))
    se = math.sqrt(lam32 / n)
    assert abs(k.mean() - lam32) < 5 * se
    assert abs(k.var() / lam32 - 1.0) < 5 * math.sqrt(2.0 / n)
    if lam < 50:
        # chi-square goodness of fit on the bulk of the support
        lo, hi = int(max(0, lam - 4 * math.sqrt(lam))), int(
            lam + 4 * math.sqrt(lam)) + 1
        obs = np.array([(k == v).sum() for v in range(lo, hi + 1)])
        exp = np.array([stats.poisson.pmf(v, lam32) for v in
                        range(lo, hi + 1)]) * n
        keep = exp > 20
        chi = ((obs[keep] - exp[keep]) ** 2 / exp[keep]).sum()
        assert stats.chi2.sf(chi, keep.sum() - 1) > 1e-4


def test_first_order_chain_exact_moments(oracle_mod):
    """s1 -> s2 -> s3 (simple_sbml.xml): s1(t) ~ Binomial(N, e^{-c1 t})."""
    N, c1, c2 = 1000, 1.0, 2.0
    pre = [[1, 0], [0, 1], [0, 0]]
    post = [[0, 0], [1, 0], [0, 1]]
    m = Model.mass_action(pre, post, [c1, c2], [N, 0, 0],
                          np.linspace(0, 2, 5).astype(np.float32))
    r = oracle_mod.simulate(m, 8000, 0, seed=3)
    s1 = r['samples'][0].astype(float)
    p = np.exp(-c1 * m.sample_times.astype(float))
    se = np.sqrt(N * p * (1 - p) / 8000) + 1e-12
    assert (np.abs(s1.mean(1) - N * p) < 4.5 * se + 1e-9).all()
    from oracle import moments
    mu, var = moments.moments(m)
    for i in range(3):
        x = r['samples'][i].astype(float)
        sem = np.sqrt(var[i] / 8000) + 1e-9
        assert (np.abs(x.mean(1) - mu[i]) < 4.5 * sem + 1e-6).all()


def test_telegraph_moments_and_tau_vs_ssa(oracle_mod):
    from oracle import moments
    m = networks.telegraph(t_end=20.0, n_samples=6)
    mu, var = moments.moments(m)
    for meth in (0, 1):
        r = oracle_mod.simulate(m, 4000, meth, seed=5 + meth)
        x = r['samples'][0].astype(float)
        sem = np.sqrt(var[3] / 4000) + 1e-9
        z = np.abs(x.mean(1) - mu[3]) / sem
        assert (z[1:] < 5).all(), (meth, z)


def test_schlogl_tau_matches_ssa_distribution(oracle_mod):
    m = networks.schlogl(t_end=5.0, n_samples=6)
    a = oracle_mod.simulate(m, 6000, 0, seed=1)['samples'][0]
    b = oracle_mod.simulate(m, 6000, 1, seed=2)['samples'][0]
    for f in range(1, 6):
        p = stats.ks_2samp(a[f], b[f]).pvalue
        assert p > 0.01 / 5, (f, p)


def test_warp_order_matches_thread_order_distribution(oracle_mod):
    m = networks.lotka_volterra(t_end=1.0, n_samples=5)
    a = oracle_mod.simulate(m, 3000, 0, seed=1)['samples']
    b = oracle_mod.simulate(m, 3000, 0, seed=2, warp=True)['samples']
    for k in range(2):
        for f in range(1, 5):
            assert stats.ks_2samp(a[k, f], b[k, f]).pvalue > 0.01 / 8
