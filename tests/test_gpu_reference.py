"""The engine against the reference's own kernels (compiled for sm_100a by
oracle/build_ref.py, replayed by oracle/ref_harness.py), at the
distribution level: the reference draws from curand MRG32k3a, the engine
from Philox, so trajectories differ but their laws must agree.

Bar: a two-sample KS test on every species at every sample time with
Bonferroni-corrected p > 0.01, and means and variances within 3 standard
errors (the threshold raised to the Bonferroni z when more than a handful
of comparisons are made).  Skipped when oracle/_ref was not built.
"""

import numpy as np
import pytest
from scipy import stats

pytestmark = pytest.mark.gpu


def _ref(name):
    from oracle import ref_harness
    if not ref_harness.available(name):
        pytest.skip('reference kernels not built (oracle/build_ref.py)')
    r = ref_harness.ReferenceRun(name)
    O, rounds = r.run()
    return r, O.cpu().numpy()


def _compare(a, b, skip_first=True):
    """a, b: [kappa, ita, n] samples of two simulators."""
    kappa, ita = a.shape[:2]
    tests = [(k, f) for k in range(kappa) for f in range(ita)
             if not (skip_first and f == 0)]
    n_tests = len(tests)
    alpha = 0.01 / n_tests
    zlim = max(3.0, stats.norm.isf(alpha / 2))
    worst_p, worst_z = 1.0, 0.0
    for k, f in tests:
        x = a[k, f].astype(np.float64)
        y = b[k, f].astype(np.float64)
        if x.std() == 0 and y.std() == 0:
            assert x.mean() == y.mean()
            continue
        p = stats.ks_2samp(x, y).pvalue
        worst_p = min(worst_p, p)
        assert p > alpha, (k, f, p)
        se_m = np.sqrt(x.var() / x.size + y.var() / y.size)
        zm = abs(x.mean() - y.mean()) / se_m
        se_v = np.sqrt(2.0 * x.var() ** 2 / (x.size - 1) +
                       2.0 * y.var() ** 2 / (y.size - 1))
        zv = abs(x.var() - y.var()) / se_v
        worst_z = max(worst_z, zm, zv)
        assert zm < zlim and zv < zlim, (k, f, zm, zv, zlim)
    return worst_p, worst_z


@pytest.mark.parametrize('name,method', [('schlogl_tl_8192', 'tau'),
                                         ('schlogl_ssa_8192', 'direct')])
def test_schlogl_matches_reference_kernels(torch_cuda, built_lib, name,
                                           method):
    from py_stoch_b200 import networks
    from py_stoch_b200.simulator import simulate
    r, O = _ref(name)
    m = networks.schlogl(n_samples=r.info['ita'])
    res = simulate(m, r.info['U'], method=method, seed=123)
    torch_cuda.cuda.synchronize()
    _compare(O, res['samples'].cpu().numpy())


@pytest.mark.parametrize('name', ['lv_ssa_1024', 'lv_gillespie_1024'])
def test_lotka_volterra_matches_reference_kernels(torch_cuda, built_lib,
                                                  name):
    from py_stoch_b200 import networks
    from py_stoch_b200.simulator import simulate
    r, O = _ref(name)
    m = networks.lotka_volterra()
    res = simulate(m, r.info['U'], method='direct', seed=321)
    torch_cuda.cuda.synchronize()
    _compare(O, res['samples'].cpu().numpy())
