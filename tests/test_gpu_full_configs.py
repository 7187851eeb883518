"""Parity at the full benchmarked configurations, not subsets.

* Lotka-Volterra direct method, all 1,024 trajectories (Philox ids
  0..1023, seed 0, t_end 10, 100 samples), on the thread mapping (the
  lane-group kernel, a warp per trajectory) and on the warp mapping: bit for
  bit against the oracle (samples, status, event counts, firing-sequence
  hashes; final clocks at rtol 1e-12).
* Schlogl tau-leaping, all 262,144 trajectories x 200 samples (t_end 5),
  through the mode-sorted kernel at full pool occupancy -- the kernel and
  launch the benchmark times: bit for bit against the oracle.
* The same Schlogl configuration against the reference's own kernels
  (kernel_P1_P2 + kernel_P3 with CuTauLeaping.run's host loop,
  mod/simulator/cuTauLeaping/cuTauLeaping.py:18-84, compiled for sm_100a
  from the reference's sources): two-sample KS and moment tests at every
  sample time over all 262,144 trajectories of each simulator.

The oracle runs these on all host threads in seconds.
"""

import numpy as np
import pytest

from py_stoch_b200 import networks

pytestmark = pytest.mark.gpu

T_RTOL = 1e-12


def _gpu(torch, model, n, method, mapping, seed):
    from py_stoch_b200.simulator import simulate
    res = simulate(model, n, method=method, mapping=mapping, seed=seed,
                   status=True, events=True, seqhash=True, t_final=True)
    torch.cuda.synchronize()
    out = {k: v.cpu().numpy() for k, v in res.items() if k != '_keepalive'}
    out['seqhash'] = out['seqhash'].view(np.uint64)
    return out


def _compare(g, o):
    np.testing.assert_array_equal(g['status'], o['status'])
    np.testing.assert_array_equal(g['events'], o['events'])
    np.testing.assert_array_equal(g['seqhash'], o['seqhash'])
    np.testing.assert_array_equal(g['samples'], o['samples'])
    np.testing.assert_allclose(g['t_final'], o['t_final'], rtol=T_RTOL,
                               atol=0)


@pytest.mark.parametrize('mapping', ['thread', 'warp'])
def test_lotka_volterra_all_1024(torch_cuda, built_lib, oracle_mod, mapping):
    m = networks.lotka_volterra()
    g = _gpu(torch_cuda, m, 1024, 'direct', mapping, seed=0)
    o = oracle_mod.simulate(m, 1024, 0, seed=0, warp=(mapping == 'warp'))
    _compare(g, o)
    assert (g['status'] == 0).all()
    assert g['events'].sum() > 2e8  # ~3e5 firings per trajectory


def test_schlogl_tau_all_262144(torch_cuda, built_lib, oracle_mod):
    m = networks.schlogl()
    assert m.ita == 200 and float(m.sample_times[-1]) == 5.0
    n = 262144
    g = _gpu(torch_cuda, m, n, 'tau', 'auto', seed=2024)
    o = oracle_mod.simulate(m, n, 1, seed=2024)
    _compare(g, o)
    assert (g['status'] == 0).all()
    final = g['samples'][0, -1]
    # bimodal at t = 5: both branches well populated
    assert 0.2 < (final < 400).mean() < 0.8


def test_schlogl_tau_all_262144_vs_reference_kernels(torch_cuda, built_lib):
    from scipy import stats

    from oracle import ref_harness
    from py_stoch_b200.simulator import simulate
    name = 'schlogl_tl_262144'
    if not ref_harness.available(name):
        pytest.skip('reference kernels not built (oracle/build_ref.py)')
    r = ref_harness.ReferenceRun(name)
    O, _ = r.run()
    ref = O.cpu().numpy()
    m = networks.schlogl(n_samples=r.info['ita'])
    res = simulate(m, r.info['U'], method='tau', seed=99)
    torch_cuda.cuda.synchronize()
    got = res['samples'].cpu().numpy()
    assert ref.shape == got.shape == (1, 200, 262144)
    ita = ref.shape[1]
    alpha = 0.01 / (ita - 1)
    zlim = max(3.0, stats.norm.isf(alpha / 2))
    for f in range(1, ita):
        x = ref[0, f].astype(np.float64)
        y = got[0, f].astype(np.float64)
        p = stats.ks_2samp(x, y).pvalue
        assert p > alpha, (f, p)
        se_m = np.sqrt(x.var() / x.size + y.var() / y.size)
        assert abs(x.mean() - y.mean()) / se_m < zlim, f
        se_v = np.sqrt(2.0 * x.var() ** 2 / (x.size - 1) +
                       2.0 * y.var() ** 2 / (y.size - 1))
        assert abs(x.var() - y.var()) / se_v < zlim, f
