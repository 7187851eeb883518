"""A sweep built by TLArgsList.make_list run as one batched launch equals
the reference's per-point loop (one CuTauLeaping().run(args) per point,
examples/schlogl_sim.py:66-80) bit for bit, point for point."""

import copy

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sweeps():
    from py_stoch_b200 import sbml, sim_maker
    sch = sbml.read_sbml_string(sbml.schlogl_sbml())
    lv = sbml.read_sbml_string(sbml.lotka_volterra_sbml())
    tau = sim_maker.TLArgsList.make_list(
        sch, [[250, 400]], [[3e-7], [1e-4], [1e-3, 1.1e-3], [3.5], [1e5],
                            [2e5, 2.1e5]], [0], 5, 20, 1000)
    direct = sim_maker.TLArgsList.make_list(
        lv, [[1000], [900, 1000], [1]], [[10], [0.01, 0.012], [10]], [0, 1],
        1, 11, 300, gillespie=1)
    return tau, direct


def test_sweep_batch_equals_per_point_runs(torch_cuda, built_lib, oracle_mod):
    from py_stoch_b200.batch import Batch
    from py_stoch_b200.model import Model
    from py_stoch_b200.simulator import CuTauLeaping
    tau, direct = _sweeps()
    assert len(tau) == 8 and len(direct) == 4
    for lst in (tau, direct):
        per_point = [CuTauLeaping().run(copy.deepcopy(a)) for a in lst]
        b = Batch.from_tl_args_list(copy.deepcopy(lst))
        b.run(seed=0)
        got = b.results()
        assert len(got) == len(lst)
        for g, want in zip(got, per_point):
            assert g.shape == want.shape
            np.testing.assert_array_equal(g, want)
        # the rounding side effect of calculate_sizes, as in the loop
        rounded = copy.deepcopy(lst)
        Batch.from_tl_args_list(rounded)
        assert [a.U for a in rounded] == [w.shape[2] for w in per_point]
    # and one point against the oracle directly
    a = copy.deepcopy(tau[3])
    CuTauLeaping().calculate_sizes(a)
    o = oracle_mod.simulate(Model.from_tl_args(a), a.U, 1, seed=0)
    b = Batch.from_tl_args_list(copy.deepcopy(tau))
    b.run(seed=0)
    np.testing.assert_array_equal(b.results()[3], o['samples'])


def test_save_batch_round_trip(torch_cuda, built_lib, tmp_path):
    """A batched sweep with in-kernel statistics written with save_batch
    and read back: item table, statistics, status and samples unchanged."""
    from py_stoch_b200 import saver
    from py_stoch_b200.batch import Batch
    tau, _ = _sweeps()
    b = Batch.from_tl_args_list(copy.deepcopy(tau), stats=True)
    b.run(seed=4)
    p = saver.save_batch(b, str(tmp_path / 'sweep.npz'), samples=True)
    d = saver.load_results(p)
    np.testing.assert_array_equal(d['n_traj'], b.n_traj)
    np.testing.assert_array_equal(d['method'], b.methods)
    for i in range(len(tau)):
        np.testing.assert_array_equal(d['item%d_stats' % i],
                                      b.stats(i).cpu().numpy())
        np.testing.assert_array_equal(d['item%d_samples' % i],
                                      b.samples(i).cpu().numpy())
        np.testing.assert_array_equal(d['item%d_status' % i],
                                      b.per_traj('status', i).cpu().numpy())
        x = d['item%d_samples' % i].astype(np.float64)
        np.testing.assert_allclose(d['item%d_stats' % i][..., 0],
                                   x.mean(axis=2), rtol=1e-12)
