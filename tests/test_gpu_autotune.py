"""The autotuner on the GPU.

* A mixed batch with reaction-count buckets on both sides of the register
  limit (R <= 32 and R > 32): every bucket is measured with each mapping it
  allows, the choice is cached on disk and reloaded without re-measuring,
  and the batch run with the tuned mappings equals the oracle item by item.
* A bucket forced to the warp mapping through the cache runs warp-mapped and
  still equals the oracle (the warp-order summation mode).
* The mode-sorted scheduler's geometry search: the chosen geometry, and
  every candidate, give the default run's results bit for bit.
"""

import numpy as np
import pytest

from py_stoch_b200 import networks

pytestmark = pytest.mark.gpu


def _mixed_models():
    small = networks.synthetic_networks(4, seed=21, s_range=(5, 12),
                                        r_range=(8, 24),
                                        t_range=(0.005, 0.02))
    large = networks.synthetic_networks(3, seed=22, s_range=(10, 40),
                                        r_range=(40, 90),
                                        t_range=(0.005, 0.02))
    return small + large


def _check_batch(torch, oracle_mod, b, models, n_traj, budget):
    torch.cuda.synchronize()
    for i, m in enumerate(models):
        warp = int(b.mappings[i]) == 2
        o = oracle_mod.simulate(m, n_traj, 1, seed=31,
                                traj_id_base=int(b.traj_id_base[i]),
                                warp=warp, step_budget=budget)
        np.testing.assert_array_equal(b.samples(i).cpu().numpy(),
                                      o['samples'])
        np.testing.assert_array_equal(b.per_traj('status', i).cpu().numpy(),
                                      o['status'])


def test_tune_mixed_buckets_cache_and_parity(torch_cuda, built_lib,
                                             oracle_mod, tmp_path):
    from py_stoch_b200 import _lib
    from py_stoch_b200.autotune import Autotuner, bucket
    from py_stoch_b200.batch import Batch
    models = _mixed_models()
    path = str(tmp_path / 'tune.json')
    tuner = Autotuner(path=path, sample=8, n_traj=32, budget=500)
    tuner.tune(models, 'tau')
    keys = {bucket(m, 'tau') for m in models}
    assert any('/R32/' in k or '/R8/' in k for k in keys)
    assert any('/R64/' in k or '/R128/' in k for k in keys)
    for k in keys:
        ent = tuner.table[k]
        assert ent['mapping'] in ('thread', 'warp')
        assert set(ent['events_per_s']) == {'thread', 'warp'}
        assert all(v > 0 for v in ent['events_per_s'].values())
    # the cache reloads without measuring again
    again = Autotuner(path=path, sample=8, n_traj=32, budget=500)
    again.tune(models, 'tau')
    assert again.timings == {} and again.table == tuner.table
    bs = tuner.tune_block(models, 'tau')
    assert bs in (64, 128)
    budget = 100000
    b = Batch(models, 48, method='tau', mapping_fn=tuner.mapping_fn,
              small_batch_warps=False)
    b.run(seed=31, step_budget=budget, block_size=bs)
    assert list(b.mappings) == [tuner.mapping(m, 'tau') for m in models]
    _check_batch(torch_cuda, oracle_mod, b, models, 48, budget)
    # force one bucket to the warp mapping through the cache
    k = bucket(models[0], 'tau')
    again.table[k] = dict(again.table[k], mapping='warp')
    b2 = Batch(models, 48, method='tau', mapping_fn=again.mapping_fn,
               small_batch_warps=False)
    assert int(b2.mappings[0]) == _lib.MAP_WARP
    b2.run(seed=31, step_budget=budget)
    _check_batch(torch_cuda, oracle_mod, b2, models, 48, budget)
    # a batch too small to fill the GPU runs its large networks warp-mapped
    b3 = Batch(models, 48, method='tau', mapping_fn=tuner.mapping_fn)
    assert [int(x) == _lib.MAP_WARP for x in b3.mappings] == [
        m.n_reactions > _lib.THREAD_MAX_REACTIONS or
        tuner.mapping(m, 'tau') == _lib.MAP_WARP for m in models]
    b3.run(seed=31, step_budget=budget)
    _check_batch(torch_cuda, oracle_mod, b3, models, 48, budget)


def test_sorted_geometry_search(torch_cuda, built_lib, oracle_mod, tmp_path):
    from py_stoch_b200.autotune import Autotuner
    from py_stoch_b200.simulator import simulate
    m = networks.schlogl(t_end=1.0, n_samples=21)
    n = 20000
    tuner = Autotuner(path=str(tmp_path / 'tune.json'))
    g = tuner.tune_geometry(m, n, 'tau')
    assert set(g) == {'round_ssa', 'round_leap', 'pool_slots',
                      'sorted_block'}
    assert len(tuner.timings) == 1
    assert tuner.geometry(m, n, 'tau') == g
    ref = simulate(m, n, method='tau', seed=6, seqhash=True)
    torch_cuda.cuda.synchronize()
    want = {k: ref[k].cpu().numpy() for k in ('samples', 'seqhash',
                                               'events')}
    o = oracle_mod.simulate(m, n, 1, seed=6)
    np.testing.assert_array_equal(want['samples'], o['samples'])
    for geo in (g, {'round_ssa': 7, 'round_leap': 1, 'pool_slots': 1,
                    'sorted_block': 96},
                {'round_ssa': 64, 'round_leap': 4, 'pool_slots': 2,
                 'sorted_block': 448}):
        got = simulate(m, n, method='tau', seed=6, seqhash=True,
                       geometry=geo)
        torch_cuda.cuda.synchronize()
        for k, v in want.items():
            np.testing.assert_array_equal(got[k].cpu().numpy(), v)
