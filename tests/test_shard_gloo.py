"""Multi-rank runs of the sharded path on CPU (gloo):

* each rank runs its shard of trajectory ids through the oracle, the shards
  reassemble into the single-process result bit for bit, and the
  timing/count reduction takes the max and the sum;
* the sufficient-statistics reduction (py_stoch_b200.shard.ShardReducer:
  int64 all-reduce of exact sample sums, all-gather of the gradient's
  256-trajectory partial rows) on 2 and 3 ranks gives the single-process
  moments and likelihood-ratio gradient bit for bit.  The per-rank
  operations here are NumPy restatements of the CUDA kernels (same
  operations in the same order); the GPU tests check those kernels against
  the same restatements.
"""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from py_stoch_b200.shard import SCORE_CHUNK, shard_items, shard_range


def test_shard_range_covers_everything():
    for align in (1, 256):
        for n in (0, 1, 7, 1000, 1024, 262144, 1048577):
            for w in (1, 2, 3, 8):
                got = [shard_range(n, r, w, align) for r in range(w)]
                assert sum(c for _, c in got) == n
                pos = 0
                for s, c in got:
                    assert s == pos and s % align == 0 or c == 0
                    pos += c


class NumpyOps(object):
    """NumPy restatement of the per-rank kernels of the reduction
    (k_sample_sums, k_moments_from_sums, k_score_partial, k_score_final in
    py_stoch_b200/csrc/pyst_k_misc.cu): the same IEEE operations in the
    same order."""

    def sample_sums(self, samples):
        import torch
        x = np.asarray(samples, dtype=np.int64)
        k, f, _ = x.shape
        x2 = x * x
        out = np.stack([x.sum(axis=2), (x2 >> 32).sum(axis=2),
                        (x2 & 0xFFFFFFFF).sum(axis=2)], axis=-1)
        return torch.from_numpy(out.reshape(k * f, 3).copy())

    def moments(self, sums, n_total, kappa, ita):
        s = np.asarray(sums).astype(np.float64)
        m = s[:, 0] / float(n_total)
        x2 = s[:, 1] * 4294967296.0 + s[:, 2]
        v = x2 / float(n_total) - m * m
        return m.reshape(kappa, ita), v.reshape(kappa, ita)

    def score_partials(self, samples, score, mean, var, gmean, gvar):
        import torch
        x = np.asarray(samples, dtype=np.float64)
        kappa, ita, U = x.shape
        h = np.zeros(U)
        for kf in range(kappa * ita):
            k, f = divmod(kf, ita)
            d = x[k, f] - mean[k, f]
            h = h + gmean[k, f] * d
            if gvar is not None:
                h = h + gvar[k, f] * (d * d - var[k, f])
        nb = -(-U // SCORE_CHUNK)
        hp = np.zeros(nb * SCORE_CHUNK)
        hp[:U] = h
        sp = np.zeros((nb * SCORE_CHUNK, score.shape[1]))
        sp[:U] = score
        hp = hp.reshape(nb, SCORE_CHUNK)
        sp = sp.reshape(nb, SCORE_CHUNK, -1)
        acc = np.zeros((nb, score.shape[1]))
        for q in range(SCORE_CHUNK):  # padded terms add +0.0 exactly
            acc = acc + hp[:, q, None] * sp[:, q]
        return torch.from_numpy(acc)

    def score_combine(self, parts, n_total):
        p = np.asarray(parts)
        acc = np.zeros(p.shape[1])
        for b in range(p.shape[0]):
            acc = acc + p[b]
        return acc / float(n_total)


def _telegraph_small():
    from py_stoch_b200 import networks
    return networks.telegraph(t_end=5.0, n_samples=6)


GM_SEED = 41
N_TOTAL = 1000  # not a multiple of 256: the last rank's range ends short


def _weights(m):
    rng = np.random.default_rng(GM_SEED)
    return (rng.normal(size=(m.kappa, m.ita)),
            rng.normal(size=(m.kappa, m.ita)) / 50.0)


def _reduce_worker(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist

    from oracle import oracle
    from py_stoch_b200.shard import ShardReducer
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    m = _telegraph_small()
    counts = [shard_range(N_TOTAL, r, world, SCORE_CHUNK)[1]
              for r in range(world)]
    start, count = shard_range(N_TOTAL, rank, world, SCORE_CHUNK)
    r = oracle.simulate(m, count, 0, seed=3, traj_id_base=start, threads=2)
    red = ShardReducer(counts, ops=NumpyOps())
    mean, var = red.moments(r['samples'])
    gm, gv = _weights(m)
    grad = red.gradient(r['samples'], r['score'], mean, var, gm, gv)
    np.save(os.path.join(out_dir, 'mv_%d.npy' % rank), np.stack([mean, var]))
    np.save(os.path.join(out_dir, 'grad_%d.npy' % rank), np.asarray(grad))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize('world', [2, 3])
def test_sufficient_statistics_reduce_bit_exact(tmp_path, oracle_mod, world):
    from py_stoch_b200.shard import ShardReducer
    ctx = mp.get_context('spawn')
    port = _free_port()
    procs = [ctx.Process(target=_reduce_worker,
                         args=(r, world, port, str(tmp_path)))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    m = _telegraph_small()
    full = oracle_mod.simulate(m, N_TOTAL, 0, seed=3)
    red = ShardReducer([N_TOTAL], ops=NumpyOps())
    mean, var = red.moments(full['samples'])
    gm, gv = _weights(m)
    grad = np.asarray(red.gradient(full['samples'], full['score'], mean, var,
                                   gm, gv))
    for r in range(world):
        mv = np.load(tmp_path / ('mv_%d.npy' % r))
        np.testing.assert_array_equal(mv[0], mean)
        np.testing.assert_array_equal(mv[1], var)
        np.testing.assert_array_equal(np.load(tmp_path / ('grad_%d.npy' % r)),
                                      grad)
    # and the reduction is the LR gradient of sum(gm * mean + gv * var)
    x = full['samples'].astype(np.float64)
    d = x - x.mean(axis=2, keepdims=True)
    h = np.einsum('kf,kfu->u', gm, d) + np.einsum(
        'kf,kfu->u', gv, d * d - x.var(axis=2)[..., None])
    np.testing.assert_allclose(grad, h @ full['score'] / N_TOTAL, rtol=1e-9,
                               atol=1e-9)
    np.testing.assert_allclose(mean, x.mean(axis=2), rtol=1e-15)


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist

    from oracle import oracle
    from py_stoch_b200 import networks
    from py_stoch_b200.shard import reduce_time_and_count, shard_range
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    m = networks.schlogl(t_end=1.0, n_samples=11)
    n_total = 301
    start, count = shard_range(n_total, rank, world)
    r = oracle.simulate(m, count, 1, seed=9, traj_id_base=start, threads=2)
    np.save(os.path.join(out_dir, 'samples_%d.npy' % rank), r['samples'])
    np.save(os.path.join(out_dir, 'events_%d.npy' % rank), r['events'])
    ms, ev = reduce_time_and_count(10.0 * (rank + 1), r['events'].sum())
    np.save(os.path.join(out_dir, 'reduced_%d.npy' % rank),
            np.array([ms, ev]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_shards_reassemble(tmp_path, oracle_mod):
    from py_stoch_b200 import networks
    world = 2
    ctx = mp.get_context('spawn')
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, str(tmp_path)))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    full = oracle_mod.simulate(networks.schlogl(t_end=1.0, n_samples=11), 301,
                               1, seed=9)
    parts = [np.load(tmp_path / ('samples_%d.npy' % r)) for r in range(world)]
    np.testing.assert_array_equal(np.concatenate(parts, axis=2),
                                  full['samples'])
    ev = sum(np.load(tmp_path / ('events_%d.npy' % r)).sum()
             for r in range(world))
    for r in range(world):
        ms, tot = np.load(tmp_path / ('reduced_%d.npy' % r))
        assert ms == 20.0 and tot == ev == full['events'].sum()


def test_shard_items_offsets():
    items = list(range(10))
    a, sa = shard_items(items, 0, 3)
    b, sb = shard_items(items, 1, 3)
    c, sc = shard_items(items, 2, 3)
    assert a + b + c == items and (sa, sb, sc) == (0, 4, 7)
