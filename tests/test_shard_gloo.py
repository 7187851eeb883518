"""World-size-2 runs of the sharded path on CPU (gloo): each rank runs its
shard of trajectory ids through the oracle, the shards reassemble into the
single-process result bit for bit, and the timing/count reduction takes
the max and the sum."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from py_stoch_b200.shard import shard_items, shard_range


def test_shard_range_covers_everything():
    for n in (0, 1, 7, 1024, 262144):
        for w in (1, 2, 3, 8):
            got = [shard_range(n, r, w) for r in range(w)]
            assert sum(c for _, c in got) == n
            pos = 0
            for s, c in got:
                assert s == pos
                pos += c


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
