"""The model-staging timeout, made to run out on purpose.

Every kernel stages its model blob into shared memory with one bulk-async
copy and waits on an mbarrier with a bounded number of polls.  The test hook
pyst_test_set_staging_polls(0) makes each of those waits give up at once
(the copy itself still lands: the block drains it, bounded, before it moves
on).  Every kernel family must then mark each of its trajectories
PYST_TRAJ_STAGING and return, and the GPU context must stay usable: a run
after the default is restored equals the oracle bit for bit.  No GPU fault
or hang is involved; the wait simply ends early.  The reference has no such
path (its host loop, cuTauLeaping.py:49, has no bound at all).
"""

import numpy as np
import pytest

from py_stoch_b200 import _lib, networks

pytestmark = pytest.mark.gpu


def _status(res):
    return res['status'].cpu().numpy()


def test_staging_timeout_marks_every_trajectory(torch_cuda, built_lib,
                                                oracle_mod):
    from py_stoch_b200.batch import Batch
    from py_stoch_b200.simulator import simulate
    torch = torch_cuda
    L = built_lib
    lv = networks.lotka_volterra(t_end=0.5, n_samples=5)
    sch = networks.schlogl(t_end=1.0, n_samples=11)
    big = networks.synthetic_networks(1, seed=3, r_range=(40, 40),
                                      t_range=(0.01, 0.02))[0]
    cases = [
        # (model, n, method, keyword arguments): the kernel each reaches
        (lv, 64, 'direct', {}),                           # lane groups
        (lv, 5000, 'direct', {}),                         # thread, queue
        (sch, 3000, 'tau', {}),                           # mode-sorted
        (sch, 700, 'tau', {'sorted_blocks': False}),      # simple tau loop
        (sch, 300, 'tau', {'mapping': 'warp'}),           # warp mapping
        (big, 200, 'direct', {'mapping': 'thread'}),      # large-R thread
    ]
    L.pyst_test_set_staging_polls(0)
    try:
        for m, n, meth, kw in cases:
            res = simulate(m, n, method=meth, seed=1, status=True, **kw)
            torch.cuda.synchronize()
            st = _status(res)
            assert (st == _lib.TRAJ_STAGING).all(), (m.name, meth, kw,
                                                     np.unique(st))
            assert res.error_count() == n
        b = Batch([lv, sch, big], [40, 100, 30], method=['direct', 'tau',
                                                         'tau'])
        b.run(seed=2)
        torch.cuda.synchronize()
        assert (b.out['status'].cpu().numpy() == _lib.TRAJ_STAGING).all()
    finally:
        L.pyst_test_set_staging_polls(-1)
    assert L.pyst_test_set_staging_polls(-1) == 1 << 22  # the default
    # the context is intact: the same runs now complete and match the oracle
    for m, n, meth, kw in cases[:3]:
        res = simulate(m, n, method=meth, seed=1, status=True, events=True,
                       **kw)
        torch.cuda.synchronize()
        o = oracle_mod.simulate(m, n, 0 if meth == 'direct' else 1, seed=1)
        np.testing.assert_array_equal(res['samples'].cpu().numpy(),
                                      o['samples'])
        np.testing.assert_array_equal(_status(res), o['status'])
