"""The sufficient-statistics kernels of the multi-GPU reduction on one GPU.

* pyst_sample_sums / pyst_moments_from_sums / pyst_score_partials /
  pyst_score_combine equal their NumPy restatements (tests/test_shard_gloo.py
  NumpyOps, which the two- and three-rank gloo tests drive) bit for bit;
* pyst_score_backward equals pyst_score_partials + pyst_score_combine bit
  for bit;
* trajectories split into chunk-aligned shards, each simulated with its own
  global Philox ids, give integer sums that add up to the whole run's and
  partial rows that concatenate to the whole run's, so the reduced moments
  and gradient are the single-GPU ones exactly;
* sharded_sampled_moments on one rank equals sampled_moments, forward and
  backward.
"""

import numpy as np
import pytest

from py_stoch_b200 import networks

pytestmark = pytest.mark.gpu

U = 70001  # not a multiple of the 256-trajectory chunk


@pytest.fixture(scope='module')
def telegraph_scores(torch_cuda, built_lib):
    from py_stoch_b200.simulator import simulate
    m = networks.telegraph(t_end=10.0, n_samples=8)
    res = simulate(m, U, method='direct', seed=17, score=True)
    torch_cuda.cuda.synchronize()
    return m, res


def _weights(m, torch):
    rng = np.random.default_rng(5)
    gm = torch.from_numpy(rng.normal(size=(m.kappa, m.ita))).cuda()
    gv = torch.from_numpy(rng.normal(size=(m.kappa, m.ita)) / 30.0).cuda()
    return gm, gv


def test_kernels_match_numpy_restatement(torch_cuda, telegraph_scores):
    from py_stoch_b200.shard import KernelOps
    from test_shard_gloo import NumpyOps
    torch = torch_cuda
    m, res = telegraph_scores
    k, n = KernelOps(), NumpyOps()
    smp, sc = res['samples'], res['score']
    sums = k.sample_sums(smp)
    np_smp, np_sc = smp.cpu().numpy(), sc.cpu().numpy()
    np.testing.assert_array_equal(sums.cpu().numpy(),
                                  n.sample_sums(np_smp).numpy())
    mean, var = k.moments(sums, U, m.kappa, m.ita)
    nm, nv = n.moments(sums.cpu().numpy(), U, m.kappa, m.ita)
    np.testing.assert_array_equal(mean.cpu().numpy(), nm)
    np.testing.assert_array_equal(var.cpu().numpy(), nv)
    gm, gv = _weights(m, torch)
    part = k.score_partials(smp, sc, mean, var, gm, gv)
    npart = n.score_partials(np_smp, np_sc, nm, nv, gm.cpu().numpy(),
                             gv.cpu().numpy()).numpy()
    np.testing.assert_array_equal(part.cpu().numpy(), npart)
    np.testing.assert_array_equal(k.score_combine(part, U).cpu().numpy(),
                                  n.score_combine(npart, U))


def test_backward_is_partials_plus_combine(torch_cuda, telegraph_scores):
    from py_stoch_b200.autograd import _moments, score_backward
    from py_stoch_b200.shard import KernelOps
    torch = torch_cuda
    m, res = telegraph_scores
    mean, var = _moments(res['samples'])
    x = res['samples'].double()
    np.testing.assert_allclose(mean.cpu().numpy(),
                               x.mean(dim=2).cpu().numpy(), rtol=1e-14)
    np.testing.assert_allclose(var.cpu().numpy(),
                               x.var(dim=2, unbiased=False).cpu().numpy(),
                               rtol=1e-10)
    gm, gv = _weights(m, torch)
    g1 = score_backward(res['samples'], res['score'], mean, var, gm, gv)
    k = KernelOps()
    g2 = k.score_combine(k.score_partials(res['samples'], res['score'], mean,
                                          var, gm, gv), U)
    np.testing.assert_array_equal(g1.cpu().numpy(), g2.cpu().numpy())


@pytest.mark.parametrize('world', [2, 3, 7])
def test_chunk_aligned_shards_reduce_exactly(torch_cuda, telegraph_scores,
                                             world):
    """Each shard simulated on its own (ids start..start+count) reduces to
    the whole run's statistics bit for bit: integer sums add exactly and
    the 256-trajectory partial rows concatenate in order."""
    from py_stoch_b200.shard import SCORE_CHUNK, KernelOps, shard_range
    from py_stoch_b200.simulator import simulate
    torch = torch_cuda
    m, res = telegraph_scores
    k = KernelOps()
    full_sums = k.sample_sums(res['samples'])
    mean, var = k.moments(full_sums, U, m.kappa, m.ita)
    gm, gv = _weights(m, torch)
    full_part = k.score_partials(res['samples'], res['score'], mean, var, gm,
                                 gv)
    sums, parts = 0, []
    for r in range(world):
        start, count = shard_range(U, r, world, SCORE_CHUNK)
        sh = simulate(m, count, method='direct', seed=17, traj_id_base=start,
                      score=True)
        sums = sums + k.sample_sums(sh['samples'])
        parts.append(k.score_partials(sh['samples'], sh['score'], mean, var,
                                      gm, gv))
    torch.cuda.synchronize()
    np.testing.assert_array_equal(sums.cpu().numpy(), full_sums.cpu().numpy())
    allp = torch.cat(parts)
    np.testing.assert_array_equal(allp.cpu().numpy(),
                                  full_part.cpu().numpy())
    np.testing.assert_array_equal(k.score_combine(allp, U).cpu().numpy(),
                                  k.score_combine(full_part, U).cpu().numpy())


def test_sharded_autograd_on_one_rank(torch_cuda, built_lib):
    from py_stoch_b200.autograd import sampled_moments
    from py_stoch_b200.shard import sharded_sampled_moments
    torch = torch_cuda
    m = networks.telegraph(t_end=10.0, n_samples=8)
    outs = []
    for fn in (sampled_moments, sharded_sampled_moments):
        logk = torch.tensor(np.log(m.rate), dtype=torch.float64,
                            device='cuda', requires_grad=True)
        mean, var = fn(m, logk, 20000, seed=2)
        w = torch.linspace(0.1, 1.0, m.ita, dtype=torch.float64,
                           device='cuda')[None]
        (g,) = torch.autograd.grad((mean * w).sum() + (var * w).sum() / 100,
                                   logk)
        outs.append((mean.detach().cpu().numpy(), var.detach().cpu().numpy(),
                     g.cpu().numpy()))
    for a, b in zip(*outs):
        np.testing.assert_array_equal(a, b)
