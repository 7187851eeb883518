"""Sharding trajectories (or models) across ranks, one process per GPU, and
the reduction of their sufficient statistics.

Trajectories are independent and every random number is keyed by the
global trajectory id, so a shard is a contiguous id range: the simulation
has no collective and its results do not depend on how the work is split.
The reference's only cross-trajectory reduction is the termination sum
``gpuarray.sum(d_Q)`` (``mod/simulator/cuTauLeaping/cuTauLeaping.py:72``);
here the sample moments and their likelihood-ratio gradients are reduced
across ranks instead, so one parameter set (or one item of a sweep) can be
split over GPUs and still give one gradient:

* forward: each rank sums its samples exactly in integers
  (``pyst_sample_sums``: sum x, and x^2 in two 32-bit halves); one
  ``all_reduce(SUM)`` of those int64 sums is exact and order-free, and
  every rank turns the totals into the mean and variance
  (``pyst_moments_from_sums``);
* backward: each rank computes the gradient's partial sums, one row per
  256 trajectories (``pyst_score_partials``); the rows are all-gathered and
  summed in global trajectory order (``pyst_score_combine``).

With shard ranges that start on multiples of 256 (``shard_range(...,
align=SCORE_CHUNK)``) the moments and the gradient are bit-identical to a
single GPU running every trajectory, for any number of ranks.  An
all-reduce of floating-point partial gradients would not be: its summation
order follows the ring.  Volumes are KB (C4: 4096 rows x 6 doubles).

The per-rank operations default to the CUDA kernels (:class:`KernelOps`);
the collectives are ``torch.distributed`` (NCCL between GPUs; gloo in the
CPU tests, which pass NumPy restatements of the same operations).
"""

import ctypes as C

import numpy as np

from . import _lib

SCORE_CHUNK = _lib.SCORE_CHUNK


def shard_range(n_total, rank, world, align=1):
    """(first id, count) of rank's contiguous share of n_total items.  Every
    range starts on a multiple of ``align`` (the last one may end short)."""
    n_total, world, align = int(n_total), int(world), int(align)
    units = -(-n_total // align)
    base, extra = divmod(units, world)
    u0 = rank * base + min(rank, extra)
    u1 = u0 + base + (1 if rank < extra else 0)
    start = min(u0 * align, n_total)
    return start, min(u1 * align, n_total) - start


def shard_items(items, rank, world):
    start, count = shard_range(len(items), rank, world)
    return items[start:start + count], start


def _dist():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist
    return None


def reduce_time_and_count(ms, count, device=None):
    """(max of ms over ranks, sum of count over ranks); identity when
    torch.distributed is not initialised."""
    import torch
    dist = _dist()
    if dist is None:
        return float(ms), float(count)
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    c = torch.tensor([float(count)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t.item()), float(c.item())


class KernelOps(object):
    """The per-rank operations of the reduction, on the GPU (C ABI)."""

    @staticmethod
    def _stream(t):
        import torch
        return C.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)

    def sample_sums(self, samples):
        """int64 [kappa*ita, 3]: sum x, sum (x^2 >> 32), sum (x^2 & 2^32-1)
        over the trajectories of ``samples`` [kappa, ita, U] int32."""
        import torch
        kappa, ita, U = samples.shape
        out = torch.empty((kappa * ita, 3), dtype=torch.int64,
                          device=samples.device)
        _lib.check(_lib.lib().pyst_sample_sums(
            samples.data_ptr(), U, U, kappa, ita, out.data_ptr(),
            self._stream(samples)), 'pyst_sample_sums')
        return out

    def moments(self, sums, n_total, kappa, ita):
        import torch
        mean = torch.empty((kappa, ita), dtype=torch.float64,
                           device=sums.device)
        var = torch.empty_like(mean)
        _lib.check(_lib.lib().pyst_moments_from_sums(
            sums.data_ptr(), kappa * ita, int(n_total), mean.data_ptr(),
            var.data_ptr(), self._stream(sums)), 'pyst_moments_from_sums')
        return mean, var

    def score_partials(self, samples, score, mean, var, gmean, gvar):
        """float64 [ceil(U / 256), R] partial gradient sums."""
        import torch
        kappa, ita, U = samples.shape
        R = score.shape[1]
        part = torch.empty((-(-U // SCORE_CHUNK), R), dtype=torch.float64,
                           device=samples.device)
        gm = gmean.to(torch.float64).contiguous()
        gv = None if gvar is None else gvar.to(torch.float64).contiguous()
        _lib.check(_lib.lib().pyst_score_partials(
            samples.data_ptr(), score.data_ptr(), U, kappa, ita, R,
            mean.data_ptr(), var.data_ptr(), gm.data_ptr(),
            gv.data_ptr() if gv is not None else None, part.data_ptr(),
            self._stream(samples)), 'pyst_score_partials')
        return part

    def score_combine(self, parts, n_total):
        import torch
        B, R = parts.shape
        grad = torch.empty(R, dtype=torch.float64, device=parts.device)
        _lib.check(_lib.lib().pyst_score_combine(
            parts.contiguous().data_ptr(), B, R, int(n_total),
            grad.data_ptr(), self._stream(parts)), 'pyst_score_combine')
        return grad


def allreduce_sums(sums, group=None):
    """Sum int64 sufficient statistics over ranks (exact, order-free)."""
    dist = _dist()
    if dist is not None:
        dist.all_reduce(sums, op=dist.ReduceOp.SUM, group=group)
    return sums


def gather_rows(rows, counts, group=None):
    """Concatenate every rank's ``rows`` [n_r, R] in rank order; ``counts``
    lists n_r for every rank (the all-gather pads to the largest)."""
    import torch
    dist = _dist()
    if dist is None:
        return rows
    world = dist.get_world_size(group)
    width = rows.shape[1]
    n_max = max(int(c) for c in counts)
    pad = torch.zeros((n_max, width), dtype=rows.dtype, device=rows.device)
    pad[:rows.shape[0]] = rows
    bufs = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(bufs, pad, group=group)
    return torch.cat([b[:int(c)] for b, c in zip(bufs, counts)], dim=0)


class ShardReducer(object):
    """Moments and their gradients over trajectories split across ranks.

    ``counts`` lists every rank's trajectory count (ranges contiguous in
    rank order, each starting on a multiple of SCORE_CHUNK); ``ops``
    supplies the per-rank operations (default: the CUDA kernels)."""

    def __init__(self, counts, ops=None, group=None):
        self.counts = [int(c) for c in counts]
        self.n_total = sum(self.counts)
        self.ops = ops if ops is not None else KernelOps()
        self.group = group

    def moments(self, samples):
        kappa, ita, _ = samples.shape
        sums = allreduce_sums(self.ops.sample_sums(samples), self.group)
        return self.ops.moments(sums, self.n_total, kappa, ita)

    def gradient(self, samples, score, mean, var, gmean, gvar=None):
        part = self.ops.score_partials(samples, score, mean, var, gmean,
                                       gvar)
        rows = [-(-c // SCORE_CHUNK) for c in self.counts]
        allp = gather_rows(part, rows, self.group)
        return self.ops.score_combine(allp, self.n_total)


def _sharded_function():
    import torch

    from .simulator import simulate

    class ShardedMoments(torch.autograd.Function):
        """(log_rates [R]) -> (mean, var) [kappa, ita] of all ranks'
        trajectories; each rank simulates its own id range."""

        @staticmethod
        def forward(ctx, log_rates, model, n_total, seed, method, group):
            dist = _dist()
            rank = dist.get_rank(group) if dist is not None else 0
            world = dist.get_world_size(group) if dist is not None else 1
            counts = [shard_range(n_total, r, world, SCORE_CHUNK)[1]
                      for r in range(world)]
            start, count = shard_range(n_total, rank, world, SCORE_CHUNK)
            rates = np.exp(log_rates.detach().double().cpu().numpy())
            m = model.with_rates(rates)
            res = simulate(m, count, method=method, seed=seed,
                           traj_id_base=start, device=log_rates.device,
                           score=True, status=True, events=False)
            bad = torch.tensor([res.error_count()], dtype=torch.int64,
                               device=log_rates.device)
            if dist is not None:
                dist.all_reduce(bad, op=dist.ReduceOp.SUM, group=group)
            if int(bad.item()):
                raise RuntimeError('%d trajectories failed' % int(bad.item()))
            red = ShardReducer(counts, group=group)
            mean, var = red.moments(res['samples'])
            ctx.save_for_backward(res['samples'], res['score'], mean, var)
            ctx.red = red
            return mean, var

        @staticmethod
        def backward(ctx, grad_mean, grad_var):
            samples, score, mean, var = ctx.saved_tensors
            if grad_mean is None:
                grad_mean = torch.zeros_like(mean)
            g = ctx.red.gradient(samples, score, mean, var, grad_mean,
                                 grad_var)
            return g, None, None, None, None, None

    return ShardedMoments


_SHARDED = None


def sharded_sampled_moments(model, log_rates, n_total, seed=0,
                            method='direct', group=None):
    """Differentiable (mean, var) [kappa, ita] of ``n_total`` trajectories
    split across the ranks of ``group`` (every rank calls it with the same
    arguments; ``log_rates`` on this rank's GPU).  The results and the
    gradient are the same on every rank and equal, bit for bit, those of
    one GPU running all trajectories."""
    global _SHARDED
    if _SHARDED is None:
        _SHARDED = _sharded_function()
    return _SHARDED.apply(log_rates, model, int(n_total), int(seed), method,
                          group)
