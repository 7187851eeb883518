"""Likelihood-ratio gradients of sampled summary statistics.

For a mass-action network the log-likelihood of a trajectory on [0, T] is
``sum_events log a_{j_e} - int_0^T a_0 dt`` and, since ``a_j`` is linear in
its rate ``k_j``, its derivative in ``log k_j`` is exactly

    s_j = N_j - int_0^T a_j(x(t)) dt

(N_j = firings of reaction j).  The forward kernels accumulate ``s`` per
trajectory next to the simulation (integer state untouched, no relaxation).
For a statistic ``E[f(X)]`` the gradient is ``E[(f - b) s]``; with the
baseline ``b`` the sample mean this gives the gradients of the sample mean
and variance used here:

    d mean = E[(O - m) s],   d var = E[((O - m)^2 - var) s].

:class:`SampledMoments` is a ``torch.autograd.Function``: forward simulates
and returns the per-sample mean and variance ``[kappa, ita]`` (float64);
backward reduces ``grad_mean * (O - m) + grad_var * ((O - m)^2 - var)``
against the scores on the GPU (``pyst_score_backward``).  Tau-leaping runs
give the corresponding Poisson-leap score (exact for the leap likelihood,
an approximation of the SSA gradient).
"""

import ctypes as C

import numpy as np

from . import _lib
from .simulator import _torch, simulate


def _moments(samples):
    """Population mean and variance [kappa, ita] of ``samples`` [kappa, ita,
    U] from exact integer sums on the GPU (the same kernels, and so the same
    bits, as the multi-GPU reduction in :mod:`py_stoch_b200.shard`)."""
    from .shard import KernelOps
    kappa, ita, U = samples.shape
    ops = KernelOps()
    return ops.moments(ops.sample_sums(samples), U, kappa, ita)


def score_backward(samples, score, mean, var, grad_mean, grad_var,
                   stream=None):
    """grad[j] = (1/U) sum_u h_u score[u, j] on the GPU (deterministic)."""
    torch = _torch()
    L = _lib.lib()
    kappa, ita, U = samples.shape
    R = score.shape[1]
    dev = samples.device
    need = C.c_size_t(0)
    _lib.check(L.pyst_score_backward_workspace_size(U, R, C.byref(need)),
               'pyst_score_backward_workspace_size')
    ws = torch.empty(need.value // 8 + 1, dtype=torch.float64, device=dev)
    grad = torch.empty(R, dtype=torch.float64, device=dev)
    gm = grad_mean.to(torch.float64).contiguous()
    gv = None if grad_var is None else grad_var.to(torch.float64).contiguous()
    if stream is None:
        stream = torch.cuda.current_stream(dev)
    _lib.check(L.pyst_score_backward(
        samples.data_ptr(), score.data_ptr(), U, kappa, ita, R,
        mean.data_ptr(), var.data_ptr(), gm.data_ptr(),
        gv.data_ptr() if gv is not None else None, grad.data_ptr(),
        ws.data_ptr(), need.value, C.c_void_p(stream.cuda_stream)),
        'pyst_score_backward')
    return grad


def _function():
    torch = _torch()

    class SampledMoments(torch.autograd.Function):
        """(log_rates [R]) -> (mean [kappa, ita], var [kappa, ita])."""

        @staticmethod
        def forward(ctx, log_rates, model, n_traj, seed, method, traj_id_base,
                    ssa_fallback_steps):
            rates = np.exp(log_rates.detach().double().cpu().numpy())
            m = model.with_rates(rates)
            res = simulate(m, n_traj, method=method, seed=seed,
                           traj_id_base=traj_id_base, device=log_rates.device
                           if log_rates.is_cuda else None, score=True,
                           status=True, events=False,
                           ssa_fallback_steps=ssa_fallback_steps)
            if res.error_count():
                raise RuntimeError('%d trajectories failed'
                                   % res.error_count())
            mean, var = _moments(res['samples'])
            ctx.save_for_backward(res['samples'], res['score'], mean, var)
            ctx.device = log_rates.device
            return mean, var

        @staticmethod
        def backward(ctx, grad_mean, grad_var):
            samples, score, mean, var = ctx.saved_tensors
            if grad_mean is None:
                grad_mean = torch.zeros_like(mean)
            g = score_backward(samples, score, mean, var, grad_mean, grad_var)
            return (g.to(ctx.device), None, None, None, None, None, None)

    return SampledMoments


_FN = None


def sampled_moments(model, log_rates, n_traj, seed=0, method='direct',
                    traj_id_base=0, ssa_fallback_steps=100):
    """Differentiable (mean, var) of the sampled species at every sample
    time, as a function of ``log_rates`` (tensor [R] on a CUDA device)."""
    global _FN
    if _FN is None:
        _FN = _function()
    return _FN.apply(log_rates, model, int(n_traj), int(seed), method,
                     int(traj_id_base), int(ssa_fallback_steps))


def lr_gradient_with_se(samples, score, weights_mean, weights_var=None):
    """Per-trajectory contributions of the LR gradient of
    sum(w_m * mean + w_v * var) and their standard error (NumPy, for
    checks).  Returns (grad [R], se [R])."""
    x = samples.astype(np.float64)
    m = x.mean(axis=2)
    v = (x * x).mean(axis=2) - m * m
    d = x - m[..., None]
    h = np.einsum('kf,kfu->u', weights_mean, d)
    if weights_var is not None:
        h = h + np.einsum('kf,kfu->u', weights_var, d * d - v[..., None])
    contrib = h[:, None] * score
    U = x.shape[2]
    return contrib.mean(axis=0), contrib.std(axis=0, ddof=1) / np.sqrt(U)
