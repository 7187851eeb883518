"""Likelihood-ratio gradients through torch.autograd on the GPU.

Telegraph gene-expression model (G_off, G_on, mRNA, protein; rates 0.5,
0.2, 20, 1, 5, 0.1; t_end = 50, 20 samples).  Checks:

* forward moments against the exact FP64 moment equations;
* the autograd gradient of a weighted sum of protein means and variances
  against the FP64 gradient of those equations (within 4 standard errors of
  the LR estimator);
* the gradient of the mean against central finite differences in log k
  (h = 1e-3, common random numbers), within 2 combined standard errors
  summed in quadrature plus a 1% allowance for the FD truncation.
"""

import numpy as np
import pytest

from py_stoch_b200 import networks

pytestmark = pytest.mark.gpu

U = 1048576  # the benchmarked gradient configuration


@pytest.fixture(scope='module')
def telegraph_run(torch_cuda, built_lib):
    torch = torch_cuda
    from py_stoch_b200.autograd import sampled_moments
    m = networks.telegraph()
    logk = torch.tensor(np.log(m.rate), dtype=torch.float64, device='cuda',
                        requires_grad=True)
    mean, var = sampled_moments(m, logk, U, seed=4)
    return m, logk, mean, var


def test_forward_moments_exact(telegraph_run):
    from oracle import moments
    m, _, mean, var = telegraph_run
    mu, vv = moments.moments(m)
    got_m = mean.detach().cpu().numpy()[0]
    got_v = var.detach().cpu().numpy()[0]
    se = np.sqrt(vv[3] / U) + 1e-9
    z = np.abs(got_m - mu[3]) / se
    assert (z[1:] < 5).all(), z
    rel = np.abs(got_v[5:] - vv[3][5:]) / vv[3][5:]
    assert (rel < 0.03).all(), rel


def test_autograd_matches_fp64_gradient(torch_cuda, telegraph_run):
    from oracle import moments
    from py_stoch_b200.autograd import lr_gradient_with_se
    from py_stoch_b200.simulator import simulate
    torch = torch_cuda
    m, logk, mean, var = telegraph_run
    rng = np.random.default_rng(0)
    wm = rng.normal(size=mean.shape)
    wv = rng.normal(size=var.shape) / 100.0
    loss = (mean * torch.from_numpy(wm).cuda()).sum() + (
        var * torch.from_numpy(wv).cuda()).sum()
    (g,) = torch.autograd.grad(loss, logk, retain_graph=True)
    g = g.cpu().numpy()
    gm, gv = moments.moment_gradients(m)
    want = np.einsum('f,jf->j', wm[0], gm[:, 3]) + np.einsum(
        'f,jf->j', wv[0], gv[:, 3])
    # standard error of the LR estimator from the same trajectories
    res = simulate(m, U, method='direct', seed=4, score=True)
    torch.cuda.synchronize()
    est, se = lr_gradient_with_se(res['samples'].cpu().numpy(),
                                  res['score'].cpu().numpy(), wm, wv)
    np.testing.assert_allclose(g, est, rtol=1e-9, atol=1e-9)
    z = np.abs(g - want) / se
    assert (z < 4).all(), (g, want, se)


def test_autograd_mean_matches_finite_differences(torch_cuda, telegraph_run):
    from py_stoch_b200.autograd import lr_gradient_with_se
    from py_stoch_b200.simulator import simulate
    torch = torch_cuda
    m, logk, mean, _ = telegraph_run
    w = np.zeros(mean.shape)
    w[0, -1] = 1.0  # protein mean at t_end
    (g,) = torch.autograd.grad((mean * torch.from_numpy(w).cuda()).sum(),
                               logk, retain_graph=True)
    g = g.cpu().numpy()
    res = simulate(m, U, method='direct', seed=4, score=True)
    torch.cuda.synchronize()
    _, se_lr = lr_gradient_with_se(res['samples'].cpu().numpy(),
                                   res['score'].cpu().numpy(), w)
    h = 1e-3
    for j in range(m.n_reactions):
        up = m.rate.copy()
        dn = m.rate.copy()
        up[j] *= np.exp(h)
        dn[j] *= np.exp(-h)
        a = simulate(m.with_rates(up), U, seed=4)['samples'][0, -1]
        b = simulate(m.with_rates(dn), U, seed=4)['samples'][0, -1]
        d = (a.double() - b.double()).cpu().numpy() / (2 * h)
        fd, se_fd = d.mean(), d.std(ddof=1) / np.sqrt(U)
        tol = 2 * np.hypot(se_lr[j], se_fd) + 0.01 * abs(fd)
        assert abs(g[j] - fd) < tol, (j, g[j], fd, se_lr[j], se_fd)
