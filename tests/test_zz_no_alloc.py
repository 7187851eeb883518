"""pyst_score_backward_noalloc: the gradient reduction for callers that
cannot allocate device memory themselves (for example a host runtime whose
own pool already owns the GPU's memory), so cannot pass a workspace.  It
keeps its scratch in a fixed array inside the library; this test checks it
against pyst_score_backward (caller workspace) on two calls in a row, the
second with different, smaller inputs, since the array keeps the previous
call's contents.  The file sorts last so a failure here stops a -x run only
after every other test has run."""

import ctypes as C

import numpy as np
import pytest

from py_stoch_b200 import _lib

pytestmark = pytest.mark.gpu

RTOL = 1e-10  # as in the workspace reduction's test


def _inputs(torch, rng, U, kappa, ita, R):
    smp = rng.integers(0, 500, size=(kappa, ita, U)).astype(np.int32)
    score = rng.normal(size=(U, R))
    mean = smp.mean(axis=2)
    var = smp.var(axis=2)
    gm = rng.normal(size=(kappa, ita))
    gv = rng.normal(size=(kappa, ita))
    return {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in
            dict(smp=smp, score=score, mean=mean, var=var, gm=gm,
                 gv=gv).items()}


def _with_workspace(L, torch, t, U, kappa, ita, R, stream):
    need = C.c_size_t(0)
    assert L.pyst_score_backward_workspace_size(U, R, C.byref(need)) == 0
    ws = torch.empty(need.value // 8 + 1, dtype=torch.float64, device='cuda')
    grad = torch.empty(R, dtype=torch.float64, device='cuda')
    assert L.pyst_score_backward(
        t['smp'].data_ptr(), t['score'].data_ptr(), U, kappa, ita, R,
        t['mean'].data_ptr(), t['var'].data_ptr(), t['gm'].data_ptr(),
        t['gv'].data_ptr(), grad.data_ptr(), ws.data_ptr(), need.value,
        stream) == 0
    return grad


def _no_alloc(L, torch, t, U, kappa, ita, R, stream):
    grad = torch.empty(R, dtype=torch.float64, device='cuda')
    assert L.pyst_score_backward_noalloc(
        t['smp'].data_ptr(), t['score'].data_ptr(), U, kappa, ita, R,
        t['mean'].data_ptr(), t['var'].data_ptr(), t['gm'].data_ptr(),
        t['gv'].data_ptr(), grad.data_ptr(), stream) == 0
    return grad


def test_noalloc_matches_workspace_twice(torch_cuda, built_lib):
    torch = torch_cuda
    L = built_lib
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(12)
    for U, kappa, ita, R in ((70000, 2, 6, 9), (1500, 1, 4, 5)):
        t = _inputs(torch, rng, U, kappa, ita, R)
        want = _with_workspace(L, torch, t, U, kappa, ita, R, stream)
        got = _no_alloc(L, torch, t, U, kappa, ita, R, stream)
        torch.cuda.synchronize()
        np.testing.assert_allclose(got.cpu().numpy(), want.cpu().numpy(),
                                   rtol=RTOL)


def test_noalloc_rejects_oversize(torch_cuda, built_lib):
    # 4097 blocks of 256 trajectories x 32 reactions x 8 bytes > 1 MiB;
    # rejected before any pointer is used
    U = 4097 * 256
    assert built_lib.pyst_score_backward_noalloc(
        8, 8, U, 1, 1, 32, 8, 8, 8, 8, 8, None) == _lib.PYST_EUNSUPPORTED
