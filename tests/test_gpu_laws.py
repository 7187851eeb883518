"""General kinetic laws on the GPU: every engine (thread mapping, the
mode-sorted tau-leaping scheduler, the simple tau loop, warp mapping, the
batched launch) against the CPU oracle, bit for bit: samples, status, event
counts and the firing-sequence hash; final clocks at rtol 1e-12.
"""

import numpy as np
import pytest

from py_stoch_b200 import kinetic
from py_stoch_b200.model import Model

pytestmark = pytest.mark.gpu
T_RTOL = 1e-12


def _law_model(laws, pre, post, rate, x0, t_end=4.0, n_samples=9):
    """Model whose reaction j uses the law string laws[j] (None: mass
    action with rate[j]); parameter_k of a law is rate[k]."""
    pre = np.asarray(pre)
    S, R = pre.shape
    progs = []
    for j, text in enumerate(laws):
        if text is None:
            progs.append(None)
        else:
            code, consts, _ = kinetic.compile_law(text, S, list(rate))
            progs.append((code, consts))
    order = np.where([[l is None for l in laws]] * S, pre, 0)
    times = np.linspace(0.0, t_end, n_samples).astype(np.float32)
    return Model(order, pre, np.asarray(post) - pre,
                 [r if l is None else 0.0 for r, l in zip(rate, laws)], x0,
                 times, np.arange(S), laws=progs)


def _models():
    # birth-death with the non-polynomial death law k1 * |x|
    bd = _law_model([None, 'parameter_1 * abs(species_0)'],
                    [[0, 1]], [[1, 0]], [2000.0, 0.5], [0])
    # enzyme-like conversion with saturation, C integer division and a
    # square root; a catalyst species keeps the reactions alive
    mm = _law_model(
        ['parameter_0 * species_0 / (parameter_1 + species_0)',
         'species_1 / 3 * parameter_2 + sqrt(species_2)',
         None],
        [[1, 0, 0], [0, 1, 0], [0, 0, 1]],
        [[0, 1, 0], [1, 0, 0], [0, 0, 1]],
        [4000.0, 5000.0, 0.7], [30000, 2000, 4])
    return {'birth_death_abs': bd, 'saturating': mm}


def _gpu(torch_cuda, model, n, method, mapping, seed=0, **kw):
    from py_stoch_b200.simulator import simulate
    res = simulate(model, n, method=method, mapping=mapping, seed=seed,
                   status=True, events=True, seqhash=True, t_final=True, **kw)
    torch_cuda.cuda.synchronize()
    out = {k: v.cpu().numpy() for k, v in res.items() if k != '_keepalive'}
    out['seqhash'] = out['seqhash'].view(np.uint64)
    return out


def _compare(g, o):
    np.testing.assert_array_equal(g['status'], o['status'])
    np.testing.assert_array_equal(g['events'], o['events'])
    np.testing.assert_array_equal(g['seqhash'], o['seqhash'])
    np.testing.assert_array_equal(g['samples'], o['samples'])
    np.testing.assert_allclose(g['t_final'], o['t_final'], rtol=T_RTOL,
                               atol=0)


@pytest.mark.parametrize('name', ['birth_death_abs', 'saturating'])
@pytest.mark.parametrize('method,mapping,sorted_blocks', [
    ('direct', 'thread', True), ('direct', 'warp', True),
    ('tau', 'thread', True), ('tau', 'thread', False), ('tau', 'warp', True)])
def test_laws_bit_exact(torch_cuda, built_lib, oracle_mod, name, method,
                        mapping, sorted_blocks):
    m = _models()[name]
    n = 600
    g = _gpu(torch_cuda, m, n, method, mapping, seed=3,
             sorted_blocks=sorted_blocks)
    o = oracle_mod.simulate(m, n, 0 if method == 'direct' else 1, seed=3,
                            warp=(mapping == 'warp'))
    assert (o['status'] == 0).all()
    _compare(g, o)


@pytest.mark.parametrize('method,mapping', [('direct', 'thread'),
                                            ('tau', 'thread'),
                                            ('direct', 'warp')])
def test_invalid_law_status(torch_cuda, built_lib, oracle_mod, method,
                            mapping):
    """A law that goes negative stops the trajectory with PYST_TRAJ_RATE
    (7) on both sides."""
    m = _law_model([None, 'parameter_1 * (species_0 - 5)'],
                   [[0, 1]], [[1, 0]], [20.0, 0.5], [0])
    g = _gpu(torch_cuda, m, 64, method, mapping, seed=1)
    o = oracle_mod.simulate(m, 64, 0 if method == 'direct' else 1, seed=1,
                            warp=(mapping == 'warp'))
    assert (o['status'] == 7).all()
    _compare(g, o)


def test_laws_in_a_batch(torch_cuda, built_lib, oracle_mod):
    from py_stoch_b200.batch import Batch
    ms = list(_models().values())
    b = Batch(ms, 200, method='tau', device='cuda', seqhash=True)
    b.run(seed=9)
    torch_cuda.cuda.synchronize()
    for i, m in enumerate(ms):
        o = oracle_mod.simulate(m, 200, 1, seed=9, traj_id_base=i * 200)
        np.testing.assert_array_equal(b.samples(i).cpu().numpy(),
                                      o['samples'])


def test_scores_refused_for_laws(torch_cuda, built_lib):
    from py_stoch_b200.simulator import simulate
    with pytest.raises(ValueError):
        simulate(_models()['saturating'], 32, score=True)


def test_batched_scores_refused_for_laws(torch_cuda, built_lib):
    """A scored batched launch (the C ABI, bypassing the Python guard) does
    not simulate an item whose model has general kinetic laws: its
    trajectories read PYST_TRAJ_UNSUPPORTED with samples -1 and NaN scores,
    while the mass-action item of the same launch runs normally."""
    import ctypes as C

    from py_stoch_b200 import _lib, networks
    from py_stoch_b200.batch import Batch
    torch = torch_cuda
    law = _models()['saturating']
    ma = networks.telegraph(t_end=2.0, n_samples=5)
    b = Batch([ma, law], 64, method='direct', order='given')
    R = max(ma.n_reactions, law.n_reactions)
    score = torch.full((2 * 64 * R,), 7.0, dtype=torch.float64,
                       device='cuda')
    o = b.out
    outs = _lib.Outputs(o['samples'].data_ptr(), 0, o['status'].data_ptr(),
                        o['events'].data_ptr(), 0, 0, score.data_ptr(), 0, 0)
    r = _lib.RunDesc(0, 0, 5, 0, 0, 100, 63, 0, 0, 0)
    L = built_lib
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.pyst_batch_run(b.d_blobs.data_ptr(), b.d_items.data_ptr(), 2,
                            C.byref(b.limits), C.byref(r), C.byref(outs),
                            b.workspace.data_ptr(), b.workspace.numel(),
                            s) == 0
    torch.cuda.synchronize()
    st = b.per_traj('status', 1).cpu().numpy()
    assert (st == _lib.TRAJ_UNSUPPORTED).all()
    assert (b.samples(1).cpu().numpy() == -1).all()
    sc = score.cpu().numpy()
    a = int(b.score_offset[1])
    assert np.isnan(sc[a:a + 64 * law.n_reactions]).all()
    assert (b.per_traj('status', 0).cpu().numpy() == 0).all()
    assert np.isfinite(sc[:64 * ma.n_reactions]).all()
