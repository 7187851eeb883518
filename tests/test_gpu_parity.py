"""GPU engine against the CPU oracle, bit for bit, through the C ABI.

Tolerances: integer outputs (samples, status, event counts, firing-sequence
hashes) must be equal; final clocks and likelihood-ratio scores are compared
with rtol 1e-12 (they are in fact bit-identical because every floating-point
operation is explicitly rounded on both sides).
"""

import numpy as np
import pytest

from py_stoch_b200 import networks
from py_stoch_b200.model import Model

pytestmark = pytest.mark.gpu

T_RTOL = 1e-12


def _gpu(torch_cuda, model, n, method, mapping, seed=0, score=False, **kw):
    from py_stoch_b200.simulator import simulate
    res = simulate(model, n, method=method, mapping=mapping, seed=seed,
                   status=True, events=True, seqhash=True, t_final=True,
                   score=score, **kw)
    torch_cuda.cuda.synchronize()
    out = {k: v.cpu().numpy() for k, v in res.items() if k != '_keepalive'}
    out['seqhash'] = out['seqhash'].view(np.uint64)
    return out


def _oracle(oracle_mod, model, n, method, mapping, seed=0, **kw):
    return oracle_mod.simulate(model, n, 0 if method == 'direct' else 1,
                               seed=seed, warp=(mapping == 'warp'), **kw)


def _compare(g, o, score=False):
    np.testing.assert_array_equal(g['status'], o['status'])
    np.testing.assert_array_equal(g['events'], o['events'])
    np.testing.assert_array_equal(g['seqhash'], o['seqhash'])
    np.testing.assert_array_equal(g['samples'], o['samples'])
    np.testing.assert_allclose(g['t_final'], o['t_final'], rtol=T_RTOL,
                               atol=0)
    if score:
        np.testing.assert_allclose(g['score'], o['score'], rtol=T_RTOL,
                                   atol=1e-12)


def test_philox_stream_and_curand(torch_cuda, built_lib, oracle_mod):
    import ctypes as C
    torch = torch_cuda
    n = 4096
    d = torch.empty(4 * n, dtype=torch.int32, device='cuda')
    s = torch.cuda.current_stream().cuda_stream
    assert built_lib.pyst_test_philox(0x1234567890ABCDEF, 77, 5, n,
                                      d.data_ptr(), C.c_void_p(s)) == 0
    got = d.cpu().numpy().view(np.uint32).reshape(n, 4)
    want = oracle_mod.philox_stream(0x1234567890ABCDEF, 77, 5, n)
    np.testing.assert_array_equal(got, want)
    rng = np.random.default_rng(0)
    ck = rng.integers(0, 2**32, size=(n, 6), dtype=np.uint64).astype(
        np.uint32)
    for c, k, _ in oracle_mod.PHILOX_KAT:
        ck[0, :4], ck[0, 4:] = c, k
    dck = torch.from_numpy(ck.view(np.int32)).cuda()
    for use_curand in (0, 1):
        assert built_lib.pyst_test_philox_raw(
            dck.data_ptr(), n, d.data_ptr(), use_curand, C.c_void_p(s)) == 0
        got = d.cpu().numpy().view(np.uint32).reshape(n, 4)
        np.testing.assert_array_equal(
            got, oracle_mod.philox_np(ck[:, :4], ck[:, 4:]))
    for i, (_, _, e) in enumerate(oracle_mod.PHILOX_KAT[-1:]):
        np.testing.assert_array_equal(got[0], np.array(e, np.uint32))


def test_math_bit_exact(torch_cuda, built_lib, oracle_mod):
    import ctypes as C
    torch = torch_cuda
    rng = np.random.default_rng(1)
    xs = {0: np.concatenate([rng.uniform(2**-53, 1, 100000),
                             np.exp(rng.uniform(-700, 700, 100000))]),
          1: -rng.uniform(0, 700, 200000),
          2: np.arange(0, 200000, dtype=np.float64)}
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for which, x in xs.items():
        dx = torch.from_numpy(x).cuda()
        dy = torch.empty_like(dx)
        assert built_lib.pyst_test_math(dx.data_ptr(), x.size, which,
                                        dy.data_ptr(), s) == 0
        np.testing.assert_array_equal(dy.cpu().numpy(),
                                      oracle_mod.math(x, which))


def test_poisson_bit_exact(torch_cuda, built_lib, oracle_mod):
    import ctypes as C
    torch = torch_cuda
    rng = np.random.default_rng(2)
    lam = np.concatenate([
        np.float32([0, -1, 1e-30, 9.999999, 10, 10.000001, 1e9, 2e9]),
        np.exp(rng.uniform(np.log(1e-6), np.log(1e7), 200000)).astype(
            np.float32)])
    dl = torch.from_numpy(lam).cuda()
    dk = torch.empty(lam.size, dtype=torch.int32, device='cuda')
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert built_lib.pyst_test_poisson(dl.data_ptr(), lam.size, 99,
                                       dk.data_ptr(), s) == 0
    got = dk.cpu().numpy()
    np.testing.assert_array_equal(got, oracle_mod.poisson(lam, 99))
    assert got[6] >= 0 and got[7] == -2 and got[0] == 0 and got[1] == 0


@pytest.mark.parametrize('mapping,n', [('thread', 256), ('warp', 64)])
def test_lotka_volterra_direct(torch_cuda, built_lib, oracle_mod, mapping, n):
    """Lotka-Volterra, x0=y0=1000, t_end=10, 100 samples (the CPU-sized
    workload) on a subset of its 1024 trajectories."""
    m = networks.lotka_volterra()
    g = _gpu(torch_cuda, m, n, 'direct', mapping, seed=0)
    o = _oracle(oracle_mod, m, n, 'direct', mapping, seed=0)
    _compare(g, o)
    assert (g['events'] > 100000).all()


@pytest.mark.parametrize('mapping,n', [('thread', 2048), ('warp', 512)])
def test_schlogl_tau(torch_cuda, built_lib, oracle_mod, mapping, n):
    m = networks.schlogl()
    g = _gpu(torch_cuda, m, n, 'tau', mapping, seed=3)
    o = _oracle(oracle_mod, m, n, 'tau', mapping, seed=3)
    _compare(g, o)
    final = g['samples'][0, -1]
    assert (final < 200).any() and (final > 400).any()  # bimodal


@pytest.mark.parametrize('mapping', ['thread', 'warp'])
def test_schlogl_direct(torch_cuda, built_lib, oracle_mod, mapping):
    m = networks.schlogl()
    g = _gpu(torch_cuda, m, 512, 'direct', mapping, seed=5)
    o = _oracle(oracle_mod, m, 512, 'direct', mapping, seed=5)
    _compare(g, o)


@pytest.mark.parametrize('which', ['small', 'limit', 'limit+1', 'large'])
def test_direct_thread_run_sizes(torch_cuda, built_lib, oracle_mod, which):
    """Direct-method thread runs on both sides of the small-run limit: up to
    16 trajectories per SM (the device's SM count x 16) each trajectory gets
    a whole warp (the lane tree for packable models), above it one thread
    per trajectory."""
    sms = torch_cuda.cuda.get_device_properties(0).multi_processor_count
    limit = sms * 16
    n = {'small': 100, 'limit': limit, 'limit+1': limit + 1,
         'large': limit + 1700}[which]
    m = networks.schlogl(t_end=1.0, n_samples=21)
    g = _gpu(torch_cuda, m, n, 'direct', 'thread', seed=3)
    o = _oracle(oracle_mod, m, n, 'direct', 'thread', seed=3)
    _compare(g, o)


@pytest.mark.parametrize('mapping', ['thread', 'warp'])
@pytest.mark.parametrize('method', ['direct', 'tau'])
def test_telegraph_score(torch_cuda, built_lib, oracle_mod, mapping, method):
    m = networks.telegraph(t_end=10.0)
    g = _gpu(torch_cuda, m, 512, method, mapping, seed=11, score=True)
    o = _oracle(oracle_mod, m, 512, method, mapping, seed=11)
    _compare(g, o, score=True)


def _small_synthetic(k=6):
    out = []
    for m in networks.synthetic_networks(k, seed=5, t_range=(0.002, 0.01)):
        out.append(m)
    return out


@pytest.mark.parametrize('method', ['direct', 'tau'])
def test_synthetic_networks(torch_cuda, built_lib, oracle_mod, method):
    for i, m in enumerate(_small_synthetic()):
        for mp in ('warp', 'thread'):
            g = _gpu(torch_cuda, m, 64, method, mp, seed=i,
                     step_budget=200000)
            o = _oracle(oracle_mod, m, 64, method, mp, seed=i,
                        step_budget=200000)
            _compare(g, o)


def test_small_thread_networks(torch_cuda, built_lib, oracle_mod):
    """Random networks with R <= 32 through every thread-kernel size."""
    for R, seed in ((3, 1), (7, 2), (12, 3), (20, 4), (32, 5)):
        ms = networks.synthetic_networks(1, seed=seed, s_range=(3, 12),
                                         r_range=(R, R),
                                         t_range=(0.01, 0.05))
        m = ms[0]
        for method in ('direct', 'tau'):
            g = _gpu(torch_cuda, m, 96, method, 'thread', seed=seed,
                     step_budget=100000)
            o = _oracle(oracle_mod, m, 96, method, 'thread', seed=seed,
                        step_budget=100000)
            _compare(g, o)


def test_edge_cases(torch_cuda, built_lib, oracle_mod):
    # absorbing from the start: degradation only with x0 = 0
    m = Model.mass_action([[1]], [[0]], [1.0], [0], [0, 1, 2])
    for mp in ('thread', 'warp'):
        g = _gpu(torch_cuda, m, 33, 'direct', mp)
        assert (g['status'] == 1).all() and (g['samples'] == 0).all()
        _compare(g, _oracle(oracle_mod, m, 33, 'direct', mp))
    # one trajectory, one sample, sizes not a multiple of the block
    lv = networks.lotka_volterra(t_end=0.5, n_samples=1)
    for n in (1, 130):
        for mp in ('thread', 'warp'):
            g = _gpu(torch_cuda, lv, n, 'direct', mp, seed=9)
            _compare(g, _oracle(oracle_mod, lv, n, 'direct', mp, seed=9))
    # step budget: status 2 and -1 fill
    g = _gpu(torch_cuda, networks.lotka_volterra(), 40, 'direct', 'thread',
             step_budget=1000)
    o = _oracle(oracle_mod, networks.lotka_volterra(), 40, 'direct',
                'thread', step_budget=1000)
    _compare(g, o)
    assert (g['status'] == 2).all() and (g['samples'][:, -1] == -1).all()
    # int32 overflow of a pure birth process
    b = Model.mass_action([[1]], [[2]], [1.0], [2147483000], [0, 10])
    for method in ('direct', 'tau'):
        g = _gpu(torch_cuda, b, 8, method, 'thread', seed=1)
        o = _oracle(oracle_mod, b, 8, method, 'thread', seed=1)
        _compare(g, o)
        assert (g['status'] == 3).all()


def test_drop_in_classes(torch_cuda, built_lib, oracle_mod):
    from py_stoch_b200 import sbml, sim_maker
    from py_stoch_b200.simulator import CuGillespie, CuTauLeaping
    m = sbml.read_sbml_string(sbml.schlogl_sbml())
    lst = sim_maker.TLArgsList.make_list(
        m, [[250]], [[3e-7], [1e-4], [1e-3, 1.1e-3], [3.5], [1e5], [2e5]],
        [0], 5, 20, 1000)
    for args in lst:
        O = CuTauLeaping().run(args)
        assert args.U == 1024 and O.shape == (1, 20, 1024)
        model = Model.from_tl_args(args)
        o = oracle_mod.simulate(model, args.U, 1, seed=0)
        np.testing.assert_array_equal(O, o['samples'])
    g_lst = sim_maker.TLArgsList.make_list(
        m, [[250]], [[3e-7], [1e-4], [1e-3], [3.5], [1e5], [2e5]], [0], 5,
        20, 100, gillespie=1)
    O = CuTauLeaping().run(g_lst[0])
    o = oracle_mod.simulate(Model.from_tl_args(g_lst[0]), g_lst[0].U, 0,
                            seed=0)
    np.testing.assert_array_equal(O, o['samples'])
    O2 = CuGillespie().run(g_lst[0])
    np.testing.assert_array_equal(O2, o['samples'])


def test_score_backward(torch_cuda, built_lib):
    import ctypes as C
    torch = torch_cuda
    rng = np.random.default_rng(4)
    U, kappa, ita, R = 1000, 2, 5, 7
    smp = rng.integers(0, 100, size=(kappa, ita, U)).astype(np.int32)
    score = rng.normal(size=(U, R))
    mean = smp.mean(axis=2)
    var = smp.var(axis=2)
    gm = rng.normal(size=(kappa, ita))
    gv = rng.normal(size=(kappa, ita))
    d = (smp - mean[..., None]).astype(np.float64)
    h = np.einsum('kf,kfu->u', gm, d) + np.einsum(
        'kf,kfu->u', gv, d * d - var[..., None])
    want = h @ score / U
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in
         dict(smp=smp, score=score, mean=mean, var=var, gm=gm,
              gv=gv).items()}
    ws_bytes = C.c_size_t(0)
    built_lib.pyst_score_backward_workspace_size(U, R, C.byref(ws_bytes))
    ws = torch.empty(ws_bytes.value // 8 + 1, dtype=torch.float64,
                     device='cuda')
    grad = torch.empty(R, dtype=torch.float64, device='cuda')
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = built_lib.pyst_score_backward(
        t['smp'].data_ptr(), t['score'].data_ptr(), U, kappa, ita, R,
        t['mean'].data_ptr(), t['var'].data_ptr(), t['gm'].data_ptr(),
        t['gv'].data_ptr(), grad.data_ptr(), ws.data_ptr(), ws_bytes.value, s)
    assert rc == 0
    np.testing.assert_allclose(grad.cpu().numpy(), want, rtol=1e-10)


@pytest.mark.parametrize('score', [True, False])
def test_batch_matches_single_runs(torch_cuda, built_lib, oracle_mod, score):
    """Uneven models, both methods and both mappings in one persistent
    launch; every item equals its oracle re-run."""
    from py_stoch_b200.batch import Batch
    models = ([networks.lotka_volterra(t_end=0.2, n_samples=7),
               networks.schlogl(t_end=1.0, n_samples=11),
               networks.telegraph(t_end=5.0)] + _small_synthetic(5))
    methods = ['direct', 'tau'] * 4
    n_traj = [40, 100, 64, 33, 64, 17, 50, 64]
    b = Batch(models, n_traj, method=methods, score=score, seqhash=True,
              t_final=True)
    b.run(seed=21, step_budget=200000)
    torch_cuda.cuda.synchronize()
    for i, m in enumerate(models):
        warp = int(b.mappings[i]) == 2
        o = oracle_mod.simulate(m, n_traj[i], 0 if methods[i] == 'direct'
                                else 1, seed=21,
                                traj_id_base=int(b.traj_id_base[i]),
                                warp=warp, step_budget=200000)
        np.testing.assert_array_equal(b.samples(i).cpu().numpy(),
                                      o['samples'])
        for k in ('status', 'events'):
            np.testing.assert_array_equal(b.per_traj(k, i).cpu().numpy(),
                                          o[k])
        np.testing.assert_array_equal(
            b.per_traj('seqhash', i).cpu().numpy().view(np.uint64),
            o['seqhash'])
        np.testing.assert_allclose(b.per_traj('t_final', i).cpu().numpy(),
                                   o['t_final'], rtol=T_RTOL)
        if score:
            np.testing.assert_allclose(b.score(i).cpu().numpy(), o['score'],
                                       rtol=T_RTOL, atol=1e-12)


@pytest.mark.parametrize('score', [False, True])
def test_sorted_scheduler_matches_unsorted(torch_cuda, built_lib, oracle_mod,
                                           score):
    """The mode-sorted block scheduler only reorders work: every output
    equals the one-trajectory-per-thread loop and the oracle."""
    m = networks.schlogl(t_end=2.0, n_samples=50)
    n = 3000  # more trajectories than one block so slots are refilled
    a = _gpu(torch_cuda, m, n, 'tau', 'thread', seed=8, score=score)
    b = _gpu(torch_cuda, m, n, 'tau', 'thread', seed=8, score=score,
             sorted_blocks=False)
    for k in ('samples', 'status', 'events', 'seqhash', 't_final'):
        np.testing.assert_array_equal(a[k], b[k])
    if score:
        np.testing.assert_array_equal(a['score'], b['score'])
    _compare(a, _oracle(oracle_mod, m, n, 'tau', 'thread', seed=8),
             score=score)


@pytest.mark.parametrize('mapping', ['thread', 'warp'])
def test_split_models_match_unsplit(torch_cuda, built_lib, oracle_mod,
                                    mapping):
    """Models split into chunks that different blocks run (and whose
    statistics the last chunk's block reduces) give the unsplit batch's
    outputs bit for bit, and the oracle's."""
    from py_stoch_b200.batch import Batch
    models = [networks.schlogl(t_end=1.0, n_samples=9),
              networks.telegraph(t_end=3.0, n_samples=6),
              networks.lotka_volterra(t_end=0.2, n_samples=5)]
    n_traj = [300, 257, 70]
    outs = []
    for chunk in (0, 128, 7):
        b = Batch(models, n_traj, method=['tau', 'direct', 'tau'],
                  mapping=mapping, score=True, stats=True, jacobian=True,
                  seqhash=True, chunk=chunk)
        if chunk == 7:
            assert b.n_items > 60
        b.run(seed=13)
        torch_cuda.cuda.synchronize()
        outs.append({k: v.cpu().numpy() for k, v in b.out.items()})
        if chunk == 128:
            for i, m in enumerate(models):
                o = oracle_mod.simulate(
                    m, n_traj[i], 1 if i != 1 else 0, seed=13,
                    traj_id_base=int(b.traj_id_base[i]),
                    warp=mapping == 'warp')
                np.testing.assert_array_equal(b.samples(i).cpu().numpy(),
                                              o['samples'])
    for other in outs[1:]:
        for k, v in outs[0].items():
            np.testing.assert_array_equal(other[k], v, err_msg=k)


def test_batch_stats_and_jacobian(torch_cuda, built_lib):
    """In-kernel per-item statistics and score Jacobians equal the same
    reductions done in NumPy on the batch's own samples and scores."""
    from py_stoch_b200.batch import Batch
    models = [networks.lotka_volterra(t_end=0.5, n_samples=9),
              networks.schlogl(t_end=1.0, n_samples=12),
              networks.telegraph(t_end=5.0, n_samples=7)]
    b = Batch(models, [200, 300, 129], method=['tau', 'tau', 'direct'],
              score=True, stats=True, jacobian=True)
    b.run(seed=3)
    torch_cuda.cuda.synchronize()
    for i in range(len(models)):
        x = b.samples(i).cpu().numpy().astype(np.float64)
        s = b.score(i).cpu().numpy()
        st = b.stats(i).cpu().numpy()
        jac = b.jacobian(i).cpu().numpy()
        m = x.mean(axis=2)
        v = (x * x).mean(axis=2) - m * m
        np.testing.assert_allclose(st[..., 0], m, rtol=1e-12)
        np.testing.assert_allclose(st[..., 1], v, rtol=1e-9, atol=1e-9)
        cov = (x[:, :-1] * x[:, 1:]).mean(axis=2) - m[:, :-1] * m[:, 1:]
        den = v[:, :-1] * v[:, 1:]
        corr = np.where(den > 0, cov / np.sqrt(np.where(den > 0, den, 1)), 0)
        np.testing.assert_allclose(st[:, :-1, 2], corr, rtol=1e-7, atol=1e-9)
        d = x - m[..., None]
        want_m = np.einsum('kfu,uj->kfj', d, s) / x.shape[2]
        want_v = np.einsum('kfu,uj->kfj', d * d - v[..., None], s) / x.shape[2]
        np.testing.assert_allclose(jac[0], want_m, rtol=1e-8, atol=1e-8)
        np.testing.assert_allclose(jac[1], want_v, rtol=1e-8, atol=1e-6)


def test_small_runs_at_the_packing_boundary(torch_cuda, built_lib,
                                            oracle_mod):
    """Small direct-method runs (a warp per trajectory) of models on both
    sides of the packed-descriptor limits: the host picks the lane tree for
    packable ones and the lockstep lane groups otherwise; both equal the
    oracle.  Also every lane-tree depth: R = 1 and 2 (5 levels), 3 and 4
    (3 levels), 5 to 8 (2 levels), each with 2, 4 and 8 species registers
    (S = 2, 3-4, 5-8)."""
    from py_stoch_b200 import _lib
    t = np.linspace(0, 0.05, 6).astype(np.float32)
    models = []
    for delta in (15, 16):
        models.append(Model.mass_action([[1], [0]], [[1 + delta], [0]],
                                        [2.0], [100, 5], t))
    for order in (3, 4):
        models.append(Model.mass_action([[order], [0]], [[order - 1], [1]],
                                        [1e-3], [60, 0], t))
    models.append(Model.mass_action([[1], [1], [1]], [[0], [0], [2]], [1.0],
                                    [90, 90, 90], t))
    for R in (1, 2, 3, 4, 5, 8):
        for k, sr in enumerate(((2, 2), (3, 4), (5, 8))):
            models += networks.synthetic_networks(
                1, seed=40 + 3 * R + k, s_range=sr, r_range=(R, R),
                t_range=(0.002, 0.01))
    kinds = set()
    for i, m in enumerate(models):
        kinds.add(built_lib.pyst_test_model_packable(m.blob().ctypes.data))
        g = _gpu(torch_cuda, m, 64, 'direct', 'thread', seed=i,
                 step_budget=200000)
        o = _oracle(oracle_mod, m, 64, 'direct', 'thread', seed=i,
                    step_budget=200000)
        _compare(g, o)
    assert kinds == {0, 1}


@pytest.mark.parametrize('R', [2, 3, 4, 5, 6, 7, 8, 16, 32])
def test_exact_reaction_counts(torch_cuda, built_lib, oracle_mod, R):
    """Packable models with 2 to 8 reactions run thread-mapped kernels with
    the reaction count fixed at compile time (the direct method and the
    simple tau loop, with and without scores), and the mode-sorted kernel
    does so when R equals its register-array size (4, 8, 16, 32): each
    equals the oracle.  2,500 trajectories put the direct method above the
    small-run limit of the lane tree."""
    # seeds whose networks take both SSA steps and leaps (oracle, 100
    # trajectories: 150-520 leaps and 1,200-1,800 SSA steps each)
    seed = {2: 69, 3: 76, 4: 78, 5: 66, 6: 70, 7: 69, 8: 71, 16: 106,
            32: 123}[R]
    m = networks.synthetic_networks(1, seed=seed, s_range=(3, 8),
                                    r_range=(R, R), t_range=(0.002, 0.02),
                                    x0_max=100000, k_range=(1e-5, 1e1))[0]
    n = 2500
    for method, kw in (('direct', {}), ('tau', {}),
                       ('tau', {'sorted_blocks': False})):
        g = _gpu(torch_cuda, m, n, method, 'thread', seed=R,
                 step_budget=100000, **kw)
        o = _oracle(oracle_mod, m, n, method, 'thread', seed=R,
                    step_budget=100000)
        _compare(g, o)
    if R <= 8:
        # with scores: the direct method's exact-R kernels, and the sorted
        # kernel's score flavour (exact R for R = 4 and 8)
        for method in ('direct', 'tau'):
            g = _gpu(torch_cuda, m, n, method, 'thread', seed=R + 1,
                     step_budget=100000, score=True)
            o = _oracle(oracle_mod, m, n, method, 'thread', seed=R + 1,
                        step_budget=100000)
            _compare(g, o, score=True)


def test_batch_exact_reaction_counts(torch_cuda, built_lib, oracle_mod):
    """Batched thread-mapped items of 2 to 8 reactions run with the reaction
    count fixed at compile time; each item equals the oracle (tau-leaping
    and the direct method, with scores)."""
    from py_stoch_b200.batch import Batch
    seeds = {2: 69, 3: 76, 4: 78, 5: 66, 6: 70, 7: 69, 8: 71}
    models = [networks.synthetic_networks(
        1, seed=s, s_range=(3, 8), r_range=(R, R), t_range=(0.002, 0.02),
        x0_max=100000, k_range=(1e-5, 1e1))[0] for R, s in seeds.items()]
    n, budget = 96, 100000
    for method in ('tau', 'direct'):
        b = Batch(models, n, method=method, mapping='thread', score=True,
                  small_batch_warps=False)
        b.run(seed=5, step_budget=budget)
        torch_cuda.cuda.synchronize()
        for i, m in enumerate(models):
            o = oracle_mod.simulate(m, n, 1 if method == 'tau' else 0,
                                    seed=5,
                                    traj_id_base=int(b.traj_id_base[i]),
                                    step_budget=budget)
            np.testing.assert_array_equal(b.samples(i).cpu().numpy(),
                                          o['samples'])
            np.testing.assert_array_equal(
                b.per_traj('status', i).cpu().numpy(), o['status'])
            np.testing.assert_array_equal(
                b.per_traj('events', i).cpu().numpy(), o['events'])
            np.testing.assert_allclose(b.score(i).cpu().numpy(), o['score'],
                                       rtol=T_RTOL, atol=1e-12)
