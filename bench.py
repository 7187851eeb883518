"""Benchmark: SSA reaction events/s (and trajectories/s) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload NAME]

Default workload (the one the headline metric is quoted on that fits one
GPU): plain cuTauLeaping on the bistable Schlogl model, 262,144
trajectories, X0=250, eps=0.03, n_c=10, 100-step SSA fallback, t_end=5 with
200 samples.  A step is one full simulation of that workload (one kernel
launch).  Events are reaction firings (SSA steps plus the Poisson firings of
each leap).  At N GPUs every rank simulates its own 262,144 trajectories
(distinct Philox ids; weak scaling, no data-path collective) and the value
is all events over the slowest rank's device time.

One JSON line on rank 0.  ``--impl reference`` times the reference's own
implementation of the path: its CUDA kernels (kernel_P1_P2 / kernel_P3, or
kernel_Gillespie), compiled for sm_100a from the reference's sources by
oracle/build_ref.py, driven by a replay of CuTauLeaping.run's host round
loop (oracle/ref_harness.py).  Where those kernels are not built for the
workload it falls back to the CPU oracle port on all host cores over a
bounded sample.
"""

import argparse
import json
import os
import subprocess
import sys
import threading
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import numpy as np  # noqa: E402

METRIC = 'SSA reaction events/s'
UNIT = 'events/s'


def workloads():
    from py_stoch_b200 import networks
    return {
        'schlogl_tau': dict(
            model=networks.schlogl(), n=262144, method='tau',
            desc='plain cuTauLeaping, Schlogl (c1=3e-7,c2=1e-4,c3=1e-3,'
                 'c4=3.5,A=1e5,B=2e5), X0=250, eps=0.03, n_c=10, 100-step '
                 'SSA fallback, 262144 trajectories, t_end=5, 200 samples',
            cpu_pilot=1024, ref_config='schlogl_tl_262144',
            # from one ncu capture of the simulation kernel on 229,376
            # trajectories: DRAM read + write per trajectory, and warp
            # instructions per reaction event
            dram_bytes_per_traj=(466.38e6 + 1003.97e6) / 229376,
            warp_inst_per_event=32554582830 / 4209068063),
        'lv_ssa': dict(
            model=networks.lotka_volterra(), n=1024, method='direct',
            desc='plain Gillespie direct method, Lotka-Volterra (k1=10, '
                 'k2=0.01, k3=10), X0=Y0=1000, 1024 trajectories, t_end=10,'
                 ' 100 samples, Philox ids 0..1023',
            cpu_pilot=64, ref_config='lv_ssa_1024'),
        'telegraph_grad': dict(
            model=networks.telegraph(), n=1048576, method='direct', grad=True,
            desc='adjoint gradient: telegraph gene expression (k_on=0.5, '
                 'k_off=0.2, 20, 1, 5, 0.1), gene off, 1048576 direct-method'
                 ' trajectories with likelihood-ratio scores, t_end=50, 20 '
                 'samples of protein; step = forward kernel + moments + '
                 'score-backward reduction of d(mean+var)/d log k',
            cpu_pilot=256, ref_config=None),
    }


def measured_peaks():
    p = os.path.join(HERE, 'MEASURED_PEAKS.json')
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d['hbm_gbs']), 'measured'
    return 6650.0, 'fallback'


class ClockSampler(object):
    """nvidia-smi sampling of SM clock and throttle reasons while running."""

    Q = ('index,clocks.sm,clocks.max.sm,power.draw,'
         'clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,'
         'clocks_event_reasons.hw_thermal_slowdown,'
         'clocks_event_reasons.sw_thermal_slowdown,'
         'clocks_event_reasons.sw_power_cap')

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ['nvidia-smi', '--query-gpu=' + self.Q, '--format=csv,noheader,'
                 'nounits', '-i', str(self.idx), '-lms', '100'],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(',')])

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], 0.0, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown',
                 'sw_power_cap']
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
            except (ValueError, IndexError):
                continue
            for k, name in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith('active'):
                    reasons.add(name)
        if not sm:
            return None
        return {'sm_mhz': float(np.median(sm)), 'sm_max_mhz': mx,
                'reasons': sorted(reasons), 'samples': len(sm)}


def expected_events(wl, n=2048):
    """Mean reaction firings per trajectory of the workload, from the CPU
    oracle (same law as the reference; the reference kernels do not count
    firings).  Returns (mean, standard error)."""
    from oracle import oracle
    m, meth = wl['model'], 0 if wl['method'] == 'direct' else 1
    r = oracle.simulate(m, n, meth, seed=77)
    ev = r['events'].astype(np.float64)
    return ev.mean(), ev.std(ddof=1) / np.sqrt(n)


def run_reference_kernels(args, wl):
    """The reference's own kernels on the GPU (oracle/_ref), replaying
    CuTauLeaping.run / CuGillespie.run; wall clock per run, since the
    reference synchronises the host every round."""
    import torch
    from oracle import ref_harness
    r = ref_harness.ReferenceRun(wl['ref_config'])
    U = r.info['U']
    for _ in range(args.warmup):
        O, _ = r.run()
        O.cpu()
    times, rounds = [], []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        O, nr = r.run()
        host = O.cpu()  # CuTauLeaping.run returns O copied to the host
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
        rounds.append(nr)
    del host
    mean_ev, se_ev = expected_events(wl)
    tot = float(np.sum(times))
    val = mean_ev * U * args.steps / tot
    line = {'impl': 'reference', 'metric': METRIC, 'value': val,
            'unit': UNIT, 'n_gpus': args.gpus, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': 1e3 * tot / args.steps,
            'higher_is_better': True, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'f64/f32', 'data': 'synthetic',
            'config': {'workload': wl['desc']},
            'trajectories_per_s': U * args.steps / tot,
            'reference': {'kernels': 'the reference\'s kernel_P1_P2/'
                          'kernel_P3/init_rng (or kernel_Gillespie) CUDA '
                          'source, compiled for sm_100a, host loop of '
                          'CuTauLeaping.run replayed (oracle/ref_harness.py)',
                          'host_rounds_per_step': float(np.mean(rounds)),
                          'events_per_trajectory_estimate': mean_ev,
                          'events_estimate_se': se_ev},
            'cpu_baseline': {'value': val, 'unit': UNIT, 'cores': 1,
                             'kind': 'reference',
                             'sample': 'full workload (%d trajectories) '
                                       'on the GPU, one host thread '
                                       'driving it' % U},
            'e2e': {'value': val, 'unit': UNIT, 'h2d_bytes_per_step': 0,
                    'd2h_bytes_per_step': 0}}
    print(json.dumps(line))
    return 0


def run_reference(args, wl):
    rank = int(os.environ.get('RANK', '0'))
    if rank != 0:
        return 0
    try:
        import torch
        from oracle import ref_harness
        if (wl.get('ref_config') and torch.cuda.is_available()
                and ref_harness.available(wl['ref_config'])):
            return run_reference_kernels(args, wl)
    except ImportError:
        pass
    from oracle import oracle
    m, meth = wl['model'], 0 if wl['method'] == 'direct' else 1
    n = wl['cpu_pilot']
    # size one step to ~ (a few minutes / steps) of CPU work
    t0 = time.perf_counter()
    oracle.simulate(m, n, meth, seed=0)
    dt = time.perf_counter() - t0
    per_step = max(2.0, min(20.0, 150.0 / max(1, args.steps + args.warmup)))
    n = int(min(wl['n'], max(n, n * per_step / max(dt, 1e-3))))
    for w in range(args.warmup):
        oracle.simulate(m, min(n, 256), meth, seed=1000 + w)
    tot_ev, tot_t = 0.0, 0.0
    for s in range(args.steps):
        t0 = time.perf_counter()
        r = oracle.simulate(m, n, meth, seed=s)
        tot_t += time.perf_counter() - t0
        tot_ev += float(r['events'].sum())
    val = tot_ev / tot_t
    cores = oracle.max_threads()
    line = {'impl': 'reference', 'metric': METRIC, 'value': val, 'unit': UNIT,
            'n_gpus': args.gpus, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': 1e3 * tot_t / args.steps,
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
            'dtype': 'f32/f64', 'data': 'synthetic',
            'config': {'workload': wl['desc']},
            'trajectories_per_s': n * args.steps / tot_t,
            'cpu_baseline': {'value': val, 'unit': UNIT, 'cores': cores,
                             'kind': 'port',
                             'sample': '%d of %d trajectories per step'
                                       % (n, wl['n'])},
            'e2e': {'value': val, 'unit': UNIT, 'h2d_bytes_per_step': 0,
                    'd2h_bytes_per_step': 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# batched persistent form vs plain one-launch-per-model form
# ---------------------------------------------------------------------------
def _events_timed(fn, stream):
    import torch
    torch.cuda.synchronize()
    st = torch.cuda.Event(enable_timing=True)
    en = torch.cuda.Event(enable_timing=True)
    st.record(stream)
    out = fn()
    en.record(stream)
    en.synchronize()
    return st.elapsed_time(en), out


def completed_events(events, status):
    """Firings of the trajectories that reached t_end or absorption (status
    DONE / ABSORBED): a leap count of a trajectory that grows until int32
    overflow or runs out of step budget is not throughput."""
    return float(events[status <= 1].sum().item())


def _form_record(ms, events, ok_events, status_counts, n_models, n_traj,
                 launches):
    st = [int(c) for c in status_counts]
    tot = float(sum(st))
    return {'ms': ms, 'models': n_models, 'launches': launches,
            'events': events, 'events_per_s': events / ms * 1e3,
            'completed_events_per_s': ok_events / ms * 1e3,
            'trajectories_per_s': n_models * n_traj / ms * 1e3,
            'status_counts': st,
            'unfinished_fraction': st[2] / tot if tot else 0.0,
            'error_fraction': sum(st[2:]) / tot if tot else 0.0}


def batch_vs_plain(kind, dev, subset=256, steps=1, full=True, budget=20000):
    """Events/s of the batched form (one persistent launch, CUDA graph) and
    of the plain form (one launch per model) on the same models.

    kind 'sweep': Lotka-Volterra / Schlogl parameter sets within a decade of
    the nominals, 256 trajectories each, tau-leaping with SSA fallback,
    likelihood-ratio scores plus in-kernel statistics and Jacobians
    (batched+grad).  kind 'synthetic': 4096 uneven synthetic networks, 64
    trajectories each, tau-leaping.  Both forms run the same trajectories
    with the same step budget and produce identical per-trajectory results;
    only the scheduling differs.  `completed_events_per_s` counts the
    firings of trajectories that reached t_end or absorption; trajectories
    stopped by the step budget are reported as `unfinished_fraction`, and
    int32 overflows (Lotka-Volterra sets whose prey grows without bound)
    in `status_counts`."""
    import torch
    from py_stoch_b200 import _lib, networks
    from py_stoch_b200.autotune import Autotuner
    from py_stoch_b200.batch import Batch
    from py_stoch_b200.simulator import simulate
    stream = torch.cuda.current_stream(dev)
    if kind == 'sweep':
        models, _ = networks.parameter_sweep(16384, seed=1)
        n_traj, grad = 256, True
        desc = ('16384 parameter sets (Lotka-Volterra / Schlogl nominals '
                '+-1 decade) x 256 trajectories, 50 samples, tau-leaping '
                'with SSA fallback, scores + in-kernel mean/var/lag-1 + '
                'Jacobians')
    else:
        models = networks.synthetic_networks(4096, seed=0)
        n_traj, grad = 64, False
        desc = ('4096 synthetic networks (S 5-64, R 8-256) x 64 '
                'trajectories, 50 samples, tau-leaping with SSA fallback')
    tuner = Autotuner(device=dev, score=grad)
    tuner.tune(models, 'tau')
    rng = np.random.default_rng(7)
    pick = sorted(rng.permutation(len(models))[:subset].tolist())
    sub = [models[i] for i in pick]
    res = {'workload': desc, 'step_budget': budget,
           'subset_models': len(sub)}

    def batched(ms, ids=None):
        b = Batch(ms, n_traj, method='tau', mapping_fn=tuner.mapping_fn,
                  device=dev, score=grad, stats=grad, jacobian=grad,
                  traj_id_base=ids)
        batched_maps['same' if ids is not None else 'full'] = [
            int(x) for x in b.mappings]
        g = b.graph(seed=11, step_budget=budget)
        g.replay()  # untimed: the first replay after capture ran slower
        clk = ClockSampler(dev.index or 0)
        clk.start()
        tot_ms, ev, ev_ok = 0.0, 0.0, 0.0
        for _ in range(steps):
            ms_, _ = _events_timed(g.replay, stream)
            tot_ms += ms_
            ev += float(b.out['events'].sum().item())
            ev_ok += completed_events(b.out['events'], b.out['status'])
        clocks = clk.stop()
        st = torch.bincount(b.out['status'].long(), minlength=9).tolist()
        del g
        rec = _form_record(tot_ms / steps, ev / steps, ev_ok / steps, st,
                           len(ms), n_traj, 1)
        rec['work_items'] = int(b.n_items)
        rec['clocks'] = clocks
        return rec, b

    ids = [i * n_traj for i in pick]
    batched_maps = {}
    res['batched_same_models'], sub_batch = batched(sub, ids)
    # plain form: one simulate() launch per model, same ids and budget
    outs = [{'samples': torch.empty((m.kappa, m.ita, n_traj),
                                    dtype=torch.int32, device=dev),
             'events': torch.empty(n_traj, dtype=torch.int64, device=dev),
             'status': torch.empty(n_traj, dtype=torch.uint8, device=dev)}
            for m in sub]

    # the plain form's mapping per model: what the library picks for one
    # launch of n_traj trajectories (a warp per trajectory for networks
    # beyond the register engine's 32 reactions, since such a launch cannot
    # fill the GPU thread by thread); the batch tuner's choices are for
    # full batches
    plain_map = ['warp' if (m.n_reactions > _lib.THREAD_MAX_REACTIONS or
                            m.n_species > 64) else 'thread' for m in sub]

    def plain():
        for k, (m, i) in enumerate(zip(sub, pick)):
            simulate(m, n_traj, method='tau', seed=11,
                     traj_id_base=i * n_traj, device=dev, stream=stream,
                     out=outs[k], score=grad, status=True,
                     step_budget=budget, mapping=plain_map[k])
    ms_p, _ = _events_timed(plain, stream)
    ev_p = float(sum(int(o['events'].sum().item()) for o in outs))
    ok_p = sum(completed_events(o['events'], o['status']) for o in outs)
    st_p = np.sum([torch.bincount(o['status'].long(), minlength=9).tolist()
                   for o in outs], axis=0)
    res['plain'] = _form_record(ms_p, ev_p, ok_p, st_p, len(sub), n_traj,
                                len(sub))
    bs = res['batched_same_models']
    res['batched_over_plain'] = bs['events_per_s'] / res['plain'][
        'events_per_s']
    res['batched_over_plain_completed'] = (
        bs['completed_events_per_s'] /
        max(res['plain']['completed_events_per_s'], 1e-30))
    # identical per-trajectory results where both forms map a model alike
    # (warp-mapped runs sum propensities in another order)
    bmaps = batched_maps['same']
    alike = [k for k in range(len(sub))
             if (bmaps[k] == _lib.MAP_WARP) == (plain_map[k] == 'warp')]
    ok = True
    for k in alike:
        ok &= bool(torch.equal(outs[k]['events'],
                               sub_batch.per_traj('events', k)))
        ok &= bool(torch.equal(outs[k]['samples'], sub_batch.samples(k)))
    res['same_results'] = {'models_compared': len(alike), 'equal': ok}
    del sub_batch
    if full:
        res['batched_full'], fb = batched(models)
        del fb
    res['autotune'] = {k: v['mapping'] for k, v in tuner.table.items()
                       if 'mapping' in v}
    torch.cuda.empty_cache()
    return res


# ---------------------------------------------------------------------------
# instruction roofline: measured pipe peaks and algorithmic operations
# ---------------------------------------------------------------------------
PIPES = ('int32', 'fp32', 'fp64')


def measure_pipe_peaks(dev, reps=3):
    """Issue rates of the arithmetic pipes on this GPU, measured now with
    the library's probe kernel (pyst_test_pipe: 8 independent chains per
    thread, 8 blocks of 256 threads per SM), CUDA events on the launching
    stream, best of `reps`.  Operations per second: an FMA counts one."""
    import ctypes as C

    import torch

    from py_stoch_b200 import _lib
    L = _lib.lib()
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    blocks, iters = sms * 8, 2048
    sink = torch.empty(blocks * 256, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = C.c_void_p(stream.cuda_stream)
    rates = {}
    for which, name, per in ((0, 'fp32_fma', 1), (1, 'int32_mad', 1),
                             (2, 'fp64_fma', 1), (3, 'int32_alu', 2)):
        best = 0.0
        for r in range(reps + 1):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            _lib.check(L.pyst_test_pipe(which, iters, blocks,
                                        sink.data_ptr(), sp),
                       'pyst_test_pipe')
            b.record(stream)
            b.synchronize()
            if r:  # the first launch is a warm-up
                ops = 8.0 * per * iters * 256 * blocks
                best = max(best, ops / (a.elapsed_time(b) * 1e-3))
        rates[name] = best
    # Philox's multiplies run on the multiply-add pipe, its xors and key
    # additions on the ALU pipe; the larger of the two rates is the INT32
    # denominator (the less flattering choice if both pipes issue at once)
    return {'int32': max(rates['int32_mad'], rates['int32_alu']),
            'fp32': rates['fp32_fma'], 'fp64': rates['fp64_fma'],
            'probes': rates}


# Operation counts of this engine's building blocks (pyst_math.cuh,
# pyst_engine.cuh), counted from their arithmetic: an FMA, add, multiply,
# divide, compare or conversion is one operation.
PHILOX_INT = 98      # 10 rounds x (2 mul.lo + 2 mul.hi + 4 xor) + 9 x 2 key adds
U53_INT = 2          # 53-bit uniform: shift, or
LOG64 = 22           # pyst_log: split, (f-1)/(f+1), 11-term series, scaling
EXP64 = 20           # pyst_exp: reduction, 15-term series, scaling


def ops_per_trajectory(model, mix, tau, grad=False, fallback=100):
    """Algorithmic operations per trajectory, by pipe, of this engine's
    method on `model`, given the measured per-trajectory step mix (means of
    the oracle's counters: SSA steps, leaps, inversion Poisson draws and
    their search iterations, PTRS draws and their iterations).

    SSA step: one Philox block and two 53-bit uniforms, the FP32
    propensities (one multiply per reactant factor), the FP64 total and
    cumulative selection (2M), tau = e/a0, r = u a0 and the clock add, one
    log; the fired reaction's net changes.  A DECIDE (before every leap and
    every SSA fallback round): propensities, the critical-reaction test,
    the leap mean/variance sums (4 FP32 per net-change entry) and the tau
    candidate of each reactant species (8 FP32).  A leap: its Poisson
    draws (inversion: one Philox block, an exp, 3 FP64 per search step;
    PTRS: 12 FP32 set-up, half a Philox block and 11 FP32 per iteration),
    the state update and the critical-reaction clock.  Scores add, per SSA
    step, an FP64 multiply-add per reaction and an integer count."""
    M, S = model.n_reactions, model.n_species
    order = np.asarray(model.order).sum(axis=0).astype(float)
    nnz = (np.asarray(model.net) != 0).sum(axis=0).astype(float)
    nneg = float((np.asarray(model.net) < 0).sum())
    react = float((np.asarray(model.hor) > 0).sum())
    prop32 = float(order.sum())
    ssa, leaps = mix['ssa'], mix['leaps']
    ops = {p: 0.0 for p in PIPES}

    def add(n, i=0.0, f32=0.0, f64=0.0):
        ops['int32'] += n * i
        ops['fp32'] += n * f32
        ops['fp64'] += n * f64

    add(ssa, i=PHILOX_INT + 2 * U53_INT + nnz.mean(), f32=prop32,
        f64=2 * M + 3 + 2 + LOG64)
    if grad:
        add(ssa, i=1, f64=2 * M)
    if tau:
        n_decide = leaps + ssa / float(fallback)
        add(n_decide, i=2 * nneg, f32=prop32 + 4 * nnz.sum() + 8 * react,
            f64=M + 1)
        add(leaps, i=2 * nnz.sum() + S, f64=M + 3)
        add(mix['inv_draws'], i=PHILOX_INT + 1, f64=EXP64 + 2)
        add(mix['inv_iters'], f64=3)
        add(mix['ptrs_draws'], f32=12)
        add(mix['ptrs_iters'], i=PHILOX_INT / 2.0, f32=11)
    return ops


def step_mix(oracle_result):
    """Per-trajectory means of the oracle's step counters and firings."""
    st = oracle_result['steps'].astype(np.float64)
    names = ('ssa', 'leaps', 'inv_draws', 'inv_iters', 'ptrs_draws',
             'ptrs_iters')
    mix = {k: float(st[:, q].mean()) for q, k in enumerate(names)}
    mix['events'] = float(oracle_result['events'].astype(np.float64).mean())
    return mix


def ops_roofline(events_per_s, model, mix, peaks, tau, grad=False):
    """The instruction roofline of a simulation: algorithmic operations per
    event on each pipe x events/s against the measured pipe peak; the bound
    is the pipe with the largest fraction."""
    per_traj = ops_per_trajectory(model, mix, tau, grad)
    per_event = {p: per_traj[p] / mix['events'] for p in PIPES}
    pipes = {}
    for p in PIPES:
        a = events_per_s * per_event[p]
        pipes[p] = {'achieved_gops': a / 1e9, 'peak_gops': peaks[p] / 1e9,
                    'frac': a / peaks[p]}
    bound = max(PIPES, key=lambda p: pipes[p]['frac'])
    return {'bound': 'issue', 'pipe': bound,
            'achieved': pipes[bound]['achieved_gops'],
            'peak': pipes[bound]['peak_gops'], 'unit': 'Gop/s',
            'frac': pipes[bound]['frac'], 'peak_source': 'measured now '
            '(pyst_test_pipe probe on this GPU)',
            'algorithmic_ops_per_event': per_event,
            'step_mix_per_trajectory': mix, 'pipes': pipes}


# ---------------------------------------------------------------------------
# plain single-model workloads
# ---------------------------------------------------------------------------
def run_plain(wl, steps, warmup, dev, world=1, rank=0, e2e=True,
              geometry=None):
    """Time `steps` simulations of workload `wl` (one kernel launch each,
    plus the score reduction for gradient workloads) after `warmup`
    untimed ones; L2 flushed before every step; device time by CUDA events
    on the launching stream, max over ranks.  With `e2e`, the same again
    through the public API with the model blob copied in from pinned host
    memory and the outputs copied back inside the timed region."""
    import torch
    import torch.distributed as dist

    from py_stoch_b200.simulator import simulate
    m, n, meth = wl['model'], wl['n'], wl['method']
    base = rank * n
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    out = {'samples': torch.empty((m.kappa, m.ita, n), dtype=torch.int32,
                                  device=dev),
           'status': torch.empty(n, dtype=torch.uint8, device=dev),
           'events': torch.empty(n, dtype=torch.int64, device=dev)}
    grad = bool(wl.get('grad'))
    if grad:
        from py_stoch_b200.autograd import _moments, score_backward
        out['score'] = torch.empty((n, m.n_reactions), dtype=torch.float64,
                                   device=dev)
        ones = torch.ones((m.kappa, m.ita), dtype=torch.float64, device=dev)

    def step(seed, d_blob=None, outs=None):
        res = simulate(m, n, method=meth, seed=seed, traj_id_base=base,
                       device=dev, stream=stream, out=outs or out,
                       score=grad, d_blob=d_blob, geometry=geometry)
        if grad:
            # backward of mean + var of every sample: the score reduction
            mean, var = _moments(res['samples'])
            res['grad'] = score_backward(res['samples'], res['score'], mean,
                                         var, ones, ones, stream=stream)
        return res

    for w in range(warmup):
        step(10_000 + w)
    torch.cuda.synchronize(dev)
    clk = ClockSampler(dev.index or 0)
    clk.start()
    total_ms, events, errs = 0.0, 0, 0
    status_counts = np.zeros(9, np.int64)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    for s in range(steps):
        flush.fill_(s & 0xFF)
        st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(
            enable_timing=True)
        st.record(stream)
        res = step(s)
        en.record(stream)
        en.synchronize()
        total_ms += st.elapsed_time(en)
        events += int(res['events'].sum().item())
        status_counts += np.bincount(res['status'].cpu().numpy(),
                                     minlength=9)[:9]
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clocks = clk.stop()
    errs = int(status_counts[2:].sum())
    t = torch.tensor([total_ms, float(events), float(errs)],
                     dtype=torch.float64, device=dev)
    if world > 1:
        tm = t[:1].clone()
        dist.all_reduce(tm, op=dist.ReduceOp.MAX)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        t[0] = tm[0]
    total_ms, events, errs = float(t[0]), float(t[1]), float(t[2])
    r = {'ms_per_step': total_ms / steps, 'events_per_step': events / steps,
         'value': events / (total_ms / 1e3),
         'trajectories_per_s': n * world * steps / (total_ms / 1e3),
         'error_trajectories': int(errs), 'clocks': clocks,
         'status_counts': status_counts.tolist(),
         # this library's kernels per step: the simulation, plus the
         # moments (sums, moments) and the two-kernel score reduction of
         # the gradient form
         'gpu_launches': steps * (5 if grad else 1),
         'out_bytes': sum(v.numel() * v.element_size()
                          for v in out.values())}
    if not e2e:
        return r
    # End to end through the public API, as an application pipelines it:
    # every step copies the model blob in from pinned host memory and all
    # its outputs (samples, status, event counts; the gradient) back to
    # pinned host memory; outputs are double-buffered and each step's copy
    # back runs on a copy stream while the next step computes.  One timed
    # region over all steps, from the first copy in to the last copy out.
    blob = torch.from_numpy(m.blob().view(np.int32)).pin_memory()
    d_blob = torch.empty_like(blob, device=dev)
    bufs = [out, {k: torch.empty_like(v) for k, v in out.items()}]
    h_bufs = [{k: torch.empty(v.shape, dtype=v.dtype, pin_memory=True)
               for k, v in out.items()} for _ in range(2)]
    h_grads = [torch.empty(m.n_reactions, dtype=torch.float64,
                           pin_memory=True) for _ in range(2)]
    xstream = torch.cuda.Stream(dev)
    copied = [None, None]
    ev_acc = torch.zeros((), dtype=torch.int64, device=dev)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    st = torch.cuda.Event(enable_timing=True)
    en = torch.cuda.Event(enable_timing=True)
    seed = None
    st.record(stream)
    for s in range(steps):
        b = s & 1
        flush.fill_(s & 0xFF)
        if copied[b] is not None:  # buffer b's previous copy is out
            stream.wait_event(copied[b])
        seed = 100 + s
        d_blob.copy_(blob, non_blocking=True)
        res = step(seed, d_blob=d_blob, outs=bufs[b])
        ev_acc += bufs[b]['events'].sum()
        done = torch.cuda.Event()
        done.record(stream)
        xstream.wait_event(done)
        with torch.cuda.stream(xstream):
            for k in h_bufs[b]:
                h_bufs[b][k].copy_(bufs[b][k], non_blocking=True)
            if grad:
                # (the gradient tensor is read on the copy stream: keep the
                # allocator from reusing it before that copy is done)
                res['grad'].record_stream(xstream)
                h_grads[b].copy_(res['grad'], non_blocking=True)
        copied[b] = torch.cuda.Event()
        copied[b].record(xstream)
    stream.wait_stream(xstream)
    en.record(stream)
    en.synchronize()
    e2e_ms, e2e_ev = st.elapsed_time(en), int(ev_acc.item())
    h_out = h_bufs[(steps - 1) & 1]
    h_grad = h_grads[0]
    e2 = torch.tensor([e2e_ms, float(e2e_ev)], dtype=torch.float64,
                      device=dev)
    if world > 1:
        tm = e2[:1].clone()
        dist.all_reduce(tm, op=dist.ReduceOp.MAX)
        dist.all_reduce(e2, op=dist.ReduceOp.SUM)
        e2[0] = tm[0]
    d2h = sum(v.numel() * v.element_size() for v in h_out.values())
    r['e2e'] = {'value': float(e2[1]) / (float(e2[0]) / 1e3), 'unit': UNIT,
                'h2d_bytes_per_step': blob.numel() * 4,
                'd2h_bytes_per_step': d2h + (h_grad.numel() * 8 if grad
                                             else 0),
                'ms_per_step': float(e2[0]) / steps,
                'pipelined': 'outputs double-buffered; each step copied '
                             'back on a copy stream while the next step '
                             'computes; one timed region over all steps'}
    # the last end-to-end step's host outputs, for the CPU check
    r['_last'] = {'seed': seed, 'base': base, 'samples':
                  h_out['samples'].numpy(), 'events':
                  h_out['events'].numpy()}
    return r


def cpu_baseline(wl, check=None, target_s=12.0, threads=0):
    """The oracle port on host cores over a bounded sample of the workload
    (all of it when that fits ~`target_s`), which also gives the step mix
    of the instruction roofline.  With `check` (the last end-to-end step's
    seed, id base and host samples) the sample reruns exactly those
    trajectories, so the bench's own GPU output is compared with the oracle
    bit for bit."""
    from oracle import oracle
    m, meth = wl['model'], 0 if wl['method'] == 'direct' else 1
    seed = check['seed'] if check else 1
    base = check['base'] if check else 0
    n = wl['cpu_pilot']
    t0 = time.perf_counter()
    r = oracle.simulate(m, wl['n'], meth, seed=seed, traj_id_base=base,
                        threads=threads, u1=n)
    dt = time.perf_counter() - t0
    if dt < target_s / 4:
        n = int(min(wl['n'], max(n, n * target_s / max(dt, 1e-3))))
        t0 = time.perf_counter()
        r = oracle.simulate(m, wl['n'], meth, seed=seed, traj_id_base=base,
                            threads=threads, u1=n)
        dt = time.perf_counter() - t0
    part = {'samples': r['samples'][:, :, :n], 'events': r['events'][:n],
            'steps': r['steps'][:n]}
    ev = float(part['events'].sum())
    cores = threads if threads > 0 else oracle.max_threads()
    res = {'value': ev / dt, 'unit': UNIT, 'cores': cores, 'kind': 'port',
           'sample': '%d of %d trajectories of the same workload, %.1f s'
                     % (n, wl['n'], dt),
           'trajectories_per_s': n / dt}
    if check:
        res['bench_output_checked'] = {
            'trajectories': n,
            'bit_exact': bool(np.array_equal(
                part['samples'], check['samples'][:, :, :n]) and
                np.array_equal(part['events'], check['events'][:n]))}
    return res, step_mix(part)


def plain_record(name, wl, args, dev, peaks, steps, warmup, world=1,
                 rank=0):
    """One workload's numbers: device-timed value, e2e, the instruction
    roofline and, on one GPU, the CPU baseline with the output check.
    Tau-leaping workloads run with the mode-sorted scheduler geometry the
    autotuner picks for them (measured before the timed region)."""
    geometry = None
    if wl['method'] == 'tau' and not args.no_tune:
        from py_stoch_b200.autotune import Autotuner
        geometry = Autotuner(device=dev).tune_geometry(wl['model'], wl['n'],
                                                       'tau')
    r = run_plain(wl, steps, warmup, dev, world, rank, geometry=geometry)
    last = r.pop('_last', None)
    rec = {'workload': wl['desc'], 'trajectories_per_gpu': wl['n']}
    if geometry:
        rec['geometry'] = geometry
    rec.update(r)
    if world == 1 and not args.no_cpu_baseline:
        cb, mix = cpu_baseline(wl, check=last)
        rec['cpu_baseline'] = cb
        rec['roofline'] = ops_roofline(r['value'] / world, wl['model'], mix,
                                       peaks, wl['method'] == 'tau',
                                       bool(wl.get('grad')))
    return rec


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=5)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--workload', default='schlogl_tau')
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--n-traj', type=int, default=0,
                    help='override trajectories per GPU (profiling runs)')
    ap.add_argument('--no-configs', action='store_true',
                    help='headline only: skip the other configurations')
    ap.add_argument('--no-tune', action='store_true',
                    help='default scheduler geometry (profiling runs)')
    args = ap.parse_args()
    if args.workload in ('sweep', 'synthetic'):
        return forms_main(args)
    wl = workloads()[args.workload]
    if args.n_traj:
        wl['n'] = args.n_traj
    if args.impl == 'reference':
        return run_reference(args, wl)

    import torch
    import torch.distributed as dist

    from py_stoch_b200 import build as _build

    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group('nccl',
                                timeout=datetime.timedelta(seconds=120))
    dev = torch.device('cuda', local)
    torch.cuda.set_device(dev)
    # one rank (re)builds the library if its sources changed; the others
    # wait, so no two processes compile into the same build directory
    if rank == 0:
        _build.build()
    if world > 1:
        dist.barrier()
    peaks = measure_pipe_peaks(dev)
    head = plain_record(args.workload, wl, args, dev, peaks, args.steps,
                        args.warmup, world, rank)
    line = None
    if rank == 0:
        hbm, hbm_kind = measured_peaks()
        per_launch_s = head['ms_per_step'] / 1e3
        achieved = head['out_bytes'] / per_launch_s / 1e9
        traffic = (wl['dram_bytes_per_traj'] * wl['n']
                   if 'dram_bytes_per_traj' in wl else None)
        roof = head.get('roofline') or {}
        roof['traffic'] = traffic
        roof['hbm'] = {'bound': 'hbm', 'achieved': achieved, 'peak': hbm,
                       'unit': 'GB/s', 'frac': achieved / hbm,
                       'peak_source': hbm_kind,
                       'algorithmic_bytes': head['out_bytes'],
                       'traffic': traffic,
                       'note': 'HBM carries only the sample output; '
                               'traffic from an ncu capture of 229376 '
                               'trajectories scaled by trajectories'}
        if 'warp_inst_per_event' in wl and (head['clocks'] or {}).get(
                'sm_mhz'):
            sms = torch.cuda.get_device_properties(
                dev).multi_processor_count
            a = head['value'] / world * wl['warp_inst_per_event'] / 1e12
            pk = sms * 4 * head['clocks']['sm_mhz'] * 1e6 / 1e12
            roof['executed_issue'] = {
                'achieved': a, 'peak': pk, 'unit': 'T warp-inst/s',
                'frac': a / pk,
                'warp_inst_per_event': wl['warp_inst_per_event'],
                'source': 'ncu executed-instruction count per event x '
                          'measured events/s; peak 4 issue slots/SM/cycle '
                          'at the sampled clock'}
        line = {
            'metric': METRIC, 'value': head['value'], 'unit': UNIT,
            'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': head['ms_per_step'], 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32/f64',
            'data': 'synthetic',
            'config': {'workload': wl['desc'],
                       'trajectories_per_gpu': wl['n'],
                       'sorted_geometry': head.get('geometry'),
                       'l2': 'flushed (256 MiB write) before every step',
                       'parallelism': 'trajectory shards, one per GPU'},
            'trajectories_per_s': head['trajectories_per_s'],
            'events_per_step': head['events_per_step'],
            'error_trajectories': head['error_trajectories'],
            'status_counts': head['status_counts'],
            'gpu_launches': head['gpu_launches'],
            'e2e': head['e2e'], 'roofline': roof,
            'clocks': head['clocks'], 'pipe_peaks': peaks,
        }
        if 'cpu_baseline' in head:
            line['cpu_baseline'] = head['cpu_baseline']
    if world == 1 and not args.no_configs:
        line['configs'] = other_configs(args, dev, peaks)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


def other_configs(args, dev, peaks):
    """The other configurations of the metric, each as its own record:
    Lotka-Volterra direct method (1024 trajectories), the telegraph
    gradient (1M trajectories, forward + backward), the 16384-set sweep
    and the 4096 synthetic networks (batched, with the plain
    one-launch-per-model form on a subset of the same models)."""
    import torch
    wls = workloads()
    steps = max(1, min(args.steps, 5))
    out = {}
    for name in ('lv_ssa', 'telegraph_grad'):
        out[name] = plain_record(name, wls[name], args, dev, peaks, steps, 2)
        torch.cuda.empty_cache()
    out['sweep'] = batch_vs_plain('sweep', dev, subset=FORMS['sweep'][0],
                                  budget=FORMS['sweep'][1])
    out['synthetic'] = batch_vs_plain('synthetic', dev,
                                      subset=FORMS['synthetic'][0],
                                      budget=FORMS['synthetic'][1])
    return out


# (plain-form subset size, step budget) of the batched configurations.
# The sweep runs every trajectory to t_end (or int32 overflow) within 2e6
# steps; the synthetic networks include explosive ones that no budget
# finishes (10x the budget: 6x the time, 3% more completed firings), so
# they keep 20,000 steps and report the unfinished fraction.
FORMS = {'sweep': (64, 2_000_000), 'synthetic': (256, 20_000)}


def forms_main(args):
    """--workload sweep | synthetic: the batched-vs-plain comparison as the
    JSON line (value = batched events/s over all models, counting the
    trajectories that completed; all firings in `all_events_per_s`)."""
    import torch
    from py_stoch_b200 import build as _build
    dev = torch.device('cuda', int(os.environ.get('LOCAL_RANK', '0')))
    torch.cuda.set_device(dev)
    _build.build()
    subset, budget = FORMS[args.workload]
    r = batch_vs_plain(args.workload, dev, subset=subset, steps=args.steps,
                       full=True, budget=budget)
    full = r['batched_full']
    line = {'metric': METRIC, 'value': full['completed_events_per_s'],
            'all_events_per_s': full['events_per_s'], 'unit': UNIT,
            'n_gpus': 1, 'steps': args.steps, 'warmup': 1,
            'ms_per_step': full['ms'], 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32/f64',
            'data': 'synthetic', 'config': {'workload': r['workload']},
            'trajectories_per_s': full['trajectories_per_s'],
            'forms': r, 'gpu_launches': args.steps}
    print(json.dumps(line))
    return 0


if __name__ == '__main__':
    sys.exit(main())
