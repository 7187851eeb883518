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
            dram_bytes_per_traj=(519.8e6 + 1382.3e6) / 229376,
            warp_inst_per_event=41112782222 / 4209068063),
        'lv_ssa': dict(
            model=networks.lotka_volterra(), n=1024, method='direct',
            desc='plain Gillespie direct method, Lotka-Volterra (k1=10, '
                 'k2=0.01, k3=10), X0=Y0=1000, 1024 trajectories, t_end=10,'
                 ' 100 samples, Philox ids 0..1023',
            cpu_pilot=64, ref_config='lv_ssa_1024',
            # warp instructions per reaction event of the lane-group
            # kernel, from one ncu capture of this workload
            warp_inst_per_event=64533376180 / 307266234),
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


def cpu_baseline(wl, target_s=12.0, threads=0):
    """Oracle port on host cores over a bounded sample of the workload."""
    from oracle import oracle
    m, meth = wl['model'], 0 if wl['method'] == 'direct' else 1
    n = wl['cpu_pilot']
    t0 = time.perf_counter()
    r = oracle.simulate(m, n, meth, seed=0, threads=threads)
    dt = time.perf_counter() - t0
    if dt < target_s / 4:
        n2 = int(min(wl['n'], max(n, n * target_s / max(dt, 1e-3))))
        t0 = time.perf_counter()
        r = oracle.simulate(m, n2, meth, seed=1, threads=threads)
        dt = time.perf_counter() - t0
        n = n2
    ev = float(r['events'].sum())
    cores = threads if threads > 0 else oracle.max_threads()
    return {'value': ev / dt, 'unit': UNIT, 'cores': cores, 'kind': 'port',
            'sample': '%d of %d trajectories of the same workload, %.1f s'
                      % (n, wl['n'], dt),
            'trajectories_per_s': n / dt}


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


def batch_vs_plain(kind, dev, subset=256, steps=1, full=True, budget=20000):
    """Events/s of the batched form (one persistent launch, CUDA graph) and
    of the plain form (one launch per model) on the same models.

    kind 'sweep': Lotka-Volterra / Schlogl parameter sets within a decade of
    the nominals, 256 trajectories each, tau-leaping with SSA fallback,
    likelihood-ratio scores plus in-kernel statistics and Jacobians
    (batched+grad).  kind 'synthetic': 4096 uneven synthetic networks, 64
    trajectories each, tau-leaping.  Both forms run the same trajectories
    with the same step budget and produce identical per-trajectory results;
    only the scheduling differs."""
    import torch
    from py_stoch_b200 import networks
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
        g = b.graph(seed=11, step_budget=budget)
        g.replay()
        tot_ms, ev, ev_ok = 0.0, 0.0, 0.0
        for _ in range(steps):
            ms_, _ = _events_timed(g.replay, stream)
            tot_ms += ms_
            ev += float(b.out['events'].sum().item())
            ev_ok += completed_events(b.out['events'], b.out['status'])
        st = torch.bincount(b.out['status'].long(), minlength=7).tolist()
        del g
        return tot_ms / steps, ev / steps, st, b, ev_ok / steps

    ids = [i * n_traj for i in pick]
    ms_b, ev_b, st_b, _, ok_b = batched(sub, ids)
    # plain form: one simulate() launch per model, same ids and budget
    outs = [{'samples': torch.empty((m.kappa, m.ita, n_traj),
                                    dtype=torch.int32, device=dev),
             'events': torch.empty(n_traj, dtype=torch.int64, device=dev),
             'status': torch.empty(n_traj, dtype=torch.uint8, device=dev)}
            for m in sub]

    def plain():
        for k, (m, i) in enumerate(zip(sub, pick)):
            simulate(m, n_traj, method='tau', seed=11,
                     traj_id_base=i * n_traj, device=dev, stream=stream,
                     out=outs[k], score=grad, status=True,
                     step_budget=budget,
                     mapping=('thread' if tuner.mapping(m, 'tau') == 1
                              else 'warp'))
    plain()
    ms_p, _ = _events_timed(plain, stream)
    ev_p = float(sum(int(o['events'].sum().item()) for o in outs))
    ok_p = sum(completed_events(o['events'], o['status']) for o in outs)
    res['plain'] = {'ms': ms_p, 'events': ev_p, 'events_per_s':
                    ev_p / ms_p * 1e3, 'completed_events_per_s':
                    ok_p / ms_p * 1e3, 'launches': len(sub)}
    res['batched_same_models'] = {'ms': ms_b, 'events': ev_b,
                                  'events_per_s': ev_b / ms_b * 1e3,
                                  'completed_events_per_s':
                                      ok_b / ms_b * 1e3,
                                  'launches': 1, 'status_counts': st_b}
    res['batched_over_plain'] = (ev_b / ms_b) / (ev_p / ms_p)
    if full:
        ms_f, ev_f, st_f, b, ok_f = batched(models)
        res['batched_full'] = {'models': len(models), 'ms': ms_f,
                               'events': ev_f,
                               'events_per_s': ev_f / ms_f * 1e3,
                               'completed_events_per_s': ok_f / ms_f * 1e3,
                               'trajectories_per_s':
                                   len(models) * n_traj / ms_f * 1e3,
                               'status_counts': st_f}
        del b
    res['autotune'] = {k: v['mapping'] for k, v in tuner.table.items()
                       if 'mapping' in v}
    torch.cuda.empty_cache()
    return res


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
    ap.add_argument('--no-forms', action='store_true',
                    help='skip the batched-vs-plain comparison')
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
    from py_stoch_b200.simulator import simulate

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

    def step(seed, d_blob=None):
        res = simulate(m, n, method=meth, seed=seed, traj_id_base=base,
                       device=dev, stream=stream, out=out, score=grad,
                       d_blob=d_blob)
        if grad:
            # backward of mean + var of every sample: the score reduction
            mean, var = _moments(res['samples'])
            res['grad'] = score_backward(res['samples'], res['score'], mean,
                                         var, ones, ones, stream=stream)
        return res

    for w in range(args.warmup):
        step(10_000 + w)
    torch.cuda.synchronize(dev)
    clk = ClockSampler(local)
    clk.start()
    total_ms, events = 0.0, 0
    errs = 0
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    for s in range(args.steps):
        flush.fill_(s & 0xFF)
        st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(
            enable_timing=True)
        st.record(stream)
        res = step(s)
        en.record(stream)
        en.synchronize()
        total_ms += st.elapsed_time(en)
        events += int(res['events'].sum().item())
        errs += int((res['status'] >= 2).sum().item())
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clocks = clk.stop()
    t = torch.tensor([total_ms, float(events), float(errs)], dtype=torch.float64,
                     device=dev)
    if world > 1:
        tm = t[:1].clone()
        dist.all_reduce(tm, op=dist.ReduceOp.MAX)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        t[0] = tm[0]
    total_ms, events, errs = float(t[0]), float(t[1]), float(t[2])
    sec = total_ms / 1e3
    value = events / sec

    # end to end through the public API: pinned host model blob in, samples
    # and per-trajectory status/events out, every step
    blob = torch.from_numpy(m.blob().view(np.int32)).pin_memory()
    d_blob = torch.empty_like(blob, device=dev)
    h_out = {k: torch.empty(v.shape, dtype=v.dtype, pin_memory=True)
             for k, v in out.items()}
    h_grad = torch.empty(m.n_reactions, dtype=torch.float64,
                         pin_memory=True)
    e2e_ms, e2e_ev = 0.0, 0
    for s in range(args.steps):
        flush.fill_(s & 0xFF)
        st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(
            enable_timing=True)
        st.record(stream)
        d_blob.copy_(blob, non_blocking=True)
        res = step(100 + s, d_blob=d_blob)
        for k in h_out:
            h_out[k].copy_(out[k], non_blocking=True)
        if grad:
            h_grad.copy_(res['grad'], non_blocking=True)
        en.record(stream)
        en.synchronize()
        e2e_ms += st.elapsed_time(en)
        e2e_ev += int(h_out['events'].sum())
    e2 = torch.tensor([e2e_ms, float(e2e_ev)], dtype=torch.float64, device=dev)
    if world > 1:
        tm = e2[:1].clone()
        dist.all_reduce(tm, op=dist.ReduceOp.MAX)
        dist.all_reduce(e2, op=dist.ReduceOp.SUM)
        e2[0] = tm[0]
    e2e_value = float(e2[1]) / (float(e2[0]) / 1e3)
    h2d = blob.numel() * 4
    d2h = sum(v.numel() * v.element_size() for v in h_out.values())
    if grad:
        d2h += h_grad.numel() * 8

    if rank == 0:
        peak, peak_kind = measured_peaks()
        out_bytes = sum(v.numel() * v.element_size() for v in out.values())
        per_launch_s = sec / args.steps / 1.0
        achieved = out_bytes / per_launch_s / 1e9
        traffic = (wl['dram_bytes_per_traj'] * n
                   if 'dram_bytes_per_traj' in wl else None)
        issue = None
        if 'warp_inst_per_event' in wl and clocks.get('sm_mhz'):
            # instruction-issue roofline: warp instructions per second
            # against 4 schedulers per SM at the sampled SM clock
            sms = torch.cuda.get_device_properties(dev).multi_processor_count
            a = value / world * wl['warp_inst_per_event'] / 1e12
            pk = sms * 4 * clocks['sm_mhz'] * 1e6 / 1e12
            issue = {'bound': 'issue', 'achieved': a, 'peak': pk,
                     'unit': 'T warp-inst/s', 'frac': a / pk,
                     'warp_inst_per_event': wl['warp_inst_per_event'],
                     'source': 'ncu instruction count per event x measured '
                               'events/s; peak 4 issue slots/SM/cycle'}
        line = {
            'metric': METRIC, 'value': value, 'unit': UNIT,
            'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': total_ms / args.steps, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32/f64',
            'data': 'synthetic',
            'config': {'workload': wl['desc'], 'trajectories_per_gpu': n,
                       'l2': 'flushed (256 MiB write) before every step',
                       'parallelism': 'trajectory shards, one per GPU'},
            'trajectories_per_s': n * world * args.steps / sec,
            'events_per_step': events / args.steps,
            'error_trajectories': int(errs),
            # this library's kernels in the timed region: the simulation,
            # plus the two-kernel score reduction of the gradient form
            'gpu_launches': args.steps * (3 if grad else 1),
            'e2e': {'value': e2e_value, 'unit': UNIT,
                    'h2d_bytes_per_step': h2d, 'd2h_bytes_per_step': d2h},
            'roofline': {'bound': 'hbm', 'achieved': achieved, 'peak': peak,
                         'unit': 'GB/s', 'frac': achieved / peak,
                         'traffic': traffic, 'peak_source': peak_kind,
                         'algorithmic_bytes': out_bytes,
                         'note': 'the kernel is CUDA-core issue bound; HBM '
                                 'carries only the sample output (traffic: '
                                 'partially written 32-byte sectors of the '
                                 '[kappa][ita][U] layout, scaled from a '
                                 '229376-trajectory ncu capture)'},
            'issue': issue,
            'clocks': clocks,
        }
        if not args.no_cpu_baseline and world == 1:
            line['cpu_baseline'] = cpu_baseline(wl)
        if not args.no_forms and world == 1:
            line['forms'] = batch_vs_plain('sweep', dev, full=False)
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


def forms_main(args):
    """--workload sweep | synthetic: the batched-vs-plain comparison as the
    JSON line (value = batched events/s over all models, counting the
    trajectories that completed; all firings in `all_events_per_s`)."""
    import torch
    from py_stoch_b200 import build as _build
    dev = torch.device('cuda', int(os.environ.get('LOCAL_RANK', '0')))
    torch.cuda.set_device(dev)
    _build.build()
    r = batch_vs_plain(args.workload, dev, steps=args.steps, full=True)
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
