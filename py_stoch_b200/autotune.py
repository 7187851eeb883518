"""Autotuner: thread- vs warp-per-trajectory mapping per model bucket and
the batch block size for batched runs, and the mode-sorted tau-leaping
scheduler's geometry (round lengths, trajectory slots per thread, block
size, which set its shared-memory layout) for single-model runs, chosen by
measurement.

Buckets are (method, reaction-count bucket, species-count bucket).  For
each bucket present in a batch the tuner builds a small trial batch from up
to ``sample`` of its models, times it with each mapping under a short step
budget (events per second on the device, CUDA events), and keeps the
faster.  The block size (64 or 128 threads) is chosen the same way on a
sample of the whole batch.  Results are cached per GPU name in a JSON file
(``$PYST_AUTOTUNE_CACHE`` or ``~/.cache/py_stoch_b200/autotune.json``), so a
bucket is measured once.

Trial runs use the caller's models and a different seed; they cost a few
hundred milliseconds per bucket.
"""

import json
import os
import threading

import numpy as np

from . import _lib
from .simulator import _method, _torch

R_EDGES = (8, 32, 64, 128, 256, 1024, 4096)
S_EDGES = (16, 64, 1024)
N_EDGES = (4096, 65536, 1 << 20, 1 << 40)

# Candidate geometries of the mode-sorted scheduler: (SSA steps, leaps) per
# round x slots per thread x block size.  Every one gives the same results
# (the schedule never changes a trajectory's arithmetic).
ROUNDS = ((16, 2), (20, 2), (32, 3), (40, 4), (50, 5), (64, 4))
POOLS = (1, 2)
SORTED_BLOCKS = (896, 448)

_lock = threading.Lock()


def _edge(v, edges):
    for e in edges:
        if v <= e:
            return e
    return edges[-1]


def bucket(model, method):
    return '%d/R%d/S%d' % (_method(method), _edge(model.n_reactions, R_EDGES),
                           _edge(model.n_species, S_EDGES))


def cache_path():
    return os.environ.get('PYST_AUTOTUNE_CACHE') or os.path.join(
        os.path.expanduser('~'), '.cache', 'py_stoch_b200', 'autotune.json')


class Autotuner(object):
    def __init__(self, path=None, device=None, sample=48, n_traj=64,
                 budget=2000, score=False):
        torch = _torch()
        self.device = torch.device(device or 'cuda')
        self.gpu = torch.cuda.get_device_name(self.device)
        self.path = path or cache_path()
        self.sample = sample
        self.n_traj = n_traj
        self.budget = budget
        self.score = score
        self.table = {}
        self.timings = {}
        self._load()

    # ---- cache ----------------------------------------------------------
    def _load(self):
        try:
            with open(self.path) as f:
                self.table = json.load(f).get(self.gpu, {})
        except (OSError, ValueError):
            self.table = {}

    def _save(self):
        with _lock:
            data = {}
            try:
                with open(self.path) as f:
                    data = json.load(f)
            except (OSError, ValueError):
                data = {}
            data[self.gpu] = self.table
            try:
                os.makedirs(os.path.dirname(self.path), exist_ok=True)
                tmp = self.path + '.tmp%d' % os.getpid()
                with open(tmp, 'w') as f:
                    json.dump(data, f, indent=1, sort_keys=True)
                os.replace(tmp, self.path)
            except OSError:
                pass  # an unwritable cache only costs re-tuning

    # ---- measurement ----------------------------------------------------
    def _time(self, models, method, mapping, block_size=0):
        from .batch import Batch
        torch = _torch()
        kw = ({'mapping_fn': mapping} if callable(mapping) else
              {'mapping': mapping})
        # whole models per block (no trajectory chunks): a trial batch is
        # far smaller than the GPU, and chunks would favour whichever
        # mapping splits into more blocks, while a full batch fills the GPU
        # either way and runs at the per-block rate compared here
        b = Batch(models, self.n_traj, method=method, device=self.device,
                  score=self.score, chunk=0, **kw)
        b.run(seed=0x5EED, step_budget=self.budget, block_size=block_size)
        st = torch.cuda.Event(enable_timing=True)
        en = torch.cuda.Event(enable_timing=True)
        stream = torch.cuda.current_stream(self.device)
        st.record(stream)
        b.run(seed=0x5EEE, step_budget=self.budget, block_size=block_size)
        en.record(stream)
        en.synchronize()
        ms = st.elapsed_time(en)
        ev = float(b.out['events'].sum().item())
        return ev / max(ms, 1e-3) * 1e3

    def tune(self, models, method, force=False):
        """Measure every bucket of `models` not yet in the cache."""
        groups = {}
        for m in models:
            groups.setdefault(bucket(m, method), []).append(m)
        changed = False
        rng = np.random.default_rng(0)
        for key, ms in sorted(groups.items()):
            if key in self.table and not force:
                continue
            pick = [ms[i] for i in rng.permutation(len(ms))[:self.sample]]
            cands = {'thread': _lib.MAP_THREAD, 'warp': _lib.MAP_WARP}
            if any(m.n_species > 64 for m in pick):
                cands.pop('thread')
            if self.score and any(
                    m.n_reactions > _lib.THREAD_MAX_REACTIONS for m in pick):
                cands.pop('thread', None)
            res = {name: self._time(pick, method, mp)
                   for name, mp in cands.items()}
            best = max(res, key=res.get)
            self.table[key] = {'mapping': best, 'events_per_s': res}
            self.timings[key] = res
            changed = True
        if changed:
            self._save()
        return self

    def tune_block(self, models, method, force=False):
        key = 'block/%d' % _method(method)
        if key in self.table and not force:
            return self.table[key]['block']
        rng = np.random.default_rng(1)
        pick = [models[i] for i in
                rng.permutation(len(models))[:2 * self.sample]]
        res = {}
        for bs in (64, 128):
            res[str(bs)] = self._time(pick, method, self.mapping_fn, bs)
        best = int(max(res, key=res.get))
        self.table[key] = {'block': best, 'events_per_s': res}
        self._save()
        return best

    def _time_single(self, model, n_traj, method, geometry, reps=2):
        from .simulator import simulate
        torch = _torch()
        stream = torch.cuda.current_stream(self.device)
        out = {}
        best = 0.0
        for r in range(reps + 1):
            st = torch.cuda.Event(enable_timing=True)
            en = torch.cuda.Event(enable_timing=True)
            st.record(stream)
            res = simulate(model, n_traj, method=method, seed=0x5EED + r,
                           device=self.device, stream=stream, out=out,
                           geometry=geometry)
            en.record(stream)
            en.synchronize()
            out = {k: v for k, v in res.items() if k != '_keepalive'}
            if r:  # the first run is a warm-up
                ev = float(res['events'].sum().item())
                best = max(best, ev / max(st.elapsed_time(en), 1e-3) * 1e3)
        return best

    def tune_geometry(self, model, n_traj, method='tau', force=False):
        """Measure every candidate geometry of the mode-sorted scheduler on
        ``n_traj`` trajectories of ``model`` (whole runs, events per second
        by CUDA events, best of two after a warm-up) and cache the fastest
        for the model's bucket and run size.  Returns the geometry dict
        (keyword ``geometry`` of :func:`py_stoch_b200.simulator.simulate`).
        """
        key = 'geom/%s/N%d' % (bucket(model, method),
                               _edge(int(n_traj), N_EDGES))
        if key in self.table and not force:
            return dict(self.table[key]['geometry'])
        res = {}
        for (rs, rl) in ROUNDS:
            for pool in POOLS:
                for blk in SORTED_BLOCKS:
                    g = {'round_ssa': rs, 'round_leap': rl,
                         'pool_slots': pool, 'sorted_block': blk}
                    name = '%d/%d/p%d/b%d' % (rs, rl, pool, blk)
                    res[name] = (g, self._time_single(model, n_traj, method,
                                                      g))
        best = max(res, key=lambda k: res[k][1])
        self.table[key] = {'geometry': res[best][0],
                           'events_per_s': {k: v[1] for k, v in
                                            res.items()}}
        self.timings[key] = self.table[key]['events_per_s']
        self._save()
        return dict(res[best][0])

    def geometry(self, model, n_traj, method='tau'):
        """Cached geometry for this model bucket and run size, or None."""
        ent = self.table.get('geom/%s/N%d' % (bucket(model, method),
                                              _edge(int(n_traj), N_EDGES)))
        return dict(ent['geometry']) if ent else None

    # ---- lookup ----------------------------------------------------------
    def mapping(self, model, method):
        ent = self.table.get(bucket(model, method))
        if ent is None:
            from .batch import auto_mapping
            return auto_mapping(model, self.score)
        return _lib.MAP_THREAD if ent['mapping'] == 'thread' else \
            _lib.MAP_WARP

    def mapping_fn(self, model, method):
        return self.mapping(model, method)
