"""Batched persistent runs: many models of uneven size in one launch.

The reference runs a sweep as one JIT compile and one host-driven launch
sequence per parameter combination (``examples/schlogl_sim.py:66-80``,
``examples/PL_sim.py:73-89``).  :class:`Batch` packs every model into one
device blob table and one item table, allocates all outputs once, and runs
everything with a single ``pyst_batch_run`` launch whose blocks pull items
from a device work queue (largest estimated cost first).

Outputs of item ``i`` are views: ``batch.samples(i)`` is
``[kappa_i, ita_i, n_traj_i]``; per-trajectory arrays are sliced the same
way.
"""

import ctypes as C

import numpy as np

from . import _lib
from .simulator import DEFAULT_STEP_BUDGET, _mapping, _method, _torch


# Resident threads per SM of the batched kernel (6 blocks of 128).
BATCH_THREADS_PER_SM = 768


def estimated_cost(model, method):
    """Rough work estimate of one trajectory: total propensity at x0 times
    the simulated time (events for the direct method)."""
    x = model.x0.astype(np.float64)
    a0 = 0.0
    for j in range(model.n_reactions):
        a = float(model.rate[j])
        for i in range(model.n_species):
            n = int(model.order[i, j])
            for q in range(n):
                a *= max(x[i] - q * int(model.falling[i, j]), 0.0)
        a0 += a
    cost = max(a0, 1.0) * float(model.sample_times[-1])
    if _method(method) == _lib.METHOD_TAU_LEAP:
        cost = min(cost, 1e4 * float(model.sample_times[-1]) + 1.0)
    return cost * (1.0 + model.n_reactions / 32.0)


def auto_mapping(model, score=False):
    """Thread per trajectory unless the species columns would not fit or
    a scored model has more reactions than the register accumulators."""
    if model.n_species > 64:
        return _lib.MAP_WARP
    if score and model.n_reactions > _lib.THREAD_MAX_REACTIONS:
        return _lib.MAP_WARP
    return _lib.MAP_THREAD


class Batch(object):
    """A set of (model, trajectories, method, mapping) items."""

    def __init__(self, models, n_traj, method='direct', mapping='auto',
                 traj_id_base=None, device=None, score=False, status=True,
                 events=True, seqhash=False, t_final=False, order='cost',
                 mapping_fn=None, stats=False, jacobian=False, chunk=128,
                 small_batch_warps=True):
        torch = _torch()
        self.device = torch.device(device or 'cuda')
        self.models = list(models)
        n = len(self.models)
        if (score or jacobian) and any(getattr(m, 'has_laws', False)
                                       for m in self.models):
            raise ValueError('likelihood-ratio scores need mass-action laws; '
                             'a model of the batch has general kinetic laws')
        self.n_traj = (np.full(n, int(n_traj), np.int64)
                       if np.isscalar(n_traj) else
                       np.asarray(n_traj, np.int64))
        meths = ([method] * n if isinstance(method, (str, int)) else
                 list(method))
        self.methods = np.array([_method(m) for m in meths], np.int32)
        if mapping_fn is not None:
            maps = [mapping_fn(m, me) for m, me in zip(self.models,
                                                       self.methods)]
        elif isinstance(mapping, (str, int)):
            maps = [mapping] * n
        else:
            maps = list(mapping)
        mp = []
        for m, x in zip(self.models, maps):
            x = _mapping(x)
            if x == _lib.MAP_AUTO:
                x = auto_mapping(m, score)
            if x == _lib.MAP_THREAD and score and (
                    m.n_reactions > _lib.THREAD_MAX_REACTIONS):
                x = _lib.MAP_WARP
            mp.append(x)
        # A batch whose trajectories would fill less than half the GPU
        # thread by thread is latency-bound: networks beyond the register
        # engine's reactions then run a warp per trajectory (each step's
        # reactions over 32 lanes), whatever a full-batch tuning chose.
        chosen_here = mapping_fn is not None or (
            isinstance(mapping, (str, int)) and
            _mapping(mapping) == _lib.MAP_AUTO)
        if small_batch_warps and chosen_here:
            props = torch.cuda.get_device_properties(self.device)
            capacity = props.multi_processor_count * BATCH_THREADS_PER_SM
            if int(self.n_traj.sum()) * 2 < capacity:
                mp = [_lib.MAP_WARP if (m.n_reactions >
                                        _lib.THREAD_MAX_REACTIONS) else x
                      for m, x in zip(self.models, mp)]
        self.mappings = np.array(mp, np.int32)
        if traj_id_base is None:
            traj_id_base = np.concatenate([[0], np.cumsum(self.n_traj)[:-1]])
        self.traj_id_base = np.asarray(traj_id_base, np.int64)

        blobs = [m.blob() for m in self.models]
        self.blob_offset = np.concatenate(
            [[0], np.cumsum([len(b) for b in blobs])[:-1]]).astype(np.int64)
        self.kappa = np.array([m.kappa for m in self.models], np.int64)
        self.ita = np.array([m.ita for m in self.models], np.int64)
        self.R = np.array([m.n_reactions for m in self.models], np.int64)
        sizes = self.kappa * self.ita * self.n_traj
        self.sample_offset = np.concatenate(
            [[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
        self.traj_offset = np.concatenate(
            [[0], np.cumsum(self.n_traj)[:-1]]).astype(np.int64)
        self.score_offset = np.concatenate(
            [[0], np.cumsum(self.n_traj * self.R)[:-1]]).astype(np.int64)
        self.stats_offset = np.concatenate(
            [[0], np.cumsum(self.kappa * self.ita * 3)[:-1]]).astype(np.int64)
        self.jac_offset = np.concatenate(
            [[0], np.cumsum(2 * self.kappa * self.ita * self.R)[:-1]]
        ).astype(np.int64)
        if jacobian and not score:
            raise ValueError('jacobian needs score=True')
        self.total_traj = int(self.n_traj.sum())

        if order == 'cost':
            cost = np.array([estimated_cost(m, me) * nt for m, me, nt in
                             zip(self.models, self.methods, self.n_traj)])
            self.run_order = np.argsort(-cost, kind='stable')
        else:
            self.run_order = np.arange(n)
        # Work items: a model whose trajectories exceed `chunk` (a
        # thread-mapped block's trajectories per pass) is split into chunks
        # that different blocks run at once, so a few large models still
        # fill the GPU and the longest ones do not form the tail alone.
        spans = []
        for i in self.run_order:
            U = int(self.n_traj[i])
            cs = int(chunk) if chunk else 0
            if self.mappings[i] == _lib.MAP_WARP:
                cs = max(cs // 8, 4) if cs else 0
            if cs and U > cs:
                k = -(-U // cs)
                spans += [(i, c * cs, min(cs, U - c * cs), U, k)
                          for c in range(k)]
            else:
                spans.append((i, 0, U, 0, 0))
        self.n_items = len(spans)
        self.item_model = np.array([sp[0] for sp in spans], np.int64)
        self.item_n_traj = np.array([sp[2] for sp in spans], np.int64)
        items = (_lib.BatchItem * len(spans))()
        for slot, (i, c0, cn, U, k) in enumerate(spans):
            it = items[slot]
            it.blob_offset = int(self.blob_offset[i])
            it.n_traj = cn
            it.traj_id_base = int(self.traj_id_base[i])
            it.sample_offset = int(self.sample_offset[i])
            it.traj_offset = int(self.traj_offset[i])
            it.score_offset = int(self.score_offset[i])
            it.stats_offset = int(self.stats_offset[i])
            it.jac_offset = int(self.jac_offset[i])
            it.method = int(self.methods[i])
            it.mapping = int(self.mappings[i])
            it.chunk_begin = c0
            it.model_n_traj = U
            it.group = int(i)
            it.group_chunks = k
        raw = np.frombuffer(bytes(items), dtype=np.uint8)
        self.d_items = torch.from_numpy(raw.copy()).to(self.device)
        self.d_blobs = torch.from_numpy(
            np.concatenate(blobs).view(np.int32)).to(self.device)
        self.limits = _lib.BatchLimits(
            max(len(b) for b in blobs),
            max(m.n_species for m in self.models),
            max(m.n_reactions for m in self.models), 0)
        L = _lib.lib()
        ws = C.c_size_t(0)
        _lib.check(L.pyst_batch_workspace_size(self.n_items, C.byref(ws)),
                   'pyst_batch_workspace_size')
        self.workspace = torch.empty(int(ws.value), dtype=torch.uint8,
                                     device=self.device)
        dev = self.device
        self.out = {'samples': torch.empty(int(sizes.sum()),
                                           dtype=torch.int32, device=dev)}
        if status:
            self.out['status'] = torch.empty(self.total_traj,
                                             dtype=torch.uint8, device=dev)
        if events:
            self.out['events'] = torch.empty(self.total_traj,
                                             dtype=torch.int64, device=dev)
        if seqhash:
            self.out['seqhash'] = torch.empty(self.total_traj,
                                              dtype=torch.int64, device=dev)
        if t_final:
            self.out['t_final'] = torch.empty(self.total_traj,
                                              dtype=torch.float64, device=dev)
        if score:
            self.out['score'] = torch.empty(int((self.n_traj * self.R).sum()),
                                            dtype=torch.float64, device=dev)
        if stats:
            self.out['stats'] = torch.empty(
                int((self.kappa * self.ita * 3).sum()), dtype=torch.float64,
                device=dev)
        if jacobian:
            self.out['jacobian'] = torch.empty(
                int((2 * self.kappa * self.ita * self.R).sum()),
                dtype=torch.float64, device=dev)

    def run(self, seed=0, stream=None, ssa_fallback_steps=100,
            max_leap_retries=63, step_budget=None, block_size=0):
        """Enqueue the whole batch on ``stream`` (one kernel launch).
        ``block_size`` 0 picks 64 threads when no work item has more than 64
        trajectories (one block then covers an item), else 128."""
        torch = _torch()
        L = _lib.lib()
        if not block_size:
            block_size = 64 if int(self.item_n_traj.max()) <= 64 else 128
        if step_budget is None:
            step_budget = DEFAULT_STEP_BUDGET
        o = self.out
        outs = _lib.Outputs(
            o['samples'].data_ptr(), 0,
            o['status'].data_ptr() if 'status' in o else 0,
            o['events'].data_ptr() if 'events' in o else 0,
            o['seqhash'].data_ptr() if 'seqhash' in o else 0,
            o['t_final'].data_ptr() if 't_final' in o else 0,
            o['score'].data_ptr() if 'score' in o else 0,
            o['stats'].data_ptr() if 'stats' in o else 0,
            o['jacobian'].data_ptr() if 'jacobian' in o else 0)
        r = _lib.RunDesc(0, 0, int(seed) & 0xFFFFFFFFFFFFFFFF, 0, 0,
                         int(ssa_fallback_steps), int(max_leap_retries),
                         int(step_budget), int(block_size), 0)
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        _lib.check(L.pyst_batch_run(
            self.d_blobs.data_ptr(), self.d_items.data_ptr(),
            self.n_items, C.byref(self.limits), C.byref(r),
            C.byref(outs), self.workspace.data_ptr(),
            self.workspace.numel(), C.c_void_p(stream.cuda_stream)),
            'pyst_batch_run')
        return self

    def graph(self, seed=0, **run_kw):
        """Capture one run of the batch into a CUDA graph and return it
        (``torch.cuda.CUDAGraph``); ``graph.replay()`` re-runs the whole
        batch, same seed, with one graph launch.  Runs the batch once
        uncaptured first (kernel attributes are set outside the capture)."""
        torch = _torch()
        self.run(seed=seed, **run_kw)
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                self.run(seed=seed, stream=s, **run_kw)
        torch.cuda.current_stream(self.device).wait_stream(s)
        return g

    @classmethod
    def from_tl_args_list(cls, tl_args_list, simulator='tau', **kw):
        """One batch for a whole sweep built by
        :meth:`py_stoch_b200.sim_maker.TLArgsList.make_list`.

        The reference runs such a list one point at a time, one
        ``CuTauLeaping().run(args)`` (or ``CuGillespie().run(args)``) each
        (``examples/schlogl_sim.py:66-80``).  Item i here is point i: its
        ``args.U`` is rounded up by the same ``calculate_sizes`` rule (the
        side effect the drop-in classes keep), it takes the direct method
        when ``args.gillespie`` is set (or ``simulator='gillespie'``) and
        tau-leaping otherwise, and -- like every point of the per-point loop
        -- its trajectories have Philox ids 0..U-1.  With the same seed each
        item's samples equal that point's ``run(args)`` result bit for bit
        (:meth:`results` returns them as NumPy arrays).  Keyword arguments
        go to :class:`Batch`."""
        from .model import Model
        from .simulator import CuGillespie, CuTauLeaping
        sim = CuGillespie() if simulator == 'gillespie' else CuTauLeaping()
        models, n_traj, methods = [], [], []
        for args in tl_args_list:
            sim.calculate_sizes(args)
            models.append(Model.from_tl_args(args))
            n_traj.append(int(args.U))
            direct = simulator == 'gillespie' or getattr(args, 'gillespie',
                                                         0)
            methods.append('direct' if direct else 'tau')
        kw.setdefault('traj_id_base', np.zeros(len(models), np.int64))
        return cls(models, n_traj, method=methods, **kw)

    def results(self):
        """Per item, its samples ``[kappa, ita, n_traj]`` as int32 NumPy
        arrays (the drop-in ``run(args)`` layout); raises if any trajectory
        ended with an error status, as the drop-in classes do."""
        torch = _torch()
        torch.cuda.synchronize(self.device)
        if 'status' in self.out:
            from .simulator import ERROR_STATUSES
            st = self.out['status'].cpu().numpy()
            bad = np.isin(st, ERROR_STATUSES)
            if bad.any():
                L = _lib.lib()
                codes = sorted(set(int(c) for c in st[bad]))
                raise RuntimeError('%d of %d trajectories failed (%s)' % (
                    int(bad.sum()), st.size, ', '.join(
                        L.pyst_traj_status_string(c).decode()
                        for c in codes)))
        return [self.samples(i).cpu().numpy() for i in range(len(self.models))]

    # ---- per-item views -------------------------------------------------
    def samples(self, i):
        a = int(self.sample_offset[i])
        n = int(self.kappa[i] * self.ita[i] * self.n_traj[i])
        return self.out['samples'][a:a + n].view(
            int(self.kappa[i]), int(self.ita[i]), int(self.n_traj[i]))

    def per_traj(self, name, i):
        a = int(self.traj_offset[i])
        return self.out[name][a:a + int(self.n_traj[i])]

    def stats(self, i):
        """[kappa, ita, 3]: mean, variance, lag-1 correlation."""
        a = int(self.stats_offset[i])
        n = int(self.kappa[i] * self.ita[i] * 3)
        return self.out['stats'][a:a + n].view(int(self.kappa[i]),
                                               int(self.ita[i]), 3)

    def jacobian(self, i):
        """[2, kappa, ita, R]: d mean and d variance by d log rate."""
        a = int(self.jac_offset[i])
        n = int(2 * self.kappa[i] * self.ita[i] * self.R[i])
        return self.out['jacobian'][a:a + n].view(
            2, int(self.kappa[i]), int(self.ita[i]), int(self.R[i]))

    def score(self, i):
        a = int(self.score_offset[i])
        n = int(self.n_traj[i] * self.R[i])
        return self.out['score'][a:a + n].view(int(self.n_traj[i]),
                                               int(self.R[i]))
