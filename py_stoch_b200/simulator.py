"""Simulator entry points.

* :func:`simulate` -- run one model on the GPU through the C ABI and return
  device tensors (samples, per-trajectory status / event counts / hashes /
  final times / likelihood-ratio scores).
* :class:`CuGillespie`, :class:`CuTauLeaping` -- drop-ins for the
  reference classes of the same names (``mod/simulator/cuGillespie/
  cuGillespie.py:16-46``, ``mod/simulator/cuTauLeaping/cuTauLeaping.py:
  18-84``): ``run(args)`` takes a parsed ``TlArgs`` and returns an int32
  NumPy array ``[kappa, ita, U]`` after rounding ``args.U`` up to the
  reference's launch multiple, as ``calculate_sizes`` does.

There is no CPU path: without the CUDA library or a GPU these raise.
"""

import ctypes as C
import math

import numpy as np

from . import _lib
from .model import Model

METHODS = {'direct': _lib.METHOD_DIRECT, 'ssa': _lib.METHOD_DIRECT,
           'gillespie': _lib.METHOD_DIRECT, 'tau': _lib.METHOD_TAU_LEAP,
           'tau_leap': _lib.METHOD_TAU_LEAP}
MAPPINGS = {'auto': _lib.MAP_AUTO, 'thread': _lib.MAP_THREAD,
            'warp': _lib.MAP_WARP}

# Steps (SSA events plus leaps) one trajectory may take before it stops with
# status STEP_BUDGET; bounds the work of a run whose trajectories explode.
DEFAULT_STEP_BUDGET = 100_000_000

ERROR_STATUSES = (_lib.TRAJ_STEP_BUDGET, _lib.TRAJ_OVERFLOW,
                  _lib.TRAJ_LEAP_RETRY, _lib.TRAJ_SAMPLER, _lib.TRAJ_STAGING,
                  _lib.TRAJ_RATE, _lib.TRAJ_UNSUPPORTED)


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError('py_stoch_b200 needs a CUDA GPU; none is visible')
    return torch


def _method(m):
    return METHODS[m] if isinstance(m, str) else int(m)


def _mapping(m):
    return MAPPINGS[m] if isinstance(m, str) else int(m)


class SimResult(dict):
    """Dict of device tensors: samples [kappa, ita, U] int32 and, when
    requested, status [U] uint8, events [U] int64, seqhash [U] int64 (bit
    pattern of the uint64 hash), t_final [U] float64, score [U, R]
    float64."""

    def __getattr__(self, k):
        try:
            return self[k]
        except KeyError:
            raise AttributeError(k)

    def error_count(self):
        if 'status' not in self:
            return 0
        st = self['status']
        return int(sum(int((st == c).sum()) for c in ERROR_STATUSES))


def device_blob(model, device):
    torch = _torch()
    return torch.from_numpy(model.blob().view(np.int32)).to(device)


def simulate(model, n_traj, method='direct', seed=0, traj_id_base=0,
             mapping='auto', device=None, stream=None, status=True,
             events=True, seqhash=False, t_final=False, score=False,
             step_budget=DEFAULT_STEP_BUDGET, ssa_fallback_steps=100, max_leap_retries=63,
             block_size=0, out=None, d_blob=None, sorted_blocks=True,
             geometry=None):
    """Run ``n_traj`` trajectories of ``model`` (a :class:`Model`) on the GPU.

    Asynchronous on ``stream`` (default: torch's current stream).  ``out``
    may supply preallocated tensors by name; ``d_blob`` a device copy of
    ``model.blob()``.  ``sorted_blocks=False`` selects the simple
    one-trajectory-per-thread tau-leaping loop instead of the mode-sorted
    block scheduler (identical results).  ``geometry`` may set the sorted
    scheduler's ``round_ssa``, ``round_leap``, ``pool_slots`` and
    ``sorted_block`` (see :class:`py_stoch_b200.autotune.Autotuner`); it
    changes the speed, never the results.
    """
    torch = _torch()
    if score and getattr(model, 'has_laws', False):
        raise ValueError('likelihood-ratio scores need mass-action laws (a_j '
                         'proportional to its rate constant); this model has '
                         'general kinetic laws')
    device = torch.device(device or 'cuda')
    L = _lib.lib()
    meth = _method(method)
    n = int(n_traj)
    kappa, ita, R = model.kappa, model.ita, model.n_reactions
    out = dict(out or {})
    res = SimResult()

    def get(name, shape, dtype, want):
        if not want:
            return None
        t = out.get(name)
        if t is None:
            t = torch.empty(shape, dtype=dtype, device=device)
        res[name] = t
        return t

    smp = get('samples', (kappa, ita, n), torch.int32, True)
    st = get('status', (n,), torch.uint8, status)
    ev = get('events', (n,), torch.int64, events)
    sh = get('seqhash', (n,), torch.int64, seqhash)
    tf = get('t_final', (n,), torch.float64, t_final)
    sc = get('score', (n, R), torch.float64, score)
    h_blob = model.blob()
    if d_blob is None:
        d_blob = device_blob(model, device)
    o = _lib.Outputs(smp.data_ptr(), 0, st.data_ptr() if st is not None else 0,
                     ev.data_ptr() if ev is not None else 0,
                     sh.data_ptr() if sh is not None else 0,
                     tf.data_ptr() if tf is not None else 0,
                     sc.data_ptr() if sc is not None else 0)
    geo = dict(geometry or {})
    r = _lib.RunDesc(n, int(traj_id_base), int(seed) & 0xFFFFFFFFFFFFFFFF,
                     meth, _mapping(mapping), int(ssa_fallback_steps),
                     int(max_leap_retries), int(step_budget), int(block_size),
                     0 if sorted_blocks else _lib.FLAG_UNSORTED,
                     int(geo.pop('round_ssa', 0)),
                     int(geo.pop('round_leap', 0)),
                     int(geo.pop('pool_slots', 0)),
                     int(geo.pop('sorted_block', 0)))
    if geo:
        raise ValueError('unknown geometry keys: %s' % sorted(geo))
    if stream is None:
        stream = torch.cuda.current_stream(device)
    sptr = C.c_void_p(stream.cuda_stream)
    ws = out.get('workspace')
    if ws is None:
        ws = torch.empty(_lib.RUN_WORKSPACE_BYTES, dtype=torch.uint8,
                         device=device)
    fn = (L.pyst_ssa_direct_run if meth == _lib.METHOD_DIRECT
          else L.pyst_tau_leap_run)
    _lib.check(fn(h_blob.ctypes.data, d_blob.data_ptr(), C.byref(r),
                  C.byref(o), ws.data_ptr(), ws.numel(), sptr),
               'pyst_ssa_direct_run' if meth == _lib.METHOD_DIRECT
               else 'pyst_tau_leap_run')
    res['_keepalive'] = (d_blob, h_blob, ws)
    return res


# ---------------------------------------------------------------------------
# drop-in classes
# ---------------------------------------------------------------------------
class _DeviceData(object):
    """Limits the reference's calculate_sizes reads from
    ``pycuda.tools.DeviceData`` (per-block values on B200)."""
    max_threads = 1024
    shared_memory = 48 * 1024
    warp_size = 32


def _block_from_limit(limit, U):
    dd = _DeviceData
    max_threads = min(dd.max_threads, limit)
    warps = math.floor(max_threads / dd.warp_size)
    opt = warps * dd.warp_size
    if opt >= 256 and U >= 2560:
        block = 256
    elif opt >= 128 and U >= 1280:
        block = 128
    elif opt >= 64 and U >= 640:
        block = 64
    elif opt >= 32:
        block = 32
    else:
        block = opt
    if U <= 2:
        block = U
    return block


class Simulator(object):
    def calculate_sizes(self, tl_args):
        """Reference launch geometry (``mod/simulator/simulator.py:11-58``),
        including its operator-precedence reading of the shared-memory
        bound; rounds ``tl_args.U`` up to grid * block."""
        limit = math.floor(_DeviceData.shared_memory / (
            9 * tl_args.M + 8 * tl_args.N + 4 * len(tl_args.c)) + 10)
        return self._finish(tl_args, _block_from_limit(limit, tl_args.U))

    @staticmethod
    def _finish(tl_args, block):
        if block <= 0:
            # the reference divides by zero here for models whose shared
            # memory estimate exceeds 48 KiB; the engine has no such limit
            block = 32
        grid = int(math.ceil(float(tl_args.U) / float(block)))
        tl_args.U = int(grid * block)
        return grid, block


class StochasticSimulator(Simulator):
    @staticmethod
    def get_rng_states(size):
        """The reference allocates and seeds ``size`` MRG32k3a states
        (``simulator.py:62-96``).  The engine's Philox4x32-10 stream is
        stateless (keyed by seed and trajectory id), so there is nothing to
        allocate; returns None."""
        return None

    def __init__(self, seed=0, device=None):
        self.seed = int(seed)
        self.device = device

    def _run(self, my_args, method):
        torch = _torch()
        self.calculate_sizes(my_args)
        model = Model.from_tl_args(my_args)
        res = simulate(model, my_args.U, method=method, seed=self.seed,
                       device=self.device, status=True, events=False,
                       ssa_fallback_steps=100,
                       max_leap_retries=63)
        torch.cuda.current_stream(res['samples'].device).synchronize()
        n_err = res.error_count()
        if n_err:
            st = res['status'].cpu().numpy()
            codes = sorted(set(int(c) for c in st if c in ERROR_STATUSES))
            L = _lib.lib()
            raise RuntimeError(
                '%d of %d trajectories failed (%s)' % (
                    n_err, my_args.U,
                    ', '.join(L.pyst_traj_status_string(c).decode()
                              for c in codes)))
        self.last_result = res
        return res['samples'].cpu().numpy()


class CuGillespie(StochasticSimulator):
    """Direct-method SSA (``CuGillespie.run``, ``cuGillespie.py:16-46``)."""

    def calculate_sizes(self, tl_args):
        limit = math.floor(_DeviceData.shared_memory /
                           (8 * tl_args.M + 4 * tl_args.N + 22))
        return self._finish(tl_args, _block_from_limit(limit, tl_args.U))

    def run(self, my_args):
        return self._run(my_args, _lib.METHOD_DIRECT)


class CuTauLeaping(StochasticSimulator):
    """Adaptive tau-leaping with SSA fallback (``CuTauLeaping.run``,
    ``cuTauLeaping.py:18-84``); ``args.gillespie == 1`` forces the direct
    method as ``P1_P2.py:68-74`` does."""

    def calculate_sizes(self, tl_args):
        limit = math.floor(_DeviceData.shared_memory /
                           (16 * tl_args.M + 24 * tl_args.N + 10))
        return self._finish(tl_args, _block_from_limit(limit, tl_args.U))

    def run(self, my_args):
        meth = (_lib.METHOD_DIRECT if getattr(my_args, 'gillespie', 0)
                else _lib.METHOD_TAU_LEAP)
        return self._run(my_args, meth)
