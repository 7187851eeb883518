"""Python access to the CPU oracle (test infrastructure only).

The oracle is the checker the GPU engine is compared against; it is never
part of the product path.  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline / reference legs may import this module.

* :func:`build` compiles ``pyst_oracle.c`` into ``liboracle.so`` (gcc).
* :func:`simulate` runs trajectories of a model on host threads.
* :func:`philox_np` is a second, NumPy restatement of Philox4x32-10 (Salmon
  et al., SC'11) used to pin both the C oracle and the device generator to
  the published known-answer vectors in :data:`PHILOX_KAT`.
"""

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, 'pyst_oracle.c')
LIB = os.path.join(HERE, 'liboracle.so')

# Philox4x32-10 known-answer vectors (Random123 kat_vectors, SC'11):
# (counter[4], key[2]) -> output[4]
PHILOX_KAT = [
    ((0x00000000, 0x00000000, 0x00000000, 0x00000000),
     (0x00000000, 0x00000000),
     (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
    ((0xffffffff, 0xffffffff, 0xffffffff, 0xffffffff),
     (0xffffffff, 0xffffffff),
     (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
    ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344),
     (0xa4093822, 0x299f31d0),
     (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
]


def philox_np(ctr, key):
    """Philox4x32-10 of counter rows ``ctr`` [n,4] and keys ``key`` [n,2]
    (uint32), vectorised in NumPy uint64 arithmetic."""
    c = np.array(ctr, dtype=np.uint64).reshape(-1, 4).copy()
    k = np.array(key, dtype=np.uint64).reshape(-1, 2).copy()
    M0, M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
    W0, W1 = np.uint64(0x9E3779B9), np.uint64(0xBB67AE85)
    mask = np.uint64(0xFFFFFFFF)
    s32 = np.uint64(32)
    for r in range(10):
        if r:
            k[:, 0] = (k[:, 0] + W0) & mask
            k[:, 1] = (k[:, 1] + W1) & mask
        p0 = M0 * c[:, 0]
        p1 = M1 * c[:, 2]
        hi0, lo0 = p0 >> s32, p0 & mask
        hi1, lo1 = p1 >> s32, p1 & mask
        n0 = hi1 ^ c[:, 1] ^ k[:, 0]
        n2 = hi0 ^ c[:, 3] ^ k[:, 1]
        c = np.stack([n0, lo1, n2, lo0], axis=1)
    return c.astype(np.uint32)


class _OModel(C.Structure):
    _fields_ = [('S', C.c_int), ('R', C.c_int), ('kappa', C.c_int),
                ('ita', C.c_int), ('order', C.c_void_p),
                ('falling', C.c_void_p), ('pre', C.c_void_p),
                ('net', C.c_void_p), ('rate', C.c_void_p),
                ('x0', C.c_void_p), ('hor', C.c_void_p),
                ('hor_type', C.c_void_p), ('times', C.c_void_p),
                ('out', C.c_void_p), ('eta', C.c_float), ('n_c', C.c_int),
                ('law_ptr', C.c_void_p), ('law_code', C.c_void_p),
                ('law_const', C.c_void_p)]


class _ORun(C.Structure):
    _fields_ = [('seed', C.c_uint64), ('id_base', C.c_int64),
                ('method', C.c_int), ('warp', C.c_int),
                ('ssa_fallback', C.c_int), ('max_retries', C.c_int),
                ('step_budget', C.c_int64)]


class _OOut(C.Structure):
    _fields_ = [('samples', C.c_void_p), ('n', C.c_int64),
                ('status', C.c_void_p), ('events', C.c_void_p),
                ('seqhash', C.c_void_p), ('t_final', C.c_void_p),
                ('score', C.c_void_p), ('steps', C.c_void_p)]


_lib = None


CFLAGS = ['-O2', '-fPIC', '-ffp-contract=off', '-fno-fast-math', '-std=c11',
          '-shared']
STAMP = LIB + '.stamp'


def _source_hash():
    import hashlib
    with open(SRC, 'rb') as f:
        return hashlib.sha1(' '.join(CFLAGS).encode() + f.read()).hexdigest()


def build(force=False):
    """Compile liboracle.so unless its stamp holds the source's content
    hash (modification times are not trusted across copies of the tree)."""
    h = _source_hash()
    if not force and os.path.exists(LIB) and os.path.exists(STAMP):
        with open(STAMP) as f:
            if f.read().strip() == h:
                return LIB
    cc = os.environ.get('CC', 'gcc')
    subprocess.check_call([cc] + CFLAGS + ['-o', LIB + '.tmp', SRC, '-lm',
                                           '-lpthread'])
    os.replace(LIB + '.tmp', LIB)
    with open(STAMP, 'w') as f:
        f.write(h + '\n')
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        L.oracle_simulate.restype = C.c_int
        L.oracle_simulate.argtypes = [C.POINTER(_OModel), C.POINTER(_ORun),
                                      C.POINTER(_OOut), C.c_int64, C.c_int64,
                                      C.c_int]
        L.oracle_philox.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_philox_stream.argtypes = [C.c_uint64, C.c_uint64,
                                           C.c_uint64, C.c_int64, C.c_void_p]
        L.oracle_math.argtypes = [C.c_void_p, C.c_int64, C.c_int,
                                  C.c_void_p]
        L.oracle_poisson_batch.argtypes = [C.c_void_p, C.c_int64, C.c_uint64,
                                           C.c_void_p]
        L.oracle_max_threads.restype = C.c_int
        _lib = L
    return _lib


def max_threads():
    return int(lib().oracle_max_threads())


def philox_c(ctr, key):
    ctr = np.ascontiguousarray(ctr, dtype=np.uint32).reshape(-1, 4)
    key = np.ascontiguousarray(key, dtype=np.uint32).reshape(-1, 2)
    out = np.zeros_like(ctr)
    for i in range(ctr.shape[0]):
        lib().oracle_philox(ctr[i].ctypes.data, key[i].ctypes.data,
                            out[i].ctypes.data)
    return out


def philox_stream(seed, traj_id, n0, count):
    out = np.zeros((count, 4), dtype=np.uint32)
    lib().oracle_philox_stream(seed, traj_id, n0, count, out.ctypes.data)
    return out


def math(x, which):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros_like(x)
    lib().oracle_math(x.ctypes.data, x.size, which, out.ctypes.data)
    return out


def poisson(lam, seed):
    lam = np.ascontiguousarray(lam, dtype=np.float32)
    out = np.zeros(lam.shape, dtype=np.int32)
    lib().oracle_poisson_batch(lam.ctypes.data, lam.size, seed,
                               out.ctypes.data)
    return out


def simulate(model, n_traj, method, seed=0, traj_id_base=0, warp=False,
             ssa_fallback_steps=100, max_leap_retries=63, step_budget=0,
             u0=0, u1=None, threads=0):
    """Run trajectories [u0, u1) of ``n_traj`` on the host.

    ``model`` is anything with the dense fields of
    :class:`py_stoch_b200.model.Model` (order, falling, pre, net, rate, x0,
    hor, hor_type, sample_times, out_species, eta, n_c).  ``method`` 0 is the
    direct method, 1 tau-leaping; ``warp`` selects the summation and
    selection order of the warp-per-trajectory kernels.  Returns a dict of
    NumPy arrays shaped like the GPU outputs (samples [kappa, ita, n_traj]);
    rows outside [u0, u1) are left zero.
    """
    u1 = n_traj if u1 is None else u1
    S, R = model.order.shape
    keep = []

    def arr(a, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return a.ctypes.data

    om = _OModel(S, R, len(model.out_species), len(model.sample_times),
                 arr(model.order, np.int32), arr(model.falling, np.uint8),
                 arr(model.pre, np.int32), arr(model.net, np.int32),
                 arr(model.rate, np.float64), arr(model.x0, np.int32),
                 arr(model.hor, np.int32), arr(model.hor_type, np.int32),
                 arr(model.sample_times, np.float32),
                 arr(model.out_species, np.int32), float(model.eta),
                 int(model.n_c))
    if getattr(model, 'laws', None) is not None:
        ptr, code, consts = model.law_arrays()
        om.law_ptr = arr(ptr, np.int32)
        om.law_code = arr(code if code.size else np.zeros(1, np.uint32),
                          np.uint32)
        om.law_const = arr(consts if consts.size else np.zeros(1),
                           np.float64)
    ru = _ORun(int(seed), int(traj_id_base), int(method), 1 if warp else 0,
               int(ssa_fallback_steps), int(max_leap_retries),
               int(step_budget))
    kappa, ita = len(model.out_species), len(model.sample_times)
    res = {
        'samples': np.zeros((kappa, ita, n_traj), dtype=np.int32),
        'status': np.zeros(n_traj, dtype=np.uint8),
        'events': np.zeros(n_traj, dtype=np.int64),
        'seqhash': np.zeros(n_traj, dtype=np.uint64),
        't_final': np.zeros(n_traj, dtype=np.float64),
        'score': np.zeros((n_traj, R), dtype=np.float64),
        # SSA steps, leaps, inversion Poisson draws and their search
        # iterations, PTRS draws and their iterations
        'steps': np.zeros((n_traj, 6), dtype=np.int64),
    }
    oo = _OOut(res['samples'].ctypes.data, n_traj,
               res['status'].ctypes.data, res['events'].ctypes.data,
               res['seqhash'].ctypes.data, res['t_final'].ctypes.data,
               res['score'].ctypes.data, res['steps'].ctypes.data)
    rc = lib().oracle_simulate(C.byref(om), C.byref(ru), C.byref(oo), u0, u1,
                               int(threads))
    if rc != 0:
        raise RuntimeError('oracle_simulate failed with %d' % rc)
    return res
