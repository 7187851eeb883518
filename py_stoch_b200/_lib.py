"""ctypes binding of libpystoch_b200.so (include/pystoch_b200.h).

The library is built in-tree (``python -m py_stoch_b200.build``).  Loading it
needs no GPU; the run entry points do.  There is no fallback: if the library
is missing, :func:`lib` raises.
"""

import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, 'libpystoch_b200.so')

PYST_OK = 0
PYST_EINVAL = 1
PYST_ECUDA = 2
PYST_EUNSUPPORTED = 3
PYST_EWORKSPACE = 4
PYST_ETRAJ = 5

TRAJ_DONE = 0
TRAJ_ABSORBED = 1
TRAJ_STEP_BUDGET = 2
TRAJ_OVERFLOW = 3
TRAJ_LEAP_RETRY = 4
TRAJ_SAMPLER = 5
TRAJ_STAGING = 6
TRAJ_RATE = 7
TRAJ_UNSUPPORTED = 8

METHOD_DIRECT = 0
METHOD_TAU_LEAP = 1
MAP_AUTO = 0
MAP_THREAD = 1
MAP_WARP = 2
FLAG_UNSORTED = 1

MAX_SPECIES = 1024
MAX_REACTIONS = 4096
THREAD_MAX_REACTIONS = 32
MAX_BLOB_WORDS = 12288
RUN_WORKSPACE_BYTES = 256
ABI_VERSION = 3
NOALLOC_SCRATCH_BYTES = 1 << 20
SCORE_CHUNK = 256
SUMS_MAX_TRAJ = 2**31 - 1

# header word indices (PYST_H_*)
H_MAGIC, H_WORDS, H_S, H_R, H_KAPPA, H_ITA = 0, 1, 2, 3, 4, 5
BLOB_MAGIC = 0x31545950

_p = C.c_void_p


class ModelDesc(C.Structure):
    _fields_ = [('n_species', C.c_int32), ('n_reactions', C.c_int32),
                ('order', _p), ('falling', _p), ('pre', _p),
                ('net_change', _p), ('rate', _p), ('x0', _p), ('hor', _p),
                ('hor_type', _p), ('sample_times', _p),
                ('n_samples', C.c_int32), ('out_species', _p),
                ('n_out', C.c_int32), ('t_max', C.c_double),
                ('eta', C.c_float), ('n_c', C.c_int32),
                ('law_ptr', _p), ('law_code', _p), ('law_const', _p),
                ('n_law_const', C.c_int32)]


class RunDesc(C.Structure):
    _fields_ = [('n_traj', C.c_int64), ('traj_id_base', C.c_int64),
                ('seed', C.c_uint64), ('method', C.c_int32),
                ('mapping', C.c_int32), ('ssa_fallback_steps', C.c_int32),
                ('max_leap_retries', C.c_int32), ('step_budget', C.c_int64),
                ('block_size', C.c_int32), ('flags', C.c_int32),
                ('round_ssa', C.c_int32), ('round_leap', C.c_int32),
                ('pool_slots', C.c_int32), ('sorted_block', C.c_int32)]


class Outputs(C.Structure):
    _fields_ = [('samples', _p), ('out_stride', C.c_int64), ('status', _p),
                ('events', _p), ('seqhash', _p), ('t_final', _p),
                ('score', _p), ('stats', _p), ('jacobian', _p)]


class BatchItem(C.Structure):
    _fields_ = [('blob_offset', C.c_int64), ('n_traj', C.c_int64),
                ('traj_id_base', C.c_int64), ('sample_offset', C.c_int64),
                ('traj_offset', C.c_int64), ('score_offset', C.c_int64),
                ('stats_offset', C.c_int64), ('jac_offset', C.c_int64),
                ('method', C.c_int32), ('mapping', C.c_int32),
                ('chunk_begin', C.c_int64), ('model_n_traj', C.c_int64),
                ('group', C.c_int32), ('group_chunks', C.c_int32)]


class BatchLimits(C.Structure):
    _fields_ = [('max_blob_words', C.c_int32), ('max_species', C.c_int32),
                ('max_reactions', C.c_int32), ('reserved', C.c_int32)]


# name -> (restype, argtypes); every symbol include/*.h declares
SIGNATURES = {
    'pyst_abi_version': (C.c_int, []),
    'pyst_status_string': (C.c_char_p, [C.c_int]),
    'pyst_traj_status_string': (C.c_char_p, [C.c_int]),
    'pyst_model_blob_words': (C.c_int, [C.POINTER(ModelDesc),
                                        C.POINTER(C.c_int64)]),
    'pyst_model_build': (C.c_int, [C.POINTER(ModelDesc), _p, C.c_int64]),
    'pyst_run_workspace_size': (C.c_int, [C.POINTER(RunDesc),
                                          C.POINTER(C.c_size_t)]),
    'pyst_ssa_direct_run': (C.c_int, [_p, _p, C.POINTER(RunDesc),
                                      C.POINTER(Outputs), _p, C.c_size_t,
                                      _p]),
    'pyst_tau_leap_run': (C.c_int, [_p, _p, C.POINTER(RunDesc),
                                    C.POINTER(Outputs), _p, C.c_size_t,
                                    _p]),
    'pyst_batch_workspace_size': (C.c_int, [C.c_int64,
                                            C.POINTER(C.c_size_t)]),
    'pyst_batch_run': (C.c_int, [_p, _p, C.c_int64, C.POINTER(BatchLimits),
                                 C.POINTER(RunDesc), C.POINTER(Outputs), _p,
                                 C.c_size_t, _p]),
    'pyst_score_backward_workspace_size': (C.c_int, [
        C.c_int64, C.c_int32, C.POINTER(C.c_size_t)]),
    'pyst_score_backward': (C.c_int, [_p, _p, C.c_int64, C.c_int32,
                                      C.c_int32, C.c_int32, _p, _p, _p, _p,
                                      _p, _p, C.c_size_t, _p]),
    'pyst_score_backward_noalloc': (C.c_int, [_p, _p, C.c_int64, C.c_int32,
                                              C.c_int32, C.c_int32, _p, _p,
                                              _p, _p, _p, _p]),
    'pyst_sample_sums': (C.c_int, [_p, C.c_int64, C.c_int64, C.c_int32,
                                   C.c_int32, _p, _p]),
    'pyst_moments_from_sums': (C.c_int, [_p, C.c_int32, C.c_int64, _p, _p,
                                         _p]),
    'pyst_score_partials': (C.c_int, [_p, _p, C.c_int64, C.c_int32,
                                      C.c_int32, C.c_int32, _p, _p, _p, _p,
                                      _p, _p]),
    'pyst_score_combine': (C.c_int, [_p, C.c_int64, C.c_int32, C.c_int64,
                                     _p, _p]),
    'pyst_test_philox': (C.c_int, [C.c_uint64, C.c_uint64, C.c_uint64,
                                   C.c_int64, _p, _p]),
    'pyst_test_philox_raw': (C.c_int, [_p, C.c_int64, _p, C.c_int, _p]),
    'pyst_test_math': (C.c_int, [_p, C.c_int64, C.c_int, _p, _p]),
    'pyst_test_poisson': (C.c_int, [_p, C.c_int64, C.c_uint64, _p, _p]),
    'pyst_test_set_staging_polls': (C.c_int, [C.c_int32]),
    'pyst_test_model_packable': (C.c_int, [_p]),
    'pyst_test_pipe': (C.c_int, [C.c_int32, C.c_int32, C.c_int32, _p, _p]),
}

_lock = threading.Lock()
_lib = None


class PystError(RuntimeError):
    def __init__(self, code, where):
        self.code = code
        msg = 'unknown status'
        if _lib is not None:
            msg = _lib.pyst_status_string(code).decode()
        super().__init__('%s failed: %s (code %d)' % (where, msg, code))


def lib():
    """Load (once) and return the library with argtypes set."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    'libpystoch_b200.so is not built; run '
                    '`python -m py_stoch_b200.build` (or '
                    '__graft_entry__.build())')
            L = C.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
    return _lib


def check(code, where):
    if code != PYST_OK:
        raise PystError(code, where)
