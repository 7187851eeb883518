"""The C ABI library: loads without a GPU, exports every function the public
headers declare, and rejects bad arguments before any CUDA call."""

import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

from py_stoch_b200 import _lib, networks

INCLUDE = os.path.join(os.path.dirname(os.path.dirname(
    os.path.abspath(__file__))), 'include')


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(INCLUDE, '*.h')):
        text = open(h).read()
        text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
        for m in re.finditer(r'^\s*(?:const\s+)?\w+\s*\*?\s*(pyst_\w+)\s*\(',
                             text, flags=re.M):
            names.add(m.group(1))
    return names


def test_exports_every_declared_symbol(built_lib):
    names = declared_functions()
    assert 'pyst_tau_leap_run' in names and 'pyst_batch_run' in names
    for n in names:
        assert hasattr(built_lib, n), n
        assert n in _lib.SIGNATURES, n


def test_version_and_strings(built_lib):
    assert built_lib.pyst_abi_version() == _lib.ABI_VERSION == 3
    for code in range(6):
        assert built_lib.pyst_status_string(code) != b'unknown status'
    for code in range(9):
        assert built_lib.pyst_traj_status_string(code) != (
            b'unknown trajectory status')


def _run_args():
    r = _lib.RunDesc(16, 0, 1, 0, 0, 100, 63, 0, 0, 0, 0, 0, 0, 0)
    o = _lib.Outputs(0, 0, 0, 0, 0, 0, 0)
    return r, o


def test_run_rejects_bad_arguments(built_lib):
    L = built_lib
    m = networks.lotka_volterra()
    blob = m.blob()
    r, o = _run_args()
    # null host blob
    assert L.pyst_ssa_direct_run(None, 16, C.byref(r), C.byref(o), 8, 256,
                                 None) == _lib.PYST_EINVAL
    # corrupt magic
    bad = blob.copy()
    bad[0] = 0
    assert L.pyst_ssa_direct_run(bad.ctypes.data, 16, C.byref(r), C.byref(o),
                                 8, 256, None) == _lib.PYST_EINVAL
    # misaligned device blob pointer, null samples, missing workspace
    assert L.pyst_ssa_direct_run(blob.ctypes.data, 17, C.byref(r),
                                 C.byref(o), 8, 256,
                                 None) == _lib.PYST_EINVAL
    o.samples = 4096
    assert L.pyst_ssa_direct_run(blob.ctypes.data, 16, C.byref(r),
                                 C.byref(o), None, 256,
                                 None) == _lib.PYST_EINVAL
    assert L.pyst_ssa_direct_run(blob.ctypes.data, 16, C.byref(r),
                                 C.byref(o), 8, 16,
                                 None) == _lib.PYST_EWORKSPACE
    # method mismatch and invalid tau parameters
    assert L.pyst_tau_leap_run(blob.ctypes.data, 16, C.byref(r), C.byref(o),
                               8, 256, None) == _lib.PYST_EINVAL
    r.method = 1
    r.max_leap_retries = 64
    assert L.pyst_tau_leap_run(blob.ctypes.data, 16, C.byref(r), C.byref(o),
                               8, 256, None) == _lib.PYST_EINVAL
    r.max_leap_retries = 63
    r.ssa_fallback_steps = 0
    assert L.pyst_tau_leap_run(blob.ctypes.data, 16, C.byref(r), C.byref(o),
                               8, 256, None) == _lib.PYST_EINVAL
    r.ssa_fallback_steps = 100
    r.block_size = 100
    assert L.pyst_tau_leap_run(blob.ctypes.data, 16, C.byref(r), C.byref(o),
                               8, 256, None) == _lib.PYST_EINVAL
    r.block_size = 0
    # sorted-scheduler geometry: slots 1..2, blocks 64..896 in whole warps
    for field, bad in (('pool_slots', 3), ('pool_slots', -1),
                       ('sorted_block', 32), ('sorted_block', 100),
                       ('sorted_block', 928), ('round_ssa', -1),
                       ('round_leap', -2)):
        setattr(r, field, bad)
        assert L.pyst_tau_leap_run(blob.ctypes.data, 16, C.byref(r),
                                   C.byref(o), 8, 256,
                                   None) == _lib.PYST_EINVAL, field
        setattr(r, field, 0)
    # thread mapping with scores on a model with too many reactions
    big = networks.synthetic_networks(1, seed=1, r_range=(100, 100))[0]
    r.block_size = 0
    r.mapping = _lib.MAP_THREAD
    o.score = 4096
    assert L.pyst_tau_leap_run(big.blob().ctypes.data, 16, C.byref(r),
                               C.byref(o), 8, 256,
                               None) == _lib.PYST_EUNSUPPORTED
    o.score = 0
    ws = C.c_size_t(0)
    assert L.pyst_run_workspace_size(C.byref(r), C.byref(ws)) == 0
    assert ws.value == _lib.RUN_WORKSPACE_BYTES


def _law_model():
    """Birth-death whose death hazard is the general law k1 * |x|."""
    from py_stoch_b200 import kinetic
    from py_stoch_b200.model import Model
    code, consts, _ = kinetic.compile_law('parameter_1 * abs(species_0)', 1,
                                          [2000.0, 0.5])
    return Model([[0, 0]], [[0, 1]], [[1, -1]], [2000.0, 0.0], [0],
                 np.linspace(0, 1, 5).astype(np.float32), [0],
                 laws=[None, (code, consts)])


def test_scores_refused_for_general_laws(built_lib):
    """N_j - int a_j dt is d log p / d log rate_j only for mass action: the
    run calls refuse scores for a model with a general kinetic law (before
    any CUDA call), and accept the same call without scores."""
    L = built_lib
    m = _law_model()
    assert m.has_laws
    blob = m.blob()
    r, o = _run_args()
    o.samples = 4096
    o.score = 4096
    for fn, meth in ((L.pyst_ssa_direct_run, 0), (L.pyst_tau_leap_run, 1)):
        r.method = meth
        assert fn(blob.ctypes.data, 16, C.byref(r), C.byref(o), 8, 256,
                  None) == _lib.PYST_EUNSUPPORTED
    # n_traj 0 with scores is refused too; without scores it is a no-op
    r.n_traj = 0
    assert L.pyst_tau_leap_run(blob.ctypes.data, 16, C.byref(r), C.byref(o),
                               8, 256, None) == _lib.PYST_EUNSUPPORTED
    o.score = 0
    assert L.pyst_tau_leap_run(blob.ctypes.data, 16, C.byref(r), C.byref(o),
                               8, 256, None) == _lib.PYST_OK


def test_batch_and_backward_reject(built_lib):
    L = built_lib
    r, o = _run_args()
    lim = _lib.BatchLimits(0, 1, 1, 0)
    assert L.pyst_batch_run(None, None, 1, C.byref(lim), C.byref(r),
                            C.byref(o), None, 0, None) == _lib.PYST_EINVAL
    o.samples = 4096
    assert L.pyst_batch_run(16, 16, 1, C.byref(lim), C.byref(r), C.byref(o),
                            8, 512, None) == _lib.PYST_EUNSUPPORTED
    lim = _lib.BatchLimits(64, 1, 1, 0)
    assert L.pyst_batch_run(16, 16, 1, C.byref(lim), C.byref(r), C.byref(o),
                            8, 8, None) == _lib.PYST_EWORKSPACE
    # the workspace holds a completion counter per item (split models)
    ws = C.c_size_t(0)
    assert L.pyst_batch_workspace_size(1000, C.byref(ws)) == 0
    assert ws.value == _lib.RUN_WORKSPACE_BYTES + 4 * 1000
    assert L.pyst_batch_run(16, 16, 1000, C.byref(lim), C.byref(r),
                            C.byref(o), 8, ws.value - 1,
                            None) == _lib.PYST_EWORKSPACE
    assert C.sizeof(_lib.BatchItem) == 96
    ws = C.c_size_t(0)
    assert L.pyst_score_backward_workspace_size(1000, 6, C.byref(ws)) == 0
    assert ws.value == 4 * 6 * 8
    assert L.pyst_score_backward(None, None, 10, 1, 1, 1, None, None, None,
                                 None, None, None, 0,
                                 None) == _lib.PYST_EINVAL
    assert L.pyst_score_backward(8, 8, 10, 1, 1, 1, 8, None, 8, 8, 8, 8,
                                 4096, None) == _lib.PYST_EINVAL


def test_blob_size_query_matches_build(built_lib):
    m = networks.schlogl()
    d = m.desc()
    n = C.c_int64(0)
    assert built_lib.pyst_model_blob_words(C.byref(d), C.byref(n)) == 0
    buf = np.zeros(n.value - 4, np.uint32)
    assert built_lib.pyst_model_build(C.byref(d), buf.ctypes.data,
                                      buf.size) == _lib.PYST_EINVAL
    assert len(m.blob()) == n.value


def _packable_py(m):
    """Restatement of the packing conditions: at most two reactant entries
    of order 1..3 and two net-change entries with -16 <= delta <= 15, over
    species < 1024, and no general kinetic laws."""
    if m.has_laws:
        return False
    for j in range(m.n_reactions):
        fac = [i for i in range(m.n_species) if m.order[i, j] > 0]
        net = [i for i in range(m.n_species) if m.net[i, j] != 0]
        if len(fac) > 2 or len(net) > 2:
            return False
        if any(m.order[i, j] > 3 or i > 1023 for i in fac):
            return False
        if any(not -16 <= m.net[i, j] <= 15 or i > 1023 for i in net):
            return False
    return True


def test_host_packable_predicate(built_lib):
    """The host's packability decision (which picks the lane-tree kernel)
    against a restatement, on models at every boundary."""
    from py_stoch_b200.model import Model
    cases = [networks.lotka_volterra(), networks.schlogl(),
             networks.telegraph(), _law_model()]
    t = np.linspace(0, 1, 3).astype(np.float32)
    for delta in (15, 16, -16, -17):
        pre = [[1], [0]]
        post = [[1 + delta if delta > 0 else 1], [0]]
        if delta < 0:
            pre, post = [[-delta], [0]], [[0], [0]]
        cases.append(Model.mass_action(pre, post, [1.0], [100, 5], t))
    for order in (3, 4):
        cases.append(Model.mass_action([[order]], [[order + 1]], [1.0],
                                       [50], t))
    # three reactant species, three net-change species
    cases.append(Model.mass_action([[1], [1], [1]], [[0], [0], [2]], [1.0],
                                   [9, 9, 9], t))
    cases.append(Model.mass_action([[1], [0], [0]], [[0], [1], [1]], [1.0],
                                   [9, 0, 0], t))
    cases += networks.synthetic_networks(6, seed=4)
    seen = set()
    for m in cases:
        want = _packable_py(m)
        seen.add(want)
        assert built_lib.pyst_test_model_packable(m.blob().ctypes.data) == \
            int(want), m.name
    assert seen == {True, False}
