"""The reference's six example models (examples/*.xml), rebuilt from the
front-end golden vectors (tests/golden/frontend_golden.json: the SPN and
TlArgs the reference's own parser produced for each file), run on the GPU
with both methods and compared bit for bit with the CPU oracle.
"""

import json
import os
import types

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, 'golden', 'frontend_golden.json')


def _arr(d):
    return np.asarray(d['data'], dtype=d['dtype']).reshape(d['shape'])


def _fixtures():
    with open(GOLDEN) as f:
        return json.load(f)['fixtures']


def _model(name):
    from py_stoch_b200.model import Model
    fx = _fixtures()[name]
    spn, tl = fx['spn'], fx['tl_args']
    args = types.SimpleNamespace(
        pre_matrix=_arr(spn['Pre']).astype(np.int64),
        post_matrix=_arr(spn['Post']).astype(np.int64),
        hazard_exprs=list(spn['h']), c=_arr(tl['c']), x_0=_arr(tl['x_0']),
        I=_arr(tl['I']), E=_arr(tl['E']), H=_arr(tl['H']),
        H_type=_arr(tl['H_type']), t_max=tl['t_max'], eta=tl['eta'],
        n_c=tl['n_c'])
    return Model.from_tl_args(args)


NAMES = sorted(_fixtures())


@pytest.mark.parametrize('name', NAMES)
def test_fixture_models_build(name):
    m = _model(name)
    assert m.n_reactions == len(_fixtures()[name]['spn']['h'])
    assert m.blob().size > 0


@pytest.mark.gpu
@pytest.mark.parametrize('name', NAMES)
@pytest.mark.parametrize('method', ['direct', 'tau'])
def test_fixture_models_bit_exact(torch_cuda, built_lib, oracle_mod, name,
                                  method):
    from py_stoch_b200.simulator import simulate
    m = _model(name)
    n = 256
    # cdi and plasmid grow without bound at these parameters: both sides
    # stop them at the same step of the budget (PYST_TRAJ_STEP_BUDGET)
    budget = 100000
    res = simulate(m, n, method=method, seed=17, status=True, events=True,
                   seqhash=True, step_budget=budget)
    torch_cuda.cuda.synchronize()
    o = oracle_mod.simulate(m, n, 0 if method == 'direct' else 1, seed=17,
                            step_budget=budget)
    np.testing.assert_array_equal(res['status'].cpu().numpy(), o['status'])
    np.testing.assert_array_equal(res['events'].cpu().numpy(), o['events'])
    np.testing.assert_array_equal(
        res['seqhash'].cpu().numpy().view(np.uint64), o['seqhash'])
    np.testing.assert_array_equal(res['samples'].cpu().numpy(),
                                  o['samples'])
