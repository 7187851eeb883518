"""Model front-end against golden vectors produced by the reference's own
parser / Petri-net code (tests/golden/make_golden.py)."""

import json
import os

import numpy as np
import pytest

from conftest import reference_available, reference_dir
from py_stoch_b200 import parser, petri_net, sbml, sim_maker, simulator

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), 'golden',
                                     'frontend_golden.json')))


def arr(d):
    return np.array(d['data'], dtype=d['dtype']).reshape(d['shape'])


def _fixture_model(fx):
    if fx == 'lotkaVoltera_sbml.xml':
        return sbml.read_sbml_string(sbml.lotka_volterra_sbml())
    if fx == 'schlogl_sbmlv2.xml':
        return sbml.read_sbml_string(sbml.schlogl_sbml())
    if not reference_available():
        pytest.skip('fixture XML only in the reference checkout')
    return sbml.read_sbml(os.path.join(reference_dir(), 'examples', fx))


@pytest.mark.parametrize('fx', sorted(GOLDEN['fixtures']))
def test_spn_matches_reference(fx):
    g = GOLDEN['fixtures'][fx]['spn']
    spn = petri_net.SPN().sbml_2_stochastic_petri_net(_fixture_model(fx))
    np.testing.assert_array_equal(spn.Pre, arr(g['Pre']))
    np.testing.assert_array_equal(spn.Post, arr(g['Post']))
    np.testing.assert_array_equal(spn.StoichMConst, arr(g['StoichMConst']))
    assert list(spn.M) == g['M']
    assert list(spn.c) == g['c']
    assert spn.P == g['P']
    assert spn.T == g['T']
    assert spn.h == g['h']


@pytest.mark.parametrize('fx', sorted(GOLDEN['fixtures']))
def test_tl_args_match_reference(fx):
    g = GOLDEN['fixtures'][fx]
    spn = petri_net.SPN().sbml_2_stochastic_petri_net(_fixture_model(fx))
    args = parser.TlArgs()
    args.E = np.arange(len(spn.P)).astype(np.int32)
    args.t_max = 10
    args.ita = 11
    args.U = 1000
    args = parser.TlParser.parse(args, spn)
    ga = g['tl_args']
    for k in ('c', 'x_0', 'A', 'V', 'V_t', 'V_bar', 'H', 'H_type', 'E', 'I'):
        want = arr(ga[k])
        got = np.asarray(getattr(args, k))
        assert got.dtype == want.dtype, k
        np.testing.assert_array_equal(got, want, err_msg=k)
    for k in ('M', 'N', 'A_size', 'V_size', 'V_t_size', 'V_bar_size',
              'kappa', 't_max', 'ita', 'U', 'n_c', 'eta', 'gillespie'):
        assert getattr(args, k) == ga[k], k
    lines = sorted(l.strip() for l in args.hazards.splitlines()
                   if l.strip().startswith('a['))
    assert lines == g['hazard_lines']
    gargs = parser.GParser.parse(parser.GArgs(), spn)
    gg = g['g_args']
    for k in ('c', 'x_0', 'V'):
        np.testing.assert_array_equal(np.asarray(getattr(gargs, k)),
                                      arr(gg[k]))
    assert gargs.V_size == gg['V_size']


@pytest.mark.parametrize('i', range(len(GOLDEN['sweeps'])))
def test_sweep_points_match_reference(i):
    g = GOLDEN['sweeps'][i]
    model = _fixture_model(g['fixture'])
    lst = sim_maker.TLArgsList.make_list(
        model, g['species_init'], g['params'], g['output_species'],
        g['duration'], g['ita'], g['U'])
    assert len(lst) == len(g['points'])
    for a, p in zip(lst, g['points']):
        np.testing.assert_array_equal(a.x_0, arr(p['x_0']))
        np.testing.assert_array_equal(a.c, arr(p['c']))
        np.testing.assert_array_equal(a.I, arr(p['I']))
    assert sim_maker.rest_list(g['params']) == g['rest_list_params']


def test_calculate_sizes_match_reference():
    import types
    classes = {'CuTauLeaping': simulator.CuTauLeaping,
               'CuGillespie': simulator.CuGillespie}
    for rec in GOLDEN['calculate_sizes']:
        a = types.SimpleNamespace(M=rec['M'], N=rec['N'],
                                  c=[0.0] * rec['P'], U=rec['U_in'])
        grid, block = classes[rec['cls']]().calculate_sizes(a)
        if 'error' in rec:
            # the reference divides by zero; the engine picks 32 threads
            assert block == 32
            continue
        assert (grid, block, a.U) == (rec['grid'], rec['block'],
                                      rec['U_out']), rec


def test_flatten_limits_raise():
    big = np.zeros((130, 2))
    big[129, 0] = 1
    with pytest.raises(parser.EncodingLimitError):
        parser.Parser.flatten_matrix(big)
    many = np.ones((16, 17))
    with pytest.raises(parser.EncodingLimitError):
        parser.Parser.flatten_matrix(many)


def test_parse_settings(tmp_path):
    p = tmp_path / 's.xml'
    p.write_text('<settings><output_species><species idx="0"/>'
                 '<species idx="2"/></output_species><duration>5.5'
                 '</duration><num_output_time_points>7'
                 '</num_output_time_points><num_simulations>64'
                 '</num_simulations></settings>')
    a = parser.TlArgs()
    parser.Parser.parse_settings(str(p), a)
    assert list(a.E) == [0, 2] and a.t_max == 5.5 and a.ita == 7
    assert a.U == 64


def test_sbml_errors_raise(tmp_path):
    p = tmp_path / 'bad.xml'
    p.write_text('<sbml><model><listOfReactions><reaction id="r">'
                 '<kineticLaw><math><apply><csymbol/></apply></math>'
                 '</kineticLaw></reaction></listOfReactions></model></sbml>')
    with pytest.raises(UserWarning):
        sbml.read_sbml(str(p))
    with pytest.raises(UserWarning):
        sbml.read_sbml(str(tmp_path / 'missing.xml'))


def test_mathml_printing_roundtrip():
    m = sbml.read_sbml_string(sbml.write_sbml(
        'm', [('A', 5), ('B', 7)], [('k', 2.5)],
        [('r', [('A', 1)], [('B', 1)], 'k * A * (B - 1) / (2 + A) ^ 2')]))
    law = m.getListOfReactions()[0].getKineticLaw().getMath()
    s = sbml.formulaToL3String(law)
    assert s == 'k * A * (B - 1) / (2 + A) ^ 2'
    v = sbml.evaluate(law, {'k': 2.5, 'A': 5, 'B': 7})
    assert abs(v - 2.5 * 5 * 6 / 49.0) < 1e-12
