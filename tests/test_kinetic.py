"""General kinetic laws: the compiler (py_stoch_b200/kinetic.py), the
packer's program checks, the oracle's evaluation and the SBML front end.

The reference evaluates each hazard as C source (mod/parser/parser.py:32-55),
so laws follow C typing: species and integer literals are integers, and a
division of two integers truncates toward zero.
"""

import math

import numpy as np
import pytest

from py_stoch_b200 import kinetic


def _eval(text, x, p):
    code, consts, _ = kinetic.compile_law(text, len(x), p)
    return kinetic.evaluate(code, consts, x)


@pytest.mark.parametrize('text,x,p,want', [
    ('parameter_0 * species_0 / (parameter_1 + species_0)', [7], [2.5, 3.0],
     2.5 * 7 / 10.0),
    ('species_0 / 2 * parameter_0', [7], [3.0], 9.0),          # C: 7/2 = 3
    ('-species_0 / 2', [7], [], -3.0),                        # truncation
    ('species_0 / 2.0 * parameter_0', [7], [3.0], 10.5),       # double
    ('species_0 ^ 2 + pow(species_1, 3)', [3, 2], [], 17.0),
    ('floor(parameter_0 * species_0) + ceil(0.5) + abs(-species_1)', [3, 4],
     [0.7], 7.0),
    ('(species_0 - 1) * (species_0 - 2) / 2', [6], [], 10.0),
])
def test_compiled_laws_follow_c_semantics(text, x, p, want):
    assert _eval(text, x, p) == want


def test_transcendental_functions():
    assert math.isclose(_eval('exp(ln(parameter_0)) * sqrt(species_0)', [16],
                              [2.0]), 8.0, rel_tol=1e-15)
    assert math.isclose(_eval('log10(species_0)', [100], []), 2.0,
                        rel_tol=1e-15)
    assert math.isclose(_eval('species_0 ^ 0.5', [9], []), 3.0,
                        rel_tol=1e-15)


@pytest.mark.parametrize('text', [
    'species_0 * unknown', 'sin(species_0)', 'species_0 +', '(species_0',
    'species_9', 'parameter_3', 'pow(species_0)',
    'species_0*(species_0*(species_0*(species_0*(species_0*(species_0*'
    '(species_0*(species_0*(species_0*species_0))))))))',
])
def test_compile_errors(text):
    with pytest.raises(kinetic.KineticLawError):
        kinetic.compile_law(text, 1, [1.0])


def test_integer_division_detection():
    assert kinetic.has_int_division('species_0 / 2 * parameter_0', 1, 1)
    assert not kinetic.has_int_division('parameter_0 / 2 * species_0', 1, 1)
    assert not kinetic.has_int_division('species_0 / 2.0', 1, 0)


def _birth_death(death_law, k0=20.0, k1=0.5, t_end=4.0, n_samples=9):
    """0 -> X at k0 (mass action), X -> 0 with the given law."""
    from py_stoch_b200.model import Model
    times = np.linspace(0.0, t_end, n_samples).astype(np.float32)
    code, consts, _ = kinetic.compile_law(death_law, 1, [k0, k1])
    return Model(order=[[0, 0]], pre=[[0, 1]], net=[[1, -1]],
                 rate=[k0, 0.0], x0=[0], sample_times=times, out_species=[0],
                 laws=[None, (code, consts)])


def test_packer_checks_programs(built_lib):
    import ctypes as C
    m = _birth_death('parameter_1 * abs(species_0)')
    n = C.c_int64(0)
    assert built_lib.pyst_model_blob_words(C.byref(m.desc()), C.byref(n)) == 0
    blob = m.blob()
    assert blob[31] == 1  # one reaction with a program
    # a program that pops an empty stack is refused
    bad = _birth_death('parameter_1 * abs(species_0)')
    bad.laws[1] = (np.array([kinetic.OP_ADD << 24], np.uint32),
                   np.zeros(0, np.float64))
    bad._law_arrays = None
    assert built_lib.pyst_model_blob_words(
        C.byref(bad.desc()), C.byref(n)) == 1  # PYST_EINVAL


def test_oracle_law_matches_exact_moments(oracle_mod):
    """X -> 0 with the non-polynomial law k1 * abs(x) is the linear death
    process: X(t) ~ Poisson(k0/k1 (1 - exp(-k1 t)))."""
    m = _birth_death('parameter_1 * abs(species_0)')
    r = oracle_mod.simulate(m, 4000, 0, seed=5)
    assert (r['status'] == 0).all()
    x = r['samples'][0].astype(np.float64)            # [ita, U]
    t = m.sample_times.astype(np.float64)
    lam = 20.0 / 0.5 * (1.0 - np.exp(-0.5 * t))
    se = np.sqrt(np.maximum(lam, 1e-9) / x.shape[1])
    assert (np.abs(x.mean(axis=1) - lam) < 5 * se + 1e-12).all()
    # tau-leaping on the same law
    rt = oracle_mod.simulate(m, 4000, 1, seed=6)
    assert (rt['status'] == 0).all()
    assert abs(rt['samples'][0, -1].mean() - lam[-1]) < 5 * se[-1] * 1.5


def test_oracle_invalid_law_status(oracle_mod):
    """A law that turns negative ends the trajectory with PYST_TRAJ_RATE."""
    m = _birth_death('parameter_1 * (species_0 - 5)')
    r = oracle_mod.simulate(m, 16, 0, seed=1)
    assert (r['status'] == 7).all()
    assert (r['samples'][0, 1:] == -1).all()


def test_sbml_michaelis_menten_front_end(oracle_mod):
    from py_stoch_b200 import sbml, sim_maker
    from py_stoch_b200.model import Model
    text = sbml.write_sbml(
        'mm', [('S', 300), ('P', 0)], [('Vmax', 40.0), ('Km', 50.0)],
        [('conv', [('S', 1)], [('P', 1)], 'Vmax * S / (Km + S)')])
    m = sbml.read_sbml_string(text)
    args = sim_maker.TLArgsList.make_list(m, [[300], [0]], [[40.0], [50.0]],
                                          [0, 1], 5.0, 6, 64)[0]
    model = Model.from_tl_args(args)
    assert model.law_reactions() == [0]
    r = oracle_mod.simulate(model, args.U, 0, seed=2)
    assert (r['status'] == 0).all()
    s = r['samples']
    assert (s[0] + s[1] == 300).all()             # conservation
    assert (np.diff(s[0].astype(int), axis=0) <= 0).all()
    # rate equation dS/dt = -Vmax S / (Km + S), solved implicitly:
    # Km ln(S/S0) + S - S0 = -Vmax t; S(5) = 139.2 (fluctuations shift the
    # mean of the stochastic process by far less than the tolerance)
    from scipy.optimize import brentq
    s5 = brentq(lambda v: 50.0 * np.log(v / 300.0) + v - 300.0 + 200.0,
                1.0, 300.0)
    se = s[0, -1].std() / np.sqrt(s.shape[2])
    assert abs(s[0, -1].mean() - s5) < 4 * se + 1.0
