"""Mass-action analysis of kinetic laws and the C packer (CPU only)."""

import ctypes as C

import numpy as np
import pytest

from py_stoch_b200 import _lib, networks, sbml, sim_maker
from py_stoch_b200.model import Model, UnsupportedKineticLaw, analyse_hazard


def test_analyse_hazard_forms():
    o, f, r = analyse_hazard(
        'parameter_0 / 2 * parameter_4 * species_0 * (species_0 - 1)', (2,),
        1)
    assert o == (2,) and f == (1,)
    assert str(r) in ('parameter_0*parameter_4/2',)
    o, f, r = analyse_hazard('parameter_2 * parameter_5', (0,), 1)
    assert o == (0,)
    # Schlogl with buffered A as a constant species listed as reactant but
    # absent from the law: orders come from the law's degrees
    o, f, r = analyse_hazard(
        'parameter_1 / 6 * species_0 * (species_0 - 1) * (species_0 - 2)',
        (3, 1, 0), 3)
    assert o == (3, 0, 0) and f[0] == 1
    # deterministic-style power law
    o, f, r = analyse_hazard('parameter_0 * species_0^2', (2,), 1)
    assert o == (2,) and f == (0,)
    with pytest.raises(UnsupportedKineticLaw):
        analyse_hazard('parameter_0 * species_0 / (parameter_1 + species_0)',
                       (1,), 1)


def test_plasmid_like_rates():
    m = sbml.read_sbml_string(sbml.write_sbml(
        'p', [('Xp', 100), ('Xm', 0)],
        [('Tp', 1.0), ('Tm', 0.75), ('lambda', 0.01), ('omega', 0.0)],
        [('r0', [('Xp', 1)], [('Xp', 2)], '(1 - lambda) / Tp * Xp'),
         ('r3', [('Xm', 1)], [('Xm', 2)], '1 / Tm * Xm')]))
    a = sim_maker.TLArgsList.make_list(m, [[100], [0]],
                                       [[1.0], [0.75], [0.01], [0.0]],
                                       [0, 1], 15, 11, 32)[0]
    mod = Model.from_tl_args(a)
    np.testing.assert_allclose(mod.rate, [0.99, 1 / 0.75])
    np.testing.assert_array_equal(mod.order, [[1, 0], [0, 1]])


def _desc_roundtrip(model):
    L = _lib.lib()
    d = model.desc()
    n = C.c_int64(0)
    rc = L.pyst_model_blob_words(C.byref(d), C.byref(n))
    return rc, n.value


def test_blob_layout_lv():
    m = networks.lotka_volterra()
    b = m.blob()
    assert b[_lib.H_MAGIC] == _lib.BLOB_MAGIC
    assert b[_lib.H_WORDS] == len(b) and len(b) % 4 == 0
    assert (b[_lib.H_S], b[_lib.H_R], b[_lib.H_KAPPA], b[_lib.H_ITA]) == (
        3, 3, 2, 100)
    rate = b[b[10]:b[10] + 3].view(np.float32)
    np.testing.assert_array_equal(rate, np.float32([10, 0.01, 10]))
    # net change entries reaction-major: r0: x+1 ; r1: x-1, y+1 ; r2: y-1
    netptr = b[b[13]:b[13] + 4]
    net = b[b[14]:b[14] + netptr[-1]]
    dec = [(int(e & 0xFFFF), int(np.int16(e >> 16))) for e in net]
    assert list(netptr) == [0, 1, 3, 4]
    assert dec == [(0, 1), (0, -1), (1, 1), (1, -1)]


@pytest.mark.parametrize('bad', ['neg_x0', 'neg_rate', 'bad_out', 'times',
                                 'order', 'big'])
def test_packer_rejects(bad):
    m = networks.lotka_volterra()
    kw = {}
    if bad == 'neg_x0':
        m = m.with_x0([-1, 0, 1])
    elif bad == 'neg_rate':
        m = m.with_rates([-1.0, 1, 1])
    elif bad == 'bad_out':
        m.out_species = np.array([5], np.int32)
    elif bad == 'times':
        m.sample_times = np.float32([0, 2, 1])
    elif bad == 'order':
        m.order = m.order.copy()
        m.order[0, 0] = 300
    elif bad == 'big':
        pre = np.ones((1, _lib.MAX_REACTIONS + 1), np.int64)
        m = Model.mass_action(pre, pre, np.ones(pre.shape[1]), [1], [0, 1])
    rc, _ = _desc_roundtrip(m)
    assert rc in (_lib.PYST_EINVAL, _lib.PYST_EUNSUPPORTED)


def test_synthetic_generator_deterministic():
    a = networks.synthetic_networks(8, seed=3)
    b = networks.synthetic_networks(8, seed=3)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x.blob(), y.blob())
    for x in a:
        assert 5 <= x.n_species <= 64 and 8 <= x.n_reactions <= 256
        assert len(x.blob()) <= _lib.MAX_BLOB_WORDS


def test_schlogl_from_sbml_equals_direct():
    m = sbml.read_sbml_string(sbml.schlogl_sbml())
    a = sim_maker.TLArgsList.make_list(
        m, [[250]], [[3e-7], [1e-4], [1e-3], [3.5], [1e5], [2e5]], [0], 5,
        200, 64)[0]
    np.testing.assert_array_equal(Model.from_tl_args(a).blob(),
                                  networks.schlogl().blob())
