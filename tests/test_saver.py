"""Result writer: the reference's text format byte for byte (golden files
written by the reference's own mod/utils/saver.py, tests/golden/
make_golden.py) and the binary npz form, which round-trips exactly."""

import datetime
import json
import os
import types

import numpy as np

from py_stoch_b200 import saver

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), 'golden',
                                     'frontend_golden.json')))['saver']


def _arr(d):
    return np.array(d['data'], dtype=d['dtype']).reshape(d['shape'])


def _args():
    g = GOLDEN
    return types.SimpleNamespace(x_0=_arr(g['x_0']), c=_arr(g['c']),
                                 E=_arr(g['E']), t_max=g['t_max'],
                                 ita=g['ita'], U=g['U'])


NOW = datetime.datetime(2024, 5, 6, 7, 8)


def test_text_format_matches_reference(tmp_path):
    res = _arr(GOLDEN['result'])
    paths = saver.save_results(res, _args(), 'lv_run', fmt='text',
                               root=str(tmp_path), now=NOW)
    got = {os.path.relpath(p, tmp_path): open(p).read() for p in paths}
    assert got == GOLDEN['files']


def test_npz_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    res = rng.integers(-1, 2**31 - 1, size=(2, 7, 1000)).astype(np.int32)
    (p,) = saver.save_results(res, _args(), 'lv_run', root=str(tmp_path),
                              now=NOW)
    assert p.endswith(os.path.join('x-1000-900-1_c-1-0.01-1',
                                   'TL_2024-5-6-7-8.npz'))
    d = saver.load_results(p)
    np.testing.assert_array_equal(d['samples'], res)
    assert d['samples'].dtype == np.int32
    np.testing.assert_array_equal(d['species_init'], _args().x_0)
    np.testing.assert_array_equal(d['parameters'], _args().c)
    assert int(d['num_simulations']) == GOLDEN['U']
    assert float(d['duration']) == GOLDEN['t_max']
    # the binary form is far smaller than the text form
    t = saver.save_results(res, _args(), 'txt', fmt='text',
                           root=str(tmp_path), now=NOW)
    assert os.path.getsize(p) < sum(os.path.getsize(q) for q in t) / 2
