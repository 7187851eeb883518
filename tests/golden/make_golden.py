"""Generate golden vectors for the model front-end by running the reference's
own Python code.

The reference is Python 2 code that imports libsbml and PyCUDA, neither of
which exists here.  This script loads its source files from the reference
checkout and applies only mechanical Python-2-to-3 shims before executing
them:

* ``dict.iteritems()`` -> ``dict.items()``;
* ``string.replace(s, a, b)`` -> ``s.replace(a, b)``;
* the statement ``print x`` -> ``print(x)``;
* ``from parser import Parser`` resolves to the reference's own parser.py;
* the Petri net's ``P``/``T`` dicts return lists from ``keys()``, as
  Python 2 dicts do.

``libsbml`` is replaced by :mod:`py_stoch_b200.sbml`, whose reader exposes
the libsbml methods the reference calls, and ``pycuda.tools.DeviceData`` by a
stub reporting a B200's limits (1024 threads per block, 48 KiB static shared
memory per block, warp size 32) so ``calculate_sizes`` can run.

It writes ``frontend_golden.json`` next to itself.  Run it in a checkout that
has the reference at ``/root/reference`` (or pass another path)::

    python tests/golden/make_golden.py [/path/to/reference]
"""

import json
import os
import re
import sys
import types

import numpy

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from py_stoch_b200 import sbml as fake_libsbml  # noqa: E402

FIXTURES = ['lotkaVoltera_sbml.xml', 'schlogl_sbmlv2.xml', 'schlogl_sbml.xml',
            'simple_sbml.xml', 'cdi_sbml.xml', 'plasmid_stability.xml']


def _py3(src):
    src = src.replace('.iteritems()', '.items()')
    src = re.sub(r'except (\w+), (\w+):', r'except \1 as \2:', src)
    src = re.sub(r'string\.replace\(', '_py2_replace(', src)
    src = re.sub(r'^(\s*)print (?!\()(.*)$', r'\1print(\2)', src,
                 flags=re.M)
    return src


def _py2_replace(s, old, new):
    return s.replace(old, new)


class _Py2Dict(dict):
    def keys(self):
        return list(dict.keys(self))


def _load(path, name, extra=None):
    with open(path) as f:
        src = _py3(f.read())
    mod = types.ModuleType(name)
    mod.__file__ = path
    mod.__dict__['_py2_replace'] = _py2_replace
    if extra:
        mod.__dict__.update(extra)
    exec(compile(src, path, 'exec'), mod.__dict__)
    return mod


class _DeviceData(object):
    max_threads = 1024
    shared_memory = 48 * 1024
    warp_size = 32


def load_reference(ref):
    saved = {k: sys.modules.get(k) for k in
             ('libsbml', 'parser', 'pycuda', 'pycuda.tools', 'pycuda.driver',
              'pycuda.compiler', 'pycuda.gpuarray', 'pycuda.autoinit',
              'pycuda.characterize', 'mod', 'mod.simulator',
              'mod.simulator.cuTauLeaping', 'mod.simulator.cuGillespie',
              'mod.utils')}
    try:
        sys.modules['libsbml'] = fake_libsbml
        spn = _load(os.path.join(ref, 'mod/petri_net/SPN.py'), 'ref_SPN')
        for meth in ('get_species_vector', 'get_reactions_vector'):
            orig = getattr(spn.SPN, meth)
            setattr(spn.SPN, meth, staticmethod(
                lambda m, _f=orig: _Py2Dict(_f(m))))
        parser = _load(os.path.join(ref, 'mod/parser/parser.py'),
                       'ref_parser')
        sys.modules['parser'] = parser
        tl = _load(os.path.join(ref, 'mod/parser/tl_parser.py'),
                   'ref_tl_parser')
        g = _load(os.path.join(ref, 'mod/parser/g_parser.py'),
                  'ref_g_parser')
        pkg = types.ModuleType('ref_pkg')
        pkg.TlParser, pkg.TlArgs = tl.TlParser, tl.TlArgs
        sys.modules['mod'] = types.ModuleType('mod')
        sys.modules['mod.parser'] = pkg
        sys.modules['mod.petri_net'] = types.ModuleType('mod.petri_net')
        sys.modules['mod.petri_net'].SPN = spn
        simk = _load(os.path.join(ref, 'sim_maker.py'), 'ref_sim_maker')

        # pycuda stubs for calculate_sizes
        pycuda = types.ModuleType('pycuda')
        tools = types.ModuleType('pycuda.tools')
        tools.DeviceData = _DeviceData
        for sub in ('driver', 'compiler', 'gpuarray', 'autoinit',
                    'characterize'):
            m = types.ModuleType('pycuda.' + sub)
            m.SourceModule = None
            sys.modules['pycuda.' + sub] = m
            setattr(pycuda, sub, m)
        pycuda.tools = tools
        sys.modules['pycuda'] = pycuda
        sys.modules['pycuda.tools'] = tools
        sim = _load(os.path.join(ref, 'mod/simulator/simulator.py'),
                    'ref_simulator')
        msim = types.ModuleType('mod.simulator')
        msim.StochasticSimulator = sim.StochasticSimulator
        sys.modules['mod.simulator'] = msim
        ctl = types.ModuleType('mod.simulator.cuTauLeaping')
        ctl.P3 = ctl.P1_P2 = None
        sys.modules['mod.simulator.cuTauLeaping'] = ctl
        cg = types.ModuleType('mod.simulator.cuGillespie')
        cg.gillespie = None
        sys.modules['mod.simulator.cuGillespie'] = cg
        mu = types.ModuleType('mod.utils')
        mu.Timer = None
        sys.modules['mod.utils'] = mu
        tlsim = _load(os.path.join(
            ref, 'mod/simulator/cuTauLeaping/cuTauLeaping.py'),
            'ref_cuTauLeaping')
        gsim = _load(os.path.join(
            ref, 'mod/simulator/cuGillespie/cuGillespie.py'),
            'ref_cuGillespie')
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v
        sys.modules.pop('mod.parser', None)
        sys.modules.pop('mod.petri_net', None)
    return dict(spn=spn, parser=parser, tl=tl, g=g, sim_maker=simk,
                tl_sim=tlsim, g_sim=gsim)


def _j(v):
    if isinstance(v, numpy.ndarray):
        return {'dtype': str(v.dtype), 'shape': list(v.shape),
                'data': v.tolist()}
    if isinstance(v, (numpy.integer,)):
        return int(v)
    if isinstance(v, (numpy.floating,)):
        return float(v)
    if isinstance(v, dict):
        return {str(k): _j(x) for k, x in sorted(v.items())}
    if isinstance(v, (list, tuple)):
        return [_j(x) for x in v]
    return v


class _FixedNow(object):
    """Stands in for datetime in the reference's saver: a fixed stamp."""
    @staticmethod
    def now():
        import datetime
        return datetime.datetime(2024, 5, 6, 7, 8)


def saver_golden(ref, R):
    """Run the reference's save_results (mod/utils/saver.py) on one sweep
    point and a small deterministic result; record every file it writes
    (path under the working directory, text content)."""
    import tempfile
    saver = _load(os.path.join(ref, 'mod/utils/saver.py'), 'ref_saver')
    saver.datetime = _FixedNow
    model = fake_libsbml.read_sbml(os.path.join(ref, 'examples',
                                                'lotkaVoltera_sbml.xml'))
    args = R['sim_maker'].TLArgsList.make_list(
        model, [[1000], [900], [1]], [[10], [0.01], [10]], [0, 1], 10, 4,
        3)[0]
    result = (numpy.arange(2 * 4 * 3, dtype=numpy.int32).reshape(2, 4, 3)
              * 37 % 1001)
    cwd = os.getcwd()
    files = {}
    with tempfile.TemporaryDirectory() as tmp:
        os.chdir(tmp)
        try:
            saver.save_results(result, args, 'lv_run')
        finally:
            os.chdir(cwd)
        for root, _, names in os.walk(tmp):
            for n in names:
                p = os.path.join(root, n)
                with open(p) as f:
                    files[os.path.relpath(p, tmp)] = f.read()
    return {'result': _j(result), 'x_0': _j(args.x_0), 'c': _j(args.c),
            'E': _j(args.E), 't_max': _j(args.t_max), 'ita': _j(args.ita),
            'U': _j(args.U), 'files': files}


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else '/root/reference'
    R = load_reference(ref)
    out = {'fixtures': {}, 'sweeps': [], 'calculate_sizes': []}
    for fx in FIXTURES:
        model = fake_libsbml.read_sbml(os.path.join(ref, 'examples', fx))
        spn = R['spn'].SPN()
        spn.sbml_2_stochastic_petri_net(model)
        args = R['tl'].TlArgs()
        args.E = numpy.arange(len(spn.P)).astype(numpy.int32)
        args.t_max = 10
        args.ita = 11
        args.U = 1000
        args = R['tl'].TlParser.parse(args, spn)
        ga = R['g'].GArgs()
        ga.E = args.E
        ga.t_max = 10
        ga.ita = 11
        ga = R['g'].GParser.parse(ga, spn)
        hazard_lines = sorted(l.strip() for l in args.hazards.splitlines()
                              if l.strip().startswith('a['))
        out['fixtures'][fx] = {
            'spn': {'Pre': _j(spn.Pre), 'Post': _j(spn.Post),
                    'StoichMConst': _j(spn.StoichMConst),
                    'M': _j(spn.M), 'c': _j(spn.c), 'h': spn.h,
                    'P': _j(spn.P), 'T': _j(spn.T)},
            'tl_args': {k: _j(getattr(args, k)) for k in
                        ('c', 'x_0', 'A', 'V', 'V_t', 'V_bar', 'M', 'N',
                         'A_size', 'V_size', 'V_t_size', 'V_bar_size', 'H',
                         'H_type', 'E', 't_max', 'ita', 'U', 'kappa', 'I',
                         'n_c', 'eta', 'gillespie')},
            'hazard_lines': hazard_lines,
            'g_args': {k: _j(getattr(ga, k)) for k in
                       ('c', 'x_0', 'V', 'M', 'N', 'V_size', 'kappa', 'I')},
        }

    sweeps = [
        ('simple_sbml.xml', [[1000, 10000], [1], [0]], [[1, 2, 5], [1, 2, 5]],
         [2], 0.1, 2, 128),
        ('schlogl_sbmlv2.xml', [[250]],
         [[3e-7], [1e-4], [8e-4, 9e-4, 1e-3], [3.5], [1e5], [2e5]],
         [0], 5, 2, 256),
        ('cdi_sbml.xml', [[10], [10]], [[0.5, 1], [1], [0.001, 0.01, 0.1]],
         [0, 1], 5, 100, 32),
    ]
    for fx, si, pa, e, dur, ita, u in sweeps:
        model = fake_libsbml.read_sbml(os.path.join(ref, 'examples', fx))
        lst = R['sim_maker'].TLArgsList.make_list(model, si, pa, e, dur, ita,
                                                  u)
        out['sweeps'].append({
            'fixture': fx, 'species_init': si, 'params': pa,
            'output_species': e, 'duration': dur, 'ita': ita, 'U': u,
            'points': [{'x_0': _j(a.x_0), 'c': _j(a.c), 'I': _j(a.I)}
                       for a in lst],
            'rest_list_params': _j(R['sim_maker'].rest_list(pa)),
        })

    for cls_name, cls in (('CuTauLeaping', R['tl_sim'].CuTauLeaping),
                          ('CuGillespie', R['g_sim'].CuGillespie)):
        for (m, n, npar) in ((3, 3, 3), (4, 1, 6), (200, 64, 10)):
            for u in (1, 2, 3, 31, 100, 639, 640, 1000, 1024, 1279, 1280,
                      2559, 2560, 25600, 262144, 1000001):
                a = types.SimpleNamespace(M=m, N=n, c=[0.0] * npar, U=u)
                rec = {'cls': cls_name, 'M': m, 'N': n, 'P': npar, 'U_in': u}
                try:
                    grid, block = cls().calculate_sizes(a)
                    rec.update(grid=int(grid), block=int(block),
                               U_out=int(a.U))
                except ZeroDivisionError:
                    rec['error'] = 'ZeroDivisionError'
                out['calculate_sizes'].append(rec)

    out['saver'] = saver_golden(ref, R)

    path = os.path.join(HERE, 'frontend_golden.json')
    with open(path, 'w') as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print('wrote', path)


if __name__ == '__main__':
    main()
