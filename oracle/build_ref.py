"""Compile the reference's own CUDA kernels for sm_100a into oracle/_ref/
(test infrastructure: the reference itself, run as a checker and as the
bench's reference arm; never part of the product path).

The reference keeps its kernels as CUDA C in Python string literals
(mod/simulator/cuGillespie/gillespie.py, mod/simulator/cuTauLeaping/
P1_P2.py and P3.py, the init_rng source inside
mod/simulator/simulator.py:64-83) and specialises them per model with
string.Template (cuTauLeaping.py:142-160, cuGillespie.py:20-30) before
PyCUDA's SourceModule compiles them.  This recipe does the same steps
without PyCUDA: it parses each configuration with the reference's own
parser / Petri-net / sim_maker code (loaded by tests/golden/make_golden.py
with its Python-2 shims), runs the reference's calculate_sizes, substitutes
the templates with the reference's template_to_code / the CuGillespie
substitution, and compiles with nvcc for sm_100a (SourceModule's defaults:
-cubin, no extra optimisation flags).  Outputs only into oracle/_ref/:
<config>_<kernel>.cubin, <config>.json (launch geometry and the __constant__
data the reference uploads), rng.cubin and the size of
curandStateMRG32k3a.

    python oracle/build_ref.py [/path/to/reference]

Needs the reference checkout (present in the build container, not on GPU
machines, which use the prebuilt files).
"""

import importlib.util
import json
import os
import re
import string
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
OUT = os.path.join(HERE, '_ref')
# where this recipe looks for the reference checkout: $PYST_REFERENCE_DIR,
# else the build container's mount point
DEFAULT_REF = '/root/reference'


def reference_dir():
    return os.environ.get('PYST_REFERENCE_DIR') or DEFAULT_REF


def reference_present(ref=None):
    return os.path.isdir(os.path.join(ref or reference_dir(), 'mod'))

# name -> (fixture, species_init, params, output species, t_max, ita, U,
#          gillespie flag, simulator class)
CONFIGS = {
    'lv_ssa_1024': ('lotkaVoltera_sbml.xml', [1000, 1000, 1], [10, 0.01, 10],
                    [0, 1], 10, 100, 1024, 1, 'CuTauLeaping'),
    'lv_gillespie_1024': ('lotkaVoltera_sbml.xml', [1000, 1000, 1],
                          [10, 0.01, 10], [0, 1], 10, 100, 1024, 1,
                          'CuGillespie'),
    'schlogl_tl_262144': ('schlogl_sbmlv2.xml', [250],
                          [3e-7, 1e-4, 1e-3, 3.5, 1e5, 2e5], [0], 5, 200,
                          262144, 0, 'CuTauLeaping'),
    'schlogl_tl_8192': ('schlogl_sbmlv2.xml', [250],
                        [3e-7, 1e-4, 1e-3, 3.5, 1e5, 2e5], [0], 5, 21, 8192,
                        0, 'CuTauLeaping'),
    'schlogl_ssa_8192': ('schlogl_sbmlv2.xml', [250],
                         [3e-7, 1e-4, 1e-3, 3.5, 1e5, 2e5], [0], 5, 21, 8192,
                         1, 'CuTauLeaping'),
}


def _load_golden_module():
    path = os.path.join(REPO, 'tests', 'golden', 'make_golden.py')
    spec = importlib.util.spec_from_file_location('make_golden', path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _kernel_string(path, var='kernel'):
    ns = {}
    with open(path) as f:
        exec(compile(f.read(), path, 'exec'), ns)
    return ns[var]


def _init_rng_source(ref):
    text = open(os.path.join(ref, 'mod/simulator/simulator.py')).read()
    m = re.search(r'init_rng_src = """(.*?)"""', text, flags=re.S)
    return m.group(1)


def _nvcc(src, out):
    cu = out[:-len('.cubin')] + '.cu'
    with open(cu, 'w') as f:
        f.write(src)
    subprocess.check_call(['nvcc', '-cubin', '-arch=sm_100a', '-o', out, cu])


def _mrg_state_size():
    src = os.path.join(OUT, 'sizeof_mrg.cu')
    exe = os.path.join(OUT, 'sizeof_mrg')
    with open(src, 'w') as f:
        f.write('#include <curand_kernel.h>\n#include <cstdio>\n'
                'int main(){printf("%zu\\n", sizeof(curandStateMRG32k3a));}\n')
    subprocess.check_call(['nvcc', '-o', exe, src])
    return int(subprocess.check_output([exe]).strip())


def _arr(a):
    a = np.asarray(a)
    return {'dtype': str(a.dtype), 'data': a.ravel().tolist(),
            'shape': list(a.shape)}


def build(ref=None, names=None):
    ref = ref or reference_dir()
    os.makedirs(OUT, exist_ok=True)
    G = _load_golden_module()
    from py_stoch_b200 import sbml as fake_libsbml
    R = G.load_reference(ref)
    p1p2 = _kernel_string(os.path.join(
        ref, 'mod/simulator/cuTauLeaping/P1_P2.py'))
    p3 = _kernel_string(os.path.join(ref, 'mod/simulator/cuTauLeaping/P3.py'))
    gil = _kernel_string(os.path.join(
        ref, 'mod/simulator/cuGillespie/gillespie.py'))
    rng_cubin = os.path.join(OUT, 'rng.cubin')
    if not os.path.exists(rng_cubin):
        _nvcc(_init_rng_source(ref), rng_cubin)
    meta = {'mrg32k3a_bytes': _mrg_state_size()}
    for name, cfg in CONFIGS.items():
        if names and name not in names:
            continue
        fx, si, pa, E, t_max, ita, U, gill, cls = cfg
        model = fake_libsbml.read_sbml(os.path.join(ref, 'examples', fx))
        args = R['sim_maker'].TLArgsList.make_list(
            model, [[v] for v in si], [[v] for v in pa], E, t_max, ita, U,
            gillespie=gill)[0]
        if cls == 'CuTauLeaping':
            sim = R['tl_sim'].CuTauLeaping()
            grid, block = sim.calculate_sizes(args)
            srcs = {'p1p2': sim.template_to_code(string.Template(p1p2), args,
                                                 block),
                    'p3': sim.template_to_code(string.Template(p3), args,
                                               block)}
        else:
            sim = R['g_sim'].CuGillespie()
            grid, block = sim.calculate_sizes(args)
            srcs = {'gillespie': string.Template(gil).substitute(
                V_SIZE=args.V_size, SPECIES_NUM=args.N, THREAD_NUM=args.U,
                PARAM_NUM=len(args.c), REACT_NUM=args.M, KAPPA=args.kappa,
                ITA=args.ita, BLOCK_SIZE=block, T_MAX=args.t_max,
                UPDATE_PROPENSITIES=args.hazards)}
        for k, src in srcs.items():
            _nvcc(src, os.path.join(OUT, '%s_%s.cubin' % (name, k)))
        info = {'class': cls, 'grid': int(grid), 'block': int(block),
                'U': int(args.U), 'N': int(args.N), 'M': int(args.M),
                'kappa': int(args.kappa), 'ita': int(args.ita),
                'gillespie': int(gill),
                'const': {'d_A': _arr(args.A) if cls == 'CuTauLeaping'
                          else None,
                          'd_V': _arr(args.V),
                          'd_H': _arr(args.H), 'd_H_type': _arr(args.H_type),
                          'd_c': _arr(args.c), 'd_I': _arr(args.I),
                          'd_E': _arr(args.E), 'd_x_0': _arr(args.x_0)}}
        with open(os.path.join(OUT, name + '.json'), 'w') as f:
            json.dump(info, f)
    with open(os.path.join(OUT, 'meta.json'), 'w') as f:
        json.dump(meta, f)
    return OUT


if __name__ == '__main__':
    sys.path.insert(0, REPO)
    build(sys.argv[1] if len(sys.argv) > 1 else reference_dir())
    print('built', OUT)
