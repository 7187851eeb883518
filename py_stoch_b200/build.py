"""Build libpystoch_b200.so in-tree with nvcc for sm_100a.

    python -m py_stoch_b200.build [--force] [--verbose] [--ptxas]

The library links these objects with the static CUDA runtime, so it loads
on machines without a GPU (only the run calls need one):

* pyst_k_thread.cu, pyst_k_warp.cu  x (PYST_TAU, PYST_SCORE) in {0,1}^2
* pyst_k_batch.cu, pyst_k_sorted.cu x PYST_SCORE in {0,1}
* pyst_k_misc.cu (gradient reduction, test hooks), pyst_capi.cu (C ABI)
* pyst_pack.cpp (host-only model packer)

Objects compile in parallel into py_stoch_b200/_build/.  ``--fmad=false``
keeps every floating-point result a fixed IEEE function of its inputs; the
kernels request fused multiply-adds explicitly where they want them.
"""

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, 'csrc')
INCLUDE = os.path.join(REPO, 'include')
BUILD = os.path.join(HERE, '_build')
LIB = os.path.join(HERE, 'libpystoch_b200.so')

ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
NVCC_FLAGS = ARCH + ['-O3', '-lineinfo', '--fmad=false', '-std=c++17',
                     '-Xcompiler', '-fPIC,-O2', '--expt-relaxed-constexpr']
HEADERS = [os.path.join(CSRC, f) for f in
           ('pyst_engine.cuh', 'pyst_math.cuh', 'pyst_model.cuh',
            'pyst_launch.cuh')] + [
    os.path.join(INCLUDE, 'pystoch_b200.h'),
    os.path.join(INCLUDE, 'pystoch_b200_testing.h')]


def units():
    out = []
    for t in (0, 1):
        for s in (0, 1):
            for base in ('pyst_k_thread', 'pyst_k_warp'):
                out.append((base + '.cu', '%s_t%ds%d.o' % (base, t, s),
                            ['-DPYST_TAU=%d' % t, '-DPYST_SCORE=%d' % s]))
    for s in (0, 1):
        out.append(('pyst_k_batch.cu', 'pyst_k_batch_s%d.o' % s,
                    ['-DPYST_SCORE=%d' % s]))
        out.append(('pyst_k_sorted.cu', 'pyst_k_sorted_s%d.o' % s,
                    ['-DPYST_SCORE=%d' % s]))
    out.append(('pyst_k_misc.cu', 'pyst_k_misc.o', []))
    out.append(('pyst_capi.cu', 'pyst_capi.o', []))
    out.append(('pyst_pack.cpp', 'pyst_pack.o', []))
    return out


def nvcc():
    cand = os.path.join(os.environ.get('CUDA_HOME', '/usr/local/cuda'), 'bin',
                        'nvcc')
    return cand if os.path.exists(cand) else 'nvcc'


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, obj, defs, extra, verbose):
    cmd = [nvcc()] + NVCC_FLAGS + ['-I' + INCLUDE, '-I' + CSRC] + defs + list(
        extra) + ['-c', os.path.join(CSRC, src), '-o', obj]
    if verbose:
        print(' '.join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError('nvcc failed for %s:\n%s%s' % (src, r.stdout,
                                                          r.stderr))
    return r.stdout + r.stderr


STAMP = LIB + '.stamp'


def source_hash():
    """Content hash of every source, header and the compiler flags."""
    import hashlib
    h = hashlib.sha1(' '.join(NVCC_FLAGS).encode())
    for f in sorted(set([os.path.join(CSRC, u[0]) for u in units()] +
                        HEADERS)):
        with open(f, 'rb') as fh:
            h.update(os.path.basename(f).encode() + b'\0' + fh.read())
    return h.hexdigest()


def up_to_date():
    if not os.path.exists(LIB) or not os.path.exists(STAMP):
        return False
    with open(STAMP) as f:
        return f.read().strip() == source_hash()


def build(force=False, verbose=False, extra=(), jobs=None, lib=None,
          build_dir=None, only=None):
    """Compile stale objects in parallel and relink; return the .so path.

    The library counts as current when its stamp file holds the content
    hash of the sources (modification times are not trusted: copies of the
    tree may not keep them)."""
    if lib is not None:
        # a variant build (other -D flags) into its own directory
        return _build_variant(lib, build_dir, extra, verbose, jobs, only)
    if not force and not extra and up_to_date():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    todo = []
    objs = []
    for src, obj, defs in units():
        objp = os.path.join(BUILD, obj)
        objs.append(objp)
        if force or _stale(objp, [os.path.join(CSRC, src)] + HEADERS):
            todo.append((src, objp, defs))
    logs = []
    if todo:
        jobs = jobs or max(1, min(len(todo), os.cpu_count() or 4))
        with cf.ThreadPoolExecutor(jobs) as ex:
            futs = [ex.submit(_compile, s, o, d, extra, verbose)
                    for s, o, d in todo]
            for fu in futs:
                logs.append(fu.result())
    if todo or not os.path.exists(LIB) or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ['-shared', '-o', LIB + '.tmp'] + objs
        if verbose:
            print(' '.join(cmd), flush=True)
        subprocess.check_call(cmd)
        os.replace(LIB + '.tmp', LIB)
    with open(STAMP, 'w') as f:
        f.write(source_hash() + '\n')
    if extra and logs:
        print('\n'.join(l for l in logs if l.strip()))
    return LIB


def _build_variant(lib, build_dir, extra, verbose, jobs, only=None):
    """Link a library variant: units whose source is in `only` (default:
    all) are recompiled with `extra` flags into build_dir, the rest are
    taken from the default build."""
    build()
    os.makedirs(build_dir, exist_ok=True)
    objs = []
    todo = []
    for src, obj, defs in units():
        if only is not None and src not in only:
            objs.append(os.path.join(BUILD, obj))
            continue
        objp = os.path.join(build_dir, obj)
        objs.append(objp)
        todo.append((src, objp, defs))
    jobs = jobs or max(1, min(len(todo), os.cpu_count() or 4))
    with cf.ThreadPoolExecutor(jobs) as ex:
        for fu in [ex.submit(_compile, s, o, d, extra, verbose)
                   for s, o, d in todo]:
            fu.result()
    subprocess.check_call([nvcc()] + ARCH + ['-shared', '-o', lib] + objs)
    return lib


if __name__ == '__main__':
    ex = ['-Xptxas', '-v'] if '--ptxas' in sys.argv else []
    build(force='--force' in sys.argv or bool(ex),
          verbose='--verbose' in sys.argv, extra=ex)
    print(LIB)
