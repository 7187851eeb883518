"""Run the reference's own kernels (compiled by oracle/build_ref.py into
oracle/_ref/) on the GPU, replaying its host code without PyCUDA.

Test infrastructure and the bench's reference arm: it checks the engine at
the distribution level against the actual reference kernels and times
them; it is never part of the product path.

Replays, step for step:
* ``CuTauLeaping.run`` (mod/simulator/cuTauLeaping/cuTauLeaping.py:18-84):
  upload the __constant__ data (:86-107), allocate x = x_0 per thread, O, Q,
  t, F as zeros (:119-132), seed one MRG32k3a state per thread with
  ``init_rng`` (mod/simulator/simulator.py:62-96; grid size//64+1, block
  64), then repeat kernel_P1_P2, kernel_P3 and ``termin = -sum(Q)`` until
  every trajectory has terminated (:49-76);
* ``CuGillespie.run`` (mod/simulator/cuGillespie/cuGillespie.py:16-46):
  constants, O zeros, init_rng, one kernel_Gillespie launch.
Kernels are launched through the CUDA driver API (cuda-python) on torch's
current stream; buffers are torch tensors.
"""

import ctypes as C
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(HERE, '_ref')


def available(name):
    return os.path.exists(os.path.join(REF, name + '.json'))


def _check(res):
    err = res[0] if isinstance(res, tuple) else res
    if int(err) != 0:
        raise RuntimeError('CUDA driver call failed: %r' % (err,))
    return res[1:] if isinstance(res, tuple) and len(res) > 1 else None


class _Kernel(object):
    def __init__(self, path, name):
        import cuda.bindings.driver as drv
        self.drv = drv
        (self.mod,) = _check(drv.cuModuleLoad(path.encode()))
        (self.fn,) = _check(drv.cuModuleGetFunction(self.mod, name.encode()))

    def set_global(self, name, arr):
        drv = self.drv
        dptr, size = _check(drv.cuModuleGetGlobal(self.mod, name.encode()))
        arr = np.ascontiguousarray(arr)
        n = min(int(size), arr.nbytes)
        _check(drv.cuMemcpyHtoD(dptr, arr.ctypes.data, n))

    def launch(self, grid, block, args, stream):
        vals = []
        for a in args:
            vals.append(C.c_int(a) if isinstance(a, np.int32) else
                        C.c_void_p(int(a)))
        ptrs = (C.c_void_p * len(vals))(*[C.addressof(v) for v in vals])
        _check(self.drv.cuLaunchKernel(
            self.fn, int(grid), 1, 1, int(block), 1, 1, 0,
            self.drv.CUstream(stream), C.addressof(ptrs), 0))


class ReferenceRun(object):
    """One prebuilt reference configuration (see oracle/build_ref.py)."""

    def __init__(self, name, device=None):
        import torch
        self.torch = torch
        self.device = torch.device(device or 'cuda')
        torch.cuda.init()
        torch.empty(1, device=self.device)  # primary context current
        with open(os.path.join(REF, name + '.json')) as f:
            self.info = json.load(f)
        with open(os.path.join(REF, 'meta.json')) as f:
            self.state_bytes = json.load(f)['mrg32k3a_bytes']
        self.name = name
        self.rng = _Kernel(os.path.join(REF, 'rng.cubin'), 'init_rng')
        consts = {k: np.array(v['data'], dtype=v['dtype']) for k, v in
                  self.info['const'].items() if v is not None}
        if self.info['class'] == 'CuTauLeaping':
            self.p1p2 = _Kernel(os.path.join(REF, name + '_p1p2.cubin'),
                                'kernel_P1_P2')
            self.p3 = _Kernel(os.path.join(REF, name + '_p3.cubin'),
                              'kernel_P3')
            for k in (self.p1p2, self.p3):
                for sym in ('d_A', 'd_V', 'd_H', 'd_H_type', 'd_c', 'd_I',
                            'd_E'):
                    k.set_global(sym, consts[sym])
        else:
            self.gil = _Kernel(os.path.join(REF, name + '_gillespie.cubin'),
                               'kernel_Gillespie')
            for sym in ('d_V', 'd_c', 'd_I', 'd_E', 'd_x_0'):
                self.gil.set_global(sym, consts[sym])
        self.x0 = consts['d_x_0']

    def run(self, max_rounds=1_000_000):
        """Simulate all U trajectories; returns O as an int32 tensor
        [kappa, ita, U] on the device and the number of host rounds."""
        torch = self.torch
        i = self.info
        U, N, kappa, ita = i['U'], i['N'], i['kappa'], i['ita']
        dev = self.device
        stream = torch.cuda.current_stream(dev).cuda_stream
        O = torch.zeros((kappa, ita, U), dtype=torch.int32, device=dev)
        rng = torch.empty(U * self.state_bytes, dtype=torch.uint8,
                          device=dev)
        self.rng.launch(U // 64 + 1, 64, [np.int32(U), rng.data_ptr()],
                        stream)
        if i['class'] != 'CuTauLeaping':
            self.gil.launch(i['grid'], i['block'],
                            [O.data_ptr(), rng.data_ptr()], stream)
            return O, 1
        x = torch.from_numpy(np.tile(self.x0.astype(np.int32), (U, 1))).to(
            dev)
        Q = torch.zeros(U, dtype=torch.int32, device=dev)
        t = torch.zeros(U, dtype=torch.float64, device=dev)
        F = torch.zeros(U, dtype=torch.int32, device=dev)
        args = [x.data_ptr(), O.data_ptr(), Q.data_ptr(), t.data_ptr(),
                F.data_ptr(), rng.data_ptr()]
        termin, rounds = 0, 0
        while termin != U:
            self.p1p2.launch(i['grid'], i['block'], args, stream)
            self.p3.launch(i['grid'], i['block'], args, stream)
            termin = -int(Q.sum().item())
            rounds += 1
            if rounds >= max_rounds:
                raise RuntimeError('reference loop did not terminate')
        return O, rounds
