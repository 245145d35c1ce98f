"""The allocation-free KP07_dimsplit substep, called through the C ABI.

Callers that may not call cudaMalloc (an application that owns all device
memory through its own pool, or a run that must not allocate mid-way) use
fv_kp07_dimsplit_substep_noalloc with their own state buffers; its scratch is
a static device array inside libfvgpu.so.  This test feeds it the same state
as the allocating simulator API and checks two calls in a row (x-then-y and
y-then-x sweeps, the second reading the first one's output) against
KP07_dimsplit.substep, within the relative L-inf tolerance of the parity
tests (1e-5; the two paths run the same kernel, so they normally agree
exactly), and checks that oversized grids are refused.  This file is
collected last so that a stop-at-first-failure run has already run every
other test.
"""

import ctypes

import numpy as np
import pytest
import torch

from conftest import bump, rel_linf

import finitevolumegpu_b200 as fv
from finitevolumegpu_b200 import _lib

pytestmark = pytest.mark.gpu

REFLECTIVE = 0x03030303


def _ptrs(t):
    FP = _lib._FP
    return (FP * 3)(*[ctypes.cast(t[v].data_ptr(), FP) for v in range(3)])


def test_noalloc_substeps_match_simulator(ctx):
    nx, ny = 300, 190  # several tiles, ragged last row and column of tiles
    h, hu, hv = bump(nx, ny)
    y, x = np.mgrid[0:ny, 0:nx]
    hu = (0.05 * np.sin(2 * np.pi * y / ny)).astype(np.float32)
    hv = (-0.03 * np.cos(2 * np.pi * x / nx)).astype(np.float32)
    sim = fv.KP07_dimsplit.KP07_dimsplit(ctx, h, hu, hv, nx, ny, 1.0, 1.0, 9.81)
    dt = np.float32(sim.computeDt() * np.float32(0.45))
    kernel_dt = float(np.float32(dt * np.float32(0.5)))  # KP07_dimsplit.substep passes dt/2

    pitch = (nx + 8 + 31) // 32 * 32
    dev = torch.device("cuda:0")
    A = torch.zeros((3, ny + 4, pitch), dtype=torch.float32, device=dev)
    B = torch.zeros_like(A)
    C = torch.zeros_like(A)
    for v, arr in enumerate((h, hu, hv)):
        A[v, 2:2 + ny, 4:4 + nx] = torch.from_numpy(arr).to(dev)
    cfl = torch.zeros(2, dtype=torch.float32, device=dev)
    FP = _lib._FP
    L = _lib.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()

    _lib.check(L.fv_kp07_dimsplit_substep_noalloc(_ptrs(A), _ptrs(B), pitch, nx, ny, 1.0, 1.0, kernel_dt, 9.81, 1.3,
                                                  0, REFLECTIVE, ctypes.cast(cfl.data_ptr(), FP), stream))
    _lib.check(L.fv_kp07_dimsplit_substep_noalloc(_ptrs(B), _ptrs(C), pitch, nx, ny, 1.0, 1.0, kernel_dt, 9.81, 1.3,
                                                  1, REFLECTIVE, ctypes.cast(cfl.data_ptr() + 4, FP), stream))
    torch.cuda.synchronize()
    got_cfl = cfl.cpu().numpy()

    for k, out in enumerate((B, C)):
        sim.substep(dt, k)
        want = sim.download()
        want_dt = float(sim.computeDt())  # min(cfl) * 0.5
        got = out[:, 2:2 + ny, 4:4 + nx].cpu().numpy()
        for v in range(3):
            assert rel_linf(got[v], want[v]) <= 1e-5, (k, v, rel_linf(got[v], want[v]))
        assert abs(float(got_cfl[k]) * 0.5 - want_dt) <= 1e-5 * want_dt, (k, got_cfl[k], want_dt)


def test_noalloc_rejects_grids_beyond_the_static_scratch(ctx):
    nx, ny = 124 * 100, 60 * 100  # 10000 tiles > 8192
    t = torch.zeros((3, 8), dtype=torch.float32, device="cuda:0")
    L = _lib.lib()
    pitch = (nx + 8 + 31) // 32 * 32
    rc = L.fv_kp07_dimsplit_substep_noalloc(_ptrs(t), _ptrs(t), pitch, nx, ny, 1.0, 1.0, 0.01, 9.81, 1.3, 0,
                                            REFLECTIVE, None, None)
    assert rc == _lib.FV_ERR_INVALID
    assert "tiles" in L.fv_last_error().decode()
