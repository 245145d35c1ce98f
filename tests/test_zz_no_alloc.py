"""The allocation-free KP07_dimsplit substep, called through the C ABI.

Callers that may not call cudaMalloc (an application that owns all device
memory through its own pool, or a run that must not allocate mid-way) use
fv_kp07_dimsplit_substep_noalloc with their own state buffers; its scratch is
a static device array inside libfvgpu.so.  These tests feed it the same state
as the allocating simulator API and the CPU oracle and check two calls in a
row (x-then-y and y-then-x sweeps, the second reading the first one's output):

  * against KP07_dimsplit.substep exactly (same kernel arithmetic, and every
    tile shape gives identical cells), state and CFL minimum;
  * against the FP32 oracle within the parity tests' relative L-inf bound for
    smooth data (2e-5);

with reflective and periodic walls, at a 32-rounded pitch and at the
smallest pitch the API accepts (nx + 8).  A tile load that gives up is
reported by the next call (FVGPU_NOALLOC_WAIT_POLLS makes every load give up
at once, in a child process, without a GPU fault), and oversized grids are
refused.  This file is collected last so that a stop-at-first-failure run
has already run every other test.
"""

import ctypes
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest
import torch

from conftest import ROOT, bump, rel_linf

import finitevolumegpu_b200 as fv
from finitevolumegpu_b200 import _lib
from oracle.oracle import OracleSim

pytestmark = pytest.mark.gpu

REFLECTIVE = 0x03030303
PERIODIC = 0x02020202


def _ptrs(t):
    FP = _lib._FP
    return (FP * 3)(*[ctypes.cast(t[v].data_ptr(), FP) for v in range(3)])


def _state(nx, ny):
    h, _, _ = bump(nx, ny)
    y, x = np.mgrid[0:ny, 0:nx]
    hu = (0.05 * np.sin(2 * np.pi * y / ny)).astype(np.float32)
    hv = (-0.03 * np.cos(2 * np.pi * x / nx)).astype(np.float32)
    return h, hu, hv


@pytest.mark.parametrize("bc", [REFLECTIVE, PERIODIC], ids=["reflective", "periodic"])
@pytest.mark.parametrize("round_pitch", [True, False], ids=["pitch32", "pitch_nx8"])
def test_noalloc_substeps_match_simulator_and_oracle(ctx, bc, round_pitch):
    nx, ny = 300, 190  # several tiles, ragged last row and column of tiles
    h, hu, hv = _state(nx, ny)
    bcobj = fv.BoundaryCondition(fv.BoundaryCondition.getTypes(bc))
    sim = fv.KP07_dimsplit.KP07_dimsplit(ctx, h, hu, hv, nx, ny, 1.0, 1.0, 9.81, boundary_conditions=bcobj)
    orc = OracleSim("KP07_dimsplit", [h, hu, hv], nx, ny, 1.0, 1.0, 9.81, bc=bc)
    dt = np.float32(sim.computeDt() * np.float32(0.45))
    kernel_dt = float(np.float32(dt * np.float32(0.5)))  # a split substep advances by dt/2

    pitch = (nx + 8 + 31) // 32 * 32 if round_pitch else nx + 8
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
                                                  0, bc, ctypes.cast(cfl.data_ptr(), FP), stream))
    _lib.check(L.fv_kp07_dimsplit_substep_noalloc(_ptrs(B), _ptrs(C), pitch, nx, ny, 1.0, 1.0, kernel_dt, 9.81, 1.3,
                                                  1, bc, ctypes.cast(cfl.data_ptr() + 4, FP), stream))
    torch.cuda.synchronize()
    got_cfl = cfl.cpu().numpy()

    for k, out in enumerate((B, C)):
        sim.substep(dt, k)
        orc.substep(dt, k)
        want = sim.download()
        got = out[:, 2:2 + ny, 4:4 + nx].cpu().numpy()
        for v, o in enumerate(orc.download()):
            assert np.array_equal(got[v], want[v]), (k, v, rel_linf(got[v], want[v]))
            assert rel_linf(got[v], o) <= 2e-5, (k, v, rel_linf(got[v], o))
        # computeDt() is min(cfl) * 0.5, exactly (a power of two)
        assert float(got_cfl[k]) * 0.5 == float(sim.computeDt()), (k, got_cfl[k], sim.computeDt())
        assert abs(float(got_cfl[k]) - float(orc.cfl)) <= 1e-5 * float(orc.cfl)


def test_noalloc_rejects_grids_beyond_the_static_scratch(ctx):
    nx, ny = 124 * 100, 60 * 100  # 10000 tiles > 8192
    t = torch.zeros((3, 8), dtype=torch.float32, device="cuda:0")
    u = torch.zeros((3, 8), dtype=torch.float32, device="cuda:0")
    L = _lib.lib()
    pitch = (nx + 8 + 31) // 32 * 32
    rc = L.fv_kp07_dimsplit_substep_noalloc(_ptrs(t), _ptrs(u), pitch, nx, ny, 1.0, 1.0, 0.01, 9.81, 1.3, 0,
                                            REFLECTIVE, None, None)
    assert rc == _lib.FV_ERR_INVALID
    assert "tiles" in L.fv_last_error().decode()


_GIVE_UP_CHILD = textwrap.dedent("""
    import ctypes, sys
    sys.path.insert(0, sys.argv[1])
    import torch
    from finitevolumegpu_b200 import _lib
    nx, ny, pitch = 200, 100, 208
    A = torch.ones((3, ny + 4, pitch), dtype=torch.float32, device="cuda:0")
    A[1:].zero_()
    B = torch.zeros_like(A)
    FP = _lib._FP
    p = lambda t: (FP * 3)(*[ctypes.cast(t[v].data_ptr(), FP) for v in range(3)])
    L = _lib.lib()
    rcs = []
    for k in range(4):
        rcs.append(L.fv_kp07_dimsplit_substep_noalloc(p(A), p(B), pitch, nx, ny, 1.0, 1.0, 0.01, 9.81, 1.3,
                                                      k % 2, 0x03030303, None, None))
        if rcs[-1] == _lib.FV_ERR_DEVICE:
            assert "gave up" in L.fv_last_error().decode()
    torch.cuda.synchronize()
    print("RCS", rcs)
""")


def test_noalloc_reports_a_tile_load_that_gave_up():
    """Every tile load gives up at once (poll limit -1, a child process): the
    call that launched returns FV_OK, the next one reports FV_ERR_DEVICE and
    clears the flag without launching, so the one after launches again."""
    env = dict(os.environ, FVGPU_NOALLOC_WAIT_POLLS="-1")
    r = subprocess.run([sys.executable, "-c", _GIVE_UP_CHILD, ROOT], env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("RCS")][-1]
    assert line == "RCS [0, %d, 0, %d]" % (_lib.FV_ERR_DEVICE, _lib.FV_ERR_DEVICE), line
