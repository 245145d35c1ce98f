"""Speed of the stage kernels against the reference's own kernels on the same
B200 and the same 4096-cell-wide inputs (device time per full step, CUDA
events).  The reference kernels run with their default block and with each
other block shape built (oracle.ref_kernels.BLOCKS); the comparison is against
the fastest.  The test fails if libfvgpu is slower than that."""

import json
import os

import numpy as np
import pytest

from conftest import dam_break, kelvin_helmholtz

import finitevolumegpu_b200 as fv
from oracle import ref_kernels

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tuned_ctx():
    """A context with the autotuner on, as CudaContext() gives users by default."""
    return fv.CudaContext.CudaContext(device=0, autotuning=True)


@pytest.mark.parametrize("scheme", ["KP07_dimsplit", "HLL2", "WAF", "FORCE", "HLL", "LxF", "KP07",
                                    "EE2D_KP07_dimsplit"])
def test_faster_than_reference_kernels(tuned_ctx, scheme):
    ctx = tuned_ctx
    if scheme == "EE2D_KP07_dimsplit":
        nx, ny = 4096, 2048
        from conftest import kelvin_helmholtz as kh
        q = kh(nx, ny)
        sim = fv.SCHEMES[scheme](ctx, *q, nx, ny, 1.0 / nx, 1.0 / ny, 0.0, 1.4,
                                 boundary_conditions=fv.BoundaryCondition(
                                     fv.BoundaryCondition.getTypes(0x02020202)))
        make_ref = lambda block: ref_kernels.RefKernelSim(scheme, q, nx, ny, 1.0 / nx, 1.0 / ny, 0.0, gamma=1.4,
                                                         bc=0x02020202, block=block)
    else:
        nx, ny = 4096, 4096
        q = list(dam_break(nx, ny))
        sim = fv.SCHEMES[scheme](ctx, *q, nx, ny, 1.0, 1.0, 9.81)
        make_ref = lambda block: ref_kernels.RefKernelSim(scheme, q, nx, ny, 1.0, 1.0, 9.81, block=block)
    ref_times = {}
    dt = None
    for block in (None,) + ref_kernels.BLOCKS:
        if not ref_kernels.available(scheme, block):
            continue
        ref = make_ref(block)
        if dt is None:
            dt = np.float32(ref.computeDt() * np.float32(0.5))
        ref.time_steps(3, dt)
        ref_times["%dx%d" % (ref.bw, ref.bh)] = ref.time_steps(20, dt)
        ref.close()
    best_block = min(ref_times, key=ref_times.get)
    ref_ms = ref_times[best_block]
    sim.advance(3)
    sim.advance(20)
    my_ms = sim.last_advance_ms()
    rec = {"scheme": scheme, "nx": nx, "ny": ny, "ref_ms_per_step": ref_ms, "fvgpu_ms_per_step": my_ms,
           "speedup": ref_ms / my_ms, "ref_block": best_block, "ref_ms_per_block": ref_times,
           "tile": sim.tile_info()}
    print(json.dumps(rec))
    out = os.environ.get("FVGPU_TIMING_OUT")
    if out:
        with open(out, "a") as f:
            f.write(json.dumps(rec) + "\n")
    assert my_ms < ref_ms, rec
