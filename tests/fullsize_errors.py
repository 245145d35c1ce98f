"""Errors against FP64 at a benchmark configuration's full size (not a test:
the FP64 oracle needs minutes of host time at these sizes).

    python tests/fullsize_errors.py config3 OUT.json

config3: EE2D_KP07_dimsplit Kelvin-Helmholtz, 4096 x 2048, gamma = 1.4,
periodic walls, 500 steps of simulate()'s dt schedule (the seeded initial
condition of tests/test_gpu_configs.py).  The GPU state after 500 steps is
compared with the FP64 oracle and with the IEEE FP32 oracle (the round-off
floor of an FP32 evaluation of this scheme) run on every host thread; the
relative L1 / L-inf error per conserved variable, the step counts and the
FP64 conservation sums go to OUT.json.
"""

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.dirname(HERE), HERE]

from conftest import rel_l1, rel_linf  # noqa: E402
from test_gpu_configs import advance_host, kh  # noqa: E402

import finitevolumegpu_b200 as fv  # noqa: E402
from oracle.oracle import OracleSim  # noqa: E402

VARS = ("rho", "rho_u", "rho_v", "E")


def config3(out_path, nx=4096, ny=2048, steps=500):
    q = kh(nx, ny)
    ctx = fv.CudaContext.CudaContext(device=0, autotuning=True)
    bc = fv.BoundaryCondition(fv.BoundaryCondition.getTypes(0x02020202))
    sim = fv.EE2D_KP07_dimsplit.EE2D_KP07_dimsplit(ctx, *q, nx, ny, 1.0 / nx, 1.0 / ny, 0.0, 1.4,
                                                   boundary_conditions=bc)
    s0 = sim.conservation()
    sim.advance(steps)
    s1 = sim.conservation()
    got = sim.download()
    rec = {"config": 3, "workload": "EE2D_KP07_dimsplit Kelvin-Helmholtz %dx%d, periodic, gamma 1.4" % (nx, ny),
           "steps": steps, "t": sim.simTime(), "tile": sim.tile_info(), "sums_start": s0.tolist(),
           "sums_end": s1.tolist()}
    del sim
    for dtype, key in ((np.float64, "fp64"), (np.float32, "ieee_fp32")):
        t0 = time.time()
        o = OracleSim("EE2D_KP07_dimsplit", q, nx, ny, 1.0 / nx, 1.0 / ny, 0.0, gamma=1.4, bc=0x02020202,
                      dtype=dtype)
        advance_host(o, steps)
        ref = o.download()
        rec["%s_oracle_seconds" % key] = round(time.time() - t0, 1)
        rec["%s_oracle_t" % key] = o.simTime()
        if key == "fp64":
            want = ref
            rec["rel_l1_vs_fp64"] = dict(zip(VARS, [rel_l1(a, b) for a, b in zip(got, want)]))
            rec["rel_linf_vs_fp64"] = dict(zip(VARS, [rel_linf(a, b) for a, b in zip(got, want)]))
        else:
            rec["ieee_fp32_oracle_rel_l1_vs_fp64"] = dict(zip(VARS, [rel_l1(a, b) for a, b in zip(ref, want)]))
            rec["ieee_fp32_oracle_rel_linf_vs_fp64"] = dict(zip(VARS, [rel_linf(a, b) for a, b in zip(ref, want)]))
        del o
    rec["host_threads"] = len(os.sched_getaffinity(0))
    with open(out_path, "w") as f:
        json.dump(rec, f, indent=1)
    print(json.dumps(rec))


if __name__ == "__main__":
    if len(sys.argv) != 3 or sys.argv[1] != "config3":
        sys.exit(__doc__)
    config3(sys.argv[2])
