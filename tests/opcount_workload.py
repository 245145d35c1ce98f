"""Workload for instruction-counter captures (not a test): two steps of the
reference's own kernel for scheme argv[1] (through oracle/ref_kernels.py),
then two steps of libfvgpu's kernel (its first tile configuration, one line
per thread), on the 3072 x 3072 dam break of the tests (for
EE2D_KP07_dimsplit: the Kelvin-Helmholtz band of the tests on a 3072 x 3072
unit square, periodic).

    python tests/opcount_workload.py KP07_dimsplit
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.dirname(HERE), HERE]

from conftest import dam_break, kelvin_helmholtz  # noqa: E402

import finitevolumegpu_b200 as fv  # noqa: E402
from oracle import ref_kernels  # noqa: E402

PERIODIC = 0x02020202


def main(scheme, n=3072):
    ctx = fv.CudaContext.CudaContext(autotuning=False)
    if scheme == "EE2D_KP07_dimsplit":
        q = kelvin_helmholtz(n, n)
        ref = ref_kernels.RefKernelSim(scheme, q, n, n, 1.0 / n, 1.0 / n, 0.0, gamma=1.4, bc=PERIODIC)
        bc = fv.BoundaryCondition(fv.BoundaryCondition.getTypes(PERIODIC))
        sim = fv.SCHEMES[scheme](ctx, *q, n, n, 1.0 / n, 1.0 / n, 0.0, 1.4, boundary_conditions=bc)
    else:
        q = list(dam_break(n, n))
        ref = ref_kernels.RefKernelSim(scheme, q, n, n, 1.0, 1.0, 9.81)
        sim = fv.SCHEMES[scheme](ctx, *q, n, n, 1.0, 1.0, 9.81)
    ref.time_steps(2, np.float32(ref.computeDt() * np.float32(0.5)))
    ref.close()
    sim.advance(2)
    sim.synchronize()


if __name__ == "__main__":
    main(sys.argv[1])
