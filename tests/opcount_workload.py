"""Workload for instruction-counter captures (not a test): two steps of the
reference's own kernel for scheme argv[1] (through oracle/ref_kernels.py),
then two steps of libfvgpu's kernel, on the 3072 x 3072 dam break of the tests.

    python tests/opcount_workload.py KP07_dimsplit
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.dirname(HERE), HERE]

from conftest import dam_break  # noqa: E402

import finitevolumegpu_b200 as fv  # noqa: E402
from oracle import ref_kernels  # noqa: E402


def main(scheme, n=3072):
    q = list(dam_break(n, n))
    ref = ref_kernels.RefKernelSim(scheme, q, n, n, 1.0, 1.0, 9.81)
    ref.time_steps(2, np.float32(ref.computeDt() * np.float32(0.5)))
    ref.close()
    sim = fv.SCHEMES[scheme](fv.CudaContext.CudaContext(autotuning=False), *q, n, n, 1.0, 1.0, 9.81)
    sim.advance(2)
    sim.synchronize()


if __name__ == "__main__":
    main(sys.argv[1])
