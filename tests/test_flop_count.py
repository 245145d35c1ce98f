"""The algorithmic operation counts the benchmark reports are the oracle's.

bench.py states the floating-point operations per cell and stage launch of each
scheme (the reference's formulation: +, -, *, /, sqrt, min, max counted once)
for its FP32 roofline.  They are measured by running the CPU restatement with
an operation-counting number type; this test repeats that count.
"""

import pytest

import bench
from oracle.oracle import ops_per_cell_substep


@pytest.mark.parametrize("scheme", sorted(bench.ALG_OPS_PER_CELL_LAUNCH))
def test_bench_op_counts_match_oracle(scheme):
    got = ops_per_cell_substep(scheme)
    want = bench.ALG_OPS_PER_CELL_LAUNCH[scheme]
    assert got["flops"] == pytest.approx(want["flops"], abs=1e-6), got
    assert got["mufu"] == pytest.approx(want["mufu"], abs=1e-6), got


def test_count_is_per_cell():
    """The fitted count does not depend on the grid sizes used for the fit."""
    from oracle import oracle

    c = ops_per_cell_substep("KP07_dimsplit")
    # a single 64 x 64 substep pair costs the per-cell count times the cells plus
    # a boundary term that is small against the 4096 interior cells
    import numpy as np

    n = 64
    m = n + 4
    y, x = np.mgrid[0:m, 0:m] + 0.5 - 2
    h = 1.0 + 0.3 * np.exp(-((x - 0.45 * n) ** 2 + (y - 0.55 * n) ** 2) / (2 * (n / 8.0) ** 2))
    q = [h, np.zeros_like(h), np.zeros_like(h)]
    tot = 0
    for st in (0, 1):
        r = oracle.count_ops("KP07_dimsplit", q, n, n, 1.0, 1.0, 0.05, 9.81, 1.4, 1.3, st, 2, 0x03030303)
        tot += sum(r[k] for k in oracle.OP_NAMES)
    per_cell = tot / 2 / (n * n)
    assert c["flops"] <= per_cell <= c["flops"] * 1.12
