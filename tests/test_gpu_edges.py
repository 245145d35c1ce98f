"""Ragged and degenerate grid sizes against the CPU oracle: grids of two
cells, strips one tile wide or long, sizes one cell over a tile edge and
exactly one tile, for every scheme, with the boundary pairs periodic/reflective
both ways round.  The periodic wrap shifts an index by one domain length
(GPUSimulators/cuda/common.h:243-286), so the smallest grid here is 2 wide.

Tolerance: L-inf 2e-5 per variable (WAF 1e-4, whose limiter switches on the
sign of Courant numbers; the Euler scheme 5e-5), with the same number of
steps on both sides, relative to the variable's magnitude: the larger of the
oracle's maximum and, for the momenta, the largest initial momentum.  On
strips two or three cells wide a momentum component can stay near zero
(mirrored walls cancel it, or the initial wave has a node on every cell), and
relative to its own tiny maximum the FP32 rounding differences look large;
the reference's own kernels differ from the oracle there by as much as these
kernels do.
"""

import numpy as np
import pytest

import finitevolumegpu_b200 as fv
from oracle.oracle import OracleSim

pytestmark = pytest.mark.gpu

SCHEMES = ["LxF", "FORCE", "HLL", "HLL2", "WAF", "KP07", "KP07_dimsplit", "EE2D_KP07_dimsplit"]
SIZES = [(2, 2), (2, 9), (9, 2), (3, 130), (130, 3), (61, 29), (124, 60), (125, 61), (127, 33)]
BCS = {"ns_periodic": 0x02020303, "ew_periodic": 0x03030202}
TOL = {"WAF": 1e-4, "EE2D_KP07_dimsplit": 5e-5}


def smooth_state(scheme, nx, ny):
    y, x = np.mgrid[0:ny, 0:nx] + 0.5
    wx, wy = np.sin(2 * np.pi * x / nx), np.cos(2 * np.pi * y / ny)
    if scheme == "EE2D_KP07_dimsplit":
        rho = 1.0 + 0.2 * wx * wy
        ru = 0.1 * wy
        rv = 0.1 * wx
        E = 2.5 / 0.4 + 0.5 * (ru ** 2 + rv ** 2) / rho
        return [a.astype(np.float32) for a in (rho, ru, rv, E)]
    h = 1.0 + 0.2 * wx * wy
    return [a.astype(np.float32) for a in (h, 0.05 * wy * h, 0.05 * wx * h)]


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("size", SIZES, ids=["%dx%d" % s for s in SIZES])
@pytest.mark.parametrize("bcname", list(BCS))
def test_ragged_sizes_vs_oracle(ctx, scheme, size, bcname):
    nx, ny = size
    q = smooth_state(scheme, nx, ny)
    bc = BCS[bcname]
    b = fv.BoundaryCondition(fv.BoundaryCondition.getTypes(bc))
    if scheme == "EE2D_KP07_dimsplit":
        dx, dy, g = 1.0 / 64, 1.0 / 64, 0.0
        sim = fv.SCHEMES[scheme](ctx, *q, nx, ny, dx, dy, g, 1.4, boundary_conditions=b, cfl_scale=0.45)
        ref = OracleSim(scheme, q, nx, ny, dx, dy, g, gamma=1.4, cfl_scale=0.45, bc=bc)
        t_end = 0.03
    else:
        dx, dy, g = 1.0, 1.0, 9.81
        sim = fv.SCHEMES[scheme](ctx, *q, nx, ny, dx, dy, g, boundary_conditions=b, cfl_scale=0.45)
        ref = OracleSim(scheme, q, nx, ny, dx, dy, g, cfl_scale=0.45, bc=bc)
        t_end = 2.0
    sim.simulate(t_end)
    ref.simulate(t_end)
    assert sim.simSteps() == ref.simSteps() > 5
    tol = TOL.get(scheme, 2e-5)
    mom_scale = max(float(np.max(np.abs(q[1]))), float(np.max(np.abs(q[2]))))
    for v, (a, w) in enumerate(zip(sim.download(), ref.download())):
        assert a.shape == (ny, nx)
        assert np.all(np.isfinite(a))
        scale = max(float(np.max(np.abs(w))), mom_scale if v in (1, 2) else 0.0)
        err = float(np.max(np.abs(a.astype(np.float64) - w))) / scale
        assert err < tol, (scheme, size, bcname, v, err)
