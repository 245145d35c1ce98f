"""The largest grids: strips at the API's maximum side (2**20 cells) against
the CPU oracle, and a 16384 x 16384 KP07_dimsplit domain checked through
size-independent properties, since the oracle would take minutes there:

  * shift equivariance with periodic walls: every cell's update depends only
    on its neighbourhood and the time step is a minimum over cells, so the
    state grown from an initial condition rolled by (sy, sx) cells is the
    rolled state, bit for bit;
  * mass conservation to FP32 rounding (FP64 sums of the interior);
  * a lake at rest stays exactly at rest.
"""

import numpy as np
import pytest

import finitevolumegpu_b200 as fv
from oracle.oracle import OracleSim

pytestmark = pytest.mark.gpu

PERIODIC = 0x02020202
MIXED = 0x02020303
MAX_SIDE = 1 << 20


def smooth(nx, ny, seed=0):
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:ny, 0:nx] + 0.5
    kx, ky = rng.integers(1, 4, size=2)
    wx, wy = np.sin(2 * np.pi * kx * x / nx), np.cos(2 * np.pi * ky * y / ny)
    h = 1.0 + 0.2 * wx * wy
    return [a.astype(np.float32) for a in (h, 0.05 * wy * h, 0.05 * wx * h)]


@pytest.mark.parametrize("scheme", ["KP07_dimsplit", "HLL", "KP07"])
@pytest.mark.parametrize("shape", [(MAX_SIDE, 3), (3, MAX_SIDE)], ids=["wide", "tall"])
def test_max_side_strips_vs_oracle(ctx, scheme, shape):
    nx, ny = shape
    q = smooth(nx, ny)
    b = fv.BoundaryCondition(fv.BoundaryCondition.getTypes(MIXED))
    sim = fv.SCHEMES[scheme](ctx, *q, nx, ny, 1.0, 1.0, 9.81, boundary_conditions=b, cfl_scale=0.45)
    ref = OracleSim(scheme, q, nx, ny, 1.0, 1.0, 9.81, cfl_scale=0.45, bc=MIXED)
    dt = np.float32(ref.computeDt() * np.float32(0.45))
    for _ in range(4):
        sim.step(dt)
        ref.step(dt)
    mom = max(float(np.max(np.abs(q[1]))), float(np.max(np.abs(q[2]))))
    for v, (a, w) in enumerate(zip(sim.download(), ref.download())):
        assert np.all(np.isfinite(a))
        scale = max(float(np.max(np.abs(w))), mom if v else 0.0)
        err = float(np.max(np.abs(a.astype(np.float64) - w))) / scale
        assert err < 2e-5, (scheme, shape, v, err)


def test_16384_shift_equivariance_and_mass(ctx):
    n = 16384
    q = smooth(n, n, seed=3)
    sy, sx = 5003, 12345
    rolled = [np.ascontiguousarray(np.roll(a, (sy, sx), axis=(0, 1))) for a in q]
    b = fv.BoundaryCondition(fv.BoundaryCondition.getTypes(PERIODIC))
    outs = []
    for init in (q, rolled):
        sim = fv.KP07_dimsplit.KP07_dimsplit(ctx, *init, n, n, 1.0, 1.0, 9.81, boundary_conditions=b)
        sim.advance(3)
        outs.append((sim.download(), sim.simSteps(), sim.simTime()))
        del sim
    (a, na, ta), (r, nr, tr) = outs
    assert na == nr == 3 and ta == tr
    for x, y in zip(a, r):
        assert np.all(np.isfinite(x))
        assert np.array_equal(np.roll(x, (sy, sx), axis=(0, 1)), y)
    m0 = float(np.sum(q[0], dtype=np.float64))
    m1 = float(np.sum(a[0], dtype=np.float64))
    assert abs(m1 - m0) / m0 < 1e-6


def test_16384_lake_at_rest(ctx):
    n = 16384
    h = np.full((n, n), 1.5, dtype=np.float32)
    z = np.zeros_like(h)
    sim = fv.KP07_dimsplit.KP07_dimsplit(ctx, h, z, z, n, n, 1.0, 1.0, 9.81)
    sim.advance(3)
    out = sim.download()
    assert np.array_equal(out[0], h)
    assert not np.any(out[1]) and not np.any(out[2])
