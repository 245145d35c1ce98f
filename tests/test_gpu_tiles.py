"""Every tile configuration of every scheme computes the same cells.

The stage kernels round each formula the same way whatever tile shape, lane
width (one line, or two lines in packed f32x2 arithmetic) or kernel computes
a cell, so all tile configurations of a scheme, plain and batched, must give
bitwise-identical states.  The first configuration is also held to the CPU
oracle with the tolerances of the parity tests.
"""

import numpy as np
import pytest

from conftest import bump, kelvin_helmholtz, rel_linf

import finitevolumegpu_b200 as fv
from finitevolumegpu_b200.Autotuner import BATCH_TILE_CONFIGS, TILE_CONFIGS, _Fixed
from finitevolumegpu_b200.batch import Batch
from oracle.oracle import OracleSim

pytestmark = pytest.mark.gpu

MIXED = 0x02020303  # north/south periodic, east/west reflective


def case(scheme, nx, ny):
    if scheme == "EE2D_KP07_dimsplit":
        return kelvin_helmholtz(nx, ny), 1.0 / nx, 1.0 / ny, 0.0, 0.05
    return list(bump(nx, ny)), 1.0, 1.0, 9.81, 6.0


def run_plain(ctx, scheme, tile, q, nx, ny, dx, dy, g, t_end, bc):
    saved = ctx.autotuner
    ctx.autotuner = _Fixed(tile)
    try:
        cls = fv.SCHEMES[scheme]
        b = fv.BoundaryCondition(fv.BoundaryCondition.getTypes(bc))
        if scheme == "EE2D_KP07_dimsplit":
            sim = cls(ctx, *q, nx, ny, dx, dy, g, 1.4, boundary_conditions=b, cfl_scale=0.45)
        else:
            sim = cls(ctx, *q, nx, ny, dx, dy, g, boundary_conditions=b, cfl_scale=0.45)
    finally:
        ctx.autotuner = saved
    sim.simulate(t_end)
    return sim.download(), sim.simSteps(), sim.tile_info()


@pytest.mark.parametrize("scheme", list(TILE_CONFIGS))
def test_all_tile_configs_identical(ctx, scheme):
    nx, ny = 253, 191  # ragged against every tile width and height
    q, dx, dy, g, t_end = case(scheme, nx, ny)
    runs = [run_plain(ctx, scheme, k, q, nx, ny, dx, dy, g, t_end, MIXED) for k in range(TILE_CONFIGS[scheme])]
    shapes = {(r[2]["tile_w"], r[2]["tile_h"], r[2]["threads"]) for r in runs}
    assert len(shapes) == len(runs), shapes  # every configuration is a distinct kernel
    base, nt, _ = runs[0]
    for k, (got, nt_k, info) in enumerate(runs[1:], start=1):
        assert nt_k == nt
        for v, (a, w) in enumerate(zip(got, base)):
            assert np.array_equal(a, w), (scheme, k, info, v, rel_linf(a, w))
    ref = OracleSim(scheme, q, nx, ny, dx, dy, g, gamma=1.4, cfl_scale=0.45, bc=MIXED)
    ref.simulate(t_end)
    assert ref.simSteps() == nt
    tols = (2e-5, 2e-5, 5e-5, 2e-5) if scheme == "EE2D_KP07_dimsplit" else (2e-5,) * 3
    for a, w, tol in zip(base, ref.download(), tols):
        assert rel_linf(a, w) < tol, (scheme, rel_linf(a, w))


@pytest.mark.parametrize("scheme", list(BATCH_TILE_CONFIGS))
def test_all_batch_tile_configs_match_plain(ctx, scheme):
    sizes = [(253, 191), (70, 300), (41, 37)]
    cases = [case(scheme, nx, ny) for nx, ny in sizes]
    want = [run_plain(ctx, scheme, 0, q, nx, ny, dx, dy, g, t_end, MIXED)
            for (nx, ny), (q, dx, dy, g, t_end) in zip(sizes, cases)]
    bc = fv.BoundaryCondition(fv.BoundaryCondition.getTypes(MIXED))
    for tile in range(BATCH_TILE_CONFIGS[scheme]):
        b = Batch(ctx, scheme, g=cases[0][3], cfl_scale=0.45, max_instances=4, tile=tile)
        slots = [b.add(q, nx, ny, dx, dy, t_end, bc) for (nx, ny), (q, dx, dy, g, t_end) in zip(sizes, cases)]
        b.run_to_completion()
        for slot, (state, nt, _) in zip(slots, want):
            assert b.status(slot)["nt"] == nt
            for v, (a, w) in enumerate(zip(b.download(slot), state)):
                assert np.array_equal(a, w), (scheme, tile, b.info(), slot, v, rel_linf(a, w))
        del b
