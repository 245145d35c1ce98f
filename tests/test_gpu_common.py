"""Checkpoint/resume and snapshot output with the sm_100a simulators.

A simulator resumed from a checkpoint (state, t, nt, dt and the last CFL
minimum) must take exactly the steps the uninterrupted simulator takes: the
continued runs are compared bit for bit."""

import numpy as np
import pytest

from conftest import bump, kelvin_helmholtz

import finitevolumegpu_b200 as fv
from finitevolumegpu_b200.Common import load_checkpoint, quantize, runSimulation, save_checkpoint

pytestmark = pytest.mark.gpu

PERIODIC = fv.BoundaryCondition(fv.BoundaryCondition.getTypes(0x02020202))


def make(ctx, scheme, nx, ny):
    if scheme == "EE2D_KP07_dimsplit":
        return fv.SCHEMES[scheme](ctx, *kelvin_helmholtz(nx, ny), nx, ny, 1.0 / nx, 1.0 / ny, 0.0, 1.4,
                                  boundary_conditions=PERIODIC, cfl_scale=0.45), (0.01, 0.02)
    return fv.SCHEMES[scheme](ctx, *bump(nx, ny), nx, ny, 1.0, 1.0, 9.81, cfl_scale=0.45), (4.0, 5.0)


@pytest.mark.parametrize("scheme", ["KP07_dimsplit", "HLL", "KP07", "WAF", "EE2D_KP07_dimsplit"])
def test_resume_from_checkpoint_is_exact(ctx, tmp_path, scheme):
    nx, ny = 150, 110
    sim, (t1, t2) = make(ctx, scheme, nx, ny)
    sim.simulate(t1)
    path = save_checkpoint(sim, str(tmp_path / "ck"))
    sim.simulate(t2)
    resumed = load_checkpoint(ctx, path)
    assert type(resumed) is type(sim)
    resumed.simulate(t2)
    assert resumed.simSteps() == sim.simSteps() and resumed.simTime() == sim.simTime()
    for a, b in zip(resumed.download(), sim.download()):
        assert np.array_equal(a, b)


def test_run_simulation_frames_match_simulator(ctx, tmp_path):
    from scipy.io import netcdf_file

    nx, ny = 96, 80
    h, hu, hv = bump(nx, ny)
    args = {"context": ctx, "h0": h, "hu0": hu, "hv0": hv, "nx": nx, "ny": ny, "dx": 1.0, "dy": 1.0, "g": 9.81}
    times = np.array([0.0, 1.0, 2.5])
    fname, _, _ = runSimulation(fv.KP07_dimsplit.KP07_dimsplit, args, str(tmp_path / "kp.nc"), times,
                                ["h", "hu", "hv"])
    sim = fv.KP07_dimsplit.KP07_dimsplit(ctx, h, hu, hv, nx, ny, 1.0, 1.0, 9.81)
    with netcdf_file(fname, "r", mmap=False) as f:
        for k, dt in enumerate(np.diff(np.concatenate([[0.0], times]))):
            if dt > 0:
                sim.simulate(dt)
            for v, name in enumerate(("h", "hu", "hv")):
                assert np.array_equal(f.variables[name][k], quantize(sim.download([v])[0], 3))
