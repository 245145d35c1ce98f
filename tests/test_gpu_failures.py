"""Failure detection without a GPU fault.

Every wait in the stage kernels is bounded: a CTA whose tile load does not
arrive within the poll limit sets the simulation's error flag, waits (again
boundedly) for its copies in flight, writes nothing, and the next
synchronising call returns FV_ERR_DEVICE, raised as FVError.  These tests make
the waits run out on purpose -- a barrier that no copy completes, and a poll
limit of zero -- and check the reported status and that the CUDA context stays
usable.  Nothing here faults, traps or hangs a GPU.
"""

import ctypes

import pytest

from conftest import bump, kelvin_helmholtz, rel_linf

import finitevolumegpu_b200 as fv
from finitevolumegpu_b200 import _lib
from oracle.oracle import OracleSim

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up():
    gave_up = ctypes.c_int(-1)
    _lib.check(_lib.lib().fv_selftest_bounded_wait(1000, ctypes.byref(gave_up)))
    assert gave_up.value == 1


@pytest.mark.parametrize("scheme", ["KP07_dimsplit", "KP07", "EE2D_KP07_dimsplit"])
def test_stage_kernel_gives_up_and_context_survives(ctx, scheme):
    nx, ny = 200, 150
    if scheme == "EE2D_KP07_dimsplit":
        q = kelvin_helmholtz(nx, ny)
        args = (nx, ny, 1.0 / nx, 1.0 / ny, 0.0, 1.4)
        okw = {"gamma": 1.4}
        t_end = 0.02
    else:
        q = list(bump(nx, ny))
        args = (nx, ny, 1.0, 1.0, 9.81)
        okw = {}
        t_end = 2.0
    sim = fv.SCHEMES[scheme](ctx, *q, *args)
    _lib.check(_lib.lib().fv_sim_set_wait_limit(sim._handle, 0))
    with pytest.raises(_lib.FVError, match="gave up"):
        sim.simulate(t_end)
    del sim
    # the context stays usable: a new simulation runs and matches the oracle
    sim = fv.SCHEMES[scheme](ctx, *q, *args)
    ref = OracleSim(scheme, q, *args[:5], **okw)
    sim.simulate(t_end)
    ref.simulate(t_end)
    assert sim.simSteps() == ref.simSteps()
    for a, b in zip(sim.download(), ref.download()):
        assert rel_linf(a, b) < 5e-5


def test_default_wait_limit_restored(ctx):
    nx, ny = 96, 64
    q = list(bump(nx, ny))
    sim = fv.KP07_dimsplit.KP07_dimsplit(ctx, *q, nx, ny, 1.0, 1.0, 9.81)
    lib = _lib.lib()
    _lib.check(lib.fv_sim_set_wait_limit(sim._handle, 0))
    _lib.check(lib.fv_sim_set_wait_limit(sim._handle, -1))
    sim.simulate(1.0)
    assert sim.simSteps() > 0
