"""The initial-condition generators against golden vectors of the reference's own
(GPUSimulators/helpers/InitialConditions.py, run by tests/golden/make_ic_golden.py):
the same arrays bit for bit, the same scalars and boundary conditions."""

import os

import numpy as np
import pytest

from finitevolumegpu_b200 import InitialConditions as IC

GOLD = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ic_ref.npz"))


class Grid(object):
    def __init__(self, gy, j):
        self.grid = np.array([1, gy])
        self.j = j

    def getCoordinate(self, index=None):
        return 0, (self.j if index is None else index)


def same(a, key):
    want = GOLD[key]
    a = np.asarray(a)
    assert a.shape == want.shape, (key, a.shape, want.shape)
    assert a.dtype == want.dtype, (key, a.dtype, want.dtype)
    assert np.array_equal(a, want), (key, np.max(np.abs(a.astype(np.float64) - want)))


def check_euler(prefix, d):
    for k in ("rho", "rho_u", "rho_v", "E"):
        same(d[k], prefix + "_" + k)
    assert np.array_equal([d["nx"], d["ny"], d["dx"], d["dy"], d["g"], d["gamma"]], GOLD[prefix + "_scalars"])
    bc = d["boundary_conditions"]
    assert [int(bc.north), int(bc.south), int(bc.east), int(bc.west)] == GOLD[prefix + "_bc"].tolist()


def test_extent_and_downsample():
    same(IC.getExtent(4.0, 1.0, 40, 10, None), "extent_plain")
    same(IC.getExtent(4.0, 1.0, 40, 10, Grid(3, 1)), "extent_grid")
    same(IC.downsample(GOLD["downsample_in"], 2, 4), "downsample")


def test_bump():
    h, hu, hv, dx, dy = IC.bump(32, 24, 10.0, 8.0)
    for a, k in ((h, "bump_h"), (hu, "bump_hu"), (hv, "bump_hv")):
        same(a, k)
    assert np.array_equal([dx, dy], GOLD["bump_d"])
    h, hu, hv, dx, dy = IC.bump(16, 12, 10.0, 8.0, ref_nx=64, ref_ny=48, x_center=0.4)
    for a, k in ((h, "bump_ref_h"), (hu, "bump_ref_hu"), (hv, "bump_ref_hv")):
        same(a, k)


def test_shock_bubble():
    check_euler("shock", IC.genShockBubble(40, 12, 1.4))
    check_euler("shock_grid", IC.genShockBubble(40, 6, 1.4, grid=Grid(2, 1)))


@pytest.mark.parametrize("prefix,seed,args,kw", [
    ("kh", 11, (32, 24, 1.4), {}),
    ("kh_rough", 12, (16, 16, 1.4), {"roughness": 1.0}),
    ("kh_smooth", 13, (40, 20, 1.67), {"roughness": 0.05}),
])
def test_kelvin_helmholtz(prefix, seed, args, kw):
    np.random.seed(seed)
    check_euler(prefix, IC.genKelvinHelmholtz(*args, **kw))


def test_rayleigh_taylor():
    check_euler("rt0", IC.genRayleighTaylor(16, 48, 1.4, version=0))
    check_euler("rt1", IC.genRayleighTaylor(16, 48, 1.4, version=1))
    with pytest.raises(AssertionError):
        IC.genRayleighTaylor(8, 8, 1.4, version=2)


def test_request_from_arguments_carries_physics():
    d = IC.genRayleighTaylor(16, 48, 1.4)
    r = IC.request_from_arguments(3, d, t_end=0.5, arrival=0.1)
    assert r.batch_key() == ("EE2D_KP07_dimsplit", pytest.approx(0.1), 1.4)
    assert r.nx == 16 and r.ny == 48 and len(r.variables) == 4 and r.variables[0].dtype == np.float32
