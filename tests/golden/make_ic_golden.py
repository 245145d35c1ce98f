"""Golden vectors of the reference's initial-condition generators.

Loads GPUSimulators/helpers/InitialConditions.py from a reference checkout
(path as the first argument) with a stand-in for GPUSimulators.Simulator,
which it imports only for BoundaryCondition (the real module needs PyCUDA),
runs every generator on small cases and writes tests/golden/ic_ref.npz.
Run in an environment with the reference tree; the fixture travels with the
repository.
"""

import enum
import importlib.util
import os
import sys
import types

import numpy as np


class _BC(object):
    class Type(enum.IntEnum):
        Dirichlet = 0
        Neumann = 1
        Periodic = 2
        Reflective = 3

    def __init__(self, types=None):
        self.types = dict(types or {})

    def code(self):
        return [int(self.types[k]) for k in ("north", "south", "east", "west")]


class _Grid(object):
    def __init__(self, gy, j):
        self.grid = np.array([1, gy])
        self.j = j

    def getCoordinate(self, index=None):
        return 0, (self.j if index is None else index)


def load(ref_root):
    pkg = types.ModuleType("GPUSimulators")
    sim = types.ModuleType("GPUSimulators.Simulator")
    sim.BoundaryCondition = _BC
    pkg.Simulator = sim
    sys.modules["GPUSimulators"] = pkg
    sys.modules["GPUSimulators.Simulator"] = sim
    path = os.path.join(ref_root, "GPUSimulators", "helpers", "InitialConditions.py")
    spec = importlib.util.spec_from_file_location("ref_initial_conditions", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def cases(ic):
    out = {}
    out["extent_plain"] = np.array(ic.getExtent(4.0, 1.0, 40, 10, None))
    out["extent_grid"] = np.array(ic.getExtent(4.0, 1.0, 40, 10, _Grid(3, 1)))
    a = np.random.default_rng(1).random((12, 16)).astype(np.float32)
    out["downsample_in"] = a
    out["downsample"] = ic.downsample(a, 2, 4)
    for name, args, kw in (("bump", (32, 24, 10.0, 8.0), {}),
                           ("bump_ref", (16, 12, 10.0, 8.0), {"ref_nx": 64, "ref_ny": 48, "x_center": 0.4})):
        h, hu, hv, dx, dy = ic.bump(*args, **kw)
        out[name + "_h"], out[name + "_hu"], out[name + "_hv"] = h, hu, hv
        out[name + "_d"] = np.array([dx, dy])

    def euler(prefix, d):
        for k in ("rho", "rho_u", "rho_v", "E"):
            out[prefix + "_" + k] = np.asarray(d[k])
        out[prefix + "_scalars"] = np.array([d["nx"], d["ny"], d["dx"], d["dy"], d["g"], d["gamma"]], dtype=np.float64)
        out[prefix + "_bc"] = np.array(d["boundary_conditions"].code())

    euler("shock", ic.genShockBubble(40, 12, 1.4))
    euler("shock_grid", ic.genShockBubble(40, 6, 1.4, grid=_Grid(2, 1)))
    np.random.seed(11)
    euler("kh", ic.genKelvinHelmholtz(32, 24, 1.4))
    np.random.seed(12)
    euler("kh_rough", ic.genKelvinHelmholtz(16, 16, 1.4, roughness=1.0))
    np.random.seed(13)
    euler("kh_smooth", ic.genKelvinHelmholtz(40, 20, 1.67, roughness=0.05))
    euler("rt0", ic.genRayleighTaylor(16, 48, 1.4, version=0))
    euler("rt1", ic.genRayleighTaylor(16, 48, 1.4, version=1))
    return out


if __name__ == "__main__":
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FVGPU_REFERENCE_ROOT", "")
    if not ref_root:
        sys.exit("usage: make_ic_golden.py <reference checkout> (or set FVGPU_REFERENCE_ROOT)")
    out = cases(load(ref_root))
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ic_ref.npz")
    np.savez_compressed(dst, **out)
    print("wrote", dst, len(out), "arrays")
