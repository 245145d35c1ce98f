"""The seeded benchmark configurations, checked end to end on the GPU.

* Config 1: KP07_dimsplit, 256 x 256, dx = dy = 1, theta = 1.3,
  cfl_scale = 0.45, reflective walls, Gaussian bump h = 1 + A exp(-r^2/(2 sigma^2))
  with A ~ U(0.1, 0.5), centre ~ U(0.3, 0.7) x domain, sigma = 20 cells;
  1000 steps.  Compared with the reference's own kernels after 100 steps
  (relative L-inf <= 1e-5) and with the FP64 oracle after 1000 steps
  (relative L1 <= 1e-4); FP64 mass sum conserved to FP32 round-off.
* Config 2: the seven SWE schemes on the 4096 x 4096 seeded circular dam
  break (h = 1 inside R ~ U(0.1, 0.3) x width, 0.1 outside), reflective
  walls, cfl_scale 0.9, 200 steps, against the reference's own kernels on
  the same inputs: relative L1 <= 1e-4 per conserved variable, and relative
  L-inf within 1e-5 or twice the distance between two valid builds of the
  reference (at a dam break WAF and KP07 amplify single roundings to 1e-3).
  FORCE goes unstable at this step size in the reference (dt is refreshed
  only every 100 steps while the flow speeds up), and cells become NaN here
  as there: the cells whose finiteness differs from the reference's may be
  no more than between the reference's two builds, and the cells finite in
  both are held to twice the distance between those builds (the growing
  instability amplifies every rounding).
* Config 3: EE2D_KP07_dimsplit Kelvin-Helmholtz, gamma = 1.4, periodic:
  at 4096 x 2048 for 500 steps the FP64 sums of rho, rho*u, rho*v and E stay
  at their initial values to FP32 round-off; the relative L1/L-inf error
  against the FP64 oracle is measured on a 512 x 256 grid of the same problem
  (the FP64 oracle cannot run the full size in test time).

FVGPU_CONFIG_OUT (optional) names a JSON-lines file that receives the measured
numbers.
"""

import json
import os

import numpy as np
import pytest

from conftest import rel_l1, rel_linf

import finitevolumegpu_b200 as fv
from oracle import ref_kernels
from oracle.oracle import OracleSim

pytestmark = pytest.mark.gpu

PERIODIC = fv.BoundaryCondition(fv.BoundaryCondition.getTypes(0x02020202))


def record(rec):
    out = os.environ.get("FVGPU_CONFIG_OUT")
    print(json.dumps(rec))
    if out:
        with open(out, "a") as f:
            f.write(json.dumps(rec) + "\n")


def config1_bump(seed=1, n=256):
    rng = np.random.default_rng(seed)
    A = rng.uniform(0.1, 0.5)
    cx, cy = rng.uniform(0.3, 0.7) * n, rng.uniform(0.3, 0.7) * n
    y, x = np.mgrid[0:n, 0:n] + 0.5
    h = (1.0 + A * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * 20.0 ** 2))).astype(np.float32)
    z = np.zeros_like(h)
    return [h, z, z.copy()]


def kh(nx, ny, seed=3, gamma=1.4):
    rng = np.random.default_rng(seed)
    phi = rng.uniform(0, 2 * np.pi)
    yy = (np.arange(ny) + 0.5) / ny
    xx = (np.arange(nx) + 0.5) / nx
    X, Y = np.meshgrid(xx, yy)
    band = (Y >= 0.25) & (Y < 0.75)
    rho = np.where(band, 2.0, 1.0)
    u = np.where(band, 0.5, -0.5)
    v = 0.01 * np.sin(4 * np.pi * X + phi)
    E = 2.5 / (gamma - 1.0) + 0.5 * rho * (u ** 2 + v ** 2)
    return [a.astype(np.float32) for a in (rho, rho * u, rho * v, E)]


def advance_host(sim, n):
    """n steps of simulate()'s schedule on a host-driven simulator (oracle or reference kernels)."""
    for _ in range(n):
        if sim.nt % 100 == 0:
            sim.dt = sim.dtype.type(sim.computeDt() * sim.dtype.type(sim.cfl_scale))
        sim.step(sim.dt)


def test_config1_kp07_dimsplit_256(ctx):
    n = 256
    q = config1_bump()
    sim = fv.KP07_dimsplit.KP07_dimsplit(ctx, *q, n, n, 1.0, 1.0, 9.81, theta=1.3, cfl_scale=0.45)
    m0 = sim.conservation()[0]
    ref = ref_kernels.RefKernelSim("KP07_dimsplit", q, n, n, 1.0, 1.0, 9.81, theta=1.3, cfl_scale=0.45)
    advance_host(ref, 100)
    sim.advance(100)
    e100 = [rel_linf(a, b) for a, b in zip(sim.download(), ref.download())]
    assert max(e100) <= 1e-5, e100
    sim.advance(900)
    f64 = OracleSim("KP07_dimsplit", q, n, n, 1.0, 1.0, 9.81, theta=1.3, cfl_scale=0.45, dtype=np.float64)
    advance_host(f64, 1000)
    got = sim.download()
    l1 = [rel_l1(a, b) for a, b in zip(got, f64.download())]
    linf = [rel_linf(a, b) for a, b in zip(got, f64.download())]
    m1 = sim.conservation()[0]
    record({"config": 1, "steps": 1000, "rel_linf_vs_reference_kernels_at_100": e100,
            "rel_l1_vs_fp64_oracle_at_1000": l1, "rel_linf_vs_fp64_oracle_at_1000": linf,
            "mass_rel_change": abs(m1 - m0) / m0})
    assert max(l1) <= 1e-4, l1
    assert abs(m1 - m0) / m0 <= 1e-6


def config2_dam_break(n=4096, seed=0):
    rng = np.random.default_rng(seed)
    R = rng.uniform(0.1, 0.3) * n
    y, x = np.mgrid[0:n, 0:n] + 0.5
    h = np.where(np.hypot(x - n / 2.0, y - n / 2.0) < R, 1.0, 0.1).astype(np.float32)
    z = np.zeros_like(h)
    return [h, z, z.copy()]


@pytest.fixture(scope="module")
def config2_state():
    return config2_dam_break()


@pytest.mark.parametrize("scheme", ["LxF", "FORCE", "HLL", "HLL2", "WAF", "KP07", "KP07_dimsplit"])
def test_config2_vs_reference_kernels(ctx, config2_state, scheme):
    n, steps = 4096, 200
    q = config2_state

    def run_ref(build):
        ref = ref_kernels.RefKernelSim(scheme, q, n, n, 1.0, 1.0, 9.81, cfl_scale=0.9, build=build)
        advance_host(ref, steps)
        out = ref.download()
        ref.close()
        return out

    want = run_ref(None)
    other = run_ref("nofma")
    sim = fv.SCHEMES[scheme](ctx, *q, n, n, 1.0, 1.0, 9.81, cfl_scale=0.9)
    sim.advance(steps)
    got = sim.download()
    del sim
    l1, linf, floor, floor_l1, finite = [], [], [], [], []
    for a, b, c in zip(got, want, other):
        fa, fb, fc = np.isfinite(a), np.isfinite(b), np.isfinite(c)
        # cells whose finiteness differs from the reference's: no more than
        # between the reference's two builds (plus 1e-4 of the cells)
        assert (fa != fb).mean() <= (fc != fb).mean() + 1e-4, (scheme, (fa != fb).mean(), (fc != fb).mean())
        finite.append(float(fb.mean()))
        m, mc = fa & fb, fb & fc
        if not m.any():
            l1.append(0.0), linf.append(0.0), floor.append(0.0), floor_l1.append(0.0)
            continue
        l1.append(rel_l1(a[m], b[m]))
        linf.append(rel_linf(a[m], b[m]))
        floor.append(rel_linf(c[mc], b[mc]) if mc.any() else 0.0)
        floor_l1.append(rel_l1(c[mc], b[mc]) if mc.any() else 0.0)
    record({"config": 2, "scheme": scheme, "n": n, "steps": steps, "rel_l1_vs_reference_kernels": l1,
            "rel_linf_vs_reference_kernels": linf, "reference_build_to_build_rel_linf": floor,
            "reference_build_to_build_rel_l1": floor_l1, "finite_fraction": finite})
    for v in range(3):
        # 1e-4; the unstable FORCE run only as close as the reference's two builds are to each other
        assert l1[v] <= max(1e-4, 2.0 * floor_l1[v]), (scheme, v, l1, floor_l1)
        assert linf[v] <= max(1e-5, 2.0 * floor[v]), (scheme, v, linf, floor)


def test_config3_ee2d_conservation_full_size(ctx):
    nx, ny = 4096, 2048
    q = kh(nx, ny)
    sim = fv.EE2D_KP07_dimsplit.EE2D_KP07_dimsplit(ctx, *q, nx, ny, 1.0 / nx, 1.0 / ny, 0.0, 1.4,
                                                   boundary_conditions=PERIODIC)
    s0 = sim.conservation()
    sim.advance(500)
    s1 = sim.conservation()
    sim.check()
    scale = np.array([abs(s0[0]), max(abs(s0[1]), abs(s0[0]) * 0.5), abs(s0[0]) * 0.01, abs(s0[3])])
    drift = np.abs(s1 - s0) / scale
    record({"config": 3, "nx": nx, "ny": ny, "steps": 500, "t": sim.simTime(), "sums_start": s0.tolist(),
            "sums_end": s1.tolist(), "relative_drift": drift.tolist()})
    # FP32 state: each sum is conserved to round-off of ~8.4 M cells x 500 steps
    assert np.all(drift <= 1e-5), drift


def test_config3_ee2d_error_vs_fp64(ctx):
    nx, ny = 512, 256
    q = kh(nx, ny)
    sim = fv.EE2D_KP07_dimsplit.EE2D_KP07_dimsplit(ctx, *q, nx, ny, 1.0 / nx, 1.0 / ny, 0.0, 1.4,
                                                   boundary_conditions=PERIODIC)
    sim.advance(500)
    f64 = OracleSim("EE2D_KP07_dimsplit", q, nx, ny, 1.0 / nx, 1.0 / ny, 0.0, gamma=1.4, bc=0x02020202,
                    dtype=np.float64)
    advance_host(f64, 500)
    f32 = OracleSim("EE2D_KP07_dimsplit", q, nx, ny, 1.0 / nx, 1.0 / ny, 0.0, gamma=1.4, bc=0x02020202,
                    dtype=np.float32)
    advance_host(f32, 500)
    got, want = sim.download(), f64.download()
    l1 = [rel_l1(a, b) for a, b in zip(got, want)]
    linf = [rel_linf(a, b) for a, b in zip(got, want)]
    floor = [rel_l1(a, b) for a, b in zip(f32.download(), want)]
    record({"config": 3, "nx": nx, "ny": ny, "steps": 500, "rel_l1_vs_fp64": l1, "rel_linf_vs_fp64": linf,
            "ieee_fp32_oracle_rel_l1_vs_fp64": floor})
    # rho, rho*u, E: 1e-4.  rho*v (the 1 % Kelvin-Helmholtz perturbation) is
    # held to twice the distance between the IEEE FP32 oracle and FP64, the
    # round-off floor of any FP32 evaluation of this scheme.
    for v in (0, 1, 3):
        assert l1[v] <= 1e-4, l1
    assert l1[2] <= max(1e-4, 2.0 * floor[2]), (l1[2], floor[2])
