"""Known answers and invariants of the sm_100a kernels themselves (the same pins
the oracle is held to in test_oracle.py, here run through the CUDA path):

  * the wet Stoker dam break of the reference's ConvergenceShock1D notebook
    (L = 10 m, h = 0.005 / 0.001, t = 6 s; the analytic solution behind the
    reference's SWASHES files): L1 error falls under refinement, with the same
    bounds the FP64 oracle meets;
  * convergence order on a smooth wave (the reference's ConvergenceSmooth1D
    study): about 2 for the second-order schemes, about 1 for the first-order
    ones, against an FP64 run of the scheme at 2048 cells;
  * mirror symmetry of a symmetric bump between reflective walls;
  * transpose equivariance of the dimensionally split substeps;
  * conservation of mass with reflective and periodic walls for every scheme.

Thresholds come from the oracle on the same inputs: orders between 64 and
256 cells 1.81-2.02 (second order) and 0.80-1.00 (first order); Stoker L1
errors at 512 cells between 3.3e-6 (WAF) and 4.6e-5 (LxF).
"""

import numpy as np
import pytest

from conftest import bump, dam_break, rel_linf

import finitevolumegpu_b200 as fv
from oracle.oracle import OracleSim
from oracle.stoker import stoker

pytestmark = pytest.mark.gpu

SWE = ["LxF", "FORCE", "HLL", "HLL2", "WAF", "KP07", "KP07_dimsplit"]
FIRST_ORDER = ("LxF", "FORCE", "HLL")
REFLECTIVE = 0x03030303
PERIODIC = 0x02020202


def make_sim(ctx, scheme, vars_, nx, ny, dx=1.0, dy=1.0, bc=REFLECTIVE):
    b = fv.BoundaryCondition(fv.BoundaryCondition.getTypes(bc))
    return fv.SCHEMES[scheme](ctx, *vars_, nx, ny, dx, dy, 9.81, boundary_conditions=b)


def lines(h, ny=4):
    """A 1-D profile repeated over ny rows, at rest."""
    h = np.tile(np.asarray(h, np.float64), (ny, 1)).astype(np.float32)
    z = np.zeros_like(h)
    return [h, z, z.copy()]


@pytest.mark.parametrize("scheme", SWE)
def test_dam_break_converges_to_stoker(ctx, scheme):
    errs = []
    for nx in (128, 256, 512):
        dx = 10.0 / nx
        x = (np.arange(nx) + 0.5) * dx
        sim = make_sim(ctx, scheme, lines(np.where(x < 5.0, 0.005, 0.001)), nx, 4, dx, 1.0)
        # explicit dt from a velocity estimate, as ConvergenceShock1D.ipynb cell 8 does
        sim.simulate(6.0, dt=0.45 * dx / (0.3 + np.sqrt(9.81 * 0.005)))
        hs, _ = stoker(x, 6.0)
        errs.append(np.mean(np.abs(sim.download()[0][1] - hs)))
    order = np.log2(errs[0] / errs[1]), np.log2(errs[1] / errs[2])
    assert errs[2] < errs[1] < errs[0], (scheme, errs)
    assert min(order) > 0.5, (scheme, order)
    assert errs[2] < 6e-5, (scheme, errs)


@pytest.mark.parametrize("scheme", SWE)
def test_smooth_convergence_order(ctx, scheme):
    """Errors of the FP32 kernels at 64, 128 and 256 cells against an FP64 run
    of the scheme at 2048 cells.  The reference solution is FP64 because FP32
    itself drifts: the IEEE FP32 oracle ends 1.8e-5 (mean |h|) from FP64 after
    the 1669 steps of the 2048-cell split run, one-signed, and 1.3e-6 after the
    418 steps at 512 cells; the GPU kernels drift the same, which would mask
    the truncation error of the finer grids.  At 256 cells the drift is near
    3e-7 against errors of 1.8e-5 and more."""
    L, fine = 10.0, 2048

    def setup(nx):
        dx = L / nx
        x = (np.arange(nx) + 0.5) * dx
        return lines(1.0 + 0.05 * np.exp(-((x - 5.0) / 1.0) ** 2)), dx, 0.4 * dx / (np.sqrt(9.81 * 1.05) + 0.05)

    def run(nx):
        q, dx, dt = setup(nx)
        sim = make_sim(ctx, scheme, q, nx, 4, dx, dx)
        sim.simulate(1.0, dt=dt)
        return sim.download()[0][1].astype(np.float64)

    q, dx, dt = setup(fine)
    oracle = OracleSim(scheme, q, fine, 4, dx, dx, 9.81, dtype=np.float64)
    oracle.simulate(1.0, dt=dt)
    ref = oracle.download()[0][1]
    errs = [np.mean(np.abs(run(nx) - ref.reshape(nx, fine // nx).mean(axis=1))) for nx in (64, 128, 256)]
    orders = [np.log2(errs[i] / errs[i + 1]) for i in range(2)]
    if scheme in FIRST_ORDER:
        assert all(0.7 < o < 1.4 for o in orders), (scheme, errs, orders)
    else:
        assert all(o > 1.6 for o in orders), (scheme, errs, orders)


@pytest.mark.parametrize("scheme", SWE)
def test_mirror_symmetry(ctx, scheme):
    """A bump centred between reflective walls stays symmetric in x and y, with
    the normal momentum antisymmetric, to FP32 round-off (the face fluxes on
    either side of the axis round differently; a misplaced wall or ghost cell
    shows up at the 1e-2 level)."""
    nx = ny = 32
    sim = make_sim(ctx, scheme, bump(nx, ny, cx=16.0, cy=16.0), nx, ny)
    sim.simulate(2.0)
    H, HU, HV = sim.download()
    tol = 5e-5
    assert rel_linf(H[::-1, :], H) < tol and rel_linf(H[:, ::-1], H) < tol
    assert np.max(np.abs(HU + HU[:, ::-1])) <= tol * np.max(np.abs(HU))
    assert np.max(np.abs(HV + HV[::-1, :])) <= tol * np.max(np.abs(HV))
    assert np.max(np.abs(HU - HU[::-1, :])) <= tol * np.max(np.abs(HU))


@pytest.mark.parametrize("scheme", ["HLL2", "KP07_dimsplit", "WAF"])
def test_transpose_equivariance(ctx, scheme):
    """Transposing the grid and swapping hu and hv commutes with a split substep
    whose sweep order is swapped (substep 0 sweeps x then y, substep 1 y then x)."""
    nx, ny = 24, 18
    h, _, hv = bump(nx, ny)
    hu = ((0.03 * np.sin(np.arange(nx) / 3.0))[None, :] * np.ones((ny, 1))).astype(np.float32)
    a = make_sim(ctx, scheme, [h, hu, hv], nx, ny)
    b = make_sim(ctx, scheme, [h.T.copy(), hv.T.copy(), hu.T.copy()], ny, nx)
    a.substep(0.05, 0)
    b.substep(0.05, 1)
    A, B = a.download(), b.download()
    assert rel_linf(A[0], B[0].T) < 1e-6
    assert rel_linf(A[1], B[2].T) < 1e-6
    assert rel_linf(A[2], B[1].T) < 1e-6


@pytest.mark.parametrize("scheme", SWE)
@pytest.mark.parametrize("bc", [REFLECTIVE, PERIODIC], ids=["reflective", "periodic"])
def test_mass_conserved(ctx, scheme, bc):
    nx, ny = 96, 64
    h, hu, hv = dam_break(nx, ny)
    sim = make_sim(ctx, scheme, [h, hu, hv], nx, ny, bc=bc)
    m0 = sim.conservation()[0]
    sim.simulate(5.0)
    assert sim.simSteps() > 10
    m1 = sim.conservation()[0]
    assert abs(m1 - m0) / m0 < 1e-6, (scheme, m0, m1)
