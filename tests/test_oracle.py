"""CPU tests of the oracle: known answers, invariants and the reference's host
semantics.  These pin the checker that the GPU parity tests rely on."""

import os

import numpy as np
import pytest

from conftest import bump, dam_break, kelvin_helmholtz, rel_l1, rel_linf

from oracle.oracle import OracleSim, oracle_substep
from oracle.stoker import stoker

SWE = ["LxF", "FORCE", "HLL", "HLL2", "WAF", "KP07", "KP07_dimsplit"]
SPLIT = ["FORCE", "HLL", "HLL2", "WAF", "KP07_dimsplit"]
# A reference checkout, when present, adds the full SWASHES files to the
# committed samples of them (tests/golden/swashes_stoker.npz).
REFERENCE_ROOT = os.environ.get("FVGPU_REFERENCE_ROOT", "")
SWASHES_GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "swashes_stoker.npz")


# ---------------------------------------------------------------- known answers

def _check_stoker(d):
    h, u = stoker(d[:, 0], 6.0)
    assert np.max(np.abs(h - d[:, 1])) < 5e-8  # files print 6 significant digits
    assert np.max(np.abs(u - d[:, 2])) < 2e-6


@pytest.mark.parametrize("nx", [128, 256, 512, 1024, 2048, 4096])
def test_stoker_matches_swashes(nx):
    """The analytic Stoker solution reproduces the reference's SWASHES files:
    the committed samples of each file, and the whole file where a reference
    checkout is given."""
    _check_stoker(np.load(SWASHES_GOLDEN)["nx%d" % nx])
    path = os.path.join(REFERENCE_ROOT, "reference", "swashes_1_nx=%d.csv" % nx)
    if REFERENCE_ROOT and os.path.exists(path):
        _check_stoker(np.genfromtxt(path, comments="#", delimiter="\t", usecols=(0, 1, 2)))


def dam_1d(nx, ny=4):
    """Wet dam break of ConvergenceShock1D.ipynb cell 8: L = 10 m, dam at 5 m."""
    x = (np.arange(nx) + 0.5) * 10.0 / nx
    h = np.where(x < 5.0, 0.005, 0.001)
    h = np.tile(h, (ny, 1)).astype(np.float32)
    z = np.zeros_like(h)
    return h, z, z.copy()


@pytest.mark.parametrize("scheme", SWE)
def test_dam_break_converges_to_stoker(scheme):
    """L1 error against Stoker at t = 6 s decreases under refinement."""
    errs = []
    for nx in (128, 256, 512):
        h, hu, hv = dam_1d(nx)
        sim = OracleSim(scheme, [h, hu, hv], nx, 4, 10.0 / nx, 1.0, 9.81, dtype=np.float64)
        # explicit dt from a velocity estimate, as ConvergenceShock1D.ipynb cell 8 does
        dx = 10.0 / nx
        dt = 0.45 * dx / (0.3 + np.sqrt(9.81 * 0.005))
        sim.simulate(6.0, dt=dt)
        H = sim.download()[0][1]
        x = (np.arange(nx) + 0.5) * 10.0 / nx
        hs, _ = stoker(x, 6.0)
        errs.append(np.mean(np.abs(H - hs)))
    order = np.log2(errs[0] / errs[1]), np.log2(errs[1] / errs[2])
    assert errs[2] < errs[1] < errs[0], (scheme, errs)
    assert min(order) > 0.4, (scheme, order)
    assert errs[2] < 6e-5, (scheme, errs)


# ---------------------------------------------------------------- invariants

@pytest.mark.parametrize("scheme", SWE)
@pytest.mark.parametrize("bc", [0x03030303, 0x02020202])
def test_mass_conserved(scheme, bc):
    nx, ny = 40, 30
    h, hu, hv = dam_break(nx, ny)
    sim = OracleSim(scheme, [h, hu, hv], nx, ny, 1.0, 1.0, 9.81, bc=bc, dtype=np.float64)
    m0 = h.astype(np.float64).sum()
    sim.simulate(3.0)
    assert abs(sim.download()[0].sum() - m0) / m0 < 1e-13


@pytest.mark.parametrize("scheme", ["LxF", "KP07", "HLL2", "KP07_dimsplit"])
def test_mirror_symmetry(scheme):
    """A symmetric bump stays symmetric under reflective walls (bit-exact)."""
    nx, ny = 32, 32
    h, hu, hv = bump(nx, ny, cx=16.0, cy=16.0)
    sim = OracleSim(scheme, [h, hu, hv], nx, ny, 1.0, 1.0, 9.81, dtype=np.float32)
    sim.simulate(2.0)
    H, HU, HV = sim.download()
    assert np.array_equal(H, H[::-1, :]) and np.array_equal(H, H[:, ::-1])
    assert np.array_equal(HU, -HU[:, ::-1])
    assert np.array_equal(HV, -HV[::-1, :])


@pytest.mark.parametrize("scheme", ["HLL2", "KP07_dimsplit", "WAF"])
def test_transpose_equivariance(scheme):
    """Transposing the grid and swapping hu/hv commutes with a split substep whose sweep order is swapped."""
    nx, ny = 24, 18
    h, hu, hv = bump(nx, ny)
    hu = (0.03 * np.sin(np.arange(nx) / 3.0))[None, :] * np.ones((ny, 1), np.float32)
    hu = hu.astype(np.float32)
    g = 2
    pad = lambda a: np.pad(a, g).astype(np.float32)
    u = [pad(h), pad(hu), pad(hv)]
    ut = [pad(h.T.copy()), pad(hv.T.copy()), pad(hu.T.copy())]
    o = [np.zeros_like(a) for a in u]
    ot = [np.zeros_like(a) for a in ut]
    oracle_substep(scheme, u, o, nx, ny, 1.0, 1.0, 0.05, 9.81, 1.4, 1.3, 0, 2, 0x03030303)
    oracle_substep(scheme, ut, ot, ny, nx, 1.0, 1.0, 0.05, 9.81, 1.4, 1.3, 1, 2, 0x03030303)
    assert np.array_equal(o[0], ot[0].T)
    assert np.array_equal(o[1], ot[2].T)
    assert np.array_equal(o[2], ot[1].T)


def test_fp32_close_to_fp64():
    nx, ny = 64, 48
    q = bump(nx, ny)
    a = OracleSim("KP07_dimsplit", q, nx, ny, 1.0, 1.0, 9.81, cfl_scale=0.45, dtype=np.float32)
    b = OracleSim("KP07_dimsplit", q, nx, ny, 1.0, 1.0, 9.81, cfl_scale=0.45, dtype=np.float64)
    a.simulate(5.0)
    b.simulate(5.0)
    for x, y in zip(a.download(), b.download()):
        assert rel_l1(x, y) < 1e-5


def test_euler_conserves_periodic():
    nx, ny = 48, 32
    q = kelvin_helmholtz(nx, ny)
    sim = OracleSim("EE2D_KP07_dimsplit", q, nx, ny, 1.0 / nx, 1.0 / ny, 0.0, gamma=1.4, bc=0x02020202,
                    dtype=np.float64)
    s0 = [a.astype(np.float64).sum() for a in q]
    sim.simulate(0.1)
    for a, b in zip(sim.download(), s0):
        assert abs(a.sum() - b) <= 1e-12 * max(1.0, abs(b))


def test_euler_predictor_uses_gamma_as_pressure():
    """Parity detail: the reference predictor passes gamma where F_func expects
    the pressure (GPUSimulators/cuda/EE2D_KP07_dimsplit.cu:57-58).  A uniform
    flow with a pressure jump evolves differently from a correct predictor, and
    the oracle must follow the reference."""
    nx, ny = 16, 4
    rho = np.ones((ny, nx), np.float32)
    ru = np.full((ny, nx), 0.3, np.float32)
    rv = np.zeros((ny, nx), np.float32)
    E = np.where(np.arange(nx) < nx // 2, 3.0, 2.0)[None, :].repeat(ny, 0).astype(np.float32)
    g = 2
    pad = lambda a: np.pad(a, g, mode="edge").astype(np.float32)
    u = [pad(a) for a in (rho, ru, rv, E)]
    o1 = [np.zeros_like(a) for a in u]
    o2 = [np.zeros_like(a) for a in u]
    oracle_substep("EE2D_KP07_dimsplit", u, o1, nx, ny, 0.1, 0.1, 0.01, 0.0, 1.4, 1.3, 0, 2, 0x03030303)
    oracle_substep("EE2D_KP07_dimsplit", u, o2, nx, ny, 0.1, 0.1, 0.01, 0.0, 1.7, 1.3, 0, 2, 0x03030303)
    assert not np.array_equal(o1[3], o2[3])


# ---------------------------------------------------------------- host semantics

def test_dt_schedule_every_100_steps():
    nx, ny = 32, 24
    q = dam_break(nx, ny)
    sim = OracleSim("KP07_dimsplit", q, nx, ny, 1.0, 1.0, 9.81)
    seen = []
    orig = sim.computeDt

    def spy():
        seen.append(sim.nt)
        return orig()

    sim.computeDt = spy
    sim.simulate(60.0)
    assert seen[:3] == [0, 100, 200][: len(seen[:3])]
    assert all(n % 100 == 0 for n in seen)


def test_last_step_hits_t_end():
    nx, ny = 32, 24
    q = bump(nx, ny)
    sim = OracleSim("HLL", q, nx, ny, 1.0, 1.0, 9.81)
    sim.simulate(1.2345)
    assert sim.t == pytest.approx(1.2345, abs=1e-7)
    t1, n1 = sim.t, sim.nt
    sim.simulate(0.5, dt=0.3)
    assert sim.nt == n1 + 2 and sim.t == pytest.approx(t1 + 0.5, abs=1e-7)


def test_waf_dt_never_updates():
    """WAFKernel has no CFL output, so computeDt keeps the constructor's fill."""
    nx, ny = 32, 24
    q = dam_break(nx, ny)
    sim = OracleSim("WAF", q, nx, ny, 1.0, 1.0, 9.81)
    d0 = sim.computeDt()
    sim.simulate(5.0)
    assert sim.computeDt() == d0


def test_kp07_rk2_blend():
    """Second RK stage writes 0.5*(u^n + u**) into the buffer holding u^n."""
    nx, ny = 20, 16
    q = bump(nx, ny)
    a = OracleSim("KP07", q, nx, ny, 1.0, 1.0, 9.81, order=2)
    b = OracleSim("KP07", q, nx, ny, 1.0, 1.0, 9.81, order=1)
    dt = np.float32(0.1)
    a.step(dt)
    un = b.download()
    b.step(dt)  # u* = u^n + dt L(u^n)
    ustar = b.download()
    b.step(dt)  # u** = u* + dt L(u*)
    ustar2 = b.download()
    for x, n, s2 in zip(a.download(), un, ustar2):
        np.testing.assert_allclose(x, 0.5 * (n + s2), rtol=0, atol=1e-6)
