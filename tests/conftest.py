import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


@pytest.fixture(scope="session")
def ctx():
    """One device context for all GPU tests; fails (does not skip) without a GPU."""
    from finitevolumegpu_b200 import CudaContext

    return CudaContext.CudaContext(device=0, autotuning=False)


def bump(nx, ny, amp=0.3, cx=None, cy=None, sigma=None, base=1.0):
    """Gaussian bump of water depth on a lake at rest."""
    cx = nx * 0.45 if cx is None else cx
    cy = ny * 0.55 if cy is None else cy
    sigma = max(2.0, min(nx, ny) / 8.0) if sigma is None else sigma
    y, x = np.mgrid[0:ny, 0:nx] + 0.5
    h = base + amp * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * sigma ** 2))
    z = np.zeros_like(h)
    return h.astype(np.float32), z.astype(np.float32), z.astype(np.float32)


def dam_break(nx, ny, radius_frac=0.2, inner=1.0, outer=0.1):
    y, x = np.mgrid[0:ny, 0:nx] + 0.5
    r = np.hypot(x - nx / 2.0, y - ny / 2.0)
    h = np.where(r < radius_frac * min(nx, ny), inner, outer).astype(np.float32)
    z = np.zeros_like(h)
    return h, z, z.copy()


def kelvin_helmholtz(nx, ny, gamma=1.4, phase=0.3):
    y = (np.arange(ny) + 0.5) / ny
    x = (np.arange(nx) + 0.5) / nx
    X, Y = np.meshgrid(x, y)
    band = (Y >= 0.25) & (Y < 0.75)
    rho = np.where(band, 2.0, 1.0)
    u = np.where(band, 0.5, -0.5)
    v = 0.01 * np.sin(4 * np.pi * X + phase)
    p = 2.5
    E = p / (gamma - 1.0) + 0.5 * rho * (u ** 2 + v ** 2)
    return [a.astype(np.float32) for a in (rho, rho * u, rho * v, E)]


def rel_linf(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-30))


def rel_l1(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.sum(np.abs(a - b)) / max(float(np.sum(np.abs(b))), 1e-30))


def ulp_sensitivity(run, q):
    """Spread of a run under a one-ulp nudge of the first input variable.

    run(q) -> list of output arrays.  Returns per-variable (rel L-inf, rel L1)
    between run(q) and run(q with q[0] nudged up by one ulp): the rounding
    amplification of the scheme itself, used where a fixed bound would not
    reflect the conditioning of the problem (WAF at shocks, states next to
    zero-depth ghost cells).
    """
    a = run(q)
    q2 = [np.array(x, copy=True) for x in q]
    q2[0] = np.nextafter(q2[0], np.float32(np.inf)).astype(q2[0].dtype)
    b = run(q2)
    out = []
    for x, y in zip(a, b):
        m = np.isfinite(x) & np.isfinite(y)
        out.append((rel_linf(x[m], y[m]) if m.any() else 0.0, rel_l1(x[m], y[m]) if m.any() else 0.0))
    return out
