"""Initial conditions of the reference's test cases: the counterpart of
GPUSimulators/helpers/InitialConditions.py.

Each generator returns what the reference's returns: ``bump`` the shallow-water
fields and cell sizes, the Euler generators a dictionary of simulator
arguments (``rho, rho_u, rho_v, E, nx, ny, dx, dy, g, gamma,
boundary_conditions``) ready for ``EE2D_KP07_dimsplit(context, **arguments)``
or for a served request (``request_from_arguments``).  ``grid`` may be a
``StripeGrid`` (row stripes): the fields are then this rank's stripe of the
global case.  The arithmetic follows the reference's NumPy code (float32 fields,
float64 coordinates where it uses them), so the arrays are the same.

Two reference behaviours are kept as they are: ``getExtent`` with a grid
shortens the last y coordinate by half a *x* cell (``y1 = ... - 0.5*dx``,
InitialConditions.py:44), and ``genKelvinHelmholtz`` always uses gamma = 1.4
whatever gamma it is given (InitialConditions.py:255).
"""

from __future__ import annotations

import numpy as np

from .Simulator import BoundaryCondition


def getExtent(width, height, nx, ny, grid, index=None):
    """[x0, x1, y0, y1, dx, dy]: centres of the first and last cells of this
    rank's part of a width x height domain, and the cell size
    (InitialConditions.py:28-54)."""
    if grid is None:
        dx, dy = width / nx, height / ny
        return [0.5 * dx, width - 0.5 * dx, 0.5 * dy, height - 0.5 * dy, dx, dy]
    gx, gy = grid.grid[0], grid.grid[1]
    i, j = grid.getCoordinate(index) if index is not None else grid.getCoordinate()
    dx = (width / gx) / nx
    dy = (height / gy) / ny
    return [width * i / gx + 0.5 * dx, width * (i + 1) / gx - 0.5 * dx,
            height * j / gy + 0.5 * dy, height * (j + 1) / gy - 0.5 * dx, dx, dy]


def downsample(highres_solution, x_factor, y_factor=None):
    """Block means of x_factor x y_factor cells (InitialConditions.py:57-74)."""
    y_factor = x_factor if y_factor is None else y_factor
    a = highres_solution
    assert a.shape[1] % x_factor == 0 and a.shape[0] % y_factor == 0
    if x_factor * y_factor == 1:
        return a
    if a.ndim == 1:
        a = a.reshape((1, a.size))
    ny, nx = int(a.shape[0] / y_factor), int(a.shape[1] / x_factor)
    return a.reshape([ny, int(y_factor), nx, int(x_factor)]).mean(3).mean(1)


def bump(nx, ny, width, height, bump_size=None, ref_nx=None, ref_ny=None, x_center=0.5, y_center=0.5,
         h_ref=0.5, h_amp=0.1, u_ref=0.0, u_amp=0.1, v_ref=0.0, v_amp=0.1):
    """Raised-cosine bump in h, u and v, sampled on a ref_nx x ref_ny grid and
    averaged down to nx x ny (InitialConditions.py:79-132).  Returns
    (h, hu, hv, dx, dy)."""
    ref_nx = nx if ref_nx is None else ref_nx
    ref_ny = ny if ref_ny is None else ref_ny
    assert ref_nx >= nx and ref_ny >= ny
    bump_size = width / 5.0 if bump_size is None else bump_size
    rdx, rdy = width / float(ref_nx), height / float(ref_ny)
    xc, yc = rdx * ref_nx * x_center, rdy * ref_ny * y_center
    x = rdx * (np.arange(0, ref_nx, dtype=np.float32) + 0.5) - xc
    y = rdy * (np.arange(0, ref_ny, dtype=np.float32) + 0.5) - yc
    xv, yv = np.meshgrid(x, y, sparse=False, indexing="xy")
    r = np.sqrt(xv ** 2 + yv ** 2)
    fx, fy = ref_nx / nx, ref_ny / ny

    def raised(ref, amp):  # ref + amp/2 (1 + cos(pi r / size)) inside the bump, same operation order
        return ref + amp * 0.5 * (1.0 + np.cos(np.pi * r / bump_size)) * (r < bump_size)

    h = downsample(raised(h_ref, h_amp), fx, fy)
    hu = downsample(raised(u_ref, u_amp), fx, fy) * h
    hv = downsample(raised(v_ref, v_amp), fx, fy) * h
    return h, hu, hv, width / nx, height / ny


def _arguments(rho, u, v, p, nx, ny, dx, dy, g, gamma, bc):
    E = 0.5 * rho * (u ** 2 + v ** 2) + p / (gamma - 1.0)
    return {"rho": rho, "rho_u": rho * u, "rho_v": rho * v, "E": E, "nx": nx, "ny": ny, "dx": dx, "dy": dy,
            "g": g, "gamma": gamma, "boundary_conditions": bc}


def _bc(north, south, east, west):
    return BoundaryCondition({"north": north, "south": south, "east": east, "west": west})


def genShockBubble(nx, ny, gamma, grid=None):
    """A Mach ~1.2 shock entering from the left onto a light bubble on a 4 x 1
    channel with reflective top and bottom and periodic ends
    (InitialConditions.py:135-191)."""
    T = BoundaryCondition.Type
    width, height, g = 4.0, 1.0, 0.0
    x0, x1, y0, y1, dx, dy = getExtent(width, height, nx, ny, grid)
    xv, yv = np.meshgrid(np.linspace(x0, x1, nx, dtype=np.float32), np.linspace(y0, y1, ny, dtype=np.float32),
                         sparse=False, indexing="xy")
    rho = np.ones((ny, nx), dtype=np.float32)
    u = np.zeros((ny, nx), dtype=np.float32)
    v = np.zeros((ny, nx), dtype=np.float32)
    p = np.ones((ny, nx), dtype=np.float32)
    rho = np.where(np.sqrt((xv - 0.5) ** 2 + (yv - 0.5) ** 2) <= 0.25, 0.1, rho)
    left = xv < 0.1
    rho = np.where(left, 3.81250, rho)
    u = np.where(left, 2.57669, u)
    p = np.where(left, 10.0, p)
    return _arguments(rho, u, v, p, nx, ny, dx, dy, g, gamma, _bc(T.Reflective, T.Reflective, T.Periodic, T.Periodic))


def _smooth_random(n_points, n_controls, rng):
    """n_points values of a random curve through n_controls uniform(-0.5, 0.5)
    control points (nearest/linear/quadratic/cubic interpolation by count)."""
    n = max(1, min(n_controls, n_points))
    if n == n_points:
        return rng.random(n_points) - 0.5
    from scipy.interpolate import interp1d

    kind = {1: "nearest", 2: "linear", 3: "quadratic"}.get(n, "cubic")
    f = interp1d(np.linspace(0.0, 1.0, n), rng.random(n) - 0.5, kind=kind)
    return f(np.linspace(0.0, 1.0, n_points))


def genKelvinHelmholtz(nx, ny, gamma, roughness=0.125, grid=None, index=None, rng=None):
    """Two counter-flowing layers (rho 2, u -0.5 in the middle band; rho 1,
    u 0.5 outside) with randomly perturbed interfaces whose wiggliness is set
    by `roughness` in (0, 1], on a 2 x 1 periodic box
    (InitialConditions.py:198-301).  `rng` (default: NumPy's global generator,
    as the reference) draws the interfaces."""
    T = BoundaryCondition.Type
    rng = np.random if rng is None else rng
    width, height, g = 2.0, 1.0, 0.0
    gamma = 1.4
    x0, x1, y0, y1, _, dy = getExtent(1.0, 1.0, nx, ny, grid, index)
    _, y = np.meshgrid(np.linspace(x0, x1, nx), np.linspace(y0, y1, ny))
    n = max(1, min(nx, int(nx * roughness)))
    zone = np.zeros((ny, nx), dtype=np.int32)
    zone = np.where(y > 0.25 + _smooth_random(nx, n, rng) * dy, zone, 1)
    zone = np.where(y < 0.75 + _smooth_random(nx, n, rng) * dy, zone, 1)
    rho = np.empty((ny, nx), dtype=np.float32)
    u = np.empty((ny, nx), dtype=np.float32)
    v = np.zeros((ny, nx), dtype=np.float32)
    p = 2.5 * np.ones((ny, nx), dtype=np.float32)
    rho = np.where(zone == 0, 1.0, rho)
    u = np.where(zone == 0, 0.5, u)
    rho = np.where(zone == 1, 2.0, rho)
    u = np.where(zone == 1, -0.5, u)
    _, _, _, _, dx, dy = getExtent(width, height, nx, ny, grid, index)
    return _arguments(rho, u, v, p, nx, ny, dx, dy, g, gamma, _bc(T.Periodic, T.Periodic, T.Periodic, T.Periodic))


def genRayleighTaylor(nx, ny, gamma, version=0, grid=None):
    """Heavy fluid (rho 2) above light fluid (rho 1) under gravity g = 0.1 in
    hydrostatic balance, on a 0.5 x 1.5 box with reflective walls; version 0
    perturbs the interface, version 1 the vertical velocity
    (InitialConditions.py:304-355)."""
    T = BoundaryCondition.Type
    width, height, g = 0.5, 1.5, 0.1
    x0, x1, y0, y1, dx, dy = getExtent(width, height, nx, ny, grid)
    x = np.linspace(x0, x1, nx, dtype=np.float32) - width * 0.5
    y = np.linspace(y0, y1, ny, dtype=np.float32) - height * 0.5
    xv, yv = np.meshgrid(x, y, sparse=False, indexing="xy")
    rho = np.zeros((ny, nx), dtype=np.float32)
    u = np.zeros((ny, nx), dtype=np.float32)
    v = np.zeros((ny, nx), dtype=np.float32)
    if version == 0:
        threshold = 0.01 * np.cos(2 * np.pi * np.abs(x) / 0.5)
        rho = np.where(yv <= threshold, 1.0, rho)
        rho = np.where(yv > threshold, 2.0, rho)
    elif version == 1:
        rho = np.where(yv <= 0.0, 1.0, rho)
        rho = np.where(yv > 0.0, 2.0, rho)
        v = 0.01 * (1.0 + np.cos(2 * np.pi * xv / 0.5)) / 4
    else:
        raise AssertionError("Invalid version")
    p = 2.5 - rho * g * yv
    return _arguments(rho, u, v, p, nx, ny, dx, dy, g, gamma,
                      _bc(T.Reflective, T.Reflective, T.Reflective, T.Reflective))


def request_from_arguments(rid, arguments, t_end, arrival=0.0, scheme="EE2D_KP07_dimsplit"):
    """A served request (``server.Request``) for the case `arguments` of an
    Euler generator above, carrying its g and gamma."""
    from .server import Request

    a = arguments
    fields = [np.ascontiguousarray(a[k], dtype=np.float32) for k in ("rho", "rho_u", "rho_v", "E")]
    return Request(rid, scheme, fields, int(a["nx"]), int(a["ny"]), float(a["dx"]), float(a["dy"]), float(t_end),
                   arrival=arrival, boundary_conditions=a["boundary_conditions"], g=float(a["g"]),
                   gamma=float(a["gamma"]))
