"""CPU oracle driver for the GPUSimulators time-step path -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline legs of
``bench.py`` may import this module.  It is the checker, never the product:
``finitevolumegpu_b200`` does not import it and has no CPU fallback.

``OracleSim`` restates the host side of the reference simulators on top of the
C restatement of the stage kernels in ``fv_oracle.cpp``:

* the time loop of ``BaseSimulator.simulate`` (GPUSimulators/Simulator.py:176-217):
  dt recomputed as ``computeDt()*cfl_scale`` whenever ``nt % 100 == 0``, the last
  step shortened to hit ``t_end`` (``float32(min(dt, t_end - t))``), t kept in
  double precision;
* ``BaseSimulator.step`` (Simulator.py:220-228) and each class's ``substep`` with
  its buffer swap and substep dt (e.g. GPUSimulators/KP07_dimsplit.py:108-126);
* the two state buffers of ``ArakawaA2D`` (GPUSimulators/Common.py:741-770):
  ``u0`` holds the upload, ``u1`` starts as zeros, including ghost cells, and the
  kernels never write ghost cells;
* the initial CFL fill computed on the host (e.g. KP07_dimsplit.py:102-106) and
  each class's ``computeDt`` factor: 1.0 for FORCE (GPUSimulators/FORCE.py:129),
  0.5**(order-1) for KP07 (GPUSimulators/KP07.py:138), 0.5 for the others
  (e.g. GPUSimulators/KP07_dimsplit.py:137).

EE2D_KP07_dimsplit swaps its buffers after every substep here, which is what
MPISimulator does (GPUSimulators/MPISimulator.py:326); the plain reference class
never swaps (GPUSimulators/EE2D_KP07_dimsplit.py:112-138), so its single-GPU
``simulate`` does not advance the state it returns.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

SCHEMES = {
    "LxF": 0,
    "FORCE": 1,
    "HLL": 2,
    "HLL2": 3,
    "WAF": 4,
    "KP07": 5,
    "KP07_dimsplit": 6,
    "EE2D_KP07_dimsplit": 7,
}
GHOST = {"LxF": 1, "FORCE": 1, "HLL": 1}
DIMSPLIT_HALF_DT = {"HLL2", "WAF", "KP07_dimsplit", "EE2D_KP07_dimsplit"}
DEFAULT_THETA = {"HLL2": 1.8, "KP07": 1.3, "KP07_dimsplit": 1.3, "EE2D_KP07_dimsplit": 1.3}

_lib = None


def build(force: bool = False) -> str:
    """Compile fv_oracle.cpp into _build/liboracle.so (g++, OpenMP, no FMA contraction)."""
    if force or not os.path.exists(LIB_PATH) or (
        os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "fv_oracle.cpp"))
    ):
        subprocess.check_call(["make", "-s", "-C", HERE, "oracle"])
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        for name, fp in (("fvo_substep_f32", ctypes.c_float), ("fvo_substep_f64", ctypes.c_double)):
            f = getattr(L, name)
            P = ctypes.POINTER(fp)
            f.argtypes = [
                ctypes.c_int, ctypes.c_int, ctypes.c_int,
                ctypes.POINTER(P), ctypes.POINTER(P),
                fp, fp, fp, fp, fp, fp,
                ctypes.c_int, ctypes.c_int, ctypes.c_int,
                P, ctypes.c_int,
                ctypes.c_int, fp,
            ]
            f.restype = ctypes.c_int
        _lib = L
    return _lib


def ghost_cells(scheme: str) -> int:
    return GHOST.get(scheme, 2)


def num_vars(scheme: str) -> int:
    return 4 if scheme == "EE2D_KP07_dimsplit" else 3


def substep_factor(scheme: str) -> float:
    """Factor each class's computeDt applies to min(cfl_data) (FORCE.py:129; 0.5 elsewhere but KP07)."""
    return 1.0 if scheme == "FORCE" else 0.5


def oracle_substep(scheme, u_in, u_out, nx, ny, dx, dy, dt, g, gamma, theta, step, order, bc, want_cfl=True,
                   nthreads=0, variant=0, beta=0.0):
    """Run one stage kernel of `scheme` on full (ny+2g, nx+2g) arrays; returns the CFL minimum or None."""
    dtype = u_in[0].dtype
    f64 = dtype == np.float64
    fp = ctypes.c_double if f64 else ctypes.c_float
    P = ctypes.POINTER(fp)
    nv = len(u_in)
    for a in list(u_in) + list(u_out):
        assert a.dtype == dtype and a.flags.c_contiguous
    ins = (P * nv)(*[a.ctypes.data_as(P) for a in u_in])
    outs = (P * nv)(*[a.ctypes.data_as(P) for a in u_out])
    cfl = fp(0)
    fn = lib().fvo_substep_f64 if f64 else lib().fvo_substep_f32
    rc = fn(SCHEMES[scheme], nx, ny, ins, outs, dx, dy, dt, g, gamma, theta, step, order, bc,
            ctypes.pointer(cfl) if want_cfl else None, nthreads, int(variant), beta)
    if rc != 0:
        raise RuntimeError("oracle substep failed")
    return dtype.type(cfl.value) if want_cfl else None


def flux_eval(kind, ql, qr, g, dx=1.0, dt=0.1):
    """FP32 oracle face fluxes for n face pairs (n x 3 arrays): kind 0 HLL, 1 HLLC, 2 Godunov centred."""
    L = lib()
    P = ctypes.POINTER(ctypes.c_float)
    ql = np.ascontiguousarray(ql, dtype=np.float32)
    qr = np.ascontiguousarray(qr, dtype=np.float32)
    out = np.empty_like(ql)
    L.fvo_flux_eval.argtypes = [ctypes.c_int, ctypes.c_int, P, P, ctypes.c_float, ctypes.c_float, ctypes.c_float, P]
    L.fvo_flux_eval(int(kind), ql.shape[0], ql.ctypes.data_as(P), qr.ctypes.data_as(P), g, dx, dt, out.ctypes.data_as(P))
    return out


def limiter_eval(limiter_id, r, beta=0.0):
    """FP32 oracle flux limiter (fv_oracle.cpp flux_limiter ids) on an array of ratios."""
    L = lib()
    P = ctypes.POINTER(ctypes.c_float)
    r = np.ascontiguousarray(r, dtype=np.float32)
    out = np.empty_like(r)
    L.fvo_limiter_eval.argtypes = [ctypes.c_int, ctypes.c_int, P, ctypes.c_float, P]
    L.fvo_limiter_eval(int(limiter_id), r.size, r.ctypes.data_as(P), beta, out.ctypes.data_as(P))
    return out


OP_NAMES = ("add", "sub", "mul", "div", "sqrt", "minmax")


def count_ops(scheme, u_in, nx, ny, dx, dy, dt, g, gamma, theta, step, order, bc):
    """Floating-point operations of one stage kernel of `scheme` as the reference
    formulates it, on full (ny+2g, nx+2g) float64 arrays: a dict over OP_NAMES."""
    L = lib()
    P = ctypes.POINTER(ctypes.c_double)
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in u_in]
    ins = (P * len(arrs))(*[a.ctypes.data_as(P) for a in arrs])
    counts = (ctypes.c_longlong * 6)()
    f = L.fvo_count_ops
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(P)] + [ctypes.c_double] * 6 + [
        ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)]
    f.restype = ctypes.c_int
    if f(SCHEMES[scheme], nx, ny, ins, dx, dy, dt, g, gamma, theta, step, order, bc, counts) != 0:
        raise RuntimeError("oracle operation count failed")
    return dict(zip(OP_NAMES, (int(c) for c in counts)))


def ops_per_cell_substep(scheme, order=2):
    """Algorithmic floating-point operations per interior cell and substep of
    `scheme`, averaged over the substeps of one step: each count is fitted as
    a*n^2 + b*n + c over n x n grids (n = 16, 32, 64) so that the ghost-line and
    extra-face work of a finite grid drops out, and `a` is returned.  Also
    returns 'flops' (+, -, *, /, sqrt, min, max counted 1 each) and 'mufu'
    (divisions and square roots, the special-function work).  The state is a
    smooth bump at rest (a lake with a Gaussian mound; Kelvin-Helmholtz bands
    for the Euler scheme) with reflective walls, so every face takes the
    subsonic branch of the HLL-type fluxes."""
    steps = (0, 1) if (scheme in DIMSPLIT_HALF_DT or (scheme == "KP07" and order == 2)) else (0,)
    theta = DEFAULT_THETA.get(scheme, 1.3)
    gc = ghost_cells(scheme)
    sizes = (16, 32, 64)
    per_size = []
    for n in sizes:
        m = n + 2 * gc
        y, x = np.mgrid[0:m, 0:m] + 0.5 - gc
        if scheme == "EE2D_KP07_dimsplit":
            band = (y >= 0.25 * n) & (y < 0.75 * n)
            rho = np.where(band, 2.0, 1.0)
            u = np.where(band, 0.5, -0.5)
            v = 0.01 * np.sin(4 * np.pi * x / n)
            q = [rho, rho * u, rho * v, 2.5 / 0.4 + 0.5 * rho * (u * u + v * v)]
            dx = 1.0 / n
            g, dt = 0.0, 0.1 * dx
        else:
            h = 1.0 + 0.3 * np.exp(-((x - 0.45 * n) ** 2 + (y - 0.55 * n) ** 2) / (2 * (n / 8.0) ** 2))
            q = [h, np.zeros_like(h), np.zeros_like(h)]
            dx = 1.0
            g, dt = 9.81, 0.05
        tot = dict.fromkeys(OP_NAMES, 0)
        for st in steps:
            c = count_ops(scheme, q, n, n, dx, dx, dt, g, 1.4, theta, st, order, 0x03030303)
            for k in OP_NAMES:
                tot[k] += c[k]
        per_size.append({k: tot[k] / len(steps) for k in OP_NAMES})
    A = np.array([[n * n, n, 1.0] for n in sizes])
    out = {}
    for k in OP_NAMES:
        a, _, _ = np.linalg.solve(A, np.array([c[k] for c in per_size], dtype=np.float64))
        out[k] = round(float(a), 6)
    out["flops"] = round(sum(out[k] for k in OP_NAMES), 6)
    out["mufu"] = round(out["div"] + out["sqrt"], 6)
    return out


class OracleSim:
    """A reference simulator's host semantics, on the CPU oracle."""

    def __init__(self, scheme, variables, nx, ny, dx, dy, g, gamma=1.4, theta=None, cfl_scale=0.9, order=2,
                 bc=0x03030303, dtype=np.float32, nthreads=0, variant=0, beta=0.0):
        self.scheme = scheme
        self.dtype = np.dtype(dtype)
        self.nx, self.ny = int(nx), int(ny)
        self.gc = ghost_cells(scheme)
        self.nv = num_vars(scheme)
        assert len(variables) == self.nv
        T = self.dtype.type
        self.dx, self.dy = T(dx), T(dy)
        self.g = T(g)
        self.gamma = T(gamma)
        self.theta = T(DEFAULT_THETA.get(scheme, 1.3) if theta is None else theta)
        self.cfl_scale = cfl_scale
        self.order = int(order)
        self.bc = int(bc)
        self.nthreads = nthreads
        self.variant = int(variant)  # HLL's flux or WAF's limiter (fv_oracle.cpp Params)
        self.beta = self.dtype.type(beta)
        if scheme in ("LxF", "FORCE", "HLL"):
            self.num_substeps = 1
        elif scheme == "KP07":
            self.num_substeps = self.order
        else:
            self.num_substeps = 2
        H, W = self.ny + 2 * self.gc, self.nx + 2 * self.gc
        self.u0 = []
        self.u1 = []
        for a in variables:
            a = np.asarray(a)
            full = np.zeros((H, W), dtype=self.dtype)
            if a.shape == (self.ny, self.nx):
                full[self.gc:self.gc + self.ny, self.gc:self.gc + self.nx] = a
            elif a.shape == (H, W):
                full[:] = a
            else:
                raise AssertionError("Wrong shape of data %s" % (a.shape,))
            self.u0.append(full)
            self.u1.append(np.zeros((H, W), dtype=self.dtype))
        # Host estimate of the initial CFL (e.g. GPUSimulators/KP07_dimsplit.py:102-106;
        # EE2D uses sqrt(gamma*rho): GPUSimulators/EE2D_KP07_dimsplit.py:106-108).
        h0, hu0, hv0 = (np.asarray(v).astype(self.dtype) for v in variables[:3])
        c2 = T(gamma) if scheme == "EE2D_KP07_dimsplit" else T(g)
        with np.errstate(divide="ignore", invalid="ignore"):
            dt_x = np.min(self.dx / (np.abs(hu0 / h0) + np.sqrt(c2 * h0)))
            dt_y = np.min(self.dy / (np.abs(hv0 / h0) + np.sqrt(c2 * h0)))
        self.cfl = T(min(dt_x, dt_y))
        self.t = 0.0
        self.nt = 0
        # Only EE2D_KP07_dimsplit.py:107 sets dt in its constructor; the other
        # classes have no dt until simulate() computes one.  Seeding it with the
        # initial CFL estimate everywhere keeps simulate() usable after manual
        # step() calls.
        self.dt = self.cfl

    # -- Simulator.py:176-217
    def simulate(self, t, dt=None):
        t_start = self.t
        t_end = t_start + t
        update_dt = dt is None
        if not update_dt:
            self.dt = dt
        T = self.dtype.type
        while self.t < t_end:
            if update_dt and (self.nt % 100 == 0):
                self.dt = T(self.computeDt() * T(self.cfl_scale))
            if self.dtype == np.float32:
                current_dt = np.float32(min(self.dt, t_end - self.t))
            else:
                current_dt = np.float64(min(self.dt, t_end - self.t))
            if current_dt <= 0.0:
                break
            self.step(current_dt)
        return self.t, self.nt

    # -- Simulator.py:220-228
    def step(self, dt):
        dt = self.dtype.type(dt)
        for i in range(self.num_substeps):
            self.substep(dt, i)
        self.t = float(self.t) + float(dt)
        self.nt += 1

    def substep(self, dt, step_number):
        T = self.dtype.type
        dt = T(dt)
        kdt = T(dt * T(0.5)) if self.scheme in DIMSPLIT_HALF_DT else dt
        cfl = self._launch(kdt, int(step_number))
        if self.scheme != "WAF":  # WAFKernel writes no CFL (GPUSimulators/cuda/SWE2D_WAF.cu:103-119)
            self.cfl = cfl
        self.u0, self.u1 = self.u1, self.u0

    def _launch(self, kdt, step_number):
        return oracle_substep(self.scheme, self.u0, self.u1, self.nx, self.ny, self.dx, self.dy, kdt, self.g,
                              self.gamma, self.theta, step_number, self.order, self.bc,
                              want_cfl=True, nthreads=self.nthreads, variant=self.variant, beta=self.beta)

    def computeDt(self):
        T = self.dtype.type
        if self.scheme == "KP07":
            return T(self.cfl * T(0.5 ** (self.order - 1)))
        return T(self.cfl * T(substep_factor(self.scheme)))

    def download(self, variables=None):
        g = self.gc
        idx = range(self.nv) if variables is None else variables
        return [self.u0[i][g:g + self.ny, g:g + self.nx].copy() for i in idx]

    def simTime(self):
        return self.t

    def simSteps(self):
        return self.nt
