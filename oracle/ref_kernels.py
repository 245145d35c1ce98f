"""The reference's own CUDA kernels as a GPU parity check -- TEST INFRASTRUCTURE ONLY.

Drives oracle/_ref/libref_<scheme>.so (built by ``make -C oracle ref`` from the
unmodified reference kernel sources, see ref_launch.cu) with the reference's
host semantics, which ``OracleSim`` restates: two dense (ny+2g) x (nx+2g)
float32 buffers per variable with the reference's row pitch, the buffer swap
after each substep, min(cfl_data) over the kernel's per-block CFL output
(gpuarray.min, e.g. GPUSimulators/KP07_dimsplit.py:136) and the dt schedule of
Simulator.simulate.  Only tests/, __graft_entry__.smoke() and bench.py's
baseline legs may use it.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from .oracle import OracleSim

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
_libs = {}


# Block shapes built besides each kernel's default (oracle/Makefile REF_BLOCKS).
BLOCKS = ((32, 8), (32, 16), (32, 4), (8, 8))


# Builds of the default block besides the reference's own compile options:
# "nofma" is fast math without FMA contraction (oracle/Makefile REF_NOFMA_LIBS).
BUILDS = ("nofma",)


def ref_lib_path(scheme: str, block=None, build=None) -> str:
    if build is not None:
        assert block is None and build in BUILDS, (block, build)
        return os.path.join(REF_DIR, "libref_%s_%s.so" % (scheme, build))
    if block is None:
        return os.path.join(REF_DIR, "libref_%s.so" % scheme)
    return os.path.join(REF_DIR, "libref_%s_%dx%d.so" % (scheme, block[0], block[1]))


def available(scheme: str = "KP07_dimsplit", block=None, build=None) -> bool:
    return os.path.exists(ref_lib_path(scheme, block, build))


def ref_lib(scheme: str, block=None, build=None):
    key = (scheme, block, build)
    if key not in _libs:
        L = ctypes.CDLL(ref_lib_path(scheme, block, build))
        P = ctypes.c_void_p
        L.ref_last_error.restype = ctypes.c_char_p
        L.ref_malloc.argtypes = [ctypes.POINTER(P), ctypes.c_size_t]
        L.ref_free.argtypes = [P]
        L.ref_memset.argtypes = [P, ctypes.c_size_t]
        L.ref_h2d.argtypes = [P, P, ctypes.c_size_t]
        L.ref_d2h.argtypes = [P, P, ctypes.c_size_t]
        L.ref_event_create.argtypes = [ctypes.POINTER(P)]
        L.ref_event_record.argtypes = [P]
        L.ref_event_elapsed.argtypes = [P, P, ctypes.POINTER(ctypes.c_float)]
        L.ref_event_destroy.argtypes = [P]
        FP = ctypes.POINTER(ctypes.c_float)
        L.ref_substep.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_float] * 6 + [ctypes.c_int] * 3 + [
            ctypes.POINTER(FP), ctypes.POINTER(FP), ctypes.c_int, FP]
        _libs[key] = L
    return _libs[key]


def _ck(L, rc):
    if rc != 0:
        raise RuntimeError("reference harness: " + L.ref_last_error().decode())


class RefKernelSim(OracleSim):
    """OracleSim's host loop with the reference kernels doing the substeps;
    `block` = (w, h) picks one of the other block shapes (BLOCKS), `build`
    one of the other builds of the default block (BUILDS)."""

    def __init__(self, scheme, variables, nx, ny, dx, dy, g, block=None, build=None, **kw):
        kw["dtype"] = np.float32
        super().__init__(scheme, variables, nx, ny, dx, dy, g, **kw)
        self.L = ref_lib(scheme, block, build)
        L = self.L
        self.bw, self.bh = L.ref_block_width(), L.ref_block_height()
        H, W = self.u0[0].shape
        self.nbytes = H * W * 4
        self.pitch = W * 4
        self.d0, self.d1 = [], []
        for host in self.u0:
            p = ctypes.c_void_p()
            _ck(L, L.ref_malloc(ctypes.byref(p), self.nbytes))
            _ck(L, L.ref_h2d(p, host.ctypes.data, self.nbytes))
            self.d0.append(p)
            q = ctypes.c_void_p()
            _ck(L, L.ref_malloc(ctypes.byref(q), self.nbytes))
            _ck(L, L.ref_memset(q, self.nbytes))
            self.d1.append(q)
        gx = (self.nx + self.bw - 1) // self.bw
        gy = (self.ny + self.bh - 1) // self.bh
        self.ncfl = gx * gy
        c = ctypes.c_void_p()
        _ck(L, L.ref_malloc(ctypes.byref(c), self.ncfl * 4))
        fill = np.full(self.ncfl, self.cfl, dtype=np.float32)  # cfl_data.fill(dt)
        _ck(L, L.ref_h2d(c, fill.ctypes.data, self.ncfl * 4))
        self.dcfl = c

    def _launch(self, kdt, step_number):
        FP = ctypes.POINTER(ctypes.c_float)
        ins = (FP * self.nv)(*[ctypes.cast(p, FP) for p in self.d0])
        outs = (FP * self.nv)(*[ctypes.cast(p, FP) for p in self.d1])
        L = self.L
        _ck(L, L.ref_substep(self.nx, self.ny, float(self.dx), float(self.dy), float(kdt), float(self.g),
                             float(self.gamma), float(self.theta), step_number, self.order, self.bc, ins, outs,
                             self.pitch, ctypes.cast(self.dcfl, FP)))
        self.d0, self.d1 = self.d1, self.d0
        host = np.empty(self.ncfl, dtype=np.float32)
        _ck(L, L.ref_d2h(host.ctypes.data, self.dcfl, self.ncfl * 4))
        return np.float32(np.fmin.reduce(host))  # gpuarray.min ignores NaN like fmin

    def substep(self, dt, step_number):
        T = np.float32
        kdt = T(T(dt) * T(0.5)) if self.scheme in ("HLL2", "WAF", "KP07_dimsplit", "EE2D_KP07_dimsplit") else T(dt)
        cfl = self._launch(kdt, int(step_number))
        if self.scheme != "WAF":
            self.cfl = cfl

    def time_steps(self, n, dt):
        """Device time (ms per step) of n steps of fixed dt: the reference's
        kernel launches and buffer swaps only (no CFL read-back)."""
        L = self.L
        P = ctypes.c_void_p
        e0, e1 = P(), P()
        _ck(L, L.ref_event_create(ctypes.byref(e0)))
        _ck(L, L.ref_event_create(ctypes.byref(e1)))
        FP = ctypes.POINTER(ctypes.c_float)
        T = np.float32
        half = self.scheme in ("HLL2", "WAF", "KP07_dimsplit", "EE2D_KP07_dimsplit")
        kdt = T(T(dt) * T(0.5)) if half else T(dt)
        _ck(L, L.ref_event_record(e0))
        for _ in range(n):
            for i in range(self.num_substeps):
                ins = (FP * self.nv)(*[ctypes.cast(p, FP) for p in self.d0])
                outs = (FP * self.nv)(*[ctypes.cast(p, FP) for p in self.d1])
                _ck(L, L.ref_substep(self.nx, self.ny, float(self.dx), float(self.dy), float(kdt), float(self.g),
                                     float(self.gamma), float(self.theta), i, self.order, self.bc, ins, outs,
                                     self.pitch, ctypes.cast(self.dcfl, FP)))
                self.d0, self.d1 = self.d1, self.d0
        _ck(L, L.ref_event_record(e1))
        ms = ctypes.c_float()
        _ck(L, L.ref_event_elapsed(e0, e1, ctypes.byref(ms)))
        L.ref_event_destroy(e0)
        L.ref_event_destroy(e1)
        return ms.value / n

    def download(self, variables=None):
        g = self.gc
        idx = range(self.nv) if variables is None else variables
        out = []
        for i in idx:
            full = np.empty(self.u0[0].shape, dtype=np.float32)
            _ck(self.L, self.L.ref_d2h(full.ctypes.data, self.d0[i], self.nbytes))
            out.append(full[g:g + self.ny, g:g + self.nx].copy())
        return out

    def download_full(self):
        out = []
        for i in range(self.nv):
            full = np.empty(self.u0[0].shape, dtype=np.float32)
            _ck(self.L, self.L.ref_d2h(full.ctypes.data, self.d0[i], self.nbytes))
            out.append(full)
        return out

    def close(self):
        for p in self.d0 + self.d1 + ([self.dcfl] if self.dcfl is not None else []):
            self.L.ref_free(p)
        self.d0, self.d1, self.dcfl = [], [], None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
