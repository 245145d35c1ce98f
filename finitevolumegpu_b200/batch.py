"""Batched simulation: many grids of uneven sizes advanced together on one GPU.

The reference runs one simulator per class instance, one kernel launch per
substep.  A ``Batch`` holds many simulations of one scheme (any of the eight)
resident in HBM and advances all of them with one kernel launch per substep
(one per Runge-Kutta stage for KP07) over a device-resident tile work list;
the step sequence is replayed from CUDA graphs.  Each simulation
follows the reference's ``simulate(t_end)`` semantics on its own: its own CFL
time step recomputed every 100 of its steps, its last step shortened to hit
its t_end (GPUSimulators/Simulator.py:176-217).  Its result is therefore the
same as that of a plain simulator run alone.
"""

from __future__ import annotations

import ctypes
import threading

import numpy as np

from . import _lib
from .Simulator import BoundaryCondition

BATCH_SCHEMES = ("LxF", "FORCE", "HLL", "HLL2", "WAF", "KP07", "KP07_dimsplit", "EE2D_KP07_dimsplit")
GHOST = {"LxF": 1, "FORCE": 1, "HLL": 1}
DEFAULT_THETA = {"HLL2": 1.8}

def _L():
    return _lib.lib()


class Batch(object):
    """Simulations of one scheme advanced together by one batched kernel launch per substep.
    ``order`` is KP07's Runge-Kutta order (1 or 2, GPUSimulators/KP07.py:62),
    the same for every simulation of the batch."""

    def __init__(self, context, scheme, g=9.81, gamma=1.4, theta=None, cfl_scale=0.9, max_instances=1024,
                 tile=None, variant=0, variant_beta=0.0, order=2):
        if scheme not in BATCH_SCHEMES:
            raise ValueError("batched kernels exist for %s" % (BATCH_SCHEMES,))
        self.context = context
        self.scheme = scheme
        self.nv = 4 if scheme == "EE2D_KP07_dimsplit" else 3
        self.gc = GHOST.get(scheme, 2)
        if tile is None:
            tile = -1
            tuner = getattr(context, "autotuner", None)
            if tuner is not None and hasattr(tuner, "get_batch_tile"):
                tile = tuner.get_batch_tile(scheme, context.device_name)
        theta = DEFAULT_THETA.get(scheme, 1.3) if theta is None else theta
        # variant: HLL's flux or WAF's limiter id (HLL.FLUXES, WAF.LIMITERS)
        _lib.require(order in (1, 2), "order must be 1 or 2, got %r" % (order,))
        p = _lib.fv_params(float(g), float(gamma), float(theta), float(cfl_scale), int(order), int(tile), int(variant),
                           float(variant_beta))
        h = ctypes.c_void_p()
        _lib.check(_L().fv_batch_create(context.handle, _lib.SCHEME_IDS[scheme], ctypes.byref(p), int(max_instances),
                                        ctypes.byref(h)))
        self._h = h
        self.shapes = {}
        # slot -> (ny, nx); guarded so that a slot released by one thread and
        # taken again by another's admission keeps the new simulation's shape
        self._shapes_lock = threading.Lock()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib._lib is not None:
            _L().fv_batch_destroy(h)
            self._h = None

    def add(self, variables, nx, ny, dx, dy, t_end, boundary_conditions=None):
        """Admit one simulation; returns its slot.  Raises MemoryError when the
        GPU has no room and AssertionError for the wrong number or shape of arrays."""
        bc = (boundary_conditions or BoundaryCondition()).asCodedInt()
        _lib.require(len(variables) == self.nv,
                     "%s takes %d conserved variables, got %d" % (self.scheme, self.nv, len(variables)))
        arrays = [np.ascontiguousarray(a, dtype=np.float32) for a in variables]
        rows, cols = arrays[0].shape
        for a in arrays:
            _lib.require(a.shape in ((ny, nx), (ny + 2 * self.gc, nx + 2 * self.gc)) and a.shape == (rows, cols),
                         "Wrong shape of data %s for a %d x %d grid" % (a.shape, nx, ny))
        ptrs = (_lib._FP * self.nv)(*[a.ctypes.data_as(_lib._FP) for a in arrays])
        slot = ctypes.c_int()
        _lib.check(_L().fv_batch_add(self._h, int(nx), int(ny), float(dx), float(dy), int(bc), ptrs, rows, cols,
                                     float(t_end), ctypes.byref(slot)))
        with self._shapes_lock:
            self.shapes[slot.value] = (int(ny), int(nx))
        return slot.value

    def remove(self, slot):
        # forget the shape first: once the library releases the slot, another
        # thread's admission may receive the same slot number
        with self._shapes_lock:
            self.shapes.pop(slot, None)
        _lib.check(_L().fv_batch_remove(self._h, int(slot)))

    def run(self, n_steps):
        """Queue n_steps steps for every simulation (asynchronous)."""
        _lib.check(_L().fv_batch_run(self._h, int(n_steps)))

    def sync(self):
        _lib.check(_L().fv_batch_sync(self._h))

    def status(self, slot):
        t, nt, dt, done = ctypes.c_double(), ctypes.c_longlong(), ctypes.c_float(), ctypes.c_int()
        _lib.check(_L().fv_batch_status(self._h, int(slot), ctypes.byref(t), ctypes.byref(nt), ctypes.byref(dt),
                                        ctypes.byref(done)))
        # done: reached t_end or failed; failed: a step left a non-finite value or
        # a non-positive depth (density), or t/dt is not a number
        return {"t": t.value, "nt": nt.value, "dt": dt.value, "done": bool(done.value), "failed": done.value == 2}

    def download(self, slot, scratch=None):
        """The simulation's state as (ny, nx) float32 arrays.  With `scratch` (a
        float32 array of at least nv * ny * nx elements, e.g. reused by a
        thread) the arrays are views into it: no fresh host memory to fault in,
        valid until the scratch is reused."""
        with self._shapes_lock:
            ny, nx = self.shapes[slot]
        out = []
        for v in range(self.nv):
            if scratch is None:
                a = np.empty((ny, nx), dtype=np.float32)
            else:
                a = scratch[v * ny * nx:(v + 1) * ny * nx].reshape(ny, nx)
            _lib.check(_L().fv_batch_download(self._h, int(slot), v, a.ctypes.data_as(_lib._FP), nx))
            out.append(a)
        return out

    def download_many(self, slots, threads=4):
        """download() of several simulations, copied out on `threads` host
        threads at once (their device-to-host copies and the host copies out of
        pinned staging overlap).  Returns the states in the order of `slots`."""
        slots = list(slots)
        if threads <= 1 or len(slots) < 2:
            return [self.download(s) for s in slots]
        import concurrent.futures

        with concurrent.futures.ThreadPoolExecutor(int(threads), thread_name_prefix="fvgpu-download") as pool:
            return list(pool.map(self.download, slots))

    def info(self):
        b, a, w, ms = ctypes.c_size_t(), ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        _lib.check(_L().fv_batch_info(self._h, ctypes.byref(b), ctypes.byref(a), ctypes.byref(w), ctypes.byref(ms)))
        tw, th, nt, gr = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _lib.check(_L().fv_batch_tile(self._h, ctypes.byref(tw), ctypes.byref(th), ctypes.byref(nt),
                                      ctypes.byref(gr)))
        return {"device_bytes": b.value, "active": a.value, "work_items": w.value, "last_run_ms": ms.value,
                "tile_w": tw.value, "tile_h": th.value, "threads": nt.value, "grid": gr.value}

    def run_to_completion(self, chunk=16):
        """Advance until every simulation reached its t_end; returns the steps run."""
        steps = 0
        while True:
            self.sync()
            with self._shapes_lock:
                slots = list(self.shapes)
            if all(self.status(s)["done"] for s in slots):
                return steps
            self.run(chunk)
            steps += chunk
