"""Simulator base class and boundary conditions: the counterpart of
GPUSimulators/Simulator.py.

``BaseSimulator`` keeps the reference's public API (simulate, step, substep,
computeDt, download, synchronize, simTime, simSteps, getExtent, check,
get/setBoundaryConditions).  The state, the time t (FP64), the step count and
the CFL time step live on the GPU and are advanced there; the methods call the
C ABI of libfvgpu.so.
"""

from __future__ import annotations

import ctypes
import logging
from enum import IntEnum

import numpy as np

from . import _lib


class BoundaryCondition(object):
    """Boundary conditions of the four global boundaries (GPUSimulators/Simulator.py:38-100)."""

    class Type(IntEnum):
        """Must match the device codec (GPUSimulators/cuda/common.h:109-114)."""

        Dirichlet = 0
        Neumann = 1
        Periodic = 2
        Reflective = 3

    def __init__(self, types=None):
        if types is None:
            types = {
                "north": BoundaryCondition.Type.Reflective,
                "south": BoundaryCondition.Type.Reflective,
                "east": BoundaryCondition.Type.Reflective,
                "west": BoundaryCondition.Type.Reflective,
            }
        self.north = types["north"]
        self.south = types["south"]
        self.east = types["east"]
        self.west = types["west"]
        if BoundaryCondition.Type.Neumann in (self.north, self.south, self.east, self.west):
            raise NotImplementedError("Neumann boundary condition not supported")

    def __str__(self):
        return "[north={:s}, south={:s}, east={:s}, west={:s}]".format(
            str(self.north), str(self.south), str(self.east), str(self.west)
        )

    def asCodedInt(self):
        """Pack the four types into one int: N<<24 | S<<16 | E<<8 | W (Simulator.py:78-92)."""
        bc = 0
        bc = bc | (int(self.north) & 0x0000000F) << 24
        bc = bc | (int(self.south) & 0x0000000F) << 16
        bc = bc | (int(self.east) & 0x0000000F) << 8
        bc = bc | (int(self.west) & 0x0000000F) << 0
        return np.int32(bc)

    @staticmethod
    def getTypes(bc):
        bc = int(bc)
        return {
            "north": BoundaryCondition.Type((bc >> 24) & 0x0000000F),
            "south": BoundaryCondition.Type((bc >> 16) & 0x0000000F),
            "east": BoundaryCondition.Type((bc >> 8) & 0x0000000F),
            "west": BoundaryCondition.Type((bc >> 0) & 0x0000000F),
        }


def stepOrderToCodedInt(step, order):
    """Pack step and order into one int: step<<16 | order (Simulator.py:280-287)."""
    return np.int32((step << 16) | (order & 0x0000FFFF))


class _VariableView(object):
    """One conserved variable of a state buffer, with the download() of
    CudaArray2D (GPUSimulators/Common.py:543-584)."""

    def __init__(self, sim, var):
        self._sim = sim
        self._var = var
        self.nx, self.ny = int(sim.nx), int(sim.ny)
        self.x_halo = self.y_halo = sim._gc

    def download(self, stream=None, cpu_data=None, asynch=False, extent=None):
        """The interior, or with extent = [x, y, nx, ny] that region of the array
        including its ghost cells (GPUSimulators/Common.py:543-584)."""
        if extent is None:
            return self._sim._download_var(self._var, cpu_data)
        x, y, nx, ny = (int(v) for v in extent)
        if cpu_data is None:
            cpu_data = np.empty((ny, nx), dtype=np.float32)
        _lib.require(cpu_data.shape == (ny, nx), "cpu_data shape does not match the extent")
        _lib.require(cpu_data.dtype == np.float32 and cpu_data.flags.c_contiguous, "cpu_data must be C-ordered float32")
        _lib.check(_lib.lib().fv_sim_download_region(self._sim._handle, self._var, x, y, nx, ny,
                                                     cpu_data.ctypes.data_as(_lib._FP), nx))
        return cpu_data

    def upload(self, stream, cpu_data, extent=None):
        """The interior (cpu_data of shape (ny, nx)), or with extent = [x, y, nx, ny]
        that region of the array including its ghost cells (Common.py:587-616)."""
        if extent is None:
            return self._sim.upload(self._var, cpu_data)
        x, y, nx, ny = (int(v) for v in extent)
        data = np.ascontiguousarray(cpu_data, dtype=np.float32)
        _lib.require(data.shape == (ny, nx), "cpu_data shape does not match the extent")
        _lib.check(_lib.lib().fv_sim_upload_region(self._sim._handle, self._var, x, y, nx, ny,
                                                   data.ctypes.data_as(_lib._FP), nx))


class _StateView(object):
    """u0: the current state as ArakawaA2D-like indexable variables."""

    def __init__(self, sim):
        self._sim = sim

    def __getitem__(self, key):
        assert type(key) == int, "Indexing is int based"
        if key >= self._sim._nv or key < 0:
            raise IndexError("Out of bounds")
        return _VariableView(self._sim, key)

    def download(self, stream=None, variables=None):
        return self._sim.download(variables)

    def check(self):
        self._sim.check()


class _DeviceRows(object):
    """A device range of FP32 values seen through the CUDA array interface."""

    def __init__(self, address, count):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": "<f4", "data": (int(address), False),
                                         "version": 3, "strides": None}


class BaseSimulator(object):
    """Common state and time loop of all schemes (GPUSimulators/Simulator.py:109-266)."""

    _scheme = None  # name of the scheme, set by subclasses
    _gc = 2         # ghost cells of the scheme

    def __init__(self, context, nx, ny, dx, dy, boundary_conditions, cfl_scale, num_substeps, block_width,
                 block_height):
        self.logger = logging.getLogger(__name__ + "." + self.__class__.__name__)
        self.context = context
        self.nx = np.int32(nx)
        self.ny = np.int32(ny)
        self.dx = np.float32(dx)
        self.dy = np.float32(dy)
        self.boundary_conditions = boundary_conditions.asCodedInt()
        self.cfl_scale = cfl_scale
        self.num_substeps = num_substeps
        # The reference sizes its thread blocks from these; here they are kept
        # for API compatibility and the tile shape comes from the autotuner.
        self.block_size = (block_width, block_height, 1)
        self.grid_size = (int(np.ceil(self.nx / float(block_width))), int(np.ceil(self.ny / float(block_height))))
        self.stream = None  # the simulation's CUDA stream is owned by libfvgpu
        self.internal_stream = None
        self._handle = None
        self._nv = 3
        self._state = None  # (buffer pointers, pitch) for halo views, queried on first use
        self._cur = None    # buffer holding the current state, tracked across substeps; None = ask the device

    # -- construction helper used by the scheme classes
    def _create(self, variables, g=9.81, gamma=1.4, theta=1.3, order=2, variant=0, variant_beta=0.0):
        scheme = _lib.SCHEME_IDS[self._scheme]
        nx, ny, gc = int(self.nx), int(self.ny), self._gc
        arrays = []
        for a in variables:
            a = np.asarray(a)
            _lib.require(a.shape == (ny + 2 * gc, nx + 2 * gc) or a.shape == (ny, nx), "Wrong shape of data %s vs %s / %s" % (
                str(a.shape), str((ny, nx)), str((ny + 2 * gc, nx + 2 * gc))))
            _lib.require(a.itemsize == 4, "Wrong size of data type")
            _lib.require(not np.isfortran(a) or a.ndim < 2 or a.shape[0] == 1, "Wrong datatype (Fortran, expected C)")
            arrays.append(np.ascontiguousarray(a, dtype=np.float32))
        shapes = {a.shape for a in arrays}
        _lib.require(len(shapes) == 1, "all variables must have the same shape")
        rows, cols = arrays[0].shape
        tile = -1
        if getattr(self.context, "autotuner", None) is not None:
            tile = self.context.autotuner.get_tile(self._scheme, nx, ny, self.context.device_name)
        p = _lib.fv_params(float(g), float(gamma), float(theta), float(self.cfl_scale), int(order), int(tile),
                           int(variant), float(variant_beta))
        ptrs = (_lib._FP * len(arrays))(*[a.ctypes.data_as(_lib._FP) for a in arrays])
        h = ctypes.c_void_p()
        _lib.check(_lib.lib().fv_sim_create(self.context.handle, scheme, nx, ny, float(self.dx), float(self.dy),
                                            ctypes.byref(p), int(self.boundary_conditions), ptrs, rows, cols,
                                            ctypes.byref(h)))
        self._handle = h
        self._nv = len(arrays)

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and _lib._lib is not None:
            _lib.lib().fv_sim_destroy(h)
            self._handle = None

    def __str__(self):
        return "{:s} [{:d}x{:d}]".format(self.__class__.__name__, int(self.nx), int(self.ny))

    # -- time stepping (Simulator.py:176-228)
    def simulate(self, t, dt=None):
        """Advance by t seconds; dt=None recomputes dt = computeDt()*cfl_scale every 100 steps."""
        self._cur = None
        if dt is None:
            _lib.check(_lib.lib().fv_sim_simulate(self._handle, float(t), 0.0, 0))
        else:
            _lib.check(_lib.lib().fv_sim_simulate(self._handle, float(t), float(np.float32(dt)), 1))

    def step(self, dt):
        _lib.check(_lib.lib().fv_sim_step(self._handle, float(np.float32(dt))))
        if self._cur is not None:
            self._cur ^= self.num_substeps & 1

    def substep(self, dt, step_number):
        _lib.check(_lib.lib().fv_sim_substep(self._handle, float(np.float32(dt)), int(step_number)))
        if self._cur is not None:
            self._cur ^= 1  # every stage launch writes the other buffer

    def substep_rows(self, dt, step_number, row0, nrows, last=False):
        """One band of tile rows of a substep (fv_sim_substep_rows): bands that
        cover every tile row once, launched in order, equal substep().  `last`
        marks the substep's final band, after which the current state is the
        buffer the substep wrote."""
        _lib.check(_lib.lib().fv_sim_substep_rows(self._handle, float(np.float32(dt)), int(step_number), int(row0),
                                                  int(nrows)))
        if last and self._cur is not None:
            self._cur ^= 1

    def tile_rows(self):
        """Number of tile rows of a substep."""
        r = ctypes.c_int()
        _lib.check(_lib.lib().fv_sim_tile_rows(self._handle, ctypes.byref(r)))
        return r.value

    def advance(self, n_steps):
        """Run exactly n_steps steps with simulate()'s dt schedule (benchmark helper)."""
        self._cur = None
        _lib.check(_lib.lib().fv_sim_advance(self._handle, int(n_steps)))

    # -- device state for row-stripe halo exchange (MPISimulator.py)
    def halo_views(self, pending=False):
        """Zero-copy torch views of the rows a north-south halo exchange moves, in
        the buffer that holds the current state (pending=True: the buffer the
        substep whose bands are being launched writes): a dict with
        'south_ghost' (domain rows -2, -1), 'south_send' (rows 0, 1),
        'north_send' (rows ny-2, ny-1) and 'north_ghost' (rows ny, ny+1), each
        a list with one 1-D float32 CUDA tensor per variable covering those two
        full storage rows (ghost columns included).  Work on them must be
        ordered after the stage launches that write them."""
        import torch

        if self._state is None or self._cur is None:
            ptrs = (_lib._FP * 8)()
            pitch, cur = ctypes.c_int(), ctypes.c_int()
            _lib.check(_lib.lib().fv_sim_buffers(self._handle, ptrs, ctypes.byref(pitch), ctypes.byref(cur)))
            addrs = [ctypes.cast(ptrs[k], ctypes.c_void_p).value for k in range(8)]
            self._state = (addrs, pitch.value)
            self._cur = cur.value
        addrs, pitch = self._state
        ny = int(self.ny)
        dev = torch.device("cuda", self.context.device_id)

        buf = self._cur ^ 1 if pending else self._cur

        def rows(var, r0):
            base = addrs[buf * 4 + var] + r0 * pitch * 4
            return torch.as_tensor(_DeviceRows(base, 2 * pitch), device=dev)

        views = {"south_ghost": 0, "south_send": 2, "north_send": ny, "north_ghost": ny + 2}
        return {k: [rows(v, r0) for v in range(self._nv)] for k, r0 in views.items()}

    def comm_stream(self):
        """The simulation's CUDA stream as a torch stream."""
        import torch

        p = ctypes.c_void_p()
        _lib.check(_lib.lib().fv_sim_stream(self._handle, ctypes.byref(p)))
        return torch.cuda.ExternalStream(p.value or 0, device=torch.device("cuda", self.context.device_id))

    def computeDt(self):
        d = ctypes.c_float()
        _lib.check(_lib.lib().fv_sim_compute_dt(self._handle, ctypes.byref(d)))
        return np.float32(d.value)

    # -- state access
    def _download_var(self, var, cpu_data=None):
        nx, ny = int(self.nx), int(self.ny)
        if cpu_data is None:
            cpu_data = np.empty((ny, nx), dtype=np.float32)
        _lib.require(cpu_data.shape == (ny, nx) and cpu_data.dtype == np.float32 and cpu_data.flags.c_contiguous,
                     "cpu_data must be a C-ordered float32 array of shape (ny, nx)")
        _lib.check(_lib.lib().fv_sim_download(self._handle, int(var), cpu_data.ctypes.data_as(_lib._FP), nx))
        return cpu_data

    def download(self, variables=None):
        if variables is None:
            variables = range(self._nv)
        out = []
        for i in variables:
            assert i < self._nv, "Variable {:d} is out of range".format(i)
            out.append(self._download_var(i))
        return out

    def upload(self, var, data):
        """Replace the interior of variable `var` of the current state."""
        data = np.ascontiguousarray(data, dtype=np.float32)
        _lib.require(data.shape == (int(self.ny), int(self.nx)), "data shape does not match the grid")
        _lib.check(_lib.lib().fv_sim_upload(self._handle, int(var), data.ctypes.data_as(_lib._FP), int(self.nx)))

    def getOutput(self):
        return _StateView(self)

    @property
    def u0(self):
        return _StateView(self)

    def conservation(self):
        """FP64 sums of the conserved variables over the interior."""
        s = (ctypes.c_double * 4)()
        _lib.check(_lib.lib().fv_sim_conservation(self._handle, s))
        return np.array(s[: self._nv], dtype=np.float64)

    def check(self):
        f = ctypes.c_int()
        _lib.check(_lib.lib().fv_sim_check(self._handle, ctypes.byref(f)))
        assert f.value == 0, "Data contains NaN values!"

    def synchronize(self):
        _lib.check(_lib.lib().fv_sim_synchronize(self._handle))

    def _time(self):
        t = ctypes.c_double()
        nt = ctypes.c_longlong()
        dt = ctypes.c_float()
        _lib.check(_lib.lib().fv_sim_time(self._handle, ctypes.byref(t), ctypes.byref(nt), ctypes.byref(dt)))
        return t.value, nt.value, np.float32(dt.value)

    def simTime(self):
        return self._time()[0]

    def simSteps(self):
        return self._time()[1]

    @property
    def t(self):
        return self._time()[0]

    @property
    def nt(self):
        return self._time()[1]

    @property
    def dt(self):
        return self._time()[2]

    def get_control(self):
        """(t, nt, dt, cfl_min): the time-stepping state a checkpoint stores."""
        t, nt = ctypes.c_double(), ctypes.c_longlong()
        dt, cfl = ctypes.c_float(), ctypes.c_float()
        _lib.check(_lib.lib().fv_sim_get_control(self._handle, ctypes.byref(t), ctypes.byref(nt), ctypes.byref(dt),
                                                 ctypes.byref(cfl)))
        return t.value, nt.value, np.float32(dt.value), np.float32(cfl.value)

    def set_control(self, t, nt, dt, cfl_min):
        """Restore the time-stepping state saved by get_control (checkpoint resume)."""
        _lib.check(_lib.lib().fv_sim_set_control(self._handle, float(t), int(nt), float(np.float32(dt)),
                                                 float(np.float32(cfl_min))))

    def getExtent(self):
        return [0, 0, self.nx * self.dx, self.ny * self.dy]

    def setBoundaryConditions(self, boundary_conditions):
        self.logger.debug("Boundary conditions set to {:s}".format(str(boundary_conditions)))
        self.boundary_conditions = boundary_conditions.asCodedInt()
        if self._handle is not None:
            _lib.check(_lib.lib().fv_sim_set_boundary_conditions(self._handle, int(self.boundary_conditions)))

    def getBoundaryConditions(self):
        return BoundaryCondition(BoundaryCondition.getTypes(self.boundary_conditions))

    def tile_info(self):
        w, h, nt, lps = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _lib.check(_lib.lib().fv_sim_info(self._handle, ctypes.byref(w), ctypes.byref(h), ctypes.byref(nt),
                                          ctypes.byref(lps)))
        return {"tile_w": w.value, "tile_h": h.value, "threads": nt.value, "launches_per_step": lps.value}

    def last_advance_ms(self):
        ms = ctypes.c_double()
        _lib.check(_lib.lib().fv_sim_last_advance_ms(self._handle, ctypes.byref(ms)))
        return ms.value
