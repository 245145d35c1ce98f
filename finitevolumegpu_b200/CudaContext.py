"""Device context: the counterpart of GPUSimulators/CudaContext.py.

The reference's CudaContext creates a PyCUDA context and JIT-compiles kernels
through a hashed cubin cache (GPUSimulators/CudaContext.py:47-258).  Here the
kernels are compiled ahead of time for sm_100a into libfvgpu.so, so the
context only selects the device; ``autotuning`` makes the simulators pick
their tile shape from the project's autotuner cache (``Autotuner.py``).
"""

from __future__ import annotations

import ctypes
import logging

from . import _lib


class CudaContext(object):
    def __init__(self, device=None, context_flags=None, use_cache=True, autotuning=True):
        self.logger = logging.getLogger(__name__)
        self.device_id = 0 if device is None else int(device)
        self.use_cache = use_cache
        h = ctypes.c_void_p()
        _lib.check(_lib.lib().fv_context_create(self.device_id, ctypes.byref(h)))
        self._handle = h
        buf = ctypes.create_string_buffer(256)
        _lib.check(_lib.lib().fv_context_device_name(h, buf, 256))
        self.device_name = buf.value.decode()
        self.autotuner = None
        if autotuning:
            from .Autotuner import Autotuner

            self.autotuner = Autotuner()
        self.logger.debug("Using device %d '%s'", self.device_id, self.device_name)

    @property
    def handle(self):
        return self._handle

    def __str__(self):
        return "CudaContext id %d (%s)" % (self.device_id, self.device_name)

    def synchronize(self):
        # Every simulator synchronises its own stream; nothing is pending here.
        pass

    def get_module(self, kernel_filename, include_dirs=(), defines=None, compile_args=None, jit_compile_args=None):
        """The reference compiles one PyCUDA module per kernel file at run time
        (GPUSimulators/CudaContext.py:178-260).  libfvgpu's kernels are compiled
        ahead of time into one library, so there is no module to return."""
        raise NotImplementedError("kernels are built into libfvgpu.so; %s has no run-time module" % kernel_filename)

    def clear_kernel_cache(self):
        """No run-time kernel cache exists (GPUSimulators/CudaContext.py:263-268)."""
        pass

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and _lib._lib is not None:
            _lib.lib().fv_context_destroy(h)
            self._handle = None
