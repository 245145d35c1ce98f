"""KP07_dimsplit: dimensionally split Kurganov-Petrova 2007 scheme -- the counterpart of GPUSimulators/KP07_dimsplit.py.

Constructor arguments and defaults follow GPUSimulators/KP07_dimsplit.py:55-106;
one step is 2 launch(es) of the sm_100a stage kernel in libfvgpu.so.
"""

import numpy as np

from . import Simulator
from .Simulator import BoundaryCondition


class KP07_dimsplit(Simulator.BaseSimulator):
    _scheme = "KP07_dimsplit"
    _gc = 2

    def __init__(self,
                 context,
                 h0, hu0, hv0,
                 nx, ny,
                 dx, dy,
                 g,
                 theta=1.3,
                 cfl_scale=0.9,
                 boundary_conditions=BoundaryCondition(),
                 block_width=16, block_height=16):
        super().__init__(context, nx, ny, dx, dy, boundary_conditions, cfl_scale, 2, block_width,
                         block_height)
        self.g = np.float32(g)
        self.theta = np.float32(theta)
        self._create([h0, hu0, hv0], g=g, theta=theta)
