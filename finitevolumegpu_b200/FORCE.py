"""FORCE: first-order centred (FORCE) scheme -- the counterpart of GPUSimulators/FORCE.py.

Constructor arguments and defaults follow GPUSimulators/FORCE.py:56-89;
one step is 1 launch(es) of the sm_100a stage kernel in libfvgpu.so.
"""

import numpy as np

from . import Simulator
from .Simulator import BoundaryCondition


class FORCE(Simulator.BaseSimulator):
    _scheme = "FORCE"
    _gc = 1

    def __init__(self,
                 context,
                 h0, hu0, hv0,
                 nx, ny,
                 dx, dy,
                 g,
                 cfl_scale=0.9,
                 boundary_conditions=BoundaryCondition(),
                 block_width=16, block_height=16):
        super().__init__(context, nx, ny, dx, dy, boundary_conditions, cfl_scale, 1, block_width,
                         block_height)
        self.g = np.float32(g)
        self._create([h0, hu0, hv0], g=g)
