"""KP07: Kurganov-Petrova 2007 central-upwind scheme with RK time stepping -- the counterpart of GPUSimulators/KP07.py.

Constructor arguments and defaults follow GPUSimulators/KP07.py:54-106;
one step is `order` launch(es) of the sm_100a stage kernel in libfvgpu.so.
"""

import numpy as np

from . import Simulator
from .Simulator import BoundaryCondition


class KP07(Simulator.BaseSimulator):
    _scheme = "KP07"
    _gc = 2

    def __init__(self,
                 context,
                 h0, hu0, hv0,
                 nx, ny,
                 dx, dy,
                 g,
                 theta=1.3,
                 cfl_scale=0.9,
                 order=2,
                 boundary_conditions=BoundaryCondition(),
                 block_width=16, block_height=16):
        assert order in (1, 2), "KP07 supports order 1 or 2"
        super().__init__(context, nx, ny, dx, dy, boundary_conditions, cfl_scale, order, block_width,
                         block_height)
        self.g = np.float32(g)
        self.theta = np.float32(theta)
        self.order = np.int32(order)
        self._create([h0, hu0, hv0], g=g, theta=theta, order=order)
