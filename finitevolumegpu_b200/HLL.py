"""HLL: first-order HLL scheme with dimensional splitting -- the counterpart of GPUSimulators/HLL.py.

Constructor arguments and defaults follow GPUSimulators/HLL.py:51-84;
one step is 1 launch(es) of the sm_100a stage kernel in libfvgpu.so.
"""

import numpy as np

from . import Simulator
from .Simulator import BoundaryCondition


FLUXES = {"HLL": 0, "HLLC": 1, "GodC": 2}


class HLL(Simulator.BaseSimulator):
    _scheme = "HLL"
    _gc = 1

    def __init__(self,
                 context,
                 h0, hu0, hv0,
                 nx, ny,
                 dx, dy,
                 g,
                 cfl_scale=0.9,
                 boundary_conditions=BoundaryCondition(),
                 block_width=16, block_height=16,
                 flux="HLL"):
        """`flux` (not in the reference's class): "HLL" (the reference's), or the
        variants its SWECommon.h defines but no scheme uses: "HLLC"
        (SWECommon.h:334-387) and "GodC", Godunov's centred flux (:248-255)."""
        assert flux in FLUXES, "flux must be one of %s" % (tuple(FLUXES),)
        super().__init__(context, nx, ny, dx, dy, boundary_conditions, cfl_scale, 1, block_width,
                         block_height)
        self.g = np.float32(g)
        self.flux = flux
        self._create([h0, hu0, hv0], g=g, variant=FLUXES[flux])
