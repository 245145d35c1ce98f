"""WAF: weighted average flux scheme with dimensional splitting -- the counterpart of GPUSimulators/WAF.py.

Constructor arguments and defaults follow GPUSimulators/WAF.py:50-97;
one step is 2 launch(es) of the sm_100a stage kernel in libfvgpu.so.
"""

import numpy as np

from . import Simulator
from .Simulator import BoundaryCondition


LIMITERS = {"generalized_minmod": 0, "minmod": 1, "superbee": 2, "vanLeer": 3, "vanAlbada1": 4, "vanAlbada2": 5,
            "monotonized_central": 6, "osher": 7, "sweby": 8}


class WAF(Simulator.BaseSimulator):
    _scheme = "WAF"
    _gc = 2

    def __init__(self,
                 context,
                 h0, hu0, hv0,
                 nx, ny,
                 dx, dy,
                 g,
                 cfl_scale=0.9,
                 boundary_conditions=BoundaryCondition(),
                 block_width=16, block_height=16,
                 limiter="generalized_minmod", limiter_beta=1.5):
        """`limiter` (not in the reference's class): the flux limiter of the
        WAF weights; "generalized_minmod" (theta 1.9) is the reference's, the
        others are those its limiters.h defines (:84-118).  `limiter_beta` is
        the beta of "osher" and "sweby"."""
        assert limiter in LIMITERS, "limiter must be one of %s" % (tuple(LIMITERS),)
        super().__init__(context, nx, ny, dx, dy, boundary_conditions, cfl_scale, 2, block_width,
                         block_height)
        self.g = np.float32(g)
        self.limiter = limiter
        self.limiter_beta = np.float32(limiter_beta)
        self._create([h0, hu0, hv0], g=g, variant=LIMITERS[limiter], variant_beta=limiter_beta)
