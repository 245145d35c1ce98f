"""EE2D_KP07_dimsplit: dimensionally split Kurganov-Petrova scheme for the
2-D Euler equations -- the counterpart of GPUSimulators/EE2D_KP07_dimsplit.py.

Constructor arguments and defaults follow EE2D_KP07_dimsplit.py:57-67.  The
reference class never swaps u0/u1 in its own substep (the swap lives in a
separate swapBuffers() that only MPISimulator calls, EE2D_KP07_dimsplit.py:268-270),
so its single-GPU simulate() does not advance the returned state; this class
swaps after every substep, which is what MPISimulator does.
"""

import numpy as np

from . import Simulator
from .Simulator import BoundaryCondition


class EE2D_KP07_dimsplit(Simulator.BaseSimulator):
    _scheme = "EE2D_KP07_dimsplit"
    _gc = 2

    def __init__(self,
                 context,
                 rho, rho_u, rho_v, E,
                 nx, ny,
                 dx, dy,
                 g,
                 gamma,
                 theta=1.3,
                 cfl_scale=0.9,
                 boundary_conditions=BoundaryCondition(),
                 block_width=16, block_height=8):
        super().__init__(context, nx, ny, dx, dy, boundary_conditions, cfl_scale, 2, block_width, block_height)
        self.g = np.float32(g)
        self.gamma = np.float32(gamma)
        self.theta = np.float32(theta)
        self._create([rho, rho_u, rho_v, E], g=g, gamma=gamma, theta=theta)

    def swapBuffers(self):
        """Kept for API compatibility: buffers are swapped after every substep."""
        return
