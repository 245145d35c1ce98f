"""finitevolumegpu_b200: B200-native (sm_100a) implementation of the
GPUSimulators time-step path of babrodtk/FiniteVolumeGPU.

Module layout mirrors the reference package so that
``from finitevolumegpu_b200 import KP07_dimsplit`` gives the module and
``KP07_dimsplit.KP07_dimsplit(context, h0, hu0, hv0, nx, ny, dx, dy, g)`` the
simulator, as with GPUSimulators.
"""

from . import Simulator, CudaContext, batch  # noqa: F401
from . import LxF, FORCE, HLL, HLL2, WAF, KP07, KP07_dimsplit, EE2D_KP07_dimsplit  # noqa: F401
from .Simulator import BoundaryCondition, BaseSimulator  # noqa: F401

SCHEMES = {
    "LxF": LxF.LxF,
    "FORCE": FORCE.FORCE,
    "HLL": HLL.HLL,
    "HLL2": HLL2.HLL2,
    "WAF": WAF.WAF,
    "KP07": KP07.KP07,
    "KP07_dimsplit": KP07_dimsplit.KP07_dimsplit,
    "EE2D_KP07_dimsplit": EE2D_KP07_dimsplit.EE2D_KP07_dimsplit,
}

__version__ = "0.1.0"
