"""B200-native P3M gravity step for one CUBE image (nn=1).

The product is the CUDA library libcube_gpu.so behind the C ABI of include/cube_gpu.h;
this package builds it, binds it (ctypes) and provides the host-side pieces a CUBE
host keeps: parameters, timestep, ICs, checkpoint I/O and the step loop.
"""
from .params import DEPOSIT_FIXED, DEPOSIT_FP32, Params  # noqa: F401


def __getattr__(name):
    if name in ("Context", "CubeError"):
        from . import _lib

        return getattr(_lib, name)
    if name == "Simulation":
        from .simulation import Simulation

        return Simulation
    raise AttributeError(name)
