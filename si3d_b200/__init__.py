"""B200-native (sm_100a) implementation of pSi3D's per-timestep semi-implicit core.

The compute path lives in the CUDA library behind include/si3d_gpu.h; the C++ host behind
include/si3d_host.h reads the reference's input files and drives the time loop; this package holds
the ctypes bindings (native), the Python API (model), the workload generator (synth) and the build.
"""
from .native import SI3D_FP64, SI3D_MIXED_IR, SI3D_X0_LEARNED, SI3D_X0_PREV, SI3D_X0_ZERO, Si3dError  # noqa: F401

__all__ = ["SI3D_FP64", "SI3D_MIXED_IR", "SI3D_X0_PREV", "SI3D_X0_ZERO", "SI3D_X0_LEARNED", "Si3dError"]
