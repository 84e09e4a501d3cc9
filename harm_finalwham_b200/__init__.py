"""B200-native per-zone conservative update of HARM (pseudotensor/harm_finalwham).

The product is the C-ABI library ``lib/libharmgpu.so`` (include/harmgpu.h),
hand-written CUDA for sm_100a.  This package adds the Python plumbing used by
the tests and the benchmark: ctypes bindings (``gpu``), the in-tree build
(``build``) and a synthetic Kerr-torus input generator (``torus``).
"""
from .gpu import HarmGPU, HarmGPUError, load_library  # noqa: F401

__all__ = ["HarmGPU", "HarmGPUError", "load_library"]
