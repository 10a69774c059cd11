"""B200-native DDA-FFT hot path (libddagpu) -- Python bindings over the C ABI.

The product is the C-ABI shared library dda_fft_b200/lib/libddagpu.so (include/ddagpu.h);
this module loads it with ctypes and mirrors the reference's DDA_FFT interface for tests
and benchmarks.  There is no CPU fallback: if the library cannot be loaded, every call
raises.
"""
from .api import (  # noqa: F401
    Agglomerate,
    BatchConfig,
    Context,
    DDAGPUError,
    Group,
    RandomEllipsoid,
    StateFile,
    build,
    farfield_plan,
    fixed_rotation,
    lib,
    library_path,
    mc_rotations,
    num_angles,
    sample_loop,
)

__all__ = ["Agglomerate", "BatchConfig", "Context", "DDAGPUError", "Group", "RandomEllipsoid", "StateFile",
           "build", "farfield_plan", "fixed_rotation", "lib", "library_path", "mc_rotations", "num_angles",
           "sample_loop"]
