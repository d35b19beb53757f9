"""brae_b200 -- a B200-native GAMG-preconditioned PCG pressure solver behind a C ABI.

The product is the CUDA library ``brae_b200/libbrae_gamg.so`` (built by ``brae_b200.build``) and its
C header ``include/brae_gamg.h``; ``brae_b200.native`` binds that ABI with ctypes for Python
callers, tests and benchmarks. There is no Python or CPU fallback: if the library is missing,
``brae_b200.native`` raises on import. ``brae_b200.cases`` builds the synthetic benchmark systems.
"""
import importlib

_NATIVE = {"B2G_MEM_DEVICE", "B2G_MEM_HOST", "Controls", "GamgError", "Matrix", "Mesh",
           "SolverPerformance", "controls_default", "gamg_solve", "lib", "pcg_gamg_solve",
           "read_controls"}


def __getattr__(name):
    if name in _NATIVE:
        return getattr(importlib.import_module(".native", __name__), name)
    raise AttributeError(name)
