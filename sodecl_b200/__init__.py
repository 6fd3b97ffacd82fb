"""sodecl_b200: SODECL's fixed-step ODE/SDE integrators on NVIDIA B200 (sm_100a).

Native parts (built in-tree by sodecl_b200/build.py):
  libsodecl_cuda.so   C ABI (include/sodecl_cuda.h), NVRTC front end, kernels,
                      C++ sodecl::sodeclmgr (include/sodeclmgr.hpp)
  sodecl_interface    the reference's pybind11 module (sodeclcall)

Python: `Integrator` (numpy API), `sodecl.sodecl(...)` (the reference's
function), `system_path(name)` for the bundled system files.

The names below load libsodecl_cuda.so on first use, not at import, so that a
module of this package that needs no GPU (the seeded workload generators in
`workloads`) can be imported without mapping the library.
"""
import importlib

__all__ = ["Integrator", "fma_peak", "noise_stream", "sin_peak", "system_path"]


def __getattr__(name):
    if name in __all__:
        return getattr(importlib.import_module(".api", __name__), name)
    raise AttributeError("module %r has no attribute %r" % (__name__, name))
