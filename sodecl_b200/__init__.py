"""sodecl_b200: SODECL's fixed-step ODE/SDE integrators on NVIDIA B200 (sm_100a).

Native parts (built in-tree by sodecl_b200/build.py):
  libsodecl_cuda.so   C ABI (include/sodecl_cuda.h), NVRTC front end, kernels,
                      C++ sodecl::sodeclmgr (include/sodeclmgr.hpp)
  sodecl_interface    the reference's pybind11 module (sodeclcall)

Python: `Integrator` (numpy API), `sodecl.sodecl(...)` (the reference's
function), `system_path(name)` for the bundled system files.
"""
from .api import Integrator, fma_peak, noise_stream, system_path  # noqa: F401

__all__ = ["Integrator", "fma_peak", "noise_stream", "system_path"]
