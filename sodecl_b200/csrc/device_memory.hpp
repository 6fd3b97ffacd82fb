// Which memory a kernel may dereference: shared by the entry points that take
// caller-owned device pointers (sodecl_cuda_launch, sodecl_cuda_adjoint,
// sodecl_batch_run_noalloc).
#pragma once

#include <cuda_runtime.h>

namespace sodecl_b200 {

// Whether a kernel on `device` may dereference p: memory of that device,
// managed memory, or pinned host memory (mapped into the device's address
// space).  Pageable host memory, another device's memory or an address CUDA
// does not know would fault the kernel, so those entry points refuse them.
// Allocates nothing.  Whether a null p is allowed is for the caller to decide.
inline bool kernel_can_access(const void *p, int device)
{
    if (!p) return true;
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    switch (attr.type) {
    case cudaMemoryTypeDevice: return attr.device == device;
    case cudaMemoryTypeManaged: return true;
    case cudaMemoryTypeHost: return attr.devicePointer != nullptr;
    default: return false;
    }
}

}  // namespace sodecl_b200
