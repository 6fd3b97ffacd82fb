// sodecl_batch_run_noalloc: a launch of the heterogeneous batch kernel that
// allocates no memory.
//
// Who needs it: callers that own every device buffer themselves and must not
// have a library allocate behind their back -- a custom operator inside a
// framework whose caching allocator manages all device memory, or a service
// that allocates its working set once at start-up and never again.
// cudaMalloc/cudaFree in their launch path would synchronise the device and
// fragment memory someone else manages.  They pass inputs and outputs as
// device buffers they allocated; the only scratch the kernel needs -- one
// work-queue head per class -- lives in a file-scope device array here.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <numeric>

#include "batch_internal.hpp"
#include "device_memory.hpp"

namespace {

// The batch kernel's scratch for this entry point: one work-queue head per
// class, at most kMaxClasses (32) classes, 256 bytes.  Every GPU that loads
// the library holds it until the process exits.  All calls on a device share
// it and it keeps the last call's contents: each call clears it before its
// launch, and calls that overlap on the GPU race on it.
static __device__ __align__(256) unsigned long long g_noalloc_queue_heads[kMaxClasses];

constexpr int kMaxDevices = 128;
std::mutex g_setup_mutex;
void *g_heads_address[kMaxDevices] = {};

// The array's device address on `device` (current), looked up once per
// device.  In host code the array's name is only a host-side stand-in, not a
// device address, so it is never handed to a kernel directly.
cudaError_t queue_heads_on(int device, unsigned long long **out)
{
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_heads_address[device]) {
        void *ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_queue_heads);
        if (e != cudaSuccess) return e;
        g_heads_address[device] = ptr;
    }
    *out = static_cast<unsigned long long *>(g_heads_address[device]);
    return cudaSuccess;
}

int fail(sodecl_batch *b, int code, const std::string &msg)
{
    b->error = msg;
    return code;
}

struct CurrentDevice {
    int prev = -1;
    bool ok = false;
    explicit CurrentDevice(int dev)
    {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        ok = cudaSetDevice(dev) == cudaSuccess;
    }
    ~CurrentDevice()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

extern "C" int sodecl_batch_run_noalloc(sodecl_batch *b, const sodecl_batch_io *io, void *stream)
{
    if (!b) return SODECL_ERR_INVALID_ARG;
    if (!b->prog) return fail(b, SODECL_ERR_STATE, "no-alloc run: call sodecl_batch_compile first");
    if (!io || !io->t || !io->y || !io->nsteps || !io->class_count)
        return fail(b, SODECL_ERR_INVALID_ARG, "no-alloc run: t, y, nsteps and class_count are required");
    const int nc = static_cast<int>(b->classes.size());
    if (nc > kMaxClasses)
        return fail(b, SODECL_ERR_INVALID_ARG,
                    "no-alloc run: " + std::to_string(nc) + " classes, the scratch holds at most " +
                        std::to_string(kMaxClasses));
    bool stochastic = false, any_params = false;
    for (const auto &c : b->classes) {
        stochastic = stochastic || c.def.spec.solver == SODECL_STOCHASTIC_EULER;
        any_params = any_params || c.def.spec.num_params > 0;
    }
    if (stochastic && !io->counters) return fail(b, SODECL_ERR_INVALID_ARG, "no-alloc run: a stochastic class needs counters");
    if (any_params && !io->params) return fail(b, SODECL_ERR_INVALID_ARG, "no-alloc run: params are required");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || b->device >= count || b->device >= kMaxDevices) {
        cudaGetLastError();
        return fail(b, SODECL_ERR_NO_DEVICE, "no-alloc run: no CUDA device " + std::to_string(b->device));
    }
    CurrentDevice dev(b->device);
    if (!dev.ok) return fail(b, SODECL_ERR_NO_DEVICE, "no-alloc run: cannot select the device");
    for (const void *p : {static_cast<const void *>(io->t), static_cast<const void *>(io->y),
                          static_cast<const void *>(io->params), static_cast<const void *>(io->counters),
                          static_cast<const void *>(io->nsteps), static_cast<const void *>(io->newton_passes),
                          static_cast<const void *>(io->flags)})
        if (!sodecl_b200::kernel_can_access(p, b->device))
            return fail(b, SODECL_ERR_INVALID_ARG, "no-alloc run: a buffer is not memory this device can access "
                                                   "(device, managed or pinned host memory)");

    // first call on this device: load the batch program and look up the
    // scratch array's address
    cudaKernel_t kernel = b->kernel;
    if (!kernel) {
        if (!b->noalloc_kernel) {
            if (cudaLibraryLoadData(&b->noalloc_lib, b->prog->cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0) !=
                    cudaSuccess ||
                cudaLibraryGetKernel(&b->noalloc_kernel, b->noalloc_lib, b->prog->kernel_name.c_str()) != cudaSuccess) {
                const cudaError_t e = cudaGetLastError();
                return fail(b, SODECL_ERR_CUDA, std::string("no-alloc run: loading the program: ") + cudaGetErrorString(e));
            }
        }
        kernel = b->noalloc_kernel;
    }
    unsigned long long *heads = nullptr;
    cudaError_t e = queue_heads_on(b->device, &heads);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(b, SODECL_ERR_CUDA, std::string("no-alloc run: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    }

    // the caller's arrays hold class 0's orbits, then class 1's, ...
    BatchArgs a{};
    a.t = io->t;
    a.y = io->y;
    a.p = io->params;
    a.counters = io->counters;
    a.nsteps = reinterpret_cast<const long long *>(io->nsteps);
    a.orbit_id = nullptr;  // the noise stream is keyed by the position in these arrays
    a.newton_passes = reinterpret_cast<long long *>(io->newton_passes);
    a.flags = reinterpret_cast<int *>(io->flags);
    a.head = heads;
    a.nclasses = nc;
    long long pos = 0, yb = 0, pb = 0;
    double work[kMaxClasses];
    for (int c = 0; c < nc; ++c) {
        const long long k = io->class_count[c];
        if (k < 0) return fail(b, SODECL_ERR_INVALID_ARG, "no-alloc run: negative class count");
        const auto &s = b->classes[c].def.spec;
        a.begin[c] = pos;
        a.end[c] = pos + k;
        a.ybase[c] = yb;
        a.pbase[c] = pb;
        work[c] = static_cast<double>(k) * b->classes[c].cost_per_step;
        pos += k;
        yb += k * s.num_equat;
        pb += k * s.num_params;
    }
    if (pos == 0) return SODECL_OK;
    int order[kMaxClasses];
    std::iota(order, order + nc, 0);
    std::stable_sort(order, order + nc, [&](int x, int y) { return work[x] > work[y]; });
    for (int k = 0; k < nc; ++k) a.order[k] = order[k];

    const int block = b->block;
    int per_sm = 0;
    const size_t shared = sodecl_b200_batch::shared_bytes(b, block);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, reinterpret_cast<const void *>(kernel), block, shared) !=
            cudaSuccess ||
        per_sm < 1) {
        cudaGetLastError();
        per_sm = 1;
    }
    if (b->blocks_per_sm > 0) per_sm = std::min(per_sm, b->blocks_per_sm);
    int sms = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the heads keep the previous call's values: clear them first
    e = cudaMemsetAsync(heads, 0, sizeof(unsigned long long) * kMaxClasses, s);
    if (e == cudaSuccess) {
        void *params[] = {&a};
        e = cudaLaunchKernel(reinterpret_cast<const void *>(kernel), dim3(std::max(1, sms) * per_sm), dim3(block),
                             params, shared, s);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(b, SODECL_ERR_CUDA, std::string("no-alloc run: launch: ") + cudaGetErrorString(e));
    }
    return SODECL_OK;
}
