// libsodecl_cuda: the C ABI of include/sodecl_cuda.h.
//
// Replaces the OpenCL plumbing of the reference's sodecl::sodeclmgr
// (src/sodeclmgr.cpp): the program is built by NVRTC (program.cpp), buffers
// are plain device allocations, and the run loop -- one launch and one
// blocking read-back plus host transpose per record in the reference
// (:951-1015) -- becomes a few launches that each advance every orbit through
// many record intervals and write the records from the device in the final
// [record][equation][orbit] order, with the device-to-host copy of finished
// records overlapped with the launches still running.
#include "sodecl_cuda.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "program.hpp"

using sodecl_b200::Program;
using sodecl_b200::ProgramSpec;

namespace {

// Must match struct sodecl_args in device/solvers.cuh field for field.
struct DeviceArgs {
    double *t;
    double *y;
    const double *p;
    double *counters;
    void *records;
    long long n;
    long long orbit_offset;
    long long rec_stride;
    long long rec_col0;
    int chunk_begin;
    int chunk_end;
    int rec_first;
    int write_final;
    long long *newton_passes;
    int *flags;
};

constexpr int kDefaultBlock = 128;
constexpr int kMaxCopyGroups = 8;

}  // namespace

struct sodecl_ctx {
    sodecl_cfg cfg{};
    std::string system_src;
    std::shared_ptr<const Program> prog;
    std::string error;
    int64_t nchunks = 0;

    bool gpu_ready = false;
    int loaded_device = -1;
    cudaLibrary_t lib = nullptr;
    cudaKernel_t kernel = nullptr;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;

    double *d_t = nullptr, *d_y = nullptr, *d_p = nullptr, *d_cnt = nullptr;
    long long *d_passes = nullptr;
    int *d_flags = nullptr;
    bool uploaded = false;
    void *d_records = nullptr;
    size_t d_records_bytes = 0;

    double last_kernel_ms = 0.0;
    double last_total_ms = 0.0;

    int fail(int code, const std::string &msg)
    {
        error = msg;
        return code;
    }
};

namespace {

// Keeps the caller's current device: switch to the context's device for the
// duration of one API call.
class DeviceScope {
  public:
    explicit DeviceScope(int dev)
    {
        if (cudaGetDevice(&prev_) != cudaSuccess) prev_ = -1;
        ok_ = cudaSetDevice(dev) == cudaSuccess;
    }
    ~DeviceScope()
    {
        if (prev_ >= 0) cudaSetDevice(prev_);
    }
    bool ok() const { return ok_; }

  private:
    int prev_ = -1;
    bool ok_ = false;
};

int cuda_fail(sodecl_ctx *ctx, cudaError_t e, const char *what)
{
    cudaGetLastError();
    if (e == cudaErrorMemoryAllocation)
        return ctx->fail(SODECL_ERR_OUT_OF_MEMORY, std::string(what) + ": " + cudaGetErrorString(e));
    if (e == cudaErrorNoDevice || e == cudaErrorInvalidDevice || e == cudaErrorInsufficientDriver)
        return ctx->fail(SODECL_ERR_NO_DEVICE, std::string(what) + ": " + cudaGetErrorString(e));
    return ctx->fail(SODECL_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define SODECL_CUDA_TRY(ctx, call)                                   \
    do {                                                             \
        cudaError_t e_ = (call);                                     \
        if (e_ != cudaSuccess) return cuda_fail((ctx), e_, #call);   \
    } while (0)

int64_t count_chunks(const sodecl_cfg &c)
{
    // for (int j = 0; j < (m_int_time/(m_dt*m_kernel_steps)); j++)  (src/sodeclmgr.cpp:951)
    const double x = c.int_time / (c.dt * c.kernel_steps);
    if (!(x > 0)) return 0;
    return static_cast<int64_t>(std::ceil(x));
}

size_t copy_string(const std::string &s, char *buf, size_t n)
{
    if (buf && n > 0) {
        const size_t k = std::min(n - 1, s.size());
        std::memcpy(buf, s.data(), k);
        buf[k] = '\0';
    }
    return s.size();
}

void free_buffers(sodecl_ctx *ctx)
{
    cudaFree(ctx->d_t);
    cudaFree(ctx->d_y);
    cudaFree(ctx->d_p);
    cudaFree(ctx->d_cnt);
    cudaFree(ctx->d_passes);
    cudaFree(ctx->d_flags);
    cudaFree(ctx->d_records);
    ctx->d_t = ctx->d_y = ctx->d_p = ctx->d_cnt = nullptr;
    ctx->d_passes = nullptr;
    ctx->d_flags = nullptr;
    ctx->d_records = nullptr;
    ctx->d_records_bytes = 0;
    ctx->uploaded = false;
}

// Loads the compiled program on the context's device and makes its streams.
int ensure_gpu(sodecl_ctx *ctx)
{
    if (!ctx->prog) return ctx->fail(SODECL_ERR_STATE, "no program: call sodecl_cuda_compile first");
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        return ctx->fail(SODECL_ERR_NO_DEVICE, std::string("no CUDA device available: ") + cudaGetErrorString(e));
    }
    if (ctx->cfg.device < 0 || ctx->cfg.device >= count)
        return ctx->fail(SODECL_ERR_NO_DEVICE, "device ordinal " + std::to_string(ctx->cfg.device) + " does not exist");
    if (ctx->gpu_ready) return SODECL_OK;
    SODECL_CUDA_TRY(ctx, cudaLibraryLoadData(&ctx->lib, ctx->prog->cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
    SODECL_CUDA_TRY(ctx, cudaLibraryGetKernel(&ctx->kernel, ctx->lib, ctx->prog->kernel_name.c_str()));
    if (!ctx->stream) SODECL_CUDA_TRY(ctx, cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    if (!ctx->copy_stream) SODECL_CUDA_TRY(ctx, cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
    ctx->loaded_device = ctx->cfg.device;
    ctx->gpu_ready = true;
    return SODECL_OK;
}

int block_size(const sodecl_ctx *ctx)
{
    return ctx->cfg.local_group_size > 0 ? ctx->cfg.local_group_size : kDefaultBlock;
}

int launch(sodecl_ctx *ctx, const DeviceArgs &a, cudaStream_t stream)
{
    if (a.n <= 0) return SODECL_OK;
    const int block = block_size(ctx);
    const long long grid = (a.n + block - 1) / block;
    if (grid > 0x7fffffffLL) return ctx->fail(SODECL_ERR_INVALID_ARG, "too many orbits for one launch");
    void *args[] = {const_cast<DeviceArgs *>(&a)};
    SODECL_CUDA_TRY(ctx, cudaLaunchKernel(reinterpret_cast<const void *>(ctx->kernel), dim3(static_cast<unsigned>(grid)),
                                          dim3(block), args, 0, stream));
    return SODECL_OK;
}

}  // namespace

extern "C" {

void sodecl_cfg_init(sodecl_cfg *cfg)
{
    if (!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->solver = SODECL_EULER;
    cfg->kernel_steps = 1;
    cfg->precision = SODECL_FP64;
    cfg->fmad = 1;
    cfg->newton_tol = 1e-7;
    cfg->newton_max_iter = 1000;
}

int sodecl_cuda_abi_version(void) { return SODECL_CUDA_ABI_VERSION; }

const char *sodecl_cuda_strerror(int status)
{
    switch (status) {
    case SODECL_OK: return "success";
    case SODECL_ERR_INVALID_ARG: return "invalid argument";
    case SODECL_ERR_COMPILE: return "program compilation failed";
    case SODECL_ERR_CUDA: return "CUDA runtime error";
    case SODECL_ERR_NO_DEVICE: return "no usable CUDA device";
    case SODECL_ERR_STATE: return "call out of order";
    case SODECL_ERR_NO_JACOBIAN: return "implicit solver needs calc_jacobian in the system file";
    case SODECL_ERR_NO_STOCH: return "stochastic solver needs sode_system_stoch in the system file";
    case SODECL_ERR_OUT_OF_MEMORY: return "out of memory";
    case SODECL_ERR_UNSUPPORTED: return "unsupported";
    default: return "unknown status";
    }
}

int sodecl_cuda_device_count(int *count)
{
    if (!count) return SODECL_ERR_INVALID_ARG;
    *count = 0;
    cudaError_t e = cudaGetDeviceCount(count);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *count = 0;
        return SODECL_ERR_NO_DEVICE;
    }
    return SODECL_OK;
}

int sodecl_cuda_create(const sodecl_cfg *cfg, sodecl_ctx **out)
{
    if (!out) return SODECL_ERR_INVALID_ARG;
    *out = nullptr;
    if (!cfg) return SODECL_ERR_INVALID_ARG;
    const sodecl_cfg &c = *cfg;
    if (c.solver < 0 || c.solver > 4) return SODECL_ERR_INVALID_ARG;
    if (c.num_equat < 1 || c.num_params < 0 || c.num_noi < 0 || c.list_size < 1) return SODECL_ERR_INVALID_ARG;
    if (!(c.dt > 0) || !std::isfinite(c.dt) || !(c.int_time >= 0) || !std::isfinite(c.int_time)) return SODECL_ERR_INVALID_ARG;
    if (c.kernel_steps < 1) return SODECL_ERR_INVALID_ARG;
    if (c.solver == SODECL_STOCHASTIC_EULER && c.num_noi < 1) return SODECL_ERR_INVALID_ARG;
    if (c.precision != SODECL_FP64 && c.precision != SODECL_FP32) return SODECL_ERR_INVALID_ARG;
    if (c.local_group_size < 0 || c.local_group_size > 1024) return SODECL_ERR_INVALID_ARG;
    if (c.newton_tol < 0 || !std::isfinite(c.newton_tol) || c.newton_max_iter < 0) return SODECL_ERR_INVALID_ARG;
    if (c.min_blocks_per_sm < 0 || c.min_blocks_per_sm > 32) return SODECL_ERR_INVALID_ARG;
    const int64_t nchunks = count_chunks(c);
    if (nchunks > 0x7ffffffeLL) return SODECL_ERR_INVALID_ARG;
    auto *ctx = new (std::nothrow) sodecl_ctx();
    if (!ctx) return SODECL_ERR_OUT_OF_MEMORY;
    ctx->cfg = c;
    if (ctx->cfg.newton_tol == 0) ctx->cfg.newton_tol = 1e-7;
    if (ctx->cfg.newton_max_iter == 0) ctx->cfg.newton_max_iter = 1000;
    ctx->nchunks = nchunks;
    *out = ctx;
    return SODECL_OK;
}

int sodecl_cuda_compile(sodecl_ctx *ctx, const char *system_src, size_t len)
{
    if (!ctx) return SODECL_ERR_INVALID_ARG;
    if (!system_src) return ctx->fail(SODECL_ERR_INVALID_ARG, "system source is NULL");
    std::string src(system_src, len);
    const auto traits = sodecl_b200::inspect_system(src);
    if (!traits.has_system) return ctx->fail(SODECL_ERR_COMPILE, "the system file defines no sode_system(...)");
    const int solver = ctx->cfg.solver;
    if ((solver == SODECL_IMPLICIT_EULER || solver == SODECL_IMPLICIT_MIDPOINT) && !traits.has_jacobian)
        return ctx->fail(SODECL_ERR_NO_JACOBIAN, "implicit solvers need calc_jacobian(...) in the system file");
    if (solver == SODECL_STOCHASTIC_EULER && !traits.has_stoch)
        return ctx->fail(SODECL_ERR_NO_STOCH, "the stochastic solver needs sode_system_stoch(...) in the system file");
    ProgramSpec spec;
    spec.solver = solver;
    spec.num_equat = ctx->cfg.num_equat;
    spec.num_params = ctx->cfg.num_params;
    spec.num_noi = ctx->cfg.num_noi;
    spec.list_size = ctx->cfg.list_size;
    spec.kernel_steps = ctx->cfg.kernel_steps;
    spec.dt = ctx->cfg.dt;
    spec.fp32 = ctx->cfg.precision == SODECL_FP32;
    spec.fmad = ctx->cfg.fmad != 0;
    spec.record_f32 = ctx->cfg.record_f32 != 0;
    spec.newton_tol = ctx->cfg.newton_tol;
    spec.newton_max_iter = ctx->cfg.newton_max_iter;
    spec.block_max = std::max(256, block_size(ctx));
    spec.min_blocks = ctx->cfg.min_blocks_per_sm;
    try {
        auto prog = sodecl_b200::build(spec, src);
        if (ctx->gpu_ready && prog != ctx->prog) {
            DeviceScope dev(ctx->loaded_device);
            if (ctx->lib) cudaLibraryUnload(ctx->lib);
            ctx->lib = nullptr;
            ctx->kernel = nullptr;
            ctx->gpu_ready = false;
        }
        ctx->prog = std::move(prog);
    } catch (const std::exception &ex) {
        return ctx->fail(SODECL_ERR_COMPILE, ex.what());
    }
    ctx->system_src = std::move(src);
    return SODECL_OK;
}

int sodecl_cuda_upload(sodecl_ctx *ctx, const double *t0, const double *y0, const double *params, const double *counters)
{
    if (!ctx) return SODECL_ERR_INVALID_ARG;
    if (!t0 || !y0 || (!params && ctx->cfg.num_params > 0))
        return ctx->fail(SODECL_ERR_INVALID_ARG, "t0, y0 and params must not be NULL");
    DeviceScope dev(ctx->cfg.device);
    int rc = ensure_gpu(ctx);
    if (rc != SODECL_OK) return rc;
    if (!dev.ok()) return ctx->fail(SODECL_ERR_NO_DEVICE, "cannot select the device");
    const size_t n = static_cast<size_t>(ctx->cfg.list_size);
    const size_t neq = ctx->cfg.num_equat, npar = ctx->cfg.num_params;
    if (!ctx->uploaded) {
        SODECL_CUDA_TRY(ctx, cudaMalloc(&ctx->d_t, n * sizeof(double)));
        SODECL_CUDA_TRY(ctx, cudaMalloc(&ctx->d_y, n * neq * sizeof(double)));
        SODECL_CUDA_TRY(ctx, cudaMalloc(&ctx->d_p, std::max<size_t>(1, n * npar) * sizeof(double)));
        SODECL_CUDA_TRY(ctx, cudaMalloc(&ctx->d_cnt, n * sizeof(double)));
        SODECL_CUDA_TRY(ctx, cudaMalloc(&ctx->d_passes, n * sizeof(long long)));
        SODECL_CUDA_TRY(ctx, cudaMalloc(&ctx->d_flags, n * sizeof(int)));
    }
    SODECL_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->d_t, t0, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    SODECL_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->d_y, y0, n * neq * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    if (npar > 0)
        SODECL_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->d_p, params, n * npar * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    std::vector<double> drawn;
    if (ctx->cfg.solver == SODECL_STOCHASTIC_EULER) {
        const double *src = counters;
        if (!src) {
            // the reference's draw (src/sodeclmgr.cpp:48-59), seeded for reproducibility
            std::mt19937 gen(0);
            std::uniform_real_distribution<double> unif(-100000000000.0, 100000000000.0);
            drawn.resize(n);
            for (auto &v : drawn) v = unif(gen);
            src = drawn.data();
        }
        SODECL_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->d_cnt, src, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    } else {
        SODECL_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_cnt, 0, n * sizeof(double), ctx->stream));
    }
    SODECL_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_passes, 0, n * sizeof(long long), ctx->stream));
    SODECL_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_flags, 0, n * sizeof(int), ctx->stream));
    SODECL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->uploaded = true;
    return SODECL_OK;
}

int64_t sodecl_cuda_num_records(const sodecl_ctx *ctx)
{
    return ctx ? ctx->nchunks + 1 : 0;
}

int sodecl_cuda_run(sodecl_ctx *ctx, double *out, int64_t out_len)
{
    if (!ctx) return SODECL_ERR_INVALID_ARG;
    if (!ctx->uploaded) return ctx->fail(SODECL_ERR_STATE, "no state on the device: call sodecl_cuda_upload first");
    if (ctx->cfg.record_f32) return ctx->fail(SODECL_ERR_UNSUPPORTED, "record_f32 programs serve sodecl_cuda_launch only");
    const int64_t n = ctx->cfg.list_size, neq = ctx->cfg.num_equat;
    const int64_t nrec = ctx->nchunks + 1;
    const int64_t rec_elems = neq * n;
    if (out && out_len < nrec * rec_elems)
        return ctx->fail(SODECL_ERR_INVALID_ARG, "output holds " + std::to_string(out_len) + " doubles, the run writes " +
                                                     std::to_string(nrec * rec_elems));
    DeviceScope dev(ctx->cfg.device);
    int rc = ensure_gpu(ctx);
    if (rc != SODECL_OK) return rc;

    DeviceArgs a{};
    a.t = ctx->d_t;
    a.y = ctx->d_y;
    a.p = ctx->d_p;
    a.counters = ctx->d_cnt;
    a.n = n;
    a.orbit_offset = 0;
    a.rec_stride = n;
    a.rec_col0 = 0;
    a.rec_first = 0;
    a.newton_passes = ctx->d_passes;
    a.flags = ctx->d_flags;

    cudaPointerAttributes attr{};
    bool device_out = false;
    if (out) {
        if (cudaPointerGetAttributes(&attr, out) != cudaSuccess) {
            cudaGetLastError();
            attr.type = cudaMemoryTypeUnregistered;
        }
        device_out = attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
    }

    cudaEvent_t t_begin, t_kernels, t_end;
    SODECL_CUDA_TRY(ctx, cudaEventCreate(&t_begin));
    SODECL_CUDA_TRY(ctx, cudaEventCreate(&t_kernels));
    SODECL_CUDA_TRY(ctx, cudaEventCreate(&t_end));
    struct EventGuard {
        cudaEvent_t *e;
        int k;
        ~EventGuard() { for (int i = 0; i < k; ++i) cudaEventDestroy(e[i]); }
    };
    cudaEvent_t timing[3] = {t_begin, t_kernels, t_end};
    EventGuard timing_guard{timing, 3};

    SODECL_CUDA_TRY(ctx, cudaEventRecord(t_begin, ctx->stream));
    if (!out || device_out) {
        // one launch through every interval, records straight into the output
        a.records = out;
        a.chunk_begin = 0;
        a.chunk_end = static_cast<int>(ctx->nchunks);
        a.write_final = 1;
        if ((rc = launch(ctx, a, ctx->stream)) != SODECL_OK) return rc;
        SODECL_CUDA_TRY(ctx, cudaEventRecord(t_kernels, ctx->stream));
        SODECL_CUDA_TRY(ctx, cudaEventRecord(t_end, ctx->stream));
    } else {
        // host output: launch groups of intervals into a device record buffer;
        // the copy stream moves each group's records out while later groups run
        const size_t need = static_cast<size_t>(nrec * rec_elems) * sizeof(double);
        if (ctx->d_records_bytes < need) {
            cudaFree(ctx->d_records);
            ctx->d_records = nullptr;
            ctx->d_records_bytes = 0;
            SODECL_CUDA_TRY(ctx, cudaMalloc(&ctx->d_records, need));
            ctx->d_records_bytes = need;
        }
        const int64_t groups = std::max<int64_t>(1, std::min<int64_t>(kMaxCopyGroups, ctx->nchunks));
        std::vector<cudaEvent_t> done(groups);
        for (auto &e : done) SODECL_CUDA_TRY(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        EventGuard done_guard{done.data(), static_cast<int>(groups)};
        std::vector<int64_t> first(groups + 1);
        for (int64_t g = 0; g <= groups; ++g) first[g] = ctx->nchunks * g / groups;
        double *d_rec = static_cast<double *>(ctx->d_records);
        a.records = d_rec;
        for (int64_t g = 0; g < groups; ++g) {
            a.chunk_begin = static_cast<int>(first[g]);
            a.chunk_end = static_cast<int>(first[g + 1]);
            a.write_final = (g == groups - 1) ? 1 : 0;
            if ((rc = launch(ctx, a, ctx->stream)) != SODECL_OK) return rc;
            SODECL_CUDA_TRY(ctx, cudaEventRecord(done[g], ctx->stream));
        }
        SODECL_CUDA_TRY(ctx, cudaEventRecord(t_kernels, ctx->stream));
        for (int64_t g = 0; g < groups; ++g) {
            const int64_t r0 = first[g];
            const int64_t r1 = (g == groups - 1) ? nrec : first[g + 1];
            SODECL_CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->copy_stream, done[g], 0));
            SODECL_CUDA_TRY(ctx, cudaMemcpyAsync(out + r0 * rec_elems, d_rec + r0 * rec_elems,
                                                 static_cast<size_t>((r1 - r0) * rec_elems) * sizeof(double),
                                                 cudaMemcpyDeviceToHost, ctx->copy_stream));
        }
        SODECL_CUDA_TRY(ctx, cudaEventRecord(t_end, ctx->copy_stream));
    }
    SODECL_CUDA_TRY(ctx, cudaEventSynchronize(t_end));
    SODECL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    float kms = 0.f, tms = 0.f;
    SODECL_CUDA_TRY(ctx, cudaEventElapsedTime(&kms, t_begin, t_kernels));
    SODECL_CUDA_TRY(ctx, cudaEventElapsedTime(&tms, t_begin, t_end));
    ctx->last_kernel_ms = kms;
    ctx->last_total_ms = tms;
    return SODECL_OK;
}

int sodecl_cuda_last_run_ms(const sodecl_ctx *ctx, double *kernel_ms, double *total_ms)
{
    if (!ctx) return SODECL_ERR_INVALID_ARG;
    if (kernel_ms) *kernel_ms = ctx->last_kernel_ms;
    if (total_ms) *total_ms = ctx->last_total_ms;
    return SODECL_OK;
}

int sodecl_cuda_download_state(sodecl_ctx *ctx, double *t, double *y, double *counters)
{
    if (!ctx) return SODECL_ERR_INVALID_ARG;
    if (!ctx->uploaded) return ctx->fail(SODECL_ERR_STATE, "no state on the device");
    DeviceScope dev(ctx->cfg.device);
    const size_t n = static_cast<size_t>(ctx->cfg.list_size), neq = ctx->cfg.num_equat;
    if (t) SODECL_CUDA_TRY(ctx, cudaMemcpyAsync(t, ctx->d_t, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (y) SODECL_CUDA_TRY(ctx, cudaMemcpyAsync(y, ctx->d_y, n * neq * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (counters)
        SODECL_CUDA_TRY(ctx, cudaMemcpyAsync(counters, ctx->d_cnt, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    SODECL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return SODECL_OK;
}

int sodecl_cuda_status(sodecl_ctx *ctx, int64_t *newton_passes, int32_t *flags)
{
    if (!ctx) return SODECL_ERR_INVALID_ARG;
    if (!ctx->uploaded) return ctx->fail(SODECL_ERR_STATE, "no state on the device");
    DeviceScope dev(ctx->cfg.device);
    const size_t n = static_cast<size_t>(ctx->cfg.list_size);
    if (newton_passes)
        SODECL_CUDA_TRY(ctx, cudaMemcpyAsync(newton_passes, ctx->d_passes, n * sizeof(long long), cudaMemcpyDeviceToHost, ctx->stream));
    if (flags) SODECL_CUDA_TRY(ctx, cudaMemcpyAsync(flags, ctx->d_flags, n * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    SODECL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return SODECL_OK;
}

int sodecl_cuda_launch(sodecl_ctx *ctx, const sodecl_launch *l, void *stream)
{
    if (!ctx) return SODECL_ERR_INVALID_ARG;
    if (!l || !l->t || !l->y || (!l->params && ctx->cfg.num_params > 0))
        return ctx->fail(SODECL_ERR_INVALID_ARG, "launch: t, y and params must be device pointers");
    if (ctx->cfg.solver == SODECL_STOCHASTIC_EULER && !l->counters)
        return ctx->fail(SODECL_ERR_INVALID_ARG, "launch: the stochastic solver needs counters");
    if (l->n < 0 || l->chunk_begin < 0 || l->chunk_end < l->chunk_begin || l->rec_first > l->chunk_begin)
        return ctx->fail(SODECL_ERR_INVALID_ARG, "launch: bad orbit or interval range");
    if (l->records && (l->rec_stride < l->rec_col0 + l->n))
        return ctx->fail(SODECL_ERR_INVALID_ARG, "launch: record rows narrower than the orbit range");
    DeviceScope dev(ctx->cfg.device);
    int rc = ensure_gpu(ctx);
    if (rc != SODECL_OK) return rc;
    DeviceArgs a{};
    a.t = l->t;
    a.y = l->y;
    a.p = l->params;
    a.counters = l->counters;
    a.records = l->records;
    a.n = l->n;
    a.orbit_offset = l->orbit_offset;
    a.rec_stride = l->rec_stride;
    a.rec_col0 = l->rec_col0;
    a.chunk_begin = l->chunk_begin;
    a.chunk_end = l->chunk_end;
    a.rec_first = l->rec_first;
    a.write_final = l->write_final;
    a.newton_passes = reinterpret_cast<long long *>(l->newton_passes);
    a.flags = reinterpret_cast<int *>(l->flags);
    return launch(ctx, a, static_cast<cudaStream_t>(stream));
}

int sodecl_cuda_kernel_info(sodecl_ctx *ctx, int *regs, int *local_bytes, int *max_threads)
{
    if (!ctx) return SODECL_ERR_INVALID_ARG;
    DeviceScope dev(ctx->cfg.device);
    int rc = ensure_gpu(ctx);
    if (rc != SODECL_OK) return rc;
    cudaFuncAttributes fa{};
    SODECL_CUDA_TRY(ctx, cudaFuncGetAttributes(&fa, reinterpret_cast<const void *>(ctx->kernel)));
    if (regs) *regs = fa.numRegs;
    if (local_bytes) *local_bytes = static_cast<int>(fa.localSizeBytes);
    if (max_threads) *max_threads = fa.maxThreadsPerBlock;
    return SODECL_OK;
}

size_t sodecl_cuda_last_error(const sodecl_ctx *ctx, char *buf, size_t n)
{
    return copy_string(ctx ? ctx->error : std::string("null context"), buf, n);
}

size_t sodecl_cuda_build_log(const sodecl_ctx *ctx, char *buf, size_t n)
{
    return copy_string(ctx && ctx->prog ? ctx->prog->log : std::string(), buf, n);
}

size_t sodecl_cuda_program_source(const sodecl_ctx *ctx, char *buf, size_t n)
{
    return copy_string(ctx && ctx->prog ? ctx->prog->source : std::string(), buf, n);
}

void sodecl_cuda_destroy(sodecl_ctx *ctx)
{
    if (!ctx) return;
    if (ctx->gpu_ready || ctx->uploaded) {
        DeviceScope dev(ctx->cfg.device);
        if (ctx->stream) cudaStreamSynchronize(ctx->stream);
        if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
        free_buffers(ctx);
        if (ctx->stream) cudaStreamDestroy(ctx->stream);
        if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
        if (ctx->lib) cudaLibraryUnload(ctx->lib);
    }
    delete ctx;
}

}  // extern "C"
