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
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <random>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "device_memory.hpp"
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

// Must match struct sodecl_adjoint_args in device/adjoint.cuh field for field.
struct AdjointArgs {
    const double *t0;
    const double *y0;
    const double *p;
    const double *targets;
    double *loss;
    double *grad_p;
    double *grad_y0;
    double *ckpt;
    double *ckpt_t;
    double *seg;
    int *flags;
    long long n;
    int nchunks;
    int ckpt_every;
};

constexpr int kDefaultBlock = 128;
constexpr int kMaxCopyGroups = 8;
// Host output in pageable memory: launch groups of about this many record
// intervals each (at least kMinPageableGroups groups), so that copying out
// starts early and keeps pace with the launches.
constexpr int kMinPageableGroups = 16;

// Pinned staging for copies into pageable host memory.  A copy from the
// device into pageable memory goes through the driver's own small staging
// buffer on the calling thread.  Instead, kStageWorkers host threads each
// bring pieces of the records into two pinned slots of their own (one in
// flight while the other is copied into the destination), so the copies run
// on several streams and the page faults of a fresh destination are taken
// by several threads.  The slots are pinned once per process and shared by
// every context; one run at a time copies through them.
constexpr int kStageWorkers = 8;
constexpr size_t kStageSlotBytes = size_t(8) << 20;

struct StagingPool {
    std::mutex in_use;
    std::vector<void *> slots;  // 2 per worker, kStageSlotBytes each
};

StagingPool &staging_pool()
{
    static StagingPool pool;
    return pool;
}

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

    // discrete adjoint: its own program and scratch (checkpoints, segments)
    std::shared_ptr<const Program> adj_prog;
    int adj_min_blocks = -1;
    int adj_block = 0;
    cudaLibrary_t adj_lib = nullptr;
    cudaKernel_t adj_kernel = nullptr;
    int adj_tape = 0;
    int adj_mode = -1;
    bool adj_fast_div = false;
    bool adj_gradient = false;
    void *adj_scratch = nullptr;
    size_t adj_scratch_bytes = 0;

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

// One record buffer per device outlives the context that allocated it: the
// reference's callers make a new manager per call (sodecl.py), and freeing
// and allocating a multi-GB buffer every call was measured to take from a
// few to several hundred milliseconds.  A destroyed context leaves its record
// buffer here (the larger of two is kept), and the next context on the
// device takes it if it is large enough.  sodecl_cuda_release_cached and
// sodecl_cuda_release_scratch free it.
constexpr int kCacheDevices = 64;
struct RecordCache {
    std::mutex m;
    void *ptr[kCacheDevices] = {};
    size_t bytes[kCacheDevices] = {};
};

RecordCache &record_cache()
{
    static RecordCache *cache = new RecordCache();  // never destroyed: no teardown-order hazards
    return *cache;
}

// Takes the cached buffer of `device` if it holds `need` bytes.
void *take_cached_records(int device, size_t need, size_t *bytes)
{
    if (device < 0 || device >= kCacheDevices) return nullptr;
    RecordCache &c = record_cache();
    std::lock_guard<std::mutex> lock(c.m);
    if (!c.ptr[device] || c.bytes[device] < need) return nullptr;
    void *p = c.ptr[device];
    *bytes = c.bytes[device];
    c.ptr[device] = nullptr;
    c.bytes[device] = 0;
    return p;
}

// Leaves an idle buffer of `device` (the current device) for the next
// context, keeping the larger of it and the one already cached.
void give_cached_records(int device, void *p, size_t bytes)
{
    if (!p) return;
    if (device < 0 || device >= kCacheDevices) {
        cudaFree(p);
        return;
    }
    RecordCache &c = record_cache();
    void *drop = p;
    {
        std::lock_guard<std::mutex> lock(c.m);
        if (!c.ptr[device] || c.bytes[device] < bytes) {
            drop = c.ptr[device];
            c.ptr[device] = p;
            c.bytes[device] = bytes;
        }
    }
    if (drop) cudaFree(drop);
}

void release_cached_records(int device)
{
    if (device < 0 || device >= kCacheDevices) return;
    RecordCache &c = record_cache();
    void *drop = nullptr;
    {
        std::lock_guard<std::mutex> lock(c.m);
        drop = c.ptr[device];
        c.ptr[device] = nullptr;
        c.bytes[device] = 0;
    }
    if (drop) cudaFree(drop);
}

void free_buffers(sodecl_ctx *ctx)
{
    cudaFree(ctx->d_t);
    cudaFree(ctx->d_y);
    cudaFree(ctx->d_p);
    cudaFree(ctx->d_cnt);
    cudaFree(ctx->d_passes);
    cudaFree(ctx->d_flags);
    give_cached_records(ctx->cfg.device, ctx->d_records, ctx->d_records_bytes);
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

int lanes_of(const sodecl_cfg &c) { return c.lanes_per_orbit > 1 ? c.lanes_per_orbit : 1; }

// A piece of the record buffer: `count` doubles at element offset `off`,
// ready once launch group `group` has finished.
struct Piece {
    int64_t off;
    int64_t count;
    int group;
};

// Copies the pieces of d_rec into the pageable `out` through the pinned
// staging pool (kStageWorkers threads, two slots each).  Worker w takes
// pieces w, w + W, w + 2W, ... (so each worker meets them in the order the
// launches finish them); for each it queues the copy of its next piece into
// its other slot before copying the current one out of its slot.  `pool`
// is locked by the caller.  Returns cudaSuccess or the first error.
cudaError_t staged_copy(int device, double *out, const double *d_rec, const std::vector<Piece> &pieces,
                        const std::vector<cudaEvent_t> &done, StagingPool &pool)
{
    const int nworkers = static_cast<int>(pool.slots.size() / 2);
    std::atomic<int> first_error{static_cast<int>(cudaSuccess)};
    auto note = [&](cudaError_t e) {
        if (e != cudaSuccess) {
            int expected = static_cast<int>(cudaSuccess);
            first_error.compare_exchange_strong(expected, static_cast<int>(e));
        }
        return e == cudaSuccess;
    };
    auto work = [&](int w) {
        if (!note(cudaSetDevice(device))) return;
        cudaStream_t st = nullptr;
        cudaEvent_t ev[2] = {nullptr, nullptr};
        if (!note(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking))) return;
        bool ok = note(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming)) &&
                  note(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
        auto issue = [&](size_t j, int slot) {
            const Piece &pc = pieces[j];
            return note(cudaStreamWaitEvent(st, done[pc.group], 0)) &&
                   note(cudaMemcpyAsync(pool.slots[2 * w + slot], d_rec + pc.off,
                                        static_cast<size_t>(pc.count) * sizeof(double), cudaMemcpyDeviceToHost, st)) &&
                   note(cudaEventRecord(ev[slot], st));
        };
        size_t j = static_cast<size_t>(w);
        if (ok && j < pieces.size()) ok = issue(j, 0);
        for (int k = 0; ok && j < pieces.size(); ++k, j += nworkers) {
            const size_t next = j + nworkers;
            if (next < pieces.size() && !issue(next, (k + 1) & 1)) break;
            if (!note(cudaEventSynchronize(ev[k & 1]))) break;
            if (first_error.load() != static_cast<int>(cudaSuccess)) break;
            std::memcpy(out + pieces[j].off, pool.slots[2 * w + (k & 1)],
                        static_cast<size_t>(pieces[j].count) * sizeof(double));
        }
        cudaStreamSynchronize(st);
        for (auto e : ev)
            if (e) cudaEventDestroy(e);
        cudaStreamDestroy(st);
    };
    std::vector<std::thread> threads;
    threads.reserve(nworkers);
    for (int w = 0; w < nworkers; ++w) threads.emplace_back(work, w);
    for (auto &t : threads) t.join();
    return static_cast<cudaError_t>(first_error.load());
}

// Pins the staging pool's slots on first use; false if pinned memory is not
// available (the caller then copies without staging).
bool staging_ready(StagingPool &pool)
{
    if (!pool.slots.empty()) return true;
    const unsigned hw = std::max(2u, std::thread::hardware_concurrency());
    const int workers = std::max(1, std::min<int>(kStageWorkers, static_cast<int>(hw / 2)));
    for (int k = 0; k < 2 * workers; ++k) {
        void *p = nullptr;
        if (cudaHostAlloc(&p, kStageSlotBytes, cudaHostAllocPortable) != cudaSuccess) {
            cudaGetLastError();
            for (void *q : pool.slots) cudaFreeHost(q);
            pool.slots.clear();
            return false;
        }
        pool.slots.push_back(p);
    }
    return true;
}

// Whether the system file has the per-row functions lanes per orbit need
// with this solver.
bool lanes_supported(const sodecl_b200::SystemTraits &t, int solver)
{
    if (!t.has_row || solver == SODECL_DORMAND_PRINCE) return false;
    if (solver == SODECL_STOCHASTIC_EULER) return t.has_stoch_row;
    if (solver == SODECL_IMPLICIT_EULER || solver == SODECL_IMPLICIT_MIDPOINT) return t.has_jac_band;
    return true;
}

// Shared memory cap of one block of the lanes-per-orbit kernel (the default
// dynamic shared memory limit, no opt-in needed).
constexpr size_t kLanesSharedCap = 48 * 1024;

// Launch geometry of the configured kernel for n orbits: threads per block,
// blocks, dynamic shared memory.  One thread per orbit: the block size as
// configured.  Lanes per orbit: a multiple of 32 threads, reduced until the
// block's orbit slots fit kLanesSharedCap.
struct Geometry {
    int block = 0;
    long long grid = 0;
    size_t shared = 0;
};

Geometry geometry(const sodecl_cfg &c, int64_t n)
{
    Geometry g;
    int block = c.local_group_size > 0 ? c.local_group_size : kDefaultBlock;
    const int lanes = lanes_of(c);
    if (lanes == 1) {
        g.block = block;
        g.grid = (n + block - 1) / block;
        return g;
    }
    block = std::max(32, (block + 31) / 32 * 32);
    ProgramSpec spec;
    spec.solver = c.solver;
    spec.num_equat = c.num_equat;
    spec.num_params = c.num_params;
    spec.num_noi = c.num_noi;
    const size_t slot = static_cast<size_t>(sodecl_b200::lanes_slot_words(spec)) *
                        (c.precision == SODECL_FP32 ? sizeof(float) : sizeof(double));
    while (block > 32 && static_cast<size_t>(block / lanes) * slot > kLanesSharedCap) block -= 32;
    g.block = block;
    g.grid = (n * lanes + block - 1) / block;
    g.shared = static_cast<size_t>(block / lanes) * slot;
    return g;
}

int launch_kernel(sodecl_ctx *ctx, cudaKernel_t kernel, const sodecl_cfg &c, const DeviceArgs &a, cudaStream_t stream)
{
    if (a.n <= 0) return SODECL_OK;
    Geometry g = geometry(c, a.n);
    if (lanes_of(c) == 1 && (c.solver == SODECL_IMPLICIT_EULER || c.solver == SODECL_IMPLICIT_MIDPOINT ||
                             c.solver == SODECL_DORMAND_PRINCE)) {
        // the implicit and adaptive kernels' warps share out ranges of orbits
        // among their lanes: give every lane the same number of orbits, the
        // fewest that fit the threads resident at once, and launch just the
        // blocks for that
        int per_sm = 0, dev = 0, sms = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, reinterpret_cast<const void *>(kernel), g.block,
                                                          0) != cudaSuccess ||
            cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
            cudaGetLastError();
            per_sm = sms = 0;
        }
        const int64_t resident = static_cast<int64_t>(per_sm) * sms * g.block;
        if (resident > 0 && a.n > resident) {
            const int64_t per_lane = (a.n + resident - 1) / resident;
            g.grid = (a.n + per_lane * g.block - 1) / (per_lane * g.block);
        }
    }
    if (g.grid > 0x7fffffffLL) return ctx->fail(SODECL_ERR_INVALID_ARG, "too many orbits for one launch");
    if (g.shared > kLanesSharedCap)
        return ctx->fail(SODECL_ERR_UNSUPPORTED, "one orbit's state, parameters and noise exceed the shared memory of a "
                                                 "block: use one thread per orbit");
    void *args[] = {const_cast<DeviceArgs *>(&a)};
    SODECL_CUDA_TRY(ctx, cudaLaunchKernel(reinterpret_cast<const void *>(kernel), dim3(static_cast<unsigned>(g.grid)),
                                          dim3(g.block), args, g.shared, stream));
    return SODECL_OK;
}

int launch(sodecl_ctx *ctx, const DeviceArgs &a, cudaStream_t stream)
{
    return launch_kernel(ctx, ctx->kernel, ctx->cfg, a, stream);
}

// SODECL_DIV_DEFAULT: the reciprocal form in FP64 (faster on converging and
// diverged orbits alike), IEEE division in FP32 (the reciprocal form gains
// only on diverged orbits there; the tuner times both) and for the adaptive
// solver, whose error test divides by a new scale every attempt: there the
// wrapper's registers cost more than it saves (2^20 oculomotor orbits over
// 0.2 time units: 241 against 199 ms at 128 registers)
bool reciprocal_division(const sodecl_cfg &c)
{
    return c.division == SODECL_DIV_RECIPROCAL ||
           (c.division == SODECL_DIV_DEFAULT && c.precision == SODECL_FP64 && c.solver != SODECL_DORMAND_PRINCE);
}

ProgramSpec make_spec(const sodecl_cfg &c)
{
    ProgramSpec spec;
    spec.solver = c.solver;
    spec.num_equat = c.num_equat;
    spec.num_params = c.num_params;
    spec.num_noi = c.num_noi;
    spec.list_size = c.list_size;
    spec.kernel_steps = c.kernel_steps;
    spec.dt = c.dt;
    spec.fp32 = c.precision == SODECL_FP32;
    spec.fmad = c.fmad != 0;
    spec.record_f32 = c.record_f32 != 0;
    spec.newton_tol = c.newton_tol;
    spec.newton_max_iter = c.newton_max_iter;
    // lanes per orbit round the block up to whole warps
    const int block = c.local_group_size > 0 ? c.local_group_size : kDefaultBlock;
    spec.block_max = std::max(256, c.lanes_per_orbit > 1 ? (block + 31) / 32 * 32 : block);
    spec.min_blocks = c.min_blocks_per_sm;
    // implicit solvers, one thread per orbit: by default at most 128 registers
    // a thread (four blocks of 128 threads on an SM); above that the Newton
    // pass's hoisted terms took more registers than the occupancy they cost
    // The adaptive solver's kernel likewise: the oculomotor model at 2^20
    // orbits over 0.2 time units took 199 ms at 128 registers against 212 ms
    // uncapped (202 registers).
    if (spec.min_blocks == 0 && lanes_of(c) == 1 &&
        (c.solver == SODECL_IMPLICIT_EULER || c.solver == SODECL_IMPLICIT_MIDPOINT ||
         c.solver == SODECL_DORMAND_PRINCE))
        spec.min_blocks = std::max(1, 65536 / (spec.block_max * 128));
    // FP64 RK4 on small systems, one thread per orbit: by default at most 85
    // registers a thread (three blocks of 256).  Measured on the oculomotor
    // model at 2^20 orbits x 10^4 steps: 397 ms against 426 ms with no cap
    // and 411 ms at 64 registers (the reference's system file; the package's
    // 362 / 381 / 371 ms).
    if (spec.min_blocks == 0 && lanes_of(c) == 1 && c.solver == SODECL_RUNGE_KUTTA && !spec.fp32 &&
        c.num_equat <= 8)
        spec.min_blocks = std::max(1, 65536 / (spec.block_max * 85));
    spec.fast_div = reciprocal_division(c);
    spec.lanes = lanes_of(c);
    // paired stores need the pair's two threads at the same store with orbits
    // 2k and 2k+1: the one-thread kernel of the explicit and stochastic
    // solvers (the implicit and adaptive kernels store per lane, whenever that
    // lane's orbit reaches a record)
    spec.pair_stores = c.record_store == SODECL_STORE_PAIRS && spec.lanes == 1 &&
                       (c.solver == SODECL_EULER || c.solver == SODECL_RUNGE_KUTTA ||
                        c.solver == SODECL_STOCHASTIC_EULER);
    spec.rtol = c.rtol;
    spec.atol = c.atol;
    spec.max_steps = c.max_steps;
    return spec;
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
    cfg->division = SODECL_DIV_DEFAULT;
    cfg->rtol = 1e-6;
    cfg->atol = 1e-9;
    cfg->max_steps = 100000;
    cfg->record_store = SODECL_STORE_DIRECT;
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

int sodecl_cuda_device_describe(int device, char *buf, size_t n, int *major, int *minor)
{
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        cudaGetLastError();
        return SODECL_ERR_NO_DEVICE;
    }
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
        cudaGetLastError();
        return SODECL_ERR_CUDA;
    }
    if (buf && n > 0) {
        std::strncpy(buf, prop.name, n - 1);
        buf[n - 1] = '\0';
    }
    if (major) *major = prop.major;
    if (minor) *minor = prop.minor;
    return SODECL_OK;
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
    if (c.solver < 0 || c.solver > SODECL_DORMAND_PRINCE) return SODECL_ERR_INVALID_ARG;
    if (c.solver == SODECL_DORMAND_PRINCE &&
        (!(c.rtol > 0) || !std::isfinite(c.rtol) || !(c.atol > 0) || !std::isfinite(c.atol) || c.max_steps < 1 ||
         c.lanes_per_orbit > 1))
        return SODECL_ERR_INVALID_ARG;
    if (c.num_equat < 1 || c.num_params < 0 || c.num_noi < 0 || c.list_size < 1) return SODECL_ERR_INVALID_ARG;
    if (!(c.dt > 0) || !std::isfinite(c.dt) || !(c.int_time >= 0) || !std::isfinite(c.int_time)) return SODECL_ERR_INVALID_ARG;
    if (c.kernel_steps < 1) return SODECL_ERR_INVALID_ARG;
    if (c.solver == SODECL_STOCHASTIC_EULER && c.num_noi < 1) return SODECL_ERR_INVALID_ARG;
    if (c.precision != SODECL_FP64 && c.precision != SODECL_FP32) return SODECL_ERR_INVALID_ARG;
    if (c.local_group_size < 0 || c.local_group_size > 1024) return SODECL_ERR_INVALID_ARG;
    if (c.newton_tol < 0 || !std::isfinite(c.newton_tol) || c.newton_max_iter < 0) return SODECL_ERR_INVALID_ARG;
    if (c.min_blocks_per_sm < 0 || c.min_blocks_per_sm > 32) return SODECL_ERR_INVALID_ARG;
    if (c.division != SODECL_DIV_RECIPROCAL && c.division != SODECL_DIV_IEEE && c.division != SODECL_DIV_DEFAULT)
        return SODECL_ERR_INVALID_ARG;
    if (c.lanes_per_orbit < 0 || c.lanes_per_orbit > 32 || (c.lanes_per_orbit & (c.lanes_per_orbit - 1)) != 0)
        return SODECL_ERR_INVALID_ARG;
    if (c.record_store != SODECL_STORE_DIRECT && c.record_store != SODECL_STORE_PAIRS) return SODECL_ERR_INVALID_ARG;
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
    if (lanes_of(ctx->cfg) > 1) {
        if (!lanes_supported(traits, solver))
            return ctx->fail(SODECL_ERR_UNSUPPORTED, "lanes per orbit need sode_system_row(...) in the system file, "
                                                     "and sode_system_stoch_row(...) for the stochastic solver or "
                                                     "calc_jacobian_band(...) for the implicit ones");
        if (geometry(ctx->cfg, 1).shared > kLanesSharedCap)
            return ctx->fail(SODECL_ERR_UNSUPPORTED, "lanes per orbit: one orbit does not fit a block's shared memory");
    }
    ProgramSpec spec = make_spec(ctx->cfg);
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
    if (ctx->cfg.solver == SODECL_DORMAND_PRINCE && counters) {
        // each orbit's next step size
        SODECL_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->d_cnt, counters, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    } else if (ctx->cfg.solver == SODECL_STOCHASTIC_EULER) {
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
    bool device_out = false, pageable_out = false;
    if (out) {
        if (cudaPointerGetAttributes(&attr, out) != cudaSuccess) {
            cudaGetLastError();
            attr.type = cudaMemoryTypeUnregistered;
        }
        device_out = attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
        pageable_out = attr.type == cudaMemoryTypeUnregistered;
    }
    const auto wall0 = std::chrono::steady_clock::now();
    bool staged = false;

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
            give_cached_records(ctx->cfg.device, ctx->d_records, ctx->d_records_bytes);
            ctx->d_records = take_cached_records(ctx->cfg.device, need, &ctx->d_records_bytes);
            if (!ctx->d_records) {
                ctx->d_records_bytes = 0;
                SODECL_CUDA_TRY(ctx, cudaMalloc(&ctx->d_records, need));
                ctx->d_records_bytes = need;
            }
        }
        // Pinned output: launch groups of halving size (half the record
        // intervals, a quarter, ...; the last takes the rest): each group's
        // records are copied out on the second stream while later groups
        // compute, and only the last, small group's copy is left exposed at
        // the end.  Pageable output: equal groups of at most 1/16 of the
        // intervals, staged through pinned memory by host threads, which start
        // on the first group's records and keep pace with the launches.
        std::unique_lock<std::mutex> pool_lock;
        StagingPool &pool = staging_pool();
        if (pageable_out) {
            pool_lock = std::unique_lock<std::mutex>(pool.in_use);
            staged = staging_ready(pool);
            if (!staged) pool_lock.unlock();
        }
        std::vector<int64_t> first{0};
        if (staged) {
            // equal groups while more than two remain, then halving ones, so
            // that the records copied after the last launch are few
            const int64_t per = std::max<int64_t>(1, (ctx->nchunks + kMinPageableGroups - 1) / kMinPageableGroups);
            while (first.back() < ctx->nchunks) {
                const int64_t rest = ctx->nchunks - first.back();
                first.push_back(first.back() + (rest > 2 * per ? per : std::max<int64_t>(1, (rest + 1) / 2)));
            }
        } else {
            while (first.back() < ctx->nchunks) {
                const int64_t rest = ctx->nchunks - first.back();
                const bool last = static_cast<int64_t>(first.size()) == kMaxCopyGroups;
                first.push_back(first.back() + (last ? rest : std::max<int64_t>(1, (rest + 1) / 2)));
            }
        }
        if (first.size() == 1) first.push_back(0);  // no interval: one launch stores the final record
        const int64_t groups = static_cast<int64_t>(first.size()) - 1;
        std::vector<cudaEvent_t> done(groups);
        for (auto &e : done) SODECL_CUDA_TRY(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        EventGuard done_guard{done.data(), static_cast<int>(groups)};
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
        if (staged) {
            // pieces of at most one slot, in the order the groups finish
            const int64_t slot_elems = static_cast<int64_t>(kStageSlotBytes / sizeof(double));
            std::vector<Piece> pieces;
            for (int64_t g = 0; g < groups; ++g) {
                const int64_t e0 = first[g] * rec_elems;
                const int64_t e1 = ((g == groups - 1) ? nrec : first[g + 1]) * rec_elems;
                for (int64_t e = e0; e < e1; e += slot_elems)
                    pieces.push_back(Piece{e, std::min(slot_elems, e1 - e), static_cast<int>(g)});
            }
            const cudaError_t e = staged_copy(ctx->cfg.device, out, d_rec, pieces, done, pool);
            if (e != cudaSuccess) {
                cudaStreamSynchronize(ctx->stream);
                return cuda_fail(ctx, e, "staged record copy");
            }
            pool_lock.unlock();
            SODECL_CUDA_TRY(ctx, cudaEventRecord(t_end, ctx->stream));
        } else {
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
    }
    SODECL_CUDA_TRY(ctx, cudaEventSynchronize(t_end));
    SODECL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    float kms = 0.f, tms = 0.f;
    SODECL_CUDA_TRY(ctx, cudaEventElapsedTime(&kms, t_begin, t_kernels));
    SODECL_CUDA_TRY(ctx, cudaEventElapsedTime(&tms, t_begin, t_end));
    ctx->last_kernel_ms = kms;
    // the staged copy ends on the host: its total is the wall time
    ctx->last_total_ms =
        staged ? std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - wall0).count() : tms;
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
    for (const void *p : {static_cast<const void *>(l->t), static_cast<const void *>(l->y),
                          static_cast<const void *>(l->params), static_cast<const void *>(l->counters),
                          static_cast<const void *>(l->records), static_cast<const void *>(l->newton_passes),
                          static_cast<const void *>(l->flags)})
        if (!sodecl_b200::kernel_can_access(p, ctx->cfg.device))
            return ctx->fail(SODECL_ERR_INVALID_ARG, "launch: a buffer is not memory this device can access "
                                                     "(device, managed or pinned host memory)");
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

int sodecl_cuda_autotune(sodecl_ctx *ctx, int64_t sample_orbits, int32_t sample_steps, int32_t *block,
                         int32_t *min_blocks, int32_t *division, int32_t *lanes, double *best_ms)
{
    if (!ctx) return SODECL_ERR_INVALID_ARG;
    if (!ctx->uploaded) return ctx->fail(SODECL_ERR_STATE, "upload the orbits first: the tuner samples them");
    if (sample_orbits < 1 || sample_steps < 1) return ctx->fail(SODECL_ERR_INVALID_ARG, "empty sample");
    DeviceScope dev(ctx->cfg.device);
    const int64_t n = std::min<int64_t>(sample_orbits, ctx->cfg.list_size);
    const size_t neq = ctx->cfg.num_equat, npar = std::max(1, ctx->cfg.num_params);
    const int chunks = std::max<int>(1, (sample_steps + ctx->cfg.kernel_steps - 1) / ctx->cfg.kernel_steps);
    // scratch copies of the sample, so the real state does not advance
    double *t = nullptr, *y = nullptr, *cnt = nullptr;
    SODECL_CUDA_TRY(ctx, cudaMalloc(&t, n * sizeof(double)));
    struct Free {
        void *p[3];
        ~Free() { for (void *q : p) cudaFree(q); }
    } guard{{t, nullptr, nullptr}};
    SODECL_CUDA_TRY(ctx, cudaMalloc(&y, n * neq * sizeof(double)));
    guard.p[1] = y;
    SODECL_CUDA_TRY(ctx, cudaMalloc(&cnt, n * sizeof(double)));
    guard.p[2] = cnt;
    (void)npar;
    // the trials store their records too, as a run does (so the store form is
    // timed); without room for them they run without
    void *rec = nullptr;
    if (cudaMalloc(&rec, static_cast<size_t>(chunks) * neq * n * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        rec = nullptr;
    }
    struct FreeRec {
        void *p;
        ~FreeRec() { cudaFree(p); }
    } rec_guard{rec};

    struct Cand {
        int block, min_blocks, division, lanes, store;
    };
    std::vector<Cand> cands = {{128, 0, SODECL_DIV_IEEE, 1, SODECL_STORE_DIRECT},
                               {128, 4, SODECL_DIV_IEEE, 1, SODECL_STORE_DIRECT},
                               {256, 3, SODECL_DIV_IEEE, 1, SODECL_STORE_DIRECT},
                               {64, 0, SODECL_DIV_IEEE, 1, SODECL_STORE_DIRECT}};
    cands.push_back({128, 0, SODECL_DIV_RECIPROCAL, 1, SODECL_STORE_DIRECT});
    cands.push_back({128, 4, SODECL_DIV_RECIPROCAL, 1, SODECL_STORE_DIRECT});
    if (ctx->cfg.precision == SODECL_FP64) cands.push_back({128, 3, SODECL_DIV_RECIPROCAL, 1, SODECL_STORE_DIRECT});
    // lanes per orbit: up to the first power of two >= the equations
    const auto traits = sodecl_b200::inspect_system(ctx->system_src);
    const int solver = ctx->cfg.solver;
    // implicit and adaptive solvers and FP64 RK4 on small systems run under a
    // register cap by default (min_blocks 0); 1 lifts it
    if (solver == SODECL_IMPLICIT_EULER || solver == SODECL_IMPLICIT_MIDPOINT || solver == SODECL_DORMAND_PRINCE ||
        (solver == SODECL_RUNGE_KUTTA && ctx->cfg.precision == SODECL_FP64 && ctx->cfg.num_equat <= 8))
        cands.push_back({128, 1,
                         ctx->cfg.precision == SODECL_FP64 && solver != SODECL_DORMAND_PRINCE ? SODECL_DIV_RECIPROCAL
                                                                                             : SODECL_DIV_IEEE,
                         1, SODECL_STORE_DIRECT});
    const bool row_ok = lanes_supported(traits, solver);
    if (row_ok) {
        for (int l = 2; l <= 32 && l / 2 < ctx->cfg.num_equat; l *= 2) {
            if (l < 4) continue;
            cands.push_back({128, 0, SODECL_DIV_IEEE, l, SODECL_STORE_DIRECT});
            cands.push_back({256, 0, SODECL_DIV_IEEE, l, SODECL_STORE_DIRECT});
        }
    }
    const sodecl_cfg saved = ctx->cfg;
    auto saved_prog = ctx->prog;
    double best = 1e300;
    Cand pick = {saved.local_group_size > 0 ? saved.local_group_size : kDefaultBlock, saved.min_blocks_per_sm,
                 saved.division, lanes_of(saved), saved.record_store};
    cudaEvent_t e0, e1;
    SODECL_CUDA_TRY(ctx, cudaEventCreate(&e0));
    SODECL_CUDA_TRY(ctx, cudaEventCreate(&e1));
    int rc = SODECL_OK;
    // one candidate's time (the second of two launches); false if it does
    // not build or load, or fell back to another division mode
    auto trial = [&](const Cand &c, float &ms) -> bool {
        sodecl_cfg cfg = saved;
        cfg.local_group_size = c.block;
        cfg.min_blocks_per_sm = c.min_blocks;
        cfg.division = c.division;
        cfg.lanes_per_orbit = c.lanes;
        cfg.record_store = c.store;
        if (c.lanes > 1 && geometry(cfg, 1).shared > kLanesSharedCap) return false;
        std::shared_ptr<const Program> prog;
        try {
            prog = sodecl_b200::build(make_spec(cfg), ctx->system_src);
        } catch (const std::exception &ex) {
            return false;
        }
        if (c.division == SODECL_DIV_RECIPROCAL && !prog->fast_div) return false;  // fell back to IEEE
        cudaLibrary_t lib = nullptr;
        cudaKernel_t kern = nullptr;
        if (cudaLibraryLoadData(&lib, prog->cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0) != cudaSuccess ||
            cudaLibraryGetKernel(&kern, lib, prog->kernel_name.c_str()) != cudaSuccess) {
            cudaGetLastError();
            if (lib) cudaLibraryUnload(lib);
            return false;
        }
        for (int rep = 0; rep < 2 && rc == SODECL_OK; ++rep) {
            cudaMemcpyAsync(t, ctx->d_t, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream);
            cudaMemcpyAsync(y, ctx->d_y, n * neq * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream);
            cudaMemcpyAsync(cnt, ctx->d_cnt, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream);
            DeviceArgs a{};
            a.t = t;
            a.y = y;
            a.p = ctx->d_p;
            a.counters = cnt;
            a.n = n;
            a.records = rec;
            a.rec_stride = n;
            a.chunk_begin = 0;
            a.chunk_end = chunks;
            cudaEventRecord(e0, ctx->stream);
            rc = launch_kernel(ctx, kern, cfg, a, ctx->stream);
            cudaEventRecord(e1, ctx->stream);
            if (rc != SODECL_OK) break;
            const cudaError_t se = cudaEventSynchronize(e1);
            if (se != cudaSuccess) {
                rc = cuda_fail(ctx, se, "autotune launch");
                break;
            }
            cudaEventElapsedTime(&ms, e0, e1);
        }
        cudaLibraryUnload(lib);
        return rc == SODECL_OK;
    };
    for (const Cand &c : cands) {
        float ms = 0.f;
        if (!trial(c, ms)) {
            if (rc != SODECL_OK) break;
            continue;
        }
        if (ms < best) {
            best = ms;
            pick = c;
        }
    }
    // the winner with paired record stores (one thread per orbit)
    if (rc == SODECL_OK && rec && pick.lanes == 1 && best < 1e300 &&
        (solver == SODECL_EULER || solver == SODECL_RUNGE_KUTTA || solver == SODECL_STOCHASTIC_EULER)) {
        Cand c = pick;
        c.store = SODECL_STORE_PAIRS;
        float ms = 0.f;
        if (trial(c, ms) && ms < best) {
            best = ms;
            pick = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != SODECL_OK) return rc;
    // rebuild the context's program with the winner
    ctx->cfg.local_group_size = pick.block;
    ctx->cfg.min_blocks_per_sm = pick.min_blocks;
    ctx->cfg.division = pick.division;
    ctx->cfg.lanes_per_orbit = pick.lanes;
    ctx->cfg.record_store = pick.store;
    try {
        auto prog = sodecl_b200::build(make_spec(ctx->cfg), ctx->system_src);
        if (prog != ctx->prog) {
            if (ctx->lib) cudaLibraryUnload(ctx->lib);
            ctx->lib = nullptr;
            ctx->kernel = nullptr;
            ctx->gpu_ready = false;
            ctx->prog = prog;
        }
    } catch (const std::exception &ex) {
        ctx->cfg = saved;
        ctx->prog = saved_prog;
        return ctx->fail(SODECL_ERR_COMPILE, ex.what());
    }
    if ((rc = ensure_gpu(ctx)) != SODECL_OK) return rc;
    if (block) *block = pick.block;
    if (min_blocks) *min_blocks = pick.min_blocks;
    if (division) *division = pick.division;
    if (lanes) *lanes = pick.lanes;
    if (best_ms) *best_ms = best;
    return SODECL_OK;
}

int sodecl_cuda_program_division(const sodecl_ctx *ctx)
{
    if (!ctx || !ctx->prog) return SODECL_ERR_STATE;
    return ctx->prog->fast_div ? SODECL_DIV_RECIPROCAL : SODECL_DIV_IEEE;
}

int sodecl_cuda_adjoint(sodecl_ctx *ctx, const sodecl_adjoint_io *io, void *stream)
{
    if (!ctx) return SODECL_ERR_INVALID_ARG;
    if (!io || !io->t0 || !io->y0 || (!io->params && ctx->cfg.num_params > 0) || !io->targets || !io->loss)
        return ctx->fail(SODECL_ERR_INVALID_ARG, "adjoint: t0, y0, params, targets and loss are required");
    if (ctx->cfg.solver == SODECL_STOCHASTIC_EULER || ctx->cfg.solver == SODECL_DORMAND_PRINCE)
        return ctx->fail(SODECL_ERR_UNSUPPORTED, "the adjoint covers the fixed-step deterministic solvers");
    if (ctx->cfg.precision != SODECL_FP64) return ctx->fail(SODECL_ERR_UNSUPPORTED, "the adjoint is FP64");
    if (io->n < 1 || io->n > ctx->cfg.list_size) return ctx->fail(SODECL_ERR_INVALID_ARG, "adjoint: orbit count");
    if (io->tape_entries < 0 || io->tape_entries > 30000)
        return ctx->fail(SODECL_ERR_INVALID_ARG, "adjoint: tape size out of range");
    if (ctx->system_src.empty()) return ctx->fail(SODECL_ERR_STATE, "compile the system first");
    DeviceScope dev(ctx->cfg.device);
    for (const void *p : {static_cast<const void *>(io->t0), static_cast<const void *>(io->y0),
                          static_cast<const void *>(io->params), static_cast<const void *>(io->targets),
                          static_cast<const void *>(io->loss), static_cast<const void *>(io->grad_params),
                          static_cast<const void *>(io->grad_y0), static_cast<const void *>(io->flags)})
        if (!sodecl_b200::kernel_can_access(p, ctx->cfg.device))
            return ctx->fail(SODECL_ERR_INVALID_ARG, "adjoint: a buffer is not memory this device can access "
                                                     "(device, managed or pinned host memory)");
    const int tape = io->tape_entries > 0 ? io->tape_entries : 256;
    const auto traits = sodecl_b200::inspect_system(ctx->system_src);
    // products: the file's calc_vjp, else its two Jacobians, else the tape
    const int mode = io->use_tape ? 0 : traits.has_vjp ? 2 : (traits.has_jacobian && traits.has_pjacobian) ? 1 : 0;
    // Each thread runs its orbit's whole forward and backward sweep, so a
    // second wave would double the time: the resident blocks the compiler
    // must allow for (its register cap) are enough for every orbit to get a
    // thread in the first wave, up to 512 threads per SM (128 registers) for
    // passes with gradients and 1024 (64 registers) for the forward sweep
    // alone, e.g. the finite-difference baseline's wide launches.  Blocks of
    // local_group_size threads, 128 by default.  (Measured at 2^16 orbits:
    // blocks of 32, 64 or 96 with up to 146 registers per thread run the
    // gradient no faster than 4 blocks of 128 at 128 registers.)
    const bool with_gradient = io->grad_params || io->grad_y0;
    const int max_threads = with_gradient ? 512 : 1024;
    int sms = 148;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->cfg.device) != cudaSuccess) {
        cudaGetLastError();
        sms = 148;
    }
    sms = std::max(1, sms);
    auto resident = [&](int blk) {  // blocks per SM for one wave, within max_threads
        const long long r = (io->n + static_cast<long long>(sms) * blk - 1) / (static_cast<long long>(sms) * blk);
        return static_cast<int>(std::max<long long>(1, std::min<long long>(r, max_threads / blk)));
    };
    const int block = ctx->cfg.local_group_size > 0 ? ctx->cfg.local_group_size : 128;
    const int per_sm = resident(block);
    const int min_blocks = per_sm * block <= 256 ? 0 : per_sm;
    // Division: loss-only passes (the forward sweep) follow the context's mode;
    // passes with gradients use IEEE division, measured faster there (the
    // reciprocal wrapper costs registers the backward sweep needs).  The
    // quotients are the same either way.
    const bool fast_div = !with_gradient && reciprocal_division(ctx->cfg);
    if (!ctx->adj_prog || ctx->adj_tape != tape || ctx->adj_mode != mode || ctx->adj_min_blocks != min_blocks ||
        ctx->adj_fast_div != fast_div || ctx->adj_block != block || ctx->adj_gradient != with_gradient) {
        try {
            ProgramSpec spec = make_spec(ctx->cfg);
            spec.block_max = block;
            spec.min_blocks = min_blocks;
            spec.fast_div = fast_div;
            auto prog = sodecl_b200::build_adjoint(spec, ctx->system_src, tape, mode, with_gradient);
            if (ctx->adj_lib) cudaLibraryUnload(ctx->adj_lib);
            ctx->adj_lib = nullptr;
            ctx->adj_kernel = nullptr;
            ctx->adj_prog = prog;
            ctx->adj_tape = tape;
            ctx->adj_mode = mode;
            ctx->adj_min_blocks = min_blocks;
            ctx->adj_fast_div = fast_div;
            ctx->adj_block = block;
            ctx->adj_gradient = with_gradient;
        } catch (const std::exception &ex) {
            return ctx->fail(SODECL_ERR_COMPILE, ex.what());
        }
    }
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || ctx->cfg.device >= count) {
        cudaGetLastError();
        return ctx->fail(SODECL_ERR_NO_DEVICE, "no CUDA device");
    }
    if (!ctx->adj_lib) {
        SODECL_CUDA_TRY(ctx, cudaLibraryLoadData(&ctx->adj_lib, ctx->adj_prog->cubin.data(), nullptr, nullptr, 0,
                                                 nullptr, nullptr, 0));
        SODECL_CUDA_TRY(ctx, cudaLibraryGetKernel(&ctx->adj_kernel, ctx->adj_lib, "sodecl_adjoint"));
    }
    const long long n = io->n;
    const int64_t steps = ctx->nchunks * static_cast<int64_t>(ctx->cfg.kernel_steps);
    const size_t neq = ctx->cfg.num_equat;
    // the segment buffer holds per step the state, t and, for RK4, the three
    // stage inputs (SODECL_SEG_WIDTH in the adjoint kernel)
    const size_t seg_width = ctx->cfg.solver == SODECL_RUNGE_KUTTA ? 4 * neq + 1 : neq + 1;
    // Steps per checkpoint.  By default one segment -- the forward sweep
    // records the whole trajectory and the backward sweep recomputes nothing
    // (0.70x the time at 2^16 orbits x 5000 RK4 steps) -- when its buffer
    // takes at most half the device's free memory (or what the context
    // already holds), else ceil(sqrt(steps)) as the memory-lean schedule.
    // (The free-memory query can take milliseconds, so it is made only when
    // the context does not hold a large enough buffer already.)
    int C = io->ckpt_every;
    if (C <= 0) {
        C = std::max<int>(1, static_cast<int>(std::ceil(std::sqrt(static_cast<double>(steps)))));
        const double whole_bytes = 8.0 * n * (static_cast<double>(steps) * seg_width + neq + 1);
        bool whole = with_gradient && steps > 0 && whole_bytes <= static_cast<double>(ctx->adj_scratch_bytes);
        if (with_gradient && steps > 0 && !whole) {
            size_t free_b = 0, total_b = 0;
            if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
                cudaGetLastError();
                free_b = 0;
            }
            whole = whole_bytes <= 0.5 * static_cast<double>(free_b);
        }
        if (whole) C = static_cast<int>(steps);
    }
    if (steps > 0 && C > steps) C = static_cast<int>(steps);
    const int64_t nckpt = steps > 0 ? (steps + C - 1) / C : 1;
    const size_t need = io->grad_params || io->grad_y0
                            ? sizeof(double) * n * (nckpt * (neq + 1) + static_cast<int64_t>(C) * seg_width)
                            : 0;
    if (need > ctx->adj_scratch_bytes) {
        cudaFree(ctx->adj_scratch);
        ctx->adj_scratch = nullptr;
        ctx->adj_scratch_bytes = 0;
        SODECL_CUDA_TRY(ctx, cudaMalloc(&ctx->adj_scratch, need));
        ctx->adj_scratch_bytes = need;
    }
    AdjointArgs a{};
    a.t0 = io->t0;
    a.y0 = io->y0;
    a.p = io->params;
    a.targets = io->targets;
    a.loss = io->loss;
    a.grad_p = io->grad_params;
    a.grad_y0 = io->grad_y0;
    if (need) {
        double *base = static_cast<double *>(ctx->adj_scratch);
        a.ckpt = base;
        a.ckpt_t = a.ckpt + nckpt * neq * n;
        a.seg = a.ckpt_t + nckpt * n;
        // the kernel writes gradients only when grad_p is set; give it a sink
        if (!a.grad_p) return ctx->fail(SODECL_ERR_INVALID_ARG, "adjoint: grad_params is required with grad_y0");
    }
    a.flags = io->flags;
    a.n = n;
    a.nchunks = static_cast<int>(ctx->nchunks);
    a.ckpt_every = C;
    void *args[] = {&a};
    SODECL_CUDA_TRY(ctx, cudaLaunchKernel(reinterpret_cast<const void *>(ctx->adj_kernel),
                                          dim3(static_cast<unsigned>((n + block - 1) / block)), dim3(block), args, 0,
                                          static_cast<cudaStream_t>(stream)));
    return SODECL_OK;
}

int sodecl_cuda_release_scratch(sodecl_ctx *ctx)
{
    if (!ctx) return SODECL_ERR_INVALID_ARG;
    DeviceScope dev(ctx->cfg.device);
    if (ctx->d_records || ctx->adj_scratch) {
        // the buffers may still be in use by work queued on the context's streams
        if (ctx->stream) SODECL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
        if (ctx->copy_stream) SODECL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->copy_stream));
        SODECL_CUDA_TRY(ctx, cudaFree(ctx->d_records));
        ctx->d_records = nullptr;
        ctx->d_records_bytes = 0;
        SODECL_CUDA_TRY(ctx, cudaFree(ctx->adj_scratch));
        ctx->adj_scratch = nullptr;
        ctx->adj_scratch_bytes = 0;
    }
    release_cached_records(ctx->cfg.device);  // and what earlier contexts left
    return SODECL_OK;
}

int sodecl_cuda_release_cached(int device)
{
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        cudaGetLastError();
        return SODECL_ERR_NO_DEVICE;
    }
    DeviceScope dev(device);
    release_cached_records(device);
    return SODECL_OK;
}

int sodecl_cuda_get_cfg(const sodecl_ctx *ctx, sodecl_cfg *cfg)
{
    if (!ctx || !cfg) return SODECL_ERR_INVALID_ARG;
    *cfg = ctx->cfg;
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
    if (ctx->gpu_ready || ctx->uploaded || ctx->adj_lib) {
        DeviceScope dev(ctx->cfg.device);
        if (ctx->stream) cudaStreamSynchronize(ctx->stream);
        if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
        free_buffers(ctx);
        cudaFree(ctx->adj_scratch);
        if (ctx->adj_lib) cudaLibraryUnload(ctx->adj_lib);
        if (ctx->stream) cudaStreamDestroy(ctx->stream);
        if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
        if (ctx->lib) cudaLibraryUnload(ctx->lib);
    }
    delete ctx;
}

}  // extern "C"
