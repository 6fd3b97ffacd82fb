// Heterogeneous batches (sodecl_batch_* in include/sodecl_cuda.h): many
// orbits of several system x solver classes, each orbit with its own step
// count, integrated by one persistent kernel (device/batch.cuh) from
// per-class work queues, launched through a captured CUDA graph.
//
// The reference has no counterpart: it integrates one system with one solver
// and one step count per call (src/sodeclmgr.cpp:921-1035), so a sweep over
// uneven orbits means one call per group, each padded to its longest orbit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "batch_internal.hpp"
#include "program.hpp"
#include "sodecl_cuda.h"

namespace {

struct Scope {
    int prev = -1;
    explicit Scope(int dev)
    {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        cudaSetDevice(dev);
    }
    ~Scope()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

int cuda_err(sodecl_batch *b, cudaError_t e, const char *what)
{
    cudaGetLastError();
    return b->fail(e == cudaErrorMemoryAllocation ? SODECL_ERR_OUT_OF_MEMORY : SODECL_ERR_CUDA,
                   std::string(what) + ": " + cudaGetErrorString(e));
}

#define BATCH_TRY(b, call)                                       \
    do {                                                         \
        cudaError_t e_ = (call);                                 \
        if (e_ != cudaSuccess) return cuda_err((b), e_, #call);  \
    } while (0)

void drop_graph(sodecl_batch *b)
{
    if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->graph_exec = nullptr;
    b->graph = nullptr;
}

void free_items(sodecl_batch *b)
{
    drop_graph(b);
    cudaFree(b->d_t);
    cudaFree(b->d_y);
    cudaFree(b->d_p);
    cudaFree(b->d_cnt);
    cudaFree(b->d_nsteps);
    cudaFree(b->d_orbit);
    cudaFree(b->d_passes);
    cudaFree(b->d_flags);
    b->d_t = b->d_y = b->d_p = b->d_cnt = nullptr;
    b->d_nsteps = b->d_orbit = b->d_passes = nullptr;
    b->d_flags = nullptr;
    b->nitems = 0;
}

// Relative cost of one step of a class, to visit expensive classes first:
// right-hand sides per step x a size term (quadratic: coupled systems
// dominate), Newton passes guessed at 10.
double step_cost(const sodecl_b200::ProgramSpec &s)
{
    const double n = s.num_equat;
    const double rhs = 10.0 + n * n;
    switch (s.solver) {
    case SODECL_EULER: return rhs;
    case SODECL_RUNGE_KUTTA: return 4.0 * rhs + 6.0 * n;
    case SODECL_IMPLICIT_EULER:
    case SODECL_IMPLICIT_MIDPOINT: return 10.0 * (2.0 * rhs + 8.0 * n);
    default: return rhs + 20.0 * (s.num_noi + 1) / 2;
    }
}

// A warp's slots of a lanes-per-orbit class fit half the 48 KiB cap, so any
// block of up to 64 threads can launch.
bool lanes_fit(const sodecl_b200::ProgramSpec &s)
{
    return (32 / s.lanes) * sodecl_b200::lanes_slot_words(s) * sizeof(double) * 2 <= sodecl_b200_batch::kSharedCap;
}

// Rebuilds the program with these lanes per orbit per class and this
// register cap (no-op when they are the current ones) and loads it in place
// of the current one.
int load_program(sodecl_batch *b, const std::vector<int> &lanes, int reg_blocks)
{
    bool same = reg_blocks == b->reg_blocks;
    for (size_t k = 0; k < b->classes.size(); ++k) same = same && b->classes[k].def.spec.lanes == lanes[k];
    if (same && b->prog) return SODECL_OK;
    for (size_t k = 0; k < b->classes.size(); ++k) b->classes[k].def.spec.lanes = lanes[k];
    b->reg_blocks = reg_blocks;
    std::vector<sodecl_b200::BatchClass> defs;
    for (const auto &c : b->classes) defs.push_back(c.def);
    try {
        b->prog = sodecl_b200::build_batch(defs, b->fmad != 0, b->division == SODECL_DIV_RECIPROCAL, 256, reg_blocks);
    } catch (const std::exception &ex) {
        return b->fail(SODECL_ERR_COMPILE, ex.what());
    }
    b->warp_words = sodecl_b200::batch_warp_words(defs);
    drop_graph(b);
    if (b->lib) {
        if (b->stream) cudaStreamSynchronize(b->stream);
        cudaLibraryUnload(b->lib);
        b->lib = nullptr;
        b->kernel = nullptr;
        BATCH_TRY(b, cudaLibraryLoadData(&b->lib, b->prog->cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
        BATCH_TRY(b, cudaLibraryGetKernel(&b->kernel, b->lib, b->prog->kernel_name.c_str()));
    }
    while (b->block > 32 && sodecl_b200_batch::shared_bytes(b, b->block) > sodecl_b200_batch::kSharedCap)
        b->block -= 32;
    return SODECL_OK;
}

int grid_size(sodecl_batch *b, int block)
{
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, reinterpret_cast<const void *>(b->kernel),
                                                                  block, sodecl_b200_batch::shared_bytes(b, block));
    if (e != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        per_sm = 1;
    }
    if (b->blocks_per_sm > 0) per_sm = std::min(per_sm, b->blocks_per_sm);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
    return std::max(1, sms) * per_sm;
}

int launch_once(sodecl_batch *b, int block, int grid)
{
    BATCH_TRY(b, cudaMemsetAsync(b->d_head, 0, sizeof(unsigned long long) * kMaxClasses, b->stream));
    void *params[] = {&b->args};
    BATCH_TRY(b, cudaLaunchKernel(reinterpret_cast<const void *>(b->kernel), dim3(grid), dim3(block), params,
                                  sodecl_b200_batch::shared_bytes(b, block), b->stream));
    return SODECL_OK;
}

}  // namespace

extern "C" {

void sodecl_class_cfg_init(sodecl_class_cfg *c)
{
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->solver = SODECL_EULER;
    c->newton_tol = 1e-7;
    c->newton_max_iter = 1000;
    c->lanes_per_orbit = 0;
}

int sodecl_batch_create(int device, int fmad, int division, sodecl_batch **out)
{
    if (!out) return SODECL_ERR_INVALID_ARG;
    *out = nullptr;
    if (device < 0 || (division != SODECL_DIV_RECIPROCAL && division != SODECL_DIV_IEEE))
        return SODECL_ERR_INVALID_ARG;
    auto *b = new (std::nothrow) sodecl_batch();
    if (!b) return SODECL_ERR_OUT_OF_MEMORY;
    b->device = device;
    b->fmad = fmad ? 1 : 0;
    b->division = division;
    *out = b;
    return SODECL_OK;
}

int sodecl_batch_add_class(sodecl_batch *b, const char *system_src, size_t len, const sodecl_class_cfg *cfg,
                           int32_t *class_id)
{
    if (!b) return SODECL_ERR_INVALID_ARG;
    if (!system_src || !cfg) return b->fail(SODECL_ERR_INVALID_ARG, "NULL system source or class configuration");
    if (b->prog) return b->fail(SODECL_ERR_STATE, "classes must be added before sodecl_batch_compile");
    if (static_cast<int>(b->classes.size()) >= kMaxClasses)
        return b->fail(SODECL_ERR_INVALID_ARG, "at most 32 classes per batch");
    const sodecl_class_cfg &c = *cfg;
    if (c.solver < 0 || c.solver > 4 || c.num_equat < 1 || c.num_params < 0 || c.num_noi < 0 || !(c.dt > 0) ||
        !std::isfinite(c.dt) || (c.solver == SODECL_STOCHASTIC_EULER && c.num_noi < 1) || c.newton_max_iter < 0 ||
        c.newton_tol < 0 || c.lanes_per_orbit < 0 || c.lanes_per_orbit > 32 ||
        (c.lanes_per_orbit & (c.lanes_per_orbit - 1)) != 0)
        return b->fail(SODECL_ERR_INVALID_ARG, "invalid class configuration");
    sodecl_b200_batch::Class cl;
    cl.def.system_src.assign(system_src, len);
    const auto traits = sodecl_b200::inspect_system(cl.def.system_src);
    if (!traits.has_system) return b->fail(SODECL_ERR_COMPILE, "the system file defines no sode_system(...)");
    if ((c.solver == SODECL_IMPLICIT_EULER || c.solver == SODECL_IMPLICIT_MIDPOINT) && !traits.has_jacobian)
        return b->fail(SODECL_ERR_NO_JACOBIAN, "implicit solvers need calc_jacobian(...) in the system file");
    if (c.solver == SODECL_STOCHASTIC_EULER && !traits.has_stoch)
        return b->fail(SODECL_ERR_NO_STOCH, "the stochastic solver needs sode_system_stoch(...) in the system file");
    auto &s = cl.def.spec;
    s.solver = c.solver;
    s.num_equat = c.num_equat;
    s.num_params = c.num_params;
    s.num_noi = c.num_noi;
    s.dt = c.dt;
    s.newton_tol = c.newton_tol > 0 ? c.newton_tol : 1e-7;
    s.newton_max_iter = c.newton_max_iter > 0 ? c.newton_max_iter : 1000;
    s.fmad = b->fmad != 0;
    // lanes per orbit: the per-row functions this solver needs
    bool rows = traits.has_row;
    if (c.solver == SODECL_STOCHASTIC_EULER) rows = rows && traits.has_stoch_row;
    if (c.solver == SODECL_IMPLICIT_EULER || c.solver == SODECL_IMPLICIT_MIDPOINT) rows = rows && traits.has_jac_band;
    if (c.lanes_per_orbit > 1 && !rows)
        return b->fail(SODECL_ERR_UNSUPPORTED, "lanes per orbit need sode_system_row(...) in the system file, and "
                                               "sode_system_stoch_row(...) for the stochastic solver or "
                                               "calc_jacobian_band(...) for the implicit ones");
    cl.requested_lanes = c.lanes_per_orbit;
    cl.rows = rows;
    s.lanes = sodecl_b200_batch::class_lanes(cl, 0);
    if (s.lanes > 1 && !lanes_fit(s))
        return b->fail(SODECL_ERR_UNSUPPORTED, "lanes per orbit: one warp's orbits need more than half of a block's "
                                               "shared memory");
    cl.cost_per_step = step_cost(s);
    b->classes.push_back(std::move(cl));
    if (class_id) *class_id = static_cast<int32_t>(b->classes.size() - 1);
    return SODECL_OK;
}

int sodecl_batch_compile(sodecl_batch *b)
{
    if (!b) return SODECL_ERR_INVALID_ARG;
    if (b->classes.empty()) return b->fail(SODECL_ERR_STATE, "no classes");
    std::vector<sodecl_b200::BatchClass> defs;
    for (const auto &c : b->classes) defs.push_back(c.def);
    try {
        b->prog = sodecl_b200::build_batch(defs, b->fmad != 0, b->division == SODECL_DIV_RECIPROCAL, 256,
                                           b->reg_blocks);
    } catch (const std::exception &ex) {
        return b->fail(SODECL_ERR_COMPILE, ex.what());
    }
    b->warp_words = sodecl_b200::batch_warp_words(defs);
    while (b->block > 32 && sodecl_b200_batch::shared_bytes(b, b->block) > sodecl_b200_batch::kSharedCap)
        b->block -= 32;
    return SODECL_OK;
}

int sodecl_batch_set_items(sodecl_batch *b, int64_t n, const int32_t *item_class, const int64_t *nsteps,
                           const double *t0, const double *y0, const double *params, const double *counters)
{
    if (!b) return SODECL_ERR_INVALID_ARG;
    if (!b->prog) return b->fail(SODECL_ERR_STATE, "call sodecl_batch_compile first");
    if (n < 1 || !item_class || !nsteps || !t0 || !y0 || !params)
        return b->fail(SODECL_ERR_INVALID_ARG, "items need classes, step counts, t0, y0 and params");
    const int nc = static_cast<int>(b->classes.size());
    for (int64_t i = 0; i < n; ++i)
        if (item_class[i] < 0 || item_class[i] >= nc || nsteps[i] < 0)
            return b->fail(SODECL_ERR_INVALID_ARG, "item " + std::to_string(i) + ": bad class or step count");
    for (const auto &c : b->classes)
        if (c.def.spec.solver == SODECL_STOCHASTIC_EULER && !counters)
            return b->fail(SODECL_ERR_INVALID_ARG, "a stochastic class needs counters");

    Scope scope(b->device);
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || b->device >= count) {
        cudaGetLastError();
        return b->fail(SODECL_ERR_NO_DEVICE, "no CUDA device " + std::to_string(b->device));
    }
    if (!b->lib) {
        BATCH_TRY(b, cudaLibraryLoadData(&b->lib, b->prog->cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
        BATCH_TRY(b, cudaLibraryGetKernel(&b->kernel, b->lib, b->prog->kernel_name.c_str()));
        BATCH_TRY(b, cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
        BATCH_TRY(b, cudaMalloc(&b->d_head, sizeof(unsigned long long) * kMaxClasses));
    }
    free_items(b);

    // caller packing: item i's state at y_off[i], parameters at p_off[i]
    b->y_off.assign(n + 1, 0);
    b->p_off.assign(n + 1, 0);
    for (int64_t i = 0; i < n; ++i) {
        const auto &s = b->classes[item_class[i]].def.spec;
        b->y_off[i + 1] = b->y_off[i] + s.num_equat;
        b->p_off[i + 1] = b->p_off[i] + s.num_params;
    }
    // sorted order: by class, then by decreasing step count
    b->perm.resize(n);
    std::iota(b->perm.begin(), b->perm.end(), 0);
    std::stable_sort(b->perm.begin(), b->perm.end(), [&](int64_t x, int64_t y) {
        if (item_class[x] != item_class[y]) return item_class[x] < item_class[y];
        return nsteps[x] > nsteps[y];
    });
    b->item_class.assign(item_class, item_class + n);

    BatchArgs &a = b->args;
    std::memset(&a, 0, sizeof(a));
    a.nclasses = nc;
    std::vector<double> ht(n), hy(b->y_off[n]), hp(std::max<int64_t>(1, b->p_off[n])), hc;
    std::vector<long long> hs(n), ho(n);
    if (counters) hc.resize(n);
    std::vector<double> work(nc, 0.0);
    int64_t yb = 0, pb = 0;
    int64_t pos = 0;
    for (int c = 0; c < nc; ++c) {
        const auto &s = b->classes[c].def.spec;
        a.begin[c] = pos;
        a.ybase[c] = yb;
        a.pbase[c] = pb;
        while (pos < n && item_class[b->perm[pos]] == c) {
            const int64_t i = b->perm[pos];
            ht[pos] = t0[i];
            std::memcpy(&hy[yb], y0 + b->y_off[i], sizeof(double) * s.num_equat);
            if (s.num_params) std::memcpy(&hp[pb], params + b->p_off[i], sizeof(double) * s.num_params);
            hs[pos] = nsteps[i];
            ho[pos] = i;
            if (counters) hc[pos] = counters[i];
            work[c] += static_cast<double>(nsteps[i]) * b->classes[c].cost_per_step;
            yb += s.num_equat;
            pb += s.num_params;
            ++pos;
        }
        a.end[c] = pos;
    }
    b->total_y = yb;
    b->total_p = pb;
    // visit the classes with the most work first
    std::vector<int> order(nc);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return work[x] > work[y]; });
    for (int k = 0; k < nc; ++k) a.order[k] = order[k];

    BATCH_TRY(b, cudaMalloc(&b->d_t, sizeof(double) * n));
    BATCH_TRY(b, cudaMalloc(&b->d_y, sizeof(double) * std::max<int64_t>(1, yb)));
    BATCH_TRY(b, cudaMalloc(&b->d_p, sizeof(double) * std::max<int64_t>(1, pb)));
    BATCH_TRY(b, cudaMalloc(&b->d_nsteps, sizeof(long long) * n));
    BATCH_TRY(b, cudaMalloc(&b->d_orbit, sizeof(long long) * n));
    BATCH_TRY(b, cudaMalloc(&b->d_passes, sizeof(long long) * n));
    BATCH_TRY(b, cudaMalloc(&b->d_flags, sizeof(int) * n));
    if (counters) BATCH_TRY(b, cudaMalloc(&b->d_cnt, sizeof(double) * n));
    BATCH_TRY(b, cudaMemcpyAsync(b->d_t, ht.data(), sizeof(double) * n, cudaMemcpyHostToDevice, b->stream));
    BATCH_TRY(b, cudaMemcpyAsync(b->d_y, hy.data(), sizeof(double) * yb, cudaMemcpyHostToDevice, b->stream));
    if (pb) BATCH_TRY(b, cudaMemcpyAsync(b->d_p, hp.data(), sizeof(double) * pb, cudaMemcpyHostToDevice, b->stream));
    BATCH_TRY(b, cudaMemcpyAsync(b->d_nsteps, hs.data(), sizeof(long long) * n, cudaMemcpyHostToDevice, b->stream));
    BATCH_TRY(b, cudaMemcpyAsync(b->d_orbit, ho.data(), sizeof(long long) * n, cudaMemcpyHostToDevice, b->stream));
    if (counters)
        BATCH_TRY(b, cudaMemcpyAsync(b->d_cnt, hc.data(), sizeof(double) * n, cudaMemcpyHostToDevice, b->stream));
    BATCH_TRY(b, cudaMemsetAsync(b->d_passes, 0, sizeof(long long) * n, b->stream));
    BATCH_TRY(b, cudaMemsetAsync(b->d_flags, 0, sizeof(int) * n, b->stream));
    BATCH_TRY(b, cudaStreamSynchronize(b->stream));
    a.t = b->d_t;
    a.y = b->d_y;
    a.p = b->d_p;
    a.counters = b->d_cnt;
    a.nsteps = b->d_nsteps;
    a.orbit_id = b->d_orbit;
    a.newton_passes = b->d_passes;
    a.flags = b->d_flags;
    a.head = b->d_head;
    b->nitems = n;
    b->has_counters = counters != nullptr;
    return SODECL_OK;
}

int sodecl_batch_set_launch(sodecl_batch *b, int32_t block, int32_t blocks_per_sm)
{
    if (!b) return SODECL_ERR_INVALID_ARG;
    if (block < 32 || block > 256 || block % 32 || blocks_per_sm < 0)
        return b->fail(SODECL_ERR_INVALID_ARG, "block must be a multiple of 32 in [32, 256]");
    if (sodecl_b200_batch::shared_bytes(b, block) > sodecl_b200_batch::kSharedCap)
        return b->fail(SODECL_ERR_INVALID_ARG, "block too large: its warps' lanes-per-orbit slots exceed 48 KiB of "
                                               "shared memory");
    if (block != b->block || blocks_per_sm != b->blocks_per_sm) drop_graph(b);
    b->block = block;
    b->blocks_per_sm = blocks_per_sm;
    return SODECL_OK;
}

int sodecl_batch_run(sodecl_batch *b, int32_t use_graph)
{
    if (!b) return SODECL_ERR_INVALID_ARG;
    if (!b->nitems) return b->fail(SODECL_ERR_STATE, "no items: call sodecl_batch_set_items first");
    Scope scope(b->device);
    cudaEvent_t e0, e1;
    BATCH_TRY(b, cudaEventCreate(&e0));
    BATCH_TRY(b, cudaEventCreate(&e1));
    int rc = SODECL_OK;
    const int grid = grid_size(b, b->block);
    BATCH_TRY(b, cudaEventRecord(e0, b->stream));
    if (use_graph) {
        if (!b->graph_exec) {
            BATCH_TRY(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
            rc = launch_once(b, b->block, grid);
            cudaGraph_t g = nullptr;
            cudaError_t ec = cudaStreamEndCapture(b->stream, &g);
            if (rc != SODECL_OK) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            if (ec != cudaSuccess) return cuda_err(b, ec, "cudaStreamEndCapture");
            b->graph = g;
            BATCH_TRY(b, cudaGraphInstantiate(&b->graph_exec, b->graph, 0));
        }
        BATCH_TRY(b, cudaGraphLaunch(b->graph_exec, b->stream));
    } else {
        rc = launch_once(b, b->block, grid);
        if (rc != SODECL_OK) return rc;
    }
    BATCH_TRY(b, cudaEventRecord(e1, b->stream));
    BATCH_TRY(b, cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    b->last_ms = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return SODECL_OK;
}

int sodecl_batch_results(sodecl_batch *b, double *t, double *y, double *counters, int64_t *newton_passes,
                         int32_t *flags)
{
    if (!b) return SODECL_ERR_INVALID_ARG;
    if (!b->nitems) return b->fail(SODECL_ERR_STATE, "no items");
    Scope scope(b->device);
    const int64_t n = b->nitems;
    std::vector<double> ht(n), hy(std::max<int64_t>(1, b->total_y)), hc(b->has_counters ? n : 0);
    std::vector<long long> hpass(n);
    std::vector<int> hflags(n);
    BATCH_TRY(b, cudaMemcpy(ht.data(), b->d_t, sizeof(double) * n, cudaMemcpyDeviceToHost));
    BATCH_TRY(b, cudaMemcpy(hy.data(), b->d_y, sizeof(double) * b->total_y, cudaMemcpyDeviceToHost));
    if (b->has_counters) BATCH_TRY(b, cudaMemcpy(hc.data(), b->d_cnt, sizeof(double) * n, cudaMemcpyDeviceToHost));
    BATCH_TRY(b, cudaMemcpy(hpass.data(), b->d_passes, sizeof(long long) * n, cudaMemcpyDeviceToHost));
    BATCH_TRY(b, cudaMemcpy(hflags.data(), b->d_flags, sizeof(int) * n, cudaMemcpyDeviceToHost));
    const BatchArgs &a = b->args;
    for (int c = 0; c < a.nclasses; ++c) {
        const int neq = b->classes[c].def.spec.num_equat;
        for (int64_t pos = a.begin[c]; pos < a.end[c]; ++pos) {
            const int64_t i = b->perm[pos];
            if (t) t[i] = ht[pos];
            if (y) std::memcpy(y + b->y_off[i], &hy[a.ybase[c] + (pos - a.begin[c]) * neq], sizeof(double) * neq);
            if (counters && b->has_counters) counters[i] = hc[pos];
            if (newton_passes) newton_passes[i] = hpass[pos];
            if (flags) flags[i] = hflags[pos];
        }
    }
    return SODECL_OK;
}

int sodecl_batch_tune(sodecl_batch *b, int32_t *block, int32_t *blocks_per_sm, double *best_ms)
{
    // Times the run for each candidate and keeps the fastest: first the lanes
    // per orbit of the automatic classes (the heuristic, one lane, twice and
    // half the heuristic; each a rebuilt program, cached on disk), then the
    // launch shape.  Each trial integrates the current items from their
    // current state, so callers tune on a copy of the workload (e.g.
    // shortened step counts) and then upload the real items.
    if (!b) return SODECL_ERR_INVALID_ARG;
    if (!b->nitems) return b->fail(SODECL_ERR_STATE, "no items to tune on");
    bool tunable = false;
    for (const auto &c : b->classes) tunable = tunable || (c.requested_lanes == 0 && c.rows);
    if (tunable) {
        std::vector<std::vector<int>> tried;
        std::vector<int> best_lanes;
        double best_lanes_ms = 1e300;
        for (int v = 0; v < 4; ++v) {
            std::vector<int> lanes;
            bool fits = true;
            for (const auto &c : b->classes) {
                sodecl_b200::ProgramSpec sp = c.def.spec;
                sp.lanes = sodecl_b200_batch::class_lanes(c, v);
                fits = fits && (sp.lanes == 1 || lanes_fit(sp));
                lanes.push_back(sp.lanes);
            }
            if (!fits || std::find(tried.begin(), tried.end(), lanes) != tried.end()) continue;
            tried.push_back(lanes);
            int rc = load_program(b, lanes, b->reg_blocks);
            if (rc != SODECL_OK) return rc;
            rc = sodecl_batch_set_launch(b, std::min(b->block, 128), 0);
            if (rc != SODECL_OK) return rc;
            rc = sodecl_batch_run(b, 0);
            if (rc != SODECL_OK) return rc;
            if (b->last_ms < best_lanes_ms) {
                best_lanes_ms = b->last_ms;
                best_lanes = lanes;
            }
        }
        const int rc = load_program(b, best_lanes, b->reg_blocks);
        if (rc != SODECL_OK) return rc;
    }
    // Then the register cap of the program (none, 128 or 85 registers per
    // thread: one program holds every class, so without a cap the most
    // demanding class sets the count, and with it the resident warps, for
    // all) and, for each, the launch shape.
    std::vector<int> lanes_now;
    for (const auto &c : b->classes) lanes_now.push_back(c.def.spec.lanes);
    static const int caps[] = {0, 2, 3};
    static const int shapes[][2] = {{64, 0}, {128, 0}, {256, 0}, {128, 2}, {256, 1}, {64, 4}};
    double best = 1e300;
    int best_block = b->block, best_bps = b->blocks_per_sm, best_cap = b->reg_blocks;
    for (int cap : caps) {
        int rc = load_program(b, lanes_now, cap);
        if (rc != SODECL_OK) return rc;
        for (const auto &sh : shapes) {
            if (sodecl_b200_batch::shared_bytes(b, sh[0]) > sodecl_b200_batch::kSharedCap) continue;
            rc = sodecl_batch_set_launch(b, sh[0], sh[1]);
            if (rc != SODECL_OK) return rc;
            rc = sodecl_batch_run(b, 0);
            if (rc != SODECL_OK) return rc;
            if (b->last_ms < best) {
                best = b->last_ms;
                best_block = sh[0];
                best_bps = sh[1];
                best_cap = cap;
            }
        }
    }
    const int rc = load_program(b, lanes_now, best_cap);
    if (rc != SODECL_OK) return rc;
    sodecl_batch_set_launch(b, best_block, best_bps);
    if (block) *block = best_block;
    if (blocks_per_sm) *blocks_per_sm = best_bps;
    if (best_ms) *best_ms = best;
    return SODECL_OK;
}

int sodecl_batch_class_lanes(const sodecl_batch *b, int32_t *lanes)
{
    if (!b || !lanes) return SODECL_ERR_INVALID_ARG;
    for (size_t k = 0; k < b->classes.size(); ++k) lanes[k] = b->classes[k].def.spec.lanes;
    return SODECL_OK;
}

int sodecl_batch_last_ms(const sodecl_batch *b, double *ms)
{
    if (!b || !ms) return SODECL_ERR_INVALID_ARG;
    *ms = b->last_ms;
    return SODECL_OK;
}

int sodecl_batch_kernel_info(sodecl_batch *b, int *regs, int *local_bytes)
{
    if (!b || !b->kernel) return SODECL_ERR_STATE;
    Scope scope(b->device);
    cudaFuncAttributes fa{};
    BATCH_TRY(b, cudaFuncGetAttributes(&fa, reinterpret_cast<const void *>(b->kernel)));
    if (regs) *regs = fa.numRegs;
    if (local_bytes) *local_bytes = static_cast<int>(fa.localSizeBytes);
    return SODECL_OK;
}

size_t sodecl_batch_last_error(const sodecl_batch *b, char *buf, size_t n)
{
    const std::string &s = b ? b->error : std::string("null batch");
    if (buf && n) {
        const size_t k = std::min(n - 1, s.size());
        std::memcpy(buf, s.data(), k);
        buf[k] = '\0';
    }
    return s.size();
}

size_t sodecl_batch_program_source(const sodecl_batch *b, char *buf, size_t n)
{
    const std::string s = b && b->prog ? b->prog->source : std::string();
    if (buf && n) {
        const size_t k = std::min(n - 1, s.size());
        std::memcpy(buf, s.data(), k);
        buf[k] = '\0';
    }
    return s.size();
}

void sodecl_batch_destroy(sodecl_batch *b)
{
    if (!b) return;
    if (b->noalloc_lib) {
        Scope scope(b->device);
        cudaLibraryUnload(b->noalloc_lib);
    }
    if (b->lib) {
        Scope scope(b->device);
        if (b->stream) cudaStreamSynchronize(b->stream);
        free_items(b);
        cudaFree(b->d_head);
        if (b->stream) cudaStreamDestroy(b->stream);
        cudaLibraryUnload(b->lib);
    }
    delete b;
}

}  // extern "C"
