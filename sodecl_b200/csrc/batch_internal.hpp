// Internal to libsodecl_cuda: the batch object and the kernel-argument block
// of the persistent batch kernel, shared by batch.cpp and batch_noalloc.cu.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <memory>
#include <string>
#include <vector>

#include "program.hpp"
#include "sodecl_cuda.h"

namespace sodecl_b200_batch {

constexpr int kMaxClasses = 32;

// Must match struct sodecl_batch_args in device/batch.cuh field for field.
struct BatchArgs {
    double *t;
    double *y;
    const double *p;
    double *counters;
    const long long *nsteps;
    const long long *orbit_id;
    long long *newton_passes;
    int *flags;
    unsigned long long *head;
    int nclasses;
    int order[kMaxClasses];
    long long begin[kMaxClasses];
    long long end[kMaxClasses];
    long long ybase[kMaxClasses];
    long long pbase[kMaxClasses];
};

struct Class {
    sodecl_b200::BatchClass def;
    double cost_per_step = 1.0;  // relative estimate, orders the classes
    int requested_lanes = 0;     // sodecl_class_cfg.lanes_per_orbit (0: automatic, tunable)
    bool rows = false;           // the system file has the per-row functions this solver needs
};

// Lanes per orbit for an automatic class: about two rows per lane from 12
// equations up (variant 0); the tuner also tries one lane (1), twice (2) and
// half (3) that.  Explicit choices are kept.
inline int class_lanes(const Class &c, int variant)
{
    if (c.requested_lanes > 0) return c.requested_lanes;
    if (!c.rows) return 1;
    const int neq = c.def.spec.num_equat;
    int lanes = 1;
    if (neq >= 12) {
        lanes = 4;
        while (lanes < 32 && 2 * lanes < neq) lanes *= 2;
    }
    switch (variant) {
    case 1: return 1;
    case 2: return neq >= 4 ? std::min(32, lanes * 2 > 1 ? lanes * 2 : 4) : lanes;
    case 3: return lanes >= 4 ? lanes / 2 : lanes;
    default: return lanes;
    }
}

}  // namespace sodecl_b200_batch

using sodecl_b200_batch::BatchArgs;
using sodecl_b200_batch::kMaxClasses;

struct sodecl_batch {
    int device = 0;
    int fmad = 1;
    int division = SODECL_DIV_RECIPROCAL;
    int block = 128;
    int blocks_per_sm = 0;  // 0 = occupancy limit
    // register cap of the program: resident blocks of 256 threads the
    // compiler must allow for (0: none, up to 255 registers per thread)
    int reg_blocks = 0;
    std::vector<sodecl_b200_batch::Class> classes;
    std::shared_ptr<const sodecl_b200::Program> prog;
    cudaLibrary_t lib = nullptr;
    cudaKernel_t kernel = nullptr;
    cudaStream_t stream = nullptr;
    std::string error;

    // items, sorted by (class, descending steps); perm[sorted] = caller index
    int64_t nitems = 0;
    std::vector<int64_t> perm;
    std::vector<int32_t> item_class;
    std::vector<int64_t> y_off, p_off;  // caller packing offsets
    BatchArgs args{};
    double *d_t = nullptr, *d_y = nullptr, *d_p = nullptr, *d_cnt = nullptr;
    long long *d_nsteps = nullptr, *d_orbit = nullptr, *d_passes = nullptr;
    int *d_flags = nullptr;
    unsigned long long *d_head = nullptr;
    int64_t total_y = 0, total_p = 0;
    bool has_counters = false;

    int warp_words = 0;  // doubles of dynamic shared memory per warp (lanes-per-orbit classes)

    // program loaded by sodecl_batch_run_noalloc when the caller never
    // uploaded items through sodecl_batch_set_items
    cudaLibrary_t noalloc_lib = nullptr;
    cudaKernel_t noalloc_kernel = nullptr;

    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    int graph_grid = 0, graph_block = 0;
    double last_ms = 0.0;

    int fail(int code, const std::string &m)
    {
        error = m;
        return code;
    }
};

namespace sodecl_b200_batch {

// Dynamic shared memory of one block of the batch kernel, and its cap (the
// default limit, no opt-in).
constexpr size_t kSharedCap = 48 * 1024;
inline size_t shared_bytes(const sodecl_batch *b, int block)
{
    return static_cast<size_t>(block / 32) * static_cast<size_t>(b->warp_words) * sizeof(double);
}

}  // namespace sodecl_b200_batch
