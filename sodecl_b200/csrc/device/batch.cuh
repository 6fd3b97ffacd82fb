// Heterogeneous batch: one persistent kernel integrates orbits of several
// classes -- each class a (system file, solver, sizes, step) combination --
// with per-orbit step counts, from device work queues.
//
// Program layout (assembled by program.cpp, build_batch):
//   prelude, noise generator, this file's shared part;
//   for each class k: namespace sodecl_cls_k { the class's size #defines,
//       the user's system file, solvers.cuh (step functions only), the
//       class body below };
//   the kernel `sodecl_batch`, which walks the classes in the host's order
//   (most expensive first) and runs each class's body.
//
// Load balance: the host sorts each class's orbits by decreasing step count.
// Every lane takes its own orbit from the class queue (an atomic counter)
// and, when that orbit is done, stores it and takes the next one, so lanes
// of a warp stay busy although their orbits have different lengths; a warp
// moves on to the next class when the queue is empty for all its lanes.
// Big orbits go first, small ones fill the tail.  Classes of wide systems
// can run with several lanes per orbit (SODECL_LANES > 1), each group of
// lanes taking orbits from the queue as one; their vectors live in the
// warp's region of dynamic shared memory (SODECL_BATCH_WARP_WORDS doubles per
// warp, the largest need of any such class), and the kernel joins the warp
// after each class so that no group's slot overlaps the next class's.

#ifndef SODECL_BATCH_SHARED
#define SODECL_BATCH_SHARED
#define SODECL_MAX_CLASSES 32

struct sodecl_batch_args {
    double *t;                       // [items] time, in/out
    double *y;                       // states, packed by class: class k's item j at ybase[k] + j*neq_k
    const double *p;                 // parameters, packed the same way with npar_k
    double *counters;                // [items] noise draw counters, in/out, or null
    const long long *nsteps;         // [items] steps to take
    const long long *orbit_id;       // [items] global orbit index (noise stream key)
    long long *newton_passes;        // [items] Newton passes taken, or null
    int *flags;                      // [items] status flags, or null
    unsigned long long *head;        // [nclasses] queue heads, zero at launch
    int nclasses;
    int order[SODECL_MAX_CLASSES];   // class visiting order
    long long begin[SODECL_MAX_CLASSES];
    long long end[SODECL_MAX_CLASSES];
    long long ybase[SODECL_MAX_CLASSES];
    long long pbase[SODECL_MAX_CLASSES];
};
#endif

#ifdef SODECL_BATCH_CLASS_BODY
// Stores orbit `item` (position j in its class) with its status.
__device__ __forceinline__ void sodecl_batch_store(const sodecl_batch_args &a, long long item, long long j,
                                                   long long ybase, real_t t, const real_t *y, double counter,
                                                   long long passes, int capped)
{
    a.t[item] = (double)t;
    bool finite = true;
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e) {
        finite = finite && isfinite(y[e]);
        a.y[ybase + j * _numeq_ + e] = (double)y[e];
    }
    if (a.counters) a.counters[item] = counter;
    if (a.newton_passes) a.newton_passes[item] = passes;
    if (a.flags) a.flags[item] = (capped ? SODECL_FLAG_NEWTON_CAP : 0) | (finite ? 0 : SODECL_FLAG_NONFINITE);
}

#if SODECL_LANES == 1 && (SODECL_SOLVER == 3 || SODECL_SOLVER == 4)
// Implicit solvers, one lane per orbit: Newton passes drive the loop, as in
// the single-system kernel.  A lane whose iteration has converged commits
// its step and starts the next at the following pass (sodecl_step_newton's
// arithmetic, in the same order), so the lanes of a warp do not wait at
// every step for the one that needs the most passes.  Parameters stay fixed
// in the inner pass loop (their reciprocals stay out of it); the lanes whose
// orbit is done take their next one from the class queue between inner
// loops.  Called by all 32 lanes of a warp together.
__device__ __forceinline__ void sodecl_class_run(const sodecl_batch_args &a, const int cls, double *)
{
    const long long begin = a.begin[cls];
    const unsigned long long count = (unsigned long long)(a.end[cls] - begin);
    unsigned long long *head = a.head + cls;
    const long long ybase = a.ybase[cls], pbase = a.pbase[cls];

    real_t y[_numeq_], x[_numeq_];
    real_t p[SODECL_NPAR_ALLOC];
    real_t t = 0;
    long long item = -1, left = 0, passes = 0;
    int capped = 0, pass = 0;
    bool need = true;
#pragma unroll 1
    for (;;) {
        if (need) {
            // take orbits until one has a step to take or the queue is empty;
            // an orbit with no step (a count of zero or less) is stored as it is
            need = false;
#pragma unroll 1
            for (;;) {
                const unsigned long long k = atomicAdd(head, 1ULL);
                if (k >= count) {
                    item = -1;
                    break;
                }
                item = begin + (long long)k;
                t = (real_t)a.t[item];
#pragma unroll SODECL_EQ_UNROLL
                for (int e = 0; e < _numeq_; ++e) y[e] = x[e] = (real_t)a.y[ybase + (long long)k * _numeq_ + e];
#pragma unroll SODECL_PAR_UNROLL
                for (int jj = 0; jj < _numpar_; ++jj) p[jj] = (real_t)__ldg(a.p + pbase + (long long)k * _numpar_ + jj);
                left = a.nsteps[item];
                passes = 0;
                capped = pass = 0;
                if (left > 0) break;
                sodecl_batch_store(a, item, (long long)k, ybase, t, y, a.counters ? a.counters[item] : 0.0, 0, 0);
            }
        }
        if (!__any_sync(0xffffffffu, item >= 0)) break;
#pragma unroll 1
        for (;;) {
            bool finished = false;
            if (item >= 0) {
                // a pass limit below one takes no pass: the step is capped at once
                const bool done = SODECL_NEWTON_MAX >= 1 && sodecl_newton_pass(_m_dt_, t, y, x, p);
                if (SODECL_NEWTON_MAX >= 1) ++pass;
                if (done || pass >= SODECL_NEWTON_MAX) {
                    if (!done) capped = 1;
                    passes += pass;
                    pass = 0;
                    t = t + _m_dt_;
#pragma unroll SODECL_EQ_UNROLL
                    for (int e = 0; e < _numeq_; ++e) y[e] = x[e];
                    if (--left <= 0) {
                        sodecl_batch_store(a, item, item - begin, ybase, t, y, a.counters ? a.counters[item] : 0.0,
                                           passes, capped);
                        item = -1;
                        finished = true;
                    }
                }
            }
            if (__any_sync(0xffffffffu, finished)) {
                need = finished;
                break;
            }
        }
    }
}
#elif SODECL_LANES == 1
// Runs class `cls` until its queue is empty for every lane of the warp.
// Called by all 32 lanes of a warp together.
__device__ __forceinline__ void sodecl_class_run(const sodecl_batch_args &a, const int cls, double *)
{
    const long long begin = a.begin[cls];
    const unsigned long long count = (unsigned long long)(a.end[cls] - begin);
    unsigned long long *head = a.head + cls;
    const long long ybase = a.ybase[cls], pbase = a.pbase[cls];

    real_t y[_numeq_];
    real_t p[SODECL_NPAR_ALLOC];
    real_t t = 0;
    long long item = -1, left = 0, passes = 0;
    int capped = 0;
    double counter = 0.0;

    unsigned long long k = atomicAdd(head, 1ULL);
    if (k < count) item = begin + (long long)k;
    if (item >= 0) {
        t = (real_t)a.t[item];
#pragma unroll SODECL_EQ_UNROLL
        for (int e = 0; e < _numeq_; ++e) y[e] = (real_t)a.y[ybase + (long long)k * _numeq_ + e];
#pragma unroll SODECL_PAR_UNROLL
        for (int j = 0; j < _numpar_; ++j) p[j] = (real_t)__ldg(a.p + pbase + (long long)k * _numpar_ + j);
        left = a.nsteps[item];
        if (a.counters) counter = a.counters[item];
    }
    while (__any_sync(0xffffffffu, item >= 0)) {
        if (item >= 0) {
            if (left > 0) {
                sodecl_advance(t, y, p, a.orbit_id ? a.orbit_id[item] : item, counter, passes, capped);
                --left;
            }
            if (left <= 0) {
                // store this orbit, take the next one (a count below zero
                // takes no step, like zero)
                sodecl_batch_store(a, item, item - begin, ybase, t, y, counter, passes, capped);
                passes = 0;
                capped = 0;
                k = atomicAdd(head, 1ULL);
                item = (k < count) ? begin + (long long)k : -1;
                if (item >= 0) {
                    t = (real_t)a.t[item];
#pragma unroll SODECL_EQ_UNROLL
                    for (int e = 0; e < _numeq_; ++e) y[e] = (real_t)a.y[ybase + (long long)k * _numeq_ + e];
#pragma unroll SODECL_PAR_UNROLL
                    for (int jj = 0; jj < _numpar_; ++jj) p[jj] = (real_t)__ldg(a.p + pbase + (long long)k * _numpar_ + jj);
                    left = a.nsteps[item];
                    counter = a.counters ? a.counters[item] : 0.0;
                }
            }
        }
    }
}
#else  // SODECL_LANES > 1
// Lanes per orbit (wide systems; the step functions of solvers.cuh): each
// group of SODECL_LANES lanes takes its own orbits from the class queue, one
// atomic per orbit, and integrates them with the group's barriers only, so the
// groups of a warp run orbits of different lengths independently.  The
// group's slot lies in the warp's shared memory region `warp_smem`.
__device__ __forceinline__ void sodecl_class_run(const sodecl_batch_args &a, const int cls, double *warp_smem)
{
    const int wl = threadIdx.x % 32;
    const int lane = wl % SODECL_LANES;
    const unsigned gmask = SODECL_LANES == 32 ? 0xffffffffu
                                              : ((1u << SODECL_LANES) - 1u) << (wl / SODECL_LANES * SODECL_LANES);
    const sodecl_lanes_view v = sodecl_lanes_slot(
        reinterpret_cast<real_t *>(warp_smem) + (wl / SODECL_LANES) * SODECL_SLOT, lane, gmask);
    const long long begin = a.begin[cls];
    const unsigned long long count = (unsigned long long)(a.end[cls] - begin);
    unsigned long long *head = a.head + cls;
    const long long ybase = a.ybase[cls], pbase = a.pbase[cls];
#pragma unroll 1
    for (;;) {
        unsigned long long k = 0;
        if (lane == 0) k = atomicAdd(head, 1ULL);
        k = __shfl_sync(gmask, k, 0, SODECL_LANES);
        if (k >= count) break;
        const long long item = begin + (long long)k;
        real_t yown[SODECL_ROWS];
#pragma unroll
        for (int q = 0; q < SODECL_ROWS; ++q) {
            const int r = lane + q * SODECL_LANES;
            yown[q] = (real_t)0;
            if (r < _numeq_) {
                yown[q] = (real_t)a.y[ybase + (long long)k * _numeq_ + r];
                v.Y[r] = yown[q];
            }
        }
        for (int j = lane; j < _numpar_; j += SODECL_LANES)
            v.P[j] = (real_t)__ldg(a.p + pbase + (long long)k * _numpar_ + j);
        __syncwarp(gmask);
        real_t t = (real_t)a.t[item];
        double counter = a.counters ? a.counters[item] : 0.0;
        const long long left = a.nsteps[item];
        const sodecl_i64 gid = a.orbit_id ? a.orbit_id[item] : item;
        sodecl_i64 passes = 0;
        int capped = 0;
#pragma unroll 1
        for (long long s = 0; s < left; ++s) sodecl_lanes_advance(t, yown, v, gid, counter, passes, capped);
        int nonfinite = 0;
#pragma unroll
        for (int q = 0; q < SODECL_ROWS; ++q) {
            const int r = lane + q * SODECL_LANES;
            if (r < _numeq_) {
                if (!isfinite(yown[q])) nonfinite = 1;
                a.y[ybase + (long long)k * _numeq_ + r] = (double)yown[q];
            }
        }
#pragma unroll
        for (int o = SODECL_LANES / 2; o > 0; o >>= 1) nonfinite |= __shfl_xor_sync(gmask, nonfinite, o, SODECL_LANES);
        if (lane == 0) {
            a.t[item] = (double)t;
            if (a.counters) a.counters[item] = counter;
            if (a.newton_passes) a.newton_passes[item] = passes;
            if (a.flags)
                a.flags[item] = (capped ? SODECL_FLAG_NEWTON_CAP : 0) | (nonfinite ? SODECL_FLAG_NONFINITE : 0);
        }
        __syncwarp(gmask);  // the slot is reused by the group's next orbit
    }
}
#endif  // SODECL_LANES
#endif
