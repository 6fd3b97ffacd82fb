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
// Big orbits go first, small ones fill the tail.

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
// Runs class `cls` until its queue is empty for every lane of the warp.
// Called by all 32 lanes of a warp together.
__device__ __forceinline__ void sodecl_class_run(const sodecl_batch_args &a, const int cls)
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
            if (left == 0) {
                // store this orbit, take the next one
                const long long j = item - begin;
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
#endif
