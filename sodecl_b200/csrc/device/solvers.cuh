// Solver kernels of every SODECL NVRTC program (appended after the user's
// system file by the host front end, program.cpp).
//
// One thread integrates one orbit.  Its state, parameters and every stage
// vector live in registers: the sizes are the compile-time macros _numeq_,
// _numpar_ and _numnoi_ of the reference's program text, so all loops over
// equations unroll and no array is indexed dynamically.  A launch advances
// every orbit through record intervals [chunk_begin, chunk_end) of _numsteps_
// steps each and stores the state before each interval (and, on request,
// after the last) straight into the output in the reference's
// [record][equation][orbit] order: consecutive threads write consecutive
// addresses, so each warp store is fully coalesced.
//
// Config macros set by the front end:
//   SODECL_SOLVER        0 Euler-Maruyama, 1 Euler, 2 RK4, 3 implicit Euler,
//                        4 implicit midpoint (solver_Type numbering)
//   SODECL_FP32          compute in float
//   SODECL_FAST_DIV      FP64 through sodecl_f64 (exact reciprocal quotients)
//   SODECL_RECORD_F32    store records as float (else double)
//   SODECL_HAS_JACOBIAN  the system file defines calc_jacobian
//   SODECL_HAS_STOCH     the system file defines sode_system_stoch
//   SODECL_NEWTON_MAX    Newton pass limit (reference: 1000)
//   SODECL_BLOCK_MAX, SODECL_MIN_BLOCKS   launch bounds

#ifndef SODECL_MIN_BLOCKS
#define SODECL_MIN_BLOCKS 1
#endif

#if SODECL_RECORD_F32
typedef float sodecl_record_t;
#else
typedef double sodecl_record_t;
#endif

// IEEE quotient in every build, for divisors that change at every use (the
// banded solve's pivots), where a reciprocal could not be hoisted.
__device__ __forceinline__ double sodecl_qdiv(double a, double b) { return a / b; }
__device__ __forceinline__ float sodecl_qdiv(float a, float b) { return a / b; }
#if SODECL_FAST_DIV
__device__ __forceinline__ sodecl_f64 sodecl_qdiv(sodecl_f64 a, sodecl_f64 b) { return sodecl_f64(a.v / b.v); }
#endif

// Loops over equations unroll fully up to 16 equations (state, stages and
// the Jacobian's bands then live in registers); wider systems keep their
// arrays in local memory anyway, and full unrolling would only inflate the
// program, so they unroll by 4.
#undef SODECL_EQ_UNROLL
#define SODECL_EQ_UNROLL ((_numeq_) <= 16 ? (_numeq_) : 4)
#undef SODECL_PAR_UNROLL
#define SODECL_PAR_UNROLL ((_numpar_) < 1 ? 1 : ((_numpar_) <= 32 ? (_numpar_) : 4))

#define SODECL_NPAR_ALLOC ((_numpar_) > 0 ? (_numpar_) : 1)
#define SODECL_NNOI_ALLOC ((_numnoi_) > 0 ? (_numnoi_) : 1)

#define SODECL_FLAG_NEWTON_CAP 1
#define SODECL_FLAG_NONFINITE 2

#ifndef SODECL_STEPS_ONLY
struct sodecl_args {
    double *t;                  // [n] time of each orbit, in/out
    double *y;                  // [n][_numeq_] state, in/out
    const double *p;            // [n][_numpar_] parameters
    double *counters;           // [n] noise draw counters, in/out (solver 0)
    sodecl_record_t *records;   // record window base: [record][_numeq_][rec_stride]
    sodecl_i64 n;               // orbits in this launch
    sodecl_i64 orbit_offset;    // global index of this launch's orbit 0
    sodecl_i64 rec_stride;      // columns (orbits) of one record row
    sodecl_i64 rec_col0;        // column of this launch's orbit 0
    int chunk_begin;            // first record interval run by this launch
    int chunk_end;              // one past the last
    int rec_first;              // record index stored at `records`
    int write_final;            // also store record chunk_end
    sodecl_i64 *newton_passes;  // [n] accumulated Newton passes, or null
    int *flags;                 // [n] or-ed status flags, or null
};
#endif

// ---------------------------------------------------------------------------
// Explicit Euler: y1 = y0 + f(t, y0) h            (src/kernels/euler.cl:10-18)
__device__ __forceinline__ void sodecl_step_euler(real_t h, real_t t, real_t *y, real_t *ynew, real_t *p)
{
    sode_system(t, y, ynew, p);
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e)
        ynew[e] = y[e] + ynew[e] * h;
}

// RK4 with the reference's buffer reuse and accumulation order: the k1 slot
// accumulates k1 + 2 k2 + 2 k3 in place; result y + (acc + k4) h / 6.
//                                                   (src/kernels/rk4.cl:17-64)
__device__ __forceinline__ void sodecl_step_rk4(real_t h, real_t t, real_t *y, real_t *ynew, real_t *p)
{
    real_t stage[_numeq_], probe[_numeq_];
    sode_system(t, y, ynew, p);
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e) {
        stage[e] = ynew[e];
        probe[e] = y[e] + (h * (real_t)0.50) * stage[e];
    }
    sode_system(t + (real_t)0.50 * h, probe, stage, p);
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e) {
        ynew[e] = ynew[e] + (real_t)2.00 * stage[e];
        probe[e] = y[e] + (h * (real_t)0.50) * stage[e];
    }
    sode_system(t + (real_t)0.50 * h, probe, stage, p);
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e) {
        ynew[e] = ynew[e] + (real_t)2.00 * stage[e];
        probe[e] = y[e] + h * stage[e];
    }
    sode_system(t + h, probe, stage, p);
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e)
        ynew[e] = y[e] + (ynew[e] + stage[e]) * h / (real_t)6.00;
}

#if SODECL_SOLVER == 3 || SODECL_SOLVER == 4
#if !SODECL_HAS_JACOBIAN
#error "implicit solvers need calc_jacobian in the system file"
#endif
// The reference's banded elimination (src/kernels/ie.cl:10-48,
// im.cl:3-41): reads only the super-diagonal of rows 0.._numeq_-3, the
// sub-diagonal and the diagonal; the forward sweep pairs the super-diagonal
// entry of row i with the pivot of row i-1.  Kept exactly, because it
// defines the iterates.  Only three bands are read, so the compiler drops
// every other entry of the Jacobian (and the work computing it).
__device__ __forceinline__ void sodecl_band_solve(real_t (*m)[_numeq_], real_t *v, real_t *x)
{
    real_t up[_numeq_], lo[_numeq_], d[_numeq_];
#pragma unroll SODECL_EQ_UNROLL
    for (int i = 0; i < _numeq_; ++i) {
        up[i] = (i < _numeq_ - 2) ? m[i][(i + 1) % _numeq_] : (real_t)0;
        lo[i] = (i < _numeq_ - 1) ? m[(i + 1) % _numeq_][i] : (real_t)0;
        d[i] = m[i][i];
    }
#pragma unroll SODECL_EQ_UNROLL
    for (int i = 1; i < _numeq_; ++i) {
        const real_t f = sodecl_qdiv(up[i], d[i - 1]);
        d[i] = d[i] - f * lo[i - 1];
        v[i] = v[i] - f * v[i - 1];
    }
    x[_numeq_ - 1] = sodecl_qdiv(v[_numeq_ - 1], d[_numeq_ - 1]);
#pragma unroll SODECL_EQ_UNROLL
    for (int i = _numeq_ - 2; i >= 0; --i)
        x[i] = sodecl_qdiv(v[i] - lo[i] * x[i + 1], d[i]);
}

// Implicit Euler (src/kernels/ie.cl:50-117) and implicit midpoint
// (src/kernels/im.cl:43-118): iterate x <- x - M^-1 r with
//   IE: r = x - y - h f(t, x),         M = I - h J(x),          L1 test
//   IM: r = x - y - h f(t, (y+x)/2),   M = I - (h/2) J((y+x)/2), L2 test
// until the residual norm drops below _epsilon1_ or SODECL_NEWTON_MAX passes.
// Returns the passes taken; sets `capped` when the limit was reached.
__device__ __forceinline__ int sodecl_step_newton(real_t h, real_t t, real_t *y, real_t *ynew, real_t *p, int &capped)
{
    real_t x[_numeq_], f[_numeq_], r[_numeq_], dx[_numeq_];
    real_t m[_numeq_][_numeq_];
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e) x[e] = y[e];
    int pass = 0;
    bool done = false;
#pragma unroll 1
    for (pass = 0; pass < SODECL_NEWTON_MAX; ++pass) {
#if SODECL_SOLVER == 4
        real_t mid[_numeq_];
#pragma unroll SODECL_EQ_UNROLL
        for (int e = 0; e < _numeq_; ++e) mid[e] = (y[e] + x[e]) * (real_t)0.5;
        sode_system(t, mid, f, p);
#else
        sode_system(t, x, f, p);
#endif
        real_t norm = 0;
#pragma unroll SODECL_EQ_UNROLL
        for (int e = 0; e < _numeq_; ++e) {
            r[e] = x[e] - y[e] - f[e] * h;
#if SODECL_SOLVER == 4
            norm = norm + r[e] * r[e];
#else
            norm = norm + fabs(r[e]);
#endif
        }
#if SODECL_SOLVER == 4
        if (sqrt(norm) < (real_t)_epsilon1_) { done = true; break; }
        calc_jacobian(mid, m, p);
        const real_t scale = (real_t)(-0.50);
#else
        if (norm < (real_t)_epsilon1_) { done = true; break; }
        calc_jacobian(x, m, p);
        const real_t scale = (real_t)(-1.00);
#endif
#pragma unroll SODECL_EQ_UNROLL
        for (int i = 0; i < _numeq_; ++i) {
#pragma unroll SODECL_EQ_UNROLL
            for (int j = 0; j < _numeq_; ++j) m[i][j] = m[i][j] * scale * h;
            m[i][i] = m[i][i] + 1;
        }
        sodecl_band_solve(m, r, dx);
#pragma unroll SODECL_EQ_UNROLL
        for (int e = 0; e < _numeq_; ++e) x[e] = x[e] - dx[e];
    }
    if (!done) capped = 1;
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e) ynew[e] = x[e];
    return done ? pass + 1 : pass;
}
#endif

#if SODECL_SOLVER == 0
#if !SODECL_HAS_STOCH
#error "the stochastic solver needs sode_system_stoch in the system file"
#endif
// One step's Gaussian increments for orbit `gid`: ceil(_numnoi_/2) Threefry
// draws with counter {gid, counter++} and key {0, 0xf00dcafe}, each turned
// into a Box-Muller pair scaled by sqrt(h): cos partner first, the sin
// partner dropped for an odd count.  (stochastic_solver_caller.cl:31-66)
__device__ __forceinline__ void sodecl_draw_noise(sodecl_i64 gid, double &counter, real_t sqrt_h, real_t *noise)
{
#pragma unroll SODECL_EQ_UNROLL
    for (int c = 0; c < (_numnoi_ + 1) / 2; ++c) {
        sodecl_u64 w0, w1;
        sodecl_threefry2x64_20((sodecl_u64)gid, sodecl_counter_word(counter), SODECL_TF_KEY0, SODECL_TF_KEY1, w0, w1);
        counter = counter + 1;
        real_t n0, n1;
        sodecl_gaussian_pair<real_t>(w0, w1, sqrt_h, n0, n1);
        noise[2 * c] = n0;
        if (2 * c + 1 < _numnoi_)
            noise[2 * c + 1] = n1;
    }
}

// Euler-Maruyama: y1 = y0 + f h + g(y0, noise)     (stochastic_euler.cl:10-22)
__device__ __forceinline__ void sodecl_step_em(real_t h, real_t t, real_t *y, real_t *ynew, real_t *p, real_t *noise)
{
    real_t g[_numeq_];
    sode_system(t, y, ynew, p);
    sode_system_stoch(t, y, g, p, noise);
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e)
        ynew[e] = y[e] + ynew[e] * h + g[e];
}
#endif

// One step of the configured solver from (t, y): y <- y(t + h), t <- t + h,
// with t advanced as the reference's callers advance it
// (solver_caller.cl:38, stochastic_solver_caller.cl:71).
__device__ __forceinline__ void sodecl_advance(real_t &t, real_t *y, real_t *p, sodecl_i64 gid, double &counter,
                                               sodecl_i64 &passes, int &capped)
{
    real_t ynew[_numeq_];
#if SODECL_SOLVER == 1
    sodecl_step_euler(_m_dt_, t, y, ynew, p);
#elif SODECL_SOLVER == 2
    sodecl_step_rk4(_m_dt_, t, y, ynew, p);
#elif SODECL_SOLVER == 3 || SODECL_SOLVER == 4
    passes += sodecl_step_newton(_m_dt_, t, y, ynew, p, capped);
#elif SODECL_SOLVER == 0
    real_t noise[SODECL_NNOI_ALLOC];
    sodecl_draw_noise(gid, counter, sqrt((real_t)_m_dt_), noise);
    sodecl_step_em(_m_dt_, t, y, ynew, p, noise);
#endif
    t = t + _m_dt_;
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e) y[e] = ynew[e];
}

#ifndef SODECL_STEPS_ONLY
__device__ __forceinline__ void sodecl_store_record(const sodecl_args &a, int rec, sodecl_i64 i, const real_t *y, int &flags)
{
    sodecl_record_t *row = a.records + (sodecl_i64)(rec - a.rec_first) * _numeq_ * a.rec_stride + a.rec_col0 + i;
    bool finite = true;
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e) {
        finite = finite && isfinite(y[e]);
        __stcs(row + (sodecl_i64)e * a.rec_stride, (sodecl_record_t)y[e]);
    }
    if (!finite) flags |= SODECL_FLAG_NONFINITE;
}

extern "C" __global__ void __launch_bounds__(SODECL_BLOCK_MAX, SODECL_MIN_BLOCKS)
sodecl_orbits(const sodecl_args a)
{
    const sodecl_i64 i = (sodecl_i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n)
        return;

    real_t y[_numeq_];
    real_t p[SODECL_NPAR_ALLOC];
    real_t t = (real_t)a.t[i];
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e) y[e] = (real_t)a.y[i * _numeq_ + e];
#pragma unroll SODECL_PAR_UNROLL
    for (int k = 0; k < _numpar_; ++k) p[k] = (real_t)__ldg(a.p + i * _numpar_ + k);

    int flags = 0, capped = 0;
    sodecl_i64 passes = 0;
    const sodecl_i64 gid = a.orbit_offset + i;
#if SODECL_SOLVER == 0
    double counter = a.counters[i];
#else
    double counter = 0.0;
#endif

#pragma unroll 1
    for (int c = a.chunk_begin; c < a.chunk_end; ++c) {
        if (a.records)
            sodecl_store_record(a, c, i, y, flags);
#pragma unroll 1
        for (int s = 0; s < _numsteps_; ++s)
            sodecl_advance(t, y, p, gid, counter, passes, capped);
    }
    if (a.write_final && a.records)
        sodecl_store_record(a, a.chunk_end, i, y, flags);

    a.t[i] = (double)t;
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e) a.y[i * _numeq_ + e] = (double)y[e];
#if SODECL_SOLVER == 0
    a.counters[i] = counter;
#endif
    if (capped) flags |= SODECL_FLAG_NEWTON_CAP;
    if (a.newton_passes) a.newton_passes[i] += passes;
    if (a.flags && flags) a.flags[i] |= flags;
}
#endif  // SODECL_STEPS_ONLY
