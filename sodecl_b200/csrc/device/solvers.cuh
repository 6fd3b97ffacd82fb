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
//   SODECL_FAST_DIV      arithmetic through sodecl_num (exact reciprocal quotients)
//   SODECL_RECORD_F32    store records as float (else double)
//   SODECL_HAS_JACOBIAN  the system file defines calc_jacobian
//   SODECL_HAS_STOCH     the system file defines sode_system_stoch
//   SODECL_NEWTON_MAX    Newton pass limit (reference: 1000)
//   SODECL_BLOCK_MAX, SODECL_MIN_BLOCKS   launch bounds
//   SODECL_LANES         lanes per orbit: 1 (one thread per orbit, the
//                        default) or 2..32, a power of two (wide systems;
//                        see the kernel at the end of this file)
//   SODECL_HAS_ROW, SODECL_HAS_STOCH_ROW, SODECL_HAS_JAC_BAND  the system
//                        file defines sode_system_row / sode_system_stoch_row /
//                        calc_jacobian_band
//   SODECL_HAS_ROW_BAND  the system file defines sode_system_row_band
//   SODECL_PAIR_STORES   one-thread kernel: records written two orbits per
//                        vector store (sodecl_store_pairs)

#ifndef SODECL_MIN_BLOCKS
#define SODECL_MIN_BLOCKS 1
#endif
template <class T> struct sodecl_pair_of;
template <> struct sodecl_pair_of<double> { typedef double2 type; };
template <> struct sodecl_pair_of<float> { typedef float2 type; };
#ifndef SODECL_LANES
#define SODECL_LANES 1
#endif
#ifndef SODECL_PAIR_STORES
#define SODECL_PAIR_STORES 0
#endif
#if SODECL_PAIR_STORES && (SODECL_LANES != 1 || SODECL_SOLVER > 2)
#error "paired record stores serve the one-thread kernel of the explicit and stochastic solvers"
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
__device__ __forceinline__ sodecl_num sodecl_qdiv(sodecl_num a, sodecl_num b) { return sodecl_num(a.v / b.v); }
#endif

// A pivot that divides twice (the banded solve's forward multiplier and back
// substitution): in reciprocal-division programs its reciprocal is taken once
// and each quotient finished from it (sodecl_div_by, the IEEE quotient's bits).
#if SODECL_FAST_DIV
__device__ __forceinline__ real_t sodecl_pivot_rcp(real_t d) { return sodecl_num((sodecl_num_t)1 / d.v); }
__device__ __forceinline__ real_t sodecl_pdiv(real_t a, real_t d, real_t r) { return sodecl_num(sodecl_div_by(a.v, d.v, r.v)); }
#else
__device__ __forceinline__ real_t sodecl_pivot_rcp(real_t d) { return d; }
__device__ __forceinline__ real_t sodecl_pdiv(real_t a, real_t d, real_t) { return sodecl_qdiv(a, d); }
#endif

// 0 / d, IEEE: a zero with d's sign; NaN (through the division itself) for a
// zero or NaN d.  The banded solve pads its super-diagonal with literal zeros.
__device__ __forceinline__ real_t sodecl_zero_over(real_t d)
{
    if (d == (real_t)0 || d != d) return sodecl_qdiv((real_t)0, d);
    return copysign((real_t)0, d);
}

// The implicit midpoint's stop test sqrt(norm) < _epsilon1_.  The square root
// is correctly rounded and monotone, so the test holds exactly when norm is
// below the least value whose root reaches _epsilon1_; the host computes that
// bound (SODECL_L2_BOUND) whenever it is a normal number.
#ifdef SODECL_L2_BOUND
__device__ __forceinline__ bool sodecl_l2_below(real_t norm) { return norm < (real_t)SODECL_L2_BOUND; }
#else
__device__ __forceinline__ bool sodecl_l2_below(real_t norm) { return sqrt(norm) < (real_t)_epsilon1_; }
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
// x2, x3, x4 (optional) receive the stage inputs y + (h/2) k1, y + (h/2) k2,
// y + h k3 (the adjoint reuses them).             (src/kernels/rk4.cl:17-64)
__device__ __forceinline__ void sodecl_step_rk4(real_t h, real_t t, real_t *y, real_t *ynew, real_t *p,
                                                real_t *x2 = nullptr, real_t *x3 = nullptr, real_t *x4 = nullptr)
{
    real_t stage[_numeq_], probe[_numeq_];
    sode_system(t, y, ynew, p);
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e) {
        stage[e] = ynew[e];
        probe[e] = y[e] + (h * (real_t)0.50) * stage[e];
        if (x2) x2[e] = probe[e];
    }
    sode_system(t + (real_t)0.50 * h, probe, stage, p);
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e) {
        ynew[e] = ynew[e] + (real_t)2.00 * stage[e];
        probe[e] = y[e] + (h * (real_t)0.50) * stage[e];
        if (x3) x3[e] = probe[e];
    }
    sode_system(t + (real_t)0.50 * h, probe, stage, p);
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e) {
        ynew[e] = ynew[e] + (real_t)2.00 * stage[e];
        probe[e] = y[e] + h * stage[e];
        if (x4) x4[e] = probe[e];
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
    // rd[i]: the reciprocal of pivot i, for the pivots whose row below has a
    // super-diagonal entry (i + 1 < _numeq_ - 2), which divide twice
    real_t rd[_numeq_];
#pragma unroll SODECL_EQ_UNROLL
    for (int i = 1; i < _numeq_; ++i) {
        real_t f;
        if (i < _numeq_ - 2) {
            rd[i - 1] = sodecl_pivot_rcp(d[i - 1]);
            f = sodecl_pdiv(up[i], d[i - 1], rd[i - 1]);
        } else {
            f = sodecl_zero_over(d[i - 1]);
        }
        d[i] = d[i] - f * lo[i - 1];
        v[i] = v[i] - f * v[i - 1];
    }
    x[_numeq_ - 1] = sodecl_qdiv(v[_numeq_ - 1], d[_numeq_ - 1]);
#pragma unroll SODECL_EQ_UNROLL
    for (int i = _numeq_ - 2; i >= 0; --i) {
        const real_t num = v[i] - lo[i] * x[i + 1];
        x[i] = (i + 1 < _numeq_ - 2) ? sodecl_pdiv(num, d[i], rd[i]) : sodecl_qdiv(num, d[i]);
    }
}

// Implicit Euler (src/kernels/ie.cl:50-117) and implicit midpoint
// (src/kernels/im.cl:43-118): iterate x <- x - M^-1 r with
//   IE: r = x - y - h f(t, x),         M = I - h J(x),          L1 test
//   IM: r = x - y - h f(t, (y+x)/2),   M = I - (h/2) J((y+x)/2), L2 test
// until the residual norm drops below _epsilon1_ or SODECL_NEWTON_MAX passes.
//
// One pass at iterate x: true when the residual norm is below _epsilon1_ (x
// unchanged), else x <- x - M^-1 r and false.
__device__ __forceinline__ bool sodecl_newton_pass(real_t h, real_t t, real_t *y, real_t *x, real_t *p)
{
    real_t f[_numeq_], r[_numeq_], dx[_numeq_];
    real_t m[_numeq_][_numeq_];
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
    if (sodecl_l2_below(norm)) return true;
    calc_jacobian(mid, m, p);
    const real_t scale = (real_t)(-0.50);
#else
    if (norm < (real_t)_epsilon1_) return true;
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
    return false;
}

// One step from y into ynew.  Returns the passes taken (residual evaluations);
// sets `capped` when the limit was reached.
__device__ __forceinline__ int sodecl_step_newton(real_t h, real_t t, real_t *y, real_t *ynew, real_t *p, int &capped)
{
    real_t x[_numeq_];
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e) x[e] = y[e];
    int pass = 0;
    bool done = false;
#pragma unroll 1
    for (pass = 0; pass < SODECL_NEWTON_MAX; ++pass)
        if (sodecl_newton_pass(h, t, y, x, p)) { done = true; break; }
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

#if SODECL_SOLVER == 5
#if SODECL_LANES > 1 || defined(SODECL_STEPS_ONLY)
#error "the adaptive solver runs one thread per orbit, in single-system programs"
#endif
// Dormand-Prince 5(4) with adaptive steps (J. R. Dormand, P. J. Prince, "A
// family of embedded Runge-Kutta formulae", J. Comput. Appl. Math. 6(1), 1980;
// step control as in Hairer, Norsett, Wanner, "Solving Ordinary Differential
// Equations I", II.4).  No counterpart in the reference, which lists
// variable-step solvers as future work.
//
// The adaptive solver integrates each record interval [t, t + span) in
// attempted steps, the last cut to land on the interval's end exactly.  A
// step of size hh is accepted when the RMS over equations of
// e_i / (atol + rtol max(|y_i|, |y5_i|)) is at most 1 (e the difference of
// the embedded 5th- and 4th-order results); the next step is
// hh * min(5, max(0.2, 0.9 err^(-1/5))), not larger than hh after a
// rejection; a step cut to the interval's end leaves the proposal `h` as it
// was.  The first stage is re-evaluated at each interval's start, so results
// do not depend on how intervals are grouped into launches.  An interval that
// needs more than SODECL_MAX_STEPS attempts, or a step too small to advance
// t, fails: the state becomes NaN.
#define SODECL_DP(c) ((real_t)(c))
struct sodecl_dp_state {
    real_t k1[_numeq_];  // the first stage at (t, y) (first same as last)
    real_t t_end;        // the interval's end
    int n;               // attempts in this interval
    bool rejected;       // the last attempt was rejected
};

// Opens the interval of length span from t.  Returns false when it needs no
// attempt: a diverged orbit stays as it is (t moves to the interval's end),
// and an interval too short to advance t ends at once.
__device__ __forceinline__ bool sodecl_dp_begin(real_t &t, const real_t *y, real_t *p, real_t &h, const real_t span,
                                                sodecl_dp_state &st)
{
    st.t_end = t + span;
    bool finite = true;
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e) finite = finite && isfinite(y[e]);
    if (!finite) {
        t = st.t_end;
        return false;
    }
    if (!(h > (real_t)0) || !isfinite(h)) h = (real_t)_m_dt_;
    sode_system(t, const_cast<real_t *>(y), st.k1, p);
    st.n = 0;
    st.rejected = false;
    return t < st.t_end;
}

// One attempted step of the open interval.  Returns 0 while the interval
// goes on, 1 when it has reached its end, 2 when it failed (state NaN, t at
// the interval's end).
__device__ __forceinline__ int sodecl_dp_attempt(real_t &t, real_t *y, real_t *p, real_t &h, sodecl_dp_state &st,
                                                 sodecl_i64 &accepted)
{
    real_t k2[_numeq_], k3[_numeq_], k4[_numeq_], k5[_numeq_], k6[_numeq_], k7[_numeq_];
    real_t yt[_numeq_], y5[_numeq_];
    const real_t t_end = st.t_end;
    const bool last = t + h >= t_end;
    const real_t hh = last ? t_end - t : h;
    if (st.n >= SODECL_MAX_STEPS || !(hh > (real_t)0) || t + hh == t) {
#pragma unroll SODECL_EQ_UNROLL
        for (int e = 0; e < _numeq_; ++e) y[e] = (real_t)__longlong_as_double(0x7ff8000000000000ULL);
        t = t_end;
        return 2;
    }
    real_t *k1 = st.k1;
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e) yt[e] = y[e] + hh * (SODECL_DP(1.0 / 5.0) * k1[e]);
    sode_system(t + SODECL_DP(1.0 / 5.0) * hh, yt, k2, p);
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e)
        yt[e] = y[e] + hh * (SODECL_DP(3.0 / 40.0) * k1[e] + SODECL_DP(9.0 / 40.0) * k2[e]);
    sode_system(t + SODECL_DP(3.0 / 10.0) * hh, yt, k3, p);
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e)
        yt[e] = y[e] + hh * (SODECL_DP(44.0 / 45.0) * k1[e] + SODECL_DP(-56.0 / 15.0) * k2[e] +
                             SODECL_DP(32.0 / 9.0) * k3[e]);
    sode_system(t + SODECL_DP(4.0 / 5.0) * hh, yt, k4, p);
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e)
        yt[e] = y[e] + hh * (SODECL_DP(19372.0 / 6561.0) * k1[e] + SODECL_DP(-25360.0 / 2187.0) * k2[e] +
                             SODECL_DP(64448.0 / 6561.0) * k3[e] + SODECL_DP(-212.0 / 729.0) * k4[e]);
    sode_system(t + SODECL_DP(8.0 / 9.0) * hh, yt, k5, p);
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e)
        yt[e] = y[e] + hh * (SODECL_DP(9017.0 / 3168.0) * k1[e] + SODECL_DP(-355.0 / 33.0) * k2[e] +
                             SODECL_DP(46732.0 / 5247.0) * k3[e] + SODECL_DP(49.0 / 176.0) * k4[e] +
                             SODECL_DP(-5103.0 / 18656.0) * k5[e]);
    sode_system(t + hh, yt, k6, p);
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e)
        y5[e] = y[e] + hh * (SODECL_DP(35.0 / 384.0) * k1[e] + SODECL_DP(500.0 / 1113.0) * k3[e] +
                             SODECL_DP(125.0 / 192.0) * k4[e] + SODECL_DP(-2187.0 / 6784.0) * k5[e] +
                             SODECL_DP(11.0 / 84.0) * k6[e]);
    sode_system(t + hh, y5, k7, p);
    real_t acc = 0;
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e) {
        const real_t err = hh * (SODECL_DP(71.0 / 57600.0) * k1[e] + SODECL_DP(-71.0 / 16695.0) * k3[e] +
                                 SODECL_DP(71.0 / 1920.0) * k4[e] + SODECL_DP(-17253.0 / 339200.0) * k5[e] +
                                 SODECL_DP(22.0 / 525.0) * k6[e] + SODECL_DP(-1.0 / 40.0) * k7[e]);
        const real_t sc = SODECL_DP(SODECL_ATOL) + SODECL_DP(SODECL_RTOL) * fmax(fabs(y[e]), fabs(y5[e]));
        const real_t q = err / sc;
        acc = acc + q * q;
    }
    const real_t err = sqrt(acc / (real_t)_numeq_);
    real_t fac = (err > (real_t)0) ? SODECL_DP(0.9) * exp(SODECL_DP(-0.2) * log(err)) : SODECL_DP(5.0);
    fac = fmin(SODECL_DP(5.0), fmax(SODECL_DP(0.2), fac));
    if (err <= (real_t)1) {
        t = last ? t_end : t + hh;
#pragma unroll SODECL_EQ_UNROLL
        for (int e = 0; e < _numeq_; ++e) {
            y[e] = y5[e];
            k1[e] = k7[e];
        }
        ++accepted;
        if (!last) h = hh * (st.rejected ? fmin((real_t)1, fac) : fac);
        st.rejected = false;
    } else {
        // a NaN error shrinks the step too
        h = hh * (err == err ? fmin((real_t)1, fac) : SODECL_DP(0.2));
        st.rejected = true;
    }
    ++st.n;
    return t < t_end ? 0 : 1;
}
#undef SODECL_DP
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

#if SODECL_LANES > 1
// ---------------------------------------------------------------------------
// Lanes per orbit, for wide systems.  With one thread per orbit, a system of
// dozens of equations keeps its state and stage vectors in local memory, and
// every right-hand-side term goes through it.  Here SODECL_LANES consecutive
// lanes of a warp share one orbit: lane l owns the rows l, l + L, l + 2L, ...
// and evaluates them with the system file's per-row functions --
// `sode_system_row(i, t, y, p)` (= yout[i] of sode_system),
// `sode_system_stoch_row(i, t, y, p, noise)` and, for the implicit solvers,
// `calc_jacobian_band(i, y, band, p)` (band = row i's entries in columns
// i-1, i, i+1 of calc_jacobian) -- against the orbit's vectors staged in
// shared memory, where the lanes of a group read the same word (a broadcast).
// Every row sees the single-thread solver's arithmetic, and sums over rows
// (the Newton residual norm) are taken in the same order, gathered with warp
// shuffles, so results are the same as one thread per orbit.  Noise pairs are
// drawn by the lanes in turn with the counter values the single thread uses;
// the banded solve, a sequential recurrence, runs on the group's first lane.
#if SODECL_LANES > 32 || (SODECL_LANES & (SODECL_LANES - 1)) != 0
#error "SODECL_LANES must be a power of two up to 32"
#endif
#if !SODECL_HAS_ROW
#error "lanes per orbit need sode_system_row in the system file"
#endif
#if SODECL_SOLVER == 0 && !SODECL_HAS_STOCH_ROW
#error "lanes per orbit with the stochastic solver need sode_system_stoch_row in the system file"
#endif
#if (SODECL_SOLVER == 3 || SODECL_SOLVER == 4) && !SODECL_HAS_JAC_BAND
#error "lanes per orbit with an implicit solver need calc_jacobian_band in the system file"
#endif

#undef SODECL_ROWS
#undef SODECL_NPAIRS
#undef SODECL_LANES_NVEC
#undef SODECL_SLOT_RAW
#undef SODECL_SLOT
#define SODECL_ROWS ((_numeq_ + SODECL_LANES - 1) / SODECL_LANES)
#define SODECL_NPAIRS ((_numnoi_ + 1) / 2)
// One orbit's shared slot, in real_t words: SODECL_LANES_NVEC vectors of
// _numeq_ (state; RK4: two probes; Newton: iterate, midpoint, diagonal,
// super- and sub-diagonal, right-hand side, update), the parameters and the
// noise, padded to an odd length so that groups of a warp reading word j of
// their slots hit different banks.
#if SODECL_SOLVER == 2
#define SODECL_LANES_NVEC 3
#elif SODECL_SOLVER == 3 || SODECL_SOLVER == 4
#define SODECL_LANES_NVEC 8
#else
#define SODECL_LANES_NVEC 1
#endif
#define SODECL_SLOT_RAW (SODECL_LANES_NVEC * (_numeq_) + (_numpar_) + (_numnoi_))
#define SODECL_SLOT ((SODECL_SLOT_RAW) | 1)

struct sodecl_lanes_view {
    real_t *Y;       // state
    real_t *A, *B;   // RK4: probes; Newton: iterate x, midpoint
    real_t *D, *UP, *LO, *V, *DX;  // Newton: the banded system and its solution
    real_t *P;       // parameters
    real_t *NZ;      // noise of the step
    int lane;        // lane within the group
    unsigned mask;   // lanes taking part in the group's barriers and shuffles
};

__device__ __forceinline__ sodecl_lanes_view sodecl_lanes_slot(real_t *slot, int lane, unsigned mask)
{
    sodecl_lanes_view v;
    v.Y = slot;
    v.A = slot + (SODECL_LANES_NVEC > 1 ? 1 : 0) * _numeq_;
    v.B = slot + (SODECL_LANES_NVEC > 2 ? 2 : 0) * _numeq_;
    v.D = slot + (SODECL_LANES_NVEC > 3 ? 3 : 0) * _numeq_;
    v.UP = slot + (SODECL_LANES_NVEC > 4 ? 4 : 0) * _numeq_;
    v.LO = slot + (SODECL_LANES_NVEC > 5 ? 5 : 0) * _numeq_;
    v.V = slot + (SODECL_LANES_NVEC > 6 ? 6 : 0) * _numeq_;
    v.DX = slot + (SODECL_LANES_NVEC > 7 ? 7 : 0) * _numeq_;
    v.P = slot + SODECL_LANES_NVEC * _numeq_;
    v.NZ = v.P + _numpar_;
    v.lane = lane;
    v.mask = mask;
    return v;
}

__device__ __forceinline__ double sodecl_shfl(unsigned m, double x, int src) { return __shfl_sync(m, x, src, SODECL_LANES); }
__device__ __forceinline__ float sodecl_shfl(unsigned m, float x, int src) { return __shfl_sync(m, x, src, SODECL_LANES); }
#if SODECL_FAST_DIV
__device__ __forceinline__ sodecl_num sodecl_shfl(unsigned m, sodecl_num x, int src)
{
    return sodecl_num(__shfl_sync(m, x.v, src, SODECL_LANES));
}
#endif

// The counter after c increments of 1.0, as c sequential additions give it:
// one addition when the counter is an integer and every partial sum stays
// within +-2^53 (all exact), else the additions themselves.
__device__ __forceinline__ double sodecl_counter_plus(double counter, int c)
{
    if (counter == floor(counter) && counter >= -9007199254740992.0 && counter <= 9007199254740992.0 - (double)c)
        return counter + (double)c;
    double cc = counter;
    for (int q = 0; q < c; ++q) cc = cc + 1.0;
    return cc;
}

#if SODECL_SOLVER == 3 || SODECL_SOLVER == 4
// sodecl_band_solve on the shared band system (D, UP, LO, V), in two parts: the
// forward sweep, a recurrence through the pivots, by one lane (IEEE quotients
// on the recurrence's chain: a reciprocal there was measured slower), and
// sodecl_lanes_back_subst -> DX.
__device__ __forceinline__ void sodecl_lanes_band_solve(const sodecl_lanes_view &v)
{
    real_t dprev = v.D[0], vprev = v.V[0];
#pragma unroll 1
    for (int i = 1; i < _numeq_; ++i) {
        const real_t up = (i < _numeq_ - 2) ? v.UP[i] : (real_t)0;
        const real_t f = sodecl_qdiv(up, dprev);
        const real_t lo = v.LO[i - 1];
        dprev = v.D[i] - f * lo;
        vprev = v.V[i] - f * vprev;
        v.D[i] = dprev;
        v.V[i] = vprev;
    }
}

// The back substitution, after the forward sweep: every lane of the group
// takes the reciprocals of its rows' pivots at once (into UP, which only the
// forward sweep reads), then the first lane finishes each quotient from them
// (sodecl_pdiv: the IEEE quotient's bits; a plain quotient in other builds),
// which shortens its dependent chain.  Called by every lane of the group.
__device__ __forceinline__ void sodecl_lanes_back_subst(const sodecl_lanes_view &v)
{
#pragma unroll
    for (int k = 0; k < SODECL_ROWS; ++k) {
        const int row = v.lane + k * SODECL_LANES;
        if (row < _numeq_) v.UP[row] = sodecl_pivot_rcp(v.D[row]);
    }
    __syncwarp(v.mask);
    if (v.lane == 0) {
        real_t x = sodecl_qdiv(v.V[_numeq_ - 1], v.D[_numeq_ - 1]);
        v.DX[_numeq_ - 1] = x;
#pragma unroll 1
        for (int i = _numeq_ - 2; i >= 0; --i) {
            x = sodecl_pdiv(v.V[i] - v.LO[i] * x, v.D[i], v.UP[i]);
            v.DX[i] = x;
        }
    }
}

// sodecl_step_newton, row by row (src/kernels/ie.cl:50-117, im.cl:43-118).
__device__ __forceinline__ int sodecl_lanes_newton(real_t h, real_t t, const real_t *yown, real_t *xnew,
                                                   const sodecl_lanes_view &v, int &capped)
{
    real_t x[SODECL_ROWS], r[SODECL_ROWS];
#pragma unroll
    for (int k = 0; k < SODECL_ROWS; ++k) {
        const int row = v.lane + k * SODECL_LANES;
        x[k] = (real_t)0;
        r[k] = (real_t)0;
        if (row < _numeq_) {
            x[k] = yown[k];
            v.A[row] = x[k];
        }
    }
    __syncwarp(v.mask);
    int pass = 0;
    bool done = false;
#pragma unroll 1
    for (pass = 0; pass < SODECL_NEWTON_MAX; ++pass) {
#if SODECL_SOLVER == 4
        real_t *at = v.B;
#pragma unroll
        for (int k = 0; k < SODECL_ROWS; ++k) {
            const int row = v.lane + k * SODECL_LANES;
            if (row < _numeq_) v.B[row] = (yown[k] + x[k]) * (real_t)0.5;
        }
        __syncwarp(v.mask);
#else
        real_t *at = v.A;
#endif
#if SODECL_HAS_ROW_BAND
        // the row's right-hand side and its band entries from one evaluation
        // (the Jacobian is taken at the residual's point), used if the pass
        // does not converge
        real_t bands[SODECL_ROWS][3];
#pragma unroll
        for (int k = 0; k < SODECL_ROWS; ++k) {
            const int row = v.lane + k * SODECL_LANES;
            if (row < _numeq_) r[k] = x[k] - yown[k] - sode_system_row_band(row, t, at, bands[k], v.P) * h;
        }
#else
#pragma unroll
        for (int k = 0; k < SODECL_ROWS; ++k) {
            const int row = v.lane + k * SODECL_LANES;
            if (row < _numeq_) r[k] = x[k] - yown[k] - sode_system_row(row, t, at, v.P) * h;
        }
#endif
        // the residual norm in row order, every lane of the group the same
        real_t norm = 0;
#pragma unroll
        for (int e = 0; e < _numeq_; ++e) {
            const real_t re = sodecl_shfl(v.mask, r[e / SODECL_LANES], e % SODECL_LANES);
#if SODECL_SOLVER == 4
            norm = norm + re * re;
#else
            norm = norm + fabs(re);
#endif
        }
#if SODECL_SOLVER == 4
        if (sodecl_l2_below(norm)) { done = true; break; }
        const real_t scale = (real_t)(-0.50);
#else
        if (norm < (real_t)_epsilon1_) { done = true; break; }
        const real_t scale = (real_t)(-1.00);
#endif
#pragma unroll
        for (int k = 0; k < SODECL_ROWS; ++k) {
            const int row = v.lane + k * SODECL_LANES;
            if (row < _numeq_) {
#if SODECL_HAS_ROW_BAND
                const real_t *band = bands[k];
#else
                real_t band[3];
                calc_jacobian_band(row, at, band, v.P);
#endif
                real_t d = band[1] * scale * h;
                d = d + 1;
                v.D[row] = d;
                if (row < _numeq_ - 2) v.UP[row] = band[2] * scale * h;
                if (row > 0) v.LO[row - 1] = band[0] * scale * h;
                v.V[row] = r[k];
            }
        }
        __syncwarp(v.mask);
        if (v.lane == 0) sodecl_lanes_band_solve(v);
        __syncwarp(v.mask);
        sodecl_lanes_back_subst(v);
        __syncwarp(v.mask);
#pragma unroll
        for (int k = 0; k < SODECL_ROWS; ++k) {
            const int row = v.lane + k * SODECL_LANES;
            if (row < _numeq_) {
                x[k] = x[k] - v.DX[row];
                v.A[row] = x[k];
            }
        }
        __syncwarp(v.mask);
    }
    if (!done) capped = 1;
#pragma unroll
    for (int k = 0; k < SODECL_ROWS; ++k) xnew[k] = x[k];
    return done ? pass + 1 : pass;
}
#endif

// One step of the configured solver for the group's orbit: every lane of the
// group (all of v.mask) calls it together.
__device__ __forceinline__ void sodecl_lanes_advance(real_t &t, real_t *yown, const sodecl_lanes_view &v, sodecl_i64 gid,
                                                     double &counter, sodecl_i64 &passes, int &capped)
{
    const real_t h = _m_dt_;
    real_t ynew[SODECL_ROWS];
#if SODECL_SOLVER == 1
    // src/kernels/euler.cl:10-18, row by row
#pragma unroll
    for (int k = 0; k < SODECL_ROWS; ++k) {
        const int r = v.lane + k * SODECL_LANES;
        if (r < _numeq_) ynew[k] = yown[k] + sode_system_row(r, t, v.Y, v.P) * h;
    }
#elif SODECL_SOLVER == 2
    // src/kernels/rk4.cl:17-64, row by row; the probe alternates between two
    // buffers so that one barrier per stage suffices
    real_t stage[SODECL_ROWS];
#pragma unroll
    for (int k = 0; k < SODECL_ROWS; ++k) {
        const int r = v.lane + k * SODECL_LANES;
        if (r < _numeq_) {
            ynew[k] = sode_system_row(r, t, v.Y, v.P);
            stage[k] = ynew[k];
            v.A[r] = yown[k] + (h * (real_t)0.50) * stage[k];
        }
    }
    __syncwarp(v.mask);
#pragma unroll
    for (int k = 0; k < SODECL_ROWS; ++k) {
        const int r = v.lane + k * SODECL_LANES;
        if (r < _numeq_) {
            stage[k] = sode_system_row(r, t + (real_t)0.50 * h, v.A, v.P);
            ynew[k] = ynew[k] + (real_t)2.00 * stage[k];
            v.B[r] = yown[k] + (h * (real_t)0.50) * stage[k];
        }
    }
    __syncwarp(v.mask);
#pragma unroll
    for (int k = 0; k < SODECL_ROWS; ++k) {
        const int r = v.lane + k * SODECL_LANES;
        if (r < _numeq_) {
            stage[k] = sode_system_row(r, t + (real_t)0.50 * h, v.B, v.P);
            ynew[k] = ynew[k] + (real_t)2.00 * stage[k];
            v.A[r] = yown[k] + h * stage[k];
        }
    }
    __syncwarp(v.mask);
#pragma unroll
    for (int k = 0; k < SODECL_ROWS; ++k) {
        const int r = v.lane + k * SODECL_LANES;
        if (r < _numeq_) {
            stage[k] = sode_system_row(r, t + h, v.A, v.P);
            ynew[k] = yown[k] + (ynew[k] + stage[k]) * h / (real_t)6.00;
        }
    }
#elif SODECL_SOLVER == 3 || SODECL_SOLVER == 4
    passes += sodecl_lanes_newton(h, t, yown, ynew, v, capped);
#elif SODECL_SOLVER == 0
    // stochastic_solver_caller.cl:31-66: pair c of this step uses the counter
    // advanced c times; the lanes draw the pairs in turn
    const real_t sqrt_h = sqrt((real_t)_m_dt_);
#pragma unroll 1
    for (int c = v.lane; c < SODECL_NPAIRS; c += SODECL_LANES) {
        sodecl_u64 w0, w1;
        sodecl_threefry2x64_20((sodecl_u64)gid, sodecl_counter_word(sodecl_counter_plus(counter, c)), SODECL_TF_KEY0,
                               SODECL_TF_KEY1, w0, w1);
        real_t n0, n1;
        sodecl_gaussian_pair<real_t>(w0, w1, sqrt_h, n0, n1);
        v.NZ[2 * c] = n0;
        if (2 * c + 1 < _numnoi_) v.NZ[2 * c + 1] = n1;
    }
    counter = sodecl_counter_plus(counter, SODECL_NPAIRS);
    __syncwarp(v.mask);
    // stochastic_euler.cl:10-22, row by row
#pragma unroll
    for (int k = 0; k < SODECL_ROWS; ++k) {
        const int r = v.lane + k * SODECL_LANES;
        if (r < _numeq_) {
            const real_t f = sode_system_row(r, t, v.Y, v.P);
            const real_t g = sode_system_stoch_row(r, t, v.Y, v.P, v.NZ);
            ynew[k] = yown[k] + f * h + g;
        }
    }
#endif
    (void)gid;
    (void)counter;
    (void)passes;
    (void)capped;
    t = t + _m_dt_;
    __syncwarp(v.mask);  // the group is done reading the state, probes and noise
#pragma unroll
    for (int k = 0; k < SODECL_ROWS; ++k) {
        const int r = v.lane + k * SODECL_LANES;
        if (r < _numeq_) {
            yown[k] = ynew[k];
            v.Y[r] = ynew[k];
        }
    }
    __syncwarp(v.mask);
}
#endif  // SODECL_LANES > 1

#ifndef SODECL_STEPS_ONLY
#if SODECL_PAIR_STORES
// Paired stores: the two threads of orbits 2k and 2k+1 (lanes 2j, 2j+1) swap
// one value per two equations with a shuffle, so that the even thread writes
// equation e of both orbits and the odd thread equation e+1 of both, each as
// one vector store (16 bytes for double records): half the store
// instructions, the same bytes and sectors.  Needs an even block size, an
// even first column and row stride and a base aligned to a pair, all uniform
// across the launch; an orbit whose partner is past the end stores alone.
__device__ __forceinline__ bool sodecl_store_pairs(const sodecl_args &a, sodecl_record_t *row, sodecl_i64 i,
                                                   const real_t *y)
{
    typedef typename sodecl_pair_of<sodecl_record_t>::type pair_t;
    const bool layout = (blockDim.x % 2u) == 0u && (a.rec_col0 % 2) == 0 && (a.rec_stride % 2) == 0 &&
                        ((unsigned long long)a.records % sizeof(pair_t)) == 0ull;
    const int odd = (int)(i & 1);
    if (!layout || (!odd && i + 1 >= a.n)) return false;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned pair_mask = 3u << (lane & 30u);
    sodecl_record_t *base = row - odd;  // column of the pair's even orbit
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e + 1 < _numeq_; e += 2) {
        const sodecl_record_t v0 = (sodecl_record_t)y[e], v1 = (sodecl_record_t)y[e + 1];
        const sodecl_record_t got = __shfl_xor_sync(pair_mask, odd ? v0 : v1, 1);
        pair_t w;
        w.x = odd ? got : v0;
        w.y = odd ? v1 : got;
        __stcs(reinterpret_cast<pair_t *>(base + (sodecl_i64)(e + odd) * a.rec_stride), w);
    }
    if (_numeq_ % 2) __stcs(row + (sodecl_i64)(_numeq_ - 1) * a.rec_stride, (sodecl_record_t)y[_numeq_ - 1]);
    return true;
}
#endif

__device__ __forceinline__ void sodecl_store_record(const sodecl_args &a, int rec, sodecl_i64 i, const real_t *y, int &flags)
{
    sodecl_record_t *row = a.records + (sodecl_i64)(rec - a.rec_first) * _numeq_ * a.rec_stride + a.rec_col0 + i;
    bool finite = true;
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e) finite = finite && isfinite(y[e]);
    if (!finite) flags |= SODECL_FLAG_NONFINITE;
#if SODECL_PAIR_STORES
    if (sodecl_store_pairs(a, row, i, y)) return;
#endif
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e) __stcs(row + (sodecl_i64)e * a.rec_stride, (sodecl_record_t)y[e]);
}

// The end of an orbit's launch: the closing record (on request), the state,
// draw counter, Newton pass count and flags.
__device__ __forceinline__ void sodecl_orbit_out(const sodecl_args &a, sodecl_i64 i, real_t t, const real_t *y,
                                                 double counter, sodecl_i64 passes, int capped, int flags)
{
    if (a.write_final && a.records)
        sodecl_store_record(a, a.chunk_end, i, y, flags);
    a.t[i] = (double)t;
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e) a.y[i * _numeq_ + e] = (double)y[e];
#if SODECL_SOLVER == 0
    a.counters[i] = counter;
#elif SODECL_SOLVER == 5
    if (a.counters) a.counters[i] = counter;
#endif
    (void)counter;
    if (capped) flags |= SODECL_FLAG_NEWTON_CAP;
    if (a.newton_passes) a.newton_passes[i] += passes;
    if (a.flags && flags) a.flags[i] |= flags;
}

// [lo of part k, when n items are split into parts parts as evenly as possible)
__device__ __forceinline__ sodecl_i64 sodecl_split(sodecl_i64 n, sodecl_i64 k, sodecl_i64 parts)
{
    const sodecl_i64 q = n / parts, r = n % parts;
    return k * q + (k < r ? k : r);
}

#if SODECL_LANES == 1 && (SODECL_SOLVER == 3 || SODECL_SOLVER == 4)
// Implicit solvers, one thread per orbit.  The orbits of a warp need
// different numbers of Newton passes per step, and a few need hundreds in
// some step (the pass limit), so this kernel keeps the warp's lanes busy two
// ways:
//  - Newton passes drive the loop, not steps: a lane whose iteration has
//    converged commits its step and starts the next one at the following
//    pass (sodecl_step_newton's arithmetic, in the same order);
//  - each warp owns a contiguous range of the launch's orbits, and a lane
//    whose orbit is done takes the range's next orbit (a ballot hands them
//    out in lane order), so a slow orbit holds up no other.
// The host launches at most the blocks that are resident at once, so each
// warp's range holds several orbits per lane.  Any block size works: the warp
// operations name only the lanes that exist.
extern "C" __global__ void __launch_bounds__(SODECL_BLOCK_MAX, SODECL_MIN_BLOCKS)
sodecl_orbits(const sodecl_args a)
{
    const int lane = threadIdx.x % 32;
    const int in_warp = min(32, (int)blockDim.x - (int)(threadIdx.x / 32) * 32);
    const unsigned wmask = in_warp == 32 ? 0xffffffffu : (1u << in_warp) - 1u;
    const sodecl_i64 warps_per_block = (blockDim.x + 31) / 32;
    const sodecl_i64 nwarps = (sodecl_i64)gridDim.x * warps_per_block;
    const sodecl_i64 w = (sodecl_i64)blockIdx.x * warps_per_block + threadIdx.x / 32;
    sodecl_i64 next = sodecl_split(a.n, w, nwarps);
    const sodecl_i64 hi = sodecl_split(a.n, w + 1, nwarps);

    real_t y[_numeq_], x[_numeq_];
    real_t p[SODECL_NPAR_ALLOC];
    real_t t = 0;
    sodecl_i64 i = 0, passes = 0;
    int c = 0, s = 0, pass = 0, flags = 0, capped = 0;
    bool active = false;
#pragma unroll 1
    for (;;) {
        // hand the range's next orbits to the idle lanes
        const unsigned idle = __ballot_sync(wmask, !active);
        if (idle != 0u && next < hi) {
            const sodecl_i64 mine = next + __popc(idle & ((1u << lane) - 1u));
            next += __popc(idle);
            if (!active && mine < hi) {
                i = mine;
                t = (real_t)a.t[i];
#pragma unroll SODECL_EQ_UNROLL
                for (int e = 0; e < _numeq_; ++e) y[e] = x[e] = (real_t)a.y[i * _numeq_ + e];
#pragma unroll SODECL_PAR_UNROLL
                for (int k = 0; k < _numpar_; ++k) p[k] = (real_t)__ldg(a.p + i * _numpar_ + k);
                c = a.chunk_begin;
                s = pass = flags = capped = 0;
                passes = 0;
                if (c < a.chunk_end) {
                    if (a.records) sodecl_store_record(a, c, i, y, flags);
                    active = true;
                } else {
                    sodecl_orbit_out(a, i, t, y, 0.0, passes, capped, flags);
                }
            }
        }
        if (!__any_sync(wmask, active)) {
            if (next >= hi) break;
            continue;
        }
        // Newton passes with every lane's parameters fixed (what depends on
        // them alone is computed once, out of this loop), until a lane is idle
        // while the range has orbits left, or every lane is done
#pragma unroll 1
        for (;;) {
            if (active) {
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
                    if (++s == _numsteps_) {
                        s = 0;
                        if (++c < a.chunk_end) {
                            if (a.records) sodecl_store_record(a, c, i, y, flags);
                        } else {
                            sodecl_orbit_out(a, i, t, y, 0.0, passes, capped, flags);
                            active = false;
                        }
                    }
                }
            }
            const unsigned now_idle = __ballot_sync(wmask, !active);
            if (now_idle == wmask || (now_idle != 0u && next < hi)) break;
        }
    }
}
#elif SODECL_LANES == 1 && SODECL_SOLVER == 5
// From record interval c on: stores record c and opens its interval; an
// interval that needs no attempt ends at once and the next one follows.
// Past the launch's last interval the orbit is written out and the lane is
// free (returns false).
__device__ __forceinline__ bool sodecl_dp_open(const sodecl_args &a, sodecl_i64 i, int &c, real_t &t, real_t *y,
                                               real_t *p, real_t &h, sodecl_dp_state &st, int &flags,
                                               sodecl_i64 accepted, int capped)
{
    const real_t span = (real_t)_numsteps_ * (real_t)_m_dt_;
#pragma unroll 1
    for (; c < a.chunk_end; ++c) {
        if (a.records) sodecl_store_record(a, c, i, y, flags);
        if (sodecl_dp_begin(t, y, p, h, span, st)) return true;
    }
    // the orbit's next step size rides in the counters array
    sodecl_orbit_out(a, i, t, y, (double)h, accepted, capped, flags);
    return false;
}

// The adaptive solver, one thread per orbit.  Orbits need very different
// numbers of attempted steps per interval, so, as in the implicit kernel,
// attempts drive the loop (a lane whose interval has ended records and opens
// the next at the following attempt), and each warp owns a contiguous range
// of the launch's orbits that its lanes take in turn (a ballot hands them out
// in lane order) when their orbit is done.  Each orbit's arithmetic is that of
// integrating it alone.
extern "C" __global__ void __launch_bounds__(SODECL_BLOCK_MAX, SODECL_MIN_BLOCKS)
sodecl_orbits(const sodecl_args a)
{
    const int lane = threadIdx.x % 32;
    const int in_warp = min(32, (int)blockDim.x - (int)(threadIdx.x / 32) * 32);
    const unsigned wmask = in_warp == 32 ? 0xffffffffu : (1u << in_warp) - 1u;
    const sodecl_i64 warps_per_block = (blockDim.x + 31) / 32;
    const sodecl_i64 nwarps = (sodecl_i64)gridDim.x * warps_per_block;
    const sodecl_i64 w = (sodecl_i64)blockIdx.x * warps_per_block + threadIdx.x / 32;
    sodecl_i64 next = sodecl_split(a.n, w, nwarps);
    const sodecl_i64 hi = sodecl_split(a.n, w + 1, nwarps);

    real_t y[_numeq_];
    real_t p[SODECL_NPAR_ALLOC];
    real_t t = 0, h = 0;
    sodecl_dp_state st;
    sodecl_i64 i = 0, accepted = 0;
    int c = 0, flags = 0, capped = 0;
    bool active = false;
#pragma unroll 1
    for (;;) {
        // hand the range's next orbits to the idle lanes
        const unsigned idle = __ballot_sync(wmask, !active);
        if (idle != 0u && next < hi) {
            const sodecl_i64 mine = next + __popc(idle & ((1u << lane) - 1u));
            next += __popc(idle);
            if (!active && mine < hi) {
                i = mine;
                t = (real_t)a.t[i];
#pragma unroll SODECL_EQ_UNROLL
                for (int e = 0; e < _numeq_; ++e) y[e] = (real_t)a.y[i * _numeq_ + e];
#pragma unroll SODECL_PAR_UNROLL
                for (int k = 0; k < _numpar_; ++k) p[k] = (real_t)__ldg(a.p + i * _numpar_ + k);
                h = a.counters ? (real_t)a.counters[i] : (real_t)0;
                c = a.chunk_begin;
                flags = capped = 0;
                accepted = 0;
                active = sodecl_dp_open(a, i, c, t, y, p, h, st, flags, accepted, capped);
            }
        }
        if (!__any_sync(wmask, active)) {
            if (next >= hi) break;
            continue;
        }
        // attempts, until a lane is idle while the range has orbits left, or
        // every lane is done
#pragma unroll 1
        for (;;) {
            if (active) {
                const int r = sodecl_dp_attempt(t, y, p, h, st, accepted);
                if (r != 0) {
                    if (r == 2) capped = 1;
                    ++c;
                    active = sodecl_dp_open(a, i, c, t, y, p, h, st, flags, accepted, capped);
                }
            }
            const unsigned now_idle = __ballot_sync(wmask, !active);
            if (now_idle == wmask || (now_idle != 0u && next < hi)) break;
        }
    }
}
#elif SODECL_LANES == 1
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
    sodecl_orbit_out(a, i, t, y, counter, passes, capped, flags);
}
#else  // SODECL_LANES > 1
__device__ __forceinline__ void sodecl_lanes_store(const sodecl_args &a, int rec, sodecl_i64 i, const real_t *yown,
                                                   int lane, int &flags)
{
    sodecl_record_t *col = a.records + (sodecl_i64)(rec - a.rec_first) * _numeq_ * a.rec_stride + a.rec_col0 + i;
    bool finite = true;
#pragma unroll
    for (int k = 0; k < SODECL_ROWS; ++k) {
        const int r = lane + k * SODECL_LANES;
        if (r < _numeq_) {
            finite = finite && isfinite(yown[k]);
            __stcs(col + (sodecl_i64)r * a.rec_stride, (sodecl_record_t)yown[k]);
        }
    }
    if (!finite) flags |= SODECL_FLAG_NONFINITE;
}

// Launch: blockDim.x a multiple of 32, grid * blockDim.x >= n * SODECL_LANES,
// dynamic shared memory blockDim.x / SODECL_LANES * SODECL_SLOT words.  The
// groups past the last orbit shadow it (all lanes of a group run to the end)
// and store nothing.
extern "C" __global__ void __launch_bounds__(SODECL_BLOCK_MAX, SODECL_MIN_BLOCKS)
sodecl_orbits(const sodecl_args a)
{
    extern __shared__ __align__(16) unsigned char sodecl_smem[];
    const int lane = threadIdx.x % SODECL_LANES;
    // the group's own lanes: groups of a warp leave a Newton iteration after
    // different numbers of passes, so no barrier or shuffle names another group
    const unsigned gmask = SODECL_LANES == 32 ? 0xffffffffu
                                              : ((1u << SODECL_LANES) - 1u) << ((threadIdx.x % 32) / SODECL_LANES * SODECL_LANES);
    const sodecl_lanes_view v = sodecl_lanes_slot(
        reinterpret_cast<real_t *>(sodecl_smem) + (threadIdx.x / SODECL_LANES) * SODECL_SLOT, lane, gmask);
    const sodecl_i64 orbit = ((sodecl_i64)blockIdx.x * blockDim.x + threadIdx.x) / SODECL_LANES;
    const bool live = orbit < a.n;
    const sodecl_i64 i = live ? orbit : a.n - 1;

    real_t yown[SODECL_ROWS];
#pragma unroll
    for (int k = 0; k < SODECL_ROWS; ++k) {
        const int r = lane + k * SODECL_LANES;
        yown[k] = (real_t)0;
        if (r < _numeq_) {
            yown[k] = (real_t)a.y[i * _numeq_ + r];
            v.Y[r] = yown[k];
        }
    }
    for (int k = lane; k < _numpar_; k += SODECL_LANES) v.P[k] = (real_t)__ldg(a.p + i * _numpar_ + k);
    __syncwarp(gmask);
    real_t t = (real_t)a.t[i];
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
        if (a.records && live) sodecl_lanes_store(a, c, i, yown, lane, flags);
#pragma unroll 1
        for (int s = 0; s < _numsteps_; ++s)
            sodecl_lanes_advance(t, yown, v, gid, counter, passes, capped);
    }
    if (a.write_final && a.records && live) sodecl_lanes_store(a, a.chunk_end, i, yown, lane, flags);

#pragma unroll
    for (int o = SODECL_LANES / 2; o > 0; o >>= 1) flags |= __shfl_xor_sync(gmask, flags, o, SODECL_LANES);
    if (!live) return;
#pragma unroll
    for (int k = 0; k < SODECL_ROWS; ++k) {
        const int r = lane + k * SODECL_LANES;
        if (r < _numeq_) a.y[i * _numeq_ + r] = (double)yown[k];
    }
    if (lane == 0) {
        a.t[i] = (double)t;
#if SODECL_SOLVER == 0
        a.counters[i] = counter;
#endif
        if (capped) flags |= SODECL_FLAG_NEWTON_CAP;
        if (a.newton_passes) a.newton_passes[i] += passes;
        if (a.flags && flags) a.flags[i] |= flags;
    }
}
#endif  // SODECL_LANES
#endif  // SODECL_STEPS_ONLY
