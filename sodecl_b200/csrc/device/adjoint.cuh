// Discrete adjoint of the explicit solvers (Euler, RK4) for model fitting:
// d(loss)/d(params, y0) per orbit, loss = mean squared error of the records
// against target trajectories.
//
// Reverse-mode differentiation of the user's right-hand side: the system
// file is compiled a second time with `double` mapped to sodecl_ad, a value
// that records every operation (its partial derivatives and operands) on a
// per-thread tape.  A reverse sweep over the tape gives the vector-Jacobian
// products v^T df/dy and v^T df/dp exactly (to rounding) for any system file,
// branches included (the tape follows the branch taken).
//
// The integrator steps are differentiated in their discrete form (the
// adjoint of the arithmetic the forward pass performs, not of the ODE), and
// the state is checkpointed every `ckpt_every` steps: the backward pass
// recomputes each segment's states from its checkpoint, then walks the
// segment's steps in reverse.  Memory per orbit: T/C checkpoints and C
// segment states (C ~ sqrt(T) balances the two).  With C >= T there is one
// segment, which the forward sweep records as it goes: T segment states and
// no recomputation.
//
// Part 1 (before the user file): the tape and the sodecl_ad type.
// Part 2 (SODECL_ADJOINT_KERNEL, after both copies of the user file): the
// step adjoints and the kernel.
//
// Where the products come from (SODECL_ADJ_MODE):
//   2  the system file's calc_vjp(t, y, v, ybar, pbar, p), which accumulates
//      v^T df/dy and v^T df/dp itself (only the nonzero terms, shared
//      subexpressions): the fastest;
//   1  its calc_jacobian (df/dy, as the implicit solvers use it) and
//      calc_jacobian_params (df/dp): dense products in registers;
//   0  the tape, for every other system file.

#ifndef SODECL_ADJOINT_TYPES
#define SODECL_ADJOINT_TYPES

#ifndef SODECL_TAPE_CAP
#define SODECL_TAPE_CAP 256
#endif

// One operation: result = g(operand a, operand b); d = dg/da, e = dg/db.
// Operand -1 means none (a constant).  Leaves have both operands -1.
struct sodecl_tape {
    int n;
    int overflow;
    short a[SODECL_TAPE_CAP];
    short b[SODECL_TAPE_CAP];
    double da[SODECL_TAPE_CAP];
    double db[SODECL_TAPE_CAP];
};

__device__ __forceinline__ int sodecl_tape_push(sodecl_tape *t, int a, double da, int b, double db)
{
    if (!t) return -1;
    const int k = t->n;
    if (k >= SODECL_TAPE_CAP) {
        t->overflow = 1;
        return -1;
    }
    t->a[k] = (short)a;
    t->b[k] = (short)b;
    t->da[k] = da;
    t->db[k] = db;
    t->n = k + 1;
    return k;
}

struct sodecl_ad {
    double v;
    int id;               // tape entry, -1 for a constant
    sodecl_tape *tp;
    __device__ __forceinline__ sodecl_ad() : v(0.0), id(-1), tp(nullptr) {}
    __device__ __forceinline__ sodecl_ad(double x) : v(x), id(-1), tp(nullptr) {}
    __device__ __forceinline__ sodecl_ad(float x) : v(x), id(-1), tp(nullptr) {}
    __device__ __forceinline__ sodecl_ad(int x) : v(x), id(-1), tp(nullptr) {}
    __device__ __forceinline__ sodecl_ad(unsigned x) : v(x), id(-1), tp(nullptr) {}
    __device__ __forceinline__ sodecl_ad(long x) : v((double)x), id(-1), tp(nullptr) {}
    __device__ __forceinline__ sodecl_ad(long long x) : v((double)x), id(-1), tp(nullptr) {}
    __device__ __forceinline__ sodecl_ad(double x, int i, sodecl_tape *t) : v(x), id(i), tp(t) {}
    __device__ __forceinline__ explicit operator double() const { return v; }
    __device__ __forceinline__ explicit operator float() const { return (float)v; }
    __device__ __forceinline__ explicit operator int() const { return (int)v; }
    __device__ __forceinline__ explicit operator long() const { return (long)v; }
    __device__ __forceinline__ explicit operator long long() const { return (long long)v; }
    __device__ __forceinline__ explicit operator bool() const { return v != 0.0; }
};

__device__ __forceinline__ sodecl_tape *sodecl_ad_tape(const sodecl_ad &a, const sodecl_ad &b)
{
    return a.tp ? a.tp : b.tp;
}

// result of a binary operation with partials da, db
__device__ __forceinline__ sodecl_ad sodecl_ad_bin(double v, const sodecl_ad &a, double da, const sodecl_ad &b,
                                                   double db)
{
    if (a.id < 0 && b.id < 0) return sodecl_ad(v);
    sodecl_tape *t = sodecl_ad_tape(a, b);
    return sodecl_ad(v, sodecl_tape_push(t, a.id, da, b.id, db), t);
}

__device__ __forceinline__ sodecl_ad sodecl_ad_un(double v, const sodecl_ad &a, double da)
{
    if (a.id < 0) return sodecl_ad(v);
    return sodecl_ad(v, sodecl_tape_push(a.tp, a.id, da, -1, 0.0), a.tp);
}

__device__ __forceinline__ sodecl_ad operator+(const sodecl_ad &a) { return a; }
__device__ __forceinline__ sodecl_ad operator-(const sodecl_ad &a) { return sodecl_ad_un(-a.v, a, -1.0); }
__device__ __forceinline__ sodecl_ad operator+(const sodecl_ad &a, const sodecl_ad &b)
{
    return sodecl_ad_bin(a.v + b.v, a, 1.0, b, 1.0);
}
__device__ __forceinline__ sodecl_ad operator-(const sodecl_ad &a, const sodecl_ad &b)
{
    return sodecl_ad_bin(a.v - b.v, a, 1.0, b, -1.0);
}
__device__ __forceinline__ sodecl_ad operator*(const sodecl_ad &a, const sodecl_ad &b)
{
    return sodecl_ad_bin(a.v * b.v, a, b.v, b, a.v);
}
__device__ __forceinline__ sodecl_ad operator/(const sodecl_ad &a, const sodecl_ad &b)
{
    const double q = a.v / b.v;
    return sodecl_ad_bin(q, a, 1.0 / b.v, b, -q / b.v);
}
__device__ __forceinline__ sodecl_ad &operator+=(sodecl_ad &a, const sodecl_ad &b) { return a = a + b; }
__device__ __forceinline__ sodecl_ad &operator-=(sodecl_ad &a, const sodecl_ad &b) { return a = a - b; }
__device__ __forceinline__ sodecl_ad &operator*=(sodecl_ad &a, const sodecl_ad &b) { return a = a * b; }
__device__ __forceinline__ sodecl_ad &operator/=(sodecl_ad &a, const sodecl_ad &b) { return a = a / b; }
__device__ __forceinline__ bool operator<(const sodecl_ad &a, const sodecl_ad &b) { return a.v < b.v; }
__device__ __forceinline__ bool operator>(const sodecl_ad &a, const sodecl_ad &b) { return a.v > b.v; }
__device__ __forceinline__ bool operator<=(const sodecl_ad &a, const sodecl_ad &b) { return a.v <= b.v; }
__device__ __forceinline__ bool operator>=(const sodecl_ad &a, const sodecl_ad &b) { return a.v >= b.v; }
__device__ __forceinline__ bool operator==(const sodecl_ad &a, const sodecl_ad &b) { return a.v == b.v; }
__device__ __forceinline__ bool operator!=(const sodecl_ad &a, const sodecl_ad &b) { return a.v != b.v; }

// elementary functions with their derivatives
__device__ __forceinline__ sodecl_ad exp(const sodecl_ad &a) { const double e = ::exp(a.v); return sodecl_ad_un(e, a, e); }
__device__ __forceinline__ sodecl_ad log(const sodecl_ad &a) { return sodecl_ad_un(::log(a.v), a, 1.0 / a.v); }
__device__ __forceinline__ sodecl_ad sqrt(const sodecl_ad &a) { const double s = ::sqrt(a.v); return sodecl_ad_un(s, a, 0.5 / s); }
__device__ __forceinline__ sodecl_ad sin(const sodecl_ad &a) { return sodecl_ad_un(::sin(a.v), a, ::cos(a.v)); }
__device__ __forceinline__ sodecl_ad cos(const sodecl_ad &a) { return sodecl_ad_un(::cos(a.v), a, -::sin(a.v)); }
__device__ __forceinline__ sodecl_ad sincos(const sodecl_ad &a, sodecl_ad *c) { *c = cos(a); return sin(a); }
__device__ __forceinline__ sodecl_ad tan(const sodecl_ad &a) { const double c = ::cos(a.v); return sodecl_ad_un(::tan(a.v), a, 1.0 / (c * c)); }
__device__ __forceinline__ sodecl_ad tanh(const sodecl_ad &a) { const double h = ::tanh(a.v); return sodecl_ad_un(h, a, 1.0 - h * h); }
__device__ __forceinline__ sodecl_ad sinh(const sodecl_ad &a) { return sodecl_ad_un(::sinh(a.v), a, ::cosh(a.v)); }
__device__ __forceinline__ sodecl_ad cosh(const sodecl_ad &a) { return sodecl_ad_un(::cosh(a.v), a, ::sinh(a.v)); }
__device__ __forceinline__ sodecl_ad atan(const sodecl_ad &a) { return sodecl_ad_un(::atan(a.v), a, 1.0 / (1.0 + a.v * a.v)); }
__device__ __forceinline__ sodecl_ad exp2(const sodecl_ad &a) { const double e = ::exp2(a.v); return sodecl_ad_un(e, a, e * 0.6931471805599453); }
__device__ __forceinline__ sodecl_ad log10(const sodecl_ad &a) { return sodecl_ad_un(::log10(a.v), a, 0.4342944819032518 / a.v); }
__device__ __forceinline__ sodecl_ad fabs(const sodecl_ad &a) { return sodecl_ad_un(::fabs(a.v), a, a.v < 0.0 ? -1.0 : 1.0); }
__device__ __forceinline__ sodecl_ad pow(const sodecl_ad &a, const sodecl_ad &b)
{
    const double r = ::pow(a.v, b.v);
    const double da = (b.v == 0.0) ? 0.0 : b.v * ::pow(a.v, b.v - 1.0);
    const double db = (a.v > 0.0) ? r * ::log(a.v) : 0.0;
    return sodecl_ad_bin(r, a, da, b, db);
}
__device__ __forceinline__ sodecl_ad fmin(const sodecl_ad &a, const sodecl_ad &b) { return a.v <= b.v ? a : b; }
__device__ __forceinline__ sodecl_ad fmax(const sodecl_ad &a, const sodecl_ad &b) { return a.v >= b.v ? a : b; }
__device__ __forceinline__ bool isfinite(const sodecl_ad &a) { return ::isfinite(a.v); }
__device__ __forceinline__ bool isnan(const sodecl_ad &a) { return ::isnan(a.v); }

// reverse sweep: adj[k] holds d(output . seed)/d(entry k) on return
__device__ __forceinline__ void sodecl_tape_sweep(const sodecl_tape &t, double *adj)
{
    for (int k = t.n - 1; k >= 0; --k) {
        const double g = adj[k];
        if (g == 0.0) continue;
        const int a = t.a[k], b = t.b[k];
        if (a >= 0) adj[a] += t.da[k] * g;
        if (b >= 0) adj[b] += t.db[k] * g;
    }
}
#endif  // SODECL_ADJOINT_TYPES

#ifdef SODECL_ADJOINT_KERNEL
// ---------------------------------------------------------------------------
// Part 2.  Needs: the plain system (sode_system), the recording copy
// (sodecl_adsys::sode_system), the solver step functions (solvers.cuh).

#if SODECL_ADJ_MODE == 2
// For the seed v: xbar += v^T df/dx, pbar += v^T df/dp, by the system file's
// own vector-Jacobian product.
__device__ __forceinline__ void sodecl_vjp(double t, const double *x, const double *p, const double *v, double *xbar,
                                           double *pbar, sodecl_tape *tape, double *adj, int &overflow)
{
    (void)tape;
    (void)adj;
    (void)overflow;
    real_t xx[_numeq_], pp[SODECL_NPAR_ALLOC], vv[_numeq_], xb[_numeq_], pb[SODECL_NPAR_ALLOC];
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e) {
        xx[e] = (real_t)x[e];
        vv[e] = (real_t)v[e];
        xb[e] = (real_t)0;
    }
#pragma unroll SODECL_PAR_UNROLL
    for (int j = 0; j < _numpar_; ++j) {
        pp[j] = (real_t)p[j];
        pb[j] = (real_t)0;
    }
    calc_vjp((real_t)t, xx, vv, xb, pb, pp);
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e) xbar[e] += (double)xb[e];
#pragma unroll SODECL_PAR_UNROLL
    for (int j = 0; j < _numpar_; ++j) pbar[j] += (double)pb[j];
}
#elif SODECL_ADJ_MODE == 1
// For the seed v: xbar += v^T df/dx, pbar += v^T df/dp, from the system
// file's own Jacobians (calc_jacobian, calc_jacobian_params): two small
// dense products, everything in registers.
__device__ __forceinline__ void sodecl_vjp(double t, const double *x, const double *p, const double *v, double *xbar,
                                           double *pbar, sodecl_tape *tape, double *adj, int &overflow)
{
    (void)t;
    (void)tape;
    (void)adj;
    (void)overflow;
    real_t xx[_numeq_], pp[SODECL_NPAR_ALLOC];
    real_t jy[_numeq_][_numeq_], jp[_numeq_][SODECL_NPAR_ALLOC];
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e) xx[e] = (real_t)x[e];
#pragma unroll SODECL_PAR_UNROLL
    for (int j = 0; j < _numpar_; ++j) pp[j] = (real_t)p[j];
    calc_jacobian(xx, jy, pp);
    calc_jacobian_params(xx, jp, pp);
#pragma unroll SODECL_EQ_UNROLL
    for (int i = 0; i < _numeq_; ++i) {
#pragma unroll SODECL_EQ_UNROLL
        for (int j = 0; j < _numeq_; ++j) xbar[j] += (double)jy[i][j] * v[i];
#pragma unroll SODECL_PAR_UNROLL
        for (int j = 0; j < _numpar_; ++j) pbar[j] += (double)jp[i][j] * v[i];
    }
}
#else
// f(t, x) and, for the seed v, xbar += v^T df/dx, pbar += v^T df/dp.
__device__ __forceinline__ void sodecl_vjp(double t, const double *x, const double *p, const double *v, double *xbar,
                                           double *pbar, sodecl_tape *tape, double *adj, int &overflow)
{
    tape->n = 0;
    tape->overflow = 0;
    sodecl_ad xa[_numeq_], pa[SODECL_NPAR_ALLOC], fa[_numeq_];
    for (int e = 0; e < _numeq_; ++e) xa[e] = sodecl_ad(x[e], sodecl_tape_push(tape, -1, 0.0, -1, 0.0), tape);
    for (int j = 0; j < _numpar_; ++j) pa[j] = sodecl_ad(p[j], sodecl_tape_push(tape, -1, 0.0, -1, 0.0), tape);
    sodecl_adsys::sode_system(sodecl_ad(t), xa, fa, pa);
    for (int k = 0; k < tape->n; ++k) adj[k] = 0.0;
    for (int e = 0; e < _numeq_; ++e)
        if (fa[e].id >= 0) adj[fa[e].id] += v[e];
    sodecl_tape_sweep(*tape, adj);
    for (int e = 0; e < _numeq_; ++e) xbar[e] += adj[e];
    for (int j = 0; j < _numpar_; ++j) pbar[j] += adj[_numeq_ + j];
    if (tape->overflow) overflow = 1;
}
#endif

#if SODECL_SOLVER == 3 || SODECL_SOLVER == 4
// mu <- A^{-T} mu for A = I - c J (J row-major, _numeq_ x _numeq_): Gaussian
// elimination with partial pivoting on A^T.  Row swaps are written as
// selects over the rows below the pivot, so small systems stay in registers.
__device__ __forceinline__ void sodecl_transposed_solve(const real_t (*J)[_numeq_], double c, double *mu)
{
    double a[_numeq_][_numeq_];
#pragma unroll SODECL_EQ_UNROLL
    for (int i = 0; i < _numeq_; ++i)
#pragma unroll SODECL_EQ_UNROLL
        for (int j = 0; j < _numeq_; ++j) a[i][j] = (i == j ? 1.0 : 0.0) - c * (double)J[j][i];
#pragma unroll SODECL_EQ_UNROLL
    for (int k = 0; k < _numeq_; ++k) {
        int piv = k;
        double best = fabs(a[k][k]);
#pragma unroll SODECL_EQ_UNROLL
        for (int i = k + 1; i < _numeq_; ++i)
            if (fabs(a[i][k]) > best) {
                best = fabs(a[i][k]);
                piv = i;
            }
#pragma unroll SODECL_EQ_UNROLL
        for (int i = k + 1; i < _numeq_; ++i) {
            const bool sw = i == piv;
#pragma unroll SODECL_EQ_UNROLL
            for (int j = k; j < _numeq_; ++j) {
                const double u = a[k][j];
                a[k][j] = sw ? a[i][j] : u;
                a[i][j] = sw ? u : a[i][j];
            }
            const double u = mu[k];
            mu[k] = sw ? mu[i] : u;
            mu[i] = sw ? u : mu[i];
        }
#pragma unroll SODECL_EQ_UNROLL
        for (int i = k + 1; i < _numeq_; ++i) {
            const double f = a[i][k] / a[k][k];
#pragma unroll SODECL_EQ_UNROLL
            for (int j = k + 1; j < _numeq_; ++j) a[i][j] -= f * a[k][j];
            mu[i] -= f * mu[k];
        }
    }
#pragma unroll SODECL_EQ_UNROLL
    for (int k = _numeq_ - 1; k >= 0; --k) {
        double sum = mu[k];
#pragma unroll SODECL_EQ_UNROLL
        for (int j = k + 1; j < _numeq_; ++j) sum -= a[k][j] * mu[j];
        mu[k] = sum / a[k][k];
    }
}
#endif

// lambda <- (d step / d y)^T lambda, pbar += (d step / d p)^T lambda, for the
// step taken from (t, y) to ynext with step h: the adjoint of
// sodecl_step_euler / sodecl_step_rk4's arithmetic, and of the implicit steps
// taken as solved exactly.
__device__ __forceinline__ void sodecl_step_adjoint(double h, double t, const double *y, const double *ynext,
                                                    const double *stages, const double *p, double *lambda,
                                                    double *pbar, sodecl_tape *tape, double *adj, int &overflow)
{
    (void)ynext;
    (void)stages;
#if SODECL_SOLVER == 1
    // y1 = y + h f(t, y)
    double seed[_numeq_], ybar[_numeq_];
    for (int e = 0; e < _numeq_; ++e) {
        seed[e] = h * lambda[e];
        ybar[e] = lambda[e];
    }
    sodecl_vjp(t, y, p, seed, ybar, pbar, tape, adj, overflow);
    for (int e = 0; e < _numeq_; ++e) lambda[e] = ybar[e];
#elif SODECL_SOLVER == 2
    // y1 = y + (k1 + 2 k2 + 2 k3 + k4) h / 6 with stage inputs
    // x1 = y, x2 = y + (h/2) k1, x3 = y + (h/2) k2, x4 = y + h k3, recorded
    // by the segment's recomputation (stages = x2 | x3 | x4)
    const double *x2 = stages, *x3 = stages + _numeq_, *x4 = stages + 2 * _numeq_;
    double pv[SODECL_NPAR_ALLOC];
    for (int j = 0; j < _numpar_; ++j) pv[j] = p[j];
    double ybar[_numeq_], kbar[_numeq_], seed[_numeq_], xbar[_numeq_];
    const double w1 = h / 6.0, w2 = 2.0 * h / 6.0;
    for (int e = 0; e < _numeq_; ++e) ybar[e] = lambda[e];
    // stage 4: k4 = f(t + h, x4), weight h/6; x4 depends on y and k3 (factor h)
    for (int e = 0; e < _numeq_; ++e) { seed[e] = w1 * lambda[e]; xbar[e] = 0.0; }
    sodecl_vjp(t + h, x4, pv, seed, xbar, pbar, tape, adj, overflow);
    for (int e = 0; e < _numeq_; ++e) { ybar[e] += xbar[e]; kbar[e] = w2 * lambda[e] + h * xbar[e]; }
    // stage 3: k3 = f(t + h/2, x3); x3 = y + (h/2) k2
    for (int e = 0; e < _numeq_; ++e) xbar[e] = 0.0;
    sodecl_vjp(t + 0.5 * h, x3, pv, kbar, xbar, pbar, tape, adj, overflow);
    for (int e = 0; e < _numeq_; ++e) { ybar[e] += xbar[e]; kbar[e] = w2 * lambda[e] + 0.5 * h * xbar[e]; }
    // stage 2: k2 = f(t + h/2, x2); x2 = y + (h/2) k1
    for (int e = 0; e < _numeq_; ++e) xbar[e] = 0.0;
    sodecl_vjp(t + 0.5 * h, x2, pv, kbar, xbar, pbar, tape, adj, overflow);
    for (int e = 0; e < _numeq_; ++e) { ybar[e] += xbar[e]; kbar[e] = w1 * lambda[e] + 0.5 * h * xbar[e]; }
    // stage 1: k1 = f(t, y)
    for (int e = 0; e < _numeq_; ++e) xbar[e] = 0.0;
    sodecl_vjp(t, y, pv, kbar, xbar, pbar, tape, adj, overflow);
    for (int e = 0; e < _numeq_; ++e) lambda[e] = ybar[e] + xbar[e];
#elif SODECL_SOLVER == 3 || SODECL_SOLVER == 4
    // The implicit step taken as solved exactly (the Newton passes of
    // src/kernels/ie.cl:50-117 / im.cl:43-118 stop at a residual bound; the
    // gradient is that of the step they approximate):
    //   IE: y1 = y + h f(t, y1):           (I - h J(y1)) dy1 = dy + h f_p dp
    //   IM: y1 = y + h f(t, (y + y1)/2):   (I - h/2 J(m)) dy1 = (I + h/2 J(m)) dy + h f_p dp
    // so mu = (I - c J)^{-T} lambda, lambda <- mu (IE) or mu + c J^T mu (IM),
    // pbar += h f_p^T mu, with J from calc_jacobian (the full matrix: every
    // entry counts here, unlike in the banded Newton solve).
#if SODECL_SOLVER == 4
    const double c = 0.5 * h;
#else
    const double c = h;
#endif
    double x[_numeq_], mu[_numeq_];
    real_t xx[_numeq_], pp[SODECL_NPAR_ALLOC], jj[_numeq_][_numeq_];
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e) {
#if SODECL_SOLVER == 4
        x[e] = (y[e] + ynext[e]) * 0.5;
#else
        x[e] = ynext[e];
#endif
        xx[e] = (real_t)x[e];
        mu[e] = lambda[e];
    }
#pragma unroll SODECL_PAR_UNROLL
    for (int j = 0; j < _numpar_; ++j) pp[j] = (real_t)p[j];
    calc_jacobian(xx, jj, pp);
    sodecl_transposed_solve(jj, c, mu);
    // J^T mu and f_p^T mu at x from the product source
    double jtmu[_numeq_], fp[SODECL_NPAR_ALLOC];
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e) jtmu[e] = 0.0;
#pragma unroll SODECL_PAR_UNROLL
    for (int j = 0; j < _numpar_; ++j) fp[j] = 0.0;
    sodecl_vjp(t, x, p, mu, jtmu, fp, tape, adj, overflow);
#pragma unroll SODECL_PAR_UNROLL
    for (int j = 0; j < _numpar_; ++j) pbar[j] += h * fp[j];
#pragma unroll SODECL_EQ_UNROLL
    for (int e = 0; e < _numeq_; ++e) {
#if SODECL_SOLVER == 4
        lambda[e] = mu[e] + c * jtmu[e];
#else
        lambda[e] = mu[e];
#endif
    }
#else
#error "the adjoint covers the Euler, RK4, implicit Euler and implicit midpoint solvers"
#endif
}

#define SODECL_FLAG_TAPE_OVERFLOW 4

// doubles per orbit per segment step: the state, t, and for RK4 the three
// stage inputs (recorded by the recomputation, read by the reverse step)
#if SODECL_SOLVER == 2
#define SODECL_SEG_WIDTH (4 * _numeq_ + 1)
#else
#define SODECL_SEG_WIDTH (_numeq_ + 1)
#endif

// One step of the forward arithmetic (sodecl_advance's), recording into st
// (stride n between values) unless it is null: the state and t before the
// step and, for RK4, its three stage inputs.  The forward sweep and the
// segment recomputation both step through here, so they agree bit for bit.
__device__ __forceinline__ void sodecl_adjoint_step(real_t &t, real_t *y, real_t *p, long long i, double &counter,
                                                    sodecl_i64 &passes, int &capped, double *st, long long n)
{
    if (st) {
        st[_numeq_ * n] = (double)t;
        for (int e = 0; e < _numeq_; ++e) st[e * n] = (double)y[e];
    }
#if SODECL_SOLVER == 2
    (void)i;
    (void)counter;
    (void)passes;
    (void)capped;
    real_t x2[_numeq_], x3[_numeq_], x4[_numeq_], ynew[_numeq_];
    sodecl_step_rk4(_m_dt_, t, y, ynew, p, x2, x3, x4);
    t = t + _m_dt_;
    for (int e = 0; e < _numeq_; ++e) y[e] = ynew[e];
    if (st)
        for (int e = 0; e < _numeq_; ++e) {
            st[(_numeq_ + 1 + e) * n] = (double)x2[e];
            st[(2 * _numeq_ + 1 + e) * n] = (double)x3[e];
            st[(3 * _numeq_ + 1 + e) * n] = (double)x4[e];
        }
#else
    sodecl_advance(t, y, p, i, counter, passes, capped);
#endif
}

struct sodecl_adjoint_args {
    const double *t0;         // [n]
    const double *y0;         // [n][neq]
    const double *p;          // [n][npar]
    const double *targets;    // [nrec][neq][n]
    double *loss;             // [n] per-orbit mean squared error
    double *grad_p;           // [n][npar] or null (forward only)
    double *grad_y0;          // [n][neq] or null
    double *ckpt;             // scratch [nckpt][neq][n]
    double *ckpt_t;           // scratch [nckpt][n]
    double *seg;              // scratch [min(ckpt_every, steps)][SODECL_SEG_WIDTH][n]: state, t, (RK4) stage inputs
    int *flags;               // [n] or null
    long long n;
    int nchunks;              // records - 1; steps = nchunks * _numsteps_
    int ckpt_every;           // C
};

// Loss and, if grad_p is set, its gradient for every orbit.
extern "C" __global__ void __launch_bounds__(SODECL_BLOCK_MAX, SODECL_MIN_BLOCKS) sodecl_adjoint(const sodecl_adjoint_args a)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const long long n = a.n;
    const int steps = a.nchunks * _numsteps_;
    const int C = a.ckpt_every;
    const double w = 1.0 / ((double)(a.nchunks + 1) * _numeq_);  // mean over records x equations

    real_t y[_numeq_], p[SODECL_NPAR_ALLOC];
    real_t t = (real_t)a.t0[i];
    for (int e = 0; e < _numeq_; ++e) y[e] = (real_t)a.y0[i * _numeq_ + e];
    for (int j = 0; j < _numpar_; ++j) p[j] = (real_t)a.p[i * _numpar_ + j];
    double counter = 0.0;
    sodecl_i64 passes = 0;
    int capped = 0;

    // forward: loss at every record, checkpoints every C steps; with one
    // segment (C >= steps) the sweep records the segment itself, and the
    // backward pass has nothing to recompute
#if SODECL_ADJ_GRADIENT
    const bool whole = a.grad_p && C >= steps;
#else
    // the loss-only kernel: the forward sweep alone, nothing recorded
    const bool whole = false;
#endif
    double loss = 0.0;
    for (int s = 0; s <= steps; ++s) {
        if (s % _numsteps_ == 0) {
            const int r = s / _numsteps_;
            for (int e = 0; e < _numeq_; ++e) {
                const double d = (double)y[e] - a.targets[((long long)r * _numeq_ + e) * n + i];
                loss += d * d;
            }
        }
        if (SODECL_ADJ_GRADIENT && a.grad_p && !whole && s % C == 0 && s < steps) {
            const long long c = s / C;
            a.ckpt_t[c * n + i] = (double)t;
            for (int e = 0; e < _numeq_; ++e) a.ckpt[(c * _numeq_ + e) * n + i] = (double)y[e];
        }
        if (s < steps)
            sodecl_adjoint_step(t, y, p, i, counter, passes, capped,
                                whole ? a.seg + (long long)s * SODECL_SEG_WIDTH * n + i : nullptr, n);
    }
    a.loss[i] = loss * w;
    if (!SODECL_ADJ_GRADIENT || !a.grad_p) {
        if (a.flags) a.flags[i] = capped ? SODECL_FLAG_NEWTON_CAP : 0;
        return;
    }
#if SODECL_ADJ_GRADIENT

    // backward, segment by segment from the last
#if SODECL_ADJ_MODE != 0
    sodecl_tape *tape = nullptr;  // the analytic products record nothing
    double *adj = nullptr;
#else
    sodecl_tape tape_storage;
    double adj[SODECL_TAPE_CAP];
    sodecl_tape *tape = &tape_storage;
#endif
    double lambda[_numeq_], pbar[SODECL_NPAR_ALLOC], pd[SODECL_NPAR_ALLOC];
    for (int e = 0; e < _numeq_; ++e) lambda[e] = 0.0;
    for (int j = 0; j < _numpar_; ++j) { pbar[j] = 0.0; pd[j] = (double)p[j]; }
    int overflow = 0;
    double ynext[_numeq_];  // state after the step being reversed
    for (int e = 0; e < _numeq_; ++e) ynext[e] = (double)y[e];
    const int nseg = (steps + C - 1) / C;
    for (int sg = nseg - 1; sg >= 0; --sg) {
        const int s0 = sg * C, s1 = min(steps, s0 + C);
        // recompute the segment's states from its checkpoint
        if (!whole) {
            real_t ys[_numeq_];
            real_t ts = (real_t)a.ckpt_t[(long long)sg * n + i];
            for (int e = 0; e < _numeq_; ++e) ys[e] = (real_t)a.ckpt[((long long)sg * _numeq_ + e) * n + i];
            for (int s = s0; s < s1; ++s)
                sodecl_adjoint_step(ts, ys, p, i, counter, passes, capped,
                                    a.seg + (long long)(s - s0) * SODECL_SEG_WIDTH * n + i, n);
        }
        // reverse the segment's steps
        for (int s = s1 - 1; s >= s0; --s) {
            // record at state s+1
            if ((s + 1) % _numsteps_ == 0) {
                const int r = (s + 1) / _numsteps_;
                for (int e = 0; e < _numeq_; ++e)
                    lambda[e] += 2.0 * w * (ynext[e] - a.targets[((long long)r * _numeq_ + e) * n + i]);
            }
            const double *st = a.seg + (long long)(s - s0) * SODECL_SEG_WIDTH * n + i;
            double ystep[_numeq_], stages[SODECL_SEG_WIDTH - _numeq_ - 1 > 0 ? SODECL_SEG_WIDTH - _numeq_ - 1 : 1];
            for (int e = 0; e < _numeq_; ++e) ystep[e] = st[e * n];
            for (int e = 0; e < SODECL_SEG_WIDTH - _numeq_ - 1; ++e) stages[e] = st[(_numeq_ + 1 + e) * n];
            sodecl_step_adjoint((double)_m_dt_, st[_numeq_ * n], ystep, ynext, stages, pd, lambda, pbar, tape, adj,
                                overflow);
            for (int e = 0; e < _numeq_; ++e) ynext[e] = ystep[e];
        }
    }
    // record 0 is the initial state
    for (int e = 0; e < _numeq_; ++e) lambda[e] += 2.0 * w * (ynext[e] - a.targets[(long long)e * n + i]);
    for (int j = 0; j < _numpar_; ++j) a.grad_p[i * _numpar_ + j] = pbar[j];
    if (a.grad_y0)
        for (int e = 0; e < _numeq_; ++e) a.grad_y0[i * _numeq_ + e] = lambda[e];
    if (a.flags) a.flags[i] = (overflow ? SODECL_FLAG_TAPE_OVERFLOW : 0) | (capped ? SODECL_FLAG_NEWTON_CAP : 0);
#endif  // SODECL_ADJ_GRADIENT
}
#endif  // SODECL_ADJOINT_KERNEL
