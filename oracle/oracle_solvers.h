/*
 * oracle_solvers.h -- TEST INFRASTRUCTURE ONLY (CPU oracle).
 *
 * A plain-C restatement of SODECL's fixed-step integrators, used by the
 * tests, the smoke check and the CPU-baseline leg of bench.py as the checker
 * for the CUDA path.  The shipped library never includes, links or calls it.
 *
 * Compiled once per SODECL system file: oracle/build.py makes one
 * translation unit of   oracle_prelude.h + <system file> + this file
 * and builds a shared library with the C entry points at the bottom.
 * With -DORACLE_FP32 the system is compiled in single precision (the build
 * script rewrites `double` and unsuffixed literals, as the CUDA front end
 * does for its fp32 programs).
 *
 * Each routine cites the reference code it restates (paths relative to the
 * sodecl repository).  Evaluation order follows the reference exactly, so a
 * build without FMA contraction reproduces the reference bit for bit.
 */
#ifndef SODECL_ORACLE_SOLVERS_H
#define SODECL_ORACLE_SOLVERS_H

#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifdef ORACLE_FP32
typedef float orc_real;
#else
typedef double orc_real;
#endif
/* a literal in the working precision */
#define ORC_C(x) ((orc_real)(x))

int g_sodecl_numeq;
int g_sodecl_numpar;
int g_sodecl_numnoi;
int g_sodecl_numsteps;
long g_sodecl_listsize;
double g_sodecl_dt;
double g_sodecl_eps;

enum { ORC_STOCH_EULER = 0, ORC_EULER = 1, ORC_RK4 = 2, ORC_IMPLICIT_EULER = 3, ORC_IMPLICIT_MIDPOINT = 4,
       ORC_DORMAND_PRINCE = 5 };
enum { ORC_FLAG_NEWTON_CAP = 1, ORC_FLAG_NONFINITE = 2 };

/* ---------------------------------------------------------------------- */
/* Explicit Euler: y1 = y0 + f(t, y0) * h.   src/kernels/euler.cl:10-18     */
static void orc_euler(orc_real h, orc_real t, orc_real *y, orc_real *ynew, orc_real *p)
{
    const int n = g_sodecl_numeq;
    sode_system(t, y, ynew, p);
    for (int e = 0; e < n; ++e)
        ynew[e] = y[e] + ynew[e] * h;
}

/* Classic RK4 with the reference's buffer reuse and accumulation order:
 * acc = k1 + 2 k2 + 2 k3 accumulated in place, then y + (acc + k4) h / 6.
 * src/kernels/rk4.cl:17-64                                                */
static void orc_rk4(orc_real h, orc_real t, orc_real *y, orc_real *ynew, orc_real *p)
{
    const int n = g_sodecl_numeq;
    orc_real stage[n], probe[n];
    sode_system(t, y, ynew, p);                                  /* k1 -> ynew */
    for (int e = 0; e < n; ++e) stage[e] = ynew[e];
    for (int e = 0; e < n; ++e) probe[e] = y[e] + (h * ORC_C(0.50)) * stage[e];
    sode_system(t + ORC_C(0.50) * h, probe, stage, p);                  /* k2 */
    for (int e = 0; e < n; ++e) ynew[e] = ynew[e] + ORC_C(2.00) * stage[e];
    for (int e = 0; e < n; ++e) probe[e] = y[e] + (h * ORC_C(0.50)) * stage[e];
    sode_system(t + ORC_C(0.50) * h, probe, stage, p);                  /* k3 */
    for (int e = 0; e < n; ++e) ynew[e] = ynew[e] + ORC_C(2.00) * stage[e];
    for (int e = 0; e < n; ++e) probe[e] = y[e] + h * stage[e];
    sode_system(t + h, probe, stage, p);                         /* k4 */
    for (int e = 0; e < n; ++e) ynew[e] = y[e] + (ynew[e] + stage[e]) * h / ORC_C(6.00);
}

/* The reference's "Thomas" solve (src/kernels/ie.cl:10-48, im.cl:3-41):
 * only three bands of the matrix are read -- super-diagonal `up` (rows
 * 0..n-3; the last two are zero), sub-diagonal `lo`, diagonal `d` -- and the
 * forward sweep pairs up[i] with d[i-1].  This is the reference's arithmetic,
 * not a textbook tridiagonal solve; the right-hand side v is overwritten.  */
static void orc_band_solve(int n, orc_real m[n][n], orc_real *v, orc_real *x)
{
    orc_real up[n], lo[n], d[n];
    for (int i = 0; i < n; ++i) {
        up[i] = (i < n - 2) ? m[i][i + 1] : 0;
        lo[i] = (i < n - 1) ? m[i + 1][i] : 0;
        d[i] = m[i][i];
    }
    for (int i = 1; i < n; ++i) {
        orc_real f = up[i] / d[i - 1];
        d[i] = d[i] - f * lo[i - 1];
        v[i] = v[i] - f * v[i - 1];
    }
    x[n - 1] = v[n - 1] / d[n - 1];
    for (int i = n - 2; i >= 0; --i)
        x[i] = (v[i] - lo[i] * x[i + 1]) / d[i];
}

#ifdef ORACLE_HAS_JACOBIAN
/* Implicit Euler: solve x - y - h f(t, x) = 0 by repeated banded Newton
 * corrections with matrix I - h J(x); stop when the L1 norm of the residual
 * drops below tol or after max_iter passes.   src/kernels/ie.cl:50-117    */
static int orc_implicit_euler(orc_real h, orc_real t, orc_real *y, orc_real *ynew, orc_real *p,
                              double tol, int max_iter, int *capped)
{
    const int n = g_sodecl_numeq;
    orc_real x[n], f[n], r[n], dx[n], m[n][n];
    int pass = 0, done = 0;
    for (int e = 0; e < n; ++e) x[e] = y[e];
    for (pass = 0; pass < max_iter; ++pass) {
        sode_system(t, x, f, p);
        for (int e = 0; e < n; ++e) r[e] = x[e] - y[e] - f[e] * h;
        orc_real l1 = 0;
        for (int e = 0; e < n; ++e) l1 = l1 + fabs(r[e]);
        if (l1 < (orc_real)tol) { done = 1; break; }
        calc_jacobian(x, m, p);
        for (int i = 0; i < n; ++i) {
            for (int j = 0; j < n; ++j) m[i][j] = m[i][j] * ORC_C(-1.00) * h;
            m[i][i] = m[i][i] + 1;
        }
        orc_band_solve(n, m, r, dx);
        for (int e = 0; e < n; ++e) x[e] = x[e] - dx[e];
    }
    if (!done) *capped = 1;
    for (int e = 0; e < n; ++e) ynew[e] = x[e];
    return done ? pass + 1 : pass;
}

/* Implicit midpoint: solve x - y - h f(t, (y + x)/2) = 0 with matrix
 * I - (h/2) J((y + x)/2) and an L2 residual test.  The right-hand side is
 * evaluated at time t (not t + h/2), as in the reference.
 * src/kernels/im.cl:43-118                                               */
static int orc_implicit_midpoint(orc_real h, orc_real t, orc_real *y, orc_real *ynew, orc_real *p,
                                 double tol, int max_iter, int *capped)
{
    const int n = g_sodecl_numeq;
    orc_real x[n], mid[n], f[n], r[n], dx[n], m[n][n];
    int pass = 0, done = 0;
    for (int e = 0; e < n; ++e) x[e] = y[e];
    for (pass = 0; pass < max_iter; ++pass) {
        for (int e = 0; e < n; ++e) mid[e] = (y[e] + x[e]) * ORC_C(0.5);
        sode_system(t, mid, f, p);
        for (int e = 0; e < n; ++e) r[e] = x[e] - y[e] - f[e] * h;
        orc_real l2 = 0;
        for (int e = 0; e < n; ++e) l2 = l2 + r[e] * r[e];
        if (sqrt(l2) < (orc_real)tol) { done = 1; break; }
        calc_jacobian(mid, m, p);
        for (int i = 0; i < n; ++i) {
            for (int j = 0; j < n; ++j) m[i][j] = m[i][j] * ORC_C(-0.50) * h;
            m[i][i] = m[i][i] + 1;
        }
        orc_band_solve(n, m, r, dx);
        for (int e = 0; e < n; ++e) x[e] = x[e] - dx[e];
    }
    if (!done) *capped = 1;
    for (int e = 0; e < n; ++e) ynew[e] = x[e];
    return done ? pass + 1 : pass;
}
#endif

/* ---------------------------------------------------------------------- */
/* Dormand-Prince 5(4) with adaptive steps over one record interval [t, t +
 * span] (Dormand & Prince, J. Comput. Appl. Math. 6(1), 1980; step control as
 * in Hairer, Norsett & Wanner, Solving ODEs I, II.4).  The reference has no
 * variable-step solver; this restates the library's own, in the same order
 * of operations: RMS error over equations of e_i / (atol + rtol max(|y_i|,
 * |y5_i|)) accepted at <= 1, next step hh * min(5, max(0.2, 0.9 err^-0.2)),
 * not larger after a rejection, the proposal kept when the step was cut to
 * the interval's end; first stage re-evaluated at each interval's start.
 * Returns 0 (state NaN) when the interval needs more than max_steps attempts
 * or a step too small to advance t.                                        */
static int orc_dp_interval(orc_real *t_io, orc_real *y, orc_real *p, orc_real *h_io, orc_real span, double rtol,
                           double atol, int max_steps, long *accepted)
{
    const int n = g_sodecl_numeq;
    orc_real k1[n], k2[n], k3[n], k4[n], k5[n], k6[n], k7[n], yt[n], y5[n];
    orc_real t = *t_io, h = *h_io;
    const orc_real t_end = t + span;
    int finite = 1;
    for (int e = 0; e < n; ++e) finite = finite && isfinite(y[e]);
    if (!finite) {
        *t_io = t_end;
        return 1;
    }
    if (!(h > 0) || !isfinite(h)) h = (orc_real)g_sodecl_dt;
    sode_system(t, y, k1, p);
    int rejected = 0;
    for (int it = 0; t < t_end; ++it) {
        if (it >= max_steps) break;
        const int last = t + h >= t_end;
        const orc_real hh = last ? t_end - t : h;
        if (!(hh > 0) || t + hh == t) break;
        for (int e = 0; e < n; ++e) yt[e] = y[e] + hh * (ORC_C(1.0 / 5.0) * k1[e]);
        sode_system(t + ORC_C(1.0 / 5.0) * hh, yt, k2, p);
        for (int e = 0; e < n; ++e) yt[e] = y[e] + hh * (ORC_C(3.0 / 40.0) * k1[e] + ORC_C(9.0 / 40.0) * k2[e]);
        sode_system(t + ORC_C(3.0 / 10.0) * hh, yt, k3, p);
        for (int e = 0; e < n; ++e)
            yt[e] = y[e] + hh * (ORC_C(44.0 / 45.0) * k1[e] + ORC_C(-56.0 / 15.0) * k2[e] + ORC_C(32.0 / 9.0) * k3[e]);
        sode_system(t + ORC_C(4.0 / 5.0) * hh, yt, k4, p);
        for (int e = 0; e < n; ++e)
            yt[e] = y[e] + hh * (ORC_C(19372.0 / 6561.0) * k1[e] + ORC_C(-25360.0 / 2187.0) * k2[e] +
                                 ORC_C(64448.0 / 6561.0) * k3[e] + ORC_C(-212.0 / 729.0) * k4[e]);
        sode_system(t + ORC_C(8.0 / 9.0) * hh, yt, k5, p);
        for (int e = 0; e < n; ++e)
            yt[e] = y[e] + hh * (ORC_C(9017.0 / 3168.0) * k1[e] + ORC_C(-355.0 / 33.0) * k2[e] +
                                 ORC_C(46732.0 / 5247.0) * k3[e] + ORC_C(49.0 / 176.0) * k4[e] +
                                 ORC_C(-5103.0 / 18656.0) * k5[e]);
        sode_system(t + hh, yt, k6, p);
        for (int e = 0; e < n; ++e)
            y5[e] = y[e] + hh * (ORC_C(35.0 / 384.0) * k1[e] + ORC_C(500.0 / 1113.0) * k3[e] +
                                 ORC_C(125.0 / 192.0) * k4[e] + ORC_C(-2187.0 / 6784.0) * k5[e] +
                                 ORC_C(11.0 / 84.0) * k6[e]);
        sode_system(t + hh, y5, k7, p);
        orc_real acc = 0;
        for (int e = 0; e < n; ++e) {
            const orc_real err = hh * (ORC_C(71.0 / 57600.0) * k1[e] + ORC_C(-71.0 / 16695.0) * k3[e] +
                                       ORC_C(71.0 / 1920.0) * k4[e] + ORC_C(-17253.0 / 339200.0) * k5[e] +
                                       ORC_C(22.0 / 525.0) * k6[e] + ORC_C(-1.0 / 40.0) * k7[e]);
            const orc_real sc = ORC_C(atol) + ORC_C(rtol) * fmax(fabs(y[e]), fabs(y5[e]));
            const orc_real q = err / sc;
            acc = acc + q * q;
        }
        const orc_real err = sqrt(acc / (orc_real)n);
        orc_real fac = (err > 0) ? ORC_C(0.9) * exp(ORC_C(-0.2) * log(err)) : ORC_C(5.0);
        fac = fmin(ORC_C(5.0), fmax(ORC_C(0.2), fac));
        if (err <= 1) {
            t = last ? t_end : t + hh;
            for (int e = 0; e < n; ++e) {
                y[e] = y5[e];
                k1[e] = k7[e];
            }
            ++*accepted;
            if (!last) h = hh * (rejected ? fmin((orc_real)1, fac) : fac);
            rejected = 0;
        } else {
            h = hh * (err == err ? fmin((orc_real)1, fac) : ORC_C(0.2));
            rejected = 1;
        }
    }
    *h_io = h;
    if (t < t_end) {
        for (int e = 0; e < n; ++e) y[e] = (orc_real)NAN;
        *t_io = t_end;
        return 0;
    }
    *t_io = t;
    return 1;
}

/* ---------------------------------------------------------------------- */
/* Threefry-2x64 with 20 rounds (Salmon, Moraes, Dror, Shaw, "Parallel random
 * numbers: as easy as 1, 2, 3", SC'11): the Threefish-derived block cipher
 * with rotation schedule 16,42,12,31,16,32,24,21, key-schedule parity word
 * 0x1BD11BDAA9FC1A22 and a key injection after every fourth round.  This
 * is the generator the reference takes from its vendored Random123 headers
 * (external/include/Random123/threefry.h, used by
 * src/kernels/stochastic_solver_caller.cl:51).                           */
static const unsigned orc_tf_rot[8] = {16, 42, 12, 31, 16, 32, 24, 21};

static void orc_threefry2x64_20(uint64_t c0, uint64_t c1, uint64_t k0, uint64_t k1, uint64_t out[2])
{
    const uint64_t ks[3] = {k0, k1, 0x1BD11BDAA9FC1A22ULL ^ k0 ^ k1};
    uint64_t x0 = c0 + ks[0];
    uint64_t x1 = c1 + ks[1];
    for (int r = 0; r < 20; ++r) {
        const unsigned s = orc_tf_rot[r & 7];
        x0 += x1;
        x1 = (x1 << s) | (x1 >> (64 - s));
        x1 ^= x0;
        if ((r & 3) == 3) {
            const unsigned inj = (unsigned)(r >> 2) + 1;
            x0 += ks[inj % 3];
            x1 += ks[(inj + 1) % 3] + inj;
        }
    }
    out[0] = x0;
    out[1] = x1;
}

/* 64-bit word -> double in the open interval (0, 1): the top 53 bits plus
 * one, times (2^53 - 1) * 2^-106.  Random123 u01.h:129-131 (open_open_64_53). */
static double orc_u01_open_open(uint64_t w)
{
    return (double)(1 + (w >> 11)) * 0x1.fffffffffffffp-54;
}

/* The per-orbit noise counter is stored as a double and converted to a
 * 64-bit counter word at every draw (stochastic_solver_caller.cl:49).  The
 * conversion is written out as x86-64 performs it, so negative counters
 * (the reference draws them from U(-1e11, 1e11), src/sodeclmgr.cpp:48-59)
 * wrap modulo 2^64 instead of depending on the compiler.                  */
static uint64_t orc_counter_word(double c)
{
    if (c >= 9223372036854775808.0)
        return ((uint64_t)(int64_t)(c - 9223372036854775808.0)) ^ 0x8000000000000000ULL;
    return (uint64_t)(int64_t)c;
}

/* One step's worth of Gaussian increments for orbit `gid`: ceil(nnoi/2)
 * Threefry draws with counter {gid, counter} and key {0, 0xf00dcafe}, the
 * counter advanced by one per draw, each pair turned into sqrt(h)-scaled
 * normals by Box-Muller (cos first, the sin partner dropped for an odd
 * count).   src/kernels/stochastic_solver_caller.cl:31-66                */
static void orc_noise(long gid, double *counter, orc_real sqrt_h, orc_real *noise)
{
    const int nnoi = g_sodecl_numnoi;
    const int ncalls = (int)ceil((float)((float)nnoi * 0.5));
    int k = 0;
    orc_real u0 = 0, u1 = 0;
    for (int c = 0; c < ncalls; ++c) {
        uint64_t w[2];
        orc_threefry2x64_20((uint64_t)gid, orc_counter_word(*counter), 0, 0xf00dcafeULL, w);
        *counter = *counter + 1;
        if (k < nnoi) {
            u0 = (orc_real)orc_u01_open_open(w[0]);
            u1 = (orc_real)orc_u01_open_open(w[1]);
            noise[k] = (sqrt(-2 * log(u0)) * cos(ORC_C(2 * M_PI) * u1)) * sqrt_h;
            k = k + 1;
        }
        if (k < nnoi) {
            noise[k] = (sqrt(-2 * log(u0)) * sin(ORC_C(2 * M_PI) * u1)) * sqrt_h;
            k = k + 1;
        }
    }
}

#ifdef ORACLE_HAS_STOCH
/* Euler-Maruyama: y1 = y0 + f h + g(y0, noise).   stochastic_euler.cl:10-22 */
static void orc_euler_maruyama(orc_real h, orc_real t, orc_real *y, orc_real *ynew, orc_real *p, orc_real *noise)
{
    const int n = g_sodecl_numeq;
    orc_real g[n];
    sode_system(t, y, ynew, p);
    sode_system_stoch(t, y, g, p, noise);
    for (int e = 0; e < n; ++e)
        ynew[e] = y[e] + ynew[e] * h + g[e];
}
#endif

/* ---------------------------------------------------------------------- */
/* The whole run for a block of orbits.                                    */
typedef struct oracle_job {
    int solver;              /* 0..4, solver_Type numbering */
    int neq, npar, nnoi;
    int ksteps;              /* steps per record interval */
    double dt;               /* the step the program is built with */
    long nchunks;            /* record intervals; records = nchunks + 1 */
    long n;                  /* orbits in this job */
    long orbit_offset;       /* global index of the job's first orbit */
    double *t;               /* [n] in/out */
    double *y;               /* [n][neq] in/out */
    const double *p;         /* [n][npar] */
    double *counters;        /* [n] in/out, stochastic solver only */
    double *records;         /* [(nchunks+1)][neq][n] or NULL */
    double newton_tol;
    int newton_max_iter;
    long *newton_passes;     /* [n] or NULL */
    int *flags;              /* [n] or NULL */
    int nthreads;            /* 0: OpenMP default */
    double rtol, atol;       /* solver 5: error tolerances */
    int max_steps;           /* solver 5: step attempts per record interval */
} oracle_job;

/* Runs every orbit of the job: the record before each interval of ksteps
 * steps and one after the last, the layout [record][equation][orbit] of
 * src/sodeclmgr.cpp:951-1015; the state carried across intervals as the
 * reference carries it in its device buffers (solver_caller.cl:19-50).   */
int oracle_run(const oracle_job *job)
{
    if (job->neq <= 0 || job->npar < 0 || job->n < 0 || job->ksteps < 0) return -1;
    if (job->solver == ORC_STOCH_EULER) {
#ifndef ORACLE_HAS_STOCH
        return -7;
#else
        if (job->nnoi <= 0 || !job->counters) return -1;
#endif
    }
    if (job->solver == ORC_IMPLICIT_EULER || job->solver == ORC_IMPLICIT_MIDPOINT) {
#ifndef ORACLE_HAS_JACOBIAN
        return -6;
#endif
    }
    if (job->solver < 0 || job->solver > 5) return -1;

    g_sodecl_numeq = job->neq;
    g_sodecl_numpar = job->npar;
    g_sodecl_numnoi = job->nnoi;
    g_sodecl_numsteps = job->ksteps;
    g_sodecl_listsize = job->n;
    g_sodecl_dt = job->dt;
    g_sodecl_eps = job->newton_tol;

    const int neq = job->neq, npar = job->npar > 0 ? job->npar : 1, nnoi = job->nnoi > 0 ? job->nnoi : 1;
    const long n = job->n;
    const orc_real h = (orc_real)job->dt;
    const orc_real sqrt_h = (orc_real)sqrt(h);

#ifdef _OPENMP
    if (job->nthreads > 0) omp_set_num_threads(job->nthreads);
#pragma omp parallel for schedule(dynamic, 16)
#endif
    for (long i = 0; i < n; ++i) {
        orc_real y[neq], ynew[neq], p[npar], noise[nnoi];
        orc_real t = (orc_real)job->t[i];
        for (int e = 0; e < neq; ++e) y[e] = (orc_real)job->y[i * neq + e];
        for (int k = 0; k < job->npar; ++k) p[k] = (orc_real)job->p[i * job->npar + k];
        double counter = job->counters ? job->counters[i] : 0.0;
        long passes = 0;
        int capped = 0;
        (void)noise; (void)sqrt_h; (void)capped;

        /* solver 5: the orbit's next step size rides in the counters array */
        orc_real hstate = (orc_real)counter;
        const orc_real span = (orc_real)job->ksteps * h;
        for (long c = 0; c <= job->nchunks; ++c) {
            if (job->records)
                for (int e = 0; e < neq; ++e)
                    job->records[((size_t)c * neq + e) * n + i] = (double)y[e];
            if (c == job->nchunks) break;
            if (job->solver == ORC_DORMAND_PRINCE) {
                if (!orc_dp_interval(&t, y, p, &hstate, span, job->rtol, job->atol, job->max_steps, &passes))
                    capped = 1;
                counter = (double)hstate;
                continue;
            }
            for (int s = 0; s < job->ksteps; ++s) {
                switch (job->solver) {
                case ORC_EULER: orc_euler(h, t, y, ynew, p); break;
                case ORC_RK4: orc_rk4(h, t, y, ynew, p); break;
#ifdef ORACLE_HAS_JACOBIAN
                case ORC_IMPLICIT_EULER:
                    passes += orc_implicit_euler(h, t, y, ynew, p, job->newton_tol, job->newton_max_iter, &capped);
                    break;
                case ORC_IMPLICIT_MIDPOINT:
                    passes += orc_implicit_midpoint(h, t, y, ynew, p, job->newton_tol, job->newton_max_iter, &capped);
                    break;
#endif
#ifdef ORACLE_HAS_STOCH
                case ORC_STOCH_EULER:
                    orc_noise(job->orbit_offset + i, &counter, sqrt_h, noise);
                    orc_euler_maruyama(h, t, y, ynew, p, noise);
                    break;
#endif
                default: break;
                }
                t = t + h;
                for (int e = 0; e < neq; ++e) y[e] = ynew[e];
            }
        }
        job->t[i] = (double)t;
        int nonfinite = 0;
        for (int e = 0; e < neq; ++e) {
            job->y[i * neq + e] = (double)y[e];
            if (!isfinite(y[e])) nonfinite = 1;
        }
        if (job->counters) job->counters[i] = counter;
        if (job->newton_passes) job->newton_passes[i] = passes;
        if (job->flags) job->flags[i] = (capped ? ORC_FLAG_NEWTON_CAP : 0) | (nonfinite ? ORC_FLAG_NONFINITE : 0);
    }
    return 0;
}

/* Raw generator access for the known-answer tests. */
void oracle_threefry2x64_20(const uint64_t ctr[2], const uint64_t key[2], uint64_t out[2])
{
    orc_threefry2x64_20(ctr[0], ctr[1], key[0], key[1], out);
}

double oracle_u01_open_open_64_53(uint64_t w) { return orc_u01_open_open(w); }

uint64_t oracle_counter_word(double c) { return orc_counter_word(c); }

/* Noise increments for `nsteps` steps of orbit gid, starting from `counter`:
 * out[step * nnoi + k]. */
void oracle_noise_stream(long gid, double counter, int nnoi, double dt, long nsteps, double *out)
{
    orc_real noise[nnoi > 0 ? nnoi : 1];
    g_sodecl_numnoi = nnoi;
    const orc_real sqrt_h = (orc_real)sqrt((orc_real)dt);
    for (long s = 0; s < nsteps; ++s) {
        orc_noise(gid, &counter, sqrt_h, noise);
        for (int k = 0; k < nnoi; ++k) out[s * nnoi + k] = (double)noise[k];
    }
}

int oracle_precision_bits(void) { return (int)(sizeof(orc_real) * 8); }

#endif
