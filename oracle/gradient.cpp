// gradient.cpp -- TEST INFRASTRUCTURE ONLY.
//
// FP64 reference gradient for the discrete adjoint: forward-mode dual numbers
// (value + NUMPAR + NUMEQ tangents) pushed through the system file and a
// restatement of the Euler / RK4 steps (src/kernels/euler.cl:10-18,
// rk4.cl:17-64, same evaluation order) and of the implicit Euler / midpoint
// Newton passes (ie.cl, im.cl).  Exact to rounding; slow, so the tests use a
// few orbits.
//
// Build: g++ -O2 -std=c++17 -DSYSTEM_FILE='"x.cl"' -DNUMEQ=6 -DNUMPAR=6 gradient.cpp
// Run:   gradient <solver 1|2|3|4> <in.bin> <out.bin> [<newton tol> <newton pass limit>]
//   in:  int64 n, nchunks, ksteps; double dt; t0[n]; y0[n][neq]; p[n][npar];
//        targets[nchunks+1][neq][n]
//   out: loss[n]; grad_p[n][npar]; grad_y0[n][neq]
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

constexpr int K = NUMPAR + NUMEQ;

struct Dual {
    double v;
    double d[K];
    Dual() : v(0) { for (double &x : d) x = 0; }
    Dual(double x) : v(x) { for (double &z : d) z = 0; }
    Dual(int x) : Dual((double)x) {}
    explicit operator double() const { return v; }
    explicit operator int() const { return (int)v; }
};
inline Dual lin(double v, const Dual &a, double da)
{
    Dual r(v);
    for (int k = 0; k < K; ++k) r.d[k] = da * a.d[k];
    return r;
}
inline Dual lin2(double v, const Dual &a, double da, const Dual &b, double db)
{
    Dual r(v);
    for (int k = 0; k < K; ++k) r.d[k] = da * a.d[k] + db * b.d[k];
    return r;
}
inline Dual operator+(const Dual &a, const Dual &b) { return lin2(a.v + b.v, a, 1, b, 1); }
inline Dual operator-(const Dual &a, const Dual &b) { return lin2(a.v - b.v, a, 1, b, -1); }
inline Dual operator*(const Dual &a, const Dual &b) { return lin2(a.v * b.v, a, b.v, b, a.v); }
inline Dual operator/(const Dual &a, const Dual &b)
{
    const double q = a.v / b.v;
    return lin2(q, a, 1.0 / b.v, b, -q / b.v);
}
inline Dual operator-(const Dual &a) { return lin(-a.v, a, -1); }
inline Dual operator+(const Dual &a) { return a; }
#define DUAL_MIXED(op)                                                        \
    inline Dual operator op(const Dual &a, double b) { return a op Dual(b); } \
    inline Dual operator op(double a, const Dual &b) { return Dual(a) op b; } \
    inline Dual operator op(const Dual &a, int b) { return a op Dual(b); }    \
    inline Dual operator op(int a, const Dual &b) { return Dual(a) op b; }
DUAL_MIXED(+) DUAL_MIXED(-) DUAL_MIXED(*) DUAL_MIXED(/)
inline Dual &operator+=(Dual &a, const Dual &b) { return a = a + b; }
inline Dual &operator-=(Dual &a, const Dual &b) { return a = a - b; }
inline Dual &operator*=(Dual &a, const Dual &b) { return a = a * b; }
inline Dual &operator/=(Dual &a, const Dual &b) { return a = a / b; }
#define DUAL_CMP(op)                                                              \
    inline bool operator op(const Dual &a, const Dual &b) { return a.v op b.v; }  \
    inline bool operator op(const Dual &a, double b) { return a.v op b; }         \
    inline bool operator op(double a, const Dual &b) { return a op b.v; }         \
    inline bool operator op(const Dual &a, int b) { return a.v op b; }
DUAL_CMP(<) DUAL_CMP(>) DUAL_CMP(<=) DUAL_CMP(>=) DUAL_CMP(==) DUAL_CMP(!=)
inline Dual exp(const Dual &a) { const double e = std::exp(a.v); return lin(e, a, e); }
inline Dual log(const Dual &a) { return lin(std::log(a.v), a, 1.0 / a.v); }
inline Dual sqrt(const Dual &a) { const double s = std::sqrt(a.v); return lin(s, a, 0.5 / s); }
inline Dual sin(const Dual &a) { return lin(std::sin(a.v), a, std::cos(a.v)); }
inline Dual cos(const Dual &a) { return lin(std::cos(a.v), a, -std::sin(a.v)); }
inline Dual tanh(const Dual &a) { const double h = std::tanh(a.v); return lin(h, a, 1 - h * h); }
inline Dual fabs(const Dual &a) { return lin(std::fabs(a.v), a, a.v < 0 ? -1.0 : 1.0); }
using std::exp; using std::log; using std::sqrt; using std::sin; using std::cos; using std::fabs;

#define _numeq_ NUMEQ
#define _numpar_ NUMPAR
#define _numnoi_ 1
#define __kernel
#define __global
#define double Dual
#include SYSTEM_FILE
#undef double

using T = Dual;

static void step_euler(double h, const T &t, const T *y, T *ynew, T *p)
{
    T yy[NUMEQ];
    for (int e = 0; e < NUMEQ; ++e) yy[e] = y[e];
    sode_system(t, yy, ynew, p);
    for (int e = 0; e < NUMEQ; ++e) ynew[e] = y[e] + ynew[e] * h;
}

static void step_rk4(double h, const T &t, const T *y, T *ynew, T *p)
{
    T stage[NUMEQ], probe[NUMEQ], yy[NUMEQ];
    for (int e = 0; e < NUMEQ; ++e) yy[e] = y[e];
    sode_system(t, yy, ynew, p);
    for (int e = 0; e < NUMEQ; ++e) stage[e] = ynew[e];
    for (int e = 0; e < NUMEQ; ++e) probe[e] = y[e] + (h * 0.50) * stage[e];
    sode_system(t + 0.50 * h, probe, stage, p);
    for (int e = 0; e < NUMEQ; ++e) ynew[e] = ynew[e] + 2.00 * stage[e];
    for (int e = 0; e < NUMEQ; ++e) probe[e] = y[e] + (h * 0.50) * stage[e];
    sode_system(t + 0.50 * h, probe, stage, p);
    for (int e = 0; e < NUMEQ; ++e) ynew[e] = ynew[e] + 2.00 * stage[e];
    for (int e = 0; e < NUMEQ; ++e) probe[e] = y[e] + h * stage[e];
    sode_system(t + h, probe, stage, p);
    for (int e = 0; e < NUMEQ; ++e) ynew[e] = y[e] + (ynew[e] + stage[e]) * h / 6.00;
}

// The implicit solvers as the reference runs them (src/kernels/ie.cl:10-117,
// im.cl:3-118): quasi-Newton passes with the banded solve, stopping at the
// residual bound; dual numbers carry the derivatives through every pass.
static double g_newton_tol = 1e-7;
static long long g_newton_max = 1000;

static void band_solve(T (*m)[NUMEQ], T *v, T *x)
{
    T up[NUMEQ], lo[NUMEQ], d[NUMEQ];
    for (int i = 0; i < NUMEQ; ++i) {
        up[i] = (i < NUMEQ - 2) ? m[i][(i + 1) % NUMEQ] : T(0.0);
        lo[i] = (i < NUMEQ - 1) ? m[(i + 1) % NUMEQ][i] : T(0.0);
        d[i] = m[i][i];
    }
    for (int i = 1; i < NUMEQ; ++i) {
        const T f = up[i] / d[i - 1];
        d[i] = d[i] - f * lo[i - 1];
        v[i] = v[i] - f * v[i - 1];
    }
    x[NUMEQ - 1] = v[NUMEQ - 1] / d[NUMEQ - 1];
    for (int i = NUMEQ - 2; i >= 0; --i) x[i] = (v[i] - lo[i] * x[i + 1]) / d[i];
}

static void step_implicit(bool midpoint, double h, const T &t, const T *y, T *ynew, T *p)
{
    T x[NUMEQ], f[NUMEQ], r[NUMEQ], dx[NUMEQ], mid[NUMEQ], m[NUMEQ][NUMEQ];
    for (int e = 0; e < NUMEQ; ++e) x[e] = y[e];
    for (long long pass = 0; pass < g_newton_max; ++pass) {
        if (midpoint) {
            for (int e = 0; e < NUMEQ; ++e) mid[e] = (y[e] + x[e]) * 0.5;
            sode_system(t, mid, f, p);
        } else {
            sode_system(t, x, f, p);
        }
        T norm(0.0);
        for (int e = 0; e < NUMEQ; ++e) {
            r[e] = x[e] - y[e] - f[e] * h;
            norm = midpoint ? norm + r[e] * r[e] : norm + fabs(r[e]);
        }
        if ((midpoint ? sqrt(norm).v : norm.v) < g_newton_tol) break;
        calc_jacobian(midpoint ? mid : x, m, p);
        const double scale = midpoint ? -0.50 : -1.00;
        for (int i = 0; i < NUMEQ; ++i) {
            for (int j = 0; j < NUMEQ; ++j) m[i][j] = m[i][j] * scale * h;
            m[i][i] = m[i][i] + 1;
        }
        band_solve(m, r, dx);
        for (int e = 0; e < NUMEQ; ++e) x[e] = x[e] - dx[e];
    }
    for (int e = 0; e < NUMEQ; ++e) ynew[e] = x[e];
}

int main(int argc, char **argv)
{
    // argv: solver, input file, output file [, Newton tolerance, Newton pass limit]
    if (argc != 4 && argc != 6) return 2;
    const int solver = std::atoi(argv[1]);
    if (argc == 6) {
        g_newton_tol = std::atof(argv[4]);
        g_newton_max = std::atoll(argv[5]);
    }
    FILE *in = std::fopen(argv[2], "rb");
    if (!in) return 3;
    long long hdr[3];
    double dt;
    if (std::fread(hdr, sizeof(hdr), 1, in) != 1 || std::fread(&dt, sizeof(dt), 1, in) != 1) return 4;
    const long long n = hdr[0], nchunks = hdr[1], ksteps = hdr[2], nrec = nchunks + 1;
    std::vector<double> t0(n), y0(n * NUMEQ), p(n * NUMPAR), tg(nrec * NUMEQ * n);
    if (std::fread(t0.data(), 8, n, in) != (size_t)n || std::fread(y0.data(), 8, y0.size(), in) != y0.size() ||
        std::fread(p.data(), 8, p.size(), in) != p.size() || std::fread(tg.data(), 8, tg.size(), in) != tg.size())
        return 5;
    std::fclose(in);
    std::vector<double> loss(n), gp(n * NUMPAR), gy(n * NUMEQ);
    const double w = 1.0 / ((double)nrec * NUMEQ);
    for (long long i = 0; i < n; ++i) {
        T y[NUMEQ], ynew[NUMEQ], pp[NUMPAR];
        for (int j = 0; j < NUMPAR; ++j) { pp[j] = T(p[i * NUMPAR + j]); pp[j].d[j] = 1.0; }
        for (int e = 0; e < NUMEQ; ++e) { y[e] = T(y0[i * NUMEQ + e]); y[e].d[NUMPAR + e] = 1.0; }
        T t(t0[i]);
        T L(0.0);
        for (long long r = 0; r < nrec; ++r) {
            for (int e = 0; e < NUMEQ; ++e) {
                const T d = y[e] - tg[(r * NUMEQ + e) * n + i];
                L = L + d * d;
            }
            if (r == nchunks) break;
            for (long long s = 0; s < ksteps; ++s) {
                if (solver == 1) step_euler(dt, t, y, ynew, pp);
                else if (solver == 2) step_rk4(dt, t, y, ynew, pp);
                else step_implicit(solver == 4, dt, t, y, ynew, pp);
                t = t + dt;
                for (int e = 0; e < NUMEQ; ++e) y[e] = ynew[e];
            }
        }
        loss[i] = L.v * w;
        for (int j = 0; j < NUMPAR; ++j) gp[i * NUMPAR + j] = L.d[j] * w;
        for (int e = 0; e < NUMEQ; ++e) gy[i * NUMEQ + e] = L.d[NUMPAR + e] * w;
    }
    FILE *out = std::fopen(argv[3], "wb");
    if (!out) return 6;
    std::fwrite(loss.data(), 8, n, out);
    std::fwrite(gp.data(), 8, gp.size(), out);
    std::fwrite(gy.data(), 8, gy.size(), out);
    std::fclose(out);
    return 0;
}
