// opcount.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Counts the source-level floating-point operations of a SODECL system file:
// the file is compiled with `double` mapped to a scalar type that counts
// + - * / and every math-library call (each 1; negation and operations on
// compile-time constants 0, since those fold).  Prints, for the given state
// and parameters, the counts of one sode_system call and one calc_jacobian
// call, so the per-orbit-step operation counts used by the throughput
// roofline are derived from the source rather than estimated.
//
// Build (tests/test_opcount.py does this):
//   g++ -std=c++17 -O0 -DSYSTEM_FILE='"path/to/system.cl"' -DNUMEQ=6 -DNUMPAR=6 opcount.cpp
#include <cmath>
#include <cstdio>
#include <cstdlib>

struct Counted {
    double v;
    static long long add, mul, div, fun;
    Counted() : v(0) {}
    Counted(double x) : v(x) {}
    Counted(int x) : v(x) {}
    explicit operator double() const { return v; }
};
long long Counted::add = 0, Counted::mul = 0, Counted::div = 0, Counted::fun = 0;

#define OPC_BIN(op, ctr)                                                                        \
    inline Counted operator op(Counted a, Counted b) { ++Counted::ctr; return Counted(a.v op b.v); } \
    inline Counted operator op(Counted a, double b) { ++Counted::ctr; return Counted(a.v op b); }    \
    inline Counted operator op(double a, Counted b) { ++Counted::ctr; return Counted(a op b.v); }    \
    inline Counted operator op(Counted a, int b) { ++Counted::ctr; return Counted(a.v op b); }       \
    inline Counted operator op(int a, Counted b) { ++Counted::ctr; return Counted(a op b.v); }
OPC_BIN(+, add)
OPC_BIN(-, add)
OPC_BIN(*, mul)
OPC_BIN(/, div)
inline Counted operator-(Counted a) { return Counted(-a.v); }
inline Counted &operator+=(Counted &a, Counted b) { a = a + b; return a; }
inline Counted &operator-=(Counted &a, Counted b) { a = a - b; return a; }
inline Counted &operator*=(Counted &a, Counted b) { a = a * b; return a; }
#define OPC_CMP(op)                                                                  \
    inline bool operator op(Counted a, Counted b) { return a.v op b.v; }             \
    inline bool operator op(Counted a, double b) { return a.v op b; }                \
    inline bool operator op(double a, Counted b) { return a op b.v; }                \
    inline bool operator op(Counted a, int b) { return a.v op b; }
OPC_CMP(<) OPC_CMP(>) OPC_CMP(<=) OPC_CMP(>=) OPC_CMP(==) OPC_CMP(!=)
#define OPC_FUN(name)                                                                \
    inline Counted name(Counted a) { ++Counted::fun; return Counted(std::name(a.v)); }
OPC_FUN(exp) OPC_FUN(log) OPC_FUN(sin) OPC_FUN(cos) OPC_FUN(sqrt) OPC_FUN(tanh) OPC_FUN(tan)
inline Counted fabs(Counted a) { return Counted(std::fabs(a.v)); }
// OpenCL C's sincos(x, &c): two math calls
inline Counted sincos(Counted a, Counted *c)
{
    Counted::fun += 2;
    *c = Counted(std::cos(a.v));
    return Counted(std::sin(a.v));
}
inline Counted pow(Counted a, Counted b) { ++Counted::fun; return Counted(std::pow(a.v, b.v)); }
using std::exp; using std::log; using std::sin; using std::cos; using std::sqrt; using std::fabs;

#define _numeq_ NUMEQ
#define _numpar_ NUMPAR
#define _numnoi_ 1
#define __kernel
#define __global
#define double Counted
#include SYSTEM_FILE
#undef double

static long long total() { return Counted::add + Counted::mul + Counted::div + Counted::fun; }
static void reset() { Counted::add = Counted::mul = Counted::div = Counted::fun = 0; }

#ifdef HAS_JACOBIAN
// One Newton pass of the reference's implicit solvers, written out with the
// counting type in the order of src/kernels/ie.cl:50-105 (implicit Euler,
// midpoint = false) and src/kernels/im.cl:43-106 (implicit midpoint).  dt
// stands for the program's literal _m_dt_ (a plain double); converged = the
// pass that meets the stop test and returns before the Jacobian.
static long long newton_pass_ops(bool midpoint, bool converged, Counted *y, Counted *p, double dt)
{
    const int n = NUMEQ;
    Counted guess[NUMEQ], mid[NUMEQ], f[NUMEQ], r[NUMEQ], jac[NUMEQ][NUMEQ], a[NUMEQ], b[NUMEQ], c[NUMEQ], x[NUMEQ];
    for (int i = 0; i < n; ++i) guess[i] = y[i] + Counted(1e-3 * (i + 1)).v;  // an iterate away from y
    reset();
    if (midpoint)
        for (int i = 0; i < n; ++i) mid[i] = (y[i] + guess[i]) * 0.5;  // im.cl:67-70
    sode_system(Counted(0.0), midpoint ? mid : guess, f, p);
    for (int i = 0; i < n; ++i) r[i] = guess[i] - y[i] - f[i] * dt;   // ie.cl:56, im.cl:47
    Counted err(0.0);
    for (int i = 0; i < n; ++i) err = midpoint ? err + r[i] * r[i] : err + fabs(r[i]);
    if (midpoint) err = sqrt(err);                                    // im.cl:76-82, ie.cl:73-78
    if (converged) return total();
    calc_jacobian(midpoint ? mid : guess, jac, p);
    for (int i = 0; i < n; ++i) {                                     // ie.cl:84-92, im.cl:86-93
        for (int j = 0; j < n; ++j) jac[i][j] = jac[i][j] * (midpoint ? -0.50 : -1.00) * dt;
        jac[i][i] = jac[i][i] + 1;
    }
    // the banded solve, ie.cl:10-48 (band copies are not arithmetic)
    for (int i = 0; i < n; ++i) {
        a[i] = (i < n - 2) ? jac[i][i + 1] : Counted(0.0);
        c[i] = (i < n - 1) ? jac[i + 1][i] : Counted(0.0);
        b[i] = jac[i][i];
    }
    for (int i = 1; i < n; ++i) {
        Counted m = a[i] / b[i - 1];
        b[i] = b[i] - m * c[i - 1];
        r[i] = r[i] - m * r[i - 1];
    }
    x[n - 1] = r[n - 1] / b[n - 1];
    for (int i = n - 2; i >= 0; --i) x[i] = (r[i] - c[i] * x[i + 1]) / b[i];
    for (int i = 0; i < n; ++i) guess[i] = guess[i] - x[i];          // ie.cl:95-98
    return total();
}
#endif

int main(int argc, char **argv)
{
    // argv: NUMEQ state values then NUMPAR parameter values
    if (argc != 1 + NUMEQ + NUMPAR) {
        std::fprintf(stderr, "need %d numbers\n", NUMEQ + NUMPAR);
        return 2;
    }
    Counted y[NUMEQ], f[NUMEQ], p[NUMPAR];
    for (int i = 0; i < NUMEQ; ++i) y[i] = Counted(std::atof(argv[1 + i]));
    for (int i = 0; i < NUMPAR; ++i) p[i] = Counted(std::atof(argv[1 + NUMEQ + i]));
    reset();
    sode_system(Counted(0.0), y, f, p);
    std::printf("rhs %lld add %lld mul %lld div %lld fun %lld\n", total(), Counted::add, Counted::mul, Counted::div,
                Counted::fun);
#ifdef HAS_JACOBIAN
    Counted jac[NUMEQ][NUMEQ];
    reset();
    calc_jacobian(y, jac, p);
    std::printf("jacobian %lld add %lld mul %lld div %lld fun %lld\n", total(), Counted::add, Counted::mul,
                Counted::div, Counted::fun);
    std::printf("ie_pass_converged %lld\n", newton_pass_ops(false, true, y, p, 1e-3));
    std::printf("ie_pass_full %lld\n", newton_pass_ops(false, false, y, p, 1e-3));
    std::printf("im_pass_converged %lld\n", newton_pass_ops(true, true, y, p, 1e-3));
    std::printf("im_pass_full %lld\n", newton_pass_ops(true, false, y, p, 1e-3));
#endif
    return 0;
}
