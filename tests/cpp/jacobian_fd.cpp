// Central-difference check of a system file's calc_jacobian (df/dy) and
// calc_jacobian_params (df/dp) against its sode_system, compiled as C++ on the
// host.  Build: g++ -DNUMEQ=6 -DNUMPAR=6 -DSYSTEM_FILE='"path.cl"' ...
// Reads states and parameters from stdin (NUMEQ then NUMPAR numbers per case)
// and prints, per case, the largest relative difference for J, for Jp and
// for the vector-Jacobian product.
#include <cmath>
#include <cstdio>

// OpenCL C's sincos(x, &c): returns sin(x), stores cos(x)
static double sincos(double x, double *c)
{
    *c = std::cos(x);
    return std::sin(x);
}

#define _numeq_ NUMEQ
#define _numpar_ NUMPAR
#define _numnoi_ 1
#include SYSTEM_FILE

static double rel(double fd, double an) { return std::fabs(fd - an) / (std::fabs(fd) + 1.0); }

int main()
{
    double y[NUMEQ], p[NUMPAR];
    for (;;) {
        for (int k = 0; k < NUMEQ; ++k)
            if (std::scanf("%lf", &y[k]) != 1) return 0;
        for (int k = 0; k < NUMPAR; ++k)
            if (std::scanf("%lf", &p[k]) != 1) return 1;
        double J[NUMEQ][NUMEQ], Jp[NUMEQ][NUMPAR], fa[NUMEQ], fb[NUMEQ];
        double Jfd[NUMEQ][NUMEQ], Jpfd[NUMEQ][NUMPAR];
        calc_jacobian(y, J, p);
        double ej = 0.0, ep = 0.0, ev = 0.0;
        for (int j = 0; j < NUMEQ; ++j) {
            const double h = 1e-6 * std::fmax(1.0, std::fabs(y[j]));
            double ya[NUMEQ], yb[NUMEQ];
            for (int k = 0; k < NUMEQ; ++k) ya[k] = yb[k] = y[k];
            ya[j] += h;
            yb[j] -= h;
            sode_system(0.0, ya, fa, p);
            sode_system(0.0, yb, fb, p);
            for (int i = 0; i < NUMEQ; ++i) {
                Jfd[i][j] = (fa[i] - fb[i]) / (2 * h);
                ej = std::fmax(ej, rel(Jfd[i][j], J[i][j]));
            }
        }
        for (int j = 0; j < NUMPAR; ++j) {
            const double h = 1e-6 * std::fmax(1.0, std::fabs(p[j]));
            double pa[NUMPAR], pb[NUMPAR];
            for (int k = 0; k < NUMPAR; ++k) pa[k] = pb[k] = p[k];
            pa[j] += h;
            pb[j] -= h;
            sode_system(0.0, y, fa, pa);
            sode_system(0.0, y, fb, pb);
            for (int i = 0; i < NUMEQ; ++i) Jpfd[i][j] = (fa[i] - fb[i]) / (2 * h);
        }
#ifdef HAS_JACP
        calc_jacobian_params(y, Jp, p);
        for (int j = 0; j < NUMPAR; ++j)
            for (int i = 0; i < NUMEQ; ++i) ep = std::fmax(ep, rel(Jpfd[i][j], Jp[i][j]));
#else
        (void)Jp;
#endif
#ifdef HAS_VJP
        double v[NUMEQ], yb[NUMEQ], pb[NUMPAR];
        for (int i = 0; i < NUMEQ; ++i) v[i] = 1.0 - 0.37 * i + 0.05 * i * i;
        for (int j = 0; j < NUMEQ; ++j) yb[j] = 0.25 * j;  // accumulated into, not overwritten
        for (int k = 0; k < NUMPAR; ++k) pb[k] = -0.5 * k;
        calc_vjp(0.0, y, v, yb, pb, p);
        for (int j = 0; j < NUMEQ; ++j) {
            double want = 0.25 * j;
            for (int i = 0; i < NUMEQ; ++i) want += v[i] * Jfd[i][j];
            ev = std::fmax(ev, rel(want, yb[j]));
        }
        for (int k = 0; k < NUMPAR; ++k) {
            double want = -0.5 * k;
            for (int i = 0; i < NUMEQ; ++i) want += v[i] * Jpfd[i][k];
            ev = std::fmax(ev, rel(want, pb[k]));
        }
#endif
        std::printf("%.3e %.3e %.3e\n", ej, ep, ev);
    }
}
