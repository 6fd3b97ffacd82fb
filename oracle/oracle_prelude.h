/*
 * oracle_prelude.h -- TEST INFRASTRUCTURE ONLY (CPU oracle).
 *
 * Lets a SODECL system file (OpenCL C: `sode_system`, `calc_jacobian`,
 * `sode_system_stoch`) compile as plain C99 on the host, so the oracle in
 * oracle_solvers.h can integrate it.  Nothing in the shipped library
 * includes this file.
 *
 * The reference bakes the sizes and the step into the program text as
 * #defines (src/sodeclmgr.cpp:379-430).  Here they name process globals,
 * so one compiled oracle serves every size: array parameters such as
 * `double jac[_numeq_][_numeq_]` become C99 variably-modified parameters,
 * with the same arithmetic.
 */
#ifndef SODECL_ORACLE_PRELUDE_H
#define SODECL_ORACLE_PRELUDE_H

#include <stdint.h>
/* type-generic math: sin/exp/... follow the argument type, as OpenCL C's
 * overloaded built-ins do, so a float build evaluates in float */
#include <tgmath.h>

/* OpenCL C address-space / function qualifiers have no meaning on the host */
#define __kernel
#define __global
#define __local
#define __private
#define __constant const

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* OpenCL C's sincos(x, &c): returns sin(x), stores cos(x) */
static inline double sodecl_sincos_d(double x, double *c) { *c = cos(x); return sin(x); }
static inline float sodecl_sincos_f(float x, float *c) { *c = cos(x); return sin(x); }
#define sincos(x, c) _Generic((x), float: sodecl_sincos_f, default: sodecl_sincos_d)(x, c)

extern int g_sodecl_numeq;
extern int g_sodecl_numpar;
extern int g_sodecl_numnoi;
extern int g_sodecl_numsteps;
extern long g_sodecl_listsize;
extern double g_sodecl_dt;
extern double g_sodecl_eps;

#define _numeq_ g_sodecl_numeq
#define _numpar_ g_sodecl_numpar
#define _numnoi_ g_sodecl_numnoi
#define _numsteps_ g_sodecl_numsteps
#define _listsize_ g_sodecl_listsize
#define _m_dt_ g_sodecl_dt
#define _epsilon1_ g_sodecl_eps

#endif
