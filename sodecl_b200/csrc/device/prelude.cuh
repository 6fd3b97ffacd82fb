// Prelude of every SODECL NVRTC program.
//
// The program is assembled by the host front end (program.cpp) as
//   config macros, this prelude, the noise generator, the reference's size
//   #defines, the user's system file (verbatim; in fp32 programs with
//   `double` mapped to `float` and float literals suffixed), the solver
//   kernels.
// It lets a SODECL system file written in OpenCL C (the functions
// sode_system / calc_jacobian / sode_system_stoch over `double` arrays)
// compile as CUDA C++: NVRTC runs with -default-device, so unannotated
// functions are device functions, and the OpenCL qualifiers and the
// built-ins a system file is likely to use are provided here.

typedef unsigned long long sodecl_u64;
typedef long long sodecl_i64;

#if SODECL_FAST_DIV
#if SODECL_FP32
typedef float sodecl_num_t;
#else
typedef double sodecl_num_t;
#endif
// A double (a float in FP32 programs) with the quotient above as its `/`.
// Every other operation is the plain operation on the scalar (so FMA
// contraction and results are unchanged).  Conversions out of it are
// explicit, so mixed expressions stay unambiguous; a system file that needs an
// implicit conversion fails to compile with it and the front end builds the
// plain program instead.
struct sodecl_num {
    sodecl_num_t v;
    __device__ __forceinline__ sodecl_num() = default;
    __device__ __forceinline__ constexpr sodecl_num(double x) : v((sodecl_num_t)x) {}
    __device__ __forceinline__ constexpr sodecl_num(float x) : v((sodecl_num_t)x) {}
    __device__ __forceinline__ constexpr sodecl_num(int x) : v((sodecl_num_t)x) {}
    __device__ __forceinline__ constexpr sodecl_num(unsigned x) : v((sodecl_num_t)x) {}
    __device__ __forceinline__ constexpr sodecl_num(long x) : v((sodecl_num_t)x) {}
    __device__ __forceinline__ constexpr sodecl_num(long long x) : v((sodecl_num_t)x) {}
    __device__ __forceinline__ constexpr sodecl_num(unsigned long x) : v((sodecl_num_t)x) {}
    __device__ __forceinline__ constexpr sodecl_num(unsigned long long x) : v((sodecl_num_t)x) {}
    __device__ __forceinline__ explicit operator double() const { return (double)v; }
    __device__ __forceinline__ explicit operator float() const { return (float)v; }
    __device__ __forceinline__ explicit operator int() const { return (int)v; }
    __device__ __forceinline__ explicit operator unsigned() const { return (unsigned)v; }
    __device__ __forceinline__ explicit operator long() const { return (long)v; }
    __device__ __forceinline__ explicit operator long long() const { return (long long)v; }
    __device__ __forceinline__ explicit operator unsigned long long() const { return (unsigned long long)v; }
    __device__ __forceinline__ explicit operator bool() const { return v != (sodecl_num_t)0; }
    __device__ __forceinline__ sodecl_num &operator+=(sodecl_num o) { v = v + o.v; return *this; }
    __device__ __forceinline__ sodecl_num &operator-=(sodecl_num o) { v = v - o.v; return *this; }
    __device__ __forceinline__ sodecl_num &operator*=(sodecl_num o) { v = v * o.v; return *this; }
    __device__ __forceinline__ sodecl_num &operator/=(sodecl_num o) { v = sodecl_div_rcp(v, o.v); return *this; }
    __device__ __forceinline__ sodecl_num &operator++() { v = v + (sodecl_num_t)1; return *this; }
    __device__ __forceinline__ sodecl_num &operator--() { v = v - (sodecl_num_t)1; return *this; }
};
__device__ __forceinline__ sodecl_num operator+(sodecl_num a) { return a; }
__device__ __forceinline__ sodecl_num operator-(sodecl_num a) { return sodecl_num(-a.v); }
__device__ __forceinline__ sodecl_num operator+(sodecl_num a, sodecl_num b) { return sodecl_num(a.v + b.v); }
__device__ __forceinline__ sodecl_num operator-(sodecl_num a, sodecl_num b) { return sodecl_num(a.v - b.v); }
__device__ __forceinline__ sodecl_num operator*(sodecl_num a, sodecl_num b) { return sodecl_num(a.v * b.v); }
__device__ __forceinline__ sodecl_num operator/(sodecl_num a, sodecl_num b) { return sodecl_num(sodecl_div_rcp(a.v, b.v)); }
__device__ __forceinline__ bool operator<(sodecl_num a, sodecl_num b) { return a.v < b.v; }
__device__ __forceinline__ bool operator>(sodecl_num a, sodecl_num b) { return a.v > b.v; }
__device__ __forceinline__ bool operator<=(sodecl_num a, sodecl_num b) { return a.v <= b.v; }
__device__ __forceinline__ bool operator>=(sodecl_num a, sodecl_num b) { return a.v >= b.v; }
__device__ __forceinline__ bool operator==(sodecl_num a, sodecl_num b) { return a.v == b.v; }
__device__ __forceinline__ bool operator!=(sodecl_num a, sodecl_num b) { return a.v != b.v; }
#define SODECL_NUM_UNARY(fn) \
    __device__ __forceinline__ sodecl_num fn(sodecl_num a) { return sodecl_num(::fn(a.v)); }
SODECL_NUM_UNARY(exp) SODECL_NUM_UNARY(exp2) SODECL_NUM_UNARY(expm1) SODECL_NUM_UNARY(log)
SODECL_NUM_UNARY(log2) SODECL_NUM_UNARY(log10) SODECL_NUM_UNARY(log1p) SODECL_NUM_UNARY(sqrt)
SODECL_NUM_UNARY(rsqrt) SODECL_NUM_UNARY(cbrt) SODECL_NUM_UNARY(sin) SODECL_NUM_UNARY(cos)
SODECL_NUM_UNARY(tan) SODECL_NUM_UNARY(asin) SODECL_NUM_UNARY(acos) SODECL_NUM_UNARY(atan)
SODECL_NUM_UNARY(sinh) SODECL_NUM_UNARY(cosh) SODECL_NUM_UNARY(tanh) SODECL_NUM_UNARY(asinh)
SODECL_NUM_UNARY(acosh) SODECL_NUM_UNARY(atanh) SODECL_NUM_UNARY(fabs) SODECL_NUM_UNARY(floor)
SODECL_NUM_UNARY(ceil) SODECL_NUM_UNARY(trunc) SODECL_NUM_UNARY(round) SODECL_NUM_UNARY(rint)
SODECL_NUM_UNARY(erf) SODECL_NUM_UNARY(erfc) SODECL_NUM_UNARY(tgamma) SODECL_NUM_UNARY(lgamma)
#define SODECL_NUM_BINARY(fn) \
    __device__ __forceinline__ sodecl_num fn(sodecl_num a, sodecl_num b) { return sodecl_num(::fn(a.v, b.v)); }
SODECL_NUM_BINARY(pow) SODECL_NUM_BINARY(fmin) SODECL_NUM_BINARY(fmax) SODECL_NUM_BINARY(fmod)
SODECL_NUM_BINARY(atan2) SODECL_NUM_BINARY(hypot) SODECL_NUM_BINARY(copysign) SODECL_NUM_BINARY(fdim)
SODECL_NUM_BINARY(remainder)
__device__ __forceinline__ sodecl_num fma(sodecl_num a, sodecl_num b, sodecl_num c) { return sodecl_num(::fma(a.v, b.v, c.v)); }
__device__ __forceinline__ sodecl_num abs(sodecl_num a) { return sodecl_num(::fabs(a.v)); }
__device__ __forceinline__ sodecl_num ldexp(sodecl_num a, int k) { return sodecl_num(::ldexp(a.v, k)); }
__device__ __forceinline__ bool isnan(sodecl_num a) { return ::isnan(a.v); }
__device__ __forceinline__ bool isinf(sodecl_num a) { return ::isinf(a.v); }
__device__ __forceinline__ bool isfinite(sodecl_num a) { return ::isfinite(a.v); }
__device__ __forceinline__ bool signbit(sodecl_num a) { return ::signbit(a.v); }
__device__ __forceinline__ void sincos(sodecl_num a, sodecl_num *s, sodecl_num *c) { ::sincos(a.v, &s->v, &c->v); }
#endif

#if SODECL_FAST_DIV
typedef sodecl_num real_t;
#elif SODECL_FP32
typedef float real_t;
#else
typedef double real_t;
#endif

// OpenCL C qualifiers: no meaning for a per-thread device function
#define __kernel
#define __global
#define __local
#define __private
#define __constant const
#define __read_only
#define __write_only

// OpenCL C scalar type names
typedef unsigned char uchar;
typedef unsigned short ushort;
typedef unsigned int uint;
typedef unsigned long long ulong;

#if SODECL_FP32
#define M_PI 3.14159265358979323846f
#define M_E 2.71828182845904523536f
#else
#define M_PI 3.14159265358979323846
#define M_E 2.71828182845904523536
#endif
#define M_PI_F 3.14159265358979323846f
#define M_E_F 2.71828182845904523536f

// OpenCL C built-ins without a CUDA counterpart of the same name
__device__ __forceinline__ double mad(double a, double b, double c) { return a * b + c; }
__device__ __forceinline__ float mad(float a, float b, float c) { return a * b + c; }
__device__ __forceinline__ double pown(double x, int n) { return pow(x, (double)n); }
__device__ __forceinline__ float pown(float x, int n) { return powf(x, (float)n); }
__device__ __forceinline__ double clamp(double x, double lo, double hi) { return fmin(fmax(x, lo), hi); }
__device__ __forceinline__ float clamp(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
__device__ __forceinline__ double mix(double a, double b, double t) { return a + (b - a) * t; }
__device__ __forceinline__ float mix(float a, float b, float t) { return a + (b - a) * t; }
__device__ __forceinline__ double sign(double x) { return x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : (x == x ? 0.0 : x)); }
__device__ __forceinline__ float sign(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : (x == x ? 0.0f : x)); }
// OpenCL C's sincos: returns sin(x) and stores cos(x), each the same value as
// sin(x) and cos(x) alone, with one argument reduction for both (CUDA's
// three-argument sincos stays available)
__device__ __forceinline__ double sincos(double x, double *c) { double s; ::sincos(x, &s, c); return s; }
__device__ __forceinline__ float sincos(float x, float *c) { float s; ::sincosf(x, &s, c); return s; }
#if SODECL_FAST_DIV
__device__ __forceinline__ sodecl_num sincos(sodecl_num x, sodecl_num *c) { sodecl_num_t s; ::sincos(x.v, &s, &c->v); return sodecl_num(s); }
__device__ __forceinline__ sodecl_num mad(sodecl_num a, sodecl_num b, sodecl_num c) { return a * b + c; }
__device__ __forceinline__ sodecl_num pown(sodecl_num x, int n) { return pow(x, sodecl_num((sodecl_num_t)n)); }
__device__ __forceinline__ sodecl_num clamp(sodecl_num x, sodecl_num lo, sodecl_num hi) { return fmin(fmax(x, lo), hi); }
__device__ __forceinline__ sodecl_num mix(sodecl_num a, sodecl_num b, sodecl_num t) { return a + (b - a) * t; }
__device__ __forceinline__ sodecl_num sign(sodecl_num x) { return sodecl_num(sign(x.v)); }
#endif
// native_/half_ variants: OpenCL allows them to be inaccurate; here they
// are the accurate functions, so results do not depend on the spelling
#define native_exp exp
#define native_log log
#define native_sin sin
#define native_cos cos
#define native_sqrt sqrt
#define native_rsqrt rsqrt
#define native_powr pow
#define half_exp exp
#define half_log log
#define half_sin sin
#define half_cos cos
#define half_sqrt sqrt
#define powr pow
