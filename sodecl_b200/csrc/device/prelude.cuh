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
// A double with the quotient above as its `/`.  Every other operation is the
// plain double operation (so FMA contraction and results are unchanged).
// Conversions out of it are explicit, so mixed expressions stay unambiguous;
// a system file that needs an implicit conversion fails to compile with it
// and the front end builds the plain-double program instead.
struct sodecl_f64 {
    double v;
    __device__ __forceinline__ sodecl_f64() = default;
    __device__ __forceinline__ constexpr sodecl_f64(double x) : v(x) {}
    __device__ __forceinline__ constexpr sodecl_f64(float x) : v(x) {}
    __device__ __forceinline__ constexpr sodecl_f64(int x) : v(x) {}
    __device__ __forceinline__ constexpr sodecl_f64(unsigned x) : v(x) {}
    __device__ __forceinline__ constexpr sodecl_f64(long x) : v((double)x) {}
    __device__ __forceinline__ constexpr sodecl_f64(long long x) : v((double)x) {}
    __device__ __forceinline__ constexpr sodecl_f64(unsigned long x) : v((double)x) {}
    __device__ __forceinline__ constexpr sodecl_f64(unsigned long long x) : v((double)x) {}
    __device__ __forceinline__ explicit operator double() const { return v; }
    __device__ __forceinline__ explicit operator float() const { return (float)v; }
    __device__ __forceinline__ explicit operator int() const { return (int)v; }
    __device__ __forceinline__ explicit operator unsigned() const { return (unsigned)v; }
    __device__ __forceinline__ explicit operator long() const { return (long)v; }
    __device__ __forceinline__ explicit operator long long() const { return (long long)v; }
    __device__ __forceinline__ explicit operator unsigned long long() const { return (unsigned long long)v; }
    __device__ __forceinline__ explicit operator bool() const { return v != 0.0; }
    __device__ __forceinline__ sodecl_f64 &operator+=(sodecl_f64 o) { v = v + o.v; return *this; }
    __device__ __forceinline__ sodecl_f64 &operator-=(sodecl_f64 o) { v = v - o.v; return *this; }
    __device__ __forceinline__ sodecl_f64 &operator*=(sodecl_f64 o) { v = v * o.v; return *this; }
    __device__ __forceinline__ sodecl_f64 &operator/=(sodecl_f64 o) { v = sodecl_div_rcp(v, o.v); return *this; }
    __device__ __forceinline__ sodecl_f64 &operator++() { v = v + 1.0; return *this; }
    __device__ __forceinline__ sodecl_f64 &operator--() { v = v - 1.0; return *this; }
};
__device__ __forceinline__ sodecl_f64 operator+(sodecl_f64 a) { return a; }
__device__ __forceinline__ sodecl_f64 operator-(sodecl_f64 a) { return sodecl_f64(-a.v); }
__device__ __forceinline__ sodecl_f64 operator+(sodecl_f64 a, sodecl_f64 b) { return sodecl_f64(a.v + b.v); }
__device__ __forceinline__ sodecl_f64 operator-(sodecl_f64 a, sodecl_f64 b) { return sodecl_f64(a.v - b.v); }
__device__ __forceinline__ sodecl_f64 operator*(sodecl_f64 a, sodecl_f64 b) { return sodecl_f64(a.v * b.v); }
__device__ __forceinline__ sodecl_f64 operator/(sodecl_f64 a, sodecl_f64 b) { return sodecl_f64(sodecl_div_rcp(a.v, b.v)); }
__device__ __forceinline__ bool operator<(sodecl_f64 a, sodecl_f64 b) { return a.v < b.v; }
__device__ __forceinline__ bool operator>(sodecl_f64 a, sodecl_f64 b) { return a.v > b.v; }
__device__ __forceinline__ bool operator<=(sodecl_f64 a, sodecl_f64 b) { return a.v <= b.v; }
__device__ __forceinline__ bool operator>=(sodecl_f64 a, sodecl_f64 b) { return a.v >= b.v; }
__device__ __forceinline__ bool operator==(sodecl_f64 a, sodecl_f64 b) { return a.v == b.v; }
__device__ __forceinline__ bool operator!=(sodecl_f64 a, sodecl_f64 b) { return a.v != b.v; }
#define SODECL_F64_UNARY(fn) \
    __device__ __forceinline__ sodecl_f64 fn(sodecl_f64 a) { return sodecl_f64(::fn(a.v)); }
SODECL_F64_UNARY(exp) SODECL_F64_UNARY(exp2) SODECL_F64_UNARY(expm1) SODECL_F64_UNARY(log)
SODECL_F64_UNARY(log2) SODECL_F64_UNARY(log10) SODECL_F64_UNARY(log1p) SODECL_F64_UNARY(sqrt)
SODECL_F64_UNARY(rsqrt) SODECL_F64_UNARY(cbrt) SODECL_F64_UNARY(sin) SODECL_F64_UNARY(cos)
SODECL_F64_UNARY(tan) SODECL_F64_UNARY(asin) SODECL_F64_UNARY(acos) SODECL_F64_UNARY(atan)
SODECL_F64_UNARY(sinh) SODECL_F64_UNARY(cosh) SODECL_F64_UNARY(tanh) SODECL_F64_UNARY(asinh)
SODECL_F64_UNARY(acosh) SODECL_F64_UNARY(atanh) SODECL_F64_UNARY(fabs) SODECL_F64_UNARY(floor)
SODECL_F64_UNARY(ceil) SODECL_F64_UNARY(trunc) SODECL_F64_UNARY(round) SODECL_F64_UNARY(rint)
SODECL_F64_UNARY(erf) SODECL_F64_UNARY(erfc) SODECL_F64_UNARY(tgamma) SODECL_F64_UNARY(lgamma)
#define SODECL_F64_BINARY(fn) \
    __device__ __forceinline__ sodecl_f64 fn(sodecl_f64 a, sodecl_f64 b) { return sodecl_f64(::fn(a.v, b.v)); }
SODECL_F64_BINARY(pow) SODECL_F64_BINARY(fmin) SODECL_F64_BINARY(fmax) SODECL_F64_BINARY(fmod)
SODECL_F64_BINARY(atan2) SODECL_F64_BINARY(hypot) SODECL_F64_BINARY(copysign) SODECL_F64_BINARY(fdim)
SODECL_F64_BINARY(remainder)
__device__ __forceinline__ sodecl_f64 fma(sodecl_f64 a, sodecl_f64 b, sodecl_f64 c) { return sodecl_f64(::fma(a.v, b.v, c.v)); }
__device__ __forceinline__ sodecl_f64 abs(sodecl_f64 a) { return sodecl_f64(::fabs(a.v)); }
__device__ __forceinline__ sodecl_f64 ldexp(sodecl_f64 a, int k) { return sodecl_f64(::ldexp(a.v, k)); }
__device__ __forceinline__ bool isnan(sodecl_f64 a) { return ::isnan(a.v); }
__device__ __forceinline__ bool isinf(sodecl_f64 a) { return ::isinf(a.v); }
__device__ __forceinline__ bool isfinite(sodecl_f64 a) { return ::isfinite(a.v); }
__device__ __forceinline__ bool signbit(sodecl_f64 a) { return ::signbit(a.v); }
__device__ __forceinline__ void sincos(sodecl_f64 a, sodecl_f64 *s, sodecl_f64 *c) { ::sincos(a.v, &s->v, &c->v); }
#endif

#if SODECL_FP32
typedef float real_t;
#elif SODECL_FAST_DIV
typedef sodecl_f64 real_t;
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
__device__ __forceinline__ sodecl_f64 sincos(sodecl_f64 x, sodecl_f64 *c) { double s; ::sincos(x.v, &s, &c->v); return sodecl_f64(s); }
__device__ __forceinline__ sodecl_f64 mad(sodecl_f64 a, sodecl_f64 b, sodecl_f64 c) { return a * b + c; }
__device__ __forceinline__ sodecl_f64 pown(sodecl_f64 x, int n) { return pow(x, sodecl_f64((double)n)); }
__device__ __forceinline__ sodecl_f64 clamp(sodecl_f64 x, sodecl_f64 lo, sodecl_f64 hi) { return fmin(fmax(x, lo), hi); }
__device__ __forceinline__ sodecl_f64 mix(sodecl_f64 a, sodecl_f64 b, sodecl_f64 t) { return a + (b - a) * t; }
__device__ __forceinline__ sodecl_f64 sign(sodecl_f64 x) { return sodecl_f64(sign(x.v)); }
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
