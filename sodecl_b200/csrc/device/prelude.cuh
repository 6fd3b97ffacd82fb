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

#if SODECL_FP32
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
