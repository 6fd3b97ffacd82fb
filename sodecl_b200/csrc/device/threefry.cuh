// Counter-based Gaussian noise for the Euler-Maruyama solver.
//
// Shared, as text, by the NVRTC programs (embedded by the build) and by the
// statically compiled test kernels in aux_kernels.cu, so both run the same
// code.  Self-contained: no includes, usable under NVRTC and nvcc.
//
// Generator: Threefry-2x64 with 20 rounds (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11) -- the Threefish
// mixing function with rotation schedule 16 42 12 31 16 32 24 21, key
// parity word 0x1BD11BDAA9FC1A22 and a key injection after every fourth
// round.  Stream layout of the reference (src/kernels/
// stochastic_solver_caller.cl:31-66): key {0, 0xf00dcafe}, counter
// {orbit index, per-orbit draw counter}; each draw yields two 64-bit words,
// mapped to (0,1) doubles and turned into a Box-Muller pair.
#ifndef SODECL_THREEFRY_CUH
#define SODECL_THREEFRY_CUH

#define SODECL_TF_KEY0 0ULL
#define SODECL_TF_KEY1 0xf00dcafeULL

// One Threefry round pair step: x0 += x1; x1 = rotl(x1, r) ^ x0.
#define SODECL_TF_MIX(r)                                      \
    x0 += x1;                                                 \
    x1 = (x1 << (r)) | (x1 >> (64 - (r)));                    \
    x1 ^= x0;

__device__ __forceinline__ void sodecl_threefry2x64_20(unsigned long long c0, unsigned long long c1,
                                                       unsigned long long k0, unsigned long long k1,
                                                       unsigned long long &o0, unsigned long long &o1)
{
    const unsigned long long k2 = 0x1BD11BDAA9FC1A22ULL ^ k0 ^ k1;
    unsigned long long x0 = c0 + k0;
    unsigned long long x1 = c1 + k1;
    SODECL_TF_MIX(16) SODECL_TF_MIX(42) SODECL_TF_MIX(12) SODECL_TF_MIX(31)
    x0 += k1; x1 += k2 + 1ULL;
    SODECL_TF_MIX(16) SODECL_TF_MIX(32) SODECL_TF_MIX(24) SODECL_TF_MIX(21)
    x0 += k2; x1 += k0 + 2ULL;
    SODECL_TF_MIX(16) SODECL_TF_MIX(42) SODECL_TF_MIX(12) SODECL_TF_MIX(31)
    x0 += k0; x1 += k1 + 3ULL;
    SODECL_TF_MIX(16) SODECL_TF_MIX(32) SODECL_TF_MIX(24) SODECL_TF_MIX(21)
    x0 += k1; x1 += k2 + 4ULL;
    SODECL_TF_MIX(16) SODECL_TF_MIX(42) SODECL_TF_MIX(12) SODECL_TF_MIX(31)
    x0 += k2; x1 += k0 + 5ULL;
    o0 = x0;
    o1 = x1;
}

// 64-bit word -> double in (0, 1): (1 + top 53 bits) * (2^53 - 1) * 2^-106.
// Exact integer conversion and one correctly rounded multiply, so the value
// is bit-identical on every IEEE machine.
__device__ __forceinline__ double sodecl_u01_open_open(unsigned long long w)
{
    return (double)(1ULL + (w >> 11)) * 0x1.fffffffffffffp-54;
}

// The per-orbit draw counter is kept as a double (as the reference keeps it)
// and converted to the 64-bit counter word at every draw.  Conversion as
// x86-64 performs it: truncation toward zero, negative values wrapping
// modulo 2^64, values >= 2^63 through the unsigned range.  Valid for
// |c| < 2^64.
__device__ __forceinline__ unsigned long long sodecl_counter_word(double c)
{
    if (c >= 9223372036854775808.0)
        return ((unsigned long long)(long long)(c - 9223372036854775808.0)) ^ 0x8000000000000000ULL;
    return (unsigned long long)(long long)c;
}

// One draw's two words -> a Box-Muller pair scaled by sqrt(h), in precision R:
//   n0 = sqrt(-2 ln u0) cos(2 pi u1) sqrt(h),  n1 = ... sin(...)
// (stochastic_solver_caller.cl:56-63).
template <class R>
__device__ __forceinline__ void sodecl_gaussian_pair(unsigned long long w0, unsigned long long w1, R sqrt_h, R &n0, R &n1)
{
    const R u0 = (R)sodecl_u01_open_open(w0);
    const R u1 = (R)sodecl_u01_open_open(w1);
    const R rad = sqrt((R)(-2) * log(u0));
    const R ang = (R)(2 * 3.14159265358979323846) * u1;
    n0 = (rad * cos(ang)) * sqrt_h;
    n1 = (rad * sin(ang)) * sqrt_h;
}

#endif
