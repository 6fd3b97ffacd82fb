// Exact division through a reciprocal.  Shared, as text, by the NVRTC
// programs (embedded by the build) and the statically compiled test kernel in
// aux_kernels.cu.  Self-contained: no includes.
#ifndef SODECL_FASTDIV_CUH
#define SODECL_FASTDIV_CUH

// ---------------------------------------------------------------------------
// q = a*r, e = fma(-q, b, a), q' = fma(e, r, q) with r = RN(1/b) gives the
// correctly rounded a/b (Markstein, "Computation of elementary functions on
// the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990): r is
// within half an ulp of 1/b, q within one ulp of a/b, and the FMA residual
// is exact as long as nothing under- or overflows -- guaranteed here by
// requiring |a| and |b| in [2^-500, 2^500); anything else takes the IEEE
// division, except NaN operands, which return NaN at once.  The point:
// r = 1/b is a plain division of loop-invariant operands whenever the
// divisor is a parameter or a constant, so the
// compiler hoists it out of the step loop and each quotient costs one
// multiply and two FMAs instead of a full division.  Results are bit-for-bit
// those of IEEE division (a NaN's payload aside).
// sodecl_div_by takes r = 1.0 / b from its caller, for a divisor that serves
// several quotients (its reciprocal is then taken once); sodecl_div_rcp takes
// the reciprocal itself.
__device__ __forceinline__ double sodecl_div_by(double a, double b, double r)
{
    const double q = a * r;
    const double e = __fma_rn(-q, b, a);
    const double q2 = __fma_rn(e, r, q);
    const unsigned ea = ((unsigned)__double2hiint(a) >> 20) & 0x7ffu;
    const unsigned eb = ((unsigned)__double2hiint(b) >> 20) & 0x7ffu;
    if ((ea - 523u) < 1000u && (eb - 523u) < 1000u)
        return q2;
    // a NaN operand makes the quotient NaN (IEEE 754); spare it the division's
    // special-case path, which orbits that have diverged would take every step
    if (a != a || b != b)
        return a + b;
    return a / b;
}

__device__ __forceinline__ double sodecl_div_rcp(double a, double b) { return sodecl_div_by(a, b, 1.0 / b); }

// The same in binary32, with the range [2^-60, 2^60) for |a| and |b|: there
// r, q, the product q*b and the residual stay normal floats, so the residual is
// exact and q' the correctly rounded quotient.
__device__ __forceinline__ float sodecl_div_by(float a, float b, float r)
{
    const float q = a * r;
    const float e = __fmaf_rn(-q, b, a);
    const float q2 = __fmaf_rn(e, r, q);
    const unsigned ea = ((unsigned)__float_as_int(a) >> 23) & 0xffu;
    const unsigned eb = ((unsigned)__float_as_int(b) >> 23) & 0xffu;
    if ((ea - 67u) < 120u && (eb - 67u) < 120u)
        return q2;
    if (a != a || b != b)
        return a + b;
    return a / b;
}

__device__ __forceinline__ float sodecl_div_rcp(float a, float b) { return sodecl_div_by(a, b, 1.0f / b); }

#endif
