// f32x2.cuh -- paired single-precision arithmetic (sm_100 f32x2 instructions).
//
// One instruction performs the same IEEE operation on the two halves of a 64-bit
// register pair, each half rounded to nearest exactly as the scalar operation
// (__fadd_rn, __fmul_rn, __fmaf_rn) would be, denormals kept.  Pairing two
// independent scalar computations of identical shape therefore changes no bit
// of either result while halving the instructions issued for them.
//
// Caution, measured with ptxas 12.9 for sm_100a: unlike the scalar mul.rn.f32,
// a mul.rn.f32x2 whose product feeds an add/sub.rn.f32x2 may be contracted into
// one fused multiply-add (seen in a five-operation chain: both ends fused; the
// ptxas option --fmad=false does not prevent it).  Where the unfused rounding
// matters, form products with mulz2: fma(a, b, z) with z = -0.0 supplied at run
// time rounds exactly as a*b (x + -0 = x for every x, zeros keep their sign), and
// since the compiler cannot know z, nothing can be fused into it.
#pragma once

namespace piv {

__device__ __forceinline__ unsigned long long f2_bits(float2 a)
{
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
    return r;
}

__device__ __forceinline__ float2 f2_of(unsigned long long r)
{
    float2 a;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
    return a;
}

__device__ __forceinline__ float2 add2(float2 a, float2 b)
{
    unsigned long long r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2_bits(a)), "l"(f2_bits(b)));
    return f2_of(r);
}

__device__ __forceinline__ float2 sub2(float2 a, float2 b)
{
    unsigned long long r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2_bits(a)), "l"(f2_bits(b)));
    return f2_of(r);
}

__device__ __forceinline__ float2 mul2(float2 a, float2 b)
{
    unsigned long long r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2_bits(a)), "l"(f2_bits(b)));
    return f2_of(r);
}

// a * b + c with one rounding per half
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c)
{
    unsigned long long r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(f2_bits(a)), "l"(f2_bits(b)), "l"(f2_bits(c)));
    return f2_of(r);
}

__device__ __forceinline__ float2 dup2(float a) { return make_float2(a, a); }

// a * b, rounded once, never contracted with a following add (nz = {-0, -0}
// from a run-time value)
__device__ __forceinline__ float2 mulz2(float2 a, float2 b, float2 nz) { return fma2(a, b, nz); }

}  // namespace piv
