// fft_reg.cuh -- register-resident mixed-radix FFTs and cross-lane combines.
//
// A length-M transform (M in {2,3,4,6,8,12,16,24,32}) runs entirely in one
// thread's registers: decimation in time, radix 4 / 2 / 3 stages, twiddles are
// compile-time constants (piv::cx_cossin), fully unrolled.  Longer transforms
// (N = P*M, P in {2, 4}) split the input over P adjacent lanes by decimation in
// time; each lane transforms its M samples and a radix-P butterfly across the P
// lanes (warp shuffles) finishes the job.  SIGN = -1 is the forward transform
// exp(-2*pi*i*k*n/N), SIGN = +1 the inverse; neither is normalised.
#pragma once

#include "f32x2.cuh"
#include "piv_common.cuh"

namespace piv {

// Complex sums as one paired FP32 instruction each (f32x2): the same two IEEE
// additions, half the issue slots (measured +9% at 32 px, +6% at 64 px).
__device__ __forceinline__ float2 c_add(float2 a, float2 b) { return add2(a, b); }
__device__ __forceinline__ float2 c_sub(float2 a, float2 b) { return sub2(a, b); }

// v * exp(SIGN * 2*pi*i * m / N), constant twiddle.
template <int N, int m, int SIGN>
__device__ __forceinline__ float2 c_twiddle(float2 v)
{
    constexpr int mm = ((m % N) + N) % N;
    if constexpr (mm == 0) {
        return v;
    } else if constexpr (4 * mm == N) {            // SIGN * i
        return SIGN < 0 ? make_float2(v.y, -v.x) : make_float2(-v.y, v.x);
    } else if constexpr (2 * mm == N) {            // -1
        return make_float2(-v.x, -v.y);
    } else if constexpr (4 * mm == 3 * N) {        // -SIGN * i
        return SIGN < 0 ? make_float2(-v.y, v.x) : make_float2(v.y, -v.x);
    } else {
        constexpr cx_cs cs = cx_cossin(mm, N);
        constexpr float c = (float)cs.c;
        constexpr float s = (float)(SIGN * cs.s);
        return make_float2(v.x * c - v.y * s, v.x * s + v.y * c);
    }
}

template <int R, int SIGN>
__device__ __forceinline__ void butterfly(float2 (&t)[R])
{
    if constexpr (R == 2) {
        float2 a = t[0], b = t[1];
        t[0] = c_add(a, b);
        t[1] = c_sub(a, b);
    } else if constexpr (R == 3) {
        constexpr float k = 0.866025403784438646763723170752936f;   // sqrt(3)/2
        float2 s = c_add(t[1], t[2]), d = c_sub(t[1], t[2]);
        const float2 m = fma2(dup2(-0.5f), s, t[0]);           // t0 - s/2, one rounding
        t[0] = c_add(t[0], s);
        // y1 = m + SIGN*i*k*d, y2 = m - SIGN*i*k*d (scalar: each a fused multiply-add)
        constexpr float sk = (float)SIGN * k;
        t[1] = make_float2(m.x - sk * d.y, m.y + sk * d.x);
        t[2] = make_float2(m.x + sk * d.y, m.y - sk * d.x);
    } else {  // R == 4
        float2 a = c_add(t[0], t[2]), b = c_sub(t[0], t[2]);
        float2 c = c_add(t[1], t[3]), d = c_sub(t[1], t[3]);
        t[0] = c_add(a, c);
        t[2] = c_sub(a, c);
        // SIGN*i*d
        float2 id = SIGN < 0 ? make_float2(d.y, -d.x) : make_float2(-d.y, d.x);
        t[1] = c_add(b, id);
        t[3] = c_sub(b, id);
    }
}

// In-place transform of x[0..N) in registers.
template <int N, int SIGN>
struct RegFFT {
    static __device__ __forceinline__ void run(float2 (&x)[N])
    {
        if constexpr (N == 1) {
        } else if constexpr (N == 2 || N == 3 || N == 4) {
            butterfly<N, SIGN>(x);
        } else {
            constexpr int R = (N % 4 == 0) ? 4 : ((N % 2 == 0) ? 2 : 3);
            constexpr int M = N / R;
            float2 s[R][M];
#pragma unroll
            for (int r = 0; r < R; ++r)
#pragma unroll
                for (int m = 0; m < M; ++m) s[r][m] = x[R * m + r];
#pragma unroll
            for (int r = 0; r < R; ++r) RegFFT<M, SIGN>::run(s[r]);
            sfor<M>([&](auto kc) {
                constexpr int k = decltype(kc)::value;
                float2 t[R];
                t[0] = s[0][k];
                sfor<R - 1>([&](auto rc) {
                    constexpr int r = decltype(rc)::value + 1;
                    t[r] = c_twiddle<N, r * k, SIGN>(s[r][k]);
                });
                butterfly<R, SIGN>(t);
#pragma unroll
                for (int q = 0; q < R; ++q) x[k + M * q] = t[q];
            });
        }
    }
};

// Cross-lane completion of a length N = P*M transform.  On entry lane p holds
// the length-M transform of samples x[P*n + p]; the P lanes of one transform are
// adjacent (lane index mod P = p), or, for P = 2 with XM = 16, lanes l and l + 16.
// On exit it holds X[M*q + k], k = 0..M-1, for the block q = out_block<P>(p).
template <int P>
__device__ __forceinline__ int out_block(int p)
{
    if constexpr (P == 4) return (p >> 1) + 2 * (p & 1);
    else return p;
}

template <int P, int M, int SIGN, int XM = 1>
__device__ __forceinline__ void lane_combine(float2 (&y)[M], int p)
{
    if constexpr (P == 1) {
        return;
    } else {
        constexpr int N = P * M;
        // twiddle W_N^{p*k}
        sfor<M>([&](auto kc) {
            constexpr int k = decltype(kc)::value;
            if constexpr (k != 0) {
                float2 v = y[k];
                float2 w1 = c_twiddle<N, k, SIGN>(v);
                if constexpr (P == 2) {
                    y[k] = p ? w1 : v;
                } else {
                    float2 w2 = c_twiddle<N, 2 * k, SIGN>(v);
                    float2 w3 = c_twiddle<N, 3 * k, SIGN>(v);
                    y[k] = (p == 1) ? w1 : (p == 2) ? w2 : (p == 3) ? w3 : v;
                }
            }
        });
        if constexpr (P == 2) {
#pragma unroll
            for (int k = 0; k < M; ++k) {
                float2 o;
                o.x = __shfl_xor_sync(0xffffffffu, y[k].x, XM);
                o.y = __shfl_xor_sync(0xffffffffu, y[k].y, XM);
                y[k] = p ? c_sub(o, y[k]) : c_add(y[k], o);
            }
        } else {  // P == 4: radix-2 over p1 (xor 2), twiddle, radix-2 over p0 (xor 1)
            const int p1 = p >> 1, p0 = p & 1;
#pragma unroll
            for (int k = 0; k < M; ++k) {
                float2 o;
                o.x = __shfl_xor_sync(0xffffffffu, y[k].x, 2);
                o.y = __shfl_xor_sync(0xffffffffu, y[k].y, 2);
                float2 u = p1 ? c_sub(o, y[k]) : c_add(y[k], o);
                if (p == 3)  // W4^{p0*q0} with p0 = q0 = 1: multiply by SIGN*i
                    u = SIGN < 0 ? make_float2(u.y, -u.x) : make_float2(-u.y, u.x);
                o.x = __shfl_xor_sync(0xffffffffu, u.x, 1);
                o.y = __shfl_xor_sync(0xffffffffu, u.y, 1);
                y[k] = p0 ? c_sub(o, u) : c_add(u, o);
            }
        }
    }
}

// Forward (SIGN = -1) four-lane combine with the lane twiddles W_N^{p k} read from
// a table tw[p * M + k] instead of being selected among compile-time candidates:
// one complex product per sample, the same arithmetic as c_twiddle's.
template <int P, int M>
__device__ __forceinline__ void lane_combine_fwd_tab(float2 (&y)[M], int p, const float2 *__restrict__ tw)
{
    static_assert(P == 4, "table combine is the four-lane form");
#pragma unroll
    for (int k = 1; k < M; ++k) {
        const float2 w = tw[p * (M + 1) + k];     // rows padded to M + 1 entries
        const float2 v = y[k];
        y[k] = make_float2(v.x * w.x - v.y * w.y, v.x * w.y + v.y * w.x);
    }
    const int p1 = p >> 1, p0 = p & 1;
#pragma unroll
    for (int k = 0; k < M; ++k) {
        float2 o;
        o.x = __shfl_xor_sync(0xffffffffu, y[k].x, 2);
        o.y = __shfl_xor_sync(0xffffffffu, y[k].y, 2);
        float2 u = p1 ? c_sub(o, y[k]) : c_add(y[k], o);
        if (p == 3) u = make_float2(u.y, -u.x);          // W4^1 = -i
        o.x = __shfl_xor_sync(0xffffffffu, u.x, 1);
        o.y = __shfl_xor_sync(0xffffffffu, u.y, 1);
        y[k] = p0 ? c_sub(o, u) : c_add(u, o);
    }
}

}  // namespace piv
