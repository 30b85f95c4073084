// xcorr_rect.cuh -- rectangular interrogation windows (nWindowSize = {h, w},
// h != w) for libbulkxcorr2d.
//
// The square-window engine keeps each window's plane in shared memory with one
// thread group per window; a rectangular window has columns and rows of two
// different lengths, so it takes a staged form instead, over a chunk of windows
// whose planes live in the caller's scratch:
//
//   rect_gather_kernel   one CTA per window: extraction at the reference's
//                        rounded origin, weights, mean removal (not in ensemble
//                        mode), energies and 1/sqrt(E_A E_B); packs z = a + i b
//                        (PIV_2d_cross_correlate.c:299-354);
//   rect_line_fft<L>     length-L register FFT of every column (L = h) or row
//                        (L = w) of every window, P adjacent lanes per line for
//                        L > 32 (the register FFT and lane combine of fft_reg.cuh);
//   rect_product_kernel  conj(C'), C' = 4 F_B conj(F_A), from the packed
//                        spectrum Z(k), Z(-k), for each (k, -k) pair in place;
//   rect_line_fft<L>     rows, then columns again: the inverse taken as
//                        conj(FFT(conj C')) with only the real part used;
//   rect_shift_kernel    real part / 4 / (h w), fftshift, into float planes (and
//                        the caller's plane dump);
//   fit_planes_kernel    the fitter on each raw plane with the correlation weight
//                        on its 5x5 patch, and the detectability ratio
//                        (lsqpeaklocate_lm, peak_detectability);
//   rect_finish_kernel   outputs: x = col - w/2, y = row - h/2, height * enorm
//                        (PIV_2d_cross_correlate.c:80-125).
// Windows that are masked or reach outside the frame are skipped and their
// outputs left untouched, as in the reference.
#pragma once

#include "xcorr_kernels.cuh"

namespace piv {

struct RectParams {
    const float *A, *B;
    long long img_stride;
    const float *mask;          // [nwy * nwx] (1 = skip) or null
    int H, W, nwy, nwx;
    long long nwt;
    const float *ctr_x, *ctr_y, *wA, *wB;
    int h, w, ensemble;
    long long w0;               // first window (image-major global index) of the chunk
    int count;                  // windows in the chunk
    float2 *Z;                  // [count][h * w] packed spectra
    float *pl;                  // [count][h * w] float planes
    float *enorm;               // [count]
    int *valid;                 // [count]
    float *planes_out;          // caller's plane dump [n][nwy][nwx][h][w] or null
};

constexpr int kRectThreads = 256;

__device__ __forceinline__ float2 rect_block_sum2(float a, float b, float2 *red)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = make_float2(a, b);
    __syncthreads();
    float2 t = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int k = 0; k < kRectThreads / 32; ++k) {
        t.x += red[k].x;
        t.y += red[k].y;
    }
    __syncthreads();
    return t;
}

__global__ void __launch_bounds__(kRectThreads) rect_gather_kernel(RectParams p)
{
    __shared__ float2 red[kRectThreads / 32];
    const int c = blockIdx.x;
    const long long idx = p.w0 + c;
    const int n = (int)(idx / p.nwt);
    const int iw = (int)(idx - (long long)n * p.nwt);
    const int ii = iw % p.nwx, jj = iw / p.nwx;
    const int hw = p.h * p.w;
    bool ok = !(p.mask && p.mask[iw] == 1.0f);
    const int r0 = (int)floor((double)p.ctr_y[jj] - ((double)p.h - 1.0) / 2.0 + 0.5);
    const int c0 = (int)floor((double)p.ctr_x[ii] - ((double)p.w - 1.0) / 2.0 + 0.5);
    if (r0 < 0 || c0 < 0 || r0 + p.h > p.H || c0 + p.w > p.W) ok = false;
    if (!ok) {
        if (threadIdx.x == 0) p.valid[c] = 0;
        return;
    }
    float2 *Z = p.Z + (long long)c * hw;
    const float *fa = p.A + (long long)n * p.img_stride + (long long)r0 * p.W + c0;
    const float *fb = p.B + (long long)n * p.img_stride + (long long)r0 * p.W + c0;
    float sa = 0.0f, sb = 0.0f;
    for (int e = threadIdx.x; e < hw; e += kRectThreads) {
        const int r = e / p.w, col = e - r * p.w;
        const float a = __fmul_rn(__ldg(fa + (long long)r * p.W + col), __ldg(p.wA + e));
        const float b = __fmul_rn(__ldg(fb + (long long)r * p.W + col), __ldg(p.wB + e));
        Z[e] = make_float2(a, b);
        sa += a;
        sb += b;
    }
    const float2 s = rect_block_sum2(sa, sb, red);
    const float ma = s.x / (float)hw, mb = s.y / (float)hw;
    float ea = 0.0f, eb = 0.0f;
    for (int e = threadIdx.x; e < hw; e += kRectThreads) {
        float2 z = Z[e];
        if (!p.ensemble) {
            z = make_float2(__fsub_rn(z.x, ma), __fsub_rn(z.y, mb));
            Z[e] = z;
        }
        ea = __fmaf_rn(z.x, z.x, ea);
        eb = __fmaf_rn(z.y, z.y, eb);
    }
    const float2 en = rect_block_sum2(ea, eb, red);
    if (threadIdx.x == 0) {
        p.enorm[c] = 1.0f / sqrtf(en.x * en.y);
        p.valid[c] = 1;
    }
}

// Forward length-L transform of every line of every valid window of the chunk:
// AXIS 0 the columns (length h, stride w), AXIS 1 the rows (length w, stride 1).
template <int L>
struct RectLine {
    static constexpr int P = (L <= 32) ? 1 : ((L == 48 || L == 64) ? 2 : 4);
    static constexpr int M = L / P;
};

template <int L, int AXIS>
__global__ void __launch_bounds__(128) rect_line_fft(RectParams p)
{
    constexpr int P = RectLine<L>::P, M = RectLine<L>::M;
    const long long gt = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = (int)(gt % P);
    const long long line_id = gt / P;
    const int nl = AXIS == 0 ? p.w : p.h;
    const long long n_lines = (long long)p.count * nl;
    const int win = line_id < n_lines ? (int)(line_id / nl) : 0;
    const int line = line_id < n_lines ? (int)(line_id % nl) : 0;
    const bool active = line_id < n_lines && p.valid[win] != 0;
    const long long stride = AXIS == 0 ? p.w : 1;
    float2 *base = p.Z + (long long)win * p.h * p.w + (AXIS == 0 ? line : (long long)line * p.w);
    float2 z[M];
#pragma unroll
    for (int k = 0; k < M; ++k) z[k] = active ? base[(long long)(P * k + lane) * stride] : make_float2(0.0f, 0.0f);
    RegFFT<M, -1>::run(z);
    lane_combine<P, M, -1>(z, lane);          // every lane of the warp takes part in the shuffles
    const int q = out_block<P>(lane);
    if (active) {
#pragma unroll
        for (int k = 0; k < M; ++k) base[(long long)(M * q + k) * stride] = z[k];
    }
}

// conj(C') at k and -k from the packed spectrum (Zm = conj Z(-k)):
// conj(C') = conj(-i (Z - Zm) conj(Z + Zm)).
__device__ __forceinline__ float2 rect_conj_cross(float2 zk, float2 zn)
{
    const float2 d = make_float2(zk.x - zn.x, zk.y + zn.y);
    const float2 s = make_float2(zk.x + zn.x, zk.y - zn.y);
    const float re = d.x * s.x + d.y * s.y;
    const float im = d.y * s.x - d.x * s.y;
    return make_float2(im, re);
}

__global__ void __launch_bounds__(256) rect_product_kernel(RectParams p)
{
    const int hw = p.h * p.w;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)p.count * hw) return;
    const int win = (int)(e / hw), k = (int)(e % hw);
    if (!p.valid[win]) return;
    const int ky = k / p.w, kx = k - ky * p.w;
    const int km = ((p.h - ky) % p.h) * p.w + (p.w - kx) % p.w;
    if (km < k) return;                        // its partner handles the pair
    float2 *Z = p.Z + (long long)win * hw;
    const float2 zk = Z[k], zn = Z[km];
    Z[k] = rect_conj_cross(zk, zn);
    if (km != k) Z[km] = rect_conj_cross(zn, zk);
}

__global__ void __launch_bounds__(256) rect_shift_kernel(RectParams p)
{
    const int hw = p.h * p.w;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)p.count * hw) return;
    const int win = (int)(e / hw), k = (int)(e % hw);
    const int r = k / p.w, col = k - r * p.w;
    const int o = ((r + p.h / 2) % p.h) * p.w + (col + p.w / 2) % p.w;
    float *pl = p.pl + (long long)win * hw;
    if (!p.valid[win]) {
        pl[o] = 0.0f;                          // keeps the fitter's pass over skipped windows short
        return;
    }
    const float v = (p.Z[(long long)win * hw + k].x * 0.25f) * (1.0f / (float)hw);
    pl[o] = v;
    if (p.planes_out) p.planes_out[(p.w0 + win) * hw + o] = v;
}

struct RectOut {
    float *pk_x, *pk_y, *pk_h, *sx, *sy, *sxy, *pk_ratio;
    const float *loc, *sd, *ratio;
    int n_peaks;
};

__global__ void __launch_bounds__(128) rect_finish_kernel(RectParams p, RectOut o)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= p.count || !p.valid[c]) return;
    const long long idx = p.w0 + c;
    const int n = (int)(idx / p.nwt);
    const int iw = (int)(idx - (long long)n * p.nwt);
    const float en = p.enorm[c];
    o.pk_ratio[(long long)n * p.nwt + iw] = o.ratio[c];
    const float hh = (float)p.h / 2.0f, hw2 = (float)p.w / 2.0f;
    for (int k = 0; k < o.n_peaks; ++k) {
        const long long out = (long long)n * o.n_peaks * p.nwt + (long long)k * p.nwt + iw;
        const long long l0 = (long long)c * 3 * o.n_peaks + k, l1 = l0 + o.n_peaks, l2 = l1 + o.n_peaks;
        o.pk_x[out] = __fsub_rn(o.loc[l1], hw2);
        o.pk_y[out] = __fsub_rn(o.loc[l0], hh);
        o.pk_h[out] = __fmul_rn(o.loc[l2], en);
        o.sx[out] = o.sd[l0];
        o.sy[out] = o.sd[l1];
        o.sxy[out] = o.sd[l2];
    }
}

}  // namespace piv
