// fusedwarp.cu -- libfusedwarp for sm_100a.
//
// Predictor-corrector image deformation (pivtools_cli/lib/fused_warp.c): per
// output pixel, upsample the coarse predictor (dy, dx) bicubically (Keys
// a = -0.75, replicate border), take half of it, and sample frame A at
// pixel - half and frame B at pixel + half (bicubic 4x4 or Lanczos-3 6x6 with a
// 4097-entry weight table; zero outside the image).
//
// impl 0 evaluates every product and sum in the order of the reference's scalar
// route (fused_warp.c:70-105, 175-207, 224-250) with unfused float operations,
// so results are bit-identical to it.  impl 1 (the default, as in the reference)
// uses, for stencils that lie inside the image, the association of the
// reference's AVX2 route (simd_warp.h:74-160): a column accumulator
// c[n] = sum_m wy[m]*img[m][n] built with fused multiply-adds, then
// val = (p0 + p1) + (p2 + p3) with p = wx*c (Lanczos: ((p0+p4) + (p1+p5)) + (p2+p3)).
// Border stencils use the scalar route in both.
#include <math.h>
#include <stdio.h>

#include <atomic>
#include <mutex>

#include "device_state.h"
#include "f32x2.cuh"
#include "piv_common.cuh"

namespace {

constexpr int kLutN = 4096;

__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }

// fused_warp.c:52-64
__device__ __forceinline__ void keys4(float d, float *w)
{
    const float s0 = fa(1.0f, d), q2 = fs(1.0f, d), s3 = fs(2.0f, d);
    w[1] = fa(fm(fm(fs(fm(1.25f, d), 2.25f), d), d), 1.0f);
    w[2] = fa(fm(fm(fs(fm(1.25f, q2), 2.25f), q2), q2), 1.0f);
    w[0] = fa(fm(fs(fm(fa(fm(-0.75f, s0), 3.75f), s0), 6.0f), s0), 3.0f);
    w[3] = fa(fm(fs(fm(fa(fm(-0.75f, s3), 3.75f), s3), 6.0f), s3), 3.0f);
}

// keys4 on two independent offsets at once (.x and .y), the same operations in
// the same order, so each half is bit-identical to keys4 of that offset.
// nz = {-0, -0} from a run-time value: the products are mulz2, never contracted.
__device__ __forceinline__ void keys4_x2(float2 d, float2 (&w)[4], float2 nz)
{
    using namespace piv;
    const float2 one = dup2(1.0f);
    auto mu = [&](float2 a, float2 b) { return mulz2(a, b, nz); };
    const float2 s0 = add2(one, d), q2 = sub2(one, d), s3 = sub2(dup2(2.0f), d);
    w[1] = add2(mu(mu(sub2(mu(dup2(1.25f), d), dup2(2.25f)), d), d), one);
    w[2] = add2(mu(mu(sub2(mu(dup2(1.25f), q2), dup2(2.25f)), q2), q2), one);
    w[0] = add2(mu(sub2(mu(add2(mu(dup2(-0.75f), s0), dup2(3.75f)), s0), dup2(6.0f)), s0), dup2(3.0f));
    w[3] = add2(mu(sub2(mu(add2(mu(dup2(-0.75f), s3), dup2(3.75f)), s3), dup2(6.0f)), s3), dup2(3.0f));
}

__device__ __forceinline__ void lanczos_w(float d, const float *lut, float *w)
{
    const float pos = fm(d, (float)kLutN);
    int k = (int)pos;
    float fr = fs(pos, (float)k);
    if (k >= kLutN) { k = kLutN - 1; fr = 0.0f; }
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        const float a = lut[k * 6 + q], b = lut[(k + 1) * 6 + q];
        w[q] = fa(a, fm(fr, fs(b, a)));
    }
}

// One bicubic sample from precomputed weights and stencil origin (iy, ix):
// sample_bicubic<1> after its weight step.
__device__ __forceinline__ float bicubic_from_weights(const float *__restrict__ img, int iy, int ix, const float *wy,
                                                      const float *wx, int H, int W)
{
    if (iy >= 0 && iy + 3 < H && ix >= 0 && ix + 3 < W) {
        const float *r = img + (iy * W + ix);
        float c[4];
#pragma unroll
        for (int n = 0; n < 4; ++n) c[n] = fm(__ldg(r + n), wy[0]);
#pragma unroll
        for (int m = 1; m < 4; ++m)
#pragma unroll
            for (int n = 0; n < 4; ++n) c[n] = __fmaf_rn(__ldg(r + m * W + n), wy[m], c[n]);
        const float p0 = fm(c[0], wx[0]), p1 = fm(c[1], wx[1]), p2 = fm(c[2], wx[2]), p3 = fm(c[3], wx[3]);
        return fa(fa(p0, p1), fa(p2, p3));
    }
    float v = 0.0f;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        const int row = iy + m;
        if (row < 0 || row >= H) continue;
#pragma unroll
        for (int n = 0; n < 4; ++n) {
            const int col = ix + n;
            if (col < 0 || col >= W) continue;
            v = fa(v, fm(fm(wy[m], wx[n]), __ldg(img + (long long)row * W + col)));
        }
    }
    return v;
}

template <int IMPL>
__device__ __forceinline__ float sample_bicubic(const float *__restrict__ img, float fy, float fx, int H, int W)
{
    const float fyf = floorf(fy), fxf = floorf(fx);
    const int iy = (int)fyf - 1, ix = (int)fxf - 1;
    float wy[4], wx[4];
    keys4(fs(fy, fyf), wy);
    keys4(fs(fx, fxf), wx);
    if (IMPL == 1 && iy >= 0 && iy + 3 < H && ix >= 0 && ix + 3 < W) {
        const float *r = img + (iy * W + ix);
        float c[4];
#pragma unroll
        for (int n = 0; n < 4; ++n) c[n] = fm(__ldg(r + n), wy[0]);
#pragma unroll
        for (int m = 1; m < 4; ++m)
#pragma unroll
            for (int n = 0; n < 4; ++n) c[n] = __fmaf_rn(__ldg(r + m * W + n), wy[m], c[n]);
        const float p0 = fm(c[0], wx[0]), p1 = fm(c[1], wx[1]), p2 = fm(c[2], wx[2]), p3 = fm(c[3], wx[3]);
        return fa(fa(p0, p1), fa(p2, p3));
    }
    float v = 0.0f;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        const int row = iy + m;
        if (row < 0 || row >= H) continue;
#pragma unroll
        for (int n = 0; n < 4; ++n) {
            const int col = ix + n;
            if (col < 0 || col >= W) continue;
            v = fa(v, fm(fm(wy[m], wx[n]), __ldg(img + (long long)row * W + col)));
        }
    }
    return v;
}

template <int IMPL>
__device__ __forceinline__ float sample_lanczos(const float *__restrict__ img, float fy, float fx, int H, int W,
                                                const float *lut)
{
    const float fyf = floorf(fy), fxf = floorf(fx);
    const int iy = (int)fyf - 2, ix = (int)fxf - 2;
    float wy[6], wx[6];
    lanczos_w(fs(fy, fyf), lut, wy);
    lanczos_w(fs(fx, fxf), lut, wx);
    if (IMPL == 1 && iy >= 0 && iy + 5 < H && ix >= 0 && ix + 5 < W) {
        const float *r = img + (iy * W + ix);
        float c[6];
#pragma unroll
        for (int n = 0; n < 6; ++n) c[n] = 0.0f;
#pragma unroll
        for (int m = 0; m < 6; ++m)
#pragma unroll
            for (int n = 0; n < 6; ++n) c[n] = __fmaf_rn(__ldg(r + m * W + n), wy[m], c[n]);
        float p[6];
#pragma unroll
        for (int n = 0; n < 6; ++n) p[n] = fm(c[n], wx[n]);
        return fa(fa(fa(p[0], p[4]), fa(p[1], p[5])), fa(p[2], p[3]));
    }
    float v = 0.0f;
#pragma unroll
    for (int m = 0; m < 6; ++m) {
        const int row = iy + m;
        if (row < 0 || row >= H) continue;
#pragma unroll
        for (int n = 0; n < 6; ++n) {
            const int col = ix + n;
            if (col < 0 || col >= W) continue;
            v = fa(v, fm(fm(wy[m], wx[n]), __ldg(img + (long long)row * W + col)));
        }
    }
    return v;
}

// np.interp(pixel, ctrs, arange(n)) with clamped ends (fused_warp.c:259-307); the
// segment is the one the reference's forward scan reaches for ascending centres.
__global__ void pred_index_kernel(const float *ctrs, int nc, float *lut, int n)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    if (nc == 1) { lut[p] = 0.0f; return; }
    const float x = (float)p;
    if (x <= ctrs[0]) { lut[p] = 0.0f; return; }
    if (x >= ctrs[nc - 1]) { lut[p] = (float)(nc - 1); return; }
    int lo = 0, hi = nc - 2;     // largest seg <= nc-2 with seg == 0 or ctrs[seg] < x
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (ctrs[mid] < x) lo = mid;
        else hi = mid - 1;
    }
    const int seg = lo;
    const float den = fs(ctrs[seg + 1], ctrs[seg]);
    if (den < 1e-12f) { lut[p] = (float)seg; return; }
    lut[p] = fa((float)seg, __fdiv_rn(fs(x, ctrs[seg]), den));
}

// Lanczos-3 weight table at d = i / 4096, i = 0..4096 (fused_warp.c:120-158).
// An input-independent constant of the algorithm: it is built once per process
// with the host libm's sinf -- the function the reference's table is built
// with, and not correctly rounded, so a device sin would differ from it in the
// last bit of a few hundred entries -- and copied into each call's tables.
float g_lut_host[(kLutN + 1) * 6];
float g_lut2_host[kLutN * 12];     // row k: the six weights at k, then the six at k + 1
std::once_flag g_lut_once;
void build_lut_host()
{
    for (int i = 0; i <= kLutN; ++i) {
        const float d = (float)i / (float)kLutN;
        for (int k = 0; k < 6; ++k) {
            const float t = d - (float)(k - 2), at = fabsf(t);
            float v;
            if (at < 1e-6f) v = 1.0f;
            else if (at >= 3.0f) v = 0.0f;
            else {
                const float pt = (float)M_PI * at, pta = pt / 3.0f;
                v = (sinf(pt) / pt) * (sinf(pta) / pta);
            }
            g_lut_host[i * 6 + k] = v;
        }
    }
    for (int i = 0; i < kLutN; ++i)
        for (int k = 0; k < 12; ++k) g_lut2_host[i * 12 + k] = g_lut_host[i * 6 + k];   // rows i and i + 1
}

struct WarpParams {
    const float *ia, *ib;
    float *oa, *ob;
    const float *pdy, *pdx;
    long long pred_stride;     // 0 = shared predictor
    long long img_stride;
    int N, H, W, nPY, nPX;
    const float *ly, *lx;      // pixel -> fractional predictor index
    const float *lut;          // Lanczos table or null
    const float4 *lut2;        // the same table as 48-byte rows {w(k), w(k + 1)}, k < kLutN
    const float4 *wyb;         // per row: predictor row weights as pairs {w0,w0,w1,w1}, {w2,w2,w3,w3}
    const int *byr;            // per row: first predictor row of the 4x4 stencil
    int round_shifts;
    int rows;                  // output rows per thread
    float neg_zero;            // -0.0f, passed at run time (see mulz2)
};

// Per-row side of the bicubic predictor (fused_warp.c:224-250): the Keys weights
// of each output row's fractional predictor index, stored twice each so that the
// warp kernel reads them as ready-made f32x2 operands, and the stencil's first row.
__global__ void row_weights_kernel(const float *ly, int H, float4 *wyb, int *byr)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= H) return;
    const float f = ly[i], ff = floorf(f);
    float w[4];
    keys4(fs(f, ff), w);
    wyb[2 * i] = make_float4(w[0], w[0], w[1], w[1]);
    wyb[2 * i + 1] = make_float4(w[2], w[2], w[3], w[3]);
    byr[i] = (int)ff - 1;
}

// Output rows per thread (default).  The rows of one thread share the
// column-side work (predictor column weights and indices) and, while they fall
// in the same predictor cell row, the 4x4 predictor patch, which stays in
// registers (measured with the paired kernel: 16 rows 3% faster than 8, 4 rows
// 7% slower).  Rows per thread and the block height are launch settings
// (pivb_warp_set_launch) that the autotuner may change.
constexpr int kWarpRows = 16;

template <int MODE, int IMPL>
__global__ void __launch_bounds__(128) warp_kernel(WarpParams p)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i0 = (blockIdx.y * blockDim.y + threadIdx.y) * p.rows;
    const int n = blockIdx.z;
    if (j >= p.W || i0 >= p.H) return;
    const float *dy = p.pdy + n * p.pred_stride, *dx = p.pdx + n * p.pred_stride;
    // column side of the bicubic predictor (fused_warp.c:224-250)
    const float fx = p.lx[j], fxf = floorf(fx);
    const int bx = (int)fxf - 1;
    float wx[4];
    keys4(fs(fx, fxf), wx);
    int cq[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) cq[q] = min(max(bx + q, 0), p.nPX - 1);
    float py[4][4], px[4][4];
    int cur_by = -0x7fffffff;
    const float *a = p.ia + n * p.img_stride, *b = p.ib + n * p.img_stride;
    const int i_end = min(i0 + p.rows, p.H);
#pragma unroll 1
    for (int i = i0; i < i_end; ++i) {
        // Phase A: bicubic predictor, products and sums in the scalar route's order
        const float fiy = p.ly[i], fiyf = floorf(fiy);
        const int by = (int)fiyf - 1;
        float wy[4];
        keys4(fs(fiy, fiyf), wy);
        if (by != cur_by) {          // warp-uniform: all lanes share row i
            cur_by = by;
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const int r = min(max(by + m, 0), p.nPY - 1) * p.nPX;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    py[m][q] = __ldg(dy + r + cq[q]);
                    px[m][q] = __ldg(dx + r + cq[q]);
                }
            }
        }
        float vy = 0.0f, vx = 0.0f;
#pragma unroll
        for (int m = 0; m < 4; ++m) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float w = fm(wy[m], wx[q]);
                vy = fa(vy, fm(w, py[m][q]));
                vx = fa(vx, fm(w, px[m][q]));
            }
        }
        // Phase B: symmetric half shifts
        float hy = fm(0.5f, vy), hx = fm(0.5f, vx);
        if (p.round_shifts) { hy = roundf(hy); hx = roundf(hx); }
        // Phase C: samples
        const long long o = n * p.img_stride + (long long)i * p.W + j;
        const float fi = (float)i, fj = (float)j;
        if (MODE == 0) {
            p.oa[o] = sample_bicubic<IMPL>(a, fs(fi, hy), fs(fj, hx), p.H, p.W);
            p.ob[o] = sample_bicubic<IMPL>(b, fa(fi, hy), fa(fj, hx), p.H, p.W);
        } else {
            p.oa[o] = sample_lanczos<IMPL>(a, fs(fi, hy), fs(fj, hx), p.H, p.W, p.lut);
            p.ob[o] = sample_lanczos<IMPL>(b, fa(fi, hy), fa(fj, hx), p.H, p.W, p.lut);
        }
    }
}

// Paired (f32x2) warp kernels: the predictor's dy and dx sums run as one f32x2
// chain, and the samples of frame A (.x) and frame B (.y) share every weight,
// gather and combine instruction.  Each half performs the scalar kernel's
// operations in its order, so the output is bit-identical to warp_kernel<MODE, 1>.
// When either stencil touches the border both samples take the scalar routines.
//
// Per-thread column side and per-row predictor of the paired kernels: the
// symmetric half shifts {hy, hx} of output pixel (i, j).
struct PredX2 {
    float2 wxb[4];
    int cq[4];
    float2 pyx[4][4];      // {dy, dx} at the 4x4 predictor stencil
    int cur_by;
};

__device__ __forceinline__ void pred_x2_init(const WarpParams &p, int j, PredX2 &st)
{
    using namespace piv;
    const float fx = p.lx[j], fxf = floorf(fx);
    const int bx = (int)fxf - 1;
    float wx[4];
    keys4(fs(fx, fxf), wx);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        st.wxb[q] = dup2(wx[q]);
        st.cq[q] = min(max(bx + q, 0), p.nPX - 1);
    }
    st.cur_by = -0x7fffffff;
}

__device__ __forceinline__ float2 pred_x2_row(const WarpParams &p, const float *dy, const float *dx, int i,
                                              PredX2 &st, float2 nz)
{
    using namespace piv;
    const int by = p.byr[i];
    const float4 w01 = p.wyb[2 * i], w23 = p.wyb[2 * i + 1];
    const float2 wyb[4] = {make_float2(w01.x, w01.y), make_float2(w01.z, w01.w), make_float2(w23.x, w23.y),
                           make_float2(w23.z, w23.w)};
    if (by != st.cur_by) {          // warp-uniform: all lanes share row i
        st.cur_by = by;
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const int r = min(max(by + m, 0), p.nPY - 1) * p.nPX;
#pragma unroll
            for (int q = 0; q < 4; ++q)
                st.pyx[m][q] = make_float2(__ldg(dy + r + st.cq[q]), __ldg(dx + r + st.cq[q]));
        }
    }
    float2 v = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int q = 0; q < 4; ++q) v = add2(v, mulz2(mulz2(wyb[m], st.wxb[q], nz), st.pyx[m][q], nz));
    float2 h = mulz2(dup2(0.5f), v, nz);     // {hy, hx}
    if (p.round_shifts) { h.x = roundf(h.x); h.y = roundf(h.y); }
    return h;
}

// (96 registers, 5 CTAs per SM; capping them for 6 or 8 spills and ran 5% slower)
__global__ void __launch_bounds__(128) warp_bicubic_x2_kernel(WarpParams p)
{
    using namespace piv;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i0 = (blockIdx.y * blockDim.y + threadIdx.y) * p.rows;
    const int n = blockIdx.z;
    if (j >= p.W || i0 >= p.H) return;
    const float2 nz = dup2(p.neg_zero);
    const float *dy = p.pdy + n * p.pred_stride, *dx = p.pdx + n * p.pred_stride;
    PredX2 st;
    pred_x2_init(p, j, st);
    const float *a = p.ia + n * p.img_stride, *b = p.ib + n * p.img_stride;
    const int H = p.H, W = p.W;
    const float fj = (float)j;
    const int i_end = min(i0 + p.rows, H);
#pragma unroll 1
    for (int i = i0; i < i_end; ++i) {
        const float2 h = pred_x2_row(p, dy, dx, i, st, nz);
        const float fi = (float)i;
        const float2 Y = make_float2(fs(fi, h.x), fa(fi, h.x));     // {frame A, frame B}
        const float2 X = make_float2(fs(fj, h.y), fa(fj, h.y));
        const float2 FY = make_float2(floorf(Y.x), floorf(Y.y)), FX = make_float2(floorf(X.x), floorf(X.y));
        float2 wy2[4], wx2[4];
        keys4_x2(sub2(Y, FY), wy2, nz);
        keys4_x2(sub2(X, FX), wx2, nz);
        const int iya = (int)FY.x - 1, iyb = (int)FY.y - 1, ixa = (int)FX.x - 1, ixb = (int)FX.y - 1;
        const long long o = n * p.img_stride + (long long)i * W + j;
        const bool inside = iya >= 0 && iya + 3 < H && ixa >= 0 && ixa + 3 < W && iyb >= 0 && iyb + 3 < H &&
                            ixb >= 0 && ixb + 3 < W;
        if (inside) {
            const float *ra = a + (iya * W + ixa), *rb = b + (iyb * W + ixb);
            float2 c[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) c[q] = mulz2(make_float2(__ldg(ra + q), __ldg(rb + q)), wy2[0], nz);
#pragma unroll
            for (int m = 1; m < 4; ++m)
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    c[q] = fma2(make_float2(__ldg(ra + m * W + q), __ldg(rb + m * W + q)), wy2[m], c[q]);
            const float2 r = add2(add2(mulz2(c[0], wx2[0], nz), mulz2(c[1], wx2[1], nz)),
                                  add2(mulz2(c[2], wx2[2], nz), mulz2(c[3], wx2[3], nz)));
            p.oa[o] = r.x;
            p.ob[o] = r.y;
        } else {
            const float wya[4] = {wy2[0].x, wy2[1].x, wy2[2].x, wy2[3].x}, wyb_[4] = {wy2[0].y, wy2[1].y, wy2[2].y, wy2[3].y};
            const float wxa[4] = {wx2[0].x, wx2[1].x, wx2[2].x, wx2[3].x}, wxb_[4] = {wx2[0].y, wx2[1].y, wx2[2].y, wx2[3].y};
            p.oa[o] = bicubic_from_weights(a, iya, ixa, wya, wxa, H, W);
            p.ob[o] = bicubic_from_weights(b, iyb, ixb, wyb_, wxb_, H, W);
        }
    }
}

// lanczos_w on two offsets at once (.x frame A, .y frame B): the table lookups
// per frame, the interpolation in paired instructions, each half equal to
// lanczos_w of its offset.
__device__ __forceinline__ void lanczos_w_x2(float2 d, const float4 *lut2, float2 (&w)[6], float2 nz)
{
    using namespace piv;
    const float2 pos = mulz2(d, dup2((float)kLutN), nz);
    int ka = (int)pos.x, kb = (int)pos.y;
    float2 fr = sub2(pos, make_float2((float)ka, (float)kb));
    if (ka >= kLutN) { ka = kLutN - 1; fr.x = 0.0f; }
    if (kb >= kLutN) { kb = kLutN - 1; fr.y = 0.0f; }
    // one 48-byte row per frame holds the twelve table values the interpolation
    // reads (three 16-byte loads instead of twelve 4-byte ones)
    const float4 a0 = __ldg(lut2 + 3 * ka), a1 = __ldg(lut2 + 3 * ka + 1), a2 = __ldg(lut2 + 3 * ka + 2);
    const float4 b0 = __ldg(lut2 + 3 * kb), b1 = __ldg(lut2 + 3 * kb + 1), b2 = __ldg(lut2 + 3 * kb + 2);
    const float2 lo[6] = {make_float2(a0.x, b0.x), make_float2(a0.y, b0.y), make_float2(a0.z, b0.z),
                          make_float2(a0.w, b0.w), make_float2(a1.x, b1.x), make_float2(a1.y, b1.y)};
    const float2 hi[6] = {make_float2(a1.z, b1.z), make_float2(a1.w, b1.w), make_float2(a2.x, b2.x),
                          make_float2(a2.y, b2.y), make_float2(a2.z, b2.z), make_float2(a2.w, b2.w)};
#pragma unroll
    for (int q = 0; q < 6; ++q) w[q] = add2(lo[q], mulz2(fr, sub2(hi[q], lo[q]), nz));
}

// The Lanczos-3 route (interp_mode 1) of the paired kernel: 6 x 6 taps per frame,
// sample_lanczos<1>'s fused row sums, products and combine tree.
__global__ void __launch_bounds__(128) warp_lanczos_x2_kernel(WarpParams p)
{
    using namespace piv;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i0 = (blockIdx.y * blockDim.y + threadIdx.y) * p.rows;
    const int n = blockIdx.z;
    if (j >= p.W || i0 >= p.H) return;
    const float2 nz = dup2(p.neg_zero);
    const float *dy = p.pdy + n * p.pred_stride, *dx = p.pdx + n * p.pred_stride;
    PredX2 st;
    pred_x2_init(p, j, st);
    const float *a = p.ia + n * p.img_stride, *b = p.ib + n * p.img_stride;
    const int H = p.H, W = p.W;
    const float fj = (float)j;
    const int i_end = min(i0 + p.rows, H);
#pragma unroll 1
    for (int i = i0; i < i_end; ++i) {
        const float2 h = pred_x2_row(p, dy, dx, i, st, nz);
        const float fi = (float)i;
        const float2 Y = make_float2(fs(fi, h.x), fa(fi, h.x));     // {frame A, frame B}
        const float2 X = make_float2(fs(fj, h.y), fa(fj, h.y));
        const float2 FY = make_float2(floorf(Y.x), floorf(Y.y)), FX = make_float2(floorf(X.x), floorf(X.y));
        const int iya = (int)FY.x - 2, iyb = (int)FY.y - 2, ixa = (int)FX.x - 2, ixb = (int)FX.y - 2;
        const long long o = n * p.img_stride + (long long)i * W + j;
        const bool inside = iya >= 0 && iya + 5 < H && ixa >= 0 && ixa + 5 < W && iyb >= 0 && iyb + 5 < H &&
                            ixb >= 0 && ixb + 5 < W;
        if (inside) {
            float2 wy2[6], wx2[6];
            lanczos_w_x2(sub2(Y, FY), p.lut2, wy2, nz);
            lanczos_w_x2(sub2(X, FX), p.lut2, wx2, nz);
            const float *ra = a + (iya * W + ixa), *rb = b + (iyb * W + ixb);
            float2 c[6];
#pragma unroll
            for (int q = 0; q < 6; ++q) c[q] = make_float2(0.0f, 0.0f);
#pragma unroll
            for (int m = 0; m < 6; ++m)
#pragma unroll
                for (int q = 0; q < 6; ++q)
                    c[q] = fma2(make_float2(__ldg(ra + m * W + q), __ldg(rb + m * W + q)), wy2[m], c[q]);
            float2 pr[6];
#pragma unroll
            for (int q = 0; q < 6; ++q) pr[q] = mulz2(c[q], wx2[q], nz);
            const float2 r = add2(add2(add2(pr[0], pr[4]), add2(pr[1], pr[5])), add2(pr[2], pr[3]));
            p.oa[o] = r.x;
            p.ob[o] = r.y;
        } else {
            p.oa[o] = sample_lanczos<1>(a, Y.x, X.x, H, W, p.lut);
            p.ob[o] = sample_lanczos<1>(b, Y.y, X.y, H, W, p.lut);
        }
    }
}

std::mutex g_mu;
volatile int g_impl = 1;
// launch settings of the warp kernels (process-wide): rows per thread, block height
std::atomic<int> g_rows{kWarpRows}, g_block_y{4};
struct Ws {
    void *dev = nullptr;
    size_t cap = 0;
    cudaStream_t s = nullptr;
    int ensure(size_t b)
    {
        if (!s && cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return 1;
        if (b > cap) {
            if (dev) cudaFree(dev);
            dev = nullptr;
            cap = 0;
            if (cudaMalloc(&dev, b + b / 4) != cudaSuccess) { cudaGetLastError(); return 1; }
            cap = b + b / 4;
        }
        return 0;
    }
} g_ws_dev[piv::kMaxDevices];
// the current device's staging workspace (nullptr without a usable device)
inline Ws *cur_ws()
{
    const int d = piv::current_device();
    return d < 0 ? nullptr : &g_ws_dev[d];
}

inline size_t pad256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace

// fused_warp.h:21-22
PIV_EXPORT void fused_warp_set_impl(int impl) { g_impl = impl ? 1 : 0; }
PIV_EXPORT int fused_warp_get_impl(void) { return g_impl; }

// Bytes of device tables pivb_warp_dev needs: lut_y [H], lut_x [W], Lanczos
// [4097*6] and its paired rows [4096*12], predictor row weight pairs [H*8],
// predictor stencil rows [H].
PIV_EXPORT size_t pivb_warp_table_bytes(int H, int W)
{
    return pad256((size_t)H * 4) + pad256((size_t)W * 4) + pad256((size_t)(kLutN + 1) * 6 * 4) +
           pad256((size_t)kLutN * 12 * 4) + pad256((size_t)H * 32) + pad256((size_t)H * 4);
}

namespace {
struct WarpTables {
    float *ly, *lx, *lut;
    float4 *lut2;
    float4 *wyb;
    int *byr;
};
WarpTables warp_tables(void *t_, int H, int W)
{
    char *t = static_cast<char *>(t_);
    WarpTables r;
    size_t off = 0;
    r.ly = reinterpret_cast<float *>(t + off); off += pad256((size_t)H * 4);
    r.lx = reinterpret_cast<float *>(t + off); off += pad256((size_t)W * 4);
    r.lut = reinterpret_cast<float *>(t + off); off += pad256((size_t)(kLutN + 1) * 6 * 4);
    r.lut2 = reinterpret_cast<float4 *>(t + off); off += pad256((size_t)kLutN * 12 * 4);
    r.wyb = reinterpret_cast<float4 *>(t + off); off += pad256((size_t)H * 32);
    r.byr = reinterpret_cast<int *>(t + off);
    return r;
}
}  // namespace

// Build the per-call tables on the device (pixel -> predictor index, Lanczos weights).
PIV_EXPORT int pivb_warp_setup_dev(const float *d_ctrs_y, int nPY, const float *d_ctrs_x, int nPX, int H,
                                   int W, void *d_tables, void *stream)
{
    if (H <= 0 || W <= 0 || nPY <= 0 || nPX <= 0 || !d_ctrs_y || !d_ctrs_x || !d_tables) return 1;
    cudaStream_t s = (cudaStream_t)stream;
    const WarpTables t = warp_tables(d_tables, H, W);
    pred_index_kernel<<<(H + 255) / 256, 256, 0, s>>>(d_ctrs_y, nPY, t.ly, H);
    pred_index_kernel<<<(W + 255) / 256, 256, 0, s>>>(d_ctrs_x, nPX, t.lx, W);
    row_weights_kernel<<<(H + 255) / 256, 256, 0, s>>>(t.ly, H, t.wyb, t.byr);
    std::call_once(g_lut_once, build_lut_host);
    if (cudaMemcpyAsync(t.lut, g_lut_host, sizeof(g_lut_host), cudaMemcpyHostToDevice, s) != cudaSuccess) return 1;
    if (cudaMemcpyAsync(t.lut2, g_lut2_host, sizeof(g_lut2_host), cudaMemcpyHostToDevice, s) != cudaSuccess) return 1;
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// Warp N pairs on device pointers.  img_stride = elements between frames (>= H*W);
// tables from pivb_warp_setup_dev.  Frames must hold fewer than 2^31 pixels.
// Returns 0 or 1 (bad arguments / launch failure).
PIV_EXPORT int pivb_warp_dev(const float *d_ia, const float *d_ib, float *d_oa, float *d_ob,
                             const float *d_pdy, const float *d_pdx, int N, int H, int W, int nPY, int nPX,
                             long long img_stride, const void *d_tables, int interp_mode, int shared_predictor,
                             int round_shifts, int impl, void *stream)
{
    if (N <= 0 || H <= 0 || W <= 0 || nPY <= 0 || nPX <= 0) return 1;
    if (!d_ia || !d_ib || !d_oa || !d_ob || !d_pdy || !d_pdx || !d_tables) return 1;
    if ((long long)H * W >= (1LL << 31) - 64 || (long long)nPY * nPX >= (1LL << 31)) return 1;  // 32-bit offsets
    if (img_stride < (long long)H * W) return 1;
    const WarpTables t = warp_tables(const_cast<void *>(d_tables), H, W);
    WarpParams p;
    p.ia = d_ia; p.ib = d_ib; p.oa = d_oa; p.ob = d_ob; p.pdy = d_pdy; p.pdx = d_pdx;
    p.pred_stride = shared_predictor ? 0 : (long long)nPY * nPX;
    p.img_stride = img_stride;
    p.N = N; p.H = H; p.W = W; p.nPY = nPY; p.nPX = nPX;
    p.ly = t.ly; p.lx = t.lx; p.lut = t.lut; p.lut2 = t.lut2; p.wyb = t.wyb; p.byr = t.byr;
    p.round_shifts = round_shifts;
    p.rows = g_rows.load(std::memory_order_relaxed);
    p.neg_zero = -0.0f;
    const int by = g_block_y.load(std::memory_order_relaxed);
    dim3 blk(32, by), grd((W + 31) / 32, (H + by * p.rows - 1) / (by * p.rows), N);   // 32 x 4 x 16 measured best
    cudaStream_t s = (cudaStream_t)stream;
    if (interp_mode == 0) {
        if (impl) warp_bicubic_x2_kernel<<<grd, blk, 0, s>>>(p);
        else warp_kernel<0, 0><<<grd, blk, 0, s>>>(p);
    } else {
        if (impl) warp_lanczos_x2_kernel<<<grd, blk, 0, s>>>(p);
        else warp_kernel<1, 0><<<grd, blk, 0, s>>>(p);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// Launch settings of the warp kernels, for the autotuner (no counterpart in the
// reference): output rows per thread (1..64) and threads per block column
// (1, 2 or 4 rows of 32 threads).  Process-wide; returns 0, or 1 when out of range.
PIV_EXPORT int pivb_warp_set_launch(int rows, int block_y)
{
    if (rows < 1 || rows > 64 || (block_y != 1 && block_y != 2 && block_y != 4)) return 1;
    g_rows.store(rows);
    g_block_y.store(block_y);
    return 0;
}

PIV_EXPORT void pivb_warp_get_launch(int *rows, int *block_y)
{
    if (rows) *rows = g_rows.load();
    if (block_y) *block_y = g_block_y.load();
}

// fused_warp.h:78-93
PIV_EXPORT int fused_symmetric_warp_batch(const float *imgs_a, const float *imgs_b, float *outs_a, float *outs_b,
                                          const float *pred_dy, const float *pred_dx, int N, int H, int W,
                                          int nPY, int nPX, const float *ctrs_y, const float *ctrs_x,
                                          int interp_mode, int shared_predictor, int round_shifts)
{
    if (N <= 0 || H <= 0 || W <= 0 || nPY <= 0 || nPX <= 0) return 1;
    if (!imgs_a || !imgs_b || !outs_a || !outs_b || !pred_dy || !pred_dx || !ctrs_y || !ctrs_x) return 1;
    std::lock_guard<std::mutex> lock(g_mu);
    const int impl = g_impl;
    const size_t img = (size_t)N * H * W;
    const size_t npred = (size_t)(shared_predictor ? 1 : N) * nPY * nPX;
    const size_t tb = pivb_warp_table_bytes(H, W);
    const size_t bytes = 4 * pad256(img * 4) + 2 * pad256(npred * 4) + pad256(nPY * 4) + pad256(nPX * 4) + tb + 4096;
    Ws *wsp = cur_ws();
    if (wsp == nullptr || wsp->ensure(bytes)) return 1;
    cudaStream_t s = wsp->s;
    char *base = static_cast<char *>(wsp->dev);
    size_t off = 0;
    auto take = [&](size_t b) { char *p = base + off; off += pad256(b); return p; };
    float *ia = (float *)take(img * 4), *ib = (float *)take(img * 4);
    float *oa = (float *)take(img * 4), *ob = (float *)take(img * 4);
    float *py = (float *)take(npred * 4), *px = (float *)take(npred * 4);
    float *cy = (float *)take((size_t)nPY * 4), *cx = (float *)take((size_t)nPX * 4);
    void *tables = take(tb);
    if (cudaMemcpyAsync(ia, imgs_a, img * 4, cudaMemcpyHostToDevice, s) != cudaSuccess) return 1;
    if (cudaMemcpyAsync(ib, imgs_b, img * 4, cudaMemcpyHostToDevice, s) != cudaSuccess) return 1;
    if (cudaMemcpyAsync(py, pred_dy, npred * 4, cudaMemcpyHostToDevice, s) != cudaSuccess) return 1;
    if (cudaMemcpyAsync(px, pred_dx, npred * 4, cudaMemcpyHostToDevice, s) != cudaSuccess) return 1;
    if (cudaMemcpyAsync(cy, ctrs_y, (size_t)nPY * 4, cudaMemcpyHostToDevice, s) != cudaSuccess) return 1;
    if (cudaMemcpyAsync(cx, ctrs_x, (size_t)nPX * 4, cudaMemcpyHostToDevice, s) != cudaSuccess) return 1;
    if (pivb_warp_setup_dev(cy, nPY, cx, nPX, H, W, tables, s)) return 1;
    if (pivb_warp_dev(ia, ib, oa, ob, py, px, N, H, W, nPY, nPX, (long long)H * W, tables, interp_mode,
                      shared_predictor, round_shifts, impl, s))
        return 1;
    if (cudaMemcpyAsync(outs_a, oa, img * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess) return 1;
    if (cudaMemcpyAsync(outs_b, ob, img * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess) return 1;
    return cudaStreamSynchronize(s) == cudaSuccess ? 0 : 1;
}

// fused_warp.h:55-64
PIV_EXPORT int fused_symmetric_warp(const float *img_a, const float *img_b, float *out_a, float *out_b,
                                    const float *pred_dy, const float *pred_dx, int H, int W, int nPY, int nPX,
                                    const float *ctrs_y, const float *ctrs_x, int interp_mode, int round_shifts)
{
    return fused_symmetric_warp_batch(img_a, img_b, out_a, out_b, pred_dy, pred_dx, 1, H, W, nPY, nPX, ctrs_y,
                                      ctrs_x, interp_mode, 1, round_shifts);
}
