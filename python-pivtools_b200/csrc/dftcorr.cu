// dftcorr.cu -- libpivb_dft: tensor-core (tcgen05) building blocks and the
// DFT-as-GEMM correlation path for sm_100a.
//
// DFT-as-GEMM correlation of 32 x 32 windows.  Each CTA takes groups of eight
// windows through four chained GEMMs on the tensor core, with the FP32
// accumulators in tensor memory and the CUDA cores doing only the splits,
// transposes and the spectrum product between them:
//
//   stage 1  Y = X W1            rows (window, y), K = x (32): the real row DFT
//                                 to the half spectrum, 16 complex columns, the
//                                 Nyquist column packed into Im of column 0;
//   stage 2  F^T = Y^T W2        rows (window, image, kx), K = (Re, Im) x y (64):
//                                 the complex column DFT;
//            C = F_B conj(F_A)    per element (slot0 = B, slot1 = A as in
//                                 PIV_2d_cross_correlate.c:131-133); row kx = 0
//                                 carries DC and Nyquist together and is unpacked
//                                 by Hermitian symmetry, multiplied, repacked;
//   stage 3  G^T = C^T W3        rows (window, kx), K = (Re, Im) x ky (64): the
//                                 inverse column DFT;
//   stage 4  c = G W4            rows (window, y), K = (Re, Im) x kx (32): the
//                                 Hermitian inverse row DFT to the real plane.
//
// Every operand is split x = hi + lo into two BF16 numbers (hi = bf16(x),
// lo = bf16(x - hi)) and each GEMM accumulates the three products hi*hi +
// hi*lo + lo*hi in FP32, which keeps about 16 significant bits per operand.
// The plane is then scaled by 1/numel, fftshifted into shared memory and goes
// through the same peak search, fit and outputs as the FFT path.
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <cuda_bf16.h>
#include <mutex>

#include "piv_common.cuh"
#include "umma.cuh"
#include "xcorr_kernels.cuh"

namespace {

// One CTA: D (128 x N, FP32) = A (128 x K, BF16) * B (N x K, BF16)^T through
// shared-memory descriptors and a tensor-memory accumulator.  Checks the
// operand layout, the descriptors and the accumulator read-back of the
// correlation kernels on a product with a known answer.
__global__ void __launch_bounds__(128) umma_selftest_kernel(const uint16_t *__restrict__ A,
                                                            const uint16_t *__restrict__ B, float *__restrict__ D,
                                                            int N, int K, int a_mn, uint32_t ncols, int *status)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    unsigned char *sA = sm;
    unsigned char *sB = sm + 128 * K * 2;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sB + N * K * 2);
    uint32_t *slot = reinterpret_cast<uint32_t *>(bar + 1);
    const int t = threadIdx.x, warp = t >> 5;
    for (int e = t; e < 128 * K; e += 128)
        *reinterpret_cast<uint16_t *>(sA + (a_mn ? umma::mnmajor_offset(128, e / K, e % K)
                                                 : umma::kmajor_offset(128, e / K, e % K))) = A[e];
    for (int e = t; e < N * K; e += 128)
        *reinterpret_cast<uint16_t *>(sB + umma::kmajor_offset(N, e / K, e % K)) = B[e];
    if (t == 0) umma::mbar_init(bar, 1);
    if (warp == 0) umma::tmem_alloc(slot, ncols);
    umma::fence_smem_to_async();
    umma::fence_before();
    __syncthreads();
    umma::fence_after();
    const uint32_t tbase = *slot;
    if (t == 0) {
        const uint32_t id = umma::idesc_bf16(128, N, a_mn != 0);
        for (int s = 0; s < K / 16; ++s)
            umma::mma_bf16(tbase, umma::desc_tile(umma::smem_u32(sA), 128, s),
                           umma::desc_tile(umma::smem_u32(sB), N, s), id, s > 0 ? 1u : 0u);
        umma::commit(umma::smem_u32(bar));
    }
    const bool ok = umma::mbar_wait(umma::smem_u32(bar), 0);
    umma::fence_after();
    if (ok) {
        for (int c0 = 0; c0 < N; c0 += 32) {
            float v[32];
            umma::tmem_ld32(tbase + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, v);
#pragma unroll
            for (int j = 0; j < 32; ++j)
                if (c0 + j < N) D[(32 * warp + (t & 31)) * N + c0 + j] = v[j];
        }
    } else if ((t & 31) == 0) {
        atomicExch(status, 1);
    }
    umma::fence_before();
    __syncthreads();
    if (warp == 0) umma::tmem_free(tbase, ncols);
}

// The failure path of the bounded waits: allocate tensor memory, wait on an
// mbarrier phase that nothing completes (no MMA is issued, nothing arrives) with a
// short poll limit, record the timeout in *status, free the tensor memory and
// return.  The correlation kernels take the same path if an MMA completion is
// ever not observed.
__global__ void __launch_bounds__(128) wait_timeout_kernel(int *status, uint32_t limit)
{
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t slot;
    const int t = threadIdx.x, warp = t >> 5;
    if (t == 0) umma::mbar_init(&bar, 1);
    if (warp == 0) umma::tmem_alloc(&slot, 32);
    umma::fence_before();
    __syncthreads();
    umma::fence_after();
    const uint32_t tbase = slot;
    const bool ok = umma::mbar_wait(umma::smem_u32(&bar), 0, limit);
    if (!ok && (t & 31) == 0) atomicAdd(status, 1);
    umma::fence_before();
    __syncthreads();
    if (warp == 0) umma::tmem_free(tbase, 32);
}

// ---------------------------------------------------------------------------
// DFT-as-GEMM correlation, 32 x 32 windows
// ---------------------------------------------------------------------------
namespace dft32 {

using namespace piv;

constexpr int N = 32;
constexpr int G = 8;                      // windows per group
// constant operands (K-major, hi then lo), byte offsets in the constant block
constexpr uint32_t B1 = 0, B1_BYTES = 32 * 32 * 2;
constexpr uint32_t B2 = B1 + 2 * B1_BYTES, B2_BYTES = 64 * 64 * 2;
constexpr uint32_t B3 = B2 + 2 * B2_BYTES, B3_BYTES = 64 * 64 * 2;
constexpr uint32_t B4 = B3 + 2 * B3_BYTES, B4_BYTES = 32 * 32 * 2;
constexpr uint32_t CONST_BYTES = B4 + 2 * B4_BYTES;          // 40 KB
constexpr uint32_t WORK_BYTES = 64 * 1024;
constexpr uint32_t PLANE_LD = WinGeo<N>::STF;   // the search reads with this stride
constexpr uint32_t SMEM_BYTES = CONST_BYTES + WORK_BYTES + 64;
constexpr uint32_t TMEM_COLS = 256;
static_assert(G * N * PLANE_LD * 4 <= WORK_BYTES, "planes alias the work region");

// Split 8 values into hi = bf16(x) and lo = bf16(x - hi) and store each half
// as one 16-byte vector (paired conversions: cvt.rn.bf16x2 per two values).
__device__ __forceinline__ void store8(unsigned char *hi_dst, unsigned char *lo_dst, const float *v)
{
    uint32_t H[4], L[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
        const float2 hf = __bfloat1622float2(h);
        const __nv_bfloat162 l = __floats2bfloat162_rn(v[2 * j] - hf.x, v[2 * j + 1] - hf.y);
        H[j] = *reinterpret_cast<const uint32_t *>(&h);
        L[j] = *reinterpret_cast<const uint32_t *>(&l);
    }
    *reinterpret_cast<uint4 *>(hi_dst) = make_uint4(H[0], H[1], H[2], H[3]);
    *reinterpret_cast<uint4 *>(lo_dst) = make_uint4(L[0], L[1], L[2], L[3]);
}

// One three-product GEMM: D (128 x n) (+)= A (128 x K) B (n x K)^T, K = 16*ksteps.
__device__ __forceinline__ void gemm3(uint32_t d, uint32_t a_hi, uint32_t a_lo, uint32_t b_hi, uint32_t b_lo,
                                      uint32_t n, int ksteps, bool a_mn)
{
    const uint32_t id = umma::idesc_bf16(128, n, a_mn);
    for (int s = 0; s < ksteps; ++s) {
        const uint64_t ah = umma::desc_tile(a_hi, 128, s), al = umma::desc_tile(a_lo, 128, s);
        const uint64_t bh = umma::desc_tile(b_hi, n, s), bl = umma::desc_tile(b_lo, n, s);
        umma::mma_bf16(d, ah, bh, id, s > 0 ? 1u : 0u);
        umma::mma_bf16(d, ah, bl, id, 1u);
        umma::mma_bf16(d, al, bh, id, 1u);
    }
}

__device__ __forceinline__ void cta_sync_for_mma()
{
    umma::fence_smem_to_async();
    umma::fence_before();
    __syncthreads();
    umma::fence_after();
}

struct WinInfo {
    long long idx;
    int n, iw;
    float enorm;
    int flags;     // 1 valid, 2 in range
};

// Two warpgroups: warp w (w = 4 wg + q) owns tensor-memory lanes 32 q .. 32 q + 31
// like warp q of the other group; the groups split each stage's columns (the
// two images, the two halves of ky or y, the two plane tiles) and each warp
// gathers, searches and fits one window of the eight.
constexpr int THREADS = 256;
constexpr uint32_t XCHG = 48 * 1024;      // kx = 0 exchange area inside the work region

__global__ void __launch_bounds__(THREADS, 2) kernel(XcorrParams prm, const uint4 *__restrict__ consts, int *status)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ WinInfo info[G];
    unsigned char *cst = sm;
    unsigned char *wk = sm + CONST_BYTES;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + CONST_BYTES + WORK_BYTES);
    uint32_t *slot = reinterpret_cast<uint32_t *>(bar + 1);
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int wg = warp >> 2, wq = warp & 3;

    for (int i = t; i < (int)(CONST_BYTES / 16); i += THREADS) reinterpret_cast<uint4 *>(cst)[i] = consts[i];
    if (t == 0) umma::mbar_init(bar, 1);
    if (warp == 0) umma::tmem_alloc(slot, TMEM_COLS);
    cta_sync_for_mma();
    const uint32_t tm = *slot;
    const uint32_t lane_base = tm + ((uint32_t)(32 * wq) << 16);
    const uint32_t cst_a = umma::smem_u32(cst), wk_a = umma::smem_u32(wk), bar_a = umma::smem_u32(bar);
    uint32_t phase = 0;
    bool ok = true;
    const long long nwt = (long long)prm.nwy * prm.nwx;
    const long long ngroups = (prm.total + G - 1) / G;
    const float inv_numel = 1.0f / (float)(N * N);
    float *xchg = reinterpret_cast<float *>(wk + XCHG);   // [wg][wq][2 rows][4][16]

    for (long long grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
        // ---- stage 0: gather, weight, mean, energy (PIV_2d_cross_correlate.c:299-353).
        //      Warp w takes window w; lane = column x, so every load instruction reads
        //      one 128-byte image row segment.
        {
            const int wl = warp;
            const long long idx = grp * G + wl;
            const bool inrange = idx < prm.total;
            bool valid = inrange;
            int n = 0, iw = 0, r0 = 0, c0 = 0;
            if (inrange) {
                n = (int)(idx / nwt);
                iw = (int)(idx - (long long)n * nwt);
                const int ii = iw % prm.nwx, jj = iw / prm.nwx;
                if (prm.mask && prm.mask[iw] == 1.0f) valid = false;
                r0 = (int)floor((double)prm.ctr_y[jj] - ((double)N - 1.0) / 2.0 + 0.5);
                c0 = (int)floor((double)prm.ctr_x[ii] - ((double)N - 1.0) / 2.0 + 0.5);
                if (r0 < 0 || c0 < 0 || r0 + N > prm.H || c0 + N > prm.W) valid = false;
            }
            float a[N], b[N];
            float sa = 0.0f, sb = 0.0f;
            if (valid) {
                const float *fa = prm.A + (long long)n * prm.img_stride + (long long)r0 * prm.W + c0 + lane;
                const float *fb = prm.B + (long long)n * prm.img_stride + (long long)r0 * prm.W + c0 + lane;
#pragma unroll
                for (int y = 0; y < N; ++y) {
                    a[y] = __ldg(fa + y * prm.W) * __ldg(prm.wA + y * N + lane);
                    b[y] = __ldg(fb + y * prm.W) * __ldg(prm.wB + y * N + lane);
                    sa += a[y];
                    sb += b[y];
                }
            } else {
#pragma unroll
                for (int y = 0; y < N; ++y) { a[y] = 0.0f; b[y] = 0.0f; }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                sa += __shfl_xor_sync(0xffffffffu, sa, o);
                sb += __shfl_xor_sync(0xffffffffu, sb, o);
            }
            const float ma = sa / (float)(N * N), mb = sb / (float)(N * N);
            float ea = 0.0f, eb = 0.0f;
#pragma unroll
            for (int y = 0; y < N; ++y) {
                if (valid && !prm.ensemble) { a[y] -= ma; b[y] -= mb; }
                ea += a[y] * a[y];
                eb += b[y] * b[y];
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                ea += __shfl_xor_sync(0xffffffffu, ea, o);
                eb += __shfl_xor_sync(0xffffffffu, eb, o);
            }
            if (lane == 0) {
                info[wl].idx = idx;
                info[wl].n = n;
                info[wl].iw = iw;
                info[wl].enorm = 1.0f / sqrtf(ea * eb);
                info[wl].flags = (valid ? 1 : 0) | (inrange ? 2 : 0);
            }
            // A1 tiles (MN-major, 8 KB hi + 8 KB lo each): tile wg (image A) and 2 + wg
            // (image B) hold windows 4 wg .. 4 wg + 3; row (window % 4) * 32 + y, K = x
            unsigned char *ta = wk + wg * 16384, *tb = wk + (2 + wg) * 16384;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const uint32_t off = umma::mnmajor_offset(128, wq * 32 + 8 * q, lane);
                store8(ta + off, ta + 8192 + off, a + 8 * q);
                store8(tb + off, tb + 8192 + off, b + 8 * q);
            }
        }
        cta_sync_for_mma();
        // ---- stage 1: four tiles, N = 32, K = 32
        if (t == 0) {
            for (int tt = 0; tt < 4; ++tt)
                gemm3(tm + 32 * tt, wk_a + tt * 16384, wk_a + tt * 16384 + 8192, cst_a + B1, cst_a + B1 + B1_BYTES,
                      32, 2, true);
            umma::commit(bar_a);
        }
        ok &= umma::mbar_wait(bar_a, phase);
        phase ^= 1u;
        umma::fence_after();
        // ---- Y -> A2 (MN-major; image i: 16 KB hi + 16 KB lo at 32 KB * i).  Row
        //      (window, kx) = wglob * 16 + kx; K: Re at y, Im at 32 + y.  Group wg
        //      takes tiles wg (image A) and 2 + wg (image B): its own windows.
#pragma unroll 1
        for (int img = 0; img < 2; ++img) {
            const int tt = 2 * img + wg;
            float v[32];
            umma::tmem_ld32(lane_base + 32 * tt, v);
            const int wglob = wg * 4 + wq;
            unsigned char *hi = wk + img * 32768, *lo = hi + 16384;
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                const uint32_t o_re = umma::mnmajor_offset(128, wglob * 16 + half * 8, lane);
                const uint32_t o_im = umma::mnmajor_offset(128, wglob * 16 + half * 8, 32 + lane);
                store8(hi + o_re, lo + o_re, v + half * 8);
                store8(hi + o_im, lo + o_im, v + 16 + half * 8);
            }
        }
        cta_sync_for_mma();
        // ---- stage 2: images A, B; N = 64, K = 64; D at columns 128 (A) and 192 (B)
        if (t == 0) {
            for (int img = 0; img < 2; ++img)
                gemm3(tm + 128 + 64 * img, wk_a + img * 32768, wk_a + img * 32768 + 16384, cst_a + B2,
                      cst_a + B2 + B2_BYTES, 64, 4, true);
            umma::commit(bar_a);
        }
        ok &= umma::mbar_wait(bar_a, phase);
        phase ^= 1u;
        umma::fence_after();
        // ---- spectrum product -> A3 (K-major, 16 KB hi + 16 KB lo); row r = (window, kx);
        //      group wg takes ky in [16 wg, 16 wg + 16)
        {
            const int k0 = 16 * wg;
            float ar[16], ai[16], br[16], bi[16];
            umma::tmem_ld16(lane_base + 128 + k0, ar);
            umma::tmem_ld16(lane_base + 160 + k0, ai);
            umma::tmem_ld16(lane_base + 192 + k0, br);
            umma::tmem_ld16(lane_base + 224 + k0, bi);
            const int kx = lane & 15;
            // rows kx = 0 (lanes 0, 16) need F(-ky), held by the other group: exchange
            float *mine = xchg + ((wg * 4 + wq) * 2 + (lane >> 4)) * 64;
            if (kx == 0) {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    mine[j] = ar[j]; mine[16 + j] = ai[j]; mine[32 + j] = br[j]; mine[48 + j] = bi[j];
                }
            }
            __syncthreads();
            float cr[16], ci[16];
            if (kx != 0) {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    cr[j] = br[j] * ar[j] + bi[j] * ai[j];
                    ci[j] = bi[j] * ar[j] - br[j] * ai[j];
                }
            } else {
                // P = F(., 0) + i F(., 16); F0 = (P + conj P(-ky)) / 2, F16 = (P - conj P(-ky)) / 2i
                const float *other = xchg + (((wg ^ 1) * 4 + wq) * 2 + (lane >> 4)) * 64;
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int ky = k0 + j, m = (32 - ky) & 31;
                    // F(m) lives with this group when m is in [k0, k0 + 16), else with the other
                    const bool own = (m >> 4) == wg;
                    const int jm = m & 15;
                    const float amr = own ? ar[jm] : other[jm], ami = own ? ai[jm] : other[16 + jm];
                    const float bmr = own ? br[jm] : other[32 + jm], bmi = own ? bi[jm] : other[48 + jm];
                    const float a0r = 0.5f * (ar[j] + amr), a0i = 0.5f * (ai[j] - ami);
                    const float a1r = 0.5f * (ai[j] + ami), a1i = -0.5f * (ar[j] - amr);
                    const float b0r = 0.5f * (br[j] + bmr), b0i = 0.5f * (bi[j] - bmi);
                    const float b1r = 0.5f * (bi[j] + bmi), b1i = -0.5f * (br[j] - bmr);
                    const float c0r = b0r * a0r + b0i * a0i, c0i = b0i * a0r - b0r * a0i;
                    const float c1r = b1r * a1r + b1i * a1i, c1i = b1i * a1r - b1r * a1i;
                    cr[j] = c0r - c1i;        // Q = C0 + i C16
                    ci[j] = c0i + c1r;
                }
            }
            const uint32_t r = (uint32_t)(wq * 32 + lane);
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const uint32_t o_re = umma::kmajor_offset(128, r, k0 + 8 * c);
                const uint32_t o_im = umma::kmajor_offset(128, r, 32 + k0 + 8 * c);
                store8(wk + o_re, wk + 16384 + o_re, cr + 8 * c);
                store8(wk + o_im, wk + 16384 + o_im, ci + 8 * c);
            }
        }
        cta_sync_for_mma();
        // ---- stage 3: N = 64, K = 64, D at column 0
        if (t == 0) {
            gemm3(tm, wk_a, wk_a + 16384, cst_a + B3, cst_a + B3 + B3_BYTES, 64, 4, false);
            umma::commit(bar_a);
        }
        ok &= umma::mbar_wait(bar_a, phase);
        phase ^= 1u;
        umma::fence_after();
        // ---- G -> A4 (MN-major; tile t4 = window / 4: 8 KB hi + 8 KB lo at 16 KB * t4).
        //      Row (window % 4) * 32 + y; K: Re at kx, Im at 16 + kx.  Group wg takes
        //      y in [16 wg, 16 wg + 16).
        {
            const int y0 = 16 * wg;
            float gre[16], gim[16];
            umma::tmem_ld16(lane_base + y0, gre);
            umma::tmem_ld16(lane_base + 32 + y0, gim);
            const int r = wq * 32 + lane, wglob = r >> 4, kx = r & 15;
            unsigned char *hi = wk + (wglob >> 2) * 16384, *lo = hi + 8192;
            const int rb = (wglob & 3) * 32 + y0;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const uint32_t o_re = umma::mnmajor_offset(128, rb + 8 * q, kx);
                const uint32_t o_im = umma::mnmajor_offset(128, rb + 8 * q, 16 + kx);
                store8(hi + o_re, lo + o_re, gre + 8 * q);
                store8(hi + o_im, lo + o_im, gim + 8 * q);
            }
        }
        cta_sync_for_mma();
        // ---- stage 4: two tiles, N = 32, K = 32, D at columns 64 and 96
        if (t == 0) {
            for (int t4 = 0; t4 < 2; ++t4)
                gemm3(tm + 64 + 32 * t4, wk_a + t4 * 16384, wk_a + t4 * 16384 + 8192, cst_a + B4,
                      cst_a + B4 + B4_BYTES, 32, 2, true);
            umma::commit(bar_a);
        }
        ok &= umma::mbar_wait(bar_a, phase);
        phase ^= 1u;
        umma::fence_after();
        // ---- plane of this warp's window: scale, fftshift into shared memory (aliases
        //      the work region; tile wg holds windows 4 wg .. 4 wg + 3)
        float *planes = reinterpret_cast<float *>(wk);
        {
            float c[32];
            umma::tmem_ld32(lane_base + 64 + 32 * wg, c);
            umma::fence_before();
            __syncthreads();              // every group has finished reading the work region
            float *pl = planes + warp * (N * PLANE_LD);
            const int row = (lane + N / 2) & (N - 1);
#pragma unroll
            for (int x = 0; x < N; ++x) pl[row * PLANE_LD + ((x + N / 2) & (N - 1))] = c[x] * inv_numel;
        }
        __syncwarp();
        // ---- search and finish, warp per window (the FFT path's code): with
        //      record scratch the warp writes its window's record line at once,
        //      otherwise its lane 0 fits in place
        {
            const int wl = warp;
            float *pl = planes + wl * (N * PLANE_LD);
            const WinInfo wi = info[wl];
            if (prm.planes && (wi.flags & 1)) {
                float *dst = prm.planes + wi.idx * (long long)(N * N);
                for (int k = lane; k < N * N; k += 32) dst[k] = pl[(k / N) * PLANE_LD + (k % N)];
            }
            const Group<N> g{lane, nullptr};
            PeakAcc acc;
            bool has_nan;
            search_plane<N>(g, pl, acc, has_nan);
            if (wi.flags & 2) {
                if (prm.lm)
                    finish_window_rec<N>(lane, 32, prm, pl, PLANE_LD, acc, has_nan, wi.idx, wi.n, wi.iw, nwt,
                                         (wi.flags & 1) != 0, wi.enorm);
                else if (lane == 0)
                    finish_window<N, false>(prm, pl, PLANE_LD, acc, has_nan, wi.idx, wi.n, wi.iw, nwt,
                                            (wi.flags & 1) != 0, wi.enorm);
            }
        }
        __syncthreads();
    }
    if (!ok && lane == 0) atomicExch(status, 1);
    umma::fence_before();
    __syncthreads();
    if (warp == 0) umma::tmem_free(tm, TMEM_COLS);
}

// ---- constant operands, built on the host in double precision and split to BF16
inline uint16_t bf16_rn(float f)
{
    uint32_t u;
    memcpy(&u, &f, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}
inline float bf16_f(uint16_t h)
{
    uint32_t u = (uint32_t)h << 16;
    float f;
    memcpy(&f, &u, 4);
    return f;
}

// K-major hi/lo images of a rows x K matrix given by coef(j, k).
template <class F>
void put(unsigned char *base, uint32_t off, uint32_t bytes, int rows, int K, F coef)
{
    for (int j = 0; j < rows; ++j)
        for (int k = 0; k < K; ++k) {
            const double v = coef(j, k);
            const uint16_t h = bf16_rn((float)v);
            const uint16_t l = bf16_rn((float)(v - (double)bf16_f(h)));
            const uint32_t o = umma::kmajor_offset((uint32_t)rows, (uint32_t)j, (uint32_t)k);
            memcpy(base + off + o, &h, 2);
            memcpy(base + off + bytes + o, &l, 2);
        }
}

void build_consts(unsigned char *c)
{
    const double tp = 2.0 * M_PI / N;
    // W1: row j -> Re Y(j) (j < 16), Y(16) (j = 16), Im Y(j - 16) (j > 16); K = x
    put(c, B1, B1_BYTES, 32, 32, [&](int j, int x) {
        if (j < 16) return cos(tp * j * x);
        if (j == 16) return (x & 1) ? -1.0 : 1.0;
        return -sin(tp * (j - 16) * x);
    });
    // W2: row j -> Re F(ky = j) (j < 32), Im F(ky = j - 32); K: Re Y(y = k) (k < 32), Im Y(y = k - 32)
    put(c, B2, B2_BYTES, 64, 64, [&](int j, int k) {
        const int ky = j & 31, y = k & 31;
        const double cs = cos(tp * ky * y), sn = sin(tp * ky * y);
        if (j < 32) return k < 32 ? cs : sn;
        return k < 32 ? -sn : cs;
    });
    // W3: row j -> Re G(y = j) (j < 32), Im G(y = j - 32); K: Re C(ky = k) (k < 32), Im C(ky = k - 32)
    put(c, B3, B3_BYTES, 64, 64, [&](int j, int k) {
        const int y = j & 31, ky = k & 31;
        const double cs = cos(tp * ky * y), sn = sin(tp * ky * y);
        if (j < 32) return k < 32 ? cs : -sn;
        return k < 32 ? sn : cs;
    });
    // W4: row x -> c(x); K: Re G(kx = k) (k < 16), Im G(kx = k - 16); kx = 0 carries G(0) and G(16)
    put(c, B4, B4_BYTES, 32, 32, [&](int x, int k) {
        const int kx = k & 15;
        if (k < 16) return kx == 0 ? 1.0 : 2.0 * cos(tp * kx * x);
        return kx == 0 ? ((x & 1) ? -1.0 : 1.0) : -2.0 * sin(tp * kx * x);
    });
}

std::mutex g_mu;
void *g_consts[64] = {};

const uint4 *consts_for_current_device()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_consts[dev]) {
        static unsigned char host[CONST_BYTES];
        memset(host, 0, sizeof(host));
        build_consts(host);
        void *d = nullptr;
        if (cudaMalloc(&d, CONST_BYTES) != cudaSuccess) return nullptr;
        if (cudaMemcpy(d, host, CONST_BYTES, cudaMemcpyHostToDevice) != cudaSuccess) {
            cudaFree(d);
            return nullptr;
        }
        if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES) != cudaSuccess) {
            cudaFree(d);
            return nullptr;
        }
        g_consts[dev] = d;
    }
    return static_cast<const uint4 *>(g_consts[dev]);
}

}  // namespace dft32

// ---------------------------------------------------------------------------
// DFT-as-GEMM correlation, 64 x 64 windows
// ---------------------------------------------------------------------------
// One CTA per SM (512 threads, 16 warps; 225 KB of shared memory) takes groups
// of four windows through the same four GEMMs as the 32 px chain, sized for
// n = 64:
//
//   stage 1  Y = X W1          per image, rows (window, y) in two 128-row tiles,
//                              K = x (64), N = 64: Re Y(kx) for kx < 32, the
//                              Nyquist column Y(32) in the slot of Im Y(0),
//                              Im Y(kx) for kx > 32;
//   stage 2  F^T = Y^T W2      per image, rows (window, kx) (4 x 32), K = (Re, Im)
//                              x y (128), N = (Re, Im) x ky (128);
//            C = F_B conj(F_A) per element, row kx = 0 (DC and Nyquist packed)
//                              unpacked by Hermitian symmetry and repacked;
//   stage 3  conj(G)^T = conj(C)^T W2   the inverse column DFT as the forward DFT
//                              of the conjugate (so W2 serves both directions);
//   stage 4  c = G W4          rows (window, y) in two tiles, K = (Re, Im) x kx
//                              (64), N = x (64): the Hermitian inverse row DFT.
//
// Tensor memory: 256 columns, reused by every stage.  Shared memory: the three
// constant operands (96 KB, hi + lo) and two 64 KB work buffers, which hold in
// turn the stage-1 operands of images A and B, the stage-2 operands of A and B,
// the conjugate spectrum product (buffer 0) with the kx = 0 exchange (buffer 1),
// the stage-4 operand (buffer 1) and finally the four fftshifted float planes
// (row stride 65, across both buffers).
namespace dft64 {

using namespace piv;

constexpr int N = 64;
constexpr int G = 4;                      // windows per group
constexpr int THREADS = 512;
constexpr uint32_t C1 = 0, C1_BYTES = 64 * 64 * 2;
constexpr uint32_t C2 = C1 + 2 * C1_BYTES, C2_BYTES = 128 * 128 * 2;
constexpr uint32_t C4 = C2 + 2 * C2_BYTES, C4_BYTES = 64 * 64 * 2;
constexpr uint32_t CONST_BYTES = C4 + 2 * C4_BYTES;         // 96 KB
constexpr uint32_t BUF = 64 * 1024;
constexpr uint32_t WORK_BYTES = 2 * BUF;
constexpr int PLANE_LD = WinGeo<N>::STF;                    // 65
constexpr uint32_t MISC_BYTES = 1024;
constexpr uint32_t SMEM_BYTES = CONST_BYTES + WORK_BYTES + MISC_BYTES;
constexpr uint32_t TMEM_COLS = 256;
static_assert(G * N * PLANE_LD * 4 <= WORK_BYTES, "planes alias the work buffers");
static_assert(G * N * 4 * 4 + G * N * 2 * 4 <= BUF, "kx = 0 exchange fits buffer 1");
static_assert(SMEM_BYTES <= 232448, "one CTA per SM");

struct WinInfo {
    long long idx;
    int n, iw;
    float enorm;
    int flags;     // 1 valid, 2 in range
};

// Pull the rows of the next group's windows into L2 while this group is on the
// tensor core: thread t takes row t % 64 of image (t / 64) % 2 of window t / 128
// (its 256 bytes span two or three 128-byte lines).  Windows the gather skips
// (out of range, masked, outside the frame) are not touched.
__device__ __forceinline__ void prefetch_group(const XcorrParams &prm, long long grp, long long nwt, int t)
{
    const long long idx = grp * G + (t >> 7);
    if (idx >= prm.total) return;
    const int n = (int)(idx / nwt);
    const int iw = (int)(idx - (long long)n * nwt);
    const int ii = iw % prm.nwx, jj = iw / prm.nwx;
    if (prm.mask && prm.mask[iw] == 1.0f) return;
    const int r0 = (int)floor((double)prm.ctr_y[jj] - ((double)N - 1.0) / 2.0 + 0.5);
    const int c0 = (int)floor((double)prm.ctr_x[ii] - ((double)N - 1.0) / 2.0 + 0.5);
    if (r0 < 0 || c0 < 0 || r0 + N > prm.H || c0 + N > prm.W) return;
    const float *img = ((t >> 6) & 1) ? prm.B : prm.A;
    const char *row = reinterpret_cast<const char *>(img + (long long)n * prm.img_stride +
                                                     (long long)(r0 + (t & 63)) * prm.W + c0);
    asm volatile("prefetch.global.L2 [%0];" ::"l"(row));
    asm volatile("prefetch.global.L2 [%0];" ::"l"(row + 128));
    asm volatile("prefetch.global.L2 [%0];" ::"l"(row + 4 * N - 4));
}

// One candidate strip per thread of the window's 128 (rows and columns [16, 48)
// of the shifted plane, strips of 8 rows; the rolled 3x3 test of search_plane),
// then the warp's reduction; the caller merges the window's four warps.
__device__ __forceinline__ void search_strip(const float *pl, int t, PeakAcc &acc, bool &nan)
{
    constexpr int H2 = N / 2, Q = N / 4, S = 8;
    acc.init();
    nan = false;
    const int j = Q + t % H2, r0 = Q + (t / H2) * S;
    const float *c0 = pl + (r0 - 1) * PLANE_LD + j;
    float m0 = 0.0f, m1 = 0.0f, c1 = 0.0f;
#pragma unroll
    for (int k = 0; k < S + 2; ++k) {
        const float l = c0[k * PLANE_LD - 1], c = c0[k * PLANE_LD], r = c0[k * PLANE_LD + 1];
        nan |= (l != l) | (c != c) | (r != r);
        const float m2 = fmaxf(l, fmaxf(c, r));
        if (k >= 2) {
            const float v = c1;
            const bool mx = v >= fmaxf(m0, fmaxf(m1, m2));
            acc.add((mx && v > 0.0f) ? v : -1.0f, (r0 + k - 2) * N + j);
        }
        m0 = m1;
        m1 = m2;
        c1 = c;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float ob = __shfl_xor_sync(0xffffffffu, acc.best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, acc.idx, o);
        const float o1 = __shfl_xor_sync(0xffffffffu, acc.p1, o);
        const float o2 = __shfl_xor_sync(0xffffffffu, acc.p2, o);
        acc.merge(ob, oi, o1, o2);
    }
    nan = __any_sync(0xffffffffu, nan);
}

__global__ void __launch_bounds__(THREADS, 1) kernel(XcorrParams prm, const uint4 *__restrict__ consts, int *status)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ WinInfo info[G];
    unsigned char *cst = sm;
    unsigned char *buf0 = sm + CONST_BYTES, *buf1 = buf0 + BUF;
    float *misc = reinterpret_cast<float *>(sm + CONST_BYTES + WORK_BYTES);
    float *red = misc;                                     // [G][4 warps][4]
    int *nanred = reinterpret_cast<int *>(misc + 64);      // [G][4]
    uint64_t *bar = reinterpret_cast<uint64_t *>(misc + 96);
    uint32_t *slot = reinterpret_cast<uint32_t *>(bar + 1);
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int wg = warp >> 2, wq = warp & 3;
    const long long nwt = (long long)prm.nwy * prm.nwx;
    const long long ngroups = (prm.total + G - 1) / G;
    if (blockIdx.x < ngroups) prefetch_group(prm, blockIdx.x, nwt, t);
    for (int i = t; i < (int)(CONST_BYTES / 16); i += THREADS) reinterpret_cast<uint4 *>(cst)[i] = consts[i];
    if (t == 0) umma::mbar_init(bar, 1);
    if (warp == 0) umma::tmem_alloc(slot, TMEM_COLS);
    dft32::cta_sync_for_mma();
    const uint32_t tm = *slot;
    const uint32_t lane_base = tm + ((uint32_t)(32 * wq) << 16);
    const uint32_t cst_a = umma::smem_u32(cst), b0_a = umma::smem_u32(buf0), b1_a = umma::smem_u32(buf1);
    const uint32_t bar_a = umma::smem_u32(bar);
    uint32_t phase = 0;
    bool ok = true;
    const float inv_numel = 1.0f / (float)(N * N);

    // Wait for the stage's MMAs; every thread learns whether any wait ran out.
    auto wait_stage = [&]() -> bool {
        const bool mine = umma::mbar_wait(bar_a, phase);
        phase ^= 1u;
        umma::fence_after();
        return __syncthreads_and(mine ? 1 : 0) != 0;
    };

    for (long long grp = blockIdx.x; grp < ngroups && ok; grp += gridDim.x) {
        // ---- stage 0: gather, weight, mean, energy (PIV_2d_cross_correlate.c:299-353).
        //      Warp (wq, wg) takes rows 16 wq .. 16 wq + 15 of window wg; lane = columns
        //      lane and lane + 32.
        {
            const int wl = wg, rb = wq;
            const long long idx = grp * G + wl;
            const bool inrange = idx < prm.total;
            bool valid = inrange;
            int n = 0, iw = 0, r0 = 0, c0 = 0;
            if (inrange) {
                n = (int)(idx / nwt);
                iw = (int)(idx - (long long)n * nwt);
                const int ii = iw % prm.nwx, jj = iw / prm.nwx;
                if (prm.mask && prm.mask[iw] == 1.0f) valid = false;
                r0 = (int)floor((double)prm.ctr_y[jj] - ((double)N - 1.0) / 2.0 + 0.5);
                c0 = (int)floor((double)prm.ctr_x[ii] - ((double)N - 1.0) / 2.0 + 0.5);
                if (r0 < 0 || c0 < 0 || r0 + N > prm.H || c0 + N > prm.W) valid = false;
            }
            float a0[16], a1[16], b0[16], b1[16];
            float sa = 0.0f, sb = 0.0f;
            if (valid) {
                const long long base = (long long)n * prm.img_stride + (long long)(r0 + 16 * rb) * prm.W + c0 + lane;
                const float *fa = prm.A + base, *fb = prm.B + base;
                const float *wa = prm.wA + 16 * rb * N + lane, *wb = prm.wB + 16 * rb * N + lane;
#pragma unroll
                for (int y = 0; y < 16; ++y) {
                    a0[y] = __ldg(fa + y * prm.W) * __ldg(wa + y * N);
                    a1[y] = __ldg(fa + y * prm.W + 32) * __ldg(wa + y * N + 32);
                    b0[y] = __ldg(fb + y * prm.W) * __ldg(wb + y * N);
                    b1[y] = __ldg(fb + y * prm.W + 32) * __ldg(wb + y * N + 32);
                    sa += a0[y] + a1[y];
                    sb += b0[y] + b1[y];
                }
            } else {
#pragma unroll
                for (int y = 0; y < 16; ++y) { a0[y] = 0.0f; a1[y] = 0.0f; b0[y] = 0.0f; b1[y] = 0.0f; }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                sa += __shfl_xor_sync(0xffffffffu, sa, o);
                sb += __shfl_xor_sync(0xffffffffu, sb, o);
            }
            if (lane == 0) { red[(wl * 4 + rb) * 4 + 0] = sa; red[(wl * 4 + rb) * 4 + 1] = sb; }
            __syncthreads();
            const float *rw = red + wl * 16;
            const float ma = (((rw[0] + rw[4]) + rw[8]) + rw[12]) / (float)(N * N);
            const float mb = (((rw[1] + rw[5]) + rw[9]) + rw[13]) / (float)(N * N);
            float ea = 0.0f, eb = 0.0f;
#pragma unroll
            for (int y = 0; y < 16; ++y) {
                if (valid && !prm.ensemble) { a0[y] -= ma; a1[y] -= ma; b0[y] -= mb; b1[y] -= mb; }
                ea += a0[y] * a0[y] + a1[y] * a1[y];
                eb += b0[y] * b0[y] + b1[y] * b1[y];
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                ea += __shfl_xor_sync(0xffffffffu, ea, o);
                eb += __shfl_xor_sync(0xffffffffu, eb, o);
            }
            if (lane == 0) { red[(wl * 4 + rb) * 4 + 2] = ea; red[(wl * 4 + rb) * 4 + 3] = eb; }
            __syncthreads();
            if (t == wl * 128) {          // lane 0 of warp (0, wl)
                const float eA = ((rw[2] + rw[6]) + rw[10]) + rw[14];
                const float eB = ((rw[3] + rw[7]) + rw[11]) + rw[15];
                info[wl].idx = idx;
                info[wl].n = n;
                info[wl].iw = iw;
                info[wl].enorm = 1.0f / sqrtf(eA * eB);
                info[wl].flags = (valid ? 1 : 0) | (inrange ? 2 : 0);
            }
            // A1 tiles (MN-major, 16 KB hi + 16 KB lo): image A in buffer 0, B in buffer 1;
            // tile m = window / 2 at 32 KB * m; row (window % 2) * 64 + y, K = x
            const int m = wl >> 1;
            unsigned char *ta = buf0 + m * 32768, *tb = buf1 + m * 32768;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const uint32_t row = (uint32_t)((wl & 1) * 64 + 16 * rb + 8 * q);
                const uint32_t o0 = umma::mnmajor_offset(128, row, lane);
                const uint32_t o1 = umma::mnmajor_offset(128, row, 32 + lane);
                dft32::store8(ta + o0, ta + 16384 + o0, a0 + 8 * q);
                dft32::store8(ta + o1, ta + 16384 + o1, a1 + 8 * q);
                dft32::store8(tb + o0, tb + 16384 + o0, b0 + 8 * q);
                dft32::store8(tb + o1, tb + 16384 + o1, b1 + 8 * q);
            }
        }
        dft32::cta_sync_for_mma();
        // ---- stage 1: tiles (image, m) -> tensor-memory columns 64 (2 image + m)
        if (t == 0) {
            for (int img = 0; img < 2; ++img)
                for (int m = 0; m < 2; ++m) {
                    const uint32_t a = (img ? b1_a : b0_a) + m * 32768;
                    dft32::gemm3(tm + 64 * (2 * img + m), a, a + 16384, cst_a + C1, cst_a + C1 + C1_BYTES, 64, 4,
                                 true);
                }
            umma::commit(bar_a);
        }
        if (grp + gridDim.x < ngroups) prefetch_group(prm, grp + gridDim.x, nwt, t);
        if (!(ok = wait_stage())) break;
        // ---- Y -> A2 (MN-major, 32 KB hi + 32 KB lo per image, in that image's buffer).
        //      Row (window, kx) = window * 32 + kx; K: Re at y, Im at 64 + y.  Warp
        //      (wq, wg) reads tile wg: lane 32 wq + lane = (window % 2) * 64 + y.
        {
            const int tt = wg, img = tt >> 1, m = tt & 1;
            const int wl = 2 * m + (wq >> 1), y = (wq & 1) * 32 + lane;
            float v[32];
            unsigned char *dst = img ? buf1 : buf0;
#pragma unroll 1
            for (int h = 0; h < 2; ++h) {       // h = 0: Re Y(kx), h = 1: Im Y(kx) (Y(32) at kx = 0)
                umma::tmem_ld32(lane_base + 64 * tt + 32 * h, v);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const uint32_t o = umma::mnmajor_offset(128, (uint32_t)(wl * 32 + 8 * q), (uint32_t)(64 * h + y));
                    dft32::store8(dst + o, dst + 32768 + o, v + 8 * q);
                }
            }
        }
        dft32::cta_sync_for_mma();
        // ---- stage 2: images A, B; N = 128, K = 128; D at columns 0 (A) and 128 (B)
        if (t == 0) {
            dft32::gemm3(tm, b0_a, b0_a + 32768, cst_a + C2, cst_a + C2 + C2_BYTES, 128, 8, true);
            dft32::gemm3(tm + 128, b1_a, b1_a + 32768, cst_a + C2, cst_a + C2 + C2_BYTES, 128, 8, true);
            umma::commit(bar_a);
        }
        if (!(ok = wait_stage())) break;
        // ---- spectrum product -> conj(C) as A3 (K-major, 32 KB hi + 32 KB lo, buffer 0);
        //      lane 32 wq + lane = (window wq, kx = lane); warp group wg takes ky in
        //      [16 wg, 16 wg + 16).  Rows kx = 0 (lane 0) need F(-ky): exchanged
        //      through buffer 1.
        {
            const int k0 = 16 * wg;
            float ar[16], ai[16], br[16], bi[16];
            umma::tmem_ld16(lane_base + k0, ar);
            umma::tmem_ld16(lane_base + 64 + k0, ai);
            umma::tmem_ld16(lane_base + 128 + k0, br);
            umma::tmem_ld16(lane_base + 192 + k0, bi);
            float *xchg = reinterpret_cast<float *>(buf1) + wq * (N * 4);    // [ky][ar, ai, br, bi]
            if (lane == 0) {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    float *e = xchg + (k0 + j) * 4;
                    e[0] = ar[j]; e[1] = ai[j]; e[2] = br[j]; e[3] = bi[j];
                }
            }
            __syncthreads();
            // row kx = 0: lanes 0..15 of the warp unpack one ky each of its ky range
            // (P = F(., 0) + i F(., 32); F0 = (P + conj P(-ky)) / 2,
            // F32 = (P - conj P(-ky)) / 2i), multiply and repack Q = C0 + i C32
            float *q0 = reinterpret_cast<float *>(buf1) + G * N * 4 + wq * (N * 2);   // [ky][Re, Im]
            if (lane < 16) {
                const int ky = k0 + lane, mk = (N - ky) & (N - 1);
                const float *e = xchg + ky * 4, *m = xchg + mk * 4;
                const float a0r = 0.5f * (e[0] + m[0]), a0i = 0.5f * (e[1] - m[1]);
                const float a1r = 0.5f * (e[1] + m[1]), a1i = -0.5f * (e[0] - m[0]);
                const float b0r = 0.5f * (e[2] + m[2]), b0i = 0.5f * (e[3] - m[3]);
                const float b1r = 0.5f * (e[3] + m[3]), b1i = -0.5f * (e[2] - m[2]);
                const float c0r = b0r * a0r + b0i * a0i, c0i = b0i * a0r - b0r * a0i;
                const float c1r = b1r * a1r + b1i * a1i, c1i = b1i * a1r - b1r * a1i;
                q0[ky * 2] = c0r - c1i;
                q0[ky * 2 + 1] = c0i + c1r;
            }
            __syncwarp();
            // conj(C) = conj(F_B conj(F_A)) in place: ar <- Re C, ai <- -Im C
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const float cre = br[j] * ar[j] + bi[j] * ai[j];
                const float cim = bi[j] * ar[j] - br[j] * ai[j];
                ar[j] = cre;
                ai[j] = -cim;
            }
            if (lane == 0) {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    ar[j] = q0[(k0 + j) * 2];
                    ai[j] = -q0[(k0 + j) * 2 + 1];
                }
            }
            float *cr = ar, *ci = ai;
            const uint32_t r = (uint32_t)(wq * 32 + lane);
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const uint32_t o_re = umma::kmajor_offset(128, r, (uint32_t)(k0 + 8 * c));
                const uint32_t o_im = umma::kmajor_offset(128, r, (uint32_t)(64 + k0 + 8 * c));
                dft32::store8(buf0 + o_re, buf0 + 32768 + o_re, cr + 8 * c);
                dft32::store8(buf0 + o_im, buf0 + 32768 + o_im, ci + 8 * c);
            }
        }
        dft32::cta_sync_for_mma();
        // ---- stage 3: N = 128, K = 128, D = conj(G) at column 0
        if (t == 0) {
            dft32::gemm3(tm, b0_a, b0_a + 32768, cst_a + C2, cst_a + C2 + C2_BYTES, 128, 8, false);
            umma::commit(bar_a);
        }
        if (!(ok = wait_stage())) break;
        // ---- G -> A4 (MN-major, buffer 1; tile m = window / 2: 16 KB hi + 16 KB lo at
        //      32 KB * m).  Row (window % 2) * 64 + y; K: Re at kx, Im at 32 + kx.
        //      Lane 32 wq + lane = (window wq, kx = lane); warp group wg takes y in
        //      [16 wg, 16 wg + 16).
        {
            const int y0 = 16 * wg, wl = wq, kx = lane;
            float gre[16], gim[16];
            umma::tmem_ld16(lane_base + y0, gre);
            umma::tmem_ld16(lane_base + 64 + y0, gim);
#pragma unroll
            for (int j = 0; j < 16; ++j) gim[j] = -gim[j];        // G = conj(D)
            unsigned char *tile = buf1 + (wl >> 1) * 32768;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const uint32_t row = (uint32_t)((wl & 1) * 64 + y0 + 8 * q);
                const uint32_t o_re = umma::mnmajor_offset(128, row, (uint32_t)kx);
                const uint32_t o_im = umma::mnmajor_offset(128, row, (uint32_t)(32 + kx));
                dft32::store8(tile + o_re, tile + 16384 + o_re, gre + 8 * q);
                dft32::store8(tile + o_im, tile + 16384 + o_im, gim + 8 * q);
            }
        }
        dft32::cta_sync_for_mma();
        // ---- stage 4: two tiles, N = 64, K = 64, D at columns 0 and 64
        if (t == 0) {
            for (int m = 0; m < 2; ++m)
                dft32::gemm3(tm + 64 * m, b1_a + m * 32768, b1_a + m * 32768 + 16384, cst_a + C4,
                             cst_a + C4 + C4_BYTES, 64, 4, true);
            umma::commit(bar_a);
        }
        if (!(ok = wait_stage())) break;
        // ---- planes: scale, fftshift into shared memory (across both buffers, whose
        //      operands the finished MMAs no longer read).  Warp (wq, wg): tile wg & 1,
        //      columns 32 (wg >> 1) .. +31; lane 32 wq + lane = (window % 2) * 64 + y.
        float *planes = reinterpret_cast<float *>(buf0);
        {
            const int m = wg & 1, h = wg >> 1;
            const int wl = 2 * m + (wq >> 1), y = (wq & 1) * 32 + lane;
            float c[32];
            umma::tmem_ld32(lane_base + 64 * m + 32 * h, c);
            float *pl = planes + wl * (N * PLANE_LD) + ((y + N / 2) & (N - 1)) * PLANE_LD;
#pragma unroll
            for (int j = 0; j < 32; ++j) pl[(32 * h + j + N / 2) & (N - 1)] = c[j] * inv_numel;
        }
        __syncthreads();
        // ---- search (window wg, warps wq = 0..3 one candidate strip per thread), merge,
        //      then the FFT path's finish: with record scratch warp (0, wg) writes the
        //      window's record line, otherwise its lane 0 fits in place
        {
            const int wl = wg;
            const float *pl = planes + wl * (N * PLANE_LD);
            const WinInfo wi = info[wl];
            if (prm.planes && (wi.flags & 1)) {
                float *dst = prm.planes + wi.idx * (long long)(N * N);
                for (int k = wq * 32 + lane; k < N * N; k += 128) dst[k] = pl[(k / N) * PLANE_LD + (k % N)];
            }
            PeakAcc acc;
            bool nan;
            search_strip(pl, wq * 32 + lane, acc, nan);
            if (lane == 0) {
                float *e = red + (wl * 4 + wq) * 4;
                e[0] = acc.best; e[1] = __int_as_float(acc.idx); e[2] = acc.p1; e[3] = acc.p2;
                nanred[wl * 4 + wq] = nan ? 1 : 0;
            }
            __syncthreads();
            if (wq == 0) {
                acc.init();
                bool has_nan = false;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const float *e = red + (wl * 4 + k) * 4;
                    acc.merge(e[0], __float_as_int(e[1]), e[2], e[3]);
                    has_nan |= nanred[wl * 4 + k] != 0;
                }
                if (wi.flags & 2) {
                    if (prm.lm)
                        finish_window_rec<N>(lane, 32, prm, const_cast<float *>(pl), PLANE_LD, acc, has_nan, wi.idx,
                                             wi.n, wi.iw, nwt, (wi.flags & 1) != 0, wi.enorm);
                    else if (lane == 0)
                        finish_window<N, false>(prm, const_cast<float *>(pl), PLANE_LD, acc, has_nan, wi.idx, wi.n,
                                                wi.iw, nwt, (wi.flags & 1) != 0, wi.enorm);
                }
            }
        }
        __syncthreads();
    }
    if (!ok) {
        // a completion was not observed: record it, give the MMAs in flight a
        // bounded time to finish before the tensor memory is released
        if (t == 0) atomicExch(status, 1);
        umma::mbar_wait(bar_a, phase ^ 1u);
    }
    umma::fence_before();
    __syncthreads();
    if (warp == 0) umma::tmem_free(tm, TMEM_COLS);
}

// ---- constant operands, built on the host in double precision and split to BF16
void build_consts(unsigned char *c)
{
    const double tp = 2.0 * M_PI / N;
    // W1: row j -> Re Y(j) (j < 32), Y(32) (j = 32), Im Y(j - 32) (j > 32); K = x
    dft32::put(c, C1, C1_BYTES, 64, 64, [&](int j, int x) {
        if (j < 32) return cos(tp * j * x);
        if (j == 32) return (x & 1) ? -1.0 : 1.0;
        return -sin(tp * (j - 32) * x);
    });
    // W2: row j -> Re F(ky = j) (j < 64), Im F(ky = j - 64); K: Re Y(y = k) (k < 64), Im Y(y = k - 64)
    dft32::put(c, C2, C2_BYTES, 128, 128, [&](int j, int k) {
        const int ky = j & 63, y = k & 63;
        const double cs = cos(tp * ky * y), sn = sin(tp * ky * y);
        if (j < 64) return k < 64 ? cs : sn;
        return k < 64 ? -sn : cs;
    });
    // W4: row x -> c(x); K: Re G(kx = k) (k < 32), Im G(kx = k - 32); kx = 0 carries G(0) and G(32)
    dft32::put(c, C4, C4_BYTES, 64, 64, [&](int x, int k) {
        const int kx = k & 31;
        if (k < 32) return kx == 0 ? 1.0 : 2.0 * cos(tp * kx * x);
        return kx == 0 ? ((x & 1) ? -1.0 : 1.0) : -2.0 * sin(tp * kx * x);
    });
}

std::mutex g_mu;
void *g_consts[64] = {};

const uint4 *consts_for_current_device()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_consts[dev]) {
        static unsigned char host[CONST_BYTES];
        memset(host, 0, sizeof(host));
        build_consts(host);
        void *d = nullptr;
        if (cudaMalloc(&d, CONST_BYTES) != cudaSuccess) return nullptr;
        if (cudaMemcpy(d, host, CONST_BYTES, cudaMemcpyHostToDevice) != cudaSuccess) {
            cudaFree(d);
            return nullptr;
        }
        if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES) != cudaSuccess) {
            cudaFree(d);
            return nullptr;
        }
        g_consts[dev] = d;
    }
    return static_cast<const uint4 *>(g_consts[dev]);
}

}  // namespace dft64

}  // namespace

// Self-test of the tensor-core path: D (128 x N) = A (128 x K) B (N x K)^T with
// BF16 operands (raw 16-bit patterns, row-major) and FP32 results.  K in
// {16, 32, 48, 64}, N a multiple of 16 in [16, 128]; a_mn stages A in the
// MN-major layout instead of K-major.  *d_status is set to 1 if
// the MMA completion was not observed within the wait limit.  Returns 0, or 1
// for bad arguments / launch failure.
PIV_EXPORT int pivb_umma_selftest(const void *d_A, const void *d_B, float *d_D, int N, int K, int a_mn,
                                  int *d_status, void *stream)
{
    if (!d_A || !d_B || !d_D || !d_status) return 1;
    if (K < 16 || K > 64 || K % 16) return 1;
    if (N < 16 || N > 128 || N % 16) return 1;
    const uint32_t ncols = N <= 32 ? 32u : (N <= 64 ? 64u : 128u);
    // operands take 128*K*2 + N*K*2 <= 32 KB; the allocation is sized so that every
    // address a descriptor of these tiles can form stays inside it
    const int smem = 96 * 1024;
    if (cudaFuncSetAttribute(umma_selftest_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
        return 1;
    umma_selftest_kernel<<<1, 128, smem, (cudaStream_t)stream>>>(static_cast<const uint16_t *>(d_A),
                                                                  static_cast<const uint16_t *>(d_B), d_D, N, K,
                                                                  a_mn, ncols, d_status);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// Exercise the timeout path of the bounded mbarrier wait: each of the 4 warps of
// one CTA adds 1 to *d_status when its wait (limit polls) runs out.  Returns 0, or
// 1 for bad arguments / launch failure.
PIV_EXPORT int pivb_wait_timeout_selftest(int *d_status, int limit, void *stream)
{
    if (!d_status || limit <= 0) return 1;
    wait_timeout_kernel<<<1, 128, 0, (cudaStream_t)stream>>>(d_status, (uint32_t)limit);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// Instantaneous correlation of 32 x 32 windows on the tensor core (DFT-as-GEMM,
// split BF16, FP32 accumulation).  Arguments as pivb_xcorr_dev; supported:
// win 32 x 32, ensemble 0, n_peaks 1, peak finders 3-6 (4-6 need the LM scratch
// of pivb_xcorr_scratch_bytes).  *d_status (device int) is set to 1 if an MMA
// completion was not observed.  The first call on a device builds the constant
// DFT operands (a synchronous upload): make it before any stream capture.
PIV_EXPORT int pivb_dft_xcorr_dev(const float *d_A, const float *d_B, long long img_stride, const float *d_mask,
                                  int H, int W, int n_images, const float *d_ctr_x, const float *d_ctr_y,
                                  int n_win_y, int n_win_x, const float *d_wA, const float *d_wB, const float *d_cw,
                                  int win_h, int win_w, int ensemble, int n_peaks, int peak_finder,
                                  int peakfit_impl, float *d_pk_x, float *d_pk_y, float *d_pk_h, float *d_sx,
                                  float *d_sy, float *d_sxy, float *d_pk_ratio, float *d_planes, void *d_scratch,
                                  size_t scratch_bytes, int *d_status, void *stream)
{
    using namespace piv;
    const int nw = win_h;
    if (win_h != win_w || (nw != 32 && nw != 64)) return PIV_ERROR_NOPLAN;
    if (ensemble || n_peaks != 1 || peak_finder < 3 || peak_finder > 6 || n_images < 0 || !d_status)
        return PIV_ERROR_OUT_OF_BOUNDS;
    const long long total = (long long)n_images * n_win_y * n_win_x;
    if (total == 0) return PIV_ERROR_NONE;
    const bool lm = peak_finder >= 4;
    if (lm && (d_scratch == nullptr || scratch_bytes < (size_t)total * sizeof(LmRecord))) return PIV_ERROR_NOMEM;
    // with record scratch the 3-point fits also run in the thread-per-window record kernel
    const bool defer = lm || (d_scratch != nullptr && scratch_bytes >= (size_t)total * sizeof(LmRecord));
    const uint4 *consts = nw == 32 ? dft32::consts_for_current_device() : dft64::consts_for_current_device();
    if (!consts) return PIV_ERROR_CUDA;
    cudaStream_t s = (cudaStream_t)stream;
    XcorrParams p{};
    p.A = d_A; p.B = d_B; p.img_stride = img_stride; p.mask = d_mask;
    p.H = H; p.W = W; p.n_img = n_images;
    p.ctr_x = d_ctr_x; p.ctr_y = d_ctr_y; p.nwy = n_win_y; p.nwx = n_win_x;
    p.wA = d_wA; p.wB = d_wB; p.cw = d_cw;
    p.ensemble = 0; p.n_peaks = 1; p.finder = peak_finder;
    p.pk_x = d_pk_x; p.pk_y = d_pk_y; p.pk_h = d_pk_h; p.sx = d_sx; p.sy = d_sy; p.sxy = d_sxy;
    p.pk_ratio = d_pk_ratio; p.planes = d_planes;
    p.lm = defer ? static_cast<LmRecord *>(d_scratch) : nullptr;
    p.total = total;
    p.neg_zero = -0.0f;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (nw == 32) {
        const long long groups = (total + dft32::G - 1) / dft32::G;
        const int grid = (int)(groups < 2LL * sms ? groups : 2LL * sms);
        dft32::kernel<<<grid, dft32::THREADS, dft32::SMEM_BYTES, s>>>(p, consts, d_status);
    } else {
        const long long groups = (total + dft64::G - 1) / dft64::G;
        const int grid = (int)(groups < (long long)sms ? groups : (long long)sms);
        dft64::kernel<<<grid, dft64::THREADS, dft64::SMEM_BYTES, s>>>(p, consts, d_status);
    }
    if (cudaGetLastError() != cudaSuccess) return PIV_ERROR_CUDA;
    if (defer) {
        const unsigned blocks = (unsigned)((total + 127) / 128);
        if (peakfit_impl) lm_records_kernel<1><<<blocks, 128, 0, s>>>(p, nw);
        else lm_records_kernel<0><<<blocks, 128, 0, s>>>(p, nw);
        if (cudaGetLastError() != cudaSuccess) return PIV_ERROR_CUDA;
    }
    return PIV_ERROR_NONE;
}
