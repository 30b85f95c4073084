// passglue.cu -- libpivb_pass: the work between multipass passes, on the GPU.
//
// The reference runs these steps in Python between its C calls
// (pivtools_cli/piv/piv_backend/cpu_instantaneous.py:559-870, :1040-1071):
//   validate  -- large-displacement gate, add the window-grid predictor, peak
//                magnitude and normalised-median outlier tests
//                (outlier_detection.py:56-84, :87-243);
//   infill    -- least-squares inpainting of invalid vectors: minimise the
//                squared first (harmonic) or second (biharmonic) differences in
//                physical units over the invalid cells with the valid cells held
//                fixed (infilling.py:150-283, 336-421), solved exactly (FP64
//                conjugate gradients on the normal equations);
//   pad       -- edge-replicate padding onto the padded predictor grid
//                (cpu_instantaneous.py:836-853) and the separable Gaussian
//                smoothing of scipy.ndimage.gaussian_filter(mode='nearest')
//                (cpu_instantaneous.py:1040-1048, :1140-1152);
//   remap     -- the padded predictor at the next pass's window centres exactly
//                as cv2.remap(INTER_CUBIC, BORDER_REPLICATE) computes it: 1/32-px
//                fixed-point coordinates, Keys a = -0.75 coefficient table
//                (cpu_instantaneous.py:1050-1071).
// The device has no libraries here: each step is a plain CUDA kernel over the
// small vector grids, one launch per step for the whole batch of pairs.
#include <math.h>

#include <algorithm>

#include "piv_common.cuh"

namespace {

__device__ __forceinline__ float qnanf() { return __int_as_float(0x7fc00000); }

// Median of the finite values among v[0..24) (np.nanmedian convention; NaN if
// none).  Register bitonic sort of 32 keys with NaN and padding mapped to +inf,
// then a select of the middle order statistics: no local memory.
__device__ __forceinline__ float median24(const float (&v)[24])
{
    float k[32];
    int m = 0;
#pragma unroll
    for (int i = 0; i < 24; ++i) {
        const bool fin = v[i] == v[i];
        k[i] = fin ? v[i] : INFINITY;
        m += fin;
    }
#pragma unroll
    for (int i = 24; i < 32; ++i) k[i] = INFINITY;
#pragma unroll
    for (int size = 2; size <= 32; size <<= 1)
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1)
#pragma unroll
            for (int i = 0; i < 32; ++i) {
                const int j = i ^ stride;
                if (j > i) {
                    const bool up = (i & size) == 0;
                    const float a = k[i], b = k[j];
                    k[i] = up ? fminf(a, b) : fmaxf(a, b);
                    k[j] = up ? fmaxf(a, b) : fminf(a, b);
                }
            }
    if (m == 0) return qnanf();
    const int hi = m / 2, lo = (m - 1) / 2;
    float vh = 0.0f, vl = 0.0f;
#pragma unroll
    for (int i = 0; i < 24; ++i) {
        vh = (i == hi) ? k[i] : vh;
        vl = (i == lo) ? k[i] : vl;
    }
    return (m & 1) ? vh : 0.5f * (vl + vh);
}

struct ValParams {
    const float *pk_x, *pk_y, *pk_h;      // (N, ny, nx), primary peak
    const float *pred_dy, *pred_dx;       // (N, ny, nx) window-grid predictor, or null
    const float *mask;                    // (ny, nx) 1 = masked, or null
    int N, ny, nx;
    float thresh_x, thresh_y;             // large-displacement gate
    float peak_thr;                       // peak-magnitude threshold (<0 disables)
    float med_eps, med_thr;               // normalised median (med_thr <= 0 disables)
    int med_size;
    float *ux, *uy;                       // out: displacement, NaN where invalid, 0 at masked
    unsigned char *invalid;               // out: 1 where the vector must be infilled
    signed char *reason;                  // out (nullable): why the vector is invalid (codes below)
    long long pk_stride;                  // elements between the images' peak arrays (ny*nx for one peak)
    int hnan_late;                        // 1: a NaN peak height invalidates only at the end of the
                                          //    secondary-peak stage (not in the primary tests)
    int med_on;                           // 1: run the normalised-median test in median_kernel
    const unsigned char *extra;           // (N, ny, nx) outlier flags of further tests, or null
};

// Invalid-vector reason codes (pivtools_cli/piv/piv_backend/nan_reason_codes.py:18-25).
// The first stage that claims a vector keeps it; masked windows always read -1.
enum : signed char {
    kMasked = -1, kValid = 0, kFitFail = 1, kLargeDisp = 6, kUnclassified = 9, kOutlier = 10,
    kSecondaryOutlier = 12, kPeakMagNaN = 13
};

// Stage 1: gate + predictor.  ux/uy receive the gated field (NaN where the
// correlation failed or the displacement gate fired, 0 at masked windows);
// invalid additionally marks peak-magnitude failures and NaN peak heights
// (cpu_instantaneous.py:589-631, :728-732).  With the median test off the
// invalid vectors are NaN-ed and their reasons completed here, otherwise by
// median_kernel.
__global__ void gate_kernel(ValParams p, int apply)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nv = (long long)p.N * p.ny * p.nx;
    if (i >= nv) return;
    const long long plane = (long long)p.ny * p.nx;
    const int w = (int)(i % plane);
    const long long src = (i / plane) * p.pk_stride + w;
    const bool masked = p.mask && p.mask[w] != 0.0f;
    float x = p.pk_x[src], y = p.pk_y[src], h = p.pk_h[src];
    const bool fit_fail = (x != x) || (y != y);
    const bool large = fabsf(x) > p.thresh_x || fabsf(y) > p.thresh_y;   // false for NaN
    if (masked || large) { x = qnanf(); y = qnanf(); h = qnanf(); }
    if (p.pred_dx) { x += p.pred_dx[i]; y += p.pred_dy[i]; }
    const bool pk_fail = p.peak_thr >= 0.0f && ((h < p.peak_thr) || (h != h));
    bool bad = (x != x) || (y != y) || pk_fail || (!p.hnan_late && h != h);
    bad = bad && !masked;
    if (apply && bad) { x = qnanf(); y = qnanf(); }
    p.ux[i] = masked ? 0.0f : x;
    p.uy[i] = masked ? 0.0f : y;
    p.invalid[i] = bad ? 1 : 0;
    if (p.reason) {
        signed char rc = masked ? kMasked : fit_fail ? kFitFail : large ? kLargeDisp : kValid;
        if (rc == kValid && pk_fail) rc = kOutlier;
        if (apply && rc == kValid && bad) rc = (h != h) ? kPeakMagNaN : kUnclassified;
        p.reason[i] = rc;
    }
}

// Stage 2: normalised-median test (outlier_detection.py:87-243) on the gated
// field gx/gy (vector-norm residual over the size x size neighbourhood without
// the node, 3x3 presence guard), OR-ed with the stage-1 flags; invalid vectors
// become NaN.  As in the reference, vectors that failed before the test enter it
// as zeros, masked windows drop out of the medians and count as present.
__global__ void median_kernel(ValParams p, const float *gx, const float *gy)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nv = (long long)p.N * p.ny * p.nx;
    if (i >= nv) return;
    const int plane = p.ny * p.nx;
    const int n = (int)(i / plane), w = (int)(i % plane), r = w / p.nx, c = w % p.nx;
    const bool masked = p.mask && p.mask[w] != 0.0f;
    if (masked) return;
    const float *X = gx + (long long)n * plane, *Y = gy + (long long)n * plane;
    bool outlier = false;
    if (p.med_on) {
        const int h = p.med_size / 2;
        float nu[24], nvv[24];
        int present = 0;
#pragma unroll
        for (int t = 0; t < 25; ++t) {
            const int dr = t / 5 - 2, dc = t % 5 - 2;
            const int rr = r + dr, cc = c + dc;
            const bool inside = rr >= 0 && rr < p.ny && cc >= 0 && cc < p.nx && abs(dr) <= h && abs(dc) <= h;
            float a = qnanf(), b = qnanf();
            if (inside) {
                const bool mk = p.mask && p.mask[rr * p.nx + cc] != 0.0f;
                if (!mk) {
                    a = X[rr * p.nx + cc];
                    b = Y[rr * p.nx + cc];
                    // the reference zeroes failed vectors before its outlier tests
                    // (cpu_instantaneous.py:627-629): they enter as 0, and are present
                    if (a != a || b != b) { a = 0.0f; b = 0.0f; }
                }
                if (abs(dr) <= 1 && abs(dc) <= 1) ++present;     // finite or masked
            }
            if (t == 12) continue;
            nu[t < 12 ? t : t - 1] = a;
            nvv[t < 12 ? t : t - 1] = b;
        }
        const float mu = median24(nu), mv = median24(nvv);
        float u0 = X[w], v0 = Y[w];
        if (u0 != u0 || v0 != v0) { u0 = 0.0f; v0 = 0.0f; }
        const float r0 = sqrtf((u0 - mu) * (u0 - mu) + (v0 - mv) * (v0 - mv));
        float ri[24];
#pragma unroll
        for (int j = 0; j < 24; ++j)
            ri[j] = sqrtf((nu[j] - mu) * (nu[j] - mu) + (nvv[j] - mv) * (nvv[j] - mv));
        const float rm = median24(ri);
        const float nr = r0 / (rm + p.med_eps);
        outlier = (nr > p.med_thr) || !isfinite(nr) || present < 6;
    }
    if (p.extra && p.extra[i]) outlier = true;
    const bool bad = p.invalid[i] || outlier;
    p.invalid[i] = bad ? 1 : 0;
    p.ux[i] = bad ? qnanf() : X[w];
    p.uy[i] = bad ? qnanf() : Y[w];
    if (p.reason) {
        signed char rc = p.reason[i];
        if (rc == kValid && outlier) rc = kOutlier;
        if (rc == kValid && bad) {
            const float hr = p.pk_h[(long long)n * p.pk_stride + w];
            rc = (hr != hr) ? kPeakMagNaN : kUnclassified;
        }
        p.reason[i] = rc;
    }
}

// Least-squares infilling (infilling.py:150-283, _fill_least_squares): minimise
// the sum of squared finite differences of order 1 (harmonic; stencil -1, 1) or
// 2 (biharmonic; 1, -2, 1) along y and x, each difference divided by pitch^order,
// over the fill cells with every known cell held at its value.  Only difference
// rows that touch a fill cell enter; rows touching an excluded cell (a masked
// window, or a non-finite value outside the fill set) are dropped, which gives
// the frame edge's natural boundary condition there.  The normal equations
// A x = b (A = Lf^T Lf, b = -Lf^T Lk u_k) are solved matrix-free in FP64 by
// conjugate gradients to a relative residual `tol`, both components at once.
//
// One CTA per pair.  The fill cells are listed in grid order (each warp scans a
// contiguous segment, ballot-compacts, and a block prefix over the warps places
// the segments), threads own fixed list entries, and every dot product is a
// fixed-order block reduction: results are bit-reproducible run to run.  A
// group of fill cells that no row links to a known cell has b = 0 there and
// stays at 0 (the reference raises for such a field; a pass on the GPU cannot
// stop, so a pair without any valid vector comes out as zeros).
constexpr int kLsqThreads = 512;
constexpr int kLsqWarps = kLsqThreads / 32;

struct LsqParams {
    float *ux, *uy;                  // (N, ny, nx), in place
    const unsigned char *invalid;    // (N, ny, nx) 1 = fill
    const float *mask;               // (ny, nx) 1 = excluded, or null
    int ny, nx, order, max_iter;
    double w2y, w2x;                 // 1 / pitch^(2 order)
    double tol2;                     // squared relative residual
    char *work;                      // per pair: work_stride bytes
    size_t work_stride;
};

__device__ __forceinline__ double2 lsq_block_sum2(double a, double b, double2 *red)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[warp] = make_double2(a, b);
    __syncthreads();
    double2 t = make_double2(0.0, 0.0);
#pragma unroll
    for (int k = 0; k < kLsqWarps; ++k) {
        t.x += red[k].x;
        t.y += red[k].y;
    }
    __syncthreads();
    return t;
}

// Sum over the kept rows through fill cell (r, c) of coef(cell) * row value,
// scaled by w^2: with `known` false the row value is sum coef * V (V zero off
// the fill set: this is (A V)_cell), with `known` true it is the known cells'
// part sum coef * u (giving -b_cell).
template <int ORDER>
__device__ __forceinline__ void lsq_rows(const unsigned char *cls, int r, int c, int ny, int nx, double w2y,
                                         double w2x, const double *V0, const double *V1, const float *U0,
                                         const float *U1, bool known, double &o0, double &o1)
{
    constexpr double coef[3] = {ORDER == 1 ? -1.0 : 1.0, ORDER == 1 ? 1.0 : -2.0, 1.0};
    double a0 = 0.0, a1 = 0.0;
#pragma unroll
    for (int axis = 0; axis < 2; ++axis) {
        const int pos = axis == 0 ? r : c, len = axis == 0 ? ny : nx;
        const int step = axis == 0 ? nx : 1;
        const int cell = r * nx + c;
        double s0 = 0.0, s1 = 0.0;
#pragma unroll
        for (int j = 0; j <= ORDER; ++j) {
            const int st = pos - j;                       // first node of the row
            if (st < 0 || st + ORDER >= len) continue;
            const int q0 = cell - j * step;
            bool kept = true;
            double v0 = 0.0, v1 = 0.0;
#pragma unroll
            for (int t = 0; t <= ORDER; ++t) {
                const int q = q0 + t * step;
                const unsigned char k = cls[q];
                kept = kept && k != 2;
                if (known) {
                    if (k == 0) {
                        v0 += coef[t] * (double)U0[q];
                        v1 += coef[t] * (double)U1[q];
                    }
                } else {
                    v0 += coef[t] * V0[q];
                    v1 += coef[t] * V1[q];
                }
            }
            if (kept) {
                s0 += coef[j] * v0;
                s1 += coef[j] * v1;
            }
        }
        const double w2 = axis == 0 ? w2y : w2x;
        a0 += w2 * s0;
        a1 += w2 * s1;
    }
    o0 = a0;
    o1 = a1;
}

template <int ORDER>
__global__ void __launch_bounds__(kLsqThreads) lsq_infill_kernel(LsqParams p)
{
    const int n = blockIdx.x;
    const int plane = p.ny * p.nx;
    float *U0 = p.ux + (long long)n * plane, *U1 = p.uy + (long long)n * plane;
    const unsigned char *bad = p.invalid + (long long)n * plane;
    char *wk = p.work + (size_t)n * p.work_stride;
    auto carve = [&](size_t bytes) { char *q = wk; wk += (bytes + 255) & ~size_t(255); return q; };
    unsigned char *cls = reinterpret_cast<unsigned char *>(carve((size_t)plane));
    int *list = reinterpret_cast<int *>(carve((size_t)plane * 4));
    double *P0 = reinterpret_cast<double *>(carve((size_t)plane * 8));
    double *P1 = reinterpret_cast<double *>(carve((size_t)plane * 8));
    double *X0 = reinterpret_cast<double *>(carve((size_t)plane * 8));
    double *X1 = reinterpret_cast<double *>(carve((size_t)plane * 8));
    double *R0 = reinterpret_cast<double *>(carve((size_t)plane * 8));
    double *R1 = reinterpret_cast<double *>(carve((size_t)plane * 8));
    double *Q0 = reinterpret_cast<double *>(carve((size_t)plane * 8));
    double *Q1 = reinterpret_cast<double *>(carve((size_t)plane * 8));
    __shared__ double2 red[kLsqWarps];
    __shared__ int s_cnt[kLsqWarps];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    // classes: 1 fill, 2 excluded, 0 known; the search direction is zero off the fill set
    for (int w = tid; w < plane; w += kLsqThreads) {
        const bool m = p.mask && p.mask[w] != 0.0f;
        unsigned char k = 0;
        if (bad[w] && !m) k = 1;
        else if (m || !isfinite(U0[w]) || !isfinite(U1[w])) k = 2;
        cls[w] = k;
        P0[w] = 0.0;
        P1[w] = 0.0;
    }
    __syncthreads();
    // fill cells listed in grid order
    const int seg = (plane + kLsqWarps - 1) / kLsqWarps;
    const int a = min(plane, warp * seg), b = min(plane, a + seg);
    int cnt = 0;
    for (int w0 = a; w0 < b; w0 += 32) {
        const int w = w0 + lane;
        cnt += __popc(__ballot_sync(0xffffffffu, w < b && cls[w] == 1));
    }
    if (lane == 0) s_cnt[warp] = cnt;
    __syncthreads();
    int base = 0, nf = 0;
    for (int k = 0; k < kLsqWarps; ++k) {
        base += k < warp ? s_cnt[k] : 0;
        nf += s_cnt[k];
    }
    for (int w0 = a; w0 < b; w0 += 32) {
        const int w = w0 + lane;
        const bool f = w < b && cls[w] == 1;
        const unsigned m = __ballot_sync(0xffffffffu, f);
        if (f) list[base + __popc(m & ((1u << lane) - 1u))] = w;
        base += __popc(m);
    }
    __syncthreads();
    if (nf == 0) return;

    // r0 = b (x0 = 0), p0 = r0
    double rr0 = 0.0, rr1 = 0.0;
    for (int i = tid; i < nf; i += kLsqThreads) {
        const int w = list[i];
        double k0, k1;
        lsq_rows<ORDER>(cls, w / p.nx, w % p.nx, p.ny, p.nx, p.w2y, p.w2x, nullptr, nullptr, U0, U1, true, k0, k1);
        X0[i] = 0.0;
        X1[i] = 0.0;
        R0[i] = -k0;
        R1[i] = -k1;
        P0[w] = -k0;
        P1[w] = -k1;
        rr0 += k0 * k0;
        rr1 += k1 * k1;
    }
    double2 rr = lsq_block_sum2(rr0, rr1, red);      // includes the barrier the P writes need
    const double stop0 = p.tol2 * rr.x, stop1 = p.tol2 * rr.y;
    bool act0 = rr.x > 0.0, act1 = rr.y > 0.0;
    for (int it = 0; it < p.max_iter && (act0 || act1); ++it) {
        double pq0 = 0.0, pq1 = 0.0;
        for (int i = tid; i < nf; i += kLsqThreads) {
            const int w = list[i];
            double q0, q1;
            lsq_rows<ORDER>(cls, w / p.nx, w % p.nx, p.ny, p.nx, p.w2y, p.w2x, P0, P1, nullptr, nullptr, false, q0,
                            q1);
            Q0[i] = q0;
            Q1[i] = q1;
            pq0 += P0[w] * q0;
            pq1 += P1[w] * q1;
        }
        const double2 pq = lsq_block_sum2(pq0, pq1, red);
        act0 = act0 && pq.x > 0.0;
        act1 = act1 && pq.y > 0.0;
        const double al0 = act0 ? rr.x / pq.x : 0.0, al1 = act1 ? rr.y / pq.y : 0.0;
        double rn0 = 0.0, rn1 = 0.0;
        for (int i = tid; i < nf; i += kLsqThreads) {
            const int w = list[i];
            if (act0) {
                X0[i] += al0 * P0[w];
                R0[i] -= al0 * Q0[i];
                rn0 += R0[i] * R0[i];
            }
            if (act1) {
                X1[i] += al1 * P1[w];
                R1[i] -= al1 * Q1[i];
                rn1 += R1[i] * R1[i];
            }
        }
        const double2 rn = lsq_block_sum2(rn0, rn1, red);
        const double be0 = act0 ? rn.x / rr.x : 0.0, be1 = act1 ? rn.y / rr.y : 0.0;
        for (int i = tid; i < nf; i += kLsqThreads) {
            const int w = list[i];
            if (act0) P0[w] = R0[i] + be0 * P0[w];
            if (act1) P1[w] = R1[i] + be1 * P1[w];
        }
        if (act0) rr.x = rn.x;
        if (act1) rr.y = rn.y;
        act0 = act0 && rr.x > stop0;
        act1 = act1 && rr.y > stop1;
        __syncthreads();
    }
    for (int i = tid; i < nf; i += kLsqThreads) {
        const int w = list[i];
        U0[w] = (float)X0[i];
        U1[w] = (float)X1[i];
    }
}

// Edge-replicate padding (ny, nx) -> (nyp, nxp) with the measured grid at
// (pre_y, pre_x); channel order (dy, dx) -> two planes.
__global__ void pad_kernel(const float *ux, const float *uy, int N, int ny, int nx, int nyp, int nxp, int pre_y,
                           int pre_x, float *pdy, float *pdx)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)N * nyp * nxp) return;
    const int n = (int)(i / ((long long)nyp * nxp)), w = (int)(i % ((long long)nyp * nxp));
    const int r = min(max(w / nxp - pre_y, 0), ny - 1), c = min(max(w % nxp - pre_x, 0), nx - 1);
    const long long s = (long long)n * ny * nx + r * nx + c;
    pdy[i] = uy[s];
    pdx[i] = ux[s];
}

// One separable Gaussian pass (mode 'nearest'), along x (axis 1) or y (axis 0).
__global__ void gauss_kernel(const float *in, float *out, int N, int ny, int nx, const float *taps, int radius, int axis)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)N * ny * nx) return;
    const int n = (int)(i / ((long long)ny * nx)), w = (int)(i % ((long long)ny * nx));
    const int r = w / nx, c = w % nx;
    const float *P = in + (long long)n * ny * nx;
    double acc = 0.0;
    for (int k = -radius; k <= radius; ++k) {
        const int rr = axis == 0 ? min(max(r + k, 0), ny - 1) : r;
        const int cc = axis == 1 ? min(max(c + k, 0), nx - 1) : c;
        acc += (double)taps[k + radius] * (double)P[rr * nx + cc];
    }
    out[i] = (float)acc;
}


// OpenCV's INTER_CUBIC coefficients (Keys, A = -0.75) at fraction x, in float
// arithmetic with its operation order (no contraction).
__device__ __forceinline__ void cv_cubic(float x, float (&c)[4])
{
    const float A = -0.75f;
    const float x1 = __fadd_rn(x, 1.0f), y = __fsub_rn(1.0f, x);
    c[0] = __fsub_rn(__fmul_rn(__fadd_rn(__fmul_rn(__fsub_rn(__fmul_rn(A, x1), 5.0f * A), x1), 8.0f * A), x1),
                     4.0f * A);
    c[1] = __fadd_rn(__fmul_rn(__fmul_rn(__fsub_rn(__fmul_rn(A + 2.0f, x), A + 3.0f), x), x), 1.0f);
    c[2] = __fadd_rn(__fmul_rn(__fmul_rn(__fsub_rn(__fmul_rn(A + 2.0f, y), A + 3.0f), y), y), 1.0f);
    c[3] = __fsub_rn(__fsub_rn(__fsub_rn(1.0f, c[0]), c[1]), c[2]);
}

// Predictor remap as cv2.remap(INTER_CUBIC, BORDER_REPLICATE) computes it for
// float32 planes and float maps (cpu_instantaneous.py:1050-1071): coordinates
// rounded to 1/32 px (round half to even), 4 x 4 taps weighted by products of
// the 32-entry coefficient table; inside the plane the four row sums are formed
// left to right and added in row order, at the border every tap (clamped
// indices) is added to a running sum in row-major order.
__global__ void remap_kernel(const float *pdy, const float *pdx, int N, int nyp, int nxp, const float *map_y,
                             const float *map_x, int ny, int nx, float *oy, float *ox)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)N * ny * nx) return;
    const int n = (int)(i / ((long long)ny * nx)), w = (int)(i % ((long long)ny * nx));
    const int sx = __float2int_rn(__fmul_rn(map_x[w], 32.0f));
    const int sy = __float2int_rn(__fmul_rn(map_y[w], 32.0f));
    const int bx = (sx >> 5) - 1, by = (sy >> 5) - 1;
    float cy[4], cx[4], wt[16];
    cv_cubic(__fmul_rn((float)(sy & 31), 1.0f / 32.0f), cy);
    cv_cubic(__fmul_rn((float)(sx & 31), 1.0f / 32.0f), cx);
#pragma unroll
    for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int q = 0; q < 4; ++q) wt[m * 4 + q] = __fmul_rn(cy[m], cx[q]);
    const float *Py = pdy + (long long)n * nyp * nxp, *Px = pdx + (long long)n * nyp * nxp;
    float vy, vx;
    if (bx >= 0 && bx < nxp - 3 && by >= 0 && by < nyp - 3) {
        float ry[4], rx[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const float *a = Py + (long long)(by + m) * nxp + bx, *b = Px + (long long)(by + m) * nxp + bx;
            ry[m] = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(a[0], wt[4 * m]), __fmul_rn(a[1], wt[4 * m + 1])),
                                        __fmul_rn(a[2], wt[4 * m + 2])), __fmul_rn(a[3], wt[4 * m + 3]));
            rx[m] = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(b[0], wt[4 * m]), __fmul_rn(b[1], wt[4 * m + 1])),
                                        __fmul_rn(b[2], wt[4 * m + 2])), __fmul_rn(b[3], wt[4 * m + 3]));
        }
        vy = __fadd_rn(__fadd_rn(__fadd_rn(ry[0], ry[1]), ry[2]), ry[3]);
        vx = __fadd_rn(__fadd_rn(__fadd_rn(rx[0], rx[1]), rx[2]), rx[3]);
    } else {
        vy = 0.0f;
        vx = 0.0f;
        for (int m = 0; m < 4; ++m) {
            const int r = min(max(by + m, 0), nyp - 1);
            for (int q = 0; q < 4; ++q) {
                const int c = min(max(bx + q, 0), nxp - 1);
                vy = __fadd_rn(vy, __fmul_rn(Py[(long long)r * nxp + c], wt[m * 4 + q]));
                vx = __fadd_rn(vx, __fmul_rn(Px[(long long)r * nxp + c], wt[m * 4 + q]));
            }
        }
    }
    oy[i] = vy;
    ox[i] = vx;
}

inline unsigned blocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

// Validation of one pass for N pairs.  pred_* (nullable) is the window-grid
// predictor added to the correlation result.  Outputs ux, uy (NaN = to infill,
// 0 at masked windows), invalid flags and (nullable) int8 reason codes.
// work: 2*N*ny*nx floats.
PIV_EXPORT int pivb_validate_dev(const float *pk_x, const float *pk_y, const float *pk_h, const float *pred_dy,
                                 const float *pred_dx, const float *mask, int N, int ny, int nx, float thresh_x,
                                 float thresh_y, float peak_thr, float med_eps, float med_thr, int med_size,
                                 float *ux, float *uy, unsigned char *invalid, signed char *nan_reason,
                                 float *work, void *stream)
{
    if (N <= 0 || ny <= 0 || nx <= 0 || med_size < 3 || med_size > 5 || !(med_size & 1)) return 1;
    cudaStream_t s = (cudaStream_t)stream;
    ValParams p{pk_x, pk_y, pk_h, pred_dy, pred_dx, mask, N, ny, nx, thresh_x, thresh_y, peak_thr, med_eps,
                med_thr, med_size, ux, uy, invalid, nan_reason, (long long)ny * nx, 0, 1, nullptr};
    const long long nv = (long long)N * ny * nx;
    gate_kernel<<<blocks(nv, 256), 256, 0, s>>>(p, med_thr > 0.0f ? 0 : 1);
    if (med_thr > 0.0f) {
        float *gx = work, *gy = work + nv;
        cudaMemcpyAsync(gx, ux, nv * 4, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(gy, uy, nv * 4, cudaMemcpyDeviceToDevice, s);
        median_kernel<<<blocks(nv, 256), 256, 0, s>>>(p, gx, gy);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

namespace {
__global__ void gather_fill_kernel(const float *__restrict__ ux, const float *__restrict__ uy,
                                   const int *__restrict__ idx, long long plane, long long nv, float *out_x,
                                   float *out_y)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nv) return;
    const long long n = i / plane, w = i - n * plane;
    const long long src = n * plane + idx[w];
    out_x[i] = ux[src];
    out_y[i] = uy[src];
}
}  // namespace

// The 'nearest' fill of the masked windows of a predictor (infilling.py:808-874):
// out[n][w] = in[n][idx[w]] for N fields of `plane` windows, idx the donor map of
// the mask (each unmasked window its own donor).  Returns 0, or 1 for bad
// arguments.
PIV_EXPORT int pivb_gather_fill_dev(const float *ux, const float *uy, const int *idx, int N, long long plane,
                                    float *out_x, float *out_y, void *stream)
{
    if (!ux || !uy || !idx || !out_x || !out_y || N <= 0 || plane <= 0) return 1;
    const long long nv = (long long)N * plane;
    gather_fill_kernel<<<blocks(nv, 256), 256, 0, (cudaStream_t)stream>>>(ux, uy, idx, plane, nv, out_x, out_y);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

namespace {
// Nearest-donor infill (infilling.py:114-141, 290-333): each fill cell takes both
// components of the nearest donor -- a cell neither filled nor excluded (masked)
// and finite in both components -- in physical distance (pitch py, px).  Among
// equidistant donors the one of smallest column, then smallest row, is taken:
// the choice scipy's Euclidean feature transform makes (checked against it on
// random, striped and holed grids with isotropic and anisotropic pitches).  The
// search walks square rings of growing index radius R and stops once
// (R * min(py, px))^2 exceeds the best squared distance.  Donors are never
// written, so the fill is in place.  A pair without any donor keeps 0 there.
__global__ void nearest_infill_kernel(float *ux, float *uy, const unsigned char *__restrict__ invalid,
                                      const float *__restrict__ mask, int N, int ny, int nx, double py, double px)
{
    const long long plane = (long long)ny * nx;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= plane * N || !invalid[i]) return;
    const long long n = i / plane;
    const int w = (int)(i - n * plane), y = w / nx, x = w % nx;
    const float *X = ux + n * plane, *Y = uy + n * plane;
    const unsigned char *inv = invalid + n * plane;
    const double pmin = py < px ? py : px;
    double best = INFINITY;
    int bx = 0x7fffffff, by = 0x7fffffff;
    const int rmax = ny > nx ? ny : nx;
    for (int R = 1; R <= rmax; ++R) {
        const double ring = (double)R * pmin;
        if (ring * ring > best) break;
        for (int dy = -R; dy <= R; ++dy) {
            const int yy = y + dy;
            if (yy < 0 || yy >= ny) continue;
            const int step = (dy == -R || dy == R) ? 1 : 2 * R;      // whole edge rows, else the two sides
            for (int dx = -R; dx <= R; dx += step) {
                const int xx = x + dx;
                if (xx < 0 || xx >= nx) continue;
                const int c = yy * nx + xx;
                if (inv[c] || (mask && mask[c] != 0.0f)) continue;
                const float a = X[c], b = Y[c];
                if (a != a || b != b || isinf(a) || isinf(b)) continue;
                const double d = (dy * py) * (dy * py) + (dx * px) * (dx * px);
                if (d < best || (d == best && (xx < bx || (xx == bx && yy < by)))) {
                    best = d;
                    bx = xx;
                    by = yy;
                }
            }
        }
    }
    if (bx == 0x7fffffff) {
        ux[i] = 0.0f;
        uy[i] = 0.0f;
    } else {
        ux[i] = X[by * nx + bx];
        uy[i] = Y[by * nx + bx];
    }
}
}  // namespace

// Nearest-donor infill of the invalid vectors in place (the reference's
// infilling method 'nearest', infilling.py:290-333), mask (nullable) the
// excluded (masked) windows.  Returns 0, or 1 for bad arguments.
PIV_EXPORT int pivb_nearest_infill_dev(float *ux, float *uy, const unsigned char *invalid, const float *mask, int N,
                                       int ny, int nx, double pitch_y, double pitch_x, void *stream)
{
    if (!ux || !uy || !invalid || N <= 0 || ny <= 0 || nx <= 0 || !(pitch_y > 0.0) || !(pitch_x > 0.0)) return 1;
    const long long nv = (long long)N * ny * nx;
    nearest_infill_kernel<<<blocks(nv, 256), 256, 0, (cudaStream_t)stream>>>(ux, uy, invalid, mask, N, ny, nx,
                                                                             pitch_y, pitch_x);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// ---------------------------------------------------------------------------
// Further outlier tests: local sigma and divergence/vorticity
// (outlier_detection.py:246-381), on a field in which masked windows are NaN
// and, in the primary tests, failed vectors are 0 (zero_fill) as the driver
// zero-fills them (cpu_instantaneous.py:627-629); in the substitution rounds
// failed vectors stay NaN.  Flags are OR-ed into `flags`.
// ---------------------------------------------------------------------------
namespace {

struct ExtraParams {
    const float *X, *Y;              // (N, ny, nx)
    const float *mask;               // (ny, nx) or null
    int N, ny, nx, zero_fill;
    float sigma_thr;                 // <= 0: off
    float *div, *vort;               // work (N, ny, nx)
    float *absdev;                   // work (N, ny, nx)
    float *thr;                      // work (N, 2): divergence and vorticity thresholds
    float div_thr, vort_thr;         // < 0: from the field (6 x 1.4826 x MAD)
    unsigned char *flags;            // (N, ny, nx), OR-ed
};

// The field value the tests see at (n, r, c): NaN at masked windows, 0 for a
// failed vector when zero_fill.
__device__ __forceinline__ void test_field(const ExtraParams &q, long long base, int r, int c, float &a, float &b)
{
    const int w = r * q.nx + c;
    if (q.mask && q.mask[w] != 0.0f) { a = qnanf(); b = qnanf(); return; }
    a = q.X[base + w];
    b = q.Y[base + w];
    if (q.zero_fill && (a != a || b != b)) { a = 0.0f; b = 0.0f; }
}

// |u| of (a, b) in float32 as np.sqrt(ux**2 + uy**2), NaN kept.
__device__ __forceinline__ float vnorm(float a, float b)
{
    return __fsqrt_rn(__fadd_rn(__fmul_rn(a, a), __fmul_rn(b, b)));
}

// 3-point mean along one axis as scipy's uniform_filter1d (size 3, mode
// constant, cval 0): double sum, / 3, rounded to float32.
__device__ __forceinline__ float mean3(float l, float c, float r)
{
    return (float)((((double)l + (double)c) + (double)r) / 3.0);
}

// Local 8-neighbour sigma test on the vector norm (combine 'norm';
// outlier_detection.py:246-319): scipy's 3x3 uniform filter of v0, v0^2 and the
// finite mask (axis 0, then axis 1), x 9, minus the centre, mean and standard
// deviation over the finite neighbours.
__global__ void sigma_kernel(ExtraParams q)
{
    const long long plane = (long long)q.ny * q.nx;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= plane * q.N) return;
    const long long n = i / plane, base = n * plane;
    const int w = (int)(i - base), r = w / q.nx, c = w % q.nx;
    // first pass (axis 0) at columns c-1, c, c+1; zero outside the grid
    float t_v[3], t_v2[3], t_f[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const int cc = c + j - 1;
        float col_v[3], col_v2[3], col_f[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int rr = r + k - 1;
            col_v[k] = 0.0f; col_v2[k] = 0.0f; col_f[k] = 0.0f;
            if (rr >= 0 && rr < q.ny && cc >= 0 && cc < q.nx) {
                float a, b;
                test_field(q, base, rr, cc, a, b);
                const float v = vnorm(a, b);
                const bool fin = isfinite(v);
                const float v0 = fin ? v : 0.0f;
                col_v[k] = v0;
                col_v2[k] = __fmul_rn(v0, v0);
                col_f[k] = fin ? 1.0f : 0.0f;
            }
        }
        const bool inside = cc >= 0 && cc < q.nx;
        t_v[j] = inside ? mean3(col_v[0], col_v[1], col_v[2]) : 0.0f;
        t_v2[j] = inside ? mean3(col_v2[0], col_v2[1], col_v2[2]) : 0.0f;
        t_f[j] = inside ? mean3(col_f[0], col_f[1], col_f[2]) : 0.0f;
    }
    const float m9_v = mean3(t_v[0], t_v[1], t_v[2]);
    const float m9_v2 = mean3(t_v2[0], t_v2[1], t_v2[2]);
    const float m9_f = mean3(t_f[0], t_f[1], t_f[2]);
    float a, b;
    test_field(q, base, r, c, a, b);
    const float v = vnorm(a, b);
    const bool fin = isfinite(v);
    const float cv = fin ? v : 0.0f, cf = fin ? 1.0f : 0.0f;
    const float sum8 = __fsub_rn(__fmul_rn(m9_v, 9.0f), cv);
    const float sumsq8 = __fsub_rn(__fmul_rn(m9_v2, 9.0f), __fmul_rn(cv, cv));
    const float cnt8 = __fsub_rn(__fmul_rn(m9_f, 9.0f), cf);
    const float mean8 = __fdiv_rn(sum8, cnt8);
    float var8 = __fsub_rn(__fdiv_rn(sumsq8, cnt8), __fmul_rn(mean8, mean8));
    if (!(var8 != var8)) var8 = fmaxf(var8, 0.0f);      // np.maximum keeps NaN
    const float std8 = __fsqrt_rn(var8);
    const bool out = (fabsf(__fsub_rn(v, mean8)) > __fmul_rn(q.sigma_thr, std8)) || !fin || !isfinite(mean8) ||
                     std8 == 0.0f || cnt8 < 1.0f;
    if (out) q.flags[i] = 1;
}

// Central differences with periodic wrap (np.roll), float32:
// div = dudx + dvdy, vort = dvdx - dudy (outlier_detection.py:351-358).
__global__ void divvort_field_kernel(ExtraParams q)
{
    const long long plane = (long long)q.ny * q.nx;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= plane * q.N) return;
    const long long n = i / plane, base = n * plane;
    const int w = (int)(i - base), r = w / q.nx, c = w % q.nx;
    const int cp = (c + 1) % q.nx, cm = (c - 1 + q.nx) % q.nx, rp = (r + 1) % q.ny, rm = (r - 1 + q.ny) % q.ny;
    float uxp, uyp, uxm, uym, vxp, vyp, vxm, vym;
    test_field(q, base, r, cp, uxp, uyp);     // (ux, uy) at column c+1
    test_field(q, base, r, cm, uxm, uym);
    test_field(q, base, rp, c, vxp, vyp);     // at row r+1
    test_field(q, base, rm, c, vxm, vym);
    const float dudx = __fmul_rn(0.5f, __fsub_rn(uxp, uxm));
    const float dvdx = __fmul_rn(0.5f, __fsub_rn(uyp, uym));
    const float dudy = __fmul_rn(0.5f, __fsub_rn(vxp, vxm));
    const float dvdy = __fmul_rn(0.5f, __fsub_rn(vyp, vym));
    q.div[i] = __fadd_rn(dudx, dvdy);
    q.vort[i] = __fsub_rn(dvdx, dudy);
}

__device__ __forceinline__ unsigned fkey(float f)
{
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ float fkey_inv(unsigned k)
{
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// The k-th smallest (0-based) finite value of v[0..n) by 8-bit radix selection,
// one CTA; every thread returns it.
__device__ float select_kth(const float *v, long long n, long long k, unsigned *hist, unsigned *shared)
{
    unsigned prefix = 0, pmask = 0;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int b = threadIdx.x; b < 256; b += blockDim.x) hist[b] = 0;
        __syncthreads();
        for (long long j = threadIdx.x; j < n; j += blockDim.x) {
            const float x = v[j];
            if (!isfinite(x)) continue;
            const unsigned key = fkey(x);
            if ((key & pmask) == prefix) atomicAdd(&hist[(key >> shift) & 255u], 1u);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            long long cum = 0;
            int b = 0;
            for (; b < 255; ++b) {
                if (cum + hist[b] > k) break;
                cum += hist[b];
            }
            k -= cum;
            shared[0] = prefix | ((unsigned)b << shift);
            shared[1] = (unsigned)k;
        }
        __syncthreads();
        prefix = shared[0];
        k = shared[1];
        pmask |= 255u << shift;
        __syncthreads();
    }
    return fkey_inv(prefix);
}

// np.median of the finite values of v[0..n) (float32; mean of the two middle
// values for an even count); count = the number of finite values.
__device__ float median_finite(const float *v, long long n, long long count, unsigned *hist, unsigned *shared)
{
    if (count & 1) return select_kth(v, n, count / 2, hist, shared);
    const float lo = select_kth(v, n, count / 2 - 1, hist, shared);
    const float hi = select_kth(v, n, count / 2, hist, shared);
    return __fmul_rn(__fadd_rn(lo, hi), 0.5f);
}

// Per pair (one CTA): thresholds 6 * 1.4826 * MAD of the finite divergence and
// vorticity values (inf if none), unless given.
__global__ void divvort_thresh_kernel(ExtraParams q)
{
    __shared__ unsigned hist[256];
    __shared__ unsigned shared[2];
    __shared__ unsigned long long cnt;
    const long long plane = (long long)q.ny * q.nx;
    const int n = blockIdx.x;
    for (int f = 0; f < 2; ++f) {
        const float given = f == 0 ? q.div_thr : q.vort_thr;
        if (given >= 0.0f) {
            if (threadIdx.x == 0) q.thr[2 * n + f] = given;
            continue;
        }
        const float *v = (f == 0 ? q.div : q.vort) + n * plane;
        float *ad = q.absdev + n * plane;
        if (threadIdx.x == 0) cnt = 0;
        __syncthreads();
        unsigned long long mine = 0;
        for (long long j = threadIdx.x; j < plane; j += blockDim.x) mine += isfinite(v[j]) ? 1 : 0;
        atomicAdd(&cnt, mine);
        __syncthreads();
        const long long count = (long long)cnt;
        if (count == 0) {
            if (threadIdx.x == 0) q.thr[2 * n + f] = INFINITY;
            __syncthreads();
            continue;
        }
        const float med = median_finite(v, plane, count, hist, shared);
        for (long long j = threadIdx.x; j < plane; j += blockDim.x)
            ad[j] = isfinite(v[j]) ? fabsf(__fsub_rn(v[j], med)) : qnanf();
        __syncthreads();
        const float mad = __fmul_rn(1.4826f, median_finite(ad, plane, count, hist, shared));
        if (threadIdx.x == 0) q.thr[2 * n + f] = __fmul_rn(6.0f, mad);
        __syncthreads();
    }
}

__global__ void divvort_flag_kernel(ExtraParams q)
{
    const long long plane = (long long)q.ny * q.nx;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= plane * q.N) return;
    const long long n = i / plane;
    if (fabsf(q.div[i]) > q.thr[2 * n] || fabsf(q.vort[i]) > q.thr[2 * n + 1]) q.flags[i] = 1;
}

// Run the enabled further tests on (X, Y), OR-ing into flags (zeroed here).
void extra_outliers(ExtraParams q, int divvort, cudaStream_t s)
{
    const long long nv = (long long)q.N * q.ny * q.nx;
    cudaMemsetAsync(q.flags, 0, nv, s);
    if (q.sigma_thr > 0.0f) sigma_kernel<<<blocks(nv, 256), 256, 0, s>>>(q);
    if (divvort) {
        divvort_field_kernel<<<blocks(nv, 256), 256, 0, s>>>(q);
        divvort_thresh_kernel<<<q.N, 1024, 0, s>>>(q);
        divvort_flag_kernel<<<blocks(nv, 256), 256, 0, s>>>(q);
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// Secondary-peak substitution (cpu_instantaneous.py:676-760)
// ---------------------------------------------------------------------------
namespace {

struct SecParams {
    const float *pk_x, *pk_y, *pk_h;      // (N, P, ny, nx): every peak of the correlator
    int P;
    const float *pred_dy, *pred_dx;       // (N, ny, nx) or null
    const float *mask;                    // (ny, nx) or null
    int N, ny, nx;
    float thresh_x, thresh_y, peak_thr, med_eps, med_thr;
    int med_size;
    float *ux, *uy;                       // out
    unsigned char *invalid;               // in/out
    signed char *reason;                  // in/out
    unsigned char *choice;                // in/out: 1-based peak of each vector (0 = invalid)
    float *cx, *cy;                       // work: the field of the current choices
    unsigned char *active;                // work: substituted in this round
    int substitute;                       // 0: only copy each vector's current choice
    const unsigned char *extra;           // flags of the further tests on cx/cy, or null
};

// Peak k of vector i after the gate and the predictor (NaN where masked, gated or
// not found), and its gated height.
__device__ __forceinline__ void gated_peak(const SecParams &q, long long i, int k, float &x, float &y, float &h)
{
    const long long plane = (long long)q.ny * q.nx;
    const long long n = i / plane, w = i - n * plane;
    const long long src = (n * q.P + k) * plane + w;
    x = q.pk_x[src];
    y = q.pk_y[src];
    h = q.pk_h[src];
    const bool masked = q.mask && q.mask[w] != 0.0f;
    const bool large = fabsf(x) > q.thresh_x || fabsf(y) > q.thresh_y;
    if (masked || large) { x = qnanf(); y = qnanf(); h = qnanf(); }
    if (q.pred_dx) { x += q.pred_dx[i]; y += q.pred_dy[i]; }
}

// One substitution round: every invalid vector with peaks left takes its next
// peak and is judged afresh (NaN -> still invalid, reason 13; else valid until
// the outlier tests below); every vector's current choice is written to cx/cy.
__global__ void subst_kernel(SecParams q)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nv = (long long)q.N * q.ny * q.nx;
    if (i >= nv) return;
    const int w = (int)(i % ((long long)q.ny * q.nx));
    if (q.mask && q.mask[w] != 0.0f) {
        q.cx[i] = qnanf();
        q.cy[i] = qnanf();
        q.active[i] = 0;
        return;
    }
    int c = q.choice[i];
    const bool act = q.substitute && q.invalid[i] && c < q.P;
    if (act) q.choice[i] = (unsigned char)(++c);
    float x, y, h;
    gated_peak(q, i, c - 1, x, y, h);
    q.cx[i] = x;
    q.cy[i] = y;
    q.active[i] = act ? 1 : 0;
    if (act) {
        const bool sub_nan = (x != x) || (y != y);
        q.invalid[i] = sub_nan ? 1 : 0;
        q.reason[i] = sub_nan ? kPeakMagNaN : kValid;
    }
}

// The outlier tests on the substituted field (outlier_detection.py:382-460 with
// the masked windows NaN): the peak magnitude of the current choice and the
// normalised median over cx/cy, whose NaN cells drop out of the medians and are
// absent from the 3x3 guard (masked cells count as present).  Only vectors
// substituted in this round and finite are re-flagged (reason 12).
__global__ void sec_median_kernel(SecParams q)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nv = (long long)q.N * q.ny * q.nx;
    if (i >= nv || !q.active[i]) return;
    const int plane = q.ny * q.nx;
    const int n = (int)(i / plane), w = (int)(i % plane), r = w / q.nx, c = w % q.nx;
    const float u0 = q.cx[i], v0 = q.cy[i];
    if (u0 != u0 || v0 != v0) return;
    float x, y, h;
    gated_peak(q, i, q.choice[i] - 1, x, y, h);
    bool outlier = q.peak_thr >= 0.0f && ((h < q.peak_thr) || (h != h));
    if (q.med_thr > 0.0f) {
        const float *X = q.cx + (long long)n * plane, *Y = q.cy + (long long)n * plane;
        const int hs = q.med_size / 2;
        float nu[24], nvv[24];
        int present = 0;
#pragma unroll
        for (int t = 0; t < 25; ++t) {
            const int dr = t / 5 - 2, dc = t % 5 - 2;
            const int rr = r + dr, cc = c + dc;
            const bool inside = rr >= 0 && rr < q.ny && cc >= 0 && cc < q.nx && abs(dr) <= hs && abs(dc) <= hs;
            float a = qnanf(), b = qnanf();
            if (inside) {
                const bool mk = q.mask && q.mask[rr * q.nx + cc] != 0.0f;
                if (!mk) {
                    a = X[rr * q.nx + cc];
                    b = Y[rr * q.nx + cc];
                }
                const bool fin = (a == a) && (b == b);
                if (abs(dr) <= 1 && abs(dc) <= 1 && (fin || mk)) ++present;
            }
            if (t == 12) continue;
            nu[t < 12 ? t : t - 1] = a;
            nvv[t < 12 ? t : t - 1] = b;
        }
        const float mu = median24(nu), mv = median24(nvv);
        const float r0 = sqrtf((u0 - mu) * (u0 - mu) + (v0 - mv) * (v0 - mv));
        float ri[24];
#pragma unroll
        for (int j = 0; j < 24; ++j)
            ri[j] = sqrtf((nu[j] - mu) * (nu[j] - mu) + (nvv[j] - mv) * (nvv[j] - mv));
        const float rm = median24(ri);
        const float nr = r0 / (rm + q.med_eps);
        outlier = outlier || (nr > q.med_thr) || !isfinite(nr) || present < 6;
    }
    if (q.extra && q.extra[i]) outlier = true;
    if (outlier) {
        q.invalid[i] = 1;
        q.reason[i] = kSecondaryOutlier;
    }
}

// The end of the stage: a NaN peak height of the chosen peak invalidates (13),
// remaining invalid vectors without a reason are 9, invalid vectors become NaN
// and lose their choice, masked windows read 0 with reason -1.
__global__ void sec_final_kernel(SecParams q)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nv = (long long)q.N * q.ny * q.nx;
    if (i >= nv) return;
    const int w = (int)(i % ((long long)q.ny * q.nx));
    if (q.mask && q.mask[w] != 0.0f) {
        q.ux[i] = 0.0f;
        q.uy[i] = 0.0f;
        q.invalid[i] = 0;
        q.reason[i] = kMasked;
        q.choice[i] = 0;
        return;
    }
    const int c = q.choice[i];
    float x, y, h;
    gated_peak(q, i, (c > 0 ? c : 1) - 1, x, y, h);
    const bool hnan = h != h;
    const bool bad = q.invalid[i] || hnan;
    signed char rc = q.reason[i];
    if (hnan && rc == kValid) rc = kPeakMagNaN;
    if (bad && rc == kValid) rc = kUnclassified;
    q.reason[i] = rc;
    q.invalid[i] = bad ? 1 : 0;
    q.ux[i] = bad ? qnanf() : q.cx[i];
    q.uy[i] = bad ? qnanf() : q.cy[i];
    q.choice[i] = bad ? 0 : (unsigned char)c;
}

__global__ void choice_init_kernel(unsigned char *choice, long long nv)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nv) choice[i] = 1;
}

}  // namespace

// Validation of one pass whose correlation returned P >= 1 peaks per window
// (pk_* in the correlator's layout (N, P, ny, nx)), with the reference's
// further outlier tests and its secondary-peak substitution:
//   * the primary peak is gated, predicted and tested as by pivb_validate_dev,
//     plus, when enabled, the local sigma test (sigma_thr > 0) and the
//     divergence/vorticity test (divvort; div_thr / vort_thr < 0: 6 x 1.4826 x
//     MAD of the pair's field), all OR-ed as outliers (reason 10);
//   * with `secondary` and P > 1, P - 1 rounds in which every invalid vector
//     with peaks left takes its next peak, is judged afresh (NaN: reason 13) and
//     is tested by every enabled test on the field of the current choices
//     (reason 12 when it fails);
//   * at the end a NaN height of the chosen peak invalidates (13).
// Outputs as pivb_validate_dev plus choice (N, ny, nx): the 1-based peak each
// valid vector took, 0 for invalid and masked vectors.
// work: pivb_validate_peaks_work_floats(N, ny, nx) floats.  Returns 0, or 1 for
// bad arguments.
PIV_EXPORT long long pivb_validate_peaks_work_floats(int N, int ny, int nx)
{
    if (N <= 0 || ny <= 0 || nx <= 0) return 0;
    return 8LL * N * ny * nx + 2LL * N;
}

PIV_EXPORT int pivb_validate_peaks_dev(const float *pk_x, const float *pk_y, const float *pk_h, int n_peaks,
                                       int secondary, const float *pred_dy, const float *pred_dx,
                                       const float *mask, int N, int ny, int nx, float thresh_x, float thresh_y,
                                       float peak_thr, float med_eps, float med_thr, int med_size, float sigma_thr,
                                       int divvort, float div_thr, float vort_thr, float *ux, float *uy,
                                       unsigned char *invalid, signed char *nan_reason, unsigned char *choice,
                                       float *work, void *stream)
{
    if (N <= 0 || ny <= 0 || nx <= 0 || n_peaks < 1 || n_peaks > 255 || med_size < 3 || med_size > 5 ||
        !(med_size & 1) || !nan_reason || !choice || !work)
        return 1;
    cudaStream_t s = (cudaStream_t)stream;
    const long long plane = (long long)ny * nx, nv = (long long)N * plane;
    const bool sec = secondary && n_peaks > 1;
    const bool extra_on = sigma_thr > 0.0f || divvort != 0;
    float *gx = work, *gy = work + nv, *cx = work + 2 * nv, *cy = work + 3 * nv;
    float *divf = work + 4 * nv, *vortf = work + 5 * nv, *absdev = work + 6 * nv;
    unsigned char *flags = reinterpret_cast<unsigned char *>(work + 7 * nv);
    unsigned char *active = flags + nv;
    float *thr = work + 8 * nv;
    ValParams p{pk_x, pk_y, pk_h, pred_dy, pred_dx, mask, N, ny, nx, thresh_x, thresh_y, peak_thr, med_eps,
                med_thr, med_size, ux, uy, invalid, nan_reason, (long long)n_peaks * plane, sec ? 1 : 0,
                med_thr > 0.0f ? 1 : 0, extra_on ? flags : nullptr};
    const bool finalize = med_thr > 0.0f || extra_on;
    gate_kernel<<<blocks(nv, 256), 256, 0, s>>>(p, (finalize || sec) ? 0 : 1);
    if (finalize) {
        cudaMemcpyAsync(gx, ux, nv * 4, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(gy, uy, nv * 4, cudaMemcpyDeviceToDevice, s);
        if (extra_on) {
            ExtraParams e{gx, gy, mask, N, ny, nx, 1, sigma_thr, divf, vortf, absdev, thr, div_thr, vort_thr, flags};
            extra_outliers(e, divvort, s);
        }
        median_kernel<<<blocks(nv, 256), 256, 0, s>>>(p, gx, gy);
    }
    choice_init_kernel<<<blocks(nv, 256), 256, 0, s>>>(choice, nv);
    SecParams q{pk_x, pk_y, pk_h, n_peaks, pred_dy, pred_dx, mask, N, ny, nx, thresh_x, thresh_y, peak_thr,
                med_eps, med_thr, med_size, ux, uy, invalid, nan_reason, choice, cx, cy, active, sec ? 1 : 0,
                extra_on ? flags : nullptr};
    if (sec) {
        for (int round = 1; round < n_peaks; ++round) {
            subst_kernel<<<blocks(nv, 256), 256, 0, s>>>(q);
            if (extra_on) {
                ExtraParams e{cx, cy, mask, N, ny, nx, 0, sigma_thr, divf, vortf, absdev, thr, div_thr, vort_thr,
                              flags};
                extra_outliers(e, divvort, s);
            }
            sec_median_kernel<<<blocks(nv, 256), 256, 0, s>>>(q);
        }
    } else {
        subst_kernel<<<blocks(nv, 256), 256, 0, s>>>(q);   // substitute = 0: copies peak 1
    }
    sec_final_kernel<<<blocks(nv, 256), 256, 0, s>>>(q);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// Work bytes of pivb_infill_dev per call (per pair: a class byte, a list index
// and eight FP64 values per grid cell).
static size_t lsq_pair_bytes(int ny, int nx)
{
    const size_t plane = (size_t)ny * nx;
    auto pad = [](size_t b) { return (b + 255) & ~size_t(255); };
    return pad(plane) + pad(plane * 4) + 8 * pad(plane * 8);
}

PIV_EXPORT size_t pivb_infill_work_bytes(int N, int ny, int nx)
{
    if (N <= 0 || ny <= 0 || nx <= 0) return 0;
    return (size_t)N * lsq_pair_bytes(ny, nx);
}

// Least-squares infilling of the invalid vectors in place (order 1 harmonic,
// 2 biharmonic).  work: pivb_infill_work_bytes(N, ny, nx) bytes.
PIV_EXPORT int pivb_infill_dev(float *ux, float *uy, const unsigned char *invalid, const float *mask, int N, int ny,
                               int nx, float spacing_y, float spacing_x, int order, int max_iter, double tol,
                               void *work, size_t work_bytes, void *stream)
{
    if (N <= 0 || ny <= 0 || nx <= 0 || !(spacing_y > 0.0f) || !(spacing_x > 0.0f)) return 1;
    if (order != 1 && order != 2) return 1;
    if (work == nullptr || work_bytes < pivb_infill_work_bytes(N, ny, nx)) return 1;
    LsqParams p{};
    p.ux = ux; p.uy = uy; p.invalid = invalid; p.mask = mask;
    p.ny = ny; p.nx = nx; p.order = order; p.max_iter = max_iter;
    p.w2y = 1.0 / pow((double)spacing_y, 2.0 * order);
    p.w2x = 1.0 / pow((double)spacing_x, 2.0 * order);
    p.tol2 = tol * tol;
    p.work = static_cast<char *>(work);
    p.work_stride = lsq_pair_bytes(ny, nx);
    if (order == 1) lsq_infill_kernel<1><<<N, kLsqThreads, 0, (cudaStream_t)stream>>>(p);
    else lsq_infill_kernel<2><<<N, kLsqThreads, 0, (cudaStream_t)stream>>>(p);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// Padding onto the predictor grid and optional Gaussian smoothing.  taps
// (2*radius+1, device) are the normalised kernel; radius 0 skips smoothing.
// work: N*nyp*nxp floats.
PIV_EXPORT int pivb_pad_smooth_dev(const float *ux, const float *uy, int N, int ny, int nx, int nyp, int nxp,
                                   int pre_y, int pre_x, const float *taps, int radius, float *pdy, float *pdx,
                                   float *work, void *stream)
{
    if (N <= 0 || ny <= 0 || nx <= 0 || nyp < ny || nxp < nx) return 1;
    cudaStream_t s = (cudaStream_t)stream;
    const long long n = (long long)N * nyp * nxp;
    pad_kernel<<<blocks(n, 256), 256, 0, s>>>(ux, uy, N, ny, nx, nyp, nxp, pre_y, pre_x, pdy, pdx);
    if (radius > 0) {
        for (float *f : {pdy, pdx}) {
            gauss_kernel<<<blocks(n, 256), 256, 0, s>>>(f, work, N, nyp, nxp, taps, radius, 1);
            gauss_kernel<<<blocks(n, 256), 256, 0, s>>>(work, f, N, nyp, nxp, taps, radius, 0);
        }
    }
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// Predictor at the next pass's window centres.
PIV_EXPORT int pivb_remap_dev(const float *pdy, const float *pdx, int N, int nyp, int nxp, const float *map_y,
                              const float *map_x, int ny, int nx, float *out_dy, float *out_dx, void *stream)
{
    if (N <= 0 || ny <= 0 || nx <= 0 || nyp <= 0 || nxp <= 0) return 1;
    const long long n = (long long)N * ny * nx;
    remap_kernel<<<blocks(n, 256), 256, 0, (cudaStream_t)stream>>>(pdy, pdx, N, nyp, nxp, map_y, map_x, ny, nx,
                                                                     out_dy, out_dx);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

namespace {
__global__ void u16_to_f32_kernel(const unsigned short *__restrict__ in, float *__restrict__ out, long long n)
{
    long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * 4;
    const long long stride = (long long)gridDim.x * blockDim.x * 4;
    for (; i + 3 < n; i += stride) {
        const ushort4 v = *reinterpret_cast<const ushort4 *>(in + i);
        *reinterpret_cast<float4 *>(out + i) = make_float4(v.x, v.y, v.z, v.w);
    }
    for (; i < n; ++i) out[i] = (float)in[i];   // tail (n not a multiple of 4)
}
}  // namespace

// uint16 camera frames -> float32, as the reference's image readers convert them
// (pivtools_core/image_handling/load_images.py:594,625).  in must be 8-byte and out
// 16-byte aligned.
PIV_EXPORT int pivb_u16_to_f32_dev(const unsigned short *in, float *out, long long n, void *stream)
{
    if (n <= 0 || !in || !out) return 1;
    if (((uintptr_t)in & 7) || ((uintptr_t)out & 15)) return 1;
    const long long quads = (n + 3) / 4;
    unsigned blocks = (unsigned)((quads + 255) / 256);
    if (blocks > 148u * 32u) blocks = 148u * 32u;
    u16_to_f32_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(in, out, n);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// ---------------------------------------------------------------------------
// LaVision pixel payloads -> float32 frames
// ---------------------------------------------------------------------------
namespace {

// Pixel p of one payload in encoding enc (the .set decoders of
// pivtools_core/image_handling/readers/set_reader.py:1196-1447 and the .im7
// WORD/FLOAT buffers of im7_reader.py:216-226), as raw sensor counts.
__device__ __forceinline__ float payload_pixel(const unsigned char *__restrict__ f, long long p, int enc)
{
    switch (enc) {
    case 0: {                                            // raw-16-bit / .im7 WORD: little-endian uint16
        const unsigned char *b = f + 2 * p;
        return (float)((unsigned)b[0] | ((unsigned)b[1] << 8));
    }
    case 1: return (float)f[p];                          // raw-8-bit: widened, not rescaled
    case 2: case 3: case 4: {                            // 2 pixels in 3 bytes
        const unsigned char *b = f + 3 * (p >> 1);
        const unsigned b0 = b[0], b1 = b[1], b2 = b[2];
        unsigned v;
        if (enc == 2) v = (p & 1) ? ((b1 >> 4) | (b2 << 4)) : (b0 | ((b1 & 0x0Fu) << 8));          // mono-12p
        else if (enc == 3) v = (p & 1) ? (((b1 & 0x0Fu) << 8) | b2) : ((b0 << 4) | (b1 >> 4));    // mono-12pmsb
        else v = (p & 1) ? ((b2 << 4) | (b1 >> 4)) : ((b0 << 4) | (b1 & 0x0Fu));                  // mono-12packed
        return (float)v;
    }
    case 5: case 6: {                                    // 4 pixels in 5 bytes
        const unsigned char *b = f + 5 * (p >> 2);
        const int j = (int)(p & 3);
        const unsigned c0 = b[j], c1 = b[j + 1];
        unsigned v;
        if (enc == 5) {                                  // mono-10p: little-endian bit stream
            const unsigned w = c0 | (c1 << 8);
            v = (w >> (2 * j)) & 0x3FFu;
        } else {                                         // mono-10pmsb: big-endian bit stream
            const unsigned w = (c0 << 8) | c1;
            v = (w >> (6 - 2 * j)) & 0x3FFu;
        }
        return (float)v;
    }
    default: {                                           // .im7 FLOAT: little-endian float32
        float v;
        memcpy(&v, f + 4 * p, 4);
        return v;
    }
    }
}

__global__ void unpack_pixels_kernel(const unsigned char *__restrict__ payload, long long payload_stride, int n_frames,
                                     long long npix, int enc, int use_slope, float slope, int use_offset, float offset,
                                     float *__restrict__ out, long long out_stride)
{
    const long long total = npix * n_frames;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(i / npix);
        const long long p = i - (long long)k * npix;
        float v = payload_pixel(payload + (long long)k * payload_stride, p, enc);
        if (use_slope) v = __fmul_rn(v, slope);
        if (use_offset) v = __fadd_rn(v, offset);
        out[(long long)k * out_stride + p] = v;
    }
}

}  // namespace

// Bytes of one payload of npix pixels in encoding enc, or -1 for an unknown
// encoding or a pixel count the packing cannot hold.
PIV_EXPORT long long pivb_payload_bytes(long long npix, int enc)
{
    if (npix <= 0) return -1;
    switch (enc) {
    case 0: return 2 * npix;
    case 1: return npix;
    case 2: case 3: case 4: return (npix & 1) ? -1 : npix / 2 * 3;
    case 5: case 6: return (npix & 3) ? -1 : npix / 4 * 5;
    case 7: return 4 * npix;
    default: return -1;
    }
}

// Unpack n_frames LaVision pixel payloads (encoding: 0 raw-16-bit or .im7 WORD,
// 1 raw-8-bit, 2 mono-12p, 3 mono-12pmsb, 4 mono-12packed, 5 mono-10p,
// 6 mono-10pmsb, 7 .im7 FLOAT) into float32 frames of npix pixels, applying the
// intensity scale as the readers do in float32 (v * slope if use_slope, then
// + offset if use_offset; im7_reader.py:1148-1152).  payload_stride: bytes between
// payloads; out_stride: elements between output frames.  Returns 0, or 1 for bad
// arguments.
PIV_EXPORT int pivb_unpack_pixels_dev(const unsigned char *payload, long long payload_stride, int n_frames,
                                      long long npix, int encoding, int use_slope, float slope, int use_offset,
                                      float offset, float *out, long long out_stride, void *stream)
{
    if (!payload || !out || n_frames <= 0) return 1;
    const long long bytes = pivb_payload_bytes(npix, encoding);
    if (bytes < 0 || payload_stride < bytes || out_stride < npix) return 1;
    const long long total = npix * n_frames;
    const long long want = (total + 255) / 256;
    const unsigned grid = (unsigned)(want < 148 * 32 ? want : 148 * 32);
    unpack_pixels_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(payload, payload_stride, n_frames, npix, encoding,
                                                                  use_slope, slope, use_offset, offset, out,
                                                                  out_stride);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// ---------------------------------------------------------------------------
// Ensemble pass: frame sums and the finalise of the accumulated planes
// (pivtools_cli/piv/piv_backend/single_pass_accumulator.py:292-320, 508-800)
// ---------------------------------------------------------------------------
namespace {

// sum[p] += sum_k frames[k][p] with a Kahan compensation term per pixel.
__global__ void frame_sum_kernel(const float *__restrict__ frames, long long stride, int n_frames, long long npix,
                                 float *__restrict__ sum, float *__restrict__ comp)
{
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < npix;
         p += (long long)gridDim.x * blockDim.x) {
        float s = sum[p], c = comp[p];
        for (int k = 0; k < n_frames; ++k) {
            const float y = __ldg(frames + (long long)k * stride + p) - c;
            const float t = s + y;
            c = (t - s) - y;
            s = t;
        }
        sum[p] = s;
        comp[p] = c;
    }
}

__global__ void frame_mean_kernel(const float *__restrict__ sum, long long npix, float n, float *__restrict__ out)
{
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < npix;
         p += (long long)gridDim.x * blockDim.x)
        out[p] = sum[p] / n;
}

// dst[k] = src[k] - mean for n frames: one float32 subtraction per pixel, the
// reference's in-place `images -= A_mean` of the 'image' background methods
// (cpu_ensemble.py:1290-1291).  dst may equal src.
__global__ void center_frames_kernel(const float *src, long long src_stride, int n_frames, long long npix,
                                     const float *__restrict__ mean, float *dst, long long dst_stride)
{
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < npix;
         p += (long long)gridDim.x * blockDim.x) {
        const float m = __ldg(mean + p);
        for (int k = 0; k < n_frames; ++k) dst[(long long)k * dst_stride + p] = src[(long long)k * src_stride + p] - m;
    }
}

struct FinParams {
    const float *sum_ab, *sum_aa, *sum_bb;     // (n_win, h, w) accumulated sums
    const float *bg_ab, *bg_aa, *bg_bb;        // background planes or null
    const float *env_auto, *env_ab;            // (h, w) envelopes or null
    float n_pairs;
    int n_win, hw, centre, dc_zero;
    double *out_aa, *out_bb, *out_ab;          // normalised planes for the k-space fit
    float *norm;                               // (n_win) normalisation factors, nullable
    float ab_scale;                            // single mode: sum area / particle area, else 1
};

// One warp per window; float32 arithmetic in the reference's order.
__global__ void ensemble_finalize_kernel(FinParams p)
{
    const int warp = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (warp >= p.n_win) return;
    const long long base = (long long)warp * p.hw;
    const float *sums[3] = {p.sum_aa, p.sum_bb, p.sum_ab};
    const float *bgs[3] = {p.bg_aa, p.bg_bb, p.bg_ab};
    double *outs[3] = {p.out_aa, p.out_bb, p.out_ab};
    float centre[3] = {0.0f, 0.0f, 0.0f};
    // pass 1: mean of each plane (after averaging and background), and its centre value
    float mean[3] = {0.0f, 0.0f, 0.0f};
    for (int q = 0; q < 3; ++q) {
        float acc = 0.0f;
        for (int k = lane; k < p.hw; k += 32) {
            float v = sums[q][base + k] / p.n_pairs;
            if (bgs[q]) v = v - bgs[q][base + k];
            acc += v;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        mean[q] = p.dc_zero ? acc / (float)p.hw : 0.0f;
        float c = sums[q][base + p.centre] / p.n_pairs;
        if (bgs[q]) c = c - bgs[q][base + p.centre];
        if (p.dc_zero) c = c - mean[q];
        const float *env = q < 2 ? p.env_auto : p.env_ab;
        if (env) c = c / env[p.centre];
        centre[q] = c;
    }
    const float nf = sqrtf(fmaxf(centre[0] * centre[1], 1e-12f));
    if (p.norm && lane == 0) p.norm[warp] = nf;
    for (int q = 0; q < 3; ++q) {
        const float *env = q < 2 ? p.env_auto : p.env_ab;
        for (int k = lane; k < p.hw; k += 32) {
            float v = sums[q][base + k] / p.n_pairs;
            if (bgs[q]) v = v - bgs[q][base + k];
            if (p.dc_zero) v = v - mean[q];
            if (env) v = v / env[k];
            if (q == 2 && p.ab_scale != 1.0f) v = v * p.ab_scale;     // single_pass_accumulator.py:765-780
            outs[q][base + k] = (double)(v / nf);
        }
    }
}

}  // namespace

// sum (+)= the n_frames frames (stride elements apart) of npix pixels, with a
// Kahan compensation array comp (zero it with sum).
PIV_EXPORT int pivb_frame_sum_dev(const float *frames, long long stride, int n_frames, long long npix, float *sum,
                                  float *comp, void *stream)
{
    if (n_frames <= 0 || npix <= 0 || stride < npix || !frames || !sum || !comp) return 1;
    const long long want = (npix + 255) / 256;
    const unsigned grid = (unsigned)(want < 148 * 16 ? want : 148 * 16);
    frame_sum_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(frames, stride, n_frames, npix, sum, comp);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// out = sum / n (the mean frame of n accumulated pairs).
PIV_EXPORT int pivb_frame_mean_dev(const float *sum, long long npix, int n, float *out, void *stream)
{
    if (n <= 0 || npix <= 0 || !sum || !out) return 1;
    const long long want = (npix + 255) / 256;
    const unsigned grid = (unsigned)(want < 148 * 16 ? want : 148 * 16);
    frame_mean_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(sum, npix, (float)n, out);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// Mean-image subtraction of the two-sweep 'image' background methods: dst frame
// k = src frame k - mean, n_frames frames of npix pixels at the given strides
// (in place when dst == src; otherwise the ranges must not overlap).
PIV_EXPORT int pivb_center_frames_dev(const float *src, long long src_stride, int n_frames, long long npix,
                                      const float *mean, float *dst, long long dst_stride, void *stream)
{
    if (n_frames <= 0 || npix <= 0 || src_stride < npix || dst_stride < npix || !src || !mean || !dst) return 1;
    if (dst == src && dst_stride != src_stride) return 1;
    const long long want = (npix + 255) / 256;
    const unsigned grid = (unsigned)(want < 148 * 16 ? want : 148 * 16);
    center_frames_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(src, src_stride, n_frames, npix, mean, dst,
                                                                 dst_stride);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// Zero-padded copies of n frames for ensemble single mode
// (window_utils.py:466-525, apply_single_mode_padding with pad value 0): dst frame
// k (Hp x Wp) holds src frame k (H x W, minus the mean frame when mean is given,
// the 'image' methods' subtraction that precedes the padding) at (pad_top,
// pad_left) and zeros elsewhere.
__global__ void pad_frames_kernel(const float *__restrict__ src, long long src_stride, int n_frames, int H, int W,
                                  const float *__restrict__ mean, int pad_top, int pad_left, float *__restrict__ dst,
                                  int Hp, int Wp, long long dst_stride)
{
    const long long npix = (long long)Hp * Wp;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < npix;
         q += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(q / Wp) - pad_top, c = (int)(q % Wp) - pad_left;
        const bool in = r >= 0 && r < H && c >= 0 && c < W;
        const long long s = (long long)r * W + c;
        const float m = (in && mean) ? __ldg(mean + s) : 0.0f;
        for (int k = 0; k < n_frames; ++k)
            dst[(long long)k * dst_stride + q] = in ? (mean ? src[(long long)k * src_stride + s] - m
                                                            : src[(long long)k * src_stride + s])
                                                    : 0.0f;
    }
}

PIV_EXPORT int pivb_pad_frames_dev(const float *src, long long src_stride, int n_frames, int H, int W,
                                   const float *mean, int pad_top, int pad_left, float *dst, int Hp, int Wp,
                                   long long dst_stride, void *stream)
{
    if (n_frames <= 0 || H <= 0 || W <= 0 || pad_top < 0 || pad_left < 0 || !src || !dst) return 1;
    if (Hp < H + pad_top || Wp < W + pad_left || src_stride < (long long)H * W || dst_stride < (long long)Hp * Wp)
        return 1;
    const long long want = ((long long)Hp * Wp + 255) / 256;
    const unsigned grid = (unsigned)(want < 148 * 16 ? want : 148 * 16);
    pad_frames_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(src, src_stride, n_frames, H, W, mean, pad_top,
                                                              pad_left, dst, Hp, Wp, dst_stride);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// Finalise of one ensemble pass for n_win windows of h x w planes: average the
// sums over n_pairs, subtract the background planes (nullable), optionally zero
// each plane's mean, divide by the envelopes (nullable), normalise by
// sqrt(max(AA_c BB_c, 1e-12)) at the centre (h/2, w/2), and write the planes in
// FP64 for the k-space fit.  norm (nullable) receives the factors.
PIV_EXPORT int pivb_ensemble_finalize_dev(const float *sum_ab, const float *sum_aa, const float *sum_bb,
                                          const float *bg_ab, const float *bg_aa, const float *bg_bb, int n_pairs,
                                          int n_win, int h, int w, int dc_zero, const float *env_auto,
                                          const float *env_ab, double *out_ab, double *out_aa, double *out_bb,
                                          float *norm, float ab_scale, void *stream)
{
    if (n_pairs <= 0 || n_win <= 0 || h <= 0 || w <= 0) return 1;
    if (!sum_ab || !sum_aa || !sum_bb || !out_ab || !out_aa || !out_bb) return 1;
    if ((bg_ab == nullptr) != (bg_aa == nullptr) || (bg_aa == nullptr) != (bg_bb == nullptr)) return 1;
    if (!(ab_scale > 0.0f) || !isfinite(ab_scale)) return 1;
    FinParams p{sum_ab, sum_aa, sum_bb, bg_ab, bg_aa, bg_bb, env_auto, env_ab ? env_ab : env_auto,
                (float)n_pairs, n_win, h * w, (h / 2) * w + w / 2, dc_zero ? 1 : 0, out_aa, out_bb, out_ab, norm,
                ab_scale};
    const long long threads = (long long)n_win * 32;
    ensemble_finalize_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, (cudaStream_t)stream>>>(p);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// Coloured-floor regressor: per window the fractions fx = |x - rint(x)| of
// x = pred_dx / 2 (float32; fy likewise), the grid cell by a left search of fs,
// bilinear weights and the four-corner sum in FP64 without contraction, rounded
// through float32 (kspace_floor_psd.py:241-275, single_pass_accumulator.py:852-880).
__global__ void floor_interp_kernel(const double *fs, int nf, const double *grid, int hw, const float *pdy,
                                    const float *pdx, long long n, double *out)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const long long wdx = i / hw;
        const int k = (int)(i - wdx * hw);
        double f[2] = {0.0, 0.0};                 // fx, fy
        if (pdx) {
            const float xs = pdx[wdx] * 0.5f, ys = pdy[wdx] * 0.5f;
            f[0] = (double)fabsf(xs - rintf(xs));
            f[1] = (double)fabsf(ys - rintf(ys));
        }
        int c[2];
        double t[2];
#pragma unroll
        for (int a = 0; a < 2; ++a) {
            int j = 0;
            while (j < nf && fs[j] < f[a]) ++j;   // first fs[j] >= f
            c[a] = min(max(j - 1, 0), nf - 2);
            const double tt = (f[a] - fs[c[a]]) / (fs[c[a] + 1] - fs[c[a]]);
            t[a] = fmin(fmax(tt, 0.0), 1.0);
        }
        const double ux = __dadd_rn(1.0, -t[0]), uy = __dadd_rn(1.0, -t[1]);
        const double *g = grid + ((long long)c[1] * nf + c[0]) * hw + k;
        const long long dx = hw, dy = (long long)nf * hw;
        double s = __dmul_rn(__dmul_rn(uy, ux), g[0]);
        s = __dadd_rn(s, __dmul_rn(__dmul_rn(uy, t[0]), g[dx]));
        s = __dadd_rn(s, __dmul_rn(__dmul_rn(t[1], ux), g[dy]));
        s = __dadd_rn(s, __dmul_rn(__dmul_rn(t[1], t[0]), g[dy + dx]));
        out[i] = (double)__double2float_rn(s);
    }
}

// P_win (n_win, hw) for the k-space fit's coloured floor from the fraction grid
// P_grid (n_fracs, n_fracs, hw) [fy, fx] and the ascending fractions fs
// (n_fracs >= 2); pred_dy / pred_dx (nullable together): the pass predictor on
// the window grid, float32.  The fractions must lie in [fs[0], fs[n_fracs-1]].
PIV_EXPORT int pivb_floor_interp_dev(const double *fs, int n_fracs, const double *P_grid, int hw,
                                     const float *pred_dy, const float *pred_dx, int n_win, double *P_win,
                                     void *stream)
{
    if (!fs || !P_grid || !P_win || n_fracs < 2 || hw <= 0 || n_win <= 0) return 1;
    if ((pred_dy == nullptr) != (pred_dx == nullptr)) return 1;
    const long long n = (long long)n_win * hw;
    const unsigned nb = (unsigned)std::min<long long>((n + 255) / 256, 148LL * 16);
    floor_interp_kernel<<<nb, 256, 0, (cudaStream_t)stream>>>(fs, n_fracs, P_grid, hw, pred_dy, pred_dx, n,
                                                              P_win);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// ---------------------------------------------------------------------------
// Ingest: camera payloads -> float32 frames
// (pivtools_core/image_handling/readers/pivraw_reader.py:896-960,
//  set_reader.py:1296-1345)
// ---------------------------------------------------------------------------
namespace {

struct DecodeParams {
    const unsigned char *raw;     // frames back to back, frame k at k * stride
    long long stride;
    int n_frames, first_index;    // 1-based file index of frame 0 (its A/B role)
    int width, height;            // sensor photosites
    int format;                   // 0 Mono12p, 1 BayerRG8
    const unsigned char *dark;    // dark frames (same format), or null
    long long dark_stride;
    int dark_frames;              // 1 (time-resolved) or 2 (A, B roles)
    int rot;                      // np.rot90 turns, 0..3
    int out_h, out_w;             // output frame shape (after the rotation)
    float *out;
    long long out_stride;
};

// Photosite (y, x) of a Mono12p payload: two pixels in three bytes, LSB first.
__device__ __forceinline__ unsigned mono12p_at(const unsigned char *f, int width, int y, int x)
{
    const long long p = (long long)y * width + x;
    const unsigned char *b = f + 3 * (p >> 1);
    return (p & 1) ? ((unsigned)(b[1] >> 4) | ((unsigned)b[2] << 4)) : ((unsigned)b[0] | ((unsigned)(b[1] & 0x0F) << 8));
}

__global__ void decode_kernel(DecodeParams p)
{
    const long long npix = (long long)p.out_h * p.out_w;
    const long long total = npix * p.n_frames;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(i / npix);
        const long long o = i - (long long)k * npix;
        const int oy = (int)(o / p.out_w), ox = (int)(o - (long long)oy * p.out_w);
        // decoded image (before rotation) is dh x dw
        const int dh = p.format == 1 ? p.height / 2 : p.height, dw = p.format == 1 ? p.width / 2 : p.width;
        int sy, sx;                               // np.rot90(m, rot)[oy, ox] = m[sy, sx]
        switch (p.rot) {
        case 1: sy = ox; sx = dw - 1 - oy; break;
        case 2: sy = dh - 1 - oy; sx = dw - 1 - ox; break;
        case 3: sy = dh - 1 - ox; sx = oy; break;
        default: sy = oy; sx = ox; break;
        }
        const unsigned char *f = p.raw + (long long)k * p.stride;
        const unsigned char *d = nullptr;
        if (p.dark) {
            const int role = p.dark_frames == 2 ? (p.first_index + k - 1) % 2 : 0;
            d = p.dark + (long long)role * p.dark_stride;
        }
        float v;
        if (p.format == 0) {
            unsigned a = mono12p_at(f, p.width, sy, sx);
            if (d) {
                const unsigned dd = mono12p_at(d, p.width, sy, sx);
                a = (a > dd ? a : dd) - dd;
            }
            v = (float)a;
        } else {
            unsigned s = 0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const long long at = (long long)(2 * sy + (q >> 1)) * p.width + 2 * sx + (q & 1);
                unsigned a = f[at];
                if (d) {
                    const unsigned dd = d[at];
                    a = (a > dd ? a : dd) - dd;
                }
                s += a;
            }
            v = (float)s;                          // at most 1020: exact
        }
        p.out[(long long)k * p.out_stride + o] = v;
    }
}

}  // namespace

// Decode n_frames camera payloads (Mono12p = format 0, BayerRG8 = format 1, as the
// PIVTOOLs Acquisition containers store them) into float32 frames: optional
// in-run dark subtraction max(frame, dark) - dark per photosite in the sensor's
// type (dark_frames 2: odd 1-based file indices take dark frame A, even ones B),
// the BayerRG8 2x2 superpixel sum R+G+G+B, and the view rotation as np.rot90 turns
// (0..3).  out_stride: elements between output frames.  Returns 0, or 1 for bad
// arguments (odd Mono12p pixel count, odd Bayer geometry, short strides).
PIV_EXPORT int pivb_decode_frames_dev(const unsigned char *raw, long long stride, int n_frames, int first_index,
                                      int width, int height, int format, const unsigned char *dark,
                                      long long dark_stride, int dark_frames, int rot, float *out,
                                      long long out_stride, void *stream)
{
    if (!raw || !out || n_frames <= 0 || width <= 0 || height <= 0 || first_index < 1) return 1;
    if (format != 0 && format != 1) return 1;
    if (rot < 0 || rot > 3) return 1;
    const long long npx = (long long)width * height;
    const long long bytes = format == 0 ? npx / 2 * 3 : npx;
    if (format == 0 && (npx & 1)) return 1;
    if (format == 1 && ((width | height) & 1)) return 1;
    if (stride < bytes) return 1;
    if (dark && (dark_stride < bytes || (dark_frames != 1 && dark_frames != 2))) return 1;
    const int dh = format == 1 ? height / 2 : height, dw = format == 1 ? width / 2 : width;
    DecodeParams p{raw, stride, n_frames, first_index, width, height, format, dark, dark_stride, dark_frames, rot,
                   (rot & 1) ? dw : dh, (rot & 1) ? dh : dw, out, out_stride};
    if (out_stride < (long long)dh * dw) return 1;
    const long long total = (long long)dh * dw * n_frames;
    const long long want = (total + 255) / 256;
    const unsigned grid = (unsigned)(want < 148 * 32 ? want : 148 * 32);
    decode_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(p);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
