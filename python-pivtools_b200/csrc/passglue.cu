// passglue.cu -- libpivb_pass: the work between multipass passes, on the GPU.
//
// The reference runs these steps in Python between its C calls
// (pivtools_cli/piv/piv_backend/cpu_instantaneous.py:559-870, :1040-1071):
//   validate  -- large-displacement gate, add the window-grid predictor, peak
//                magnitude and normalised-median outlier tests
//                (outlier_detection.py:56-84, :87-243);
//   infill    -- harmonic inpainting of invalid vectors: minimise the squared
//                gradients (physical units) over the invalid cells with the valid
//                cells held fixed and zero flux at the grid edge
//                (infilling.py:336-376), solved by Jacobi iteration;
//   pad       -- edge-replicate padding onto the padded predictor grid
//                (cpu_instantaneous.py:836-853) and the separable Gaussian
//                smoothing of scipy.ndimage.gaussian_filter(mode='nearest')
//                (cpu_instantaneous.py:1040-1048, :1140-1152);
//   remap     -- Keys-cubic (a = -0.75) interpolation of the padded predictor at
//                the next pass's window centres, replicate border
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
};

// Invalid-vector reason codes (pivtools_cli/piv/piv_backend/nan_reason_codes.py:18-25).
// The first stage that claims a vector keeps it; masked windows always read -1.
enum : signed char {
    kMasked = -1, kValid = 0, kFitFail = 1, kLargeDisp = 6, kUnclassified = 9, kOutlier = 10, kPeakMagNaN = 13
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
    const int w = (int)(i % ((long long)p.ny * p.nx));
    const bool masked = p.mask && p.mask[w] != 0.0f;
    float x = p.pk_x[i], y = p.pk_y[i], h = p.pk_h[i];
    const bool fit_fail = (x != x) || (y != y);
    const bool large = fabsf(x) > p.thresh_x || fabsf(y) > p.thresh_y;   // false for NaN
    if (masked || large) { x = qnanf(); y = qnanf(); h = qnanf(); }
    if (p.pred_dx) { x += p.pred_dx[i]; y += p.pred_dy[i]; }
    const bool pk_fail = p.peak_thr >= 0.0f && ((h < p.peak_thr) || (h != h));
    bool bad = (x != x) || (y != y) || pk_fail || (h != h);
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
    const bool outlier = (nr > p.med_thr) || !isfinite(nr) || present < 6;
    const bool bad = p.invalid[i] || outlier;
    p.invalid[i] = bad ? 1 : 0;
    p.ux[i] = bad ? qnanf() : X[w];
    p.uy[i] = bad ? qnanf() : Y[w];
    if (p.reason) {
        signed char rc = p.reason[i];
        if (rc == kValid && outlier) rc = kOutlier;
        if (rc == kValid && bad) rc = (p.pk_h[i] != p.pk_h[i]) ? kPeakMagNaN : kUnclassified;
        p.reason[i] = rc;
    }
}

// Harmonic inpainting: one CTA per pair, Jacobi sweeps over the invalid cells.
// Weights 1/dx^2 (x neighbours) and 1/dy^2 (y neighbours); neighbours outside
// the grid or masked drop out (zero flux).  Cells start from the mean of the
// pair's valid vectors; iteration stops at max_iter or when the largest update
// is below tol (px).  The invalid cells are listed once in shared memory (any
// order: a Jacobi sweep's updates are independent) so that a sweep touches only
// them; grids with more invalid cells than the list holds sweep the whole grid.
constexpr int kInfillList = 6144;

__device__ __forceinline__ void infill_cell(int w, int ny, int nx, float wy, float wx, const float *mask,
                                            const float *sx, const float *sy, float *dx, float *dy, float &local)
{
    const int r = w / nx, c = w % nx;
    float su = 0.0f, sv = 0.0f, sw = 0.0f;
    const int nr[4] = {r - 1, r + 1, r, r};
    const int nc[4] = {c, c, c - 1, c + 1};
    const float ww[4] = {wy, wy, wx, wx};
    for (int k = 0; k < 4; ++k) {
        if (nr[k] < 0 || nr[k] >= ny || nc[k] < 0 || nc[k] >= nx) continue;
        const int q = nr[k] * nx + nc[k];
        if (mask && mask[q] != 0.0f) continue;
        su += ww[k] * sx[q];
        sv += ww[k] * sy[q];
        sw += ww[k];
    }
    const float nu = sw > 0.0f ? su / sw : sx[w], nv = sw > 0.0f ? sv / sw : sy[w];
    local = fmaxf(local, fmaxf(fabsf(nu - sx[w]), fabsf(nv - sy[w])));
    dx[w] = nu;
    dy[w] = nv;
}

__global__ void __launch_bounds__(512) infill_kernel(float *ux, float *uy, const unsigned char *invalid,
                                                     const float *mask, int ny, int nx, float wy, float wx,
                                                     int max_iter, float tol, float *work)
{
    const int n = blockIdx.x;
    const int plane = ny * nx;
    float *X = ux + (long long)n * plane, *Y = uy + (long long)n * plane;
    const unsigned char *bad = invalid + (long long)n * plane;
    float *X2 = work + (long long)n * 2 * plane, *Y2 = X2 + plane;
    __shared__ float s_max;
    __shared__ int s_cnt;
    __shared__ int s_list[kInfillList];
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();
    for (int w = threadIdx.x; w < plane; w += blockDim.x)
        if (bad[w]) {
            const int k = atomicAdd(&s_cnt, 1);
            if (k < kInfillList) s_list[k] = w;
        }
    __syncthreads();
    const int n_bad = s_cnt;
    if (n_bad == 0) return;
    const bool listed = n_bad <= kInfillList;
    // initial guess: mean of the valid vectors (the iteration converges to the
    // unique harmonic solution from any start; a good start shortens it)
    // deterministic block reduction (fixed order), so repeated runs agree bit for bit
    __shared__ float s_part[3][16];
    __shared__ float s_su, s_sv, s_n;
    {
        float su = 0.0f, sv = 0.0f, cnt = 0.0f;
        for (int w = threadIdx.x; w < plane; w += blockDim.x)
            if (!bad[w] && !(mask && mask[w] != 0.0f)) { su += X[w]; sv += Y[w]; cnt += 1.0f; }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            su += __shfl_xor_sync(0xffffffffu, su, o);
            sv += __shfl_xor_sync(0xffffffffu, sv, o);
            cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        }
        if ((threadIdx.x & 31) == 0) {
            s_part[0][threadIdx.x >> 5] = su;
            s_part[1][threadIdx.x >> 5] = sv;
            s_part[2][threadIdx.x >> 5] = cnt;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            float a = 0.0f, b = 0.0f, c = 0.0f;
            for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { a += s_part[0][k]; b += s_part[1][k]; c += s_part[2][k]; }
            s_su = a; s_sv = b; s_n = c;
        }
    }
    __syncthreads();
    const float mu = s_n > 0.0f ? s_su / s_n : 0.0f, mv = s_n > 0.0f ? s_sv / s_n : 0.0f;
    for (int w = threadIdx.x; w < plane; w += blockDim.x) {
        if (bad[w]) { X[w] = mu; Y[w] = mv; }
        X2[w] = X[w];
        Y2[w] = Y[w];
    }
    __syncthreads();
    for (int it = 0; it < max_iter; ++it) {
        if (threadIdx.x == 0) s_max = 0.0f;
        __syncthreads();
        float local = 0.0f;
        // valid cells are equal in both buffers and never change
        const float *sx = (it & 1) ? X2 : X, *sy = (it & 1) ? Y2 : Y;
        float *dx = (it & 1) ? X : X2, *dy = (it & 1) ? Y : Y2;
        if (listed) {
            for (int i = threadIdx.x; i < n_bad; i += blockDim.x)
                infill_cell(s_list[i], ny, nx, wy, wx, mask, sx, sy, dx, dy, local);
        } else {
            for (int w = threadIdx.x; w < plane; w += blockDim.x)
                if (bad[w]) infill_cell(w, ny, nx, wy, wx, mask, sx, sy, dx, dy, local);
        }
        atomicMax(reinterpret_cast<int *>(&s_max), __float_as_int(local));   // local >= 0
        __syncthreads();
        const bool done = s_max < tol;
        __syncthreads();
        if (done || it == max_iter - 1) {
            if (!(it & 1)) {   // result is in X2/Y2
                if (listed) {
                    for (int i = threadIdx.x; i < n_bad; i += blockDim.x) {
                        const int w = s_list[i];
                        X[w] = X2[w];
                        Y[w] = Y2[w];
                    }
                } else {
                    for (int w = threadIdx.x; w < plane; w += blockDim.x) { X[w] = X2[w]; Y[w] = Y2[w]; }
                }
            }
            break;
        }
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

__device__ __forceinline__ void keys4(float d, float *w)
{
    const float s0 = 1.0f + d, q2 = 1.0f - d, s3 = 2.0f - d;
    w[1] = (1.25f * d - 2.25f) * d * d + 1.0f;
    w[2] = (1.25f * q2 - 2.25f) * q2 * q2 + 1.0f;
    w[0] = ((-0.75f * s0 + 3.75f) * s0 - 6.0f) * s0 + 3.0f;
    w[3] = ((-0.75f * s3 + 3.75f) * s3 - 6.0f) * s3 + 3.0f;
}

// Cubic remap of both padded planes at fractional grid coordinates.
__global__ void remap_kernel(const float *pdy, const float *pdx, int N, int nyp, int nxp, const float *map_y,
                             const float *map_x, int ny, int nx, float *oy, float *ox)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)N * ny * nx) return;
    const int n = (int)(i / ((long long)ny * nx)), w = (int)(i % ((long long)ny * nx));
    const float fy = map_y[w], fx = map_x[w];
    const float fyf = floorf(fy), fxf = floorf(fx);
    float wy[4], wx[4];
    keys4(fy - fyf, wy);
    keys4(fx - fxf, wx);
    const int by = (int)fyf - 1, bx = (int)fxf - 1;
    const float *Py = pdy + (long long)n * nyp * nxp, *Px = pdx + (long long)n * nyp * nxp;
    float vy = 0.0f, vx = 0.0f;
    for (int m = 0; m < 4; ++m) {
        const int r = min(max(by + m, 0), nyp - 1);
        for (int q = 0; q < 4; ++q) {
            const int c = min(max(bx + q, 0), nxp - 1);
            const float wt = wy[m] * wx[q];
            vy += wt * Py[r * nxp + c];
            vx += wt * Px[r * nxp + c];
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
                med_thr, med_size, ux, uy, invalid, nan_reason};
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

// Harmonic infilling of the invalid vectors, in place.  work: 2*N*ny*nx floats.
PIV_EXPORT int pivb_infill_dev(float *ux, float *uy, const unsigned char *invalid, const float *mask, int N, int ny,
                               int nx, float spacing_y, float spacing_x, int max_iter, float tol, float *work,
                               void *stream)
{
    if (N <= 0 || ny <= 0 || nx <= 0 || spacing_y <= 0.0f || spacing_x <= 0.0f) return 1;
    const float wy = 1.0f / (spacing_y * spacing_y), wx = 1.0f / (spacing_x * spacing_x);
    infill_kernel<<<N, 512, 0, (cudaStream_t)stream>>>(ux, uy, invalid, mask, ny, nx, wy, wx, max_iter, tol, work);
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

struct FinParams {
    const float *sum_ab, *sum_aa, *sum_bb;     // (n_win, h, w) accumulated sums
    const float *bg_ab, *bg_aa, *bg_bb;        // background planes or null
    const float *env_auto, *env_ab;            // (h, w) envelopes or null
    float n_pairs;
    int n_win, hw, centre, dc_zero;
    double *out_aa, *out_bb, *out_ab;          // normalised planes for the k-space fit
    float *norm;                               // (n_win) normalisation factors, nullable
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

// Finalise of one ensemble pass for n_win windows of h x w planes: average the
// sums over n_pairs, subtract the background planes (nullable), optionally zero
// each plane's mean, divide by the envelopes (nullable), normalise by
// sqrt(max(AA_c BB_c, 1e-12)) at the centre (h/2, w/2), and write the planes in
// FP64 for the k-space fit.  norm (nullable) receives the factors.
PIV_EXPORT int pivb_ensemble_finalize_dev(const float *sum_ab, const float *sum_aa, const float *sum_bb,
                                          const float *bg_ab, const float *bg_aa, const float *bg_bb, int n_pairs,
                                          int n_win, int h, int w, int dc_zero, const float *env_auto,
                                          const float *env_ab, double *out_ab, double *out_aa, double *out_bb,
                                          float *norm, void *stream)
{
    if (n_pairs <= 0 || n_win <= 0 || h <= 0 || w <= 0) return 1;
    if (!sum_ab || !sum_aa || !sum_bb || !out_ab || !out_aa || !out_bb) return 1;
    if ((bg_ab == nullptr) != (bg_aa == nullptr) || (bg_aa == nullptr) != (bg_bb == nullptr)) return 1;
    FinParams p{sum_ab, sum_aa, sum_bb, bg_ab, bg_aa, bg_bb, env_auto, env_ab ? env_ab : env_auto,
                (float)n_pairs, n_win, h * w, (h / 2) * w + w / 2, dc_zero ? 1 : 0, out_aa, out_bb, out_ab, norm};
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
