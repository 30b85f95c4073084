// kspacefit.cu -- libkspacefit for sm_100a: the ensemble k-space
// Reynolds-stress Levenberg-Marquardt fit (pivtools_cli/lib/kspace_lm_fit.c),
// FP64 throughout.
//
// One warp per window.  The three correlation planes are transformed with their
// centre moved to the origin (the ifftshift load of kspace_lm_fit.c:253-286) by a
// separable FP64 DFT; lanes then own k-bins.  Per bin the transfer ratio
// T = F_AB / sqrt(|F_AA| |F_BB|), the weight F_ref / max F_ref (DC excluded) and
// the floor regressor D (1/F_ref flat, P/F_ref coloured) are kept in shared
// memory (global scratch for the largest windows).  The LM loop follows
// kspace_lm_fit.c:574-664: cost and normal equations are warp reductions over the
// bins, the damped Cholesky solve is evaluated redundantly by every lane, and the
// accept / convergence / give-up rules and the status contract
// (kspace_lm_fit.c:669-884) are the reference's.
#include <math.h>
#include <stdio.h>

#include <mutex>

#include "device_state.h"
#include "piv_common.cuh"

namespace {

constexpr int KMAX = 9;
constexpr int MAIN_MAX_ITER = 250;
constexpr double LM_XTOL = 1e-8, LM_FTOL = 1e-8;
constexpr int MIN_VALID_PTS = 10;
constexpr double MAX_DISP_FRAC = 0.75, COST_PER_PT_ACCEPT = 1.0, EXP_ARG_MAX = 300.0;
constexpr double LAM_INIT = 1e-3, LAM_MIN = 1e-12, LAM_ENOPROG = 1e12;
constexpr double GAIN_LO = 1e-3, GAIN_HI = 1e3, SIGMA_SEED_XX = 1.0, SIGMA_SEED_YY = 0.2;
constexpr double N0_HI_COLOURED = 10.0, SEED_KR_MIN = 0.35, SEED_CLIP_LO = 1e-3, SEED_CLIP_HI = 10.0;
constexpr double TWO_PI = 6.283185307179586476925286766559;
constexpr double TWO_PI2 = 2.0 * 9.869604401089358618834490999876;

bool size_ok(int n)
{
    switch (n) {
    case 8: case 12: case 16: case 24: case 32: case 48: case 64: case 96: case 128:
        return true;
    default:
        return false;
    }
}

__device__ __forceinline__ double wsum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double wmax(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ int wsumi(int v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

struct KsParams {
    const double *RAA, *RBB, *RAB;
    const unsigned char *mask;
    const double *Pw;          // centred P per window, or null (flat floor)
    int nw, H, W, ukx, uky, K;
    double *gf, *ig, *dgain, *dN0, *db4x, *db4y, *dcpp;
    int *status, *dnv, *diter;
    unsigned char *dconv;
    double *gscratch;          // per-warp-slot scratch when shared memory is too small
    int use_smem;
};

// Per-bin arrays of one warp: Fr, Tre, Tim, Wg, Dv, Pn, spectra scratch (re, im).
constexpr int PER_BIN = 8;

// Separable DFT of the centred plane: out[k] = sum_x plane[shift(x)] e^{-2 pi i k.x}.
// re/im receive the spectrum (natural order).  tmp needs 2*P doubles.
__device__ void dft_centred(const double *plane, int H, int W, const double *cw, const double *sw,
                            const double *ch, const double *sh, double *re, double *im, double *tr, double *ti)
{
    const int lane = threadIdx.x & 31, P = H * W;
    // rows: X1[r][kx] = sum_c x[r][c] e^{-2 pi i kx c / W}, x[r][c] = plane[(r+H/2)%H][(c+W/2)%W]
    for (int b = lane; b < P; b += 32) {
        const int r = b / W, kx = b % W;
        const double *src = plane + (size_t)((r + H / 2) % H) * W;
        double ar = 0.0, ai = 0.0;
        for (int c = 0; c < W; ++c) {
            const double v = src[(c + W / 2) % W];
            const int m = (kx * c) % W;
            ar += v * cw[m];
            ai -= v * sw[m];
        }
        tr[b] = ar;
        ti[b] = ai;
    }
    __syncwarp();
    for (int b = lane; b < P; b += 32) {
        const int ky = b / W, kx = b % W;
        double ar = 0.0, ai = 0.0;
        for (int r = 0; r < H; ++r) {
            const int m = (ky * r) % H;
            const double xr = tr[r * W + kx], xi = ti[r * W + kx];
            const double c = ch[m], s = sh[m];
            ar += xr * c + xi * s;     // (xr + i xi)(c - i s)
            ai += xi * c - xr * s;
        }
        re[b] = ar;
        im[b] = ai;
    }
    __syncwarp();
}

struct Bins {
    double *Fr, *Tre, *Tim, *Wg, *Dv, *Pn, *sr, *si;
};

__device__ __forceinline__ void model_bin(const double *x, int ukx, int uky, double kx, double ky, double dv,
                                          double &arg, double &att, double &phase)
{
    const double kx2 = kx * kx, ky2 = ky * ky;
    arg = -TWO_PI2 * (x[2] * kx2 + 2.0 * x[4] * kx * ky + x[3] * ky2);
    int c = 7;
    if (ukx) arg -= x[c++] * kx2 * kx2;
    if (uky) arg -= x[c] * ky2 * ky2;
    if (arg > EXP_ARG_MAX) arg = EXP_ARG_MAX;
    att = 1.0 - x[6] * dv;
    phase = -TWO_PI * (kx * x[0] + ky * x[1]);
}

__device__ double cost_eval(const Bins &B, const double *x, const KsParams &p, const double *kxv,
                            const double *kyv)
{
    const int lane = threadIdx.x & 31, P = p.H * p.W;
    double cost = 0.0;
    for (int b = lane; b < P; b += 32) {
        const double w = B.Wg[b];
        if (w == 0.0) continue;
        double arg, att, ph;
        model_bin(x, p.ukx, p.uky, kxv[b % p.W], kyv[b / p.W], B.Dv[b], arg, att, ph);
        double sp, cp;
        sincos(ph, &sp, &cp);
        const double gd = x[5] * exp(arg) * att;
        const double rr = w * (B.Tre[b] - gd * cp), ri = w * (B.Tim[b] - gd * sp);
        cost += rr * rr + ri * ri;
    }
    return wsum(cost);
}

// Normal equations (upper triangle, K x K) and gradient, reduced over the warp.
__device__ void jtj_eval(const Bins &B, const double *x, const KsParams &p, const double *kxv, const double *kyv,
                         double *A, double *g)
{
    const int lane = threadIdx.x & 31, P = p.H * p.W, K = p.K;
    double a[KMAX * (KMAX + 1) / 2], gv[KMAX];
#pragma unroll
    for (int i = 0; i < KMAX * (KMAX + 1) / 2; ++i) a[i] = 0.0;
#pragma unroll
    for (int i = 0; i < KMAX; ++i) gv[i] = 0.0;
    for (int b = lane; b < P; b += 32) {
        const double w = B.Wg[b];
        if (w == 0.0) continue;
        const double kx = kxv[b % p.W], ky = kyv[b / p.W];
        const double kx2 = kx * kx, ky2 = ky * ky, kxky = kx * ky;
        double arg, att, ph;
        const double dv = B.Dv[b];
        model_bin(x, p.ukx, p.uky, kx, ky, dv, arg, att, ph);
        double sp, cp;
        sincos(ph, &sp, &cp);
        const double dec = exp(arg);
        const double gd = x[5] * dec * att;
        const double rr = w * (B.Tre[b] - gd * cp), ri = w * (B.Tim[b] - gd * sp);
        double Jr[KMAX], Ji[KMAX];
        const double dpx = -TWO_PI * kx, dpy = -TWO_PI * ky;
        Jr[0] = -w * gd * (-sp) * dpx; Ji[0] = -w * gd * cp * dpx;
        Jr[1] = -w * gd * (-sp) * dpy; Ji[1] = -w * gd * cp * dpy;
        const double d2 = gd * (-TWO_PI2 * kx2);
        Jr[2] = -w * d2 * cp; Ji[2] = -w * d2 * sp;
        const double d3 = gd * (-TWO_PI2 * ky2);
        Jr[3] = -w * d3 * cp; Ji[3] = -w * d3 * sp;
        const double d4 = gd * (-TWO_PI2 * 2.0 * kxky);
        Jr[4] = -w * d4 * cp; Ji[4] = -w * d4 * sp;
        Jr[5] = -w * dec * att * cp; Ji[5] = -w * dec * att * sp;
        const double dn = x[5] * dec * (-dv);
        Jr[6] = -w * dn * cp; Ji[6] = -w * dn * sp;
        int cc = 7;
        if (p.ukx) { const double db = gd * (-(kx2 * kx2)); Jr[cc] = -w * db * cp; Ji[cc] = -w * db * sp; ++cc; }
        if (p.uky) { const double db = gd * (-(ky2 * ky2)); Jr[cc] = -w * db * cp; Ji[cc] = -w * db * sp; }
        int t = 0;
#pragma unroll
        for (int i = 0; i < KMAX; ++i) {
            if (i < K) gv[i] += Jr[i] * rr + Ji[i] * ri;
#pragma unroll
            for (int j = i; j < KMAX; ++j, ++t)
                if (i < K && j < K) a[t] += Jr[i] * Jr[j] + Ji[i] * Ji[j];
        }
    }
    int t = 0;
#pragma unroll
    for (int i = 0; i < KMAX; ++i) {
        g[i] = wsum(gv[i]);
#pragma unroll
        for (int j = i; j < KMAX; ++j, ++t) {
            const double v = wsum(a[t]);
            if (i < K && j < K) { A[i * K + j] = v; A[j * K + i] = v; }
        }
    }
}

// Cholesky solve of the damped system (kspace_lm_fit.c:535-562); -1 if not PD.
__device__ int chol_solve(int K, const double *M, const double *b, double *d)
{
    double L[KMAX * KMAX], y[KMAX];
    for (int i = 0; i < K; ++i)
        for (int j = 0; j <= i; ++j) {
            double s = M[i * K + j];
            for (int k = 0; k < j; ++k) s -= L[i * K + k] * L[j * K + k];
            if (i == j) {
                if (s <= 0.0 || !isfinite(s)) return -1;
                L[i * K + i] = sqrt(s);
            } else {
                L[i * K + j] = s / L[j * K + j];
            }
        }
    for (int i = 0; i < K; ++i) {
        double s = b[i];
        for (int k = 0; k < i; ++k) s -= L[i * K + k] * y[k];
        y[i] = s / L[i * K + i];
    }
    for (int i = K - 1; i >= 0; --i) {
        double s = y[i];
        for (int k = i + 1; k < K; ++k) s -= L[k * K + i] * d[k];
        d[i] = s / L[i * K + i];
    }
    return 0;
}

// Median of v[0..n) (np.median convention) by rank selection across the warp;
// v is read-only.  Ties are ranked by index.
__device__ double warp_median(const double *v, int n)
{
    const int lane = threadIdx.x & 31;
    const int want_lo = (n - 1) / 2, want_hi = n / 2;
    double lo = 0.0, hi = 0.0;
    bool got_lo = false, got_hi = false;
    for (int i = lane; i < n; i += 32) {
        const double vi = v[i];
        int rank = 0;
        for (int j = 0; j < n; ++j) {
            const double vj = v[j];
            rank += (vj < vi) || (vj == vi && j < i);
        }
        if (rank == want_lo) { lo = vi; got_lo = true; }
        if (rank == want_hi) { hi = vi; got_hi = true; }
    }
    const unsigned ml = __ballot_sync(0xffffffffu, got_lo), mh = __ballot_sync(0xffffffffu, got_hi);
    lo = __shfl_sync(0xffffffffu, lo, __ffs(ml) - 1);
    hi = __shfl_sync(0xffffffffu, hi, __ffs(mh) - 1);
    return (n & 1) ? hi : 0.5 * (lo + hi);
}

__device__ double sub3(double lo, double ce, double hi)
{
    if (lo <= 0.0 || ce <= 0.0 || hi <= 0.0) return 0.0;
    const double l = log(lo), c = log(ce), r = log(hi);
    const double den = 2.0 * (l - 2.0 * c + r);
    if (fabs(den) <= 1e-12) return 0.0;
    return (l - r) / den;
}

// Output defaults for every window (kspace_lm_fit.c:725-752).
__global__ void init_kernel(KsParams p, const int *n_proc)
{
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= p.nw) return;
    const double cxc = p.W / 2.0 + 1.0, cyc = p.H / 2.0 + 1.0;
    const double qnan = __longlong_as_double(0x7ff8000000000000LL);
    double *gf = p.gf + (size_t)w * 16, *ig = p.ig + (size_t)w * 16;
    for (int c = 0; c < 16; ++c) { gf[c] = 0.0; ig[c] = 0.0; }
    gf[6] = gf[7] = gf[8] = qnan;
    gf[12] = cxc; gf[13] = cyc; gf[14] = cxc; gf[15] = cyc;
    if (*n_proc == 0 || !p.mask[w]) {
        ig[6] = ig[7] = ig[8] = qnan;
        ig[12] = cxc; ig[13] = cyc; ig[14] = cxc; ig[15] = cyc;
    }
    p.status[w] = -1;
    p.dgain[w] = p.dN0[w] = p.db4x[w] = p.db4y[w] = p.dcpp[w] = qnan;
    p.dnv[w] = 0; p.diter[w] = 0; p.dconv[w] = 0;
}

__global__ void count_kernel(const unsigned char *mask, int n, int *n_proc)
{
    int c = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) c += !mask[i];
    c = wsumi(c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(n_proc, c);
}

__global__ void __launch_bounds__(128) fit_kernel(KsParams p, int warps_per_cta)
{
    extern __shared__ double sm[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;   // blockDim.x == 32 * warps_per_cta
    const int H = p.H, W = p.W, P = H * W, K = p.K;
    // per-CTA tables: twiddles and k grids
    double *cw = sm, *sw = cw + W, *ch = sw + W, *sh = ch + H, *kxv = sh + H, *kyv = kxv + W;
    double *per_warp = kyv + H;
    if (threadIdx.x < 32) {
        for (int m = lane; m < W; m += 32) {
            double s, c;
            sincospi(2.0 * m / W, &s, &c);
            cw[m] = c; sw[m] = s;
            kxv[m] = (m < (W + 1) / 2 ? (double)m : (double)(m - W)) / (double)W;
        }
        for (int m = lane; m < H; m += 32) {
            double s, c;
            sincospi(2.0 * m / H, &s, &c);
            ch[m] = c; sh[m] = s;
            kyv[m] = (m < (H + 1) / 2 ? (double)m : (double)(m - H)) / (double)H;
        }
    }
    __syncthreads();
    const long long slot = (long long)blockIdx.x * warps_per_cta + wid;
    double *base = p.use_smem ? per_warp + (size_t)wid * PER_BIN * P : p.gscratch + (size_t)slot * PER_BIN * P;
    Bins B{base, base + P, base + 2 * P, base + 3 * P, base + 4 * P, base + 5 * P, base + 6 * P, base + 7 * P};
    const int cy = H / 2, cx = W / 2;
    const double cxc = W / 2.0 + 1.0, cyc = H / 2.0 + 1.0;
    double lo[KMAX], hi[KMAX];
    for (int i = 0; i < KMAX; ++i) { lo[i] = -INFINITY; hi[i] = INFINITY; }
    lo[2] = 0.0; lo[3] = 0.0; lo[5] = GAIN_LO; hi[5] = GAIN_HI; lo[6] = 0.0;
    hi[6] = p.Pw ? N0_HI_COLOURED : INFINITY;
    const long long nslots = (long long)gridDim.x * warps_per_cta;

    for (long long w = slot; w < p.nw; w += nslots) {
        if (p.mask[w]) continue;
        double *gf = p.gf + w * 16, *ig = p.ig + w * 16;
        const double *aa = p.RAA + w * P, *bb = p.RBB + w * P, *ab = p.RAB + w * P;
        // amplitudes and the peak-mu seed from the raw AB plane (first-occurrence argmax)
        double best = ab[0];
        int bi = 0;
        bool nan = false;
        for (int i = lane; i < P; i += 32) {
            const double v = ab[i];
            nan |= (v != v);
            if (v > best || (v == best && i < bi)) { best = v; bi = i; }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ob = __shfl_xor_sync(0xffffffffu, best, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
        }
        if (__any_sync(0xffffffffu, nan)) {   // exact scan semantics
            best = ab[0];
            bi = 0;
            for (int i = 1; i < P; ++i)
                if (ab[i] > best) { best = ab[i]; bi = i; }
        }
        const double ampA = aa[cy * W + cx], ampB = bb[cy * W + cx], ampAB = best;
        const bool amp_ok = ampA >= 1e-12 && ampB >= 1e-12;
        double seed[KMAX];
        for (int i = 0; i < KMAX; ++i) seed[i] = 0.0;
        {
            const int py = bi / W, px = bi % W;
            double sx = 0.0, sy = 0.0;
            if (px > 0 && px < W - 1) sx = sub3(ab[py * W + px - 1], ab[py * W + px], ab[py * W + px + 1]);
            if (py > 0 && py < H - 1) sy = sub3(ab[(py - 1) * W + px], ab[py * W + px], ab[(py + 1) * W + px]);
            seed[0] = ((double)px + sx) - (double)cx;
            seed[1] = ((double)py + sy) - (double)cy;
        }
        seed[2] = SIGMA_SEED_XX;
        seed[3] = SIGMA_SEED_YY;
        // spectra: |F_AA| -> Fr, |F_BB| -> Fr = sqrt(|AA||BB|), then T
        dft_centred(aa, H, W, cw, sw, ch, sh, B.sr, B.si, B.Tre, B.Tim);
        for (int b = lane; b < P; b += 32) B.Fr[b] = hypot(B.sr[b], B.si[b]);
        __syncwarp();
        dft_centred(bb, H, W, cw, sw, ch, sh, B.sr, B.si, B.Tre, B.Tim);
        for (int b = lane; b < P; b += 32) B.Fr[b] = sqrt(B.Fr[b] * hypot(B.sr[b], B.si[b]));
        __syncwarp();
        dft_centred(ab, H, W, cw, sw, ch, sh, B.sr, B.si, B.Tre, B.Tim);
        double frmax = 0.0;
        for (int b = lane; b < P; b += 32) {
            const double fr = B.Fr[b];
            const double inv = 1.0 / (fr > 1e-30 ? fr : 1e-30);
            B.Tre[b] = B.sr[b] * inv;
            B.Tim[b] = B.si[b] * inv;
            frmax = fmax(frmax, fr);
        }
        frmax = wmax(frmax);
        if (frmax < 1e-30) frmax = 1e-30;
        int nv = 0;
        for (int b = lane; b < P; b += 32) {
            const bool v = B.Fr[b] > 1e-12 && b != 0;
            B.Wg[b] = v ? B.Fr[b] / frmax : 0.0;
            nv += v;
        }
        nv = wsumi(nv);
        __syncwarp();
        if (lane == 0) {
            gf[0] = ig[0] = ampA;
            gf[1] = ig[1] = ampB;
            gf[2] = ig[2] = ampAB;
            ig[9] = seed[2];
            ig[10] = seed[3];
            ig[14] = cxc + seed[0];
            ig[15] = cyc + seed[1];
            p.dnv[w] = nv;
        }
        if (!amp_ok) { if (lane == 0) p.status[w] = 2; continue; }
        if (nv < MIN_VALID_PTS) { if (lane == 0) p.status[w] = 1; continue; }
        // ring-1 gain median (kspace_lm_fit.c:330-346)
        {
            double v8[8];
            int k = 0;
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    if (!dy && !dx) continue;
                    const int i = ((dy + H) % H) * W + (dx + W) % W;
                    v8[k++] = hypot(B.Tre[i], B.Tim[i]);
                }
            for (int i = 1; i < 8; ++i)
                for (int j = i; j > 0 && v8[j - 1] > v8[j]; --j) { const double t = v8[j]; v8[j] = v8[j - 1]; v8[j - 1] = t; }
            double med = 0.5 * (v8[3] + v8[4]);
            seed[5] = med < 1e-2 ? 1e-2 : (med > 10.0 ? 10.0 : med);
        }
        // floor regressor and coloured N0 seed (kspace_lm_fit.c:366-404)
        if (!p.Pw) {
            for (int b = lane; b < P; b += 32) B.Dv[b] = 1.0 / (B.Fr[b] > 1e-30 ? B.Fr[b] : 1e-30);
            __syncwarp();
        } else {
            const double *pc = p.Pw + w * P;
            for (int b = lane; b < P; b += 32) {
                const int r = b / W, c = b % W;
                const double pv = pc[((r + H / 2) % H) * W + (c + W / 2) % W];
                B.Pn[b] = pv;
                B.Dv[b] = pv / (B.Fr[b] > 1e-30 ? B.Fr[b] : 1e-30);
            }
            __syncwarp();
            // tail bins |k| >= 0.35 in natural order, compacted into sr
            int n_tail = 0;
            for (int b0 = 0; b0 < P; b0 += 32) {
                const int b = b0 + lane;
                bool in = false;
                double v = 0.0;
                if (b < P) {
                    const double kx = kxv[b % W], ky = kyv[b / W];
                    in = ky * ky + kx * kx >= SEED_KR_MIN * SEED_KR_MIN;
                    v = B.Fr[b] / (B.Pn[b] > 1e-30 ? B.Pn[b] : 1e-30);
                }
                const unsigned m = __ballot_sync(0xffffffffu, in);
                if (in) B.sr[n_tail + __popc(m & ((1u << lane) - 1u))] = v;
                n_tail += __popc(m);
            }
            __syncwarp();
            double med = warp_median(B.sr, n_tail);
            seed[6] = med < SEED_CLIP_LO ? SEED_CLIP_LO : (med > SEED_CLIP_HI ? SEED_CLIP_HI : med);
        }
        // LM (kspace_lm_fit.c:574-664)
        double x[KMAX];
        for (int i = 0; i < KMAX; ++i) {
            x[i] = seed[i];
            if (i < K) {
                if (x[i] < lo[i]) x[i] = lo[i];
                if (x[i] > hi[i]) x[i] = hi[i];
            }
        }
        double cost = cost_eval(B, x, p, kxv, kyv);
        int niter = 0, conv = 0;
        if (isfinite(cost)) {
            double lam = LAM_INIT, A[KMAX * KMAX], g[KMAX], Ad[KMAX * KMAX];
            bool have = false;
            for (int it = 0; it < MAIN_MAX_ITER; ++it) {
                if (!have) { jtj_eval(B, x, p, kxv, kyv, A, g); have = true; }
                for (int i = 0; i < K * K; ++i) Ad[i] = A[i];
                for (int i = 0; i < K; ++i) {
                    double dg = A[i * K + i];
                    if (dg < 1e-30) dg = 1e-30;
                    Ad[i * K + i] += lam * dg;
                }
                double d[KMAX], ng[KMAX], xn[KMAX];
                for (int i = 0; i < K; ++i) ng[i] = -g[i];
                for (int i = K; i < KMAX; ++i) xn[i] = x[i];
                const bool solved = chol_solve(K, Ad, ng, d) == 0;
                bool acc = false;
                double cn = INFINITY;
                if (solved) {
                    bool fin = true;
                    for (int i = 0; i < K; ++i) {
                        xn[i] = x[i] + d[i];
                        if (xn[i] < lo[i]) xn[i] = lo[i];
                        if (xn[i] > hi[i]) xn[i] = hi[i];
                        if (!isfinite(xn[i])) fin = false;
                    }
                    if (fin) {
                        cn = cost_eval(B, xn, p, kxv, kyv);
                        acc = isfinite(cn) && cn <= cost;
                    }
                }
                ++niter;
                if (acc) {
                    bool small = true;
                    for (int i = 0; i < K; ++i)
                        if (fabs(xn[i] - x[i]) > LM_XTOL * (LM_XTOL + fabs(xn[i]))) { small = false; break; }
                    const double ref = cost > 1e-300 ? cost : 1e-300;
                    const bool drop = (cost - cn) <= LM_FTOL * ref;
                    for (int i = 0; i < K; ++i) x[i] = xn[i];
                    cost = cn;
                    lam /= 3.0;
                    if (lam < LAM_MIN) lam = LAM_MIN;
                    have = false;
                    if (small || drop) { conv = 1; break; }
                } else {
                    lam *= 10.0;
                    if (lam > LAM_ENOPROG) break;
                }
            }
        }
        if (lane == 0) {
            p.diter[w] = niter;
            p.dconv[w] = (unsigned char)conv;
            const double cpp = cost / (double)nv;
            p.dcpp[w] = cpp;
            const bool fit_ok = conv || (niter >= MAIN_MAX_ITER && cpp < COST_PER_PT_ACCEPT);
            if (!fit_ok) {
                p.status[w] = 1;
            } else if (fabs(x[0]) > MAX_DISP_FRAC * W || fabs(x[1]) > MAX_DISP_FRAC * H) {
                p.status[w] = 3;
            } else {
                p.status[w] = 0;
                gf[9] = x[2] > 0.0 ? x[2] : 0.0;
                gf[10] = x[3] > 0.0 ? x[3] : 0.0;
                gf[11] = x[4];
                gf[14] = cxc + x[0];
                gf[15] = cyc + x[1];
                p.dgain[w] = x[5];
                p.dN0[w] = x[6];
                int cc = 7;
                if (p.ukx) p.db4x[w] = x[cc++];
                if (p.uky) p.db4y[w] = x[cc];
            }
        }
        __syncwarp();
    }
}

// Centred FFT of one plane (kspace_fft2_centered) and the regressor probe.
__global__ void fft_probe_kernel(const double *plane, int H, int W, double *re, double *im, double *tmp)
{
    extern __shared__ double sm[];
    const int lane = threadIdx.x & 31;
    double *cw = sm, *sw = cw + W, *ch = sw + W, *sh = ch + H;
    for (int m = lane; m < W; m += 32) sincospi(2.0 * m / W, &sw[m], &cw[m]);
    for (int m = lane; m < H; m += 32) sincospi(2.0 * m / H, &sh[m], &ch[m]);
    __syncwarp();
    dft_centred(plane, H, W, cw, sw, ch, sh, re, im, tmp, tmp + H * W);
}

std::mutex g_mu;
struct Ws {
    void *dev = nullptr;
    size_t cap = 0;
    cudaStream_t s = nullptr;
    int ensure(size_t b)
    {
        if (!s && cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return -2;
        if (b > cap) {
            if (dev) cudaFree(dev);
            dev = nullptr;
            cap = 0;
            if (cudaMalloc(&dev, b + b / 4) != cudaSuccess) { cudaGetLastError(); return -2; }
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

// Device-pointer fit.  Inputs/outputs as kspace_lm_fit_batch, all on the device;
// scratch from pivb_kspace_scratch_bytes.
PIV_EXPORT size_t pivb_kspace_scratch_bytes(int n_windows, int h, int w)
{
    (void)n_windows;
    const size_t P = (size_t)h * w;
    const size_t per_warp = PER_BIN * P * 8;
    if (per_warp <= 48 * 1024) return 256;
    const int dev = piv::current_device();
    const int sms = dev < 0 ? 148 : piv::device_sms(dev);
    return 256 + pad256((size_t)sms * 8 * per_warp);
}

PIV_EXPORT int pivb_kspace_fit_dev(const double *d_RAA, const double *d_RBB, const double *d_RAB,
                                   const unsigned char *d_mask, const double *d_Pwin, int n_windows, int h, int w,
                                   int use_kx4, int use_ky4, double *d_gauss, int *d_status, double *d_init,
                                   double *d_gain, double *d_N0, double *d_b4x, double *d_b4y, double *d_cpp,
                                   int *d_nvalid, int *d_iter, unsigned char *d_conv, void *d_scratch,
                                   size_t scratch_bytes, void *stream)
{
    if (!size_ok(h) || !size_ok(w)) return -1;
    if (n_windows <= 0) return 0;
    cudaStream_t s = (cudaStream_t)stream;
    const int dev = piv::current_device();
    if (dev < 0) return -2;
    const int n_sms = piv::device_sms(dev);
    if (scratch_bytes < pivb_kspace_scratch_bytes(n_windows, h, w) || !d_scratch) return -2;
    const size_t P = (size_t)h * w;
    const size_t per_warp = PER_BIN * P * 8;
    KsParams p{};
    p.RAA = d_RAA; p.RBB = d_RBB; p.RAB = d_RAB; p.mask = d_mask; p.Pw = d_Pwin;
    p.nw = n_windows; p.H = h; p.W = w; p.ukx = use_kx4 ? 1 : 0; p.uky = use_ky4 ? 1 : 0;
    p.K = 7 + p.ukx + p.uky;
    p.gf = d_gauss; p.ig = d_init; p.dgain = d_gain; p.dN0 = d_N0; p.db4x = d_b4x; p.db4y = d_b4y;
    p.dcpp = d_cpp; p.status = d_status; p.dnv = d_nvalid; p.diter = d_iter; p.dconv = d_conv;
    int *n_proc = static_cast<int *>(d_scratch);
    if (cudaMemsetAsync(n_proc, 0, 4, s) != cudaSuccess) return -2;
    count_kernel<<<64, 256, 0, s>>>(d_mask, n_windows, n_proc);
    init_kernel<<<(n_windows + 127) / 128, 128, 0, s>>>(p, n_proc);
    int warps;
    size_t smem = (size_t)(2 * w + 2 * h + w + h) * 8;
    if (per_warp <= 48 * 1024) {
        p.use_smem = 1;
        warps = (int)((160 * 1024) / per_warp);
        warps = warps < 1 ? 1 : (warps > 4 ? 4 : warps);
        smem += warps * per_warp;
        p.gscratch = nullptr;
    } else {
        p.use_smem = 0;
        warps = 4;
        p.gscratch = reinterpret_cast<double *>(static_cast<char *>(d_scratch) + 256);
    }
    if (cudaFuncSetAttribute(fit_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return -2;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fit_kernel, warps * 32, smem) != cudaSuccess) return -2;
    if (per_sm < 1) per_sm = 1;
    long long want = ((long long)n_windows + warps - 1) / warps;
    long long cap = (long long)per_sm * n_sms;
    if (!p.use_smem) cap = (long long)n_sms * 8 / warps;   // scratch slots
    int grid = (int)(want < cap ? want : cap);
    fit_kernel<<<grid, warps * 32, smem, s>>>(p, warps);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// kspace_lm_fit.h:54-61.  n_threads is accepted for signature compatibility; the
// GPU decides its own parallelism.
PIV_EXPORT int kspace_lm_fit_batch(const double *R_AA, const double *R_BB, const double *R_AB,
                                   const unsigned char *mask_flat, const double *P_win, int n_windows, int corr_h,
                                   int corr_w, int use_kx4, int use_ky4, int n_threads, double *gauss_flat,
                                   int *status_flat, double *initial_guess_flat, double *diag_gain, double *diag_N0,
                                   double *diag_b4x, double *diag_b4y, double *diag_cost_per_pt, int *diag_n_valid,
                                   int *diag_iter, unsigned char *diag_conv)
{
    (void)n_threads;
    if (!size_ok(corr_h) || !size_ok(corr_w)) return -1;
    if (n_windows <= 0) return 0;
    std::lock_guard<std::mutex> lock(g_mu);
    const size_t P = (size_t)corr_h * corr_w, nw = (size_t)n_windows;
    Ws *wsp = cur_ws();
    if (wsp == nullptr || wsp->ensure(16)) return -2;
    const size_t scr = pivb_kspace_scratch_bytes(n_windows, corr_h, corr_w);
    const size_t bytes = 3 * pad256(nw * P * 8) + pad256(nw) + (P_win ? pad256(nw * P * 8) : 0) + 2 * pad256(nw * 128) +
                         5 * pad256(nw * 8) + 3 * pad256(nw * 4) + pad256(nw) + pad256(scr) + 4096;
    if (wsp->ensure(bytes)) return -2;
    cudaStream_t s = wsp->s;
    char *base = static_cast<char *>(wsp->dev);
    size_t off = 0;
    auto take = [&](size_t b) { char *q = base + off; off += pad256(b); return q; };
    double *aa = (double *)take(nw * P * 8), *bb = (double *)take(nw * P * 8), *ab = (double *)take(nw * P * 8);
    unsigned char *m = (unsigned char *)take(nw);
    double *pw = P_win ? (double *)take(nw * P * 8) : nullptr;
    double *gf = (double *)take(nw * 128), *ig = (double *)take(nw * 128);
    double *dg = (double *)take(nw * 8), *dn = (double *)take(nw * 8), *dbx = (double *)take(nw * 8);
    double *dby = (double *)take(nw * 8), *dc = (double *)take(nw * 8);
    int *st = (int *)take(nw * 4), *nvv = (int *)take(nw * 4), *itr = (int *)take(nw * 4);
    unsigned char *cv = (unsigned char *)take(nw);
    void *scratch = take(scr);
#define H2D(d, h, n) if (cudaMemcpyAsync(d, h, n, cudaMemcpyHostToDevice, s) != cudaSuccess) return -2
#define D2H(h, d, n) if (cudaMemcpyAsync(h, d, n, cudaMemcpyDeviceToHost, s) != cudaSuccess) return -2
    H2D(aa, R_AA, nw * P * 8);
    H2D(bb, R_BB, nw * P * 8);
    H2D(ab, R_AB, nw * P * 8);
    H2D(m, mask_flat, nw);
    if (pw) H2D(pw, P_win, nw * P * 8);
    int e = pivb_kspace_fit_dev(aa, bb, ab, m, pw, n_windows, corr_h, corr_w, use_kx4, use_ky4, gf, st, ig, dg, dn,
                                dbx, dby, dc, nvv, itr, cv, scratch, scr, s);
    if (e) return e;
    D2H(gauss_flat, gf, nw * 128);
    D2H(status_flat, st, nw * 4);
    D2H(initial_guess_flat, ig, nw * 128);
    D2H(diag_gain, dg, nw * 8);
    D2H(diag_N0, dn, nw * 8);
    D2H(diag_b4x, dbx, nw * 8);
    D2H(diag_b4y, dby, nw * 8);
    D2H(diag_cost_per_pt, dc, nw * 8);
    D2H(diag_n_valid, nvv, nw * 4);
    D2H(diag_iter, itr, nw * 4);
    D2H(diag_conv, cv, nw);
#undef H2D
#undef D2H
    return cudaStreamSynchronize(s) == cudaSuccess ? 0 : -2;
}

// kspace_lm_fit.h:65.  The loader calls it once as a liveness probe; here it
// reports the GPU's multiprocessor count (0 without a usable GPU).
PIV_EXPORT int kspace_lm_fit_max_threads(void)
{
    int d = 0, n = 0;
    if (cudaGetDevice(&d) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, d) != cudaSuccess) return 0;
    return n;
}

// kspace_lm_fit.h:86-87
PIV_EXPORT int kspace_fft2_centered(const double *plane, int H, int W, double *out_re, double *out_im)
{
    if (!size_ok(H) || !size_ok(W)) return -1;
    std::lock_guard<std::mutex> lock(g_mu);
    const size_t P = (size_t)H * W;
    Ws *wsp = cur_ws();
    if (wsp == nullptr || wsp->ensure(5 * pad256(P * 8) + 1024)) return -2;
    cudaStream_t s = wsp->s;
    double *d = static_cast<double *>(wsp->dev);
    double *re = d + P, *im = d + 2 * P, *tmp = d + 3 * P;
    if (cudaMemcpyAsync(d, plane, P * 8, cudaMemcpyHostToDevice, s) != cudaSuccess) return -2;
    fft_probe_kernel<<<1, 32, (size_t)(2 * W + 2 * H) * 8, s>>>(d, H, W, re, im, tmp);
    if (cudaGetLastError() != cudaSuccess) return -2;
    if (cudaMemcpyAsync(out_re, re, P * 8, cudaMemcpyDeviceToHost, s) != cudaSuccess) return -2;
    if (cudaMemcpyAsync(out_im, im, P * 8, cudaMemcpyDeviceToHost, s) != cudaSuccess) return -2;
    return cudaStreamSynchronize(s) == cudaSuccess ? 0 : -2;
}

// kspace_lm_fit.h:79-82: floor regressor (natural order) and N0 seed of one window.
__global__ void debug_prep_kernel(const double *aa, const double *bb, const double *ab, const double *Pc, int H,
                                  int W, double *Dv, double *seed, double *work)
{
    extern __shared__ double sm[];
    const int lane = threadIdx.x & 31, P = H * W;
    double *cw = sm, *sw = cw + W, *ch = sw + W, *sh = ch + H;
    for (int m = lane; m < W; m += 32) sincospi(2.0 * m / W, &sw[m], &cw[m]);
    for (int m = lane; m < H; m += 32) sincospi(2.0 * m / H, &sh[m], &ch[m]);
    __syncwarp();
    double *Fr = work, *re = work + P, *im = work + 2 * P, *tmp = work + 3 * P;
    dft_centred(aa, H, W, cw, sw, ch, sh, re, im, tmp, tmp + P);
    for (int b = lane; b < P; b += 32) Fr[b] = hypot(re[b], im[b]);
    __syncwarp();
    dft_centred(bb, H, W, cw, sw, ch, sh, re, im, tmp, tmp + P);
    for (int b = lane; b < P; b += 32) Fr[b] = sqrt(Fr[b] * hypot(re[b], im[b]));
    __syncwarp();
    int n_tail = 0;
    for (int b0 = 0; b0 < P; b0 += 32) {
        const int b = b0 + lane;
        bool in = false;
        double v = 0.0;
        if (b < P) {
            const int r = b / W, c = b % W;
            const double kx = (c < (W + 1) / 2 ? (double)c : (double)(c - W)) / (double)W;
            const double ky = (r < (H + 1) / 2 ? (double)r : (double)(r - H)) / (double)H;
            if (Pc) {
                const double pv = Pc[((r + H / 2) % H) * W + (c + W / 2) % W];
                Dv[b] = pv / (Fr[b] > 1e-30 ? Fr[b] : 1e-30);
                in = ky * ky + kx * kx >= SEED_KR_MIN * SEED_KR_MIN;
                v = Fr[b] / (pv > 1e-30 ? pv : 1e-30);
            } else {
                Dv[b] = 1.0 / (Fr[b] > 1e-30 ? Fr[b] : 1e-30);
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, in);
        if (in) re[n_tail + __popc(m & ((1u << lane) - 1u))] = v;
        n_tail += __popc(m);
    }
    __syncwarp();
    if (Pc) {
        double med = warp_median(re, n_tail);
        med = med < SEED_CLIP_LO ? SEED_CLIP_LO : (med > SEED_CLIP_HI ? SEED_CLIP_HI : med);
        if (lane == 0) *seed = med;
    } else if (lane == 0) {
        *seed = 0.0;
    }
}

PIV_EXPORT int kspace_debug_prep(const double *R_AA, const double *R_BB, const double *R_AB, const double *P_centred,
                                 int H, int W, double *out_Dv, double *out_n0_seed)
{
    if (!size_ok(H) || !size_ok(W)) return -1;
    std::lock_guard<std::mutex> lock(g_mu);
    const size_t P = (size_t)H * W;
    Ws *wsp = cur_ws();
    if (wsp == nullptr || wsp->ensure(12 * pad256(P * 8) + 1024)) return -2;
    cudaStream_t s = wsp->s;
    double *d = static_cast<double *>(wsp->dev);
    double *aa = d, *bb = d + P, *ab = d + 2 * P, *pc = d + 3 * P, *dv = d + 4 * P, *seed = d + 5 * P,
           *work = d + 6 * P;
    if (cudaMemcpyAsync(aa, R_AA, P * 8, cudaMemcpyHostToDevice, s) != cudaSuccess) return -2;
    if (cudaMemcpyAsync(bb, R_BB, P * 8, cudaMemcpyHostToDevice, s) != cudaSuccess) return -2;
    if (cudaMemcpyAsync(ab, R_AB, P * 8, cudaMemcpyHostToDevice, s) != cudaSuccess) return -2;
    if (P_centred && cudaMemcpyAsync(pc, P_centred, P * 8, cudaMemcpyHostToDevice, s) != cudaSuccess) return -2;
    debug_prep_kernel<<<1, 32, (size_t)(2 * W + 2 * H) * 8, s>>>(aa, bb, ab, P_centred ? pc : nullptr, H, W, dv, seed,
                                                                  work);
    if (cudaGetLastError() != cudaSuccess) return -2;
    if (cudaMemcpyAsync(out_Dv, dv, P * 8, cudaMemcpyDeviceToHost, s) != cudaSuccess) return -2;
    if (cudaMemcpyAsync(out_n0_seed, seed, 8, cudaMemcpyDeviceToHost, s) != cudaSuccess) return -2;
    return cudaStreamSynchronize(s) == cudaSuccess ? 0 : -2;
}
