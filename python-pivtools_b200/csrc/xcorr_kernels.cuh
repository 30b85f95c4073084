// xcorr_kernels.cuh -- kernels of libbulkxcorr2d.
#pragma once

#include <type_traits>

#include "xcorr_engine.cuh"

namespace piv {

// Deferred Levenberg-Marquardt work item: the compensated 5x5 patch of one
// window plus what the output writes need.  One record per window; flag 0 means
// "nothing to fit" (invalid window or gate failure already written).
struct alignas(16) LmRecord {
    float sub[PKN];
    float best;
    float enorm;
    int ij;      // (i0 << 16) | j0
    int flag;
    float pad[3];
};
static_assert(sizeof(LmRecord) == 128, "LmRecord is one 128-byte line");

struct XcorrParams {
    const float *A, *B;
    long long img_stride;      // elements between consecutive frames
    const float *mask;         // [nwy * nwx] (1 = skip) or null
    int H, W, n_img;
    const float *ctr_x, *ctr_y;
    int nwy, nwx;
    const float *wA, *wB;
    const float *cw;           // correlation weight numel / (wB * wB), [N*N]
    int ensemble, n_peaks, finder;
    float *pk_x, *pk_y, *pk_h, *sx, *sy, *sxy, *pk_ratio;
    float *planes;             // debug dump or ensemble output, nullable
    LmRecord *lm;              // deferred LM records, nullable
    long long total;           // n_img * nwy * nwx
    float neg_zero;            // -0.0f, passed at run time (see mulz2)
};

// A packed launch: several jobs (pivb_xcorr_dev calls) of one window size in one
// grid.  Job j owns the padded window range [off[j], off[j+1]); each offset is a
// multiple of the CTA's window count, so every CTA iteration lies in one job.
// Passed whole as a grid-constant kernel parameter (no device copy of the
// table, nothing to order on the stream).
constexpr int kMaxJobs = 40;
struct XcorrJobs {
    XcorrParams job[kMaxJobs];
    long long off[kMaxJobs + 1];
    long long total;           // off[n_jobs]
    int n_jobs;
};

// Job of padded window index g (binary search of the offsets); sets the
// job-local index.
__device__ __forceinline__ int job_of(const XcorrJobs &pk, long long g, long long &local)
{
    int lo = 0, hi = pk.n_jobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pk.off[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    local = g - pk.off[lo];
    return lo;
}

template <bool JOBS>
using XcorrArg = std::conditional_t<JOBS, XcorrJobs, XcorrParams>;

template <bool JOBS>
__device__ __forceinline__ const XcorrParams &params_of(const XcorrArg<JOBS> &in, int job)
{
    if constexpr (JOBS) return in.job[job];
    else return in;
}

__device__ __forceinline__ void write_sentinel(const XcorrParams &p, long long o, float enorm)
{
    p.pk_x[o] = __int_as_float(0x7fc00000);
    p.pk_y[o] = __int_as_float(0x7fc00000);
    p.pk_h[o] = fmul(0.0f, enorm);
    p.sx[o] = 0.0f;
    p.sy[o] = 0.0f;
    p.sxy[o] = 0.0f;
}

__device__ __forceinline__ void write_peak(const XcorrParams &p, long long o, int N, int bi, int bj,
                                           const float *off, const float *sig, float best, float enorm)
{
    const float half = (float)N / 2.0f;
    p.pk_x[o] = fsub(fadd(off[1], (float)bj), half);
    p.pk_y[o] = fsub(fadd(off[0], (float)bi), half);
    p.pk_h[o] = fmul(best, enorm);
    p.sx[o] = sig[0];
    p.sy[o] = sig[1];
    p.sxy[o] = sig[2];
}

// Group-leader finish of one window: peak choice and detectability (from the
// parallel search, or an exact sequential scan when the plane holds NaN), the
// height and border gates, the weighted 5x5 patch, the fit (or a deferred LM
// record), and the outputs (PIV_2d_cross_correlate.c:80-125, peak_locate_lm.c:757-918).
// pl: float plane of the window, row stride ld.
template <int N, bool MULTI>
__device__ __forceinline__ void finish_window(const XcorrParams &prm, float *pl, int ld, PeakAcc acc, bool has_nan,
                                           long long idx, int n, int iw, long long nwt, bool valid, float enorm)
{
    LmRecord *rec = prm.lm ? prm.lm + idx : nullptr;
    if (!valid) {
        if (rec) rec->flag = 0;
    } else {
        PlaneView v{pl, ld};
        int bi, bj;
        float best, ratio;
        if (has_nan) {
            best = seq_search(v, N, N, &bi, &bj);
            ratio = seq_detectability(v, N, N);
        } else {
            best = acc.best;
            bi = (acc.idx == 0x7fffffff) ? 0 : acc.idx / N;
            bj = (acc.idx == 0x7fffffff) ? 0 : acc.idx % N;
            ratio = (acc.p2 > 0.0f) ? fdiv(acc.p1, acc.p2) : 0.0f;
        }
        prm.pk_ratio[(long long)n * nwt + iw] = ratio;
        const int np = MULTI ? prm.n_peaks : 1;
        for (int k = 0; k < np; ++k) {
            if (k > 0) best = seq_search(v, N, N, &bi, &bj);
            const long long o = (long long)n * np * nwt + (long long)k * nwt + iw;
            if (!(best > 0.0f) && !(best != best)) {   // best <= 0
                write_sentinel(prm, o, enorm);
                if (rec) rec->flag = 0;
                continue;
            }
            if (bi < 2 || bi >= N - 2 || bj < 2 || bj >= N - 2) {
                write_sentinel(prm, o, enorm);
                if (rec) rec->flag = 0;
                continue;
            }
            float sub[PKN];
#pragma unroll
            for (int aa = 0; aa < PKW; ++aa)
#pragma unroll
                for (int bb = 0; bb < PKW; ++bb) {
                    const int r = bi + aa - 2, c = bj + bb - 2;
                    sub[aa * PKW + bb] = fmul(pl[r * ld + c], __ldg(prm.cw + r * N + c));
                }
            if (k == 0 && rec && !MULTI) {
                // deferred fit (single peak): the patch goes to the window's record
#pragma unroll
                for (int q = 0; q < PKN; ++q) rec->sub[q] = sub[q];
                rec->best = best;
                rec->enorm = enorm;
                rec->ij = (bi << 16) | bj;
                rec->flag = 1;
                continue;
            }
            float off[2], sig[3], fv[PKN];
            bool ok = true;
            if constexpr (MULTI) {
                if (k == 0 && prm.finder >= 4 && prm.finder <= 6) {
                    ok = lm_fit_any<0>(prm.finder, sub, off, sig, fv);
                } else {
                    float A0, s0, s1;
                    three_point(sub, PKW, PKW, PKW, off, &A0, &s0, &s1);
                    sig[0] = s0; sig[1] = s1; sig[2] = 0.0f;
                    for (int q = 0; q < PKN; ++q) {
                        float di = fdiv(fsub((float)(q / PKW - 2), off[0]), s0);
                        float dj = fdiv(fsub((float)(q % PKW - 2), off[1]), s1);
                        fv[q] = fmul(A0, expf_cr(-fadd(fmul(di, di), fmul(dj, dj))));
                    }
                }
            } else {
                float A0, s0, s1;
                three_point(sub, PKW, PKW, PKW, off, &A0, &s0, &s1);
                sig[0] = s0; sig[1] = s1; sig[2] = 0.0f;
            }
            if (!ok) write_sentinel(prm, o, enorm);
            else write_peak(prm, o, N, bi, bj, off, sig, best, enorm);
            if constexpr (MULTI) {
                float *mp = const_cast<float *>(pl);
                for (int q = 0; q < PKN; ++q) {
                    const int r = bi + q / PKW - 2, c = bj + q % PKW - 2;
                    float f = fdiv(fv[q], __ldg(prm.cw + r * N + c));
                    float d = fsub(mp[r * ld + c], f);
                    mp[r * ld + c] = (0.0f > d) ? 0.0f : d;
                }
            }
        }
    }
}

// finish_window for a single-peak call with deferred fits, spread over the
// window's group: every thread holds the same search result, so the gates are
// uniform and the 128-byte record (compensated 5x5 patch, peak, norm, position,
// flag) is written by up to 32 threads at once instead of element by element.
// Invalid windows and planes holding NaN take the leader's finish_window.
template <int N>
__device__ __forceinline__ void finish_window_rec(int t, int gw, const XcorrParams &prm, float *pl, int ld,
                                                  const PeakAcc &acc, bool has_nan, long long idx, int n, int iw,
                                                  long long nwt, bool valid, float enorm)
{
    if (!valid || has_nan) {
        if (t == 0) finish_window<N, false>(prm, pl, ld, acc, has_nan, idx, n, iw, nwt, valid, enorm);
        return;
    }
    const float best = acc.best;
    const int bi = (acc.idx == 0x7fffffff) ? 0 : acc.idx / N;
    const int bj = (acc.idx == 0x7fffffff) ? 0 : acc.idx % N;
    const long long o = (long long)n * nwt + iw;
    const bool gated = !(best > 0.0f) || bi < 2 || bi >= N - 2 || bj < 2 || bj >= N - 2;
    if (t == 0) prm.pk_ratio[o] = (acc.p2 > 0.0f) ? fdiv(acc.p1, acc.p2) : 0.0f;
    if (gated) {
        if (t == 0) {
            write_sentinel(prm, o, enorm);
            prm.lm[idx].flag = 0;
        }
        return;
    }
    float *rec = reinterpret_cast<float *>(prm.lm + idx);      // sub[25], best, enorm, ij, flag
    for (int q = t; q < PKN + 4; q += gw) {
        float val;
        if (q < PKN) {
            const int r = bi + q / PKW - 2, c = bj + q % PKW - 2;
            val = fmul(pl[r * ld + c], __ldg(prm.cw + r * N + c));
        } else if (q == PKN) {
            val = best;
        } else if (q == PKN + 1) {
            val = enorm;
        } else {
            val = __int_as_float(q == PKN + 2 ? ((bi << 16) | bj) : 1);
        }
        rec[q] = val;
    }
}

// Fused correlation kernel (PIV_2d_cross_correlate.c:203-397): gather + weight +
// mean/energy, packed forward FFT, conjugate product, inverse FFT, shift, peak
// search, 3-point fit.  LM fits of single-peak calls are deferred to
// lm_records_kernel; MULTI handles nPeaks > 1 entirely in the group leader.
template <int N, bool MULTI, bool JOBS = false>
__global__ void __launch_bounds__(WinGeo<N>::CTA_THREADS, MULTI ? 1 : WinGeo<N>::MIN_CTAS)
xcorr_kernel(const __grid_constant__ XcorrArg<JOBS> prm_in)
{
    static_assert(!(MULTI && JOBS), "packed launches are single-peak");
    using G = WinGeo<N>;
    constexpr int M = G::M, P = G::P;
    extern __shared__ float4 smem_raw[];
    char *smem = reinterpret_cast<char *>(smem_raw);
    int gi, t;
    if constexpr (G::GW <= 32) {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        gi = warp * G::WPW + lane / G::GW;
        t = lane % G::GW;
    } else {
        gi = 0;
        t = threadIdx.x;
    }
    float2 *S = reinterpret_cast<float2 *>(smem + gi * G::PLANE_BYTES);
    float *red = reinterpret_cast<float *>(smem + G::GROUPS_PER_CTA * G::PLANE_BYTES);
    float2 *tw = reinterpret_cast<float2 *>(smem + G::GROUPS_PER_CTA * G::PLANE_BYTES + G::RED_BYTES);
    fill_lane_twiddles<N>(tw, threadIdx.x, G::CTA_THREADS);
    if constexpr (G::TW_BYTES > 0) __syncthreads();
    // 32 px: both window weights staged once per CTA as pairs {wA, wB} (one
    // 64-bit shared load per sample in the gather)
    float2 *swt = reinterpret_cast<float2 *>(smem + G::GROUPS_PER_CTA * G::PLANE_BYTES + G::RED_BYTES + G::TW_BYTES);
    const float *staged_wa = nullptr, *staged_wb = nullptr;
    if constexpr (N == 32 && !JOBS) {
        for (int i = threadIdx.x; i < N * N; i += G::CTA_THREADS) swt[i] = make_float2(prm_in.wA[i], prm_in.wB[i]);
        __syncthreads();
    }
    const float2 nz = dup2(params_of<JOBS>(prm_in, 0).neg_zero);
    auto wmul = [&](float2 x, float2 w) { return mulz2(x, w, nz); };
    const Group<N> g{t, red};
    const bool active = t < G::T;
    int line, p;
    lane_slot<N>(active ? t : 0, line, p);
    const long long per_iter = (long long)gridDim.x * G::GROUPS_PER_CTA;
    const long long n_iter = (prm_in.total + per_iter - 1) / per_iter;
    const float inv_numel = 1.0f / (float)(N * N);

    for (long long it = 0; it < n_iter; ++it) {
        long long idx = it * per_iter + (long long)blockIdx.x * G::GROUPS_PER_CTA + gi;
        int job = 0;
        if constexpr (JOBS) {
            // every window of this CTA's chunk belongs to one job (job offsets
            // are multiples of the chunk), so the whole CTA sees the same job
            long long local;
            job = job_of(prm_in, it * per_iter + (long long)blockIdx.x * G::GROUPS_PER_CTA, local);
            idx = local + gi;
        }
        const XcorrParams &prm = params_of<JOBS>(prm_in, job);
        if constexpr (JOBS && N == 32) {
            // the staged weight pairs follow the job's weights (uniform over the CTA)
            if (prm.wA != staged_wa || prm.wB != staged_wb) {
                __syncthreads();
                for (int i = threadIdx.x; i < N * N; i += G::CTA_THREADS) swt[i] = make_float2(prm.wA[i], prm.wB[i]);
                staged_wa = prm.wA;
                staged_wb = prm.wB;
                __syncthreads();
            }
        }
        const long long nwt = (long long)prm.nwy * prm.nwx;
        const bool inrange = idx < prm.total;
        int n = 0, iw = 0, r0 = 0, c0 = 0;
        bool valid = inrange;
        if (inrange) {
            n = (int)(idx / nwt);
            iw = (int)(idx - (long long)n * nwt);
            const int ii = iw % prm.nwx, jj = iw / prm.nwx;
            if (prm.mask && prm.mask[iw] == 1.0f) valid = false;
            r0 = (int)floor((double)prm.ctr_y[jj] - ((double)N - 1.0) / 2.0 + 0.5);
            c0 = (int)floor((double)prm.ctr_x[ii] - ((double)N - 1.0) / 2.0 + 0.5);
            if (r0 < 0 || c0 < 0 || r0 + N > prm.H || c0 + N > prm.W) valid = false;
        }
        // ---- gather, weight, mean, energy (PIV_2d_cross_correlate.c:299-353).
        // At 32, 48, 64 and 128 px as pairs z = {A, B}, one paired instruction per
        // step for both frames (bit-identical; +3.6% at 32 px); 96 and 16 px ran
        // 9% and 3% slower that way and keep the scalar form.
        float2 z[M];
        float ea, eb;
        if constexpr (N == 32 || N == 48 || N == 64 || N == 128) {
            float2 sab = make_float2(0.0f, 0.0f);
            if (active && valid) {
                const float *fa = prm.A + (long long)n * prm.img_stride + (long long)r0 * prm.W + c0 + line;
                const float *fb = prm.B + (long long)n * prm.img_stride + (long long)r0 * prm.W + c0 + line;
                if constexpr (N == 128) {
                    // one weight for both frames: load it once (measured faster at
                    // 128 px; 32 px reads staged pairs, 48 and 64 px plain loads)
                    const bool same_w = prm.wA == prm.wB;
#pragma unroll
                    for (int k = 0; k < M; ++k) {
                        const int r = P * k + p;
                        const float wa = __ldg(prm.wA + r * N + line);
                        const float wb = same_w ? wa : __ldg(prm.wB + r * N + line);
                        z[k] = wmul(make_float2(__ldg(fa + (long long)r * prm.W), __ldg(fb + (long long)r * prm.W)),
                                    make_float2(wa, wb));
                        sab = add2(sab, z[k]);
                    }
                } else if constexpr (G::WT_BYTES > 0) {
#pragma unroll
                    for (int k = 0; k < M; ++k) {
                        const int r = P * k + p;
                        z[k] = wmul(make_float2(__ldg(fa + (long long)r * prm.W), __ldg(fb + (long long)r * prm.W)),
                                    swt[r * N + line]);
                        sab = add2(sab, z[k]);
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < M; ++k) {
                        const int r = P * k + p;
                        z[k] = wmul(make_float2(__ldg(fa + (long long)r * prm.W), __ldg(fb + (long long)r * prm.W)),
                                    make_float2(__ldg(prm.wA + r * N + line), __ldg(prm.wB + r * N + line)));
                        sab = add2(sab, z[k]);
                    }
                }
            } else {
#pragma unroll
                for (int k = 0; k < M; ++k) z[k] = make_float2(0.0f, 0.0f);
            }
            const float mean_a = g.sum(sab.x) / (float)(N * N);
            const float mean_b = g.sum(sab.y) / (float)(N * N);
            float2 e2 = make_float2(0.0f, 0.0f);
            if (!prm.ensemble) {
                const float2 mab = make_float2(mean_a, mean_b);
#pragma unroll
                for (int k = 0; k < M; ++k) {
                    if (active && valid) z[k] = sub2(z[k], mab);
                    e2 = fma2(z[k], z[k], e2);
                }
            } else {
#pragma unroll
                for (int k = 0; k < M; ++k) e2 = fma2(z[k], z[k], e2);
            }
            ea = g.sum(e2.x);
            eb = g.sum(e2.y);
        } else {
            float a[M], b[M];
            float sa = 0.0f, sb = 0.0f;
            if (active && valid) {
                const float *fa = prm.A + (long long)n * prm.img_stride + (long long)r0 * prm.W + c0 + line;
                const float *fb = prm.B + (long long)n * prm.img_stride + (long long)r0 * prm.W + c0 + line;
                if constexpr (P == 4) {
                    // one weight for both frames: load it once (faster at 96 px)
                    const bool same_w = prm.wA == prm.wB;
#pragma unroll
                    for (int k = 0; k < M; ++k) {
                        const int r = P * k + p;
                        const float wa = __ldg(prm.wA + r * N + line);
                        const float wb = same_w ? wa : __ldg(prm.wB + r * N + line);
                        a[k] = __ldg(fa + (long long)r * prm.W) * wa;
                        b[k] = __ldg(fb + (long long)r * prm.W) * wb;
                        sa += a[k];
                        sb += b[k];
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < M; ++k) {
                        const int r = P * k + p;
                        a[k] = __ldg(fa + (long long)r * prm.W) * __ldg(prm.wA + r * N + line);
                        b[k] = __ldg(fb + (long long)r * prm.W) * __ldg(prm.wB + r * N + line);
                        sa += a[k];
                        sb += b[k];
                    }
                }
            } else {
#pragma unroll
                for (int k = 0; k < M; ++k) { a[k] = 0.0f; b[k] = 0.0f; }
            }
            const float mean_a = g.sum(sa) / (float)(N * N);
            const float mean_b = g.sum(sb) / (float)(N * N);
            float e_a = 0.0f, e_b = 0.0f;
            if (!prm.ensemble) {
#pragma unroll
                for (int k = 0; k < M; ++k) {
                    if (active && valid) { a[k] -= mean_a; b[k] -= mean_b; }
                    e_a += a[k] * a[k];
                    e_b += b[k] * b[k];
                }
            } else {
#pragma unroll
                for (int k = 0; k < M; ++k) { e_a += a[k] * a[k]; e_b += b[k] * b[k]; }
            }
            ea = g.sum(e_a);
            eb = g.sum(e_b);
#pragma unroll
            for (int k = 0; k < M; ++k) z[k] = make_float2(a[k], b[k]);
        }
        const float enorm = 1.0f / sqrtf(ea * eb);

        correlate_plane<N>(g, S, z, inv_numel, tw);
        float *pl = reinterpret_cast<float *>(S);

        if (prm.planes && valid) {
            float *dst = prm.planes + idx * (long long)(N * N);
#pragma unroll 1
            for (int k = t; k < N * N; k += G::GW) dst[k] = pl[(k / N) * G::STF + (k % N)];
        }
        if (!prm.ensemble) {
            PeakAcc acc;
            bool has_nan;
            search_plane<N>(g, pl, acc, has_nan);
            if constexpr (!MULTI) {
                if (prm.lm) {
                    if (inrange && active)
                        finish_window_rec<N>(t, G::T, prm, pl, G::STF, acc, has_nan, idx, n, iw, nwt, valid, enorm);
                } else if (t == 0 && inrange) {
                    finish_window<N, false>(prm, pl, G::STF, acc, has_nan, idx, n, iw, nwt, valid, enorm);
                }
            } else if (t == 0 && inrange) {
                finish_window<N, MULTI>(prm, pl, G::STF, acc, has_nan, idx, n, iw, nwt, valid, enorm);
            }
        }
        g.sync();
    }
}

// Deferred single-peak fits (3-point or LM): one thread per window record.
template <int MODE, bool JOBS = false>
__global__ void __launch_bounds__(128) lm_records_kernel(const __grid_constant__ XcorrArg<JOBS> prm_in, int N)
{
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= prm_in.total) return;
    int job = 0;
    if constexpr (JOBS) {
        long long local;
        job = job_of(prm_in, idx, local);
        idx = local;
    }
    const XcorrParams &prm = params_of<JOBS>(prm_in, job);
    if (JOBS && idx >= prm.total) return;        // padding of the job's window range
    const LmRecord &rec = prm.lm[idx];
    if (rec.flag != 1) return;
    float sub[PKN];
    const float4 *s4 = reinterpret_cast<const float4 *>(rec.sub);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        float4 v = s4[k];
        sub[4 * k] = v.x; sub[4 * k + 1] = v.y; sub[4 * k + 2] = v.z; sub[4 * k + 3] = v.w;
    }
    sub[24] = rec.sub[24];
    float off[2], sig[3];
    bool ok = true;
    if (prm.finder == 3) {
        float A0, s0, s1;
        three_point(sub, PKW, PKW, PKW, off, &A0, &s0, &s1);
        sig[0] = s0; sig[1] = s1; sig[2] = 0.0f;
    } else {
        ok = lm_fit_any<MODE>(prm.finder, sub, off, sig, nullptr);
    }
    if (!ok) write_sentinel(prm, idx, rec.enorm);
    else write_peak(prm, idx, N, rec.ij >> 16, rec.ij & 0xffff, off, sig, rec.best, rec.enorm);
}

// Deferred LM fits (types 4-6) of single-peak calls, persistent: warp w owns the
// records [w * chunk, (w + 1) * chunk) and its lanes refill as their fits end, so
// a lane whose fit converged early takes the next record instead of idling while
// the warp's slowest fit iterates (one thread per record left about a third of
// the lanes active).  Each fit runs lm_init / lm_step / lm_finish, the same
// arithmetic as lm_fit, so the results equal lm_records_kernel's.
template <int T, int MODE>
__global__ void __launch_bounds__(128) lm_fit_kernel(const __grid_constant__ XcorrParams prm, int N, long long chunk)
{
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    long long next = warp * chunk;                            // warp-uniform
    const long long end = min(prm.total, next + chunk);
    LmState<T> st;
    float sub[PKN], pred[PKN];
    long long idx = 0;
    bool active = false;
#pragma unroll 1
    for (;;) {
        // lanes without a fit take the next records of the chunk; records that
        // need no fit (flag != 1) are passed over
#pragma unroll 1
        for (;;) {
            const unsigned need = __ballot_sync(0xffffffffu, !active);
            if (need == 0u || next >= end) break;
            const long long mine = next + __popc(need & ((1u << lane) - 1u));
            next += __popc(need);
            if (!active && mine < end) {
                const LmRecord &rec = prm.lm[mine];
                if (rec.flag == 1) {
                    const float4 *s4 = reinterpret_cast<const float4 *>(rec.sub);
#pragma unroll
                    for (int k = 0; k < 6; ++k) {
                        const float4 v = s4[k];
                        sub[4 * k] = v.x; sub[4 * k + 1] = v.y; sub[4 * k + 2] = v.z; sub[4 * k + 3] = v.w;
                    }
                    sub[24] = rec.sub[24];
                    lm_init<T, MODE>(sub, st, pred);
                    idx = mine;
                    active = true;
                }
            }
        }
        if (__ballot_sync(0xffffffffu, active) == 0u) break;
        if (active) {
            const int r = lm_step<T, MODE>(sub, st, pred);
            if (r != 0) {
                float off[2], sig[3];
                const LmRecord &rec = prm.lm[idx];
                if (!lm_finish<T, MODE>(st, r == 1, off, sig)) write_sentinel(prm, idx, rec.enorm);
                else write_peak(prm, idx, N, rec.ij >> 16, rec.ij & 0xffff, off, sig, rec.best, rec.enorm);
                active = false;
            }
        }
    }
}

// numel / (w (*) w): linear autocorrelation of the window weight at shift
// (r - h/2, c - w/2), FP64 sum (PIV_2d_cross_correlate.c:216-222, xcorr.c:55-122).
// Generic two-input form; `divide` selects the reciprocal weighting.
__global__ void lin_xcorr_kernel(const float *w1, const float *w2, int h, int w, float *out, int divide)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= h * w) return;
    const int sy = k / w - h / 2, sx = k % w - w / 2;
    double acc = 0.0;
    const int y0 = max(0, -sy), y1 = min(h, h - sy), x0 = max(0, -sx), x1 = min(w, w - sx);
    for (int y = y0; y < y1; ++y)
        for (int x = x0; x < x1; ++x)
            acc += (double)w1[(y + sy) * w + x + sx] * (double)w2[y * w + x];
    out[k] = divide ? (float)(h * w) / (float)acc : (float)acc;
}

// Circular cross-correlation, fftshifted and divided by... nothing else: the
// codelet result IFFT(FFT(a) conj(FFT(b)))/numel is the plain circular sum.
__global__ void circ_xcorr_kernel(const float *a, const float *b, int h, int w, float *out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= h * w) return;
    const int sy = k / w - h / 2, sx = k % w - w / 2;
    double acc = 0.0;
    for (int y = 0; y < h; ++y) {
        const int yy = ((y + sy) % h + h) % h;
        for (int x = 0; x < w; ++x) {
            const int xx = ((x + sx) % w + w) % w;
            acc += (double)a[yy * w + xx] * (double)b[y * w + x];
        }
    }
    out[k] = (float)acc;
}

struct GlobalPlane {
    const float *s;
    int ld;
    __device__ __forceinline__ float operator()(int i, int j) const { return s[(long long)i * ld + j]; }
};

// Block-wide reduction of PeakAcc (blockDim.x = 128).
__device__ __forceinline__ void block_reduce_peak(PeakAcc &a, float *red)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        float ob = __shfl_xor_sync(0xffffffffu, a.best, o);
        int oi = __shfl_xor_sync(0xffffffffu, a.idx, o);
        float o1 = __shfl_xor_sync(0xffffffffu, a.p1, o);
        float o2 = __shfl_xor_sync(0xffffffffu, a.p2, o);
        a.merge(ob, oi, o1, o2);
    }
    const int w = threadIdx.x >> 5;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) {
        red[4 * w] = a.best;
        red[4 * w + 1] = __int_as_float(a.idx);
        red[4 * w + 2] = a.p1;
        red[4 * w + 3] = a.p2;
    }
    __syncthreads();
    a.init();
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k)
        a.merge(red[4 * k], __float_as_int(red[4 * k + 1]), red[4 * k + 2], red[4 * k + 3]);
}

// Peak fit of arbitrary n0 x n1 planes already in device memory: one CTA per
// plane (lsqpeaklocate_lm / lsqpeaklocate_lm_batch / peak_detectability).
//   layout 0: loc/std are [3*n_peaks] per plane, contiguous per plane
//   layout 1: component-major [3][lanes] (the batch fitter's layout)
// work: scratch copy of each plane for secondary-peak subtraction (n_peaks > 1).
template <int MODE>
__global__ void __launch_bounds__(128)
fit_planes_kernel(const float *planes, int n0, int n1, int n_peaks, int fit, const float *wt,
                  float *loc, float *sd, int layout, int lanes, float *ratio, float *work)
{
    __shared__ float red[16];
    __shared__ int nan_flag;
    const int pid = blockIdx.x;
    const float *src = planes + (long long)pid * n0 * n1;
    if (threadIdx.x == 0) nan_flag = 0;
    __syncthreads();
    PeakAcc acc;
    acc.init();
    bool nan = false;
    GlobalPlane v{src, n1};
    const int h2 = n0 * 3 / 4 - n0 / 4, w2 = n1 * 3 / 4 - n1 / 4;
    for (int c = threadIdx.x; c < h2 * w2; c += blockDim.x) {
        const int i = n0 / 4 + c / w2, j = n1 / 4 + c % w2;
        acc.add(candidate(v, i, j, &nan), i * n1 + j);
    }
    if (nan) atomicOr(&nan_flag, 1);
    block_reduce_peak(acc, red);
    if (threadIdx.x != 0) return;
    const bool has_nan = nan_flag != 0;
    if (ratio) {
        ratio[pid] = has_nan ? seq_detectability(v, n0, n1)
                             : ((acc.p2 > 0.0f) ? fdiv(acc.p1, acc.p2) : 0.0f);
    }
    if (!loc) return;
    float *mp = nullptr;
    if (n_peaks > 1) {
        mp = work + (long long)pid * n0 * n1;
        for (int k = 0; k < n0 * n1; ++k) mp[k] = src[k];
    }
    GlobalPlane mv{mp ? mp : src, n1};
    int bi, bj;
    float best;
    if (has_nan) best = seq_search(v, n0, n1, &bi, &bj);
    else {
        best = acc.best;
        bi = (acc.idx == 0x7fffffff) ? 0 : acc.idx / n1;
        bj = (acc.idx == 0x7fffffff) ? 0 : acc.idx % n1;
    }
    for (int k = 0; k < n_peaks; ++k) {
        if (k > 0) best = seq_search(mv, n0, n1, &bi, &bj);
        long long o0, o1, o2;
        if (layout == 0) {
            o0 = (long long)pid * 3 * n_peaks + k;
            o1 = o0 + n_peaks;
            o2 = o1 + n_peaks;
        } else {
            o0 = pid;
            o1 = pid + lanes;
            o2 = pid + 2 * lanes;
        }
        const float qnan = __int_as_float(0x7fc00000);
        if (!(best > 0.0f) && !(best != best) || bi < 2 || bi >= n0 - 2 || bj < 2 || bj >= n1 - 2) {
            loc[o0] = qnan; loc[o1] = qnan; loc[o2] = 0.0f;
            sd[o0] = 0.0f; sd[o1] = 0.0f; sd[o2] = 0.0f;
            continue;
        }
        float sub[PKN], fv[PKN], off[2], sig[3];
        for (int q = 0; q < PKN; ++q) {
            const long long id = (long long)(bi + q / PKW - 2) * n1 + (bj + q % PKW - 2);
            const float x = mp ? mp[id] : src[id];
            sub[q] = wt ? fmul(x, wt[id]) : x;
        }
        bool ok = true;
        if (k == 0 && fit >= 4 && fit <= 6) {
            ok = lm_fit_any<MODE>(fit, sub, off, sig, fv);
        } else {
            float A0, s0, s1;
            three_point(sub, PKW, PKW, PKW, off, &A0, &s0, &s1);
            sig[0] = s0; sig[1] = s1; sig[2] = 0.0f;
            for (int q = 0; q < PKN; ++q) {
                float di = fdiv(fsub((float)(q / PKW - 2), off[0]), s0);
                float dj = fdiv(fsub((float)(q % PKW - 2), off[1]), s1);
                fv[q] = fmul(A0, expf_cr(-fadd(fmul(di, di), fmul(dj, dj))));
            }
        }
        if (!ok) {
            loc[o0] = qnan; loc[o1] = qnan; loc[o2] = 0.0f;
            sd[o0] = 0.0f; sd[o1] = 0.0f; sd[o2] = 0.0f;
        } else {
            loc[o0] = fadd(off[0], (float)bi);
            loc[o1] = fadd(off[1], (float)bj);
            loc[o2] = best;
            sd[o0] = sig[0]; sd[o1] = sig[1]; sd[o2] = sig[2];
        }
        if (mp) {
            for (int q = 0; q < PKN; ++q) {
                const long long id = (long long)(bi + q / PKW - 2) * n1 + (bj + q % PKW - 2);
                float f = wt ? fdiv(fv[q], wt[id]) : fv[q];
                float d = fsub(mp[id], f);
                mp[id] = (0.0f > d) ? 0.0f : d;
            }
        }
    }
}

// min / max fold with the reference's MIN/MAX-macro NaN behaviour
// (PIV_2d_cross_correlate.c:836-860): the result is the fold over the elements
// after the last NaN, or NaN if the last element is NaN.
__global__ void last_nan_kernel(const float *v, int n, int *last)
{
    int best = -1;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (v[i] != v[i]) best = max(best, i);
    if (best >= 0) atomicMax(last, best);
}

__global__ void minmax_fold_kernel(const float *v, int n, const int *last, int want_max, float *out)
{
    __shared__ float s[256];
    const int start = *last + 1;
    float acc = __int_as_float(0x7fc00000);
    bool have = false;
    for (int i = start + threadIdx.x; i < n; i += blockDim.x) {
        float x = v[i];
        if (!have) { acc = x; have = true; }
        else acc = want_max ? (acc > x ? acc : x) : (acc < x ? acc : x);
    }
    s[threadIdx.x] = have ? acc : (want_max ? -INFINITY : INFINITY);
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            float a = s[threadIdx.x], b = s[threadIdx.x + o];
            s[threadIdx.x] = want_max ? (a > b ? a : b) : (a < b ? a : b);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (start >= n) *out = (n > 0 && *last == n - 1) ? v[n - 1] : v[0];
        else *out = s[0];
    }
}

}  // namespace piv

namespace piv {

// Ensemble accumulation (PIV_2d_cross_correlate.c:403-484, 502-833).
struct AccumParams {
    const float *A, *B;
    long long img_stride;
    const float *mask;
    int H, W, n_img;
    const float *ctr_x, *ctr_y;
    int nwy, nwx;
    const float *w_ab_a, *w_ab_b, *w_aa, *w_bb;   // plain accumulate: wA, wB, -, -
    const float *wsums;                           // [3] sums of w_ab_b, w_aa, w_bb (device)
    int out_h, out_w, sy0, sx0;
    int mean_sub, ppn, triple;
    float *ab, *aa, *bb;                          // += outputs [nwt][out_h*out_w]
    float *comp;                                  // Kahan carries [3][nwt][out_h*out_w] or null
    float *gacc;                                  // global accumulators when shared memory is too small
    long long nwt;
};

__device__ __forceinline__ void kahan_add(float &s, float &c, float v)
{
    const float y = __fsub_rn(v, c);
    const float t = __fadd_rn(s, y);
    c = __fsub_rn(__fsub_rn(t, s), y);
    s = t;
}

// Window-stationary: one thread group per window streams all pairs of the call.
// Correlation is linear, so the planes of a run of pairs are the inverse
// transform of the sum of their spectra: each pair adds its cross spectrum and
// its two power spectra (packed as |F_A|^2 + i |F_B|^2, per-pair scales
// applied) to sums kept in shared memory (or, for the largest windows, global
// scratch), and every kAccumBlock pairs (and at the end of the call) the sums
// are transformed back once, cropped and added to the caller's planes with
// Kahan compensation in FP32 (the compensation carried across calls in `comp`).
// Per pair that leaves the two packed forward transforms (AB-weighted A + i B;
// AA/BB auto-weighted A + i B) and the spectrum products; the inverse
// transforms run once per block.  The spectral sums of a block are plain FP32
// (at most kAccumBlock terms).
constexpr int kAccumBlock = 64;

template <int N, bool SMEM_ACC>
__global__ void __launch_bounds__(WinGeo<N>::CTA_THREADS) accum_kernel(AccumParams prm)
{
    using G = WinGeo<N>;
    constexpr int M = G::M, P = G::P, T = G::T;
    constexpr int ACC_FLOATS = 4 * N * N;
    extern __shared__ float4 smem_raw[];
    char *smem = reinterpret_cast<char *>(smem_raw);
    int gi, t;
    if constexpr (G::GW <= 32) {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        gi = warp * G::WPW + lane / G::GW;
        t = lane % G::GW;
    } else {
        gi = 0;
        t = threadIdx.x;
    }
    float2 *S = reinterpret_cast<float2 *>(smem + gi * G::PLANE_BYTES);
    float *red = reinterpret_cast<float *>(smem + G::GROUPS_PER_CTA * G::PLANE_BYTES);
    float *acc;
    if constexpr (SMEM_ACC)
        acc = reinterpret_cast<float *>(smem + G::GROUPS_PER_CTA * G::PLANE_BYTES + 64 * G::RED_SLOTS * 4 + 64) +
              gi * ACC_FLOATS;
    else
        acc = prm.gacc + ((long long)blockIdx.x * G::GROUPS_PER_CTA + gi) * ACC_FLOATS;
    // spectral sums, element (lane t, sample n) at n * T + t: cross, then powers
    float2 *sab = reinterpret_cast<float2 *>(acc), *spw = sab + N * N;
    const Group<N> g{t, red};
    const bool active = t < G::T;
    int line, p;
    lane_slot<N>(active ? t : 0, line, p);
    const int q = out_block<P>(p);
    const int nout = prm.out_h * prm.out_w;
    const long long per_iter = (long long)gridDim.x * G::GROUPS_PER_CTA;
    const long long n_iter = (prm.nwt + per_iter - 1) / per_iter;
    const float inv_numel = 1.0f / (float)(N * N);
    const int col = (line + N / 2) % N - prm.sx0;
    const bool col_in = active && col >= 0 && col < prm.out_w;

    for (long long it = 0; it < n_iter; ++it) {
        const long long iw = it * per_iter + (long long)blockIdx.x * G::GROUPS_PER_CTA + gi;
        bool valid = iw < prm.nwt;
        int r0 = 0, c0 = 0;
        if (valid) {
            const int ii = (int)(iw % prm.nwx), jj = (int)(iw / prm.nwx);
            if (prm.mask && prm.mask[iw] == 1.0f) valid = false;
            r0 = (int)floorf(prm.ctr_y[jj] - ((float)N - 1.0f) / 2.0f + 0.5f);
            c0 = (int)floorf(prm.ctr_x[ii] - ((float)N - 1.0f) / 2.0f + 0.5f);
            if (r0 < 0 || c0 < 0 || r0 + N > prm.H || c0 + N > prm.W) valid = false;
        }
        int in_block = 0;
        for (int n = 0; n < prm.n_img; ++n) {
            if (in_block == 0 && active) {
#pragma unroll
                for (int k = 0; k < M; ++k) {
                    sab[k * T + t] = make_float2(0.0f, 0.0f);
                    spw[k * T + t] = make_float2(0.0f, 0.0f);
                }
            }
            float ra[M], rb[M];
            if (active && valid) {
                const float *fa = prm.A + (long long)n * prm.img_stride + (long long)r0 * prm.W + c0 + line;
                const float *fb = prm.B + (long long)n * prm.img_stride + (long long)r0 * prm.W + c0 + line;
#pragma unroll
                for (int k = 0; k < M; ++k) {
                    const int r = P * k + p;
                    ra[k] = __ldg(fa + (long long)r * prm.W);
                    rb[k] = __ldg(fb + (long long)r * prm.W);
                }
            } else {
#pragma unroll
                for (int k = 0; k < M; ++k) { ra[k] = 0.0f; rb[k] = 0.0f; }
            }
            float s_ab = 1.0f, s_aa = 1.0f, s_bb = 1.0f;
            bool skip = false;
            float m_abb = 0.0f, m_aa = 0.0f, m_bb = 0.0f;
            if (prm.triple) {
                if (prm.mean_sub) {
                    float s1 = 0.0f, s2 = 0.0f, s3 = 0.0f;
                    if (active) {
#pragma unroll
                        for (int k = 0; k < M; ++k) {
                            const int wi = (P * k + p) * N + line;
                            s1 += rb[k] * __ldg(prm.w_ab_b + wi);
                            s2 += ra[k] * __ldg(prm.w_aa + wi);
                            s3 += rb[k] * __ldg(prm.w_bb + wi);
                        }
                    }
                    s1 = g.sum(s1);
                    s2 = g.sum(s2);
                    s3 = g.sum(s3);
                    const float w1 = prm.wsums[0], w2 = prm.wsums[1], w3 = prm.wsums[2];
                    m_abb = (w1 > 0.0f) ? s1 / w1 : 0.0f;
                    m_aa = (w2 > 0.0f) ? s2 / w2 : 0.0f;
                    m_bb = (w3 > 0.0f) ? s3 / w3 : 0.0f;
                }
                if (prm.ppn) {
                    float eaa = 0.0f, ebb = 0.0f;
#pragma unroll
                    for (int k = 0; k < M; ++k) {
                        const int wi = (P * k + p) * N + line;
                        const float x3 = (ra[k] - m_aa) * (active ? __ldg(prm.w_aa + wi) : 0.0f);
                        const float x4 = (rb[k] - m_bb) * (active ? __ldg(prm.w_bb + wi) : 0.0f);
                        eaa += x3 * x3;
                        ebb += x4 * x4;
                    }
                    eaa = g.sum(eaa);
                    ebb = g.sum(ebb);
                    // a pair without signal contributes to no plane; the group still
                    // runs the transforms (groups share warps and their shuffles)
                    if (eaa <= 0.0f || ebb <= 0.0f) skip = true;
                    s_ab = 1.0f / sqrtf(eaa * ebb);
                    s_aa = 1.0f / eaa;
                    s_bb = 1.0f / ebb;
                }
            }
            // one code copy of the forward transform for both products (two
            // inlined copies stalled instruction fetch; measured 1.6-2% faster,
            // bit-identical): f = 0 the auto-weighted pair -> 4 (|F_A|^2 + i |F_B|^2),
            // f = 1 the AB-weighted pair -> the cross spectrum 4 F_B conj(F_A)
            // (slot0 = B, slot1 = A)
#pragma unroll 1
            for (int f = prm.triple ? 0 : 1; f < 2; ++f) {
                const float *wa = f == 0 ? prm.w_aa : prm.w_ab_a;
                const float *wb = f == 0 ? prm.w_bb : prm.w_ab_b;
                const float ma = m_aa, mb = f == 0 ? m_bb : m_abb;
                float u[M], v[M];
#pragma unroll
                for (int k = 0; k < M; ++k) {
                    const int wi = (P * k + p) * N + line;
                    const float w1 = active ? __ldg(wa + wi) : 0.0f, w2 = active ? __ldg(wb + wi) : 0.0f;
                    if (prm.triple) {
                        u[k] = (ra[k] - ma) * w1;
                        v[k] = (rb[k] - mb) * w2;
                    } else {
                        u[k] = ra[k] * w1;
                        v[k] = rb[k] * w2;
                    }
                }
                float2 z[M];
                fft2_forward<N>(g, S, u, v);
                if (f == 0) spectrum_product<N, 1>(g, S, z);
                else spectrum_product<N, 0>(g, S, z);
                if (active && valid && !skip) {
                    float2 *dst = f == 0 ? spw : sab;
                    const float2 sc = f == 0 ? make_float2(s_aa, s_bb) : make_float2(s_ab, s_ab);
#pragma unroll
                    for (int k = 0; k < M; ++k) {
                        float2 a = dst[k * T + t];
                        a.x += sc.x * z[k].x;
                        a.y += sc.y * z[k].y;
                        dst[k * T + t] = a;
                    }
                }
            }
            // the end of a block or of the call: one inverse of each sum, added
            // to the caller's planes
            if (++in_block == kAccumBlock || n + 1 == prm.n_img) {
                in_block = 0;
#pragma unroll 1
                for (int pass = 0; pass < (prm.triple ? 2 : 1); ++pass) {
                    const float2 *src = pass == 0 ? sab : spw;
                    float2 z[M];
#pragma unroll
                    for (int k = 0; k < M; ++k) z[k] = active ? src[k * T + t] : make_float2(0.0f, 0.0f);
                    fft2_inverse<N>(g, S, z);
                    if (valid) {
#pragma unroll
                        for (int k = 0; k < M; ++k) {
                            const int row = (M * q + k + N / 2) % N - prm.sy0;
                            if (col_in && row >= 0 && row < prm.out_h) {
                                const long long e = iw * nout + row * prm.out_w + col;
#pragma unroll
                                for (int h = 0; h < 2; ++h) {
                                    if (pass == 0 && h == 1) break;           // the cross plane is real
                                    const int a = pass == 0 ? 0 : 1 + h;      // AB, AA, BB
                                    float *out = a == 0 ? prm.ab : (a == 1 ? prm.aa : prm.bb);
                                    const float v = ((h == 0 ? z[k].x : z[k].y) * 0.25f) * inv_numel;
                                    float sum = out[e];
                                    float c = prm.comp ? prm.comp[(long long)a * prm.nwt * nout + e] : 0.0f;
                                    kahan_add(sum, c, v);
                                    out[e] = sum;
                                    if (prm.comp) prm.comp[(long long)a * prm.nwt * nout + e] = c;
                                }
                            }
                        }
                    }
                }
            }
        }
        g.sync();
    }
}

}  // namespace piv

namespace piv {
// Sequential float sums of the three mean-subtraction weights, in the order of
// PIV_2d_cross_correlate.c:671-678.
__global__ void weight_sums_kernel(const float *w1, const float *w2, const float *w3, int n, float *out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    float a = 0.0f, b = 0.0f, c = 0.0f;
    for (int i = 0; i < n; ++i) {
        a = __fadd_rn(a, w1[i]);
        b = __fadd_rn(b, w2[i]);
        c = __fadd_rn(c, w3[i]);
    }
    out[0] = a;
    out[1] = b;
    out[2] = c;
}
}  // namespace piv
