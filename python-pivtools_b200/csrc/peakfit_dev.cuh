// peakfit_dev.cuh -- device peak search and subpixel fits.
//
// Arithmetic is written with explicit round-to-nearest intrinsics (__fmul_rn,
// __fadd_rn, __dmul_rn, ...) so that nvcc cannot contract a multiply and an add
// into one FMA: the fit then evaluates every float and double expression in the
// order, and with the roundings, of the reference's scalar fitter
// (pivtools_cli/lib/peak_locate_lm.c, compiled without FMA on x86-64) and of its
// lockstep twin (peak_locate_lm_batch.c, compiled with -ffp-contract=off).
//
// expf: the scalar fitter calls libm expf (correctly rounded in glibc); here the
// exponential is exp() in double rounded once to float, which gives the
// correctly rounded float.  The batch fitter's own exponential (peak_simd.h:
// Cody-Waite reduction, degree-5 polynomial, exponent-field scaling) is restated
// for impl = 1.  log() in the 3-point estimator is double, as in the reference.
#pragma once

#include <float.h>

#include "piv_common.cuh"

namespace piv {

__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

constexpr int PKW = 5;              // fit patch side (peak_locate_lm.h:16-17)
constexpr int PKN = PKW * PKW;

// Row-major index of (i, j), j <= i, in a packed lower triangle.
__host__ __device__ constexpr int tri(int i, int j) { return i * (i + 1) / 2 + j; }

// Correctly rounded float exponential via double.
__device__ __forceinline__ float expf_cr(float x) { return (float)exp((double)x); }

// Exponential of the reference's batch fitter (restated from its published
// polynomial): arguments are clamped below at -87.3365478515625.
__device__ __forceinline__ float expf_batch(float x)
{
    const float lo = -87.3365478515625f;
    float xc = (x > lo) ? x : lo;
    float rn = fsub(fadd(fmul(1.44269504088896341f, xc), 12582912.0f), 12582912.0f);
    int n = (int)rn;
    float r = fsub(fsub(xc, fmul(rn, 0.693359375f)), fmul(rn, -2.12194440e-4f));
    float r2 = fmul(r, r);
    float p = 1.9875691500e-4f;
    p = fadd(fmul(p, r), 1.3981999507e-3f);
    p = fadd(fmul(p, r), 8.3334519073e-3f);
    p = fadd(fmul(p, r), 4.1665795894e-2f);
    p = fadd(fmul(p, r), 1.6666665459e-1f);
    p = fadd(fmul(p, r), 5.0000001201e-1f);
    float er = fadd(fadd(fmul(p, r2), r), 1.0f);
    float s = __int_as_float((int)((unsigned)(n + 127) << 23));
    return fmul(er, s);
}

template <int MODE>
__device__ __forceinline__ float fexp(float x)
{
    if constexpr (MODE == 0) return expf_cr(x);
    else return expf_batch(x);
}
// Clamp helpers: fminf/fmaxf in the scalar fitter, compare-select in the batch.
template <int MODE>
__device__ __forceinline__ float cmax(float a, float b)
{
    if constexpr (MODE == 0) return fmaxf(a, b);
    else return (a > b) ? a : b;
}
template <int MODE>
__device__ __forceinline__ float cmin(float a, float b)
{
    if constexpr (MODE == 0) return fminf(a, b);
    else return (a < b) ? a : b;
}

// 3-point log-parabola at the centre of a (rows x cols) patch with row stride ld
// (peak_locate_lm.c:35-66).  loc[0] = row offset, loc[1] = column offset.
__device__ __forceinline__ void three_point(const float *x, int rows, int cols, int ld,
                                            float *loc, float *A, float *sx, float *sy)
{
    const int cr = (rows - 1) / 2, cc = (cols - 1) / 2;
    float xf[3], yf[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float a = x[(i - 1 + cr) * ld + cc];
        float b = x[cr * ld + (i - 1 + cc)];
        xf[i] = (float)log((double)((a < FLT_EPSILON) ? FLT_EPSILON : a));
        yf[i] = (float)log((double)((b < FLT_EPSILON) ? FLT_EPSILON : b));
    }
    float dx = fadd(fsub(fmul(2.0f, xf[0]), fmul(4.0f, xf[1])), fmul(2.0f, xf[2]));
    float dy = fadd(fsub(fmul(2.0f, yf[0]), fmul(4.0f, yf[1])), fmul(2.0f, yf[2]));
    loc[0] = (fabsf(dx) > FLT_EPSILON) ? fdiv(fsub(xf[0], xf[2]), dx) : 0.0f;
    loc[1] = (fabsf(dy) > FLT_EPSILON) ? fdiv(fsub(yf[0], yf[2]), dy) : 0.0f;
    *A = x[cr * ld + cc];
    *sx = sqrtf(fdiv(-4.0f, fadd(dx, FLT_EPSILON)));
    *sy = sqrtf(fdiv(-4.0f, fadd(dy, FLT_EPSILON)));
}

// Model of fit type T at patch coordinate (i, j); p = {A, i0, j0, s1, s2, s3}.
template <int T, int MODE>
__device__ __forceinline__ float lm_model(float i, float j, const float *p)
{
    if constexpr (T == 4) {
        float di = fdiv(fsub(i, p[1]), p[3]), dj = fdiv(fsub(j, p[2]), p[3]);
        return fmul(p[0], fexp<MODE>(-fadd(fmul(di, di), fmul(dj, dj))));
    } else if constexpr (T == 5) {
        float di = fdiv(fsub(i, p[1]), p[3]), dj = fdiv(fsub(j, p[2]), p[4]);
        return fmul(p[0], fexp<MODE>(-fadd(fmul(di, di), fmul(dj, dj))));
    } else {
        float di = fsub(i, p[1]), dj = fsub(j, p[2]);
        float q = fadd(fadd(fdiv(fmul(di, di), p[3]), fdiv(fmul(dj, dj), p[4])),
                       fmul(fmul(fmul(2.0f, di), dj), p[5]));
        return fmul(p[0], fexp<MODE>(fmul(-0.5f, q)));
    }
}

template <int T, int MODE>
__device__ __forceinline__ double lm_resid(const float *sub, const float *p, float *pred)
{
    double rs = 0.0;
    // one patch row per iteration: its five model values are independent, so
    // their latency overlaps; the residual sum keeps the row-major order
    float i = -2.0f;
#pragma unroll 1
    for (int a = 0; a < PKW; ++a) {
        float v[PKW];
#pragma unroll
        for (int b = 0; b < PKW; ++b) v[b] = lm_model<T, MODE>(i, (float)(b - 2), p);
#pragma unroll
        for (int b = 0; b < PKW; ++b) {
            pred[a * PKW + b] = v[b];
            float r = fsub(v[b], sub[a * PKW + b]);
            rs = dadd(rs, dmul((double)r, (double)r));
        }
        i += 1.0f;
    }
    return rs;
}

template <int T>
__device__ __forceinline__ void lm_jac(const float *sub, const float *p, const float *pred,
                                       double *JtJ, double *Jtr)
{
    constexpr int n = (T == 4) ? 4 : (T == 5 ? 5 : 6);
#pragma unroll
    for (int a = 0; a < n * (n + 1) / 2; ++a) JtJ[a] = 0.0;
#pragma unroll
    for (int a = 0; a < n; ++a) Jtr[a] = 0.0;
    float i = -2.0f, j = -2.0f;
#pragma unroll 1
    for (int q = 0; q < PKN; ++q) {
        float v = pred[q];
        float r = fsub(v, sub[q]);
        float J[n];
        if constexpr (T == 4) {
            float di = fdiv(fsub(i, p[1]), p[3]), dj = fdiv(fsub(j, p[2]), p[3]);
            float r2 = fadd(fmul(di, di), fmul(dj, dj));
            float v2 = fmul(2.0f, v);
            J[0] = fdiv(v, p[0]);
            J[1] = fdiv(fmul(v2, di), p[3]);
            J[2] = fdiv(fmul(v2, dj), p[3]);
            J[3] = fdiv(fmul(v2, r2), p[3]);
        } else if constexpr (T == 5) {
            float di = fdiv(fsub(i, p[1]), p[3]), dj = fdiv(fsub(j, p[2]), p[4]);
            float v2 = fmul(2.0f, v);
            J[0] = fdiv(v, p[0]);
            J[1] = fdiv(fmul(v2, di), p[3]);
            J[2] = fdiv(fmul(v2, dj), p[4]);
            J[3] = fdiv(fmul(fmul(v2, di), di), p[3]);
            J[4] = fdiv(fmul(fmul(v2, dj), dj), p[4]);
        } else {
            float di = fsub(i, p[1]), dj = fsub(j, p[2]);
            float vh = fmul(0.5f, v);
            J[0] = fdiv(v, p[0]);
            J[1] = fmul(v, fadd(fdiv(di, p[3]), fmul(dj, p[5])));
            J[2] = fmul(v, fadd(fdiv(dj, p[4]), fmul(di, p[5])));
            J[3] = fdiv(fmul(fmul(vh, di), di), fmul(p[3], p[3]));
            J[4] = fdiv(fmul(fmul(vh, dj), dj), fmul(p[4], p[4]));
            J[5] = fmul(fmul(-v, di), dj);
        }
#pragma unroll
        for (int a = 0; a < n; ++a) {
            Jtr[a] = dadd(Jtr[a], dmul((double)J[a], (double)r));
#pragma unroll
            for (int b = 0; b <= a; ++b) JtJ[tri(a, b)] = dadd(JtJ[tri(a, b)], dmul((double)J[a], (double)J[b]));
        }
        j += 1.0f;
        if (j > 2.0f) { j = -2.0f; i += 1.0f; }
    }
}

// (JtJ + lambda diag) delta = -Jtr by FP64 Cholesky (peak_locate_lm.c:342-393).
// JtJ is the packed lower triangle; the factor overwrites a working copy of it
// entry by entry (each entry is read once, just before its factor value is
// written), the reference's operation order throughout.
template <int n>
__device__ __forceinline__ bool lm_solve(const double *JtJ, const double *Jtr, float lambda, float *delta)
{
    double L[n * (n + 1) / 2], y[n], d[n];
    const double l1 = dadd(1.0, (double)lambda);
#pragma unroll
    for (int a = 0; a < n * (n + 1) / 2; ++a) L[a] = JtJ[a];
#pragma unroll
    for (int i = 0; i < n; ++i) L[tri(i, i)] = dmul(L[tri(i, i)], l1);
#pragma unroll
    for (int i = 0; i < n; ++i) {
#pragma unroll
        for (int j = 0; j <= i; ++j) {
            double s = L[tri(i, j)];
#pragma unroll
            for (int k = 0; k < j; ++k) s = dsub(s, dmul(L[tri(i, k)], L[tri(j, k)]));
            if (i == j) {
                if (s <= 0.0) return false;
                L[tri(i, i)] = sqrt(s);
            } else {
                L[tri(i, j)] = ddiv(s, L[tri(j, j)]);
            }
        }
    }
#pragma unroll
    for (int i = 0; i < n; ++i) {
        double s = -Jtr[i];
#pragma unroll
        for (int j = 0; j < i; ++j) s = dsub(s, dmul(L[tri(i, j)], y[j]));
        y[i] = ddiv(s, L[tri(i, i)]);
    }
#pragma unroll
    for (int i = n - 1; i >= 0; --i) {
        double s = y[i];
#pragma unroll
        for (int j = i + 1; j < n; ++j) s = dsub(s, dmul(L[tri(j, i)], d[j]));
        d[i] = ddiv(s, L[tri(i, i)]);
    }
#pragma unroll
    for (int i = 0; i < n; ++i) delta[i] = (float)d[i];
    return true;
}

// Marquardt fit of a compensated 5x5 patch (peak_locate_lm.c:412-712 for MODE 0,
// peak_locate_lm_batch.c:362-588 per lane for MODE 1), in three pieces so that a
// caller can interleave the iterations of many fits: lm_init (start values from
// the 3-point fit, residual, normal equations), lm_step (one damped step) and
// lm_finish (the trust test).  lm_fit runs them in sequence.
template <int T>
struct LmState {
    static constexpr int n = (T == 4) ? 4 : (T == 5 ? 5 : 6);
    float p[6];
    double JtJ[n * (n + 1) / 2], Jtr[n];      // normal equations, packed lower triangle
    double resid;
    float lambda;
    int it;
};

template <int T, int MODE>
__device__ __forceinline__ void lm_init(const float *sub, LmState<T> &st, float *pred)
{
    float pk[2], A, sx, sy;
    three_point(sub, PKW, PKW, PKW, pk, &A, &sx, &sy);
#pragma unroll
    for (int k = 0; k < 6; ++k) st.p[k] = 0.0f;
    st.p[0] = A;
    st.p[1] = fminf(fmaxf(pk[0], -2.0f), 2.0f);
    st.p[2] = fminf(fmaxf(pk[1], -2.0f), 2.0f);
    if constexpr (T == 4) {
        float s = sqrtf(fadd(fmul(sx, sx), fmul(sy, sy)));
        st.p[3] = fminf(fmaxf(s, 0.5f), 3.0f);
    } else if constexpr (T == 5) {
        st.p[3] = fminf(fmaxf(sx, 0.5f), 3.0f);
        st.p[4] = fminf(fmaxf(sy, 0.5f), 3.0f);
    } else {
        st.p[3] = fminf(fmaxf(fmul(sx, sx), 0.25f), 9.0f);
        st.p[4] = fminf(fmaxf(fmul(sy, sy), 0.25f), 9.0f);
    }
    st.lambda = 0.01f;
    st.it = 0;
    st.resid = lm_resid<T, MODE>(sub, st.p, pred);
    lm_jac<T>(sub, st.p, pred, st.JtJ, st.Jtr);
}

// One iteration of at most 50: 0 = go on, 1 = converged, 2 = stopped without
// converging (singular system, damping above 1e6 or the iteration limit).
template <int T, int MODE>
__device__ __forceinline__ int lm_step(const float *sub, LmState<T> &st, float *pred)
{
    constexpr int n = LmState<T>::n;
    float delta[n];
    if (!lm_solve<n>(st.JtJ, st.Jtr, st.lambda, delta)) return 2;
    float *p = st.p;
    float q[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) q[k] = p[k];
#pragma unroll
    for (int k = 0; k < n; ++k) q[k] = fadd(p[k], delta[k]);
    q[0] = cmax<MODE>(q[0], fmul(p[0], 0.5f));
    q[1] = cmin<MODE>(cmax<MODE>(q[1], -2.5f), 2.5f);
    q[2] = cmin<MODE>(cmax<MODE>(q[2], -2.5f), 2.5f);
    if constexpr (T == 4) {
        q[3] = cmin<MODE>(cmax<MODE>(q[3], 0.25f), 4.0f);
    } else if constexpr (T == 5) {
        q[3] = cmin<MODE>(cmax<MODE>(q[3], 0.25f), 4.0f);
        q[4] = cmin<MODE>(cmax<MODE>(q[4], 0.25f), 4.0f);
    } else {
        q[3] = cmin<MODE>(cmax<MODE>(q[3], 0.1f), 16.0f);
        q[4] = cmin<MODE>(cmax<MODE>(q[4], 0.1f), 16.0f);
        float smax = fdiv(0.95f, sqrtf(fmul(q[3], q[4])));
        q[5] = cmin<MODE>(cmax<MODE>(q[5], -smax), smax);
    }
    const double nr = lm_resid<T, MODE>(sub, q, pred);
    int r = 0;
    if (nr < st.resid) {
#pragma unroll
        for (int k = 0; k < 6; ++k) p[k] = q[k];
        const double improve = ddiv(dsub(st.resid, nr), dadd(st.resid, (double)FLT_EPSILON));
        st.resid = nr;
        st.lambda = fmul(st.lambda, 0.5f);
        lm_jac<T>(sub, p, pred, st.JtJ, st.Jtr);
        if (improve < 1e-6) r = 1;
    } else {
        st.lambda = fmul(st.lambda, 2.0f);
        if (st.lambda > 1e6f) r = 2;
    }
    if (r == 0 && ++st.it == 50) r = 2;
    return r;
}

// Trust test and outputs; `converged` is lm_step's result 1.
template <int T, int MODE>
__device__ __forceinline__ bool lm_finish(const LmState<T> &st, bool converged, float *off, float *sig)
{
    const float *p = st.p;
    bool ok = converged;
    if (!ok) {
        if constexpr (MODE == 0) {
            ok = st.resid <= (double)fmul(fmul(fmul(1e-3f, p[0]), p[0]), 25.0f);
        } else {
            constexpr float frac = 1e-3f * 25.0f;
            ok = st.resid <= (double)fmul(fmul(frac, p[0]), p[0]);
        }
    }
    if (ok) {
        if constexpr (T == 6) ok = (p[3] > 0.1f && p[3] < 16.0f && p[4] > 0.1f && p[4] < 16.0f);
        else if constexpr (T == 5) ok = (p[3] > 0.25f && p[3] < 4.0f && p[4] > 0.25f && p[4] < 4.0f);
        else ok = (p[3] > 0.25f && p[3] < 4.0f);
    }
    off[0] = p[1];
    off[1] = p[2];
    if constexpr (T == 4) { sig[0] = p[3]; sig[1] = p[3]; sig[2] = 0.0f; }
    else if constexpr (T == 5) { sig[0] = p[3]; sig[1] = p[4]; sig[2] = 0.0f; }
    else { sig[0] = p[3]; sig[1] = p[4]; sig[2] = p[5]; }
    return ok;
}

// The whole fit of one patch.  Returns true if trusted.
template <int T, int MODE>
__device__ bool lm_fit(const float *sub, float *off, float *sig, float *fitval)
{
    float pred[PKN];
    LmState<T> st;
    lm_init<T, MODE>(sub, st, pred);
    int r = 0;
#pragma unroll 1
    while (r == 0) r = lm_step<T, MODE>(sub, st, pred);
    const bool ok = lm_finish<T, MODE>(st, r == 1, off, sig);
    if (fitval) {
#pragma unroll 1
        for (int q = 0; q < PKN; ++q)
            fitval[q] = lm_model<T, MODE>((float)(q / PKW - 2), (float)(q % PKW - 2), st.p);
    }
    return ok;
}

// Dispatch on the runtime fit type.  Types outside 4..6 are not LM fits.
template <int MODE>
__device__ __forceinline__ bool lm_fit_any(int type, const float *sub, float *off, float *sig, float *fitval)
{
    if (type == 6) return lm_fit<6, MODE>(sub, off, sig, fitval);
    if (type == 5) return lm_fit<5, MODE>(sub, off, sig, fitval);
    return lm_fit<4, MODE>(sub, off, sig, fitval);
}

// Sequential Westerweel search, used where plain reductions cannot reproduce the
// reference's scan order (a NaN in the search region) and for secondary peaks
// (peak_locate_lm.c:793-805).  plane(i, j) returns the value.
template <class Plane>
__device__ __forceinline__ float seq_search(const Plane &pl, int n0, int n1, int *bi, int *bj)
{
    float best = 0.0f;
    *bi = 0;
    *bj = 0;
    for (int i = n0 / 4; i < n0 * 3 / 4; ++i)
        for (int j = n1 / 4; j < n1 * 3 / 4; ++j) {
            float v = pl(i, j);
            if (v <= best) continue;
            bool mx = true;
            for (int a = -1; a <= 1 && mx; ++a)
                for (int b = -1; b <= 1; ++b)
                    if (pl(i + a, j + b) > v) { mx = false; break; }
            if (mx) { best = v; *bi = i; *bj = j; }
        }
    return best;
}

// Sequential detectability (peak_locate_lm.c:727-744).
template <class Plane>
__device__ __forceinline__ float seq_detectability(const Plane &pl, int n0, int n1)
{
    float p1 = 0.0f, p2 = 0.0f;
    for (int i = n0 / 4; i < n0 * 3 / 4; ++i)
        for (int j = n1 / 4; j < n1 * 3 / 4; ++j) {
            float v = pl(i, j);
            if (v <= p2 || v <= 0.0f) continue;
            bool mx = true;
            for (int a = -1; a <= 1 && mx; ++a)
                for (int b = -1; b <= 1; ++b)
                    if (pl(i + a, j + b) > v) { mx = false; break; }
            if (!mx) continue;
            if (v > p1) { p2 = p1; p1 = v; }
            else p2 = v;
        }
    return (p2 > 0.0f) ? fdiv(p1, p2) : 0.0f;
}

// Candidate test shared by the parallel searches: value, or -1 when (i, j) is not
// a positive non-strict 3x3 local maximum; *has_nan set if any value read is NaN.
template <class Plane>
__device__ __forceinline__ float candidate(const Plane &pl, int i, int j, bool *has_nan)
{
    float v = pl(i, j);
    bool nan = (v != v), mx = true;
#pragma unroll
    for (int a = -1; a <= 1; ++a)
#pragma unroll
        for (int b = -1; b <= 1; ++b) {
            float u = pl(i + a, j + b);
            nan |= (u != u);
            mx &= !(u > v);
        }
    *has_nan |= nan;
    return (mx && v > 0.0f) ? v : -1.0f;
}

// Running (argmax, top-2) state of the parallel search.
struct PeakAcc {
    float best;   // largest candidate value (0 if none)
    int idx;      // its row-major index (first on ties)
    float p1, p2; // two largest candidate values, with multiplicity
    __device__ __forceinline__ void init() { best = 0.0f; idx = 0x7fffffff; p1 = 0.0f; p2 = 0.0f; }
    __device__ __forceinline__ void add(float v, int k)
    {
        if (v <= 0.0f) return;
        if (v > best || (v == best && k < idx)) { best = v; idx = k; }
        if (v > p1) { p2 = p1; p1 = v; }
        else if (v > p2) p2 = v;
    }
    __device__ __forceinline__ void merge(float ob, int oi, float o1, float o2)
    {
        if (ob > best || (ob == best && oi < idx)) { best = ob; idx = oi; }
        float hi = fmaxf(p1, o1), lo = fminf(p1, o1);
        float second = fmaxf(lo, fmaxf(p2, o2));
        p1 = hi;
        p2 = second;
    }
};

}  // namespace piv
