/*
 * pivoracle.c -- CPU restatement of the PIVtools correlation hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA product (see pivoracle.h).
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 *
 * Every routine cites the reference routine it restates by file:line within the
 * reference project (pivtools_cli/lib/...).  Built with -ffp-contract=off so that
 * the float expressions are evaluated exactly in the order written, which is the
 * order the reference's scalar C evaluates them in.
 */
#include "pivoracle.h"

#include <complex.h>
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex zd;

#define ORC_ERR_NOMEM 1
#define ORC_ERR_NOPLAN_BWD 4
#define ORC_ERR_NOPLAN 8

/* ------------------------------------------------------------------------- */
/* FP64 mixed-radix (2, 3) FFT, unnormalised, sign -1 forward / +1 inverse.    */
/* ------------------------------------------------------------------------- */

#define ORC_MAXN 256

int orc_size_ok(int n)
{
    switch (n) {
    case 8: case 12: case 16: case 24: case 32: case 48: case 64: case 96: case 128:
        return 1;
    default:
        return 0;
    }
}

static int fft_len_ok(int n)
{
    if (n < 1 || n > ORC_MAXN) return 0;
    while (n % 2 == 0) n /= 2;
    while (n % 3 == 0) n /= 3;
    return n == 1;
}

/* Twiddle table for length n: tw[j] = exp(sign * 2*pi*i * j / n). */
static void twiddles(zd *tw, int n, int sign)
{
    for (int j = 0; j < n; ++j) {
        double a = 2.0 * M_PI * (double)j / (double)n;
        tw[j] = cos(a) + (double)sign * sin(a) * I;
    }
}

/* Decimation in time: y[0..n) = DFT of x[0], x[s], x[2s], ...  (tw for ntop). */
static void fft_rec(const zd *x, int n, int s, zd *y, const zd *tw, int ntop)
{
    if (n == 1) { y[0] = x[0]; return; }
    int r = (n % 2 == 0) ? 2 : 3;
    int m = n / r;
    for (int q = 0; q < r; ++q) fft_rec(x + q * s, m, s * r, y + q * m, tw, ntop);
    zd tmp[ORC_MAXN];
    int step = ntop / n;
    for (int k = 0; k < m; ++k)
        for (int p = 0; p < r; ++p) {
            zd acc = 0;
            for (int q = 0; q < r; ++q)
                acc += y[q * m + k] * tw[((long)step * q * (k + m * p)) % ntop];
            tmp[k + m * p] = acc;
        }
    memcpy(y, tmp, (size_t)n * sizeof(zd));
}

static void fft1(zd *x, int n, int stride, const zd *tw)
{
    zd in[ORC_MAXN], out[ORC_MAXN];
    for (int i = 0; i < n; ++i) in[i] = x[(size_t)i * stride];
    fft_rec(in, n, 1, out, tw, n);
    for (int i = 0; i < n; ++i) x[(size_t)i * stride] = out[i];
}

/* In-place 2-D transform of an h x w row-major array (rows, then columns). */
static void fft2(zd *x, int h, int w, int sign)
{
    zd twr[ORC_MAXN], twc[ORC_MAXN];
    twiddles(twr, w, sign);
    twiddles(twc, h, sign);
    for (int r = 0; r < h; ++r) fft1(x + (size_t)r * w, w, 1, twr);
    for (int c = 0; c < w; ++c) fft1(x + c, h, w, twc);
}

/* Circular cross-correlation (codelet_fft.c:153-192 and :335-352; the reference's
 * `xcorr_preplanned(a, b)` loads a into spectrum slot 0 and b into slot 1 and
 * emits fftshift(IFFT(spec0 .* conj(spec1)))/numel). */
static int xcorr_d(const double *a, const double *b, int h, int w, double *out)
{
    if (!fft_len_ok(h) || !fft_len_ok(w) || (h & 1) || (w & 1)) return ORC_ERR_NOPLAN_BWD;
    size_t n = (size_t)h * w;
    zd *fa = (zd *)malloc(n * sizeof(zd));
    zd *fb = (zd *)malloc(n * sizeof(zd));
    if (!fa || !fb) { free(fa); free(fb); return ORC_ERR_NOMEM; }
    for (size_t i = 0; i < n; ++i) { fa[i] = a[i]; fb[i] = b[i]; }
    fft2(fa, h, w, -1);
    fft2(fb, h, w, -1);
    for (size_t i = 0; i < n; ++i) fa[i] = fa[i] * conj(fb[i]);
    fft2(fa, h, w, +1);
    const double inv = 1.0 / (double)n;
    for (int r = 0; r < h; ++r)
        for (int c = 0; c < w; ++c)
            out[(size_t)r * w + c] =
                creal(fa[(size_t)((r + h / 2) % h) * w + (c + w / 2) % w]) * inv;
    free(fa);
    free(fb);
    return 0;
}

int orc_xcorr_plane(const float *a, const float *b, int h, int w, double *out)
{
    size_t n = (size_t)h * w;
    double *ad = (double *)malloc(n * sizeof(double));
    double *bd = (double *)malloc(n * sizeof(double));
    if (!ad || !bd) { free(ad); free(bd); return ORC_ERR_NOMEM; }
    for (size_t i = 0; i < n; ++i) { ad[i] = a[i]; bd[i] = b[i]; }
    int e = xcorr_d(ad, bd, h, w, out);
    free(ad);
    free(bd);
    return e;
}

/* numel / (W (*) W): the weight's linear autocorrelation at shift
 * (r - h/2, c - w/2), formed on a 2h x 2w zero-padded grid (xcorr.c:55-122),
 * then PIV_2d_cross_correlate.c:222's float division. */
int orc_correl_weight(const float *wt, int h, int w, float *out)
{
    int H2 = 2 * h, W2 = 2 * w;
    size_t n2 = (size_t)H2 * W2;
    double *p = (double *)calloc(n2, sizeof(double));
    double *c = (double *)malloc(n2 * sizeof(double));
    if (!p || !c) { free(p); free(c); return ORC_ERR_NOMEM; }
    for (int r = 0; r < h; ++r)
        for (int q = 0; q < w; ++q)
            p[(size_t)(r + h / 2) * W2 + q + w / 2] = wt[(size_t)r * w + q];
    int e = xcorr_d(p, p, H2, W2, c);
    if (!e) {
        const float numel = (float)(h * w);
        for (int r = 0; r < h; ++r)
            for (int q = 0; q < w; ++q) {
                float conv = (float)c[(size_t)(r + h / 2) * W2 + q + w / 2];
                out[(size_t)r * w + q] = numel / conv;
            }
    }
    free(p);
    free(c);
    return e;
}

/* ------------------------------------------------------------------------- */
/* Peak fitter (peak_locate_lm.c and peak_locate_lm_batch.c).                 */
/* ------------------------------------------------------------------------- */

#define PK 5
#define NSUB (PK * PK)

/* The batch fitter's exponential (peak_simd.h pk_vexpf): Cody-Waite range
 * reduction with a magic-number round, degree-5 polynomial, exponent-field 2^n. */
static float cephes_expf(float x)
{
    const float lo = -87.3365478515625f;
    float xc = (x > lo) ? x : lo;
    float rn = (1.44269504088896341f * xc + 12582912.0f) - 12582912.0f;
    int n = (int)rn;
    float r = xc - rn * 0.693359375f - rn * -2.12194440e-4f;
    float r2 = r * r;
    float p = 1.9875691500e-4f;
    p = p * r + 1.3981999507e-3f;
    p = p * r + 8.3334519073e-3f;
    p = p * r + 4.1665795894e-2f;
    p = p * r + 1.6666665459e-1f;
    p = p * r + 5.0000001201e-1f;
    float er = p * r2 + r + 1.0f;
    int32_t bits = (int32_t)((uint32_t)(n + 127) << 23);
    float s;
    memcpy(&s, &bits, 4);
    return er * s;
}

typedef struct {
    int mode;   /* 0 scalar fitter, 1 batch fitter */
} fit_cfg;

static inline float fexp(const fit_cfg *c, float x) { return c->mode ? cephes_expf(x) : expf(x); }
/* clamp helpers: fminf/fmaxf in the scalar fitter, compare-select in the batch */
static inline float cmax(const fit_cfg *c, float a, float b) { return c->mode ? (a > b ? a : b) : fmaxf(a, b); }
static inline float cmin(const fit_cfg *c, float a, float b) { return c->mode ? (a < b ? a : b) : fminf(a, b); }

/* peak_locate_lm.c:35-66 (3-point log-parabola on the centre of an N-plane) */
static void three_point(const float *x, const int *N, float *loc, float *A, float *sx, float *sy)
{
    float xf[3], yf[3];
    int cr = (N[0] - 1) / 2, cc = (N[1] - 1) / 2;
    for (int i = 0; i < 3; ++i) {
        xf[i] = x[(i - 1 + cr) * N[1] + cc];
        yf[i] = x[cr * N[1] + (i - 1 + cc)];
        xf[i] = (float)log((xf[i] < FLT_EPSILON) ? FLT_EPSILON : xf[i]);
        yf[i] = (float)log((yf[i] < FLT_EPSILON) ? FLT_EPSILON : yf[i]);
    }
    float dx = 2 * xf[0] - 4 * xf[1] + 2 * xf[2];
    float dy = 2 * yf[0] - 4 * yf[1] + 2 * yf[2];
    loc[0] = (fabs(dx) > FLT_EPSILON) ? (xf[0] - xf[2]) / dx : 0.0f;
    loc[1] = (fabs(dy) > FLT_EPSILON) ? (yf[0] - yf[2]) / dy : 0.0f;
    *A = x[cr * N[1] + cc];
    *sx = (float)sqrt(-4.0f / (dx + FLT_EPSILON));
    *sy = (float)sqrt(-4.0f / (dy + FLT_EPSILON));
}

/* Model value of fit type t at patch pixel (i, j); prm = {A, i0, j0, s1, s2, s3}. */
static inline float model(const fit_cfg *c, int t, float i, float j, const float *p)
{
    if (t == 4) {
        float di = (i - p[1]) / p[3], dj = (j - p[2]) / p[3];
        return p[0] * fexp(c, -(di * di + dj * dj));
    } else if (t == 5) {
        float di = (i - p[1]) / p[3], dj = (j - p[2]) / p[4];
        return p[0] * fexp(c, -(di * di + dj * dj));
    } else {
        float di = i - p[1], dj = j - p[2];
        return p[0] * fexp(c, -0.5f * (di * di / p[3] + dj * dj / p[4] + 2.0f * di * dj * p[5]));
    }
}

/* Residual pass (peak_locate_lm.c:108-137 and twins): fills pred, FP64 sum. */
static double resid_pass(const fit_cfg *c, int t, const float *sub, const float *p, float *pred)
{
    double rs = 0.0;
    for (int q = 0; q < NSUB; ++q) {
        float i = (float)(q / PK - 2), j = (float)(q % PK - 2);
        float v = model(c, t, i, j, p);
        pred[q] = v;
        float r = v - sub[q];
        rs += (double)r * (double)r;
    }
    return rs;
}

/* Jacobian pass from the cached model values (peak_locate_lm.c:139-183 and twins). */
static void jac_pass(int t, const float *sub, const float *p, const float *pred, double *JtJ, double *Jtr, int n)
{
    memset(JtJ, 0, sizeof(double) * 36);
    memset(Jtr, 0, sizeof(double) * 6);
    for (int q = 0; q < NSUB; ++q) {
        float i = (float)(q / PK - 2), j = (float)(q % PK - 2);
        float v = pred[q];
        float r = v - sub[q];
        float J[6];
        if (t == 4) {
            float di = (i - p[1]) / p[3], dj = (j - p[2]) / p[3];
            float r2 = di * di + dj * dj;
            J[0] = v / p[0];
            J[1] = 2.0f * v * di / p[3];
            J[2] = 2.0f * v * dj / p[3];
            J[3] = 2.0f * v * r2 / p[3];
        } else if (t == 5) {
            float di = (i - p[1]) / p[3], dj = (j - p[2]) / p[4];
            J[0] = v / p[0];
            J[1] = 2.0f * v * di / p[3];
            J[2] = 2.0f * v * dj / p[4];
            J[3] = 2.0f * v * di * di / p[3];
            J[4] = 2.0f * v * dj * dj / p[4];
        } else {
            float di = i - p[1], dj = j - p[2];
            J[0] = v / p[0];
            J[1] = v * (di / p[3] + dj * p[5]);
            J[2] = v * (dj / p[4] + di * p[5]);
            J[3] = 0.5f * v * di * di / (p[3] * p[3]);
            J[4] = 0.5f * v * dj * dj / (p[4] * p[4]);
            J[5] = -v * di * dj;
        }
        for (int a = 0; a < n; ++a) {
            Jtr[a] += (double)J[a] * (double)r;
            for (int b = 0; b <= a; ++b) JtJ[a * n + b] += (double)J[a] * (double)J[b];
        }
    }
    for (int a = 0; a < n; ++a)
        for (int b = a + 1; b < n; ++b) JtJ[a * n + b] = JtJ[b * n + a];
}

/* (JtJ + lambda diag JtJ) d = -Jtr by FP64 Cholesky (peak_locate_lm.c:342-393). */
static int lm_step(const double *JtJ, const double *Jtr, float lambda, float *delta, int n)
{
    double A[36], L[36], y[6], d[6];
    memcpy(A, JtJ, sizeof(double) * n * n);
    for (int i = 0; i < n; ++i) A[i * n + i] *= (1.0 + (double)lambda);
    memset(L, 0, sizeof L);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j <= i; ++j) {
            double s = A[i * n + j];
            for (int k = 0; k < j; ++k) s -= L[i * n + k] * L[j * n + k];
            if (i == j) {
                if (s <= 0.0) return -1;
                L[i * n + i] = sqrt(s);
            } else {
                L[i * n + j] = s / L[j * n + j];
            }
        }
    for (int i = 0; i < n; ++i) {
        double s = -Jtr[i];
        for (int j = 0; j < i; ++j) s -= L[i * n + j] * y[j];
        y[i] = s / L[i * n + i];
    }
    for (int i = n - 1; i >= 0; --i) {
        double s = y[i];
        for (int j = i + 1; j < n; ++j) s -= L[j * n + i] * d[j];
        d[i] = s / L[i * n + i];
    }
    for (int i = 0; i < n; ++i) delta[i] = (float)d[i];
    return 0;
}

/* Marquardt loop shared by gauss4/5/6 (peak_locate_lm.c:412-712; lockstep twin
 * peak_locate_lm_batch.c:362-588).  Returns 0 = trusted, -1 = failed.  sub is the
 * compensated 5x5 patch.  Writes the centre offsets and widths. */
static int lm_fit(const fit_cfg *c, int t, const float *sub, float *off, float *sig, float *fitval)
{
    const int N5[2] = {PK, PK};
    int n = (t == 4) ? 4 : (t == 5 ? 5 : 6);
    float p[6] = {0, 0, 0, 0, 0, 0};
    float pk[2], A, sx, sy;
    three_point(sub, N5, pk, &A, &sx, &sy);
    p[0] = A;
    p[1] = fminf(fmaxf(pk[0], -2.0f), 2.0f);
    p[2] = fminf(fmaxf(pk[1], -2.0f), 2.0f);
    if (t == 4) {
        float s = sqrtf(sx * sx + sy * sy);
        p[3] = fminf(fmaxf(s, 0.5f), 3.0f);
    } else if (t == 5) {
        p[3] = fminf(fmaxf(sx, 0.5f), 3.0f);
        p[4] = fminf(fmaxf(sy, 0.5f), 3.0f);
    } else {
        p[3] = fminf(fmaxf(sx * sx, 0.25f), 9.0f);
        p[4] = fminf(fmaxf(sy * sy, 0.25f), 9.0f);
        p[5] = 0.0f;
    }
    float pred[NSUB];
    double JtJ[36], Jtr[6];
    float delta[6];
    float lambda = 0.01f;
    int ok = 0;
    double resid = resid_pass(c, t, sub, p, pred);
    jac_pass(t, sub, p, pred, JtJ, Jtr, n);
    for (int it = 0; it < 50; ++it) {
        if (lm_step(JtJ, Jtr, lambda, delta, n) != 0) break;
        float q[6];
        for (int k = 0; k < 6; ++k) q[k] = p[k];
        for (int k = 0; k < n; ++k) q[k] = p[k] + delta[k];
        q[0] = cmax(c, q[0], p[0] * 0.5f);
        q[1] = cmin(c, cmax(c, q[1], -2.5f), 2.5f);
        q[2] = cmin(c, cmax(c, q[2], -2.5f), 2.5f);
        if (t == 4) {
            q[3] = cmin(c, cmax(c, q[3], 0.25f), 4.0f);
        } else if (t == 5) {
            q[3] = cmin(c, cmax(c, q[3], 0.25f), 4.0f);
            q[4] = cmin(c, cmax(c, q[4], 0.25f), 4.0f);
        } else {
            q[3] = cmin(c, cmax(c, q[3], 0.1f), 16.0f);
            q[4] = cmin(c, cmax(c, q[4], 0.1f), 16.0f);
            float smax = c->mode ? 0.95f / sqrtf(q[3] * q[4]) : 0.95f / sqrtf(q[3] * q[4]);
            q[5] = cmin(c, cmax(c, q[5], -smax), smax);
        }
        double nr = resid_pass(c, t, sub, q, pred);
        if (nr < resid) {
            for (int k = 0; k < 6; ++k) p[k] = q[k];
            double improve = (resid - nr) / (resid + FLT_EPSILON);
            resid = nr;
            lambda *= 0.5f;
            jac_pass(t, sub, p, pred, JtJ, Jtr, n);
            if (improve < 1e-6) { ok = 1; break; }
        } else {
            lambda *= 2.0f;
            if (lambda > 1e6f) break;
        }
    }
    if (!ok) {
        if (c->mode)
            ok = resid <= (double)((1e-3f * (float)NSUB) * p[0] * p[0]);
        else
            ok = resid <= 1e-3f * p[0] * p[0] * (float)NSUB;
    }
    if (ok) {
        if (t == 6) ok = (p[3] > 0.1f && p[3] < 16.0f && p[4] > 0.1f && p[4] < 16.0f);
        else if (t == 5) ok = (p[3] > 0.25f && p[3] < 4.0f && p[4] > 0.25f && p[4] < 4.0f);
        else ok = (p[3] > 0.25f && p[3] < 4.0f);
    }
    off[0] = p[1];
    off[1] = p[2];
    if (t == 4) { sig[0] = p[3]; sig[1] = p[3]; sig[2] = 0.0f; }
    else if (t == 5) { sig[0] = p[3]; sig[1] = p[4]; sig[2] = 0.0f; }
    else { sig[0] = p[3]; sig[1] = p[4]; sig[2] = p[5]; }
    if (fitval)
        for (int q = 0; q < NSUB; ++q)
            fitval[q] = model(c, t, (float)(q / PK - 2), (float)(q % PK - 2), p);
    return ok ? 0 : -1;
}

void orc_lsqpeaklocate_lm(const float *xc, const int *N, float *loc, int nPeaks, int fit,
                          float *sd, const float *wt, int exp_mode)
{
    fit_cfg cfg = {exp_mode ? 1 : 0};
    size_t np = (size_t)N[0] * N[1];
    float *work = NULL;
    const float *src = xc;
    if (nPeaks > 1) {
        work = (float *)malloc(np * sizeof(float));
        memcpy(work, xc, np * sizeof(float));
        src = work;
    }
    for (int k = 0; k < nPeaks; ++k) {
        /* search: largest non-strict 3x3 local max in the quarter region,
         * first in row-major order on ties (peak_locate_lm.c:793-805) */
        int bi = 0, bj = 0;
        float best = 0;
        for (int i = N[0] / 4; i < N[0] * 3 / 4; ++i)
            for (int j = N[1] / 4; j < N[1] * 3 / 4; ++j) {
                float v = src[i * N[1] + j];
                if (v <= best) continue;
                int mx = 1;
                for (int a = -1; a <= 1 && mx; ++a)
                    for (int b = -1; b <= 1; ++b)
                        if (src[(i + a) * N[1] + j + b] > v) { mx = 0; break; }
                if (mx) { best = v; bi = i; bj = j; }
            }
        if (best <= 0 || bi < 2 || bi >= N[0] - 2 || bj < 2 || bj >= N[1] - 2) {
            loc[0 * nPeaks + k] = NAN;
            loc[1 * nPeaks + k] = NAN;
            loc[2 * nPeaks + k] = 0;
            sd[0 * nPeaks + k] = 0;
            sd[1 * nPeaks + k] = 0;
            sd[2 * nPeaks + k] = 0;
            continue;
        }
        float sub[NSUB], fv[NSUB], off[2], sig[3];
        for (int a = 0; a < PK; ++a)
            for (int b = 0; b < PK; ++b) {
                size_t idx = (size_t)(bi + a - 2) * N[1] + (bj + b - 2);
                sub[a * PK + b] = wt ? src[idx] * wt[idx] : src[idx];
            }
        int st = 0;
        const int N5[2] = {PK, PK};
        if (k == 0 && fit >= 4 && fit <= 6) {
            st = lm_fit(&cfg, fit, sub, off, sig, fv);
        } else {
            float A, sx, sy;
            three_point(sub, N5, off, &A, &sx, &sy);
            sig[0] = sx; sig[1] = sy; sig[2] = 0.0f;
            if (nPeaks > 1)
                for (int q = 0; q < NSUB; ++q) {
                    float di = ((float)(q / PK - 2) - off[0]) / sx;
                    float dj = ((float)(q % PK - 2) - off[1]) / sy;
                    fv[q] = A * expf(-(di * di + dj * dj));
                }
        }
        if (st != 0) {
            loc[0 * nPeaks + k] = NAN;
            loc[1 * nPeaks + k] = NAN;
            loc[2 * nPeaks + k] = 0;
            sd[0 * nPeaks + k] = 0;
            sd[1 * nPeaks + k] = 0;
            sd[2 * nPeaks + k] = 0;
        } else {
            loc[0 * nPeaks + k] = off[0] + bi;
            loc[1 * nPeaks + k] = off[1] + bj;
            loc[2 * nPeaks + k] = best;
            sd[0 * nPeaks + k] = sig[0];
            sd[1 * nPeaks + k] = sig[1];
            sd[2 * nPeaks + k] = sig[2];
        }
        if (nPeaks > 1)
            for (int a = 0; a < PK; ++a)
                for (int b = 0; b < PK; ++b) {
                    size_t idx = (size_t)(bi + a - 2) * N[1] + (bj + b - 2);
                    float f = fv[a * PK + b];
                    if (wt) f /= wt[idx];
                    float d = work[idx] - f;
                    work[idx] = (0 > d) ? 0 : d;
                }
    }
    free(work);
}

float orc_peak_detectability(const float *x, const int *N)
{
    float p1 = 0.0f, p2 = 0.0f;
    for (int i = N[0] / 4; i < N[0] * 3 / 4; ++i)
        for (int j = N[1] / 4; j < N[1] * 3 / 4; ++j) {
            float v = x[i * N[1] + j];
            if (v <= p2 || v <= 0.0f) continue;
            int mx = 1;
            for (int a = -1; a <= 1 && mx; ++a)
                for (int b = -1; b <= 1; ++b)
                    if (x[(i + a) * N[1] + j + b] > v) { mx = 0; break; }
            if (!mx) continue;
            if (v > p1) { p2 = p1; p1 = v; }
            else p2 = v;
        }
    return (p2 > 0.0f) ? p1 / p2 : 0.0f;
}

/* ------------------------------------------------------------------------- */
/* bulkxcorr2d (PIV_2d_cross_correlate.c:203-397)                             */
/* ------------------------------------------------------------------------- */

unsigned char orc_bulkxcorr2d(const float *A, const float *B, const float *mask,
                              const int *img_size, int n_images, const float *ctr_x,
                              const float *ctr_y, const int *n_win, const float *wA,
                              int ensemble, const float *wB, const int *ws, int n_peaks,
                              int finder, float *pk_x, float *pk_y, float *pk_h, float *sx,
                              float *sy, float *sxy, float *pk_ratio, float *plane_out,
                              double *planes_f64, int impl, int n_threads)
{
    const int h = ws[0], w = ws[1];
    if (!orc_size_ok(h) || !orc_size_ok(w)) return ORC_ERR_NOPLAN_BWD;
    const int nwt = n_win[0] * n_win[1];
    const int npx = h * w;
    const int H = img_size[0], W = img_size[1];
    float *cw = (float *)malloc((size_t)npx * sizeof(float));
    if (!cw) return ORC_ERR_NOMEM;
    if (orc_correl_weight(wB, h, w, cw)) { free(cw); return ORC_ERR_NOMEM; }
    const long total = (long)n_images * nwt;
    int err = 0;
#ifdef _OPENMP
    int nt = n_threads > 0 ? n_threads : omp_get_max_threads();
#pragma omp parallel num_threads(nt) reduction(| : err)
#endif
    {
        float *pa = (float *)malloc((size_t)npx * sizeof(float));
        float *pb = (float *)malloc((size_t)npx * sizeof(float));
        double *pl = (double *)malloc((size_t)npx * sizeof(double));
        float *plf = (float *)malloc((size_t)npx * sizeof(float));
        float *loc = (float *)malloc((size_t)3 * n_peaks * sizeof(float));
        float *sd = (float *)malloc((size_t)3 * n_peaks * sizeof(float));
        if (!pa || !pb || !pl || !plf || !loc || !sd) err = ORC_ERR_NOMEM;
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (long idx = 0; idx < total; ++idx) {
            if (err) continue;
            int n = (int)(idx / nwt), iw = (int)(idx % nwt);
            int ii = iw % n_win[1], jj = iw / n_win[1];
            if (mask[jj * n_win[1] + ii] == 1) continue;
            int r0 = (int)floor(ctr_y[jj] - ((float)h - 1.0) / 2.0 + 0.5);
            int c0 = (int)floor(ctr_x[ii] - ((float)w - 1.0) / 2.0 + 0.5);
            if (r0 < 0 || c0 < 0 || r0 + h > H || c0 + w > W) continue;
            const float *ia = A + (size_t)n * H * W, *ib = B + (size_t)n * H * W;
            for (int i = 0; i < h; ++i)
                for (int j = 0; j < w; ++j) {
                    pa[i * w + j] = ia[(size_t)(r0 + i) * W + c0 + j];
                    pb[i * w + j] = ib[(size_t)(r0 + i) * W + c0 + j];
                }
            float ma = 0.0f, mb = 0.0f;
            for (int i = 0; i < npx; ++i) {
                pa[i] *= wA[i];
                pb[i] *= wB[i];
                ma += pa[i];
                mb += pb[i];
            }
            ma /= npx;
            mb /= npx;
            float ea = 0.0f, eb = 0.0f;
            for (int i = 0; i < npx; ++i) {
                if (!ensemble) { pa[i] -= ma; pb[i] -= mb; }
                ea += pa[i] * pa[i];
                eb += pb[i] * pb[i];
            }
            float enorm = 1.0f / sqrtf(ea * eb);
            if (orc_xcorr_plane(pb, pa, h, w, pl)) { err = ORC_ERR_NOMEM; continue; }
            for (int i = 0; i < npx; ++i) plf[i] = (float)pl[i];
            if (plane_out) memcpy(plane_out + (size_t)idx * npx, plf, (size_t)npx * sizeof(float));
            if (planes_f64) memcpy(planes_f64 + (size_t)idx * npx, pl, (size_t)npx * sizeof(double));
            if (ensemble) continue;
            int mode = (impl && n_peaks == 1 && finder >= 4) ? 1 : 0;
            orc_lsqpeaklocate_lm(plf, ws, loc, n_peaks, finder, sd, cw, mode);
            pk_ratio[(size_t)n * nwt + iw] = orc_peak_detectability(plf, ws);
            for (int k = 0; k < n_peaks; ++k) {
                size_t o = (size_t)n * n_peaks * nwt + (size_t)k * nwt + iw;
                pk_x[o] = loc[1 * n_peaks + k] - w / 2.0f;
                pk_y[o] = loc[0 * n_peaks + k] - h / 2.0f;
                sx[o] = sd[0 * n_peaks + k];
                sy[o] = sd[1 * n_peaks + k];
                sxy[o] = sd[2 * n_peaks + k];
                pk_h[o] = loc[2 * n_peaks + k] * enorm;
            }
        }
        free(pa); free(pb); free(pl); free(plf); free(loc); free(sd);
    }
    free(cw);
    return (unsigned char)err;
}

/* ------------------------------------------------------------------------- */
/* Ensemble accumulation (PIV_2d_cross_correlate.c:403-484, 502-833)          */
/* ------------------------------------------------------------------------- */

static int window_origin_f(float ctr, int n)
{
    return (int)floor(ctr - ((float)n - 1.0f) / 2.0f + 0.5f);
}

unsigned char orc_accumulate_triple(const float *A, const float *B, const float *mask,
                                    const int *img_size, int n_images, const float *ctr_x,
                                    const float *ctr_y, const int *n_win, const float *wa_ab,
                                    const float *wb_ab, const float *waa, const float *wbb,
                                    const int *ws, const int *fs, int mean_sub, int ppn,
                                    float *ab, float *aa, float *bb, int n_threads)
{
    const int h = ws[0], w = ws[1];
    if (!orc_size_ok(h) || !orc_size_ok(w)) return ORC_ERR_NOPLAN_BWD;
    const int oh = fs ? fs[0] : h, ow = fs ? fs[1] : w;
    const int sy0 = (h - oh) / 2, sx0 = (w - ow) / 2;
    const int npx = h * w, nout = oh * ow, nwt = n_win[0] * n_win[1];
    const int H = img_size[0], W = img_size[1];
    float swb = 0.0f, swa_auto = 0.0f, swb_auto = 0.0f;
    if (mean_sub)
        for (int i = 0; i < npx; ++i) { swb += wb_ab[i]; swa_auto += waa[i]; swb_auto += wbb[i]; }
    int err = 0;
#ifdef _OPENMP
    int nt = n_threads > 0 ? n_threads : omp_get_max_threads();
#pragma omp parallel num_threads(nt) reduction(| : err)
#endif
    {
        double *x1 = (double *)malloc(sizeof(double) * npx), *x2 = (double *)malloc(sizeof(double) * npx);
        double *x3 = (double *)malloc(sizeof(double) * npx), *x4 = (double *)malloc(sizeof(double) * npx);
        double *pab = (double *)malloc(sizeof(double) * npx), *paa = (double *)malloc(sizeof(double) * npx);
        double *pbb = (double *)malloc(sizeof(double) * npx);
        double *sab = (double *)malloc(sizeof(double) * nout), *saa = (double *)malloc(sizeof(double) * nout);
        double *sbb = (double *)malloc(sizeof(double) * nout);
        float *ra = (float *)malloc(sizeof(float) * npx), *rb = (float *)malloc(sizeof(float) * npx);
        if (!x1 || !x2 || !x3 || !x4 || !pab || !paa || !pbb || !sab || !saa || !sbb || !ra || !rb)
            err = ORC_ERR_NOMEM;
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (int iw = 0; iw < nwt; ++iw) {
            if (err) continue;
            int ii = iw % n_win[1], jj = iw / n_win[1];
            if (mask[iw] == 1) continue;
            int r0 = window_origin_f(ctr_y[jj], h), c0 = window_origin_f(ctr_x[ii], w);
            if (r0 < 0 || c0 < 0 || r0 + h > H || c0 + w > W) continue;
            memset(sab, 0, sizeof(double) * nout);
            memset(saa, 0, sizeof(double) * nout);
            memset(sbb, 0, sizeof(double) * nout);
            for (int n = 0; n < n_images; ++n) {
                const float *ia = A + (size_t)n * H * W, *ib = B + (size_t)n * H * W;
                for (int i = 0; i < h; ++i)
                    for (int j = 0; j < w; ++j) {
                        ra[i * w + j] = ia[(size_t)(r0 + i) * W + c0 + j];
                        rb[i * w + j] = ib[(size_t)(r0 + i) * W + c0 + j];
                    }
                float m_abb = 0.0f, m_aa = 0.0f, m_bb = 0.0f;
                if (mean_sub) {
                    float s1 = 0.0f, s2 = 0.0f, s3 = 0.0f;
                    for (int i = 0; i < npx; ++i) {
                        s1 += rb[i] * wb_ab[i];
                        s2 += ra[i] * waa[i];
                        s3 += rb[i] * wbb[i];
                    }
                    m_abb = (swb > 0.0f) ? s1 / swb : 0.0f;
                    m_aa = (swa_auto > 0.0f) ? s2 / swa_auto : 0.0f;
                    m_bb = (swb_auto > 0.0f) ? s3 / swb_auto : 0.0f;
                }
                float eaa = 0.0f, ebb = 0.0f;
                for (int i = 0; i < npx; ++i) {
                    float vb = (rb[i] - m_abb) * wb_ab[i];
                    float va = (ra[i] - m_aa) * wa_ab[i];
                    float vaa = (ra[i] - m_aa) * waa[i];
                    float vbb = (rb[i] - m_bb) * wbb[i];
                    x1[i] = vb; x2[i] = va; x3[i] = vaa; x4[i] = vbb;
                    eaa += vaa * vaa;
                    ebb += vbb * vbb;
                }
                float s_ab = 1.0f, s_aa = 1.0f, s_bb = 1.0f;
                if (ppn) {
                    if (eaa <= 0.0f || ebb <= 0.0f) continue;
                    s_ab = 1.0f / sqrtf(eaa * ebb);
                    s_aa = 1.0f / eaa;
                    s_bb = 1.0f / ebb;
                }
                if (xcorr_d(x1, x2, h, w, pab) || xcorr_d(x3, x3, h, w, paa) ||
                    xcorr_d(x4, x4, h, w, pbb)) { err = ORC_ERR_NOMEM; break; }
                for (int i = 0; i < oh; ++i)
                    for (int j = 0; j < ow; ++j) {
                        int src = (sy0 + i) * w + sx0 + j;
                        sab[i * ow + j] += (double)s_ab * pab[src];
                        saa[i * ow + j] += (double)s_aa * paa[src];
                        sbb[i * ow + j] += (double)s_bb * pbb[src];
                    }
            }
            for (int i = 0; i < nout; ++i) {
                ab[(size_t)iw * nout + i] += (float)sab[i];
                aa[(size_t)iw * nout + i] += (float)saa[i];
                bb[(size_t)iw * nout + i] += (float)sbb[i];
            }
        }
        free(x1); free(x2); free(x3); free(x4); free(pab); free(paa); free(pbb);
        free(sab); free(saa); free(sbb); free(ra); free(rb);
    }
    return (unsigned char)err;
}

unsigned char orc_accumulate(const float *A, const float *B, const float *mask,
                             const int *img_size, int n_images, const float *ctr_x,
                             const float *ctr_y, const int *n_win, const float *wA,
                             const float *wB, const int *ws, const int *fs, float *sum,
                             int n_threads)
{
    const int h = ws[0], w = ws[1];
    if (!orc_size_ok(h) || !orc_size_ok(w)) return ORC_ERR_NOPLAN_BWD;
    const int oh = fs ? fs[0] : h, ow = fs ? fs[1] : w;
    const int sy0 = (h - oh) / 2, sx0 = (w - ow) / 2;
    const int npx = h * w, nout = oh * ow, nwt = n_win[0] * n_win[1];
    const int H = img_size[0], W = img_size[1];
    int err = 0;
#ifdef _OPENMP
    int nt = n_threads > 0 ? n_threads : omp_get_max_threads();
#pragma omp parallel num_threads(nt) reduction(| : err)
#endif
    {
        double *xa = (double *)malloc(sizeof(double) * npx), *xb = (double *)malloc(sizeof(double) * npx);
        double *pl = (double *)malloc(sizeof(double) * npx), *acc = (double *)malloc(sizeof(double) * nout);
        if (!xa || !xb || !pl || !acc) err = ORC_ERR_NOMEM;
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (int iw = 0; iw < nwt; ++iw) {
            if (err) continue;
            int ii = iw % n_win[1], jj = iw / n_win[1];
            if (mask[iw] == 1) continue;
            int r0 = window_origin_f(ctr_y[jj], h), c0 = window_origin_f(ctr_x[ii], w);
            if (r0 < 0 || c0 < 0 || r0 + h > H || c0 + w > W) continue;
            memset(acc, 0, sizeof(double) * nout);
            for (int n = 0; n < n_images; ++n) {
                const float *ia = A + (size_t)n * H * W, *ib = B + (size_t)n * H * W;
                for (int i = 0; i < h; ++i)
                    for (int j = 0; j < w; ++j) {
                        int k = i * w + j;
                        xa[k] = ia[(size_t)(r0 + i) * W + c0 + j] * wA[k];
                        xb[k] = ib[(size_t)(r0 + i) * W + c0 + j] * wB[k];
                    }
                /* product rounded to float, as the reference stores it */
                for (int k = 0; k < npx; ++k) { xa[k] = (float)xa[k]; xb[k] = (float)xb[k]; }
                if (xcorr_d(xb, xa, h, w, pl)) { err = ORC_ERR_NOMEM; break; }
                for (int i = 0; i < oh; ++i)
                    for (int j = 0; j < ow; ++j) acc[i * ow + j] += pl[(sy0 + i) * w + sx0 + j];
            }
            for (int i = 0; i < nout; ++i) sum[(size_t)iw * nout + i] += (float)acc[i];
        }
        free(xa); free(xb); free(pl); free(acc);
    }
    return (unsigned char)err;
}

/* ------------------------------------------------------------------------- */
/* Fused symmetric warp, scalar route (fused_warp.c)                          */
/* ------------------------------------------------------------------------- */

static void keys4(float d, float *w)
{
    float s0 = 1.0f + d, q2 = 1.0f - d, s3 = 2.0f - d;
    w[1] = (1.25f * d - 2.25f) * d * d + 1.0f;
    w[2] = (1.25f * q2 - 2.25f) * q2 * q2 + 1.0f;
    w[0] = ((-0.75f * s0 + 3.75f) * s0 - 6.0f) * s0 + 3.0f;
    w[3] = ((-0.75f * s3 + 3.75f) * s3 - 6.0f) * s3 + 3.0f;
}

static float bicubic_zero(const float *img, float fy, float fx, int H, int W)
{
    float fyf = floorf(fy), fxf = floorf(fx);
    int iy = (int)fyf - 1, ix = (int)fxf - 1;
    float wy[4], wx[4], v = 0.0f;
    keys4(fy - fyf, wy);
    keys4(fx - fxf, wx);
    for (int m = 0; m < 4; ++m) {
        int r = iy + m;
        if (r < 0 || r >= H) continue;
        for (int n = 0; n < 4; ++n) {
            int c = ix + n;
            if (c < 0 || c >= W) continue;
            v += wy[m] * wx[n] * img[(size_t)r * W + c];
        }
    }
    return v;
}

static float lanczos3(float t)
{
    float at = fabsf(t);
    if (at < 1e-6f) return 1.0f;
    if (at >= 3.0f) return 0.0f;
    float pt = (float)M_PI * at;
    float pta = pt / 3.0f;
    return (sinf(pt) / pt) * (sinf(pta) / pta);
}

#define LUTN 4096

static float lanczos_sample(const float *img, float fy, float fx, int H, int W, const float (*lut)[6])
{
    float fyf = floorf(fy), fxf = floorf(fx);
    int iy = (int)fyf - 2, ix = (int)fxf - 2;
    float wy[6], wx[6], v = 0.0f;
    float ds[2] = {fy - fyf, fx - fxf};
    for (int a = 0; a < 2; ++a) {
        float pos = ds[a] * (float)LUTN;
        int k = (int)pos;
        float fr = pos - (float)k;
        if (k >= LUTN) { k = LUTN - 1; fr = 0.0f; }
        float *o = a ? wx : wy;
        for (int q = 0; q < 6; ++q) o[q] = lut[k][q] + fr * (lut[k + 1][q] - lut[k][q]);
    }
    for (int m = 0; m < 6; ++m) {
        int r = iy + m;
        if (r < 0 || r >= H) continue;
        for (int n = 0; n < 6; ++n) {
            int c = ix + n;
            if (c < 0 || c >= W) continue;
            v += wy[m] * wx[n] * img[(size_t)r * W + c];
        }
    }
    return v;
}

/* np.interp(pixel, ctrs, arange) with end clamps (fused_warp.c:259-307) */
static void pred_index(float *lut, int n, const float *c, int nc)
{
    if (nc == 1) { for (int p = 0; p < n; ++p) lut[p] = 0.0f; return; }
    int seg = 0;
    for (int p = 0; p < n; ++p) {
        float x = (float)p;
        if (x <= c[0]) { lut[p] = 0.0f; continue; }
        if (x >= c[nc - 1]) { lut[p] = (float)(nc - 1); continue; }
        while (seg < nc - 2 && c[seg + 1] < x) seg++;
        float den = c[seg + 1] - c[seg];
        if (den < 1e-12f) { lut[p] = (float)seg; continue; }
        lut[p] = (float)seg + (x - c[seg]) / den;
    }
}

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

int orc_fused_warp_batch(const float *ia, const float *ib, float *oa, float *ob,
                         const float *pdy, const float *pdx, int N, int H, int W, int nPY,
                         int nPX, const float *cy, const float *cx, int mode, int shared,
                         int round_shifts, int n_threads)
{
    if (N <= 0 || H <= 0 || W <= 0 || nPY <= 0 || nPX <= 0) return 1;
    if (!ia || !ib || !oa || !ob || !pdy || !pdx || !cy || !cx) return 1;
    float *ly = (float *)malloc(sizeof(float) * H), *lx = (float *)malloc(sizeof(float) * W);
    float (*lut)[6] = (float (*)[6])malloc(sizeof(float) * 6 * (LUTN + 1));
    if (!ly || !lx || !lut) { free(ly); free(lx); free(lut); return 1; }
    pred_index(ly, H, cy, nPY);
    pred_index(lx, W, cx, nPX);
    for (int i = 0; i <= LUTN; ++i) {
        float d = (float)i / (float)LUTN;
        for (int k = 0; k < 6; ++k) lut[i][k] = lanczos3(d - (float)(k - 2));
    }
    long stride = shared ? 0 : (long)nPY * nPX;
    long rows = (long)N * H;
#ifdef _OPENMP
    int nt = n_threads > 0 ? n_threads : omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(nt)
#endif
    for (long t = 0; t < rows; ++t) {
        int n = (int)(t / H), i = (int)(t % H);
        const float *dy = pdy + n * stride, *dx = pdx + n * stride;
        const float *a = ia + (size_t)n * H * W, *b = ib + (size_t)n * H * W;
        float *outa = oa + (size_t)n * H * W, *outb = ob + (size_t)n * H * W;
        float fiy = ly[i], fiyf = floorf(fiy);
        int by = (int)fiyf - 1;
        float wy[4];
        keys4(fiy - fiyf, wy);
        for (int j = 0; j < W; ++j) {
            float fx = lx[j], fxf = floorf(fx);
            int bx = (int)fxf - 1;
            float wx[4], vy = 0.0f, vx = 0.0f;
            keys4(fx - fxf, wx);
            for (int m = 0; m < 4; ++m) {
                int r = clampi(by + m, 0, nPY - 1);
                for (int q = 0; q < 4; ++q) {
                    int c = clampi(bx + q, 0, nPX - 1);
                    float wt = wy[m] * wx[q];
                    vy += wt * dy[r * nPX + c];
                    vx += wt * dx[r * nPX + c];
                }
            }
            float hy = 0.5f * vy, hx = 0.5f * vx;
            if (round_shifts) { hy = roundf(hy); hx = roundf(hx); }
            size_t o = (size_t)i * W + j;
            if (mode == 0) {
                outa[o] = bicubic_zero(a, (float)i - hy, (float)j - hx, H, W);
                outb[o] = bicubic_zero(b, (float)i + hy, (float)j + hx, H, W);
            } else {
                outa[o] = lanczos_sample(a, (float)i - hy, (float)j - hx, H, W, (const float (*)[6])lut);
                outb[o] = lanczos_sample(b, (float)i + hy, (float)j + hx, H, W, (const float (*)[6])lut);
            }
        }
    }
    free(ly); free(lx); free(lut);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* k-space Reynolds-stress LM fit (kspace_lm_fit.c), FP64                     */
/* ------------------------------------------------------------------------- */

#define KS_MAXK 9
static const double KS_2PI = 6.283185307179586476925286766559;
static const double KS_2PI2 = 2.0 * 9.869604401089358618834490999876;

typedef struct {
    int H, W, P;
    double *fr[3], *fi[3];
    double *Fr, *Tre, *Tim, *Wg, *Dv, *Pn, *tail;
    double *kx, *ky;
    int *tail_idx, n_tail;
} ks_ws;

static int ks_init(ks_ws *s, int H, int W)
{
    memset(s, 0, sizeof *s);
    s->H = H; s->W = W; s->P = H * W;
    size_t P = (size_t)s->P;
    for (int i = 0; i < 3; ++i) {
        s->fr[i] = (double *)malloc(P * sizeof(double));
        s->fi[i] = (double *)malloc(P * sizeof(double));
    }
    s->Fr = (double *)malloc(P * sizeof(double));
    s->Tre = (double *)malloc(P * sizeof(double));
    s->Tim = (double *)malloc(P * sizeof(double));
    s->Wg = (double *)malloc(P * sizeof(double));
    s->Dv = (double *)malloc(P * sizeof(double));
    s->Pn = (double *)malloc(P * sizeof(double));
    s->tail = (double *)malloc(P * sizeof(double));
    s->tail_idx = (int *)malloc(P * sizeof(int));
    s->kx = (double *)malloc(W * sizeof(double));
    s->ky = (double *)malloc(H * sizeof(double));
    if (!s->Fr || !s->Tre || !s->Tim || !s->Wg || !s->Dv || !s->Pn || !s->tail ||
        !s->tail_idx || !s->kx || !s->ky || !s->fr[2] || !s->fi[2])
        return -1;
    for (int k = 0; k < W; ++k) s->kx[k] = (k < (W + 1) / 2 ? (double)k : (double)(k - W)) / (double)W;
    for (int k = 0; k < H; ++k) s->ky[k] = (k < (H + 1) / 2 ? (double)k : (double)(k - H)) / (double)H;
    s->n_tail = 0;
    for (int r = 0; r < H; ++r)
        for (int c = 0; c < W; ++c)
            if (s->ky[r] * s->ky[r] + s->kx[c] * s->kx[c] >= 0.35 * 0.35)
                s->tail_idx[s->n_tail++] = r * W + c;
    return 0;
}

static void ks_free(ks_ws *s)
{
    for (int i = 0; i < 3; ++i) { free(s->fr[i]); free(s->fi[i]); }
    free(s->Fr); free(s->Tre); free(s->Tim); free(s->Wg); free(s->Dv); free(s->Pn);
    free(s->tail); free(s->tail_idx); free(s->kx); free(s->ky);
}

/* centred transform: load with the ifftshift index map, natural-order output
 * (kspace_lm_fit.c:253-286) */
static void ks_fft_centred(ks_ws *s, const double *pl, int slot)
{
    int H = s->H, W = s->W;
    zd *z = (zd *)malloc(sizeof(zd) * s->P);
    for (int r = 0; r < H; ++r)
        for (int c = 0; c < W; ++c) z[r * W + c] = pl[(size_t)((r + H / 2) % H) * W + (c + W / 2) % W];
    fft2(z, H, W, -1);
    for (int i = 0; i < s->P; ++i) { s->fr[slot][i] = creal(z[i]); s->fi[slot][i] = cimag(z[i]); }
    free(z);
}

int orc_kspace_fft2_centered(const double *plane, int h, int w, double *re, double *im)
{
    if (!orc_size_ok(h) || !orc_size_ok(w)) return -1;
    ks_ws s;
    if (ks_init(&s, h, w)) { ks_free(&s); return -2; }
    ks_fft_centred(&s, plane, 0);
    memcpy(re, s.fr[0], sizeof(double) * s.P);
    memcpy(im, s.fi[0], sizeof(double) * s.P);
    ks_free(&s);
    return 0;
}

static int cmpd(const void *a, const void *b)
{
    double x = *(const double *)a, y = *(const double *)b;
    return (x > y) - (x < y);
}

static double ks_sub3(double lo, double ce, double hi)
{
    if (lo <= 0.0 || ce <= 0.0 || hi <= 0.0) return 0.0;
    double l = log(lo), c = log(ce), r = log(hi);
    double den = 2.0 * (l - 2.0 * c + r);
    if (fabs(den) <= 1e-12) return 0.0;
    return (l - r) / den;
}

static void ks_unpack(const double *x, int ukx, int uky, double *b4x, double *b4y)
{
    int c = 7;
    *b4x = ukx ? x[c++] : 0.0;
    *b4y = uky ? x[c] : 0.0;
}

/* model residual terms of one bin (kspace_lm_fit.c:411-444) */
static double ks_cost(const ks_ws *s, const double *x, int ukx, int uky)
{
    double b4x, b4y, cost = 0.0;
    ks_unpack(x, ukx, uky, &b4x, &b4y);
    for (int r = 0; r < s->H; ++r) {
        double ky = s->ky[r], ky2 = ky * ky;
        for (int c = 0; c < s->W; ++c) {
            size_t i = (size_t)r * s->W + c;
            double w = s->Wg[i];
            if (w == 0.0) continue;
            double kx = s->kx[c], kx2 = kx * kx;
            double arg = -KS_2PI2 * (x[2] * kx2 + 2.0 * x[4] * kx * ky + x[3] * ky2);
            if (ukx) arg -= b4x * kx2 * kx2;
            if (uky) arg -= b4y * ky2 * ky2;
            if (arg > 300.0) arg = 300.0;
            double dec = exp(arg), att = 1.0 - x[6] * s->Dv[i];
            double ph = -KS_2PI * (kx * x[0] + ky * x[1]);
            double gd = x[5] * dec * att;
            double rr = w * (s->Tre[i] - gd * cos(ph)), ri = w * (s->Tim[i] - gd * sin(ph));
            cost += rr * rr + ri * ri;
        }
    }
    return cost;
}

/* normal equations (kspace_lm_fit.c:447-530) */
static void ks_jtj(const ks_ws *s, const double *x, int K, int ukx, int uky, double *A, double *g)
{
    double b4x, b4y, Jr[KS_MAXK], Ji[KS_MAXK];
    ks_unpack(x, ukx, uky, &b4x, &b4y);
    memset(A, 0, sizeof(double) * K * K);
    memset(g, 0, sizeof(double) * K);
    for (int r = 0; r < s->H; ++r) {
        double ky = s->ky[r], ky2 = ky * ky;
        for (int c = 0; c < s->W; ++c) {
            size_t i = (size_t)r * s->W + c;
            double w = s->Wg[i];
            if (w == 0.0) continue;
            double kx = s->kx[c], kx2 = kx * kx, kxky = kx * ky;
            double arg = -KS_2PI2 * (x[2] * kx2 + 2.0 * x[4] * kxky + x[3] * ky2);
            if (ukx) arg -= b4x * kx2 * kx2;
            if (uky) arg -= b4y * ky2 * ky2;
            if (arg > 300.0) arg = 300.0;
            double dec = exp(arg), dv = s->Dv[i], att = 1.0 - x[6] * dv;
            double ph = -KS_2PI * (kx * x[0] + ky * x[1]);
            double cp = cos(ph), sp = sin(ph);
            double gd = x[5] * dec * att;
            double rr = w * (s->Tre[i] - gd * cp), ri = w * (s->Tim[i] - gd * sp);
            double dpx = -KS_2PI * kx, dpy = -KS_2PI * ky;
            Jr[0] = -w * gd * (-sp) * dpx; Ji[0] = -w * gd * cp * dpx;
            Jr[1] = -w * gd * (-sp) * dpy; Ji[1] = -w * gd * cp * dpy;
            double d2 = gd * (-KS_2PI2 * kx2);
            Jr[2] = -w * d2 * cp; Ji[2] = -w * d2 * sp;
            double d3 = gd * (-KS_2PI2 * ky2);
            Jr[3] = -w * d3 * cp; Ji[3] = -w * d3 * sp;
            double d4 = gd * (-KS_2PI2 * 2.0 * kxky);
            Jr[4] = -w * d4 * cp; Ji[4] = -w * d4 * sp;
            Jr[5] = -w * dec * att * cp; Ji[5] = -w * dec * att * sp;
            double dn = x[5] * dec * (-dv);
            Jr[6] = -w * dn * cp; Ji[6] = -w * dn * sp;
            int cc = 7;
            if (ukx) { double db = gd * (-(kx2 * kx2)); Jr[cc] = -w * db * cp; Ji[cc] = -w * db * sp; ++cc; }
            if (uky) { double db = gd * (-(ky2 * ky2)); Jr[cc] = -w * db * cp; Ji[cc] = -w * db * sp; }
            for (int a = 0; a < K; ++a) {
                g[a] += Jr[a] * rr + Ji[a] * ri;
                for (int b = a; b < K; ++b) A[a * K + b] += Jr[a] * Jr[b] + Ji[a] * Ji[b];
            }
        }
    }
    for (int a = 1; a < K; ++a)
        for (int b = 0; b < a; ++b) A[a * K + b] = A[b * K + a];
}

static int ks_chol(int K, const double *M, const double *b, double *d)
{
    double L[KS_MAXK * KS_MAXK], y[KS_MAXK];
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

int orc_kspace_lm_fit_batch(const double *RAA, const double *RBB, const double *RAB,
                            const unsigned char *mask, const double *Pw, int nw, int h,
                            int w, int ukx, int uky, double *gf_all, int *status,
                            double *ig_all, double *dgain, double *dN0, double *db4x,
                            double *db4y, double *dcpp, int *dnv, int *diter,
                            unsigned char *dconv, int n_threads)
{
    if (!orc_size_ok(h) || !orc_size_ok(w)) return -1;
    const int P = h * w, cy = h / 2, cx = w / 2;
    const double ctr_x = w / 2.0 + 1.0, ctr_y = h / 2.0 + 1.0;
    const int K = 7 + (ukx ? 1 : 0) + (uky ? 1 : 0);
    double lo[KS_MAXK], hi[KS_MAXK];
    for (int i = 0; i < KS_MAXK; ++i) { lo[i] = -INFINITY; hi[i] = INFINITY; }
    lo[2] = 0.0; lo[3] = 0.0; lo[5] = 1e-3; hi[5] = 1e3; lo[6] = 0.0;
    hi[6] = Pw ? 10.0 : INFINITY;
    int nproc = 0;
    for (int i = 0; i < nw; ++i) nproc += !mask[i];
    const int all_masked = nproc == 0;
    for (int i = 0; i < nw; ++i) {
        double *gf = gf_all + (size_t)i * 16, *ig = ig_all + (size_t)i * 16;
        for (int c = 0; c < 16; ++c) { gf[c] = 0.0; ig[c] = 0.0; }
        gf[6] = gf[7] = gf[8] = NAN;
        gf[12] = ctr_x; gf[13] = ctr_y; gf[14] = ctr_x; gf[15] = ctr_y;
        if (all_masked || !mask[i]) {
            ig[6] = ig[7] = ig[8] = NAN;
            ig[12] = ctr_x; ig[13] = ctr_y; ig[14] = ctr_x; ig[15] = ctr_y;
        }
        status[i] = -1;
        dgain[i] = dN0[i] = db4x[i] = db4y[i] = dcpp[i] = NAN;
        dnv[i] = 0; diter[i] = 0; dconv[i] = 0;
    }
    int alloc_err = 0;
#ifdef _OPENMP
    int nt = n_threads > 0 ? n_threads : omp_get_max_threads();
#pragma omp parallel num_threads(nt)
#endif
    {
        ks_ws s;
        int ok_ws = ks_init(&s, h, w) == 0;
        if (!ok_ws) alloc_err = 1;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 16)
#endif
        for (int iw = 0; iw < nw; ++iw) {
            if (!ok_ws || mask[iw]) continue;
            double *gf = gf_all + (size_t)iw * 16, *ig = ig_all + (size_t)iw * 16;
            const double *aa = RAA + (size_t)iw * P, *bb = RBB + (size_t)iw * P, *ab = RAB + (size_t)iw * P;
            double ampA = aa[cy * w + cx], ampB = bb[cy * w + cx], ampAB = ab[0];
            for (int i = 1; i < P; ++i) if (ab[i] > ampAB) ampAB = ab[i];
            gf[0] = ig[0] = ampA; gf[1] = ig[1] = ampB; gf[2] = ig[2] = ampAB;
            int amp_ok = ampA >= 1e-12 && ampB >= 1e-12;
            ks_fft_centred(&s, aa, 0);
            ks_fft_centred(&s, bb, 1);
            ks_fft_centred(&s, ab, 2);
            double frmax = 0.0;
            for (int i = 0; i < P; ++i) {
                double fa = hypot(s.fr[0][i], s.fi[0][i]), fb = hypot(s.fr[1][i], s.fi[1][i]);
                double fr = sqrt(fa * fb);
                s.Fr[i] = fr;
                double inv = 1.0 / (fr > 1e-30 ? fr : 1e-30);
                s.Tre[i] = s.fr[2][i] * inv;
                s.Tim[i] = s.fi[2][i] * inv;
                if (fr > frmax) frmax = fr;
            }
            if (frmax < 1e-30) frmax = 1e-30;
            int nv = 0;
            for (int i = 0; i < P; ++i) {
                int v = s.Fr[i] > 1e-12 && i != 0;
                s.Wg[i] = v ? s.Fr[i] / frmax : 0.0;
                nv += v;
            }
            dnv[iw] = nv;
            double seed[KS_MAXK] = {0};
            {   /* peak mu seed from the raw AB plane (kspace_lm_fit.c:301-321) */
                int pi = 0;
                double best = ab[0];
                for (int i = 1; i < P; ++i) if (ab[i] > best) { best = ab[i]; pi = i; }
                int py = pi / w, px = pi % w;
                double sx = 0.0, sy = 0.0;
                if (px > 0 && px < w - 1) sx = ks_sub3(ab[py * w + px - 1], ab[py * w + px], ab[py * w + px + 1]);
                if (py > 0 && py < h - 1) sy = ks_sub3(ab[(py - 1) * w + px], ab[py * w + px], ab[(py + 1) * w + px]);
                seed[0] = ((double)px + sx) - (double)cx;
                seed[1] = ((double)py + sy) - (double)cy;
            }
            seed[2] = 1.0; seed[3] = 0.2; seed[4] = 0.0; seed[6] = 0.0;
            ig[9] = seed[2]; ig[10] = seed[3];
            ig[14] = ctr_x + seed[0];
            ig[15] = ctr_y + seed[1];
            if (!amp_ok) { status[iw] = 2; continue; }
            if (nv < 10) { status[iw] = 1; continue; }
            {   /* ring-1 gain median (kspace_lm_fit.c:330-346) */
                double v8[8];
                int k = 0;
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        if (!dy && !dx) continue;
                        size_t i = (size_t)((dy + h) % h) * w + (dx + w) % w;
                        v8[k++] = hypot(s.Tre[i], s.Tim[i]);
                    }
                qsort(v8, 8, sizeof(double), cmpd);
                double med = 0.5 * (v8[3] + v8[4]);
                seed[5] = med < 1e-2 ? 1e-2 : (med > 10.0 ? 10.0 : med);
            }
            if (!Pw) {
                for (int i = 0; i < P; ++i) s.Dv[i] = 1.0 / (s.Fr[i] > 1e-30 ? s.Fr[i] : 1e-30);
            } else {
                const double *pc = Pw + (size_t)iw * P;
                for (int r = 0; r < h; ++r)
                    for (int c = 0; c < w; ++c) {
                        size_t i = (size_t)r * w + c;
                        double p = pc[(size_t)((r + h / 2) % h) * w + (c + w / 2) % w];
                        s.Pn[i] = p;
                        s.Dv[i] = p / (s.Fr[i] > 1e-30 ? s.Fr[i] : 1e-30);
                    }
                for (int t = 0; t < s.n_tail; ++t) {
                    int i = s.tail_idx[t];
                    s.tail[t] = s.Fr[i] / (s.Pn[i] > 1e-30 ? s.Pn[i] : 1e-30);
                }
                qsort(s.tail, s.n_tail, sizeof(double), cmpd);
                int n = s.n_tail;
                double med = (n & 1) ? s.tail[n / 2] : 0.5 * (s.tail[n / 2 - 1] + s.tail[n / 2]);
                seed[6] = med < 1e-3 ? 1e-3 : (med > 10.0 ? 10.0 : med);
            }
            /* LM (kspace_lm_fit.c:574-664) */
            double x[KS_MAXK];
            for (int i = 0; i < K; ++i) {
                x[i] = seed[i];
                if (x[i] < lo[i]) x[i] = lo[i];
                if (x[i] > hi[i]) x[i] = hi[i];
            }
            double cost = ks_cost(&s, x, ukx, uky);
            int niter = 0, conv = 0;
            if (isfinite(cost)) {
                double lam = 1e-3, A[KS_MAXK * KS_MAXK], g[KS_MAXK], Ad[KS_MAXK * KS_MAXK];
                int have = 0;
                for (int it = 0; it < 250; ++it) {
                    if (!have) { ks_jtj(&s, x, K, ukx, uky, A, g); have = 1; }
                    memcpy(Ad, A, sizeof(double) * K * K);
                    for (int i = 0; i < K; ++i) {
                        double dg = A[i * K + i];
                        if (dg < 1e-30) dg = 1e-30;
                        Ad[i * K + i] += lam * dg;
                    }
                    double d[KS_MAXK], ng[KS_MAXK], xn[KS_MAXK];
                    for (int i = 0; i < K; ++i) ng[i] = -g[i];
                    int solved = ks_chol(K, Ad, ng, d) == 0;
                    int acc = 0;
                    double cn = INFINITY;
                    if (solved) {
                        int fin = 1;
                        for (int i = 0; i < K; ++i) {
                            xn[i] = x[i] + d[i];
                            if (xn[i] < lo[i]) xn[i] = lo[i];
                            if (xn[i] > hi[i]) xn[i] = hi[i];
                            if (!isfinite(xn[i])) fin = 0;
                        }
                        if (fin) {
                            cn = ks_cost(&s, xn, ukx, uky);
                            acc = isfinite(cn) && cn <= cost;
                        }
                    }
                    ++niter;
                    if (acc) {
                        int small = 1;
                        for (int i = 0; i < K; ++i)
                            if (fabs(xn[i] - x[i]) > 1e-8 * (1e-8 + fabs(xn[i]))) { small = 0; break; }
                        double ref = cost > 1e-300 ? cost : 1e-300;
                        int drop = (cost - cn) <= 1e-8 * ref;
                        memcpy(x, xn, sizeof(double) * K);
                        cost = cn;
                        lam /= 3.0;
                        if (lam < 1e-12) lam = 1e-12;
                        have = 0;
                        if (small || drop) { conv = 1; break; }
                    } else {
                        lam *= 10.0;
                        if (lam > 1e12) break;
                    }
                }
            }
            diter[iw] = niter;
            dconv[iw] = (unsigned char)conv;
            double cpp = cost / (double)nv;
            dcpp[iw] = cpp;
            int fit_ok = conv || (niter >= 250 && cpp < 1.0);
            if (!fit_ok) { status[iw] = 1; continue; }
            if (fabs(x[0]) > 0.75 * w || fabs(x[1]) > 0.75 * h) { status[iw] = 3; continue; }
            status[iw] = 0;
            gf[9] = x[2] > 0.0 ? x[2] : 0.0;
            gf[10] = x[3] > 0.0 ? x[3] : 0.0;
            gf[11] = x[4];
            gf[14] = ctr_x + x[0];
            gf[15] = ctr_y + x[1];
            dgain[iw] = x[5];
            dN0[iw] = x[6];
            int cc = 7;
            if (ukx) db4x[iw] = x[cc++];
            if (uky) db4y[iw] = x[cc];
        }
        ks_free(&s);
    }
    return alloc_err ? -2 : 0;
}

float orc_fminvec(const float *v, int n)
{
    float r = v[0];
    for (int i = 1; i < n; ++i) r = (r < v[i]) ? r : v[i];
    return r;
}

float orc_fmaxvec(const float *v, int n)
{
    float r = v[0];
    for (int i = 1; i < n; ++i) r = (r > v[i]) ? r : v[i];
    return r;
}
