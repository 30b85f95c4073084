// xcorr_engine.cuh -- one interrogation window per thread group: FFT
// cross-correlation with the plane kept in shared memory.
//
// Layout of work.  An N x N window is handled by T = N*P threads (P = 1 for
// N <= 32, 2 for 48/64, 4 for 96/128); each thread owns M = N/P complex samples
// of one column (column phase) or one row (row phase), decimated by P.  The
// forward transform packs the two real windows into one complex plane
// z = a + i*b (a = frame A, b = frame B), so one complex 2-D FFT yields both
// spectra; the Hermitian split and the conjugate product
//     C = F_B * conj(F_A)                                 (slot0 = B, slot1 = A)
// are formed in one pass that reads Z(k) and Z(-k) from shared memory
// (PIV_2d_cross_correlate.c:131-133, codelet_fft.c:342-352).  The inverse
// transform then produces the real correlation surface; it is scaled by
// 1/numel, fftshifted (codelet_fft.c:316-327) and written to shared memory as
// floats, where the peak search reads it.  The surface never leaves the SM
// unless the caller asks for the debug dump.
#pragma once

#include "fft_reg.cuh"
#include "peakfit_dev.cuh"

// Resident correlation CTAs per SM that the register allocation is capped for
// (measured on B200 with the paired FP32 FFT: 32 px 5 (96 registers, +1% over
// 4), 64 px 6 (168 registers, +0.6% over 4); before the pairing, 5 at 32 px was
// slower and 6 spilled).
#ifndef PIVB_MIN_CTAS_32
#define PIVB_MIN_CTAS_32 5
#endif
#ifndef PIVB_MIN_CTAS_64
#define PIVB_MIN_CTAS_64 6
#endif

namespace piv {

template <int N>
struct WinGeo {
    // lanes per column (measured on B200 with the deferred fits: one lane at 64 px
    // is 20% faster than two; two at 128 px 1% faster than four; 96 px keeps four)
    static constexpr int P = (N <= 32 || N == 64) ? 1 : ((N == 48 || N == 128) ? 2 : 4);
    static constexpr int M = N / P;
    static constexpr int T = N * P;                                     // active threads per window
    static constexpr int GW = (T <= 8) ? 8 : (T <= 16) ? 16 : (T <= 32) ? 32 : T;  // lanes per group
    static constexpr int WPW = (GW <= 32) ? 32 / GW : 1;                // windows per warp
    // Plane layout of correlate_plane: complex element (row, col) at
    // row * ST + c + SKEW * (c >> SKB), c = (col + ROT * (row / M)) % N.  ST, the
    // rotation of each block of M rows and the skew per 2^SKB columns come from
    // simulating the banks of every store and load phase: a 64-bit access is
    // served per half-warp, so the cost of a phase is the largest number of
    // distinct words one bank holds among 16 lanes, summed over the two halves.
    // Chosen per size (cost summed over the phases, 14 = no conflict): 48 ->
    // ST 50, skew per 32 columns (19.5); 96 -> 100, rotation 4, skew per 32
    // (20.0; the former 102 ran 6% longer).  128 px takes the split lane layout
    // below with ST 129 (no conflict in any phase): shared-memory bank conflicts
    // fell from 35.6 M to 4.0 M of the launch's wavefronts and the pass from
    // 1.157 to 1.051 ms against the adjacent-lane layout's best stride, 134.
    // At 128 px the two lanes of a column sit in opposite half-warps (lane l and
    // l + 16), so each half-warp holds 16 consecutive lines of one sample block:
    // with an odd stride every store and load phase is then free of bank
    // conflicts (a 64-bit access is served per half-warp; rows i apart start
    // 2 * ST * i words apart, distinct even banks for 16 rows).
    static constexpr bool SPLIT = (N == 128);
    static constexpr int XM = SPLIT ? 16 : 1;                           // partner-lane xor mask
    static constexpr int ST = N + ((P == 1 || SPLIT) ? 1 : (P == 2 ? 2 : 4));
    static constexpr int SKEW = (P == 1 || SPLIT) ? 0 : 1;
    static constexpr int SKB = 5;
    static constexpr int ROT = (P == 4) ? 4 : 0;
    static_assert(N - 1 + SKEW * ((N - 1) >> SKB) < ST, "a skewed plane row must fit its stride");
    // float row stride; at 32 px rows 8 apart (the two halves of a warp in the
    // peak search) then fall 16 banks apart
    static constexpr int STF = (N == 32) ? N + 2 : N + 1;
    static constexpr int WARPS_PER_CTA = (GW <= 32) ? 4 : GW / 32;
    static constexpr int CTA_THREADS = WARPS_PER_CTA * 32;
    // resident CTAs per SM the correlation kernel is compiled for (register cap)
    static constexpr int MIN_CTAS = (N == 32) ? PIVB_MIN_CTAS_32 : (N <= 16 ? 8 : (N == 64 ? PIVB_MIN_CTAS_64 : 1));
    static constexpr int GROUPS_PER_CTA = (GW <= 32) ? WARPS_PER_CTA * WPW : 1;
    static constexpr int PLANE_BYTES = N * ST * 8;
    static constexpr int RED_SLOTS = (GW > 32) ? GW / 32 : 1;
    static constexpr int RED_BYTES = 64 * RED_SLOTS * 4 + 64;
    // lane twiddles W_N^{p k} for the four-lane combine (forward sign), float2
    // [P][M + 1]: the padded row puts the four lanes' entries on distinct banks
    static constexpr int TW_LD = M + 1;
    static constexpr int TW_BYTES = (P == 4) ? P * TW_LD * 8 : 0;
    // window weights staged in shared memory at 32 px (measured slower at 64 px
    // with one lane per column and at 128 px)
    static constexpr int WT_BYTES = (N == 32) ? 2 * N * N * 4 : 0;
    static constexpr int SMEM_BYTES = GROUPS_PER_CTA * PLANE_BYTES + RED_BYTES + TW_BYTES + WT_BYTES;
    static_assert(N * STF * 4 <= PLANE_BYTES, "float plane must alias the complex plane");
};

// Thread-group services: synchronisation and reductions over the T threads of
// one window.  Groups of <= 32 lanes live inside one warp; larger groups are a
// whole CTA.
template <int N>
struct Group {
    using G = WinGeo<N>;
    int t;            // thread index within the group (0..GW-1)
    float *red;       // CTA reduction scratch (GW > 32 only)

    __device__ __forceinline__ void sync() const
    {
        if constexpr (G::GW <= 32) __syncwarp();
        else __syncthreads();
    }

    __device__ __forceinline__ float sum(float v) const
    {
        if constexpr (G::GW <= 32) {
#pragma unroll
            for (int o = G::GW / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            return v;
        } else {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            const int w = t >> 5;
            __syncthreads();
            if ((t & 31) == 0) red[w] = v;
            __syncthreads();
            float s = 0.0f;
#pragma unroll
            for (int k = 0; k < G::RED_SLOTS; ++k) s += red[k];
            return s;
        }
    }

    __device__ __forceinline__ bool any(bool b) const
    {
        if constexpr (G::GW <= 32) {
            unsigned m = __ballot_sync(0xffffffffu, b);
            if constexpr (G::GW < 32) {
                const unsigned seg = ((1u << G::GW) - 1u) << ((threadIdx.x & 31) & ~(G::GW - 1));
                m &= seg;
            }
            return m != 0u;
        } else {
            return __syncthreads_or(b) != 0;
        }
    }

    // Reduce the (argmax, top-2) accumulator over the group; result in every lane.
    __device__ __forceinline__ void reduce_peak(PeakAcc &a) const
    {
        constexpr int W = (G::GW <= 32) ? G::GW : 32;
#pragma unroll
        for (int o = W / 2; o > 0; o >>= 1) {
            float ob = __shfl_xor_sync(0xffffffffu, a.best, o);
            int oi = __shfl_xor_sync(0xffffffffu, a.idx, o);
            float o1 = __shfl_xor_sync(0xffffffffu, a.p1, o);
            float o2 = __shfl_xor_sync(0xffffffffu, a.p2, o);
            a.merge(ob, oi, o1, o2);
        }
        if constexpr (G::GW > 32) {
            const int w = t >> 5;
            float *r = red;
            __syncthreads();
            if ((t & 31) == 0) {
                r[4 * w + 0] = a.best;
                r[4 * w + 1] = __int_as_float(a.idx);
                r[4 * w + 2] = a.p1;
                r[4 * w + 3] = a.p2;
            }
            __syncthreads();
            a.init();
#pragma unroll 1
            for (int k = 0; k < G::RED_SLOTS; ++k)
                a.merge(r[4 * k], __float_as_int(r[4 * k + 1]), r[4 * k + 2], r[4 * k + 3]);
        }
    }
};

// Position of a group thread in the column/row phases: the P threads sharing
// one column (row) are adjacent lanes.
template <int N>
__device__ __forceinline__ void lane_slot(int t, int &line, int &p)
{
    using G = WinGeo<N>;
    if constexpr (G::P == 1) {
        line = t;
        p = 0;
    } else if constexpr (G::SPLIT) {
        line = (t >> 5) * 16 + (t & 15);
        p = (t >> 4) & 1;
    } else {
        line = (t >> 5) * (32 / G::P) + (t & 31) / G::P;
        p = t % G::P;
    }
}

struct PlaneView {
    const float *s;
    int ld;
    __device__ __forceinline__ float operator()(int i, int j) const { return s[i * ld + j]; }
};

// Forward packed 2-D transform: z = a + i b (column samples P*n + p of each
// thread) -> Z in shared memory, row-major natural order.
template <int N>
__device__ __forceinline__ void fft2_forward(const Group<N> &g, float2 *S, const float (&a)[WinGeo<N>::M],
                                             const float (&b)[WinGeo<N>::M])
{
    using G = WinGeo<N>;
    constexpr int M = G::M, P = G::P, ST = G::ST;
    const bool active = g.t < G::T;
    int line, p;
    lane_slot<N>(active ? g.t : 0, line, p);
    const int q = out_block<P>(p);
    float2 z[M];
#pragma unroll
    for (int n = 0; n < M; ++n) z[n] = make_float2(a[n], b[n]);
    RegFFT<M, -1>::run(z);                       // column transform (over rows)
    lane_combine<P, M, -1, G::XM>(z, p);
    if (active) {
#pragma unroll
        for (int k = 0; k < M; ++k) S[(M * q + k) * ST + line] = z[k];
    }
    g.sync();
    if (active) {
#pragma unroll
        for (int n = 0; n < M; ++n) z[n] = S[line * ST + P * n + p];
    }
    RegFFT<M, -1>::run(z);                       // row transform
    lane_combine<P, M, -1, G::XM>(z, p);
    g.sync();
    if (active) {
#pragma unroll
        for (int k = 0; k < M; ++k) S[line * ST + M * q + k] = z[k];
    }
    g.sync();
}

// Spectrum products of the packed transform, in the decimated order of the
// inverse row transform.  With Zm = conj(Z(-k)): F_a = (Z + Zm)/2 and
// F_b = (Z - Zm)/(2i).
//   KIND 0 (cross):  4 F_b conj(F_a) = -i (Z - Zm) conj(Z + Zm)
//   KIND 1 (powers): 4 (|F_a|^2 + i |F_b|^2) = |Z + Zm|^2 + i |Z - Zm|^2
template <int N, int KIND>
__device__ __forceinline__ void spectrum_product(const Group<N> &g, const float2 *S, float2 (&z)[WinGeo<N>::M])
{
    using G = WinGeo<N>;
    constexpr int M = G::M, P = G::P, ST = G::ST;
    if (g.t < G::T) {
        int line, p;
        lane_slot<N>(g.t, line, p);
        const int rm = (N - line) % N;
#pragma unroll
        for (int n = 0; n < M; ++n) {
            const int kx = P * n + p;
            const float2 zk = S[line * ST + kx];
            const float2 zn = S[rm * ST + (N - kx) % N];
            const float2 d = make_float2(zk.x - zn.x, zk.y + zn.y);   // Z - Zm
            const float2 s = make_float2(zk.x + zn.x, zk.y - zn.y);   // Z + Zm
            if constexpr (KIND == 0) {
                const float re = d.x * s.x + d.y * s.y;
                const float im = d.y * s.x - d.x * s.y;
                z[n] = make_float2(im, -re);
            } else {
                z[n] = make_float2(s.x * s.x + s.y * s.y, d.x * d.x + d.y * d.y);
            }
        }
    } else {
#pragma unroll
        for (int n = 0; n < M; ++n) z[n] = make_float2(0.0f, 0.0f);
    }
    g.sync();
}

// Inverse 2-D transform of spectrum rows held in registers (decimated order);
// on exit thread (line, p) holds sample rows M*q + k of column `line`.
template <int N>
__device__ __forceinline__ void fft2_inverse(const Group<N> &g, float2 *S, float2 (&z)[WinGeo<N>::M])
{
    using G = WinGeo<N>;
    constexpr int M = G::M, P = G::P, ST = G::ST;
    const bool active = g.t < G::T;
    int line, p;
    lane_slot<N>(active ? g.t : 0, line, p);
    const int q = out_block<P>(p);
    RegFFT<M, +1>::run(z);
    lane_combine<P, M, +1, G::XM>(z, p);
    if (active) {
#pragma unroll
        for (int k = 0; k < M; ++k) S[line * ST + M * q + k] = z[k];
    }
    g.sync();
    if (active) {
#pragma unroll
        for (int n = 0; n < M; ++n) z[n] = S[(P * n + p) * ST + line];
    }
    RegFFT<M, +1>::run(z);
    lane_combine<P, M, +1, G::XM>(z, p);
    g.sync();
}

// Forward packed transform of (a, b) -> C' = 4 F_b conj(F_a), inverse transform,
// scaling and fftshift into the float plane `pl` (aliases S).  On entry each
// active thread holds a[n], b[n] = samples (P*n + p) of its column.
//
// All four 1-D passes (forward columns, forward rows, inverse rows, inverse
// columns) run the same forward transform code inside one loop, so the kernel
// carries a single copy of the unrolled butterflies (the instruction footprint
// of four inlined copies does not fit the instruction cache).  The inverse is
// taken as conj(FFT(conj(C'))): the product stage emits conj(C') directly, and
// only the real part of the result is used, which the final conjugation leaves
// unchanged.  Negation is exact, so this equals the inverse transform bit for bit.
// Fill the lane-twiddle table of the four-lane combine: tw[p][k] = W_N^{p k}
// (forward sign), once per CTA.
template <int N>
__device__ __forceinline__ void fill_lane_twiddles(float2 *tw, int tid, int nthreads)
{
    using G = WinGeo<N>;
    if constexpr (G::TW_BYTES > 0) {
        for (int i = tid; i < G::P * G::M; i += nthreads) {
            const int pp = i / G::M, k = i % G::M;
            double sn, cs;
            sincospi(2.0 * (double)(pp * k) / (double)N, &sn, &cs);
            tw[pp * G::TW_LD + k] = make_float2((float)cs, (float)(-sn));
        }
    }
}

template <int N>
__device__ __forceinline__ void correlate_plane(const Group<N> &g, float2 *S, const float2 (&zab)[WinGeo<N>::M],
                                                float scale, const float2 *tw = nullptr)
{
    using G = WinGeo<N>;
    constexpr int M = G::M, P = G::P, ST = G::ST;
    const bool active = g.t < G::T;
    int line, p;
    lane_slot<N>(active ? g.t : 0, line, p);
    const int q = out_block<P>(p);
    const int rm = (N - line) % N;
    // Complex plane element (row, col) lives at row * ST + c + SKEW * (c >> SKB)
    // with c = (col + ROT * blk) % N, blk = row / M (known at each call site).
    // The rotation of each block of M rows separates the column-phase stores of
    // the lanes of one half-warp that write different blocks; the skew separates
    // the row-phase stores of the lanes of one line, which write columns M apart.
    constexpr int ROT = G::ROT, SKB = G::SKB;
    constexpr bool POW2 = (N & (N - 1)) == 0;
    auto at = [&](int row, int blk, int col) {
        if constexpr (P == 1) return row * ST + col;
        else {
            int c = col;
            if constexpr (ROT != 0) c = POW2 ? ((col + ROT * blk) & (N - 1)) : (col + ROT * blk) % N;
            return row * ST + c + G::SKEW * (c >> SKB);
        }
    };
    const int lb = line / M, rb = rm / M;
    // One lane per column (8 to 64 px but 12): the last pass is a complex-to-real
    // transform.  After the row pass, column x holds E(ky) = conj(D(ky, x)) with D
    // Hermitian in ky (C is), so the real column c(., x) follows from ky = 0..N/2
    // alone: Z(k) = conj(E(k)) + E(N/2 - k) + i (conj(E(k)) - E(N/2 - k)) W_N^{-k}
    // for k < N/2, z = the unnormalised length-N/2 inverse of Z, and
    // c(2m, x) = Re z(m), c(2m + 1, x) = Im z(m): half-length butterflies in place
    // of a full-length transform whose imaginary output was discarded (measured
    // on B200: 32 px final pass -5.5%, 8 / 16 / 24 px -1 to -2%; 12 px spills at
    // its register cap and ran 3.7% slower, so it keeps the full transform).
    constexpr bool C2R = (P == 1) && (N % 2 == 0) && (N != 12);
    constexpr int MH = C2R ? M / 2 : 1;
    float2 zh[MH];
    float2 z[M];
#pragma unroll
    for (int n = 0; n < M; ++n) z[n] = zab[n];
#pragma unroll 1
    for (int pass = 0;; ++pass) {
        RegFFT<M, -1>::run(z);
        if constexpr (G::TW_BYTES > 0) lane_combine_fwd_tab<P, M>(z, p, tw);
        else lane_combine<P, M, -1, G::XM>(z, p);
        if (pass == 3) break;
        g.sync();
        if (active) {
            if (pass == 0) {
#pragma unroll
                for (int k = 0; k < M; ++k) S[at(M * q + k, q, line)] = z[k];
            } else {
#pragma unroll
                for (int k = 0; k < M; ++k) S[at(line, lb, M * q + k)] = z[k];
            }
        }
        g.sync();
        if (pass == 1) {
            // conj(C') = conj(-i (Z - Zm) conj(Z + Zm)), Zm = conj(Z(-k))
            if (active) {
#pragma unroll
                for (int n = 0; n < M; ++n) {
                    const int kx = P * n + p;
                    const float2 zk = S[at(line, lb, kx)];
                    const float2 zn = S[at(rm, rb, (N - kx) % N)];
                    const float2 d = make_float2(zk.x - zn.x, zk.y + zn.y);   // Z - Zm
                    const float2 sm = make_float2(zk.x + zn.x, zk.y - zn.y);  // Z + Zm
                    const float re = d.x * sm.x + d.y * sm.y;
                    const float im = d.y * sm.x - d.x * sm.y;
                    z[n] = make_float2(im, re);
                }
            } else {
#pragma unroll
                for (int n = 0; n < M; ++n) z[n] = make_float2(0.0f, 0.0f);
            }
        } else if (active) {
            if (pass == 0) {
#pragma unroll
                for (int n = 0; n < M; ++n) z[n] = S[at(line, lb, P * n + p)];
            } else if constexpr (C2R) {
                sfor<MH>([&](auto kc) {
                    constexpr int k = decltype(kc)::value;
                    const float2 e = S[k * ST + line], f = S[(MH - k) * ST + line];
                    const float2 s = make_float2(e.x + f.x, f.y - e.y);        // conj(E(k)) + E(N/2 - k)
                    const float2 d = c_twiddle<N, k, +1>(make_float2(e.x - f.x, -e.y - f.y));
                    zh[k] = make_float2(s.x - d.y, s.y + d.x);                // s + i d
                });
                RegFFT<MH, +1>::run(zh);
                break;
            } else {
#pragma unroll
                for (int n = 0; n < M; ++n) z[n] = S[at(P * n + p, (P * n) / M, line)];
            }
        } else if constexpr (C2R) {
            if (pass == 2) break;
        }
    }
    g.sync();
    float *pl = reinterpret_cast<float *>(S);
    if (active) {
        const int col = (line + N / 2) % N;
        if constexpr (C2R) {
#pragma unroll
            for (int m = 0; m < MH; ++m) {
                pl[((2 * m + N / 2) % N) * G::STF + col] = (zh[m].x * 0.25f) * scale;
                pl[((2 * m + 1 + N / 2) % N) * G::STF + col] = (zh[m].y * 0.25f) * scale;
            }
        } else {
#pragma unroll
            for (int k = 0; k < M; ++k) {
                const int row = (M * q + k + N / 2) % N;
                pl[row * G::STF + col] = (z[k].x * 0.25f) * scale;
            }
        }
    }
    g.sync();
}

// Parallel Westerweel search + detectability over the plane in shared memory.
// Returns, in every lane, the accumulator and whether a NaN was seen.
// The candidates (rows and columns [N/4, 3N/4); a value above zero that no
// neighbour of its 3x3 block exceeds) are taken in vertical strips of up to 8
// rows of one column, rolling the maxima of three consecutive 3-wide rows: 3
// loads per row of the strip instead of 9 per candidate.  PeakAcc's result
// does not depend on the order in which candidates arrive.  A plane holding
// NaN sets the flag (over the same neighbourhoods) and is searched again by
// the caller's exact sequential scan, so only NaN-free planes rely on the
// maximum form of the test.
template <int N>
__device__ __forceinline__ void search_plane(const Group<N> &g, const float *pl, PeakAcc &acc, bool &has_nan)
{
    using G = WinGeo<N>;
    constexpr int H2 = N / 2, Q = N / 4, S = (H2 < 8) ? H2 : 8;
    constexpr int NS = (H2 + S - 1) / S, U = H2 * NS;
    acc.init();
    bool nan = false;
    if (g.t < G::T) {
#pragma unroll 1
        for (int u = g.t; u < U; u += G::T) {
            const int j = Q + u % H2, r0 = Q + (u / H2) * S;
            const int rows = min(S, Q + H2 - r0);
            const float *c0 = pl + (r0 - 1) * G::STF + j;
            float m0 = 0.0f, m1 = 0.0f, c1 = 0.0f;      // row maxima k-2, k-1; centre value k-1
            // at 32 px a partly rolled loop keeps the kernel's code within the
            // instruction cache (measured: 5.21 -> 4.92 ms per 1 M windows)
            constexpr int UNR = (N == 32) ? 2 : S + 2;
#pragma unroll UNR
            for (int k = 0; k < S + 2; ++k) {
                if (k < rows + 2) {
                    const float l = c0[k * G::STF - 1], c = c0[k * G::STF], r = c0[k * G::STF + 1];
                    nan |= (l != l) | (c != c) | (r != r);
                    const float m2 = fmaxf(l, fmaxf(c, r));
                    if (k >= 2) {
                        const float v = c1;                 // candidate row r0 + k - 2
                        const bool mx = v >= fmaxf(m0, fmaxf(m1, m2));
                        acc.add((mx && v > 0.0f) ? v : -1.0f, (r0 + k - 2) * N + j);
                    }
                    m0 = m1;
                    m1 = m2;
                    c1 = c;
                }
            }
        }
    }
    has_nan = g.any(nan);
    g.reduce_peak(acc);
}

}  // namespace piv
