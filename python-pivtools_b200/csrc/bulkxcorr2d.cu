// bulkxcorr2d.cu -- libbulkxcorr2d for sm_100a.
//
// Exports the reference library's C-ABI (pivtools_cli/lib/PIV_2d_cross_correlate.h,
// peak_locate_lm.h, peak_locate_lm_batch.h, xcorr.h, codelet_fft.h) with the same
// argument meaning, array layouts and error codes, so that the reference's ctypes
// callers load this file in place of the CPU library.  Host-pointer entry points
// stage their arrays through a device workspace owned by this library; the
// pivb_*_dev entry points take device pointers and a CUDA stream for callers that
// keep their data resident.  Every computation runs on the GPU; with no usable
// device the entry points return an error code (there is no CPU path).
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <atomic>
#include <mutex>

#include "device_state.h"
#include "xcorr_kernels.cuh"
#include "xcorr_rect.cuh"

using namespace piv;

// ---------------------------------------------------------------------------
// Library state (process-wide, like the reference's selector globals).
// ---------------------------------------------------------------------------
namespace {

std::mutex g_mu;                        // serialises host-pointer calls
volatile int g_timing = 0;
double g_t_fft = 0.0, g_t_fit = 0.0;
volatile int g_peakfit_impl = 0;

// Staging workspace of the host-pointer entry points on one device: a device
// block, a stream and timing events, all created on that device.
struct Workspace {
    void *dev = nullptr;
    size_t cap = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};

    int ensure(size_t bytes)
    {
        if (stream == nullptr) {
            if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) return PIV_ERROR_CUDA;
            for (auto &e : ev)
                if (cudaEventCreate(&e) != cudaSuccess) return PIV_ERROR_CUDA;
        }
        if (bytes > cap) {
            if (dev) cudaFree(dev);
            dev = nullptr;
            cap = 0;
            size_t want = bytes + bytes / 4;
            if (cudaMalloc(&dev, want) != cudaSuccess) {
                cudaGetLastError();
                return PIV_ERROR_NOMEM;
            }
            cap = want;
        }
        return PIV_ERROR_NONE;
    }
};
Workspace g_ws_dev[kMaxDevices];
// The current device's workspace (nullptr without a usable device).  Host-pointer
// calls use it under g_mu; the timing events are also recorded by the device
// entry points (after ensure(0) has created them).
Workspace *cur_ws()
{
    const int d = current_device();
    return d < 0 ? nullptr : &g_ws_dev[d];
}

// Bump allocator over one device block.
struct Carve {
    char *base;
    size_t off = 0;
    explicit Carve(void *b) : base(static_cast<char *>(b)) {}
    template <class T>
    T *take(size_t n)
    {
        off = (off + 255) & ~size_t(255);
        T *p = reinterpret_cast<T *>(base + off);
        off += n * sizeof(T);
        return p;
    }
};
inline size_t pad256(size_t b) { return (b + 255) & ~size_t(255); }

bool size_ok(int n)
{
    switch (n) {
    case 8: case 12: case 16: case 24: case 32: case 48: case 64: case 96: case 128:
        return true;
    default:
        return false;
    }
}

// Resident CTAs per SM of xcorr_kernel<N, MULTI> on `dev`, set up once per device
// (raises the kernel's dynamic shared-memory limit there first); -1 on failure.
template <int N, bool MULTI>
int xcorr_blocks_per_sm(int dev)
{
    using G = WinGeo<N>;
    static PerDeviceOnce per_sm;
    return per_sm.get(dev, [] {
        auto kern = xcorr_kernel<N, MULTI>;
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM_BYTES) != cudaSuccess)
            return -1;
        int nb = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, G::CTA_THREADS, G::SMEM_BYTES) != cudaSuccess)
            return -1;
        return nb > 0 ? nb : 1;
    });
}

// Launch settings the autotuner may change (process-wide): a cap on resident
// correlation CTAs per SM for each window size (0 = the occupancy maximum), and
// the block size of the per-window record (fit) kernel.
int size_index(int n)
{
    switch (n) {
    case 8: return 0; case 12: return 1; case 16: return 2; case 24: return 3; case 32: return 4;
    case 48: return 5; case 64: return 6; case 96: return 7; case 128: return 8;
    default: return -1;
    }
}
std::atomic<int> g_ctas_cap[9];
std::atomic<int> g_record_block{128};

// Resident 128-thread CTAs per SM of lm_fit_kernel<T, MODE> on `dev`, once per device.
template <int T, int MODE>
int lm_fit_blocks_per_sm(int dev)
{
    static PerDeviceOnce per_sm;
    return per_sm.get(dev, [] {
        int nb = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, lm_fit_kernel<T, MODE>, 128, 0) != cudaSuccess)
            return -1;
        return nb > 0 ? nb : 1;
    });
}

bool lm_fit_setup(int dev)
{
    return lm_fit_blocks_per_sm<4, 0>(dev) >= 0 && lm_fit_blocks_per_sm<5, 0>(dev) >= 0 &&
           lm_fit_blocks_per_sm<6, 0>(dev) >= 0 && lm_fit_blocks_per_sm<4, 1>(dev) >= 0 &&
           lm_fit_blocks_per_sm<5, 1>(dev) >= 0 && lm_fit_blocks_per_sm<6, 1>(dev) >= 0;
}

template <int T, int MODE>
int launch_lm_fit(const XcorrParams &p, int win, cudaStream_t s)
{
    const int dev = current_device();
    if (dev < 0) return PIV_ERROR_CUDA;
    const int per_sm = lm_fit_blocks_per_sm<T, MODE>(dev);
    if (per_sm < 0) return PIV_ERROR_CUDA;
    // every resident warp owns a contiguous run of at least 64 records
    const long long resident = (long long)device_sms(dev) * per_sm * 4;
    long long warps = (p.total + 63) / 64;
    if (warps > resident) warps = resident;
    const long long chunk = (p.total + warps - 1) / warps;
    const unsigned blocks = (unsigned)((warps + 3) / 4);
    lm_fit_kernel<T, MODE><<<blocks, 128, 0, s>>>(p, win, chunk);
    return cudaGetLastError() == cudaSuccess ? PIV_ERROR_NONE : PIV_ERROR_CUDA;
}

// The deferred fits of a single-peak call: LM types on the persistent refill
// kernel, 3-point fits one thread per record.
int launch_records(const XcorrParams &p, int win, int peakfit_impl, int tb, cudaStream_t s)
{
    const int impl = peakfit_impl ? 1 : 0;
    switch (p.finder * 2 + impl) {
    case 8: return launch_lm_fit<4, 0>(p, win, s);
    case 9: return launch_lm_fit<4, 1>(p, win, s);
    case 10: return launch_lm_fit<5, 0>(p, win, s);
    case 11: return launch_lm_fit<5, 1>(p, win, s);
    case 12: return launch_lm_fit<6, 0>(p, win, s);
    case 13: return launch_lm_fit<6, 1>(p, win, s);
    default: break;
    }
    const unsigned blocks = (unsigned)((p.total + tb - 1) / tb);
    if (impl) lm_records_kernel<1><<<blocks, tb, 0, s>>>(p, win);
    else lm_records_kernel<0><<<blocks, tb, 0, s>>>(p, win);
    return cudaGetLastError() == cudaSuccess ? PIV_ERROR_NONE : PIV_ERROR_CUDA;
}

template <int N, bool MULTI>
int launch_xcorr_n(const XcorrParams &p, cudaStream_t s)
{
    using G = WinGeo<N>;
    auto kern = xcorr_kernel<N, MULTI>;
    const int dev = current_device();
    if (dev < 0) return PIV_ERROR_CUDA;
    const int per_sm = xcorr_blocks_per_sm<N, MULTI>(dev);
    if (per_sm < 0) {
        cudaGetLastError();
        return PIV_ERROR_CUDA;
    }
    const int tuned = g_ctas_cap[size_index(N)].load(std::memory_order_relaxed);
    long long want = (p.total + G::GROUPS_PER_CTA - 1) / G::GROUPS_PER_CTA;
    long long cap = (long long)(tuned > 0 && tuned < per_sm ? tuned : per_sm) * device_sms(dev);
    int grid = (int)(want < cap ? want : cap);
    if (grid < 1) grid = 1;
    kern<<<grid, G::CTA_THREADS, G::SMEM_BYTES, s>>>(p);
    return cudaGetLastError() == cudaSuccess ? PIV_ERROR_NONE : PIV_ERROR_CUDA;
}

template <bool MULTI>
int launch_xcorr(int N, const XcorrParams &p, cudaStream_t s)
{
    switch (N) {
    case 8: return launch_xcorr_n<8, MULTI>(p, s);
    case 12: return launch_xcorr_n<12, MULTI>(p, s);
    case 16: return launch_xcorr_n<16, MULTI>(p, s);
    case 24: return launch_xcorr_n<24, MULTI>(p, s);
    case 32: return launch_xcorr_n<32, MULTI>(p, s);
    case 48: return launch_xcorr_n<48, MULTI>(p, s);
    case 64: return launch_xcorr_n<64, MULTI>(p, s);
    case 96: return launch_xcorr_n<96, MULTI>(p, s);
    case 128: return launch_xcorr_n<128, MULTI>(p, s);
    default: return PIV_ERROR_NOPLAN_BWD;
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// Device-pointer API
// ---------------------------------------------------------------------------

// Bytes of scratch the device correlation entry point needs for a call.
namespace {

// Rectangular windows: the staged path of xcorr_rect.cuh over chunks of windows
// whose planes fit a fixed scratch budget.
constexpr size_t kRectChunkBudget = 256u << 20;

size_t rect_window_bytes(int h, int w, int n_peaks)
{
    const size_t hw = (size_t)h * w;
    return hw * 8 + hw * 4 + (n_peaks > 1 ? hw * 4 : 0) + (size_t)6 * n_peaks * 4 + 12;
}

long long rect_chunk(long long total, int h, int w, int n_peaks)
{
    long long c = (long long)(kRectChunkBudget / rect_window_bytes(h, w, n_peaks));
    if (c < 1) c = 1;
    return c < total ? c : total;
}

size_t rect_scratch_bytes(long long total, int h, int w, int n_peaks)
{
    if (total <= 0) return 0;
    const size_t c = (size_t)rect_chunk(total, h, w, n_peaks), hw = (size_t)h * w;
    return pad256(c * hw * 8) + pad256(c * hw * 4) + (n_peaks > 1 ? pad256(c * hw * 4) : 0) +
           2 * pad256(c * 3 * n_peaks * 4) + 3 * pad256(c * 4);
}

template <int L, int AXIS>
void rect_fft_n(const RectParams &p, cudaStream_t s)
{
    const long long threads = (long long)p.count * (AXIS == 0 ? p.w : p.h) * RectLine<L>::P;
    rect_line_fft<L, AXIS><<<(unsigned)((threads + 127) / 128), 128, 0, s>>>(p);
}

template <int AXIS>
void rect_fft(int L, const RectParams &p, cudaStream_t s)
{
    switch (L) {
    case 8: rect_fft_n<8, AXIS>(p, s); break;
    case 12: rect_fft_n<12, AXIS>(p, s); break;
    case 16: rect_fft_n<16, AXIS>(p, s); break;
    case 24: rect_fft_n<24, AXIS>(p, s); break;
    case 32: rect_fft_n<32, AXIS>(p, s); break;
    case 48: rect_fft_n<48, AXIS>(p, s); break;
    case 64: rect_fft_n<64, AXIS>(p, s); break;
    case 96: rect_fft_n<96, AXIS>(p, s); break;
    default: rect_fft_n<128, AXIS>(p, s); break;
    }
}

// The whole rectangular correlation + fit of `total` windows on stream s.
int xcorr_rect(RectParams p, long long total, int n_peaks, int peak_finder, int peakfit_impl, const float *cw,
               float *pk_x, float *pk_y, float *pk_h, float *sx, float *sy, float *sxy, float *pk_ratio,
               void *scratch, cudaStream_t s)
{
    const long long chunk = rect_chunk(total, p.h, p.w, n_peaks);
    const size_t c = (size_t)chunk, hw = (size_t)p.h * p.w;
    Carve cv(scratch);
    p.Z = cv.take<float2>(c * hw);
    p.pl = cv.take<float>(c * hw);
    float *work = n_peaks > 1 ? cv.take<float>(c * hw) : nullptr;
    float *loc = cv.take<float>(c * 3 * n_peaks);
    float *sd = cv.take<float>(c * 3 * n_peaks);
    p.enorm = cv.take<float>(c);
    p.valid = cv.take<int>(c);
    float *ratio = cv.take<float>(c);
    const bool batch = peakfit_impl && n_peaks == 1 && peak_finder >= 4 && peak_finder <= 6;
    RectOut o{pk_x, pk_y, pk_h, sx, sy, sxy, pk_ratio, loc, sd, ratio, n_peaks};
    for (long long w0 = 0; w0 < total; w0 += chunk) {
        p.w0 = w0;
        p.count = (int)(total - w0 < chunk ? total - w0 : chunk);
        const unsigned elems = (unsigned)(((long long)p.count * hw + 255) / 256);
        rect_gather_kernel<<<p.count, kRectThreads, 0, s>>>(p);
        rect_fft<0>(p.h, p, s);
        rect_fft<1>(p.w, p, s);
        rect_product_kernel<<<elems, 256, 0, s>>>(p);
        rect_fft<1>(p.w, p, s);
        rect_fft<0>(p.h, p, s);
        rect_shift_kernel<<<elems, 256, 0, s>>>(p);
        if (!p.ensemble) {
            if (batch)
                fit_planes_kernel<1><<<p.count, 128, 0, s>>>(p.pl, p.h, p.w, n_peaks, peak_finder, cw, loc, sd, 0, 0,
                                                             ratio, work);
            else
                fit_planes_kernel<0><<<p.count, 128, 0, s>>>(p.pl, p.h, p.w, n_peaks, peak_finder, cw, loc, sd, 0, 0,
                                                             ratio, work);
            rect_finish_kernel<<<(p.count + 127) / 128, 128, 0, s>>>(p, o);
        }
        if (cudaGetLastError() != cudaSuccess) return PIV_ERROR_CUDA;
    }
    return PIV_ERROR_NONE;
}

}  // namespace

// ---------------------------------------------------------------------------
// Packed correlation launches (no counterpart in the reference)
// ---------------------------------------------------------------------------
// One job of a packed launch: the arguments of one single-peak pivb_xcorr_dev
// call (device pointers).  Declared the same in include/libbulkxcorr2d.h.
struct PivbXcorrJob {
    const float *A, *B;
    long long img_stride;
    const float *mask;
    int H, W, n_images;
    const float *ctr_x, *ctr_y;
    int n_win_y, n_win_x;
    const float *wA, *wB, *cw;
    float *pk_x, *pk_y, *pk_h, *sx, *sy, *sxy, *pk_ratio;
};

namespace {

int groups_per_cta(int n)
{
    switch (n) {
    case 8: return WinGeo<8>::GROUPS_PER_CTA;
    case 12: return WinGeo<12>::GROUPS_PER_CTA;
    case 16: return WinGeo<16>::GROUPS_PER_CTA;
    case 24: return WinGeo<24>::GROUPS_PER_CTA;
    case 32: return WinGeo<32>::GROUPS_PER_CTA;
    case 48: return WinGeo<48>::GROUPS_PER_CTA;
    case 64: return WinGeo<64>::GROUPS_PER_CTA;
    case 96: return WinGeo<96>::GROUPS_PER_CTA;
    case 128: return WinGeo<128>::GROUPS_PER_CTA;
    default: return -1;
    }
}

// Padded window offsets of the jobs (each range a multiple of the CTA's window
// count); returns the padded total, or -1 for bad arguments.
long long job_offsets(const PivbXcorrJob *jobs, int n_jobs, int win, long long *off)
{
    const int g = groups_per_cta(win);
    if (g < 1 || n_jobs < 1 || n_jobs > kMaxJobs) return -1;
    off[0] = 0;
    for (int j = 0; j < n_jobs; ++j) {
        if (jobs[j].n_images < 0 || jobs[j].n_win_y < 0 || jobs[j].n_win_x < 0) return -1;
        const long long t = (long long)jobs[j].n_images * jobs[j].n_win_y * jobs[j].n_win_x;
        off[j + 1] = off[j] + (t + g - 1) / g * g;
    }
    return off[n_jobs];
}

template <int N>
int launch_xcorr_jobs_n(const XcorrJobs &pj, cudaStream_t s)
{
    using G = WinGeo<N>;
    static PerDeviceOnce per_sm_dev;
    const int dev = current_device();
    if (dev < 0) return PIV_ERROR_CUDA;
    const int per_sm = per_sm_dev.get(dev, [] {
        auto kern = xcorr_kernel<N, false, true>;
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM_BYTES) != cudaSuccess)
            return -1;
        int nb = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, G::CTA_THREADS, G::SMEM_BYTES) != cudaSuccess)
            return -1;
        return nb > 0 ? nb : 1;
    });
    if (per_sm < 0) {
        cudaGetLastError();
        return PIV_ERROR_CUDA;
    }
    const long long want = pj.total / G::GROUPS_PER_CTA;
    const long long cap = (long long)per_sm * device_sms(dev);
    const int grid = (int)(want < cap ? (want < 1 ? 1 : want) : cap);
    xcorr_kernel<N, false, true><<<grid, G::CTA_THREADS, G::SMEM_BYTES, s>>>(pj);
    return cudaGetLastError() == cudaSuccess ? PIV_ERROR_NONE : PIV_ERROR_CUDA;
}

int launch_xcorr_jobs(int N, const XcorrJobs &pj, cudaStream_t s)
{
    switch (N) {
    case 8: return launch_xcorr_jobs_n<8>(pj, s);
    case 12: return launch_xcorr_jobs_n<12>(pj, s);
    case 16: return launch_xcorr_jobs_n<16>(pj, s);
    case 24: return launch_xcorr_jobs_n<24>(pj, s);
    case 32: return launch_xcorr_jobs_n<32>(pj, s);
    case 48: return launch_xcorr_jobs_n<48>(pj, s);
    case 64: return launch_xcorr_jobs_n<64>(pj, s);
    case 96: return launch_xcorr_jobs_n<96>(pj, s);
    case 128: return launch_xcorr_jobs_n<128>(pj, s);
    default: return PIV_ERROR_NOPLAN_BWD;
    }
}

}  // namespace

// Record bytes a packed launch of these jobs needs (128 per padded window).
PIV_EXPORT size_t pivb_xcorr_jobs_record_bytes(const PivbXcorrJob *jobs, int n_jobs, int win)
{
    long long off[kMaxJobs + 1];
    const long long total = job_offsets(jobs, n_jobs, win, off);
    return total < 0 ? 0 : pad256((size_t)total * sizeof(LmRecord));
}

PIV_EXPORT int pivb_xcorr_jobs_max(void) { return kMaxJobs; }

// Single-peak correlation + fit of up to pivb_xcorr_jobs_max() jobs of one
// square window size in one launch (and one launch of the fit kernel for all of
// them): jobs may differ in frames, frame size, window grid, mask, weights and
// outputs.  Every job's results equal those of its own pivb_xcorr_dev call.
// d_records: pivb_xcorr_jobs_record_bytes bytes.  The job table travels as the
// kernels' parameter, so the call issues no copy and needs no synchronisation.
PIV_EXPORT int pivb_xcorr_jobs_dev(const PivbXcorrJob *jobs, int n_jobs, int win, int peak_finder,
                                   int peakfit_impl, void *d_records, size_t record_bytes, void *stream)
{
    if (!size_ok(win)) return PIV_ERROR_NOPLAN_BWD;
    if (peak_finder < 3 || peak_finder > 6) return PIV_ERROR_NOPLAN;
    static XcorrJobs pj;                      // 10 KB: kept off the host stack; filled under the lock
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    const long long total = job_offsets(jobs, n_jobs, win, pj.off);
    if (total < 0) return PIV_ERROR_OUT_OF_BOUNDS;
    if (total == 0) return PIV_ERROR_NONE;
    if (d_records == nullptr || record_bytes < (size_t)total * sizeof(LmRecord)) return PIV_ERROR_NOMEM;
    pj.total = total;
    pj.n_jobs = n_jobs;
    LmRecord *rec = static_cast<LmRecord *>(d_records);
    for (int j = 0; j < n_jobs; ++j) {
        const PivbXcorrJob &J = jobs[j];
        XcorrParams &p = pj.job[j];
        p = XcorrParams{};
        p.A = J.A; p.B = J.B; p.img_stride = J.img_stride; p.mask = J.mask;
        p.H = J.H; p.W = J.W; p.n_img = J.n_images;
        p.ctr_x = J.ctr_x; p.ctr_y = J.ctr_y; p.nwy = J.n_win_y; p.nwx = J.n_win_x;
        p.wA = J.wA; p.wB = J.wB; p.cw = J.cw;
        p.ensemble = 0; p.n_peaks = 1; p.finder = peak_finder;
        p.pk_x = J.pk_x; p.pk_y = J.pk_y; p.pk_h = J.pk_h; p.sx = J.sx; p.sy = J.sy; p.sxy = J.sxy;
        p.pk_ratio = J.pk_ratio; p.planes = nullptr;
        p.lm = rec + pj.off[j];
        p.total = (long long)J.n_images * J.n_win_y * J.n_win_x;
        p.neg_zero = -0.0f;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int e = launch_xcorr_jobs(win, pj, s);
    if (e) return e;
    const int tb = g_record_block.load(std::memory_order_relaxed);
    const unsigned blocks = (unsigned)((total + tb - 1) / tb);
    if (peakfit_impl) lm_records_kernel<1, true><<<blocks, tb, 0, s>>>(pj, win);
    else lm_records_kernel<0, true><<<blocks, tb, 0, s>>>(pj, win);
    return cudaGetLastError() == cudaSuccess ? PIV_ERROR_NONE : PIV_ERROR_CUDA;
}

// Autotuner hooks (no counterpart in the reference): cap the resident
// correlation CTAs per SM of window size `win` (0 restores the occupancy
// maximum); read the cap and the occupancy maximum on the current device; set
// the record kernel's block size (32, 64 or 128).  Process-wide settings;
// 0 on success, 1 for arguments out of range.
PIV_EXPORT int pivb_xcorr_set_ctas_per_sm(int win, int ctas)
{
    const int k = size_index(win);
    if (k < 0 || ctas < 0 || ctas > 64) return 1;
    g_ctas_cap[k].store(ctas);
    return 0;
}

PIV_EXPORT int pivb_xcorr_get_ctas_per_sm(int win)
{
    const int k = size_index(win);
    return k < 0 ? -1 : g_ctas_cap[k].load();
}

PIV_EXPORT int pivb_xcorr_max_ctas_per_sm(int win)
{
    const int dev = current_device();
    if (dev < 0) return -1;
    switch (win) {
    case 8: return xcorr_blocks_per_sm<8, false>(dev);
    case 12: return xcorr_blocks_per_sm<12, false>(dev);
    case 16: return xcorr_blocks_per_sm<16, false>(dev);
    case 24: return xcorr_blocks_per_sm<24, false>(dev);
    case 32: return xcorr_blocks_per_sm<32, false>(dev);
    case 48: return xcorr_blocks_per_sm<48, false>(dev);
    case 64: return xcorr_blocks_per_sm<64, false>(dev);
    case 96: return xcorr_blocks_per_sm<96, false>(dev);
    case 128: return xcorr_blocks_per_sm<128, false>(dev);
    default: return -1;
    }
}

PIV_EXPORT int pivb_xcorr_set_record_block(int threads)
{
    if (threads != 32 && threads != 64 && threads != 128) return 1;
    g_record_block.store(threads);
    return 0;
}

PIV_EXPORT size_t pivb_xcorr_scratch_bytes(long long n_windows_total, int n_peaks, int peak_finder)
{
    if (n_peaks == 1 && peak_finder >= 4 && peak_finder <= 6)
        return pad256((size_t)n_windows_total * sizeof(LmRecord));
    return 0;
}

// Bytes of the per-window records with which pivb_xcorr_dev defers every
// single-peak fit (3-point included) to a thread-per-window kernel.
// Scratch bytes pivb_xcorr_dev needs for windows of h x w: for square windows
// pivb_xcorr_scratch_bytes (LM records only); for rectangular windows the planes
// of the staged path, for chunks of at most 256 MiB of windows.
PIV_EXPORT size_t pivb_xcorr_scratch_bytes_hw(long long n_windows_total, int win_h, int win_w, int n_peaks,
                                              int peak_finder)
{
    if (win_h == win_w) return pivb_xcorr_scratch_bytes(n_windows_total, n_peaks, peak_finder);
    return rect_scratch_bytes(n_windows_total, win_h, win_w, n_peaks < 1 ? 1 : n_peaks);
}

PIV_EXPORT size_t pivb_xcorr_record_bytes(long long n_windows_total)
{
    return pad256((size_t)n_windows_total * sizeof(LmRecord));
}

// Loss-of-correlation weight numel / (wB (*) wB) on the device.
PIV_EXPORT int pivb_correl_weight_dev(const float *d_wB, int h, int w, float *d_out, void *stream)
{
    if (h <= 0 || w <= 0) return PIV_ERROR_NOPLAN_BWD;
    const int n = h * w;
    lin_xcorr_kernel<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(d_wB, d_wB, h, w, d_out, 1);
    return cudaGetLastError() == cudaSuccess ? PIV_ERROR_NONE : PIV_ERROR_CUDA;
}

// Batched instantaneous correlation + peak fit on device-resident data.  Same
// meaning as bulkxcorr2d's arguments; additionally img_stride (elements between
// frames, >= H*W), the precomputed correlation weight d_cw, the peak-fit
// implementation (0 scalar, 1 batch), and scratch for deferred LM fits
// (pivb_xcorr_scratch_bytes).  Outputs of skipped windows are left untouched.
PIV_EXPORT int pivb_xcorr_dev(const float *d_A, const float *d_B, long long img_stride,
                              const float *d_mask, int H, int W, int n_images,
                              const float *d_ctr_x, const float *d_ctr_y, int n_win_y,
                              int n_win_x, const float *d_wA, const float *d_wB, const float *d_cw,
                              int win_h, int win_w, int ensemble, int n_peaks, int peak_finder,
                              int peakfit_impl, float *d_pk_x, float *d_pk_y, float *d_pk_h,
                              float *d_sx, float *d_sy, float *d_sxy, float *d_pk_ratio,
                              float *d_planes, void *d_scratch, size_t scratch_bytes, void *stream)
{
    if (!size_ok(win_h) || !size_ok(win_w)) return PIV_ERROR_NOPLAN_BWD;
    if (n_peaks < 1 || n_images < 0) return PIV_ERROR_OUT_OF_BOUNDS;
    const long long total = (long long)n_images * n_win_y * n_win_x;
    if (total == 0) return PIV_ERROR_NONE;
    if (win_h != win_w) {
        // rectangular windows: the staged path (planes in the caller's scratch)
        if (d_scratch == nullptr || scratch_bytes < rect_scratch_bytes(total, win_h, win_w, n_peaks))
            return PIV_ERROR_NOMEM;
        RectParams rp{};
        rp.A = d_A; rp.B = d_B; rp.img_stride = img_stride; rp.mask = d_mask;
        rp.H = H; rp.W = W; rp.nwy = n_win_y; rp.nwx = n_win_x; rp.nwt = (long long)n_win_y * n_win_x;
        rp.ctr_x = d_ctr_x; rp.ctr_y = d_ctr_y; rp.wA = d_wA; rp.wB = d_wB;
        rp.h = win_h; rp.w = win_w; rp.ensemble = ensemble; rp.planes_out = d_planes;
        return xcorr_rect(rp, total, n_peaks, peak_finder, peakfit_impl, d_cw, d_pk_x, d_pk_y, d_pk_h, d_sx, d_sy,
                          d_sxy, d_pk_ratio, d_scratch, (cudaStream_t)stream);
    }
    const bool lm = !ensemble && n_peaks == 1 && peak_finder >= 4 && peak_finder <= 6;
    if (lm && (d_scratch == nullptr || scratch_bytes < pivb_xcorr_scratch_bytes(total, n_peaks, peak_finder)))
        return PIV_ERROR_NOMEM;
    // 3-point fits also move to the per-window record kernel when the caller's
    // scratch holds the records (pivb_xcorr_record_bytes): the correlation kernel's
    // group leader then only extracts the patch; results are the same either way
    const bool defer = lm || (!ensemble && n_peaks == 1 && peak_finder == 3 && d_scratch != nullptr &&
                              scratch_bytes >= pivb_xcorr_record_bytes(total));
    cudaStream_t s = (cudaStream_t)stream;
    XcorrParams p{};
    p.A = d_A; p.B = d_B; p.img_stride = img_stride; p.mask = d_mask;
    p.H = H; p.W = W; p.n_img = n_images;
    p.ctr_x = d_ctr_x; p.ctr_y = d_ctr_y; p.nwy = n_win_y; p.nwx = n_win_x;
    p.wA = d_wA; p.wB = d_wB; p.cw = d_cw;
    p.ensemble = ensemble; p.n_peaks = n_peaks; p.finder = peak_finder;
    p.pk_x = d_pk_x; p.pk_y = d_pk_y; p.pk_h = d_pk_h; p.sx = d_sx; p.sy = d_sy; p.sxy = d_sxy;
    p.pk_ratio = d_pk_ratio; p.planes = d_planes;
    p.lm = defer ? static_cast<LmRecord *>(d_scratch) : nullptr;
    p.total = total;
    p.neg_zero = -0.0f;
    Workspace *tw = nullptr;
    if (g_timing != 0) {
        tw = cur_ws();
        if (tw == nullptr || tw->ensure(0)) return PIV_ERROR_CUDA;
    }
    const bool timing = tw != nullptr;
    if (timing) cudaEventRecord(tw->ev[0], s);
    int e = (n_peaks > 1 && !ensemble) ? launch_xcorr<true>(win_h, p, s) : launch_xcorr<false>(win_h, p, s);
    if (e) return e;
    if (timing) cudaEventRecord(tw->ev[1], s);
    if (defer) {
        const int er = launch_records(p, win_h, peakfit_impl, g_record_block.load(std::memory_order_relaxed), s);
        if (er) return er;
    }
    if (timing) {
        cudaEventRecord(tw->ev[2], s);
        if (cudaEventSynchronize(tw->ev[2]) != cudaSuccess) return PIV_ERROR_CUDA;
        float t0 = 0.f, t1 = 0.f;
        cudaEventElapsedTime(&t0, tw->ev[0], tw->ev[1]);
        cudaEventElapsedTime(&t1, tw->ev[1], tw->ev[2]);
        g_t_fft += t0 * 1e-3;
        g_t_fit += t1 * 1e-3;
    }
    return PIV_ERROR_NONE;
}


namespace {

template <int N>
constexpr size_t accum_smem_bytes()
{
    // the accumulation kernel has no use for the correlator's staged weights
    return (size_t)(WinGeo<N>::SMEM_BYTES - WinGeo<N>::WT_BYTES) + (size_t)WinGeo<N>::GROUPS_PER_CTA * 4 * N * N * 4;
}
template <int N>
constexpr bool accum_in_smem()
{
    return accum_smem_bytes<N>() <= 200 * 1024;
}

template <int N>
int accum_grid(long long nwt)
{
    using G = WinGeo<N>;
    constexpr bool SM = accum_in_smem<N>();
    static PerDeviceOnce per_sm_dev;
    const size_t smem = SM ? accum_smem_bytes<N>() : (size_t)(G::SMEM_BYTES - G::WT_BYTES);
    const int dev = current_device();
    if (dev < 0) return -1;
    const int per_sm = per_sm_dev.get(dev, [smem] {
        auto kern = accum_kernel<N, SM>;
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return -1;
        int nb = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, G::CTA_THREADS, smem) != cudaSuccess) return -1;
        return nb > 0 ? nb : 1;
    });
    if (per_sm < 0) {
        cudaGetLastError();
        return -1;
    }
    long long want = (nwt + G::GROUPS_PER_CTA - 1) / G::GROUPS_PER_CTA;
    long long cap = (long long)per_sm * device_sms(dev);
    return (int)(want < cap ? (want < 1 ? 1 : want) : cap);
}

template <int N>
size_t accum_scratch_n(long long nwt)
{
    size_t b = 256;   // weight sums
    if (!accum_in_smem<N>()) {
        int grid = accum_grid<N>(nwt);
        if (grid < 0) return (size_t)-1;
        b += pad256((size_t)grid * WinGeo<N>::GROUPS_PER_CTA * 4 * N * N * 4);
    }
    return b;
}

template <int N>
int accum_launch_n(AccumParams p, char *scratch, cudaStream_t s)
{
    using G = WinGeo<N>;
    constexpr bool SM = accum_in_smem<N>();
    const int grid = accum_grid<N>(p.nwt);
    if (grid < 0) return PIV_ERROR_CUDA;
    p.gacc = SM ? nullptr : reinterpret_cast<float *>(scratch + 256);
    const size_t smem = SM ? accum_smem_bytes<N>() : (size_t)(G::SMEM_BYTES - G::WT_BYTES);
    accum_kernel<N, SM><<<grid, G::CTA_THREADS, smem, s>>>(p);
    return cudaGetLastError() == cudaSuccess ? PIV_ERROR_NONE : PIV_ERROR_CUDA;
}

size_t accum_scratch(int N, long long nwt)
{
    switch (N) {
    case 8: return accum_scratch_n<8>(nwt);
    case 12: return accum_scratch_n<12>(nwt);
    case 16: return accum_scratch_n<16>(nwt);
    case 24: return accum_scratch_n<24>(nwt);
    case 32: return accum_scratch_n<32>(nwt);
    case 48: return accum_scratch_n<48>(nwt);
    case 64: return accum_scratch_n<64>(nwt);
    case 96: return accum_scratch_n<96>(nwt);
    case 128: return accum_scratch_n<128>(nwt);
    default: return 0;
    }
}

int accum_launch(int N, const AccumParams &p, char *scratch, cudaStream_t s)
{
    switch (N) {
    case 8: return accum_launch_n<8>(p, scratch, s);
    case 12: return accum_launch_n<12>(p, scratch, s);
    case 16: return accum_launch_n<16>(p, scratch, s);
    case 24: return accum_launch_n<24>(p, scratch, s);
    case 32: return accum_launch_n<32>(p, scratch, s);
    case 48: return accum_launch_n<48>(p, scratch, s);
    case 64: return accum_launch_n<64>(p, scratch, s);
    case 96: return accum_launch_n<96>(p, scratch, s);
    case 128: return accum_launch_n<128>(p, scratch, s);
    default: return PIV_ERROR_NOPLAN_BWD;
    }
}

int accumulate_dev(const float *d_A, const float *d_B, long long img_stride, const float *d_mask, int H, int W,
                   int n_images, const float *d_ctr_x, const float *d_ctr_y, int nwy, int nwx, const float *w1,
                   const float *w2, const float *w3, const float *w4, int win_h, int win_w, int out_h, int out_w,
                   int mean_sub, int ppn, int triple, float *d_ab, float *d_aa, float *d_bb, float *d_comp,
                   void *d_scratch, size_t scratch_bytes, cudaStream_t s)
{
    if (!size_ok(win_h) || !size_ok(win_w)) return PIV_ERROR_NOPLAN_BWD;
    if (win_h != win_w) return PIV_ERROR_NOPLAN;
    if (out_h <= 0 || out_w <= 0 || out_h > win_h || out_w > win_w) return PIV_ERROR_OUT_OF_BOUNDS;
    const long long nwt = (long long)nwy * nwx;
    if (nwt == 0 || n_images <= 0) return PIV_ERROR_NONE;
    const size_t need = accum_scratch(win_h, nwt);
    if (need == (size_t)-1) return PIV_ERROR_CUDA;
    if (!d_scratch || scratch_bytes < need) return PIV_ERROR_NOMEM;
    char *scr = static_cast<char *>(d_scratch);
    float *wsums = reinterpret_cast<float *>(scr);
    if (triple && mean_sub) {
        weight_sums_kernel<<<1, 32, 0, s>>>(w2, w3, w4, win_h * win_w, wsums);
        if (cudaGetLastError() != cudaSuccess) return PIV_ERROR_CUDA;
    }
    AccumParams p{};
    p.A = d_A; p.B = d_B; p.img_stride = img_stride; p.mask = d_mask;
    p.H = H; p.W = W; p.n_img = n_images; p.ctr_x = d_ctr_x; p.ctr_y = d_ctr_y; p.nwy = nwy; p.nwx = nwx;
    p.w_ab_a = w1; p.w_ab_b = w2; p.w_aa = w3; p.w_bb = w4; p.wsums = wsums;
    p.out_h = out_h; p.out_w = out_w; p.sy0 = (win_h - out_h) / 2; p.sx0 = (win_w - out_w) / 2;
    p.mean_sub = mean_sub; p.ppn = ppn; p.triple = triple;
    p.ab = d_ab; p.aa = d_aa; p.bb = d_bb; p.comp = d_comp; p.nwt = nwt;
    return accum_launch(win_h, p, scr, s);
}

}  // namespace

// Scratch bytes of the device accumulation entry points.
PIV_EXPORT size_t pivb_accumulate_scratch_bytes(int win, long long n_windows)
{
    size_t b = accum_scratch(win, n_windows);
    return b == (size_t)-1 ? 0 : b;
}

// bulkxcorr2d_accumulate_triple on device pointers; d_comp (nullable) carries the
// Kahan compensation [3][nwt][out_h*out_w] across calls.
PIV_EXPORT int pivb_accumulate_triple_dev(const float *d_A, const float *d_B, long long img_stride,
                                          const float *d_mask, int H, int W, int n_images, const float *d_ctr_x,
                                          const float *d_ctr_y, int n_win_y, int n_win_x, const float *d_w_ab_a,
                                          const float *d_w_ab_b, const float *d_w_auto_a, const float *d_w_auto_b,
                                          int win_h, int win_w, int out_h, int out_w, int mean_subtract,
                                          int per_pair_norm, float *d_ab, float *d_aa, float *d_bb, float *d_comp,
                                          void *d_scratch, size_t scratch_bytes, void *stream)
{
    return accumulate_dev(d_A, d_B, img_stride, d_mask, H, W, n_images, d_ctr_x, d_ctr_y, n_win_y, n_win_x,
                          d_w_ab_a, d_w_ab_b, d_w_auto_a, d_w_auto_b, win_h, win_w, out_h, out_w, mean_subtract,
                          per_pair_norm, 1, d_ab, d_aa, d_bb, d_comp, d_scratch, scratch_bytes, (cudaStream_t)stream);
}

// bulkxcorr2d_accumulate on device pointers (AB only, no mean subtraction).
PIV_EXPORT int pivb_accumulate_dev(const float *d_A, const float *d_B, long long img_stride, const float *d_mask,
                                   int H, int W, int n_images, const float *d_ctr_x, const float *d_ctr_y,
                                   int n_win_y, int n_win_x, const float *d_wA, const float *d_wB, int win_h,
                                   int win_w, int out_h, int out_w, float *d_sum, float *d_comp, void *d_scratch,
                                   size_t scratch_bytes, void *stream)
{
    return accumulate_dev(d_A, d_B, img_stride, d_mask, H, W, n_images, d_ctr_x, d_ctr_y, n_win_y, n_win_x, d_wA,
                          d_wB, nullptr, nullptr, win_h, win_w, out_h, out_w, 0, 0, 0, d_sum, nullptr, nullptr,
                          d_comp, d_scratch, scratch_bytes, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// Reference C-ABI (host pointers)
// ---------------------------------------------------------------------------

// PIV_2d_cross_correlate.h:18-20
PIV_EXPORT unsigned char bulkxcorr2d(const float *fImageA, const float *fImageB, const float *fMask,
                                     const int *nImageSize, int N_images, const float *fWinCtrsX,
                                     const float *fWinCtrsY, const int *nWindows, float *fWindowWeightA,
                                     bool bEnsemble, const float *fWindowWeightB, const int *nWindowSize,
                                     int nPeaks, int iPeakFinder, float *fPkLocX, float *fPkLocY,
                                     float *fPkHeight, float *fSx, float *fSy, float *fSxy,
                                     float *fPkRatio, float *fCorrelPlane_Out)
{
    const int h = nWindowSize[0], w = nWindowSize[1];
    if (!size_ok(h) || !size_ok(w)) return PIV_ERROR_NOPLAN_BWD;
    std::lock_guard<std::mutex> lock(g_mu);
    const int H = nImageSize[0], W = nImageSize[1];
    const int nwy = nWindows[0], nwx = nWindows[1];
    const long long nwt = (long long)nwy * nwx;
    const long long total = (long long)N_images * nwt;
    const size_t img = (size_t)N_images * H * W;
    const size_t nout = (size_t)N_images * nPeaks * nwt;
    const size_t nrat = (size_t)N_images * nwt;
    const size_t npl = (size_t)h * w;
    const int impl = g_peakfit_impl;
    const size_t scratch = pivb_xcorr_scratch_bytes_hw(total, h, w, nPeaks, iPeakFinder);
    size_t bytes = 2 * pad256(img * 4) + pad256(nwt * 4) + pad256(nwx * 4) + pad256(nwy * 4) +
                   3 * pad256(npl * 4) + 6 * pad256(nout * 4) + pad256(nrat * 4) +
                   (fCorrelPlane_Out ? pad256((size_t)total * npl * 4) : 0) + scratch + 4096;
    Workspace *wsp = cur_ws();
    if (wsp == nullptr) return PIV_ERROR_CUDA;
    int e = wsp->ensure(bytes);
    if (e) return (unsigned char)e;
    cudaStream_t s = wsp->stream;
    Carve c(wsp->dev);
    float *dA = c.take<float>(img), *dB = c.take<float>(img);
    float *dmask = c.take<float>(nwt), *dcx = c.take<float>(nwx), *dcy = c.take<float>(nwy);
    float *dwa = c.take<float>(npl), *dwb = c.take<float>(npl), *dcw = c.take<float>(npl);
    float *o[6];
    for (auto &q : o) q = c.take<float>(nout);
    float *drat = c.take<float>(nrat);
    float *dpl = fCorrelPlane_Out ? c.take<float>((size_t)total * npl) : nullptr;
    void *dscr = scratch ? (void *)c.take<char>(scratch) : nullptr;
    float *host_out[6] = {fPkLocX, fPkLocY, fPkHeight, fSx, fSy, fSxy};
#define H2D(dst, src, n) if (cudaMemcpyAsync(dst, src, (n) * sizeof(float), cudaMemcpyHostToDevice, s) != cudaSuccess) return PIV_ERROR_CUDA
#define D2H(dst, src, n) if (cudaMemcpyAsync(dst, src, (n) * sizeof(float), cudaMemcpyDeviceToHost, s) != cudaSuccess) return PIV_ERROR_CUDA
    H2D(dA, fImageA, img);
    H2D(dB, fImageB, img);
    H2D(dmask, fMask, nwt);
    H2D(dcx, fWinCtrsX, nwx);
    H2D(dcy, fWinCtrsY, nwy);
    H2D(dwa, fWindowWeightA, npl);
    H2D(dwb, fWindowWeightB, npl);
    if (!bEnsemble) {
        // skipped windows keep the caller's values
        for (int k = 0; k < 6; ++k) H2D(o[k], host_out[k], nout);
        H2D(drat, fPkRatio, nrat);
    }
    if (dpl) H2D(dpl, fCorrelPlane_Out, (size_t)total * npl);
    if ((e = pivb_correl_weight_dev(dwb, h, w, dcw, s))) return (unsigned char)e;
    e = pivb_xcorr_dev(dA, dB, (long long)H * W, dmask, H, W, N_images, dcx, dcy, nwy, nwx, dwa, dwb, dcw,
                       h, w, bEnsemble ? 1 : 0, nPeaks, iPeakFinder, impl, o[0], o[1], o[2], o[3], o[4],
                       o[5], drat, dpl, dscr, scratch, s);
    if (e) return (unsigned char)e;
    if (!bEnsemble) {
        for (int k = 0; k < 6; ++k) D2H(host_out[k], o[k], nout);
        D2H(fPkRatio, drat, nrat);
    }
    if (dpl) D2H(fCorrelPlane_Out, dpl, (size_t)total * npl);
#undef H2D
#undef D2H
    if (cudaStreamSynchronize(s) != cudaSuccess) return PIV_ERROR_CUDA;
    return PIV_ERROR_NONE;
}


namespace {
int accumulate_host(const float *A, const float *B, const float *mask, const int *img_size, int n_images,
                    const float *cx, const float *cy, const int *n_win, const float *w1, const float *w2,
                    const float *w3, const float *w4, const int *ws, const int *fs, int mean_sub, int ppn,
                    int triple, float *ab, float *aa, float *bb)
{
    const int h = ws[0], w = ws[1];
    if (!size_ok(h) || !size_ok(w)) return PIV_ERROR_NOPLAN_BWD;
    if (h != w) return PIV_ERROR_NOPLAN;
    std::lock_guard<std::mutex> lock(g_mu);
    const int H = img_size[0], W = img_size[1];
    const int nwy = n_win[0], nwx = n_win[1];
    const long long nwt = (long long)nwy * nwx;
    const int oh = fs ? fs[0] : h, ow = fs ? fs[1] : w;
    const size_t img = (size_t)n_images * H * W, npl = (size_t)h * w, nout = (size_t)nwt * oh * ow;
    const int nacc = triple ? 3 : 1;
    Workspace *wsp = cur_ws();
    if (wsp == nullptr) return PIV_ERROR_CUDA;
    int e = wsp->ensure(16);   // device + stream setup before the occupancy query
    if (e) return e;
    const size_t scr = accum_scratch(h, nwt);
    if (scr == (size_t)-1) return PIV_ERROR_CUDA;
    size_t bytes = 2 * pad256(img * 4) + pad256(nwt * 4) + pad256(nwx * 4) + pad256(nwy * 4) + 4 * pad256(npl * 4) +
                   nacc * pad256(nout * 4) + pad256(scr) + 4096;
    if ((e = wsp->ensure(bytes))) return e;
    cudaStream_t s = wsp->stream;
    Carve c(wsp->dev);
    float *dA = c.take<float>(img), *dB = c.take<float>(img);
    float *dm = c.take<float>(nwt), *dcx = c.take<float>(nwx), *dcy = c.take<float>(nwy);
    float *dw[4];
    for (auto &q : dw) q = c.take<float>(npl);
    float *dout[3] = {nullptr, nullptr, nullptr};
    float *hout[3] = {ab, aa, bb};
    for (int a = 0; a < nacc; ++a) dout[a] = c.take<float>(nout);
    char *dscr = c.take<char>(scr);
    const float *hw[4] = {w1, w2, w3, w4};
#define H2D(dst, src, n) if (cudaMemcpyAsync(dst, src, (n) * sizeof(float), cudaMemcpyHostToDevice, s) != cudaSuccess) return PIV_ERROR_CUDA
    H2D(dA, A, img);
    H2D(dB, B, img);
    H2D(dm, mask, nwt);
    H2D(dcx, cx, nwx);
    H2D(dcy, cy, nwy);
    for (int k = 0; k < (triple ? 4 : 2); ++k) H2D(dw[k], hw[k], npl);
    for (int a = 0; a < nacc; ++a) H2D(dout[a], hout[a], nout);
#undef H2D
    e = accumulate_dev(dA, dB, (long long)H * W, dm, H, W, n_images, dcx, dcy, nwy, nwx, dw[0], dw[1],
                       triple ? dw[2] : nullptr, triple ? dw[3] : nullptr, h, w, oh, ow, mean_sub, ppn, triple,
                       dout[0], dout[1], dout[2], nullptr, dscr, scr, s);
    if (e) return e;
    for (int a = 0; a < nacc; ++a)
        if (cudaMemcpyAsync(hout[a], dout[a], nout * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess) return PIV_ERROR_CUDA;
    return cudaStreamSynchronize(s) == cudaSuccess ? PIV_ERROR_NONE : PIV_ERROR_CUDA;
}
}  // namespace

// PIV_2d_cross_correlate.h:37-51
PIV_EXPORT unsigned char bulkxcorr2d_accumulate(const float *fImageA_stack, const float *fImageB_stack,
                                                const float *fMask, const int *nImageSize, int N_images,
                                                const float *fWinCtrsX, const float *fWinCtrsY, const int *nWindows,
                                                const float *fWindowWeightA, const float *fWindowWeightB,
                                                const int *nWindowSize, const int *nFitWindowSize,
                                                float *fCorrelPlane_Sum)
{
    return (unsigned char)accumulate_host(fImageA_stack, fImageB_stack, fMask, nImageSize, N_images, fWinCtrsX,
                                          fWinCtrsY, nWindows, fWindowWeightA, fWindowWeightB, nullptr, nullptr,
                                          nWindowSize, nFitWindowSize, 0, 0, 0, fCorrelPlane_Sum, nullptr, nullptr);
}

// PIV_2d_cross_correlate.h:66-86
PIV_EXPORT unsigned char bulkxcorr2d_accumulate_triple(const float *fImageA_stack, const float *fImageB_stack,
                                                       const float *fMask, const int *nImageSize, int N_images,
                                                       const float *fWinCtrsX, const float *fWinCtrsY,
                                                       const int *nWindows, const float *fWindowWeightA_AB,
                                                       const float *fWindowWeightB_AB, const float *fAutoWeightA,
                                                       const float *fAutoWeightB, const int *nWindowSize,
                                                       const int *nFitWindowSize, int bMeanSubtract, int bPerPairNorm,
                                                       float *fCorrAB_Sum, float *fCorrAA_Sum, float *fCorrBB_Sum)
{
    return (unsigned char)accumulate_host(fImageA_stack, fImageB_stack, fMask, nImageSize, N_images, fWinCtrsX,
                                          fWinCtrsY, nWindows, fWindowWeightA_AB, fWindowWeightB_AB, fAutoWeightA,
                                          fAutoWeightB, nWindowSize, nFitWindowSize, bMeanSubtract, bPerPairNorm, 1,
                                          fCorrAB_Sum, fCorrAA_Sum, fCorrBB_Sum);
}

PIV_EXPORT void bulkxcorr2d_set_timing_enabled(int on) { g_timing = on ? 1 : 0; }
PIV_EXPORT void bulkxcorr2d_reset_timing(void) { g_t_fft = 0.0; g_t_fit = 0.0; }
PIV_EXPORT void bulkxcorr2d_get_timing(double *fft_s, double *fit_s)
{
    if (fft_s) *fft_s = g_t_fft;
    if (fit_s) *fit_s = g_t_fit;
}

// Peak-fit implementation: 0 = scalar-fitter semantics, 1 = batch-fitter
// semantics (its exponential and trust-rule arithmetic).  Both run on the GPU.
PIV_EXPORT int bulkxcorr2d_set_peakfit_impl(int impl)
{
    g_peakfit_impl = impl ? 1 : 0;
    return 0;
}
PIV_EXPORT int bulkxcorr2d_get_peakfit_impl(void) { return g_peakfit_impl; }
PIV_EXPORT int bulkxcorr2d_peakfit_batch_available(void) { return 1; }

// Lane width reported to callers that size [3][lanes] batch arrays; the GPU
// fitter has no lane limit, this is the reference's PEAKFIT_MAX_LANES.
#define PIVB_BATCH_LANES 16
PIV_EXPORT int peakfit_batch_available(void) { return 1; }
PIV_EXPORT int peakfit_batch_lanes(void) { return PIVB_BATCH_LANES; }
PIV_EXPORT int codelet_lanes(void) { return PIVB_BATCH_LANES; }

// The reference's loader refuses a library without this symbol; there is no CPU
// instruction-set floor here.
PIV_EXPORT int pivtools_cpu_supported(void) { return 1; }

// Fit arbitrary planes on the GPU (shared by the single-plane entry points).
static int fit_planes_host(const float *planes, int n_planes, const int *N, int nPeaks, int iFitType,
                           const float *wt, float *loc, float *sd, int layout, int lanes, float *ratio,
                           int mode)
{
    std::lock_guard<std::mutex> lock(g_mu);
    const size_t npl = (size_t)N[0] * N[1];
    const size_t nloc = layout == 0 ? (size_t)n_planes * 3 * nPeaks : (size_t)3 * lanes;
    size_t bytes = pad256(n_planes * npl * 4) * (nPeaks > 1 ? 2 : 1) + pad256(npl * 4) + 2 * pad256(nloc * 4) +
                   pad256((size_t)n_planes * 4) + 4096;
    Workspace *wsp = cur_ws();
    if (wsp == nullptr) return PIV_ERROR_CUDA;
    int e = wsp->ensure(bytes);
    if (e) return e;
    cudaStream_t s = wsp->stream;
    Carve c(wsp->dev);
    float *dp = c.take<float>(n_planes * npl);
    float *dw = wt ? c.take<float>(npl) : nullptr;
    float *dl = loc ? c.take<float>(nloc) : nullptr;
    float *ds = loc ? c.take<float>(nloc) : nullptr;
    float *dr = ratio ? c.take<float>(n_planes) : nullptr;
    float *work = nPeaks > 1 ? c.take<float>(n_planes * npl) : nullptr;
    if (cudaMemcpyAsync(dp, planes, n_planes * npl * 4, cudaMemcpyHostToDevice, s) != cudaSuccess) return PIV_ERROR_CUDA;
    if (dw && cudaMemcpyAsync(dw, wt, npl * 4, cudaMemcpyHostToDevice, s) != cudaSuccess) return PIV_ERROR_CUDA;
    if (dl) {
        // entries the kernel does not write (batch lanes >= L_real) keep the caller's values
        if (cudaMemcpyAsync(dl, loc, nloc * 4, cudaMemcpyHostToDevice, s) != cudaSuccess) return PIV_ERROR_CUDA;
        if (cudaMemcpyAsync(ds, sd, nloc * 4, cudaMemcpyHostToDevice, s) != cudaSuccess) return PIV_ERROR_CUDA;
    }
    if (mode)
        fit_planes_kernel<1><<<n_planes, 128, 0, s>>>(dp, N[0], N[1], nPeaks, iFitType, dw, dl, ds, layout, lanes, dr, work);
    else
        fit_planes_kernel<0><<<n_planes, 128, 0, s>>>(dp, N[0], N[1], nPeaks, iFitType, dw, dl, ds, layout, lanes, dr, work);
    if (cudaGetLastError() != cudaSuccess) return PIV_ERROR_CUDA;
    if (dl) {
        if (cudaMemcpyAsync(loc, dl, nloc * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess) return PIV_ERROR_CUDA;
        if (cudaMemcpyAsync(sd, ds, nloc * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess) return PIV_ERROR_CUDA;
    }
    if (dr && cudaMemcpyAsync(ratio, dr, (size_t)n_planes * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return PIV_ERROR_CUDA;
    return cudaStreamSynchronize(s) == cudaSuccess ? PIV_ERROR_NONE : PIV_ERROR_CUDA;
}

static void nan_sentinel(float *loc, float *sd, int nPeaks)
{
    for (int k = 0; k < nPeaks; ++k) {
        loc[k] = NAN; loc[nPeaks + k] = NAN; loc[2 * nPeaks + k] = 0.0f;
        sd[k] = 0.0f; sd[nPeaks + k] = 0.0f; sd[2 * nPeaks + k] = 0.0f;
    }
}

// peak_locate_lm.h:39 -- scalar-fitter semantics, any plane size.
PIV_EXPORT void lsqpeaklocate_lm(const float *xcorr, const int *N, float *peak_loc, int nPeaks, int iFitType,
                                 float *std_dev, const float *fPlaneWeight)
{
    if (nPeaks < 1) return;
    if (fit_planes_host(xcorr, 1, N, nPeaks, iFitType, fPlaneWeight, peak_loc, std_dev, 0, 0, nullptr, 0)) {
        fprintf(stderr, "lsqpeaklocate_lm: GPU call failed\n");
        nan_sentinel(peak_loc, std_dev, nPeaks);
    }
}

// peak_locate_lm.h:46
PIV_EXPORT float peak_detectability(const float *xcorr, const int *N)
{
    float r = 0.0f;
    if (fit_planes_host(xcorr, 1, N, 1, 3, nullptr, nullptr, nullptr, 0, 0, &r, 0)) {
        fprintf(stderr, "peak_detectability: GPU call failed\n");
        return NAN;
    }
    return r;
}

// peak_locate_lm_batch.h:39-42 -- batch-fitter semantics; lanes >= L_real NaN.
PIV_EXPORT void lsqpeaklocate_lm_batch(const float *planes, int L_real, const int *N, int iFitType,
                                       float *peak_loc, float *std_dev, const float *fPlaneWeight)
{
    const int W = PIVB_BATCH_LANES;
    for (int l = 0; l < W; ++l) {
        peak_loc[l] = NAN; peak_loc[W + l] = NAN; peak_loc[2 * W + l] = 0.0f;
        std_dev[l] = 0.0f; std_dev[W + l] = 0.0f; std_dev[2 * W + l] = 0.0f;
    }
    if (iFitType < 4 || iFitType > 6) {
        fprintf(stderr, "lsqpeaklocate_lm_batch: unsupported iFitType %d\n", iFitType);
        return;
    }
    const int L = L_real < W ? L_real : W;
    if (L <= 0) return;
    if (fit_planes_host(planes, L, N, 1, iFitType, fPlaneWeight, peak_loc, std_dev, 1, W, nullptr, 1))
        fprintf(stderr, "lsqpeaklocate_lm_batch: GPU call failed\n");
}

// xcorr.h:26 -- linear correlation of two weights, centre of the 2N-padded result.
PIV_EXPORT unsigned convolve(const float *w1, const float *w2, float *conv, const int *N)
{
    std::lock_guard<std::mutex> lock(g_mu);
    const int h = N[0], w = N[1];
    if (h <= 0 || w <= 0) return PIV_ERROR_NOPLAN_BWD;
    const size_t n = (size_t)h * w;
    Workspace *wsp = cur_ws();
    if (wsp == nullptr) return PIV_ERROR_CUDA;
    int e = wsp->ensure(3 * pad256(n * 4) + 1024);
    if (e) return e;
    cudaStream_t s = wsp->stream;
    Carve c(wsp->dev);
    float *a = c.take<float>(n), *b = c.take<float>(n), *o = c.take<float>(n);
    if (cudaMemcpyAsync(a, w1, n * 4, cudaMemcpyHostToDevice, s) != cudaSuccess) return PIV_ERROR_CUDA;
    if (cudaMemcpyAsync(b, w2, n * 4, cudaMemcpyHostToDevice, s) != cudaSuccess) return PIV_ERROR_CUDA;
    lin_xcorr_kernel<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(a, b, h, w, o, 0);
    if (cudaGetLastError() != cudaSuccess) return PIV_ERROR_CUDA;
    if (cudaMemcpyAsync(conv, o, n * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess) return PIV_ERROR_CUDA;
    return cudaStreamSynchronize(s) == cudaSuccess ? PIV_ERROR_NONE : PIV_ERROR_CUDA;
}

// xcorr.h:27 -- circular correlation, fftshifted (built sizes only).
PIV_EXPORT unsigned xcorr(const float *w1, const float *w2, float *corr, const int *N)
{
    std::lock_guard<std::mutex> lock(g_mu);
    const int h = N[0], w = N[1];
    if (h <= 0 || w <= 0 || !size_ok(h) || !size_ok(w)) return PIV_ERROR_NOPLAN_BWD;
    const size_t n = (size_t)h * w;
    Workspace *wsp = cur_ws();
    if (wsp == nullptr) return PIV_ERROR_CUDA;
    int e = wsp->ensure(3 * pad256(n * 4) + 1024);
    if (e) return e;
    cudaStream_t s = wsp->stream;
    Carve c(wsp->dev);
    float *a = c.take<float>(n), *b = c.take<float>(n), *o = c.take<float>(n);
    if (cudaMemcpyAsync(a, w1, n * 4, cudaMemcpyHostToDevice, s) != cudaSuccess) return PIV_ERROR_CUDA;
    if (cudaMemcpyAsync(b, w2, n * 4, cudaMemcpyHostToDevice, s) != cudaSuccess) return PIV_ERROR_CUDA;
    circ_xcorr_kernel<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(a, b, h, w, o);
    if (cudaGetLastError() != cudaSuccess) return PIV_ERROR_CUDA;
    if (cudaMemcpyAsync(corr, o, n * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess) return PIV_ERROR_CUDA;
    return cudaStreamSynchronize(s) == cudaSuccess ? PIV_ERROR_NONE : PIV_ERROR_CUDA;
}

static float minmax_host(const float *v, int n, int want_max)
{
    if (n <= 0) return NAN;
    std::lock_guard<std::mutex> lock(g_mu);
    Workspace *wsp = cur_ws();
    if (wsp == nullptr || wsp->ensure(pad256((size_t)n * 4) + 1024)) return NAN;
    cudaStream_t s = wsp->stream;
    Carve c(wsp->dev);
    float *d = c.take<float>(n), *out = c.take<float>(1);
    int *last = c.take<int>(1);
    const int minus1 = -1;
    float r = NAN;
    if (cudaMemcpyAsync(d, v, (size_t)n * 4, cudaMemcpyHostToDevice, s) != cudaSuccess) return NAN;
    if (cudaMemcpyAsync(last, &minus1, 4, cudaMemcpyHostToDevice, s) != cudaSuccess) return NAN;
    last_nan_kernel<<<(n + 255) / 256 < 1024 ? (n + 255) / 256 : 1024, 256, 0, s>>>(d, n, last);
    minmax_fold_kernel<<<1, 256, 0, s>>>(d, n, last, want_max, out);
    if (cudaMemcpyAsync(&r, out, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess) return NAN;
    if (cudaStreamSynchronize(s) != cudaSuccess) return NAN;
    return r;
}

// PIV_2d_cross_correlate.h:88-89
PIV_EXPORT float fminvec(const float *fVec, int n) { return minmax_host(fVec, n, 0); }
PIV_EXPORT float fmaxvec(const float *fVec, int n) { return minmax_host(fVec, n, 1); }

// Device ordinal and name of the GPU this library computes on (diagnostics).
PIV_EXPORT int pivb_device_info(char *name, int len)
{
    int d = -1;
    if (cudaGetDevice(&d) != cudaSuccess) return -1;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, d) != cudaSuccess) return -1;
    if (name && len > 0) {
        strncpy(name, prop.name, (size_t)len - 1);
        name[len - 1] = 0;
    }
    return d;
}

// ---------------------------------------------------------------------------
// Allocation-free correlation entry point
// ---------------------------------------------------------------------------
// For callers that cannot allocate device memory themselves: a host whose
// device memory is owned by another allocator (a framework's caching pool that
// has reserved the GPU), a stream that is being captured into a CUDA graph, or a
// latency-bound pipeline that cannot afford the device-wide synchronisation
// cudaFree implies.  The scratch of the deferred LM fits then lives in a
// file-scope device array of fixed size instead of a caller-provided buffer.
//
// Limit: 16 MiB, i.e. 131072 windows (image pairs x windows per pair) per call
// when the call needs LM records (nPeaks == 1 and peak finder 4, 5 or 6); larger
// calls are refused with PIV_ERROR_NOMEM and a message on stderr.  Calls without
// LM records use no scratch and have no limit.  Every GPU that loads this library
// holds the array until the process exits.
//
// The array is shared by every call on a device and keeps the last call's
// contents.  Nothing in it needs clearing: the correlation kernel writes every
// record the LM kernel reads, earlier on the same stream.  Calls whose work
// overlaps on the GPU (different streams or host threads without ordering)
// race on the array.
//
// Set-up: the first call on a device (with that device current) resolves the
// array's device address with cudaGetSymbolAddress and sets up the launch
// configuration of the correlation kernels of every built window size, single-
// and multi-peak (their shared-memory limit and occupancy on that device); make
// that first call, of any size, before any stream capture.
// Neither this set-up nor a call allocates memory: no cudaMalloc, cudaFree or
// allocating library routine is used.
#define PIVB_NOALLOC_SCRATCH_BYTES (16u << 20)
static __device__ __align__(256) unsigned char g_noalloc_scratch[PIVB_NOALLOC_SCRATCH_BYTES];

namespace {
void *g_noalloc_addr[kMaxDevices] = {};
std::mutex g_noalloc_mu;

template <bool MULTI>
bool setup_all_sizes(int dev)
{
    return xcorr_blocks_per_sm<8, MULTI>(dev) >= 0 && xcorr_blocks_per_sm<12, MULTI>(dev) >= 0 &&
           xcorr_blocks_per_sm<16, MULTI>(dev) >= 0 && xcorr_blocks_per_sm<24, MULTI>(dev) >= 0 &&
           xcorr_blocks_per_sm<32, MULTI>(dev) >= 0 && xcorr_blocks_per_sm<48, MULTI>(dev) >= 0 &&
           xcorr_blocks_per_sm<64, MULTI>(dev) >= 0 && xcorr_blocks_per_sm<96, MULTI>(dev) >= 0 &&
           xcorr_blocks_per_sm<128, MULTI>(dev) >= 0;
}

// Device address of the scratch array on the current device, set up on the
// first call there (see above); nullptr on failure.
void *noalloc_setup()
{
    const int dev = current_device();
    if (dev < 0) return nullptr;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (g_noalloc_addr[dev] == nullptr) {
        void *addr = nullptr;
        if (cudaGetSymbolAddress(&addr, g_noalloc_scratch) != cudaSuccess || addr == nullptr) {
            cudaGetLastError();
            return nullptr;
        }
        if (!setup_all_sizes<false>(dev) || !setup_all_sizes<true>(dev) || !lm_fit_setup(dev)) {
            cudaGetLastError();
            return nullptr;
        }
        g_noalloc_addr[dev] = addr;
    }
    return g_noalloc_addr[dev];
}
}  // namespace

// pivb_xcorr_dev without the scratch arguments (see the block comment above).
PIV_EXPORT int pivb_xcorr_dev_noalloc(const float *d_A, const float *d_B, long long img_stride,
                                      const float *d_mask, int H, int W, int n_images, const float *d_ctr_x,
                                      const float *d_ctr_y, int n_win_y, int n_win_x, const float *d_wA,
                                      const float *d_wB, const float *d_cw, int win_h, int win_w, int ensemble,
                                      int n_peaks, int peak_finder, int peakfit_impl, float *d_pk_x, float *d_pk_y,
                                      float *d_pk_h, float *d_sx, float *d_sy, float *d_sxy, float *d_pk_ratio,
                                      float *d_planes, void *stream)
{
    if (!size_ok(win_h) || !size_ok(win_w)) return PIV_ERROR_NOPLAN_BWD;
    if (win_h != win_w) return PIV_ERROR_NOPLAN;
    if (n_peaks < 1 || n_images < 0) return PIV_ERROR_OUT_OF_BOUNDS;
    void *scratch = noalloc_setup();
    if (scratch == nullptr) return PIV_ERROR_CUDA;
    const long long total = (long long)n_images * n_win_y * n_win_x;
    if (total == 0) return PIV_ERROR_NONE;
    const bool lm = !ensemble && n_peaks == 1 && peak_finder >= 4 && peak_finder <= 6;
    if (lm) {
        const size_t need = (size_t)total * sizeof(LmRecord);
        if (need > PIVB_NOALLOC_SCRATCH_BYTES) {
            fprintf(stderr,
                    "pivb_xcorr_dev_noalloc: %lld windows need %zu bytes of LM scratch; the fixed array holds "
                    "%u bytes (%u windows); split the call\n",
                    total, need, PIVB_NOALLOC_SCRATCH_BYTES, (unsigned)(PIVB_NOALLOC_SCRATCH_BYTES / sizeof(LmRecord)));
            return PIV_ERROR_NOMEM;
        }
    }
    LmRecord *records = lm ? static_cast<LmRecord *>(scratch) : nullptr;
    cudaStream_t s = (cudaStream_t)stream;
    XcorrParams p{};
    p.A = d_A; p.B = d_B; p.img_stride = img_stride; p.mask = d_mask;
    p.H = H; p.W = W; p.n_img = n_images;
    p.ctr_x = d_ctr_x; p.ctr_y = d_ctr_y; p.nwy = n_win_y; p.nwx = n_win_x;
    p.wA = d_wA; p.wB = d_wB; p.cw = d_cw;
    p.ensemble = ensemble; p.n_peaks = n_peaks; p.finder = peak_finder;
    p.pk_x = d_pk_x; p.pk_y = d_pk_y; p.pk_h = d_pk_h; p.sx = d_sx; p.sy = d_sy; p.sxy = d_sxy;
    p.pk_ratio = d_pk_ratio; p.planes = d_planes;
    p.lm = records;
    p.total = total;
    p.neg_zero = -0.0f;
    const int e = (n_peaks > 1 && !ensemble) ? launch_xcorr<true>(win_h, p, s) : launch_xcorr<false>(win_h, p, s);
    if (e) return e;
    if (lm) {
        const int er = launch_records(p, win_h, peakfit_impl, 128, s);
        if (er) return er;
    }
    return PIV_ERROR_NONE;
}
