// Data ingestion before reconstruct(): the APS driver's normalisation of raw
// detector counts by bright (white) and dark fields, the standard driver's
// down-sampling of ready-made projections and weights, and the interlaced
// view generator (TIMBIR src/reconstruct/aps_data/XT_HDFIO.c read_data,
// std_data/XT_HDFIO.c read_ProjWeightData, aps_data/XT_Views.c).  The HDF5
// file access itself is the caller's: these entry points take the datasets'
// arrays as the file holds them ([frames][rows][cols]) and select the same
// hyperslabs the readers select.
//
// Arithmetic follows the readers operation for operation (float sums in the
// same order, the double-precision fabs / log / quadratic of the C code and
// their roundings to float), so the results equal the reference's; log is
// CUDA's double log, which can differ from the host C library's in the last
// bit of a double and so, rarely, move a projection by one float ulp.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <cmath>
#include <cstdio>
#include <vector>

#include "../../include/timbir_b200.h"
#include "mbir_host.h"

namespace {

thread_local char g_ing_err[256];

int ing_fail(const char *msg, cudaError_t e = cudaSuccess)
{
    snprintf(g_ing_err, sizeof g_ing_err, "%s%s%s", msg, e != cudaSuccess ? ": " : "",
             e != cudaSuccess ? cudaGetErrorString(e) : "");
    return -1;
}

#define IK(call)                                                   \
    do {                                                           \
        cudaError_t _e = (call);                                   \
        if (_e != cudaSuccess) return ing_fail(#call, _e);         \
    } while (0)

// Mean over frames of a [nf][rows][cols] uint16 stack, per (row, col) of the
// selected window (XT_HDFIO.c:178-199): float sum in frame order, then / nf.
__global__ void k_frame_mean(const uint16_t *__restrict__ frames, int nf, int rows, int cols, float *__restrict__ out)
{
    const size_t n = (size_t)rows * cols;
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    float s = 0.0f;
    for (int i = 0; i < nf; i++) s = __fadd_rn(s, (float)frames[(size_t)i * n + q]);
    out[q] = __fdiv_rn(s, (float)nf);
}

// Projections and weights (XT_HDFIO.c:203-215): per output sample (view,
// row j, column k) the ratio x ratio block of raw samples at (j ratio + m,
// k ratio + n): weights = sum |count - dark|, bright = sum |white - dark|
// (float accumulators, double fabs and adds rounded to float), t =
// log(bright / weights) rounded to float, projection = bh t^2 + t.  counts:
// [views][srows][scols] (the window), white / dark: [srows][scols] means.
// A thread owns one (j, k) for a chunk of kNormViews views: the bright sum,
// which does not depend on the view (the reference recomputes it per view,
// to the same value), once per chunk; grid (column blocks, rows, view
// chunks), so no index division.
constexpr int kNormViews = 32;

__global__ void __launch_bounds__(128) k_normalize(const uint16_t *__restrict__ counts,
                                                   const float *__restrict__ white, const float *__restrict__ dark,
                                                   int views, int srows, int scols, int ratio, int prows, int pcols,
                                                   double bh, float *__restrict__ proj, float *__restrict__ wts)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (k >= pcols) return;
    const int v0 = blockIdx.z * kNormViews, v1 = min(views, v0 + kNormViews);
    float wd = 0.0f;
    for (int m = 0; m < ratio; m++)
        for (int q = 0; q < ratio; q++) {
            const int o = (j * ratio + m) * scols + k * ratio + q;
            wd = __double2float_rn(__dadd_rn((double)wd, fabs((double)__fsub_rn(__ldg(white + o), __ldg(dark + o)))));
        }
    const size_t plane = (size_t)srows * scols, oplane = (size_t)prows * pcols;
    const size_t out0 = (size_t)j * pcols + k;
    if (ratio == 2 && (scols & 1) == 0) {
        // 2 x 2 blocks: one 32-bit load per raw row (k ratio is even and so is
        // scols, so each pair is 4-byte aligned); the dark values held
        const int o0 = (2 * j) * scols + 2 * k, o1 = o0 + scols;
        const float d00 = __ldg(dark + o0), d01 = __ldg(dark + o0 + 1), d10 = __ldg(dark + o1),
                    d11 = __ldg(dark + o1 + 1);
        for (int i = v0; i < v1; i++) {
            const uint16_t *c = counts + (size_t)i * plane;
            const ushort2 r0 = __ldcs(reinterpret_cast<const ushort2 *>(c + o0));
            const ushort2 r1 = __ldcs(reinterpret_cast<const ushort2 *>(c + o1));
            float w = 0.0f;
            w = __double2float_rn(__dadd_rn((double)w, fabs((double)__fsub_rn((float)r0.x, d00))));
            w = __double2float_rn(__dadd_rn((double)w, fabs((double)__fsub_rn((float)r0.y, d01))));
            w = __double2float_rn(__dadd_rn((double)w, fabs((double)__fsub_rn((float)r1.x, d10))));
            w = __double2float_rn(__dadd_rn((double)w, fabs((double)__fsub_rn((float)r1.y, d11))));
            const float t = __double2float_rn(log((double)__fdiv_rn(wd, w)));
            const double td = (double)t;
            __stcs(proj + (size_t)i * oplane + out0, __double2float_rn(__dadd_rn(__dmul_rn(__dmul_rn(bh, td), td), td)));
            __stcs(wts + (size_t)i * oplane + out0, w);
        }
        return;
    }
    for (int i = v0; i < v1; i++) {
        const uint16_t *c = counts + (size_t)i * plane;
        float w = 0.0f;
        for (int m = 0; m < ratio; m++)
            for (int q = 0; q < ratio; q++) {
                const int o = (j * ratio + m) * scols + k * ratio + q;
                w = __double2float_rn(__dadd_rn((double)w, fabs((double)__fsub_rn((float)__ldcs(c + o), __ldg(dark + o)))));
            }
        const float t = __double2float_rn(log((double)__fdiv_rn(wd, w)));
        const double td = (double)t;
        __stcs(proj + (size_t)i * oplane + out0, __double2float_rn(__dadd_rn(__dmul_rn(__dmul_rn(bh, td), td), td)));
        __stcs(wts + (size_t)i * oplane + out0, w);
    }
}

// Down-sampling of float projections and weights (std_data/XT_HDFIO.c:
// 128-146): sums in block order, the projection's mean (float division by
// ratio^2) through bh t^2 + t.
__global__ void k_downsample_pw(const float *__restrict__ pin, const float *__restrict__ win, int views, int srows,
                                int scols, int ratio, int prows, int pcols, double bh, float *__restrict__ proj,
                                float *__restrict__ wts)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    const size_t i = blockIdx.z;
    if (k >= pcols) return;
    const size_t idx = (i * prows + j) * pcols + k;
    const size_t base = i * (size_t)srows * scols;
    float t = 0.0f, w = 0.0f;
    for (int m = 0; m < ratio; m++)
        for (int q = 0; q < ratio; q++) {
            const size_t o = base + (size_t)(j * ratio + m) * scols + (size_t)k * ratio + q;
            t = __fadd_rn(t, pin[o]);
            w = __fadd_rn(w, win[o]);
        }
    t = __fdiv_rn(t, (float)(ratio * ratio));
    const double td = (double)t;
    proj[idx] = __double2float_rn(__dadd_rn(__dmul_rn(__dmul_rn(bh, td), td), td));
    wts[idx] = w;
}

inline unsigned nblk(size_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

// The hyperslab both readers select (XT_HDFIO.c:94-125): columns trimmed
// symmetrically to a multiple of proj_cols, ratio = kept columns / proj_cols
// (the same along rows), this rank's rows.
struct Window {
    int ratio, col0, ncols, row0, nrows, prows;
};

int window(int rows, int cols, int datafile_row0, int proj_rows, int proj_cols, int rank, int ranks, Window &w)
{
    if (ranks < 1 || rank < 0 || rank >= ranks) return ing_fail("rank outside 0 .. ranks - 1");
    if (proj_cols < 1 || cols < proj_cols) return ing_fail("the file has fewer detector columns than proj_cols");
    if (proj_rows < ranks || proj_rows % ranks) return ing_fail("proj_rows must be a multiple of the ranks");
    const int extras = cols % proj_cols;
    w.ncols = cols - extras;
    w.ratio = w.ncols / proj_cols;
    w.col0 = extras / 2;
    w.prows = proj_rows / ranks;
    w.nrows = w.prows * w.ratio;
    w.row0 = datafile_row0 + rank * w.nrows;
    if (datafile_row0 < 0 || (long long)w.row0 + w.nrows > rows)
        return ing_fail("the file has fewer detector rows than datafile_row0 + proj_rows x ratio");
    return 0;
}

// Copy frames [f0, f0 + nf) of a [frames][rows][cols] stack, rows
// [row0, row0 + nrows) and columns [col0, col0 + ncols), to a dense device
// array [nf][nrows][ncols] (one 2-D copy per frame window: the rows of a
// frame's window are one pitched block).
template <typename T>
cudaError_t copy_window(T *dst, const T *src, int f0, int nf, int rows, int cols, const Window &w, cudaMemcpyKind kind,
                        cudaStream_t s)
{
    for (int f = 0; f < nf; f++) {
        const T *sp = src + ((size_t)(f0 + f) * rows + w.row0) * cols + w.col0;
        cudaError_t e = cudaMemcpy2DAsync(dst + (size_t)f * w.nrows * w.ncols, (size_t)w.ncols * sizeof(T), sp,
                                          (size_t)cols * sizeof(T), (size_t)w.ncols * sizeof(T), w.nrows, kind, s);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

struct DevBuf {
    void *p = nullptr;
    ~DevBuf()
    {
        if (p) cudaFree(p);
    }
};

}  // namespace

extern "C" {

const char *mbir_ingest_last_error(void) { return g_ing_err; }

int mbir_normalize_counts_device(const uint16_t *counts, const float *white_mean, const float *dark_mean,
                                 int32_t views, int32_t win_rows, int32_t win_cols, int32_t ratio, double bh_quad_coef,
                                 float *projections, float *weights, void *stream)
{
    if (ratio < 1 || win_rows % ratio || win_cols % ratio) return ing_fail("window not a multiple of the ratio");
    const int pr = win_rows / ratio, pc = win_cols / ratio;
    if ((size_t)views * pr * pc == 0) return 0;
    if (pr > 65535) return ing_fail("more than 65535 output rows");
    const dim3 grid((pc + 127) / 128, pr, (views + kNormViews - 1) / kNormViews);
    k_normalize<<<grid, 128, 0, (cudaStream_t)stream>>>(counts, white_mean, dark_mean, views, win_rows, win_cols,
                                                         ratio, pr, pc, bh_quad_coef, projections, weights);
    IK(cudaGetLastError());
    return 0;
}

int mbir_frame_mean_device(const uint16_t *frames, int32_t n_frames, int32_t rows, int32_t cols, float *out,
                           void *stream)
{
    if (n_frames < 1) return ing_fail("no frames to average");
    const size_t n = (size_t)rows * cols;
    k_frame_mean<<<nblk(n), 256, 0, (cudaStream_t)stream>>>(frames, n_frames, rows, cols, out);
    IK(cudaGetLastError());
    return 0;
}

int mbir_normalize_counts(const uint16_t *counts, int32_t n_counts, const uint16_t *whites, int32_t n_whites,
                          const uint16_t *darks, int32_t n_darks, int32_t rows, int32_t cols, int32_t datafile_row0,
                          int32_t proj_rows, int32_t proj_cols, int32_t proj_start, int32_t proj_num, int32_t rank,
                          int32_t ranks, double bh_quad_coef, float *projections, float *weights)
{
    Window w;
    if (window(rows, cols, datafile_row0, proj_rows, proj_cols, rank, ranks, w)) return -1;
    if (n_whites < 3 || n_darks < 3) return ing_fail("the bright and dark stacks need at least 3 frames (first and last are dropped)");
    if (proj_start < 0 || proj_num < 0 || (long long)proj_start + proj_num > n_counts)
        return ing_fail("proj_start + proj_num beyond the counts stack");
    cudaStream_t s = nullptr;
    IK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } sg{s};
    const size_t win = (size_t)w.nrows * w.ncols, nout = (size_t)proj_num * w.prows * proj_cols;
    DevBuf dc, dw, dd, mw, md, dp, dwt;
    IK(cudaMalloc(&dc.p, std::max<size_t>(1, (size_t)proj_num * win) * sizeof(uint16_t)));
    IK(cudaMalloc(&dw.p, (size_t)(n_whites - 2) * win * sizeof(uint16_t)));
    IK(cudaMalloc(&dd.p, (size_t)(n_darks - 2) * win * sizeof(uint16_t)));
    IK(cudaMalloc(&mw.p, win * sizeof(float)));
    IK(cudaMalloc(&md.p, win * sizeof(float)));
    IK(cudaMalloc(&dp.p, std::max<size_t>(1, nout) * sizeof(float)));
    IK(cudaMalloc(&dwt.p, std::max<size_t>(1, nout) * sizeof(float)));
    // the readers drop the first and last bright and dark frames (offset 1, count n - 2)
    IK(copy_window((uint16_t *)dw.p, whites, 1, n_whites - 2, rows, cols, w, cudaMemcpyHostToDevice, s));
    IK(copy_window((uint16_t *)dd.p, darks, 1, n_darks - 2, rows, cols, w, cudaMemcpyHostToDevice, s));
    IK(copy_window((uint16_t *)dc.p, counts, proj_start, proj_num, rows, cols, w, cudaMemcpyHostToDevice, s));
    if (mbir_frame_mean_device((const uint16_t *)dw.p, n_whites - 2, w.nrows, w.ncols, (float *)mw.p, s) ||
        mbir_frame_mean_device((const uint16_t *)dd.p, n_darks - 2, w.nrows, w.ncols, (float *)md.p, s) ||
        mbir_normalize_counts_device((const uint16_t *)dc.p, (const float *)mw.p, (const float *)md.p, proj_num,
                                     w.nrows, w.ncols, w.ratio, bh_quad_coef, (float *)dp.p, (float *)dwt.p, s))
        return -1;
    IK(cudaMemcpyAsync(projections, dp.p, nout * sizeof(float), cudaMemcpyDeviceToHost, s));
    IK(cudaMemcpyAsync(weights, dwt.p, nout * sizeof(float), cudaMemcpyDeviceToHost, s));
    IK(cudaStreamSynchronize(s));
    return 0;
}

int mbir_downsample_projections(const float *projs, const float *wts, int32_t n_views, int32_t rows, int32_t cols,
                                int32_t datafile_row0, int32_t proj_rows, int32_t proj_cols, int32_t proj_start,
                                int32_t proj_num, int32_t rank, int32_t ranks, double bh_quad_coef,
                                float *projections, float *weights)
{
    Window w;
    if (window(rows, cols, datafile_row0, proj_rows, proj_cols, rank, ranks, w)) return -1;
    if (proj_start < 0 || proj_num < 0 || (long long)proj_start + proj_num > n_views)
        return ing_fail("proj_start + proj_num beyond the dataset");
    cudaStream_t s = nullptr;
    IK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } sg{s};
    const size_t win = (size_t)w.nrows * w.ncols, nout = (size_t)proj_num * w.prows * proj_cols;
    DevBuf dpi, dwi, dp, dwt;
    IK(cudaMalloc(&dpi.p, std::max<size_t>(1, (size_t)proj_num * win) * sizeof(float)));
    IK(cudaMalloc(&dwi.p, std::max<size_t>(1, (size_t)proj_num * win) * sizeof(float)));
    IK(cudaMalloc(&dp.p, std::max<size_t>(1, nout) * sizeof(float)));
    IK(cudaMalloc(&dwt.p, std::max<size_t>(1, nout) * sizeof(float)));
    IK(copy_window((float *)dpi.p, projs, proj_start, proj_num, rows, cols, w, cudaMemcpyHostToDevice, s));
    IK(copy_window((float *)dwi.p, wts, proj_start, proj_num, rows, cols, w, cudaMemcpyHostToDevice, s));
    if (nout) {
        if (w.prows > 65535 || proj_num > 65535) return ing_fail("more than 65535 output rows or views");
        const dim3 grid((proj_cols + 127) / 128, w.prows, proj_num);
        k_downsample_pw<<<grid, 128, 0, s>>>((const float *)dpi.p, (const float *)dwi.p, proj_num, w.nrows,
                                                    w.ncols, w.ratio, w.prows, proj_cols, bh_quad_coef,
                                                    (float *)dp.p, (float *)dwt.p);
        IK(cudaGetLastError());
    }
    IK(cudaMemcpyAsync(projections, dp.p, nout * sizeof(float), cudaMemcpyDeviceToHost, s));
    IK(cudaMemcpyAsync(weights, dwt.p, nout * sizeof(float), cudaMemcpyDeviceToHost, s));
    IK(cudaStreamSynchronize(s));
    return 0;
}

// gen_interlaced_views_0_to_Inf (aps_data/XT_Views.c:41-80): view i of the
// interlaced scan has index i K + bitrev(floor(i / L) mod K) on a grid of
// N_theta views per half turn (L = N_theta / K, bit reversal over
// round(log2 K) bits), angle index x pi / N_theta, time index / K; a view
// closer than rot_speed x min_acq_time to the last kept one is skipped.
// Views proj_start .. proj_start + N_p - 1 of the kept ones are returned;
// the result is the count of kept views generated (proj_start + N_p).
int32_t mbir_gen_interlaced_views(float *views, float *times, int32_t K, int32_t N_theta, int32_t proj_start,
                                  int32_t N_p, float min_acq_time, float rot_speed)
{
    if (K < 1 || N_theta < K || proj_start < 0 || N_p < 0) return -1;
    const int32_t L = N_theta / K;
    const int32_t bits = (int32_t)floor(log((double)K) / log(2.0) + 0.5);
    const float dtheta = (float)(M_PI / N_theta);
    const float min_d = rot_speed * min_acq_time;
    std::vector<float> ang((size_t)proj_start + N_p + 1), tim((size_t)proj_start + N_p + 1);
    int32_t kept = 0;
    for (int32_t i = 0; kept < proj_start + N_p; i++) {
        const int32_t q = i / L % K;
        int32_t r = 0;
        for (int32_t b = 0; b < bits; b++)
            if (q & (1 << b)) r |= 1 << (bits - 1 - b);
        const float a = (float)(i * K + r);
        tim[kept] = a / (float)K;
        ang[kept] = a * dtheta;
        if (i == 0 || ang[kept] - ang[kept - 1] > min_d) kept++;
    }
    for (int32_t i = 0; i < N_p; i++) {
        views[i] = ang[(size_t)proj_start + i];
        times[i] = tim[(size_t)proj_start + i];
    }
    return kept;
}

}  // extern "C"
