// One resolution stage of the reconstruction on the GPU: device state, the
// reference ICD schedule, cost, ring offsets and variance, behind the C ABI
// declared in include/timbir_b200.h.
//
// Reference: TIMBIR v0.0.2, src/MBIR_4D/XT_ICD_update.c (ICD_BackProject,
// updateVoxelsTimeSlices) and XT_Init.c (stage set-up).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/timbir_b200.h"
#include "mbir_host.h"
#include "mbir_internal.h"
#include "mbir_fbp.h"
#include "mbir_sv.h"

using namespace mbir;

static thread_local char g_err[512];

static int fail(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return -1;
}

#define CK(call)                                                                                 \
    do {                                                                                         \
        cudaError_t _e = (call);                                                                 \
        if (_e != cudaSuccess)                                                                   \
            return fail("%s:%d: %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(_e));    \
    } while (0)

// Device buffers come from the device's default memory pool, which keeps
// freed memory cached (release threshold raised once per device), so stages
// set up one after another reuse it instead of paying for fresh allocations.
// Allocation is stream-ordered on the legacy stream and completed before use.
// Device memory the stages hold, and an optional cap on it
// (mbir_set_device_bytes_cap: the allocator refuses what would exceed it,
// as an exhausted device would; for testing the error paths).
static std::mutex g_alloc_mu;
static std::map<void *, size_t> g_alloc_live;
static size_t g_alloc_bytes = 0, g_alloc_cap = 0;

template <typename T>
static cudaError_t dalloc(T **p, size_t n)
{
    const size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
    {
        std::lock_guard<std::mutex> lock(g_alloc_mu);
        if (g_alloc_cap && g_alloc_bytes + bytes > g_alloc_cap) {
            *p = nullptr;
            return cudaErrorMemoryAllocation;
        }
    }
    static bool pool_ready[64] = {false};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < 64 && !pool_ready[dev]) {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        pool_ready[dev] = true;
    }
    e = cudaMallocAsync((void **)p, bytes, 0);
    if (e != cudaSuccess) return e;
    {
        std::lock_guard<std::mutex> lock(g_alloc_mu);
        g_alloc_live[(void *)*p] = bytes;
        g_alloc_bytes += bytes;
    }
    return cudaStreamSynchronize(0);
}

struct MbirStage;
static int slab_sum(MbirStage *S, double *v, int n);

static void dfree(void *p)
{
    if (!p) return;
    {
        std::lock_guard<std::mutex> lock(g_alloc_mu);
        auto it = g_alloc_live.find(p);
        if (it != g_alloc_live.end()) {
            g_alloc_bytes -= it->second;
            g_alloc_live.erase(it);
        }
    }
    cudaFreeAsync(p, 0);
}

extern "C" int mbir_set_device_bytes_cap(int64_t bytes)
{
    std::lock_guard<std::mutex> lock(g_alloc_mu);
    g_alloc_cap = bytes > 0 ? (size_t)bytes : 0;
    return 0;
}

extern "C" int64_t mbir_get_device_bytes(void)
{
    std::lock_guard<std::mutex> lock(g_alloc_mu);
    return (int64_t)g_alloc_bytes;
}

struct MbirStage {
    ScanGeom sg;
    StageGeom st;
    ParkMiller rng;
    int nblk = 2, K = 10, offset_type = 0, upd_offset = 0, upd_var = 0, prepared = 0;
    double var_est = 1.0, stop_thresh = 1.0, hT = 0, hdelta = 0, last_pct = 0;
    long long updates = 0, zero_skips = 0;
    bool hr_ready = false;  // d_H holds the detector response
    std::vector<uint8_t> mask;
    std::vector<int> nr, nn;  // line counts [N_time][nblk]
    MbirGeom g{};
    MbirPrior pr{};
    MbirDev dv{};
    cudaStream_t stream = nullptr;
    // device buffers
    float *d_e = nullptr, *d_w = nullptr, *d_y = nullptr, *d_d = nullptr, *d_x = nullptr,
          *d_mag = nullptr, *d_filt = nullptr, *d_H = nullptr;
    double *d_cos = nullptr, *d_sin = nullptr, *d_num = nullptr, *d_den = nullptr,
           *d_partials = nullptr, *d_result = nullptr, *d_ochunk = nullptr;
    int *d_vidx = nullptr, *d_vnum = nullptr, *d_fov = nullptr, *d_xr = nullptr, *d_yr = nullptr,
        *d_xn = nullptr, *d_yn = nullptr;
    uint8_t *d_mask = nullptr;
    MbirTask *d_tasks = nullptr;
    MbirTaskOut *d_tout = nullptr;
    char *d_acache = nullptr;
    size_t acache_bytes = 0;
    int nparts = 592;
    int threads = 256;
    // CUDA events around the ICD kernel launches, on the stage's stream
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, tev0 = nullptr, tev1 = nullptr;
    double icd_ms = 0;
    long long launches = 0, icd_launches = 0;
    // super-voxel schedule
    int schedule = 0;  // 0: reference schedule, 1: super-voxel schedule
    SvParams sp{};
    int nzg = 1, gz = 1;
    int sv_nphase = 1;
    std::vector<SvTask> sv_all;            // every super-voxel; its id is its index
    std::vector<int> sv_all_phase;         // its colour phase
    std::vector<std::vector<int>> sv_nbr;  // ids of the super-voxels it conflicts with
    SvTask *d_sv_all = nullptr;
    int *d_sv_done = nullptr;  // per id: epoch of its last finished visit
    int sv_epoch = 0;
    // launch lists [order | dep_off | deps] of the full sweep for each phase
    // rotation (the non-homogeneous pass visits a subset of one of them)
    std::vector<std::array<size_t, 4>> sv_rot;  // {n, order, dep_off, deps offsets}
    int *d_sv_lists = nullptr;
    cudaEvent_t sv_ev[4] = {nullptr, nullptr, nullptr, nullptr};
    SvTaskOut *d_sv_out = nullptr;
    float *d_scratch = nullptr;
    // A-matrix column cache of the super-voxel kernel ([N_y N_x][N_p][eq] int4),
    // filled at the first iteration after the prologue
    int4 *d_acol = nullptr;
    size_t acol_bytes = 0;
    int acol_mode = -1;  // -1: when it fits in a third of free memory, 0: never, 1: always, 2: FP16 values
    bool acol_half = false;  // the cache holds FP16 values
    bool acol_built = false;
    int *d_err = nullptr, *d_queue = nullptr;
    int sm_count = 148;
    int sv_ctas = 0;    // persistent CTAs per launch requested; 0 = automatic
    int sv_zgroup = 0;  // slices per z-group requested; 0 = automatic
    int sv_grid = 1;    // persistent CTAs per launch (automatic)
    int sv_cap = 0;     // concurrent super-voxels allowed per (frame, z-group)
    int sv_fit = 1;     // CTAs resident on the GPU (all SMs)
    double sv_alpha = 0;      // over-relaxation of schedule 1 requested; 0 = automatic
    double sv_alpha_eff = 1.5;  // over-relaxation schedule 1 uses
    // stability guard of schedule 1: the state at the start of the current
    // window of iterations and the MAP cost there (have_cost: known), the
    // window's iterations so far and the windows checked
    float *d_snap_x = nullptr, *d_snap_e = nullptr, *d_snap_w = nullptr, *d_snap_d = nullptr;
    double snap_var = 1.0, prev_cost = 0;
    bool guard = true, have_cost = false, win_open = false;
    int win_iters = 0, guard_checks = 0, stab_events = 0;
    std::vector<int> sv_rank;  // size rank of a super-voxel within its (phase, frame, z-group)
    // NHICD pass of schedule 1: per (frame, z-group) plane, the lines whose
    // filtered update magnitude is above the plane's order statistic (a
    // fraction nh_fraction of its in-mask lines), chosen on the device; off
    // unless set (on the 3-D workload every fraction tried made the time to
    // the MAP cost longer: each selected super-voxel stages and commits its
    // whole band for a few lines)
    double nh_fraction = 0.0;
    uint8_t *d_nh_sel = nullptr;  // [planes][N_y][N_x] selected lines
    int *d_nh_nsel = nullptr, *d_nh_count = nullptr, *d_nh_pos = nullptr, *d_nh_nt = nullptr;
    float *d_nh_thresh = nullptr;
    std::vector<int> nh_nsel;  // host copy of d_nh_nsel
    // rectangular-patch constraint windows of offset mode 3 (win.M = 0: none)
    OffsetWindows win{};
    std::vector<void *> win_bufs;
    // z-slab `slab_rank` of `slab_count` (one slab per rank; 1: the whole
    // volume): the halo slices [2][N_time][N_y][N_x] and the sum over ranks
    // that takes the place of the reference's MPI reductions
    float *d_halo = nullptr;
    int slab_rank = 0, slab_count = 1;
    // fault injection (mbir_debug_sv_skip_tasks): the next sweep's work queue
    // starts this many entries in, so those super-voxels never run and the
    // ones that depend on them wait until the wait gives up
    int debug_skip = 0;
    MbirAllreduceFn allreduce = nullptr;
    void *allreduce_ctx = nullptr;

    size_t nsino() const { return (size_t)sg.N_t * sg.N_p * sg.N_r; }
    size_t nvox() const { return (size_t)sg.N_time * st.N_z * st.N_y * st.N_x; }
    size_t nxy() const { return (size_t)st.N_y * st.N_x; }
    // most detector columns of one A-matrix entry: 2 ceil(delta_xy / delta_r) + 1
    int amax() const { return 2 * (int)std::ceil(st.delta_xy / sg.delta_r) + 1; }
    size_t nmag() const { return (size_t)sg.N_time * nblk * nxy(); }
    int max_views() const
    {
        int m = 1;
        for (auto &v : sg.views) m = std::max<int>(m, (int)v.size());
        return m;
    }
    ~MbirStage()
    {
        void *bufs[] = {d_e,   d_w,   d_y,    d_d,   d_x,   d_mag, d_filt,     d_H,      d_cos,
                        d_sin, d_num, d_den,  d_partials, d_result, d_ochunk, d_vidx, d_vnum, d_fov,
                        d_xr,  d_yr,  d_xn,   d_yn,  d_mask, d_tasks, d_tout, d_acache,
                        d_sv_all, d_sv_done, d_sv_lists, d_sv_out, d_scratch, d_err, d_queue, d_acol,
                        d_snap_x, d_snap_e, d_snap_w, d_snap_d, d_nh_sel, d_nh_nsel, d_nh_count, d_nh_pos,
                        d_nh_nt, d_nh_thresh, d_halo};
        if (stream) cudaStreamSynchronize(stream);
        for (void *b : bufs) dfree(b);
        for (void *b : win_bufs) dfree(b);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (tev0) cudaEventDestroy(tev0);
        if (tev1) cudaEventDestroy(tev1);
        for (auto e : sv_ev)
            if (e) cudaEventDestroy(e);
        if (stream) cudaStreamDestroy(stream);
    }
};

// ---------------------------------------------------------------------------
// Set-up (initStatStructures + initDynStructures, XT_Init.c:211-669)
// ---------------------------------------------------------------------------
extern "C" int mbir_init_stage(MbirStage **out, const float *projections, const float *weights,
                               const float *proj_angles, const float *proj_times,
                               const float *recon_times, int32_t proj_rows, int32_t proj_cols,
                               int32_t proj_num, int32_t recon_num, float vox_wid, float rot_center,
                               float sig_s, float sig_t, float c_s, float c_t, float convg_thresh,
                               int32_t remove_rings, int32_t quad_convex, float huber_delta,
                               float huber_T, int32_t mult_xy, int32_t mult_z, int32_t num_z_blocks)
{
    *out = nullptr;
    if (proj_rows <= 0 || proj_cols <= 0 || proj_num <= 0 || recon_num <= 0)
        return fail("non-positive dimensions");
    if (mult_xy <= 0 || mult_z <= 0 || proj_cols % mult_xy != 0 || proj_rows % mult_z != 0)
        return fail("voxel scales (%d, %d) do not divide the detector (%d, %d)", mult_xy, mult_z,
                    proj_cols, proj_rows);
    if (remove_rings < 0 || remove_rings > 3) return fail("remove_rings must be 0..3");
    if (quad_convex < 0 || quad_convex > 1) return fail("quad_convex must be 0 or 1");
    // a NaN or infinite projection or weight would turn every cost and
    // update it touches into NaN (the reference does not check); refused here
    {
        const size_t n = (size_t)proj_num * proj_rows * proj_cols;
        for (size_t q = 0; q < n; q++)
            if (!std::isfinite(projections[q]) || !std::isfinite(weights[q]) || weights[q] < 0.0f)
                return fail("projection / weight %zu is not finite (or the weight is negative)", q);
    }
    MbirStage *S = new MbirStage();
    char err[256];
    if (scan_geom(S->sg, proj_angles, proj_times, recon_times, proj_rows, proj_cols, proj_num,
                  recon_num, vox_wid, rot_center, err, sizeof(err))) {
        delete S;
        return fail("%s", err);
    }
    stage_geom(S->sg, S->st, mult_xy, mult_z, sig_s, sig_t);
    if (num_z_blocks < 2 || num_z_blocks % 2 || num_z_blocks > std::max(2, S->st.N_z)) {
        const int nz = S->st.N_z;
        delete S;
        return fail("num_z_blocks %d must be even, >= 2 and <= N_z = %d", num_z_blocks, nz);
    }
    S->nblk = num_z_blocks;
    S->offset_type = remove_rings;
    S->stop_thresh = convg_thresh;
    S->hT = quad_convex == 0 ? (double)huber_T : 100000.0;
    S->hdelta = quad_convex == 0 ? (double)huber_delta : 1.0;
    S->nr.assign((size_t)recon_num * S->nblk, 0);
    S->nn.assign((size_t)recon_num * S->nblk, 0);

    const ScanGeom &sg = S->sg;
    const StageGeom &st = S->st;
    int rc = 0;
#define CKS(call)                                                                               \
    do {                                                                                        \
        cudaError_t _e = (call);                                                                \
        if (_e != cudaSuccess) {                                                                \
            rc = fail("%s: %s", #call, cudaGetErrorString(_e));                                 \
            delete S;                                                                           \
            return rc;                                                                          \
        }                                                                                       \
    } while (0)
    CKS(cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking));
    CKS(cudaEventCreate(&S->ev0));
    CKS(cudaEventCreate(&S->ev1));
    CKS(cudaEventCreate(&S->tev0));
    CKS(cudaEventCreate(&S->tev1));
    const size_t ns = S->nsino();
    CKS(dalloc(&S->d_e, ns));
    CKS(dalloc(&S->d_w, ns));
    CKS(dalloc(&S->d_y, ns));
    CKS(dalloc(&S->d_d, (size_t)sg.N_t * sg.N_r));
    CKS(dalloc(&S->d_x, S->nvox()));
    CKS(dalloc(&S->d_mag, S->nmag()));
    CKS(dalloc(&S->d_filt, S->nmag()));
    CKS(dalloc(&S->d_H, (size_t)sg.N_p * (MBIR_RESP_BINS + 1)));
    CKS(dalloc(&S->d_cos, sg.N_p));
    CKS(dalloc(&S->d_sin, sg.N_p));
    CKS(dalloc(&S->d_num, (size_t)sg.N_t * sg.N_r));
    CKS(dalloc(&S->d_den, (size_t)sg.N_t * sg.N_r));
    CKS(dalloc(&S->d_partials, (size_t)4 * S->nparts));
    {
        MbirGeom gg{};
        gg.N_p = sg.N_p;
        CKS(dalloc(&S->d_ochunk, (size_t)2 * mbir_offset_chunks(gg) * sg.N_t * sg.N_r));
    }
    CKS(dalloc(&S->d_result, 8));
    const int mv = S->max_views();
    CKS(dalloc(&S->d_vidx, (size_t)recon_num * mv));
    CKS(dalloc(&S->d_vnum, recon_num));
    CKS(dalloc(&S->d_fov, sg.N_p));
    CKS(dalloc(&S->d_xr, S->nmag()));
    CKS(dalloc(&S->d_yr, S->nmag()));
    CKS(dalloc(&S->d_xn, S->nmag()));
    CKS(dalloc(&S->d_yn, S->nmag()));
    CKS(dalloc(&S->d_mask, S->nxy()));
    CKS(dalloc(&S->d_tasks, (size_t)recon_num * S->nblk));
    CKS(dalloc(&S->d_tout, (size_t)recon_num * S->nblk));
    // per-task A-column cache: views x entries x (double value + int bin) + counts
    const int amax = mbir_amax(st.delta_xy, sg.delta_r);
    S->acache_bytes = (size_t)mv * amax * (sizeof(double) + sizeof(int)) + (size_t)mv * sizeof(int);
    S->acache_bytes = (S->acache_bytes + 255) & ~(size_t)255;
    if (S->acache_bytes > 160 * 1024)
        CKS(dalloc(&S->d_acache, S->acache_bytes * (size_t)recon_num * (S->nblk / 2)));
    S->threads = mv <= 64 ? 64 : (mv <= 128 ? 128 : 256);

    // upload inputs in the reference layout [view][row][col] and reorder on
    // the device into [row][view][col] (the variance estimate is 1 here, so
    // the weights are taken as they are, XT_Init.c:327-330)
    {
        float *raw = nullptr;
        CKS(dalloc(&raw, ns));
        cudaError_t e1 = cudaMemcpy(raw, projections, ns * sizeof(float), cudaMemcpyHostToDevice);
        if (e1 == cudaSuccess) e1 = mbir_launch_to_slice_major(raw, S->d_y, sg.N_p, sg.N_t, sg.N_r, 0);
        if (e1 == cudaSuccess) e1 = cudaMemcpy(raw, weights, ns * sizeof(float), cudaMemcpyHostToDevice);
        if (e1 == cudaSuccess) e1 = mbir_launch_to_slice_major(raw, S->d_w, sg.N_p, sg.N_t, sg.N_r, 0);
        if (e1 == cudaSuccess) e1 = cudaStreamSynchronize(0);
        dfree(raw);
        S->launches += 2;
        CKS(e1);
    }
    CKS(cudaMemset(S->d_d, 0, (size_t)sg.N_t * sg.N_r * sizeof(float)));
    CKS(cudaMemset(S->d_x, 0, S->nvox() * sizeof(float)));
    CKS(cudaMemset(S->d_mag, 0, S->nmag() * sizeof(float)));
    CKS(cudaMemcpy(S->d_cos, sg.cosv.data(), sg.N_p * sizeof(double), cudaMemcpyHostToDevice));
    CKS(cudaMemcpy(S->d_sin, sg.sinv.data(), sg.N_p * sizeof(double), cudaMemcpyHostToDevice));
    {
        std::vector<int> vidx((size_t)recon_num * mv, 0), vnum(recon_num);
        for (int i = 0; i < recon_num; i++) {
            vnum[i] = (int)sg.views[i].size();
            std::copy(sg.views[i].begin(), sg.views[i].end(), vidx.begin() + (size_t)i * mv);
        }
        CKS(cudaMemcpy(S->d_vidx, vidx.data(), vidx.size() * sizeof(int), cudaMemcpyHostToDevice));
        CKS(cudaMemcpy(S->d_vnum, vnum.data(), vnum.size() * sizeof(int), cudaMemcpyHostToDevice));
        CKS(cudaMemcpy(S->d_fov, sg.frame_of_view.data(), sg.N_p * sizeof(int), cudaMemcpyHostToDevice));
    }
    // error flags of the stage's kernels (super-voxel waits, column widths,
    // the windowed offset solve)
    CKS(dalloc(&S->d_err, 1));
    CKS(cudaMemsetAsync(S->d_err, 0, sizeof(int), S->stream));
#undef CKS
    // device-side views of the geometry and prior
    MbirGeom &g = S->g;
    g.N_p = sg.N_p; g.N_r = sg.N_r; g.N_t = sg.N_t; g.m_z = st.m_z;
    g.delta_r = sg.delta_r; g.R0 = sg.R0; g.RMax = sg.RMax; g.OffsetR = st.OffsetR;
    g.N_x = st.N_x; g.N_y = st.N_y; g.N_z = st.N_z; g.N_time = sg.N_time;
    g.x0 = st.x0; g.y0 = sg.y0; g.delta_xy = st.delta_xy;
    g.max_views = mv; g.view_idx = S->d_vidx; g.view_num = S->d_vnum;
    g.cosv = S->d_cos; g.sinv = S->d_sin; g.H_r = S->d_H;
    MbirPrior &pr = S->pr;
    pr.sSQ = st.sSQ; pr.sSQP = st.sSQP; pr.sTQ = st.sTQ; pr.sTQP = st.sTQP;
    pr.c_s = c_s; pr.c_t = c_t;
    std::copy(st.SF, st.SF + 27, pr.SF);
    pr.TF = st.TF; pr.alpha = 1.5; pr.hT = S->hT; pr.hdelta = S->hdelta;
    S->dv.e = S->d_e; S->dv.w = S->d_w; S->dv.d = S->d_d; S->dv.x = S->d_x; S->dv.mag = S->d_mag;
    S->dv.mask = S->d_mask;
    *out = S;
    return 0;
}

extern "C" void mbir_free_stage(MbirStage *S) { delete S; }

extern "C" const char *mbir_last_error(void) { return g_err; }

// Per-stage switches (XT_Init.c:236-266) and the variance estimate carried
// from the previous stage; weights are rescaled as at XT_Init.c:327-330.
extern "C" int mbir_set_stage_switches(MbirStage *S, int32_t update_proj_offset, int32_t update_var,
                                       double var_est)
{
    S->upd_offset = update_proj_offset;
    S->upd_var = update_var;
    if (var_est > 0 && var_est != S->var_est) {
        std::vector<float> w(S->nsino());
        CK(cudaMemcpy(w.data(), S->d_w, w.size() * sizeof(float), cudaMemcpyDeviceToHost));
        for (auto &v : w) v = (float)(v * S->var_est);
        for (auto &v : w) v /= var_est;
        S->var_est = var_est;
        CK(cudaMemcpy(S->d_w, w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice));
    }
    return 0;
}

extern "C" int mbir_set_convergence_threshold(MbirStage *S, double convg_thresh)
{
    S->stop_thresh = convg_thresh;
    return 0;
}

extern "C" int mbir_set_rng_state(MbirStage *S, uint32_t state)
{
    S->rng.state = state;
    return 0;
}

extern "C" uint32_t mbir_get_rng_state(MbirStage *S) { return S->rng.state; }

// Detector response H_r into d_H: trapezoids and beam from the host C library,
// the sampling and beam convolution on the GPU (XT_Profile.c:129-170).
static int compute_detector_response(MbirStage *S)
{
    std::vector<double> trap, beam;
    double r0, step, tc;
    detector_response_params(S->sg, S->st, trap, beam, r0, step, tc);
    double *d_trap = nullptr, *d_beam = nullptr;
    CK(dalloc(&d_trap, trap.size()));
    CK(dalloc(&d_beam, beam.size()));
    cudaError_t e = cudaMemcpy(d_trap, trap.data(), trap.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_beam, beam.data(), beam.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = mbir_launch_detector_response(d_trap, d_beam, S->sg.N_p, S->st.OffsetR, S->st.delta_xy, r0, step, tc,
                                          S->d_H, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    dfree(d_trap);
    dfree(d_beam);
    CK(e);
    S->launches++;
    S->hr_ready = true;
    return 0;
}

// Stage prologue of ICD_BackProject (XT_ICD_update.c:1134-1159): mask,
// detector response, initial object (zero unless given, [N_time][N_z][N_y][N_x]),
// ring offsets (zero unless given, [N_r][N_t] as the reference stores them),
// update-magnitude map (zero unless given) and the error sinogram.
// The stage prologue (ICD_BackProject, XT_ICD_update.c:1134-1159): detector
// response, mask, start object, offsets and magnitude map, error sinogram.
// fill_object / fill_mag enqueue the start object and magnitude map on the
// stage's stream.
template <class FO, class FM>
static int icd_prepare_with(MbirStage *S, const float *offset, FO &&fill_object, FM &&fill_mag)
{
    const ScanGeom &sg = S->sg;
    if (compute_detector_response(S)) return -1;
    object_mask(sg, S->st, S->mask);
    // uploads on the stage's stream, ahead of its kernels (pageable sources
    // are staged before each call returns)
    CK(cudaMemcpyAsync(S->d_mask, S->mask.data(), S->mask.size(), cudaMemcpyHostToDevice, S->stream));
    if (fill_object()) return -1;
    if (offset) {
        std::vector<float> d((size_t)sg.N_t * sg.N_r);
        for (int r = 0; r < sg.N_r; r++)
            for (int t = 0; t < sg.N_t; t++) d[(size_t)t * sg.N_r + r] = offset[(size_t)r * sg.N_t + t];
        CK(cudaMemcpyAsync(S->d_d, d.data(), d.size() * sizeof(float), cudaMemcpyHostToDevice, S->stream));
    } else {
        CK(cudaMemsetAsync(S->d_d, 0, (size_t)sg.N_t * sg.N_r * sizeof(float), S->stream));
    }
    if (fill_mag()) return -1;
    CK(mbir_forward_rows(S->g, S->d_fov, S->d_x, S->d_y, S->d_d, S->d_e, 0, S->amax(), S->stream));
    S->launches++;
    CK(cudaStreamSynchronize(S->stream));
    S->prepared = 1;
    S->have_cost = S->win_open = false;
    S->guard_checks = 0;
    return 0;
}

extern "C" int mbir_icd_prepare(MbirStage *S, const float *object, const float *offset,
                                const float *magmap)
{
    return icd_prepare_with(
        S, offset,
        [&]() -> int {
            if (object)
                CK(cudaMemcpyAsync(S->d_x, object, S->nvox() * sizeof(float), cudaMemcpyHostToDevice, S->stream));
            else
                CK(cudaMemsetAsync(S->d_x, 0, S->nvox() * sizeof(float), S->stream));
            return 0;
        },
        [&]() -> int {
            if (magmap)
                CK(cudaMemcpyAsync(S->d_mag, magmap, S->nmag() * sizeof(float), cudaMemcpyHostToDevice, S->stream));
            else
                CK(cudaMemsetAsync(S->d_mag, 0, S->nmag() * sizeof(float), S->stream));
            return 0;
        });
}

// The prologue of the stage after `prev` in one multi-resolution run, with
// the hand-off on the device (initObject, XT_ICD_update.c:540-651): the start
// object is prev's object up-sampled x2 in x and y (initICD 2) or in x, y
// and z (initICD 3), the magnitude map prev's up-sampled likewise when its
// planes per frame allow (the same count, or half), else zero.  prev must
// have finished its iterations.
int mbir_icd_prepare_from(MbirStage *S, MbirStage *prev, int initICD, const float *offset, int *mag_carried)
{
    const int Nt = S->sg.N_time, cNz = prev->st.N_z, cNy = prev->st.N_y, cNx = prev->st.N_x;
    if (2 * cNy != S->st.N_y || 2 * cNx != S->st.N_x || (initICD == 3 ? 2 * cNz : cNz) != S->st.N_z)
        return fail("stage hand-off: the previous stage is not half this one's size");
    const int pb = prev->nblk, nb = S->nblk;
    const bool mag_ok = pb == nb || 2 * pb == nb;
    if (mag_carried) *mag_carried = mag_ok ? 1 : 0;
    return icd_prepare_with(
        S, offset,
        [&]() -> int {
            for (int f = 0; f < Nt; f++)
                CK(mbir_launch_upsample(prev->d_x + (size_t)f * prev->st.N_z * prev->nxy(),
                                        S->d_x + (size_t)f * S->st.N_z * S->nxy(), cNz, cNy, cNx, initICD == 3,
                                        S->stream));
            S->launches += Nt;
            return 0;
        },
        [&]() -> int {
            if (!mag_ok) {
                CK(cudaMemsetAsync(S->d_mag, 0, S->nmag() * sizeof(float), S->stream));
                return 0;
            }
            for (int f = 0; f < Nt; f++)
                CK(mbir_launch_upsample(prev->d_mag + (size_t)f * pb * prev->nxy(),
                                        S->d_mag + (size_t)f * nb * S->nxy(), pb, cNy, cNx, pb != nb, S->stream));
            S->launches += Nt;
            return 0;
        });
}

// ---------------------------------------------------------------------------
// Reference schedule (updateVoxelsTimeSlices, XT_ICD_update.c:936-1105)
// ---------------------------------------------------------------------------
static int run_half(MbirStage *S, int j, int second, int nhicd, int iter, double *vox_mag)
{
    const int per = S->st.N_z / S->nblk;
    std::vector<MbirTask> tasks;
    for (int i = 0; i < S->sg.N_time; i++)
        for (int b = 0; b < S->nblk; b += 2) {
            const int idx = second ? ((i % 2 == 0) ? b + 1 : b) : ((i % 2 == 0) ? b : b + 1);
            MbirTask t{};
            t.frame = i;
            t.z0 = idx * per;
            t.z1 = (idx >= S->nblk - 1) ? S->st.N_z - 1 : (idx + 1) * per - 1;
            const size_t plane = ((size_t)i * S->nblk + idx);
            t.mag = S->d_mag + plane * S->nxy();
            if (!nhicd) {
                const int num = S->nr[plane];
                t.b0 = j * (num / S->K);
                t.b1 = (j == S->K - 1) ? num - 1 : (j + 1) * (num / S->K) - 1;
                t.xs = S->d_xr + plane * S->nxy();
                t.ys = S->d_yr + plane * S->nxy();
            } else {
                t.b0 = 0;
                t.b1 = S->nn[plane] - 1;
                t.xs = S->d_xn + plane * S->nxy();
                t.ys = S->d_yn + plane * S->nxy();
            }
            if (t.b1 >= t.b0) tasks.push_back(t);
        }
    if (tasks.empty()) return 0;
    CK(cudaMemcpyAsync(S->d_tasks, tasks.data(), tasks.size() * sizeof(MbirTask), cudaMemcpyHostToDevice,
                       S->stream));
    CK(cudaEventRecord(S->ev0, S->stream));
    CK(mbir_launch_icd_ref(S->g, S->pr, S->dv, S->d_tasks, (int)tasks.size(), S->d_tout, iter,
                           S->threads, S->acache_bytes, S->d_acache, S->stream));
    CK(cudaEventRecord(S->ev1, S->stream));
    S->launches++;
    S->icd_launches++;
    std::vector<MbirTaskOut> out(tasks.size());
    CK(cudaMemcpyAsync(out.data(), S->d_tout, out.size() * sizeof(MbirTaskOut), cudaMemcpyDeviceToHost,
                       S->stream));
    CK(cudaStreamSynchronize(S->stream));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, S->ev0, S->ev1));
    S->icd_ms += ms;
    for (auto &o : out) {
        *vox_mag += o.vox_mag;
        S->updates += o.updates;
        S->zero_skips += o.zero_skips;
    }
    return 0;
}

// The ring-offset update enqueued on the stage's stream (no host sync).
static int offset_update_async(MbirStage *S)
{
    CK(mbir_launch_offset(S->g, S->pr, S->dv, S->offset_type, S->d_num, S->d_den, S->d_partials,
                          S->nparts, S->stream, &S->win, S->d_err, S->d_ochunk));
    S->launches += S->offset_type == 3 && S->win.M > 0 ? 6 : 5;
    return 0;
}

extern "C" int mbir_update_sinogram_offset(MbirStage *S)
{
    if (offset_update_async(S)) return -1;
    int err = 0;
    CK(cudaMemcpyAsync(&err, S->d_err, sizeof(int), cudaMemcpyDeviceToHost, S->stream));
    CK(cudaStreamSynchronize(S->stream));
    if (err & 16) return fail("ring-offset constraint system is not positive definite");
    return 0;
}

// Constraint windows of offset mode 3 (gen_offset_constraint_windows,
// XT_OffsetError.c:46-96): sides r_size = 2 N_r / round(sqrt(N_r)) and
// t_size = 2 N_t / round(sqrt(N_t)), origins every half side, wrapping
// around the detector, tent weights; a later assignment to an element of the
// same window replaces an earlier one, as in the reference's loop.  Lists are
// in the reference's element order (detector column major, row inner).
extern "C" int mbir_set_offset_windows(MbirStage *S, int32_t on)
{
    if (on && S->slab_count > 1)
        return fail("ring-offset constraint windows reduce over the ranks; not supported on a sharded stage");
    CK(cudaStreamSynchronize(S->stream));
    for (void *b : S->win_bufs) dfree(b);
    S->win_bufs.clear();
    S->win = OffsetWindows{};
    if (!on) return 0;
    if (!S->d_err) CK(dalloc(&S->d_err, 1));
    const int Nr = S->sg.N_r, Nt = S->sg.N_t, nel = Nr * Nt;
    const int rs = 2 * Nr / (int)(std::sqrt((double)Nr) + 0.5), ts = 2 * Nt / (int)(std::sqrt((double)Nt) + 0.5);
    // per window: its elements (q = t N_r + r) in reference order and weights
    std::vector<std::vector<std::pair<int, float>>> wins;
    std::vector<float> val(nel, 0.0f);
    std::vector<int> seen(nel, -1);
    for (int i = 0; i <= Nr - rs / 2; i += rs / 2)
        for (int j = 0; j <= Nt - ts / 2; j += ts / 2) {
            const int m = (int)wins.size();
            std::vector<int> touched;
            for (int k = i; k < i + rs; k++)
                for (int l = j; l < j + ts; l++) {
                    double a = (k - i) < rs / 2 ? (k - i + 1) : rs - (k - i);
                    a *= (l - j) < ts / 2 ? (l - j + 1) : ts - (l - j);
                    const int q = (l % Nt) * Nr + k % Nr;
                    if (seen[q] != m) {
                        seen[q] = m;
                        touched.push_back(q);
                    }
                    val[q] = (float)a;
                }
            std::sort(touched.begin(), touched.end(), [&](int a, int b) {
                const int ra = a % Nr, rb = b % Nr;
                return ra != rb ? ra < rb : a / Nr < b / Nr;
            });
            std::vector<std::pair<int, float>> w;
            for (int q : touched) w.push_back({q, val[q]});
            wins.push_back(std::move(w));
        }
    const int M = (int)wins.size();
    if (M == 0) return 0;
    // per element its windows; per overlapping pair the shared elements
    std::vector<std::vector<std::pair<int, float>>> els(nel);
    for (int m = 0; m < M; m++)
        for (auto &p : wins[m]) els[p.first].push_back({m, p.second});
    std::map<std::pair<int, int>, std::vector<int>> pairs;  // (i <= j) -> element list (reference order)
    std::vector<int> order(nel);
    for (int q = 0; q < nel; q++) order[q] = q;
    std::sort(order.begin(), order.end(), [&](int a, int b) {
        const int ra = a % Nr, rb = b % Nr;
        return ra != rb ? ra < rb : a / Nr < b / Nr;
    });
    for (int q : order)
        for (size_t u = 0; u < els[q].size(); u++)
            for (size_t v = u; v < els[q].size(); v++) {
                int a = els[q][u].first, b = els[q][v].first;
                if (a > b) std::swap(a, b);
                pairs[{a, b}].push_back(q);
            }
    std::vector<int> win_off(M + 1, 0), win_el, pair_off(1, 0), pair_i, pair_j, pair_el, el_off(nel + 1, 0), el_m;
    std::vector<float> win_a, pair_ai, pair_aj, el_a;
    for (int m = 0; m < M; m++) {
        for (auto &p : wins[m]) {
            win_el.push_back(p.first);
            win_a.push_back(p.second);
        }
        win_off[m + 1] = (int)win_el.size();
    }
    auto weight = [&](int m, int q) {
        for (auto &p : els[q])
            if (p.first == m) return p.second;
        return 0.0f;
    };
    for (auto &kv : pairs) {
        pair_i.push_back(kv.first.first);
        pair_j.push_back(kv.first.second);
        for (int q : kv.second) {
            pair_el.push_back(q);
            pair_ai.push_back(weight(kv.first.first, q));
            pair_aj.push_back(weight(kv.first.second, q));
        }
        pair_off.push_back((int)pair_el.size());
    }
    for (int q = 0; q < nel; q++) {
        for (auto &p : els[q]) {
            el_m.push_back(p.first);
            el_a.push_back(p.second);
        }
        el_off[q + 1] = (int)el_m.size();
    }
    auto up = [&](auto &vec, auto **dst) -> int {
        using T = typename std::remove_reference<decltype(vec)>::type::value_type;
        T *d = nullptr;
        CK(dalloc(&d, std::max<size_t>(vec.size(), 1)));
        S->win_bufs.push_back(d);
        if (!vec.empty())
            CK(cudaMemcpyAsync(d, vec.data(), vec.size() * sizeof(T), cudaMemcpyHostToDevice, S->stream));
        *dst = d;
        return 0;
    };
    OffsetWindows W{};
    W.M = M;
    W.nel = nel;
    W.npairs = (int)pair_i.size();
    if (up(win_off, &W.win_off) || up(win_el, &W.win_el) || up(win_a, &W.win_a) || up(pair_off, &W.pair_off) ||
        up(pair_i, &W.pair_i) || up(pair_j, &W.pair_j) || up(pair_el, &W.pair_el) || up(pair_ai, &W.pair_ai) ||
        up(pair_aj, &W.pair_aj) || up(el_off, &W.el_off) || up(el_m, &W.el_m) || up(el_a, &W.el_a))
        return -1;
    double *D = nullptr, *y = nullptr, *x = nullptr;
    CK(dalloc(&D, (size_t)M * M));
    CK(dalloc(&y, (size_t)M));
    CK(dalloc(&x, (size_t)nel));
    S->win_bufs.push_back(D);
    S->win_bufs.push_back(y);
    S->win_bufs.push_back(x);
    W.D = D;
    W.y = y;
    W.x = x;
    CK(cudaStreamSynchronize(S->stream));
    S->win = W;
    return 0;
}

extern "C" int mbir_get_offset_windows(MbirStage *S) { return S->win.M; }

// ---------------------------------------------------------------------------
// z-slab sharding (XT_MPI.c:47-122)
// ---------------------------------------------------------------------------
// Sum of n doubles over the slabs, in place; the identity for a whole volume.
static int slab_sum(MbirStage *S, double *v, int n)
{
    if (S->slab_count <= 1) return 0;
    if (!S->allreduce || S->allreduce(v, n, S->allreduce_ctx) != 0)
        return fail("z-slab reduction over the ranks failed");
    return 0;
}

extern "C" int mbir_debug_sv_skip_tasks(MbirStage *S, int32_t n)
{
    if (S->schedule != 1) return fail("the super-voxel schedule is not set");
    S->debug_skip = std::max(0, n);
    return 0;
}

extern "C" int mbir_set_z_slab(MbirStage *S, int32_t rank, int32_t ranks, MbirAllreduceFn allreduce, void *ctx)
{
    if (ranks < 1 || rank < 0 || rank >= ranks) return fail("z-slab %d of %d", rank, ranks);
    if (ranks > 1 && !allreduce) return fail("a sharded stage needs a reduction over its ranks");
    if (ranks > 1 && S->win.M > 0)
        return fail("ring-offset constraint windows reduce over the ranks; not supported on a sharded stage");
    const size_t n = 2 * (size_t)S->sg.N_time * S->nxy();
    if (ranks > 1 && !S->d_halo) {
        CK(dalloc(&S->d_halo, n));
        CK(cudaMemsetAsync(S->d_halo, 0, n * sizeof(float), S->stream));
        CK(cudaStreamSynchronize(S->stream));
    }
    S->slab_rank = rank;
    S->slab_count = ranks;
    S->allreduce = ranks > 1 ? allreduce : nullptr;
    S->allreduce_ctx = ranks > 1 ? ctx : nullptr;
    S->dv.halo = ranks > 1 ? S->d_halo : nullptr;
    S->dv.halo_lo = ranks > 1 && rank > 0;
    S->dv.halo_hi = ranks > 1 && rank < ranks - 1;
    S->have_cost = false;  // the guard's cost is the whole volume's from here
    return 0;
}

extern "C" int mbir_get_slab_faces(MbirStage *S, float *lo, float *hi)
{
    const size_t plane = S->nxy() * sizeof(float), frame = (size_t)S->st.N_z * plane;
    if (lo)
        CK(cudaMemcpy2DAsync(lo, plane, S->d_x, frame, plane, S->sg.N_time, cudaMemcpyDeviceToDevice, S->stream));
    if (hi)
        CK(cudaMemcpy2DAsync(hi, plane, S->d_x + (size_t)(S->st.N_z - 1) * S->nxy(), frame, plane, S->sg.N_time,
                             cudaMemcpyDeviceToDevice, S->stream));
    CK(cudaStreamSynchronize(S->stream));
    return 0;
}

extern "C" int mbir_set_slab_halo(MbirStage *S, const float *lo, const float *hi)
{
    if (!S->d_halo) return fail("not a sharded stage (mbir_set_z_slab with ranks > 1)");
    const size_t n = (size_t)S->sg.N_time * S->nxy();
    if (lo) CK(cudaMemcpyAsync(S->d_halo, lo, n * sizeof(float), cudaMemcpyDeviceToDevice, S->stream));
    if (hi) CK(cudaMemcpyAsync(S->d_halo + n, hi, n * sizeof(float), cudaMemcpyDeviceToDevice, S->stream));
    CK(cudaStreamSynchronize(S->stream));
    return 0;
}

extern "C" int mbir_update_variance_parameter(MbirStage *S)
{
    CK(mbir_launch_variance(S->g, S->pr, S->dv, S->var_est, S->d_partials, S->nparts, S->d_result,
                            S->stream));
    S->launches += 3;
    double sum = 0;
    CK(cudaMemcpyAsync(&sum, S->d_result, sizeof(double), cudaMemcpyDeviceToHost, S->stream));
    CK(cudaStreamSynchronize(S->stream));
    // summed over the slabs (XT_ICD_update.c:738-739)
    if (slab_sum(S, &sum, 1)) return -1;
    S->var_est = sum / ((double)S->slab_count * (double)S->sg.N_p * (double)S->sg.N_r * (double)S->sg.N_t);
    CK(mbir_launch_variance_apply(S->g, S->dv, S->var_est, S->stream));
    CK(cudaStreamSynchronize(S->stream));
    return 0;
}

// NHICD line selection (VSC_based_Voxel_Line_Select, XT_NHICD.c:164-216):
// filter on the GPU, order statistic and raster-order selection on the host
// so that the generator's draws follow the reference's.
static int vsc_select(MbirStage *S)
{
    const int planes = S->sg.N_time * S->nblk;
    const size_t nxy = S->nxy();
    CK(mbir_launch_vsc_filter(S->d_mag, S->d_filt, planes, S->st.N_y, S->st.N_x, S->stream));
    S->launches++;
    std::vector<float> f((size_t)planes * nxy), work(nxy);
    CK(cudaMemcpyAsync(f.data(), S->d_filt, f.size() * sizeof(float), cudaMemcpyDeviceToHost, S->stream));
    CK(cudaStreamSynchronize(S->stream));
    std::vector<int> xs((size_t)planes * nxy), ys((size_t)planes * nxy);
    for (int pl = 0; pl < planes; pl++) {
        const float *fc = &f[(size_t)pl * nxy];
        std::copy(fc, fc + nxy, work.begin());
        const int n = S->nr[pl] / S->K;
        const double th = order_statistic(S->rng, work.data(), (uint32_t)nxy, (uint32_t)(nxy - n));
        int cnt = 0;
        for (size_t q = 0; q < nxy; q++)
            if (fc[q] > th) {
                xs[(size_t)pl * nxy + cnt] = (int)(q % S->st.N_x);
                ys[(size_t)pl * nxy + cnt] = (int)(q / S->st.N_x);
                cnt++;
            }
        S->nn[pl] = cnt;
    }
    CK(cudaMemcpyAsync(S->d_xn, xs.data(), xs.size() * sizeof(int), cudaMemcpyHostToDevice, S->stream));
    CK(cudaMemcpyAsync(S->d_yn, ys.data(), ys.size() * sizeof(int), cudaMemcpyHostToDevice, S->stream));
    CK(cudaStreamSynchronize(S->stream));
    return 0;
}

static int random_select(MbirStage *S)
{
    const int planes = S->sg.N_time * S->nblk;
    const size_t nxy = S->nxy();
    std::vector<int> xs((size_t)planes * nxy), ys((size_t)planes * nxy);
    const int per = S->st.N_z / S->nblk;
    for (int pl = 0; pl < planes; pl++)
        S->nr[pl] = random_lines(S->rng, S->mask.data(), S->st.N_y, S->st.N_x, per, &xs[(size_t)pl * nxy],
                                 &ys[(size_t)pl * nxy]);
    CK(cudaMemcpyAsync(S->d_xr, xs.data(), xs.size() * sizeof(int), cudaMemcpyHostToDevice, S->stream));
    CK(cudaMemcpyAsync(S->d_yr, ys.data(), ys.size() * sizeof(int), cudaMemcpyHostToDevice, S->stream));
    CK(cudaStreamSynchronize(S->stream));
    return 0;
}

// ---------------------------------------------------------------------------
// Super-voxel schedule
// ---------------------------------------------------------------------------
static SvParams sv_params(const MbirStage *S, int side, int nz, int vsplit)
{
    SvParams sp{};
    const double m = S->st.delta_xy / S->sg.delta_r;
    sp.S = side;
    // band width: projected extent of the block plus each voxel's footprint
    // (+-delta_xy) plus floor effects at both ends
    sp.W = (int)floor((side - 1) * sqrt(2.0) * m + 2 * m + 1e-9) + 3;
    sp.amax = 2 * (int)ceil(m) + 1;
    sp.eq = (1 + sp.amax + 3) / 4;
    sp.ring = kSvRing;
    sp.ahalf = S->acol_half ? 1 : 0;
    sp.max_views = S->max_views();
    sp.max_nz = nz;
    sp.max_rows = nz * S->st.m_z;
    // warps per slice: up to 4 (named barriers 1..15 serve one slice each)
    if (vsplit <= 0) vsplit = nz <= 15 ? 2 : 1;
    while (vsplit > 1 && (nz > 15 || 32 * nz * vsplit > 1024)) vsplit /= 2;
    sp.vsplit = std::min(vsplit, 4);
    // producer warps for the A-matrix columns: one view per lane, within the
    // 1024-thread limit
    const int want = (sp.max_views + 31) / 32;
    sp.prod_warps = std::max(0, std::min(std::min(want, 8), (1024 - 32 * nz * sp.vsplit) / 32));
    sp.band_floats = sv_scratch_floats(sp.max_rows, sp.W, sp.max_views);
    return sp;
}

// Orders super-voxel ids for a sweep: colour phases starting from phase r,
// the largest super-voxels of a phase first.
// Orders super-voxel ids for a sweep: colour phases starting from phase r;
// within a phase the (frame, z-group) groups take turns, largest super-voxels
// first, so that the super-voxels in flight spread over the groups.
static void sv_sort(const MbirStage *S, std::vector<int> &ids, int r)
{
    const int P = S->sv_nphase;
    std::stable_sort(ids.begin(), ids.end(), [&](int a, int b) {
        const int pa = (S->sv_all_phase[a] - r + P) % P, pb = (S->sv_all_phase[b] - r + P) % P;
        if (pa != pb) return pa < pb;
        if (S->sv_rank[a] != S->sv_rank[b]) return S->sv_rank[a] < S->sv_rank[b];
        return S->sv_all[a].nlines > S->sv_all[b].nlines;
    });
}

// Launch list of super-voxels `ids` in that order, appended to buf as
// [order | dep_off | deps]: for each, the conflicting super-voxels earlier in
// the list (they finish first; so no two conflicting ones run at once, and
// every wait is for a super-voxel that an earlier CTA already holds).
// meta = {n, order offset, dep_off offset, deps offset}.
static void sv_build_list(const MbirStage *S, const std::vector<int> &ids, std::vector<int> &buf,
                          std::array<size_t, 4> &meta)
{
    std::vector<int> pos(S->sv_all.size(), -1), deps;
    for (size_t k = 0; k < ids.size(); k++) pos[ids[k]] = (int)k;
    meta[0] = ids.size();
    meta[1] = buf.size();
    buf.insert(buf.end(), ids.begin(), ids.end());
    meta[2] = buf.size();
    buf.resize(buf.size() + ids.size() + 1);
    for (size_t k = 0; k < ids.size(); k++) {
        buf[meta[2] + k] = (int)deps.size();
        for (int nb : S->sv_nbr[ids[k]])
            if (pos[nb] >= 0 && pos[nb] < (int)k) deps.push_back(nb);
    }
    buf[meta[2] + ids.size()] = (int)deps.size();
    meta[3] = buf.size();
    buf.insert(buf.end(), deps.begin(), deps.end());
}

// The super-voxels of schedule 1 (tasks, colour phases, size ranks,
// conflicts) and the full-sweep launch lists of every phase rotation, into
// S and buf.  They depend only on the geometry (grid, z-groups, side, mask),
// so they are kept in a small process-wide cache: stages of the same
// geometry set up one after another (a scan series, the stages of repeated
// reconstructions) reuse them instead of rebuilding them on the host.
namespace {
struct SvScheduleCache {
    std::vector<SvTask> all;
    std::vector<int> phase, rank, buf;
    std::vector<std::vector<int>> nbr;
    std::vector<std::array<size_t, 4>> rot;
    int nphase = 1;
};
std::mutex g_sched_mu;
std::vector<std::pair<std::string, std::shared_ptr<const SvScheduleCache>>> g_sched_cache;  // most recent last
}  // namespace

static void sv_schedule_build(MbirStage *S, const SvParams &sp, int gz, std::vector<int> &buf)
{
    const int Nz = S->st.N_z;
    // super-voxels, coloured by SV x / y parity, z-group parity, frame parity
    const int side_ = sp.S, N_x = S->st.N_x, N_y = S->st.N_y, N_time = S->sg.N_time;
    const int ntx = (N_x + side_ - 1) / side_, nty = (N_y + side_ - 1) / side_;
    std::vector<int> phase_of(16, -1), cell((size_t)N_time * S->nzg * nty * ntx, -1);
    auto cell_of = [&](int i, int zg, int ty, int tx) { return (((size_t)i * S->nzg + zg) * nty + ty) * ntx + tx; };
    int nphase = 0;
    S->sv_all.clear();
    S->sv_all_phase.clear();
    for (int i = 0; i < N_time; i++)
        for (int zg = 0; zg < S->nzg; zg++)
            for (int ty = 0; ty < nty; ty++)
                for (int tx = 0; tx < ntx; tx++) {
                    const int k0 = tx * side_, j0 = ty * side_;
                    int lines = 0;
                    for (int y = j0; y < std::min(N_y, j0 + side_); y++)
                        for (int x = k0; x < std::min(N_x, k0 + side_); x++)
                            if (S->mask[(size_t)y * N_x + x]) lines++;
                    if (!lines) continue;
                    const int colour = (tx & 1) | ((ty & 1) << 1) | ((S->nzg > 1 ? (zg & 1) : 0) << 2) |
                                       ((N_time > 1 ? (i & 1) : 0) << 3);
                    if (phase_of[colour] < 0) phase_of[colour] = nphase++;
                    SvTask t{};
                    t.frame = i;
                    t.k0 = k0;
                    t.j0 = j0;
                    t.z0 = zg * gz;
                    t.nz = std::min(gz, Nz - t.z0);
                    t.nlines = lines;
                    t.mag = S->d_mag + ((size_t)i * S->nzg + zg) * S->nxy();
                    t.plane = i * S->nzg + zg;
                    cell[cell_of(i, zg, ty, tx)] = (int)S->sv_all.size();
                    S->sv_all.push_back(t);
                    S->sv_all_phase.push_back(phase_of[colour]);
                }
    S->sv_nphase = nphase;
    // size rank within (phase, frame, z-group)
    {
        std::vector<int> ids(S->sv_all.size());
        for (size_t q = 0; q < ids.size(); q++) ids[q] = (int)q;
        auto key = [&](int a) {
            return ((long long)S->sv_all_phase[a] * N_time + S->sv_all[a].frame) * S->nzg + S->sv_all[a].z0 / gz;
        };
        std::stable_sort(ids.begin(), ids.end(), [&](int a, int b) {
            if (key(a) != key(b)) return key(a) < key(b);
            return S->sv_all[a].nlines > S->sv_all[b].nlines;
        });
        S->sv_rank.assign(ids.size(), 0);
        for (size_t q = 1; q < ids.size(); q++)
            S->sv_rank[ids[q]] = key(ids[q]) == key(ids[q - 1]) ? S->sv_rank[ids[q - 1]] + 1 : 0;
    }
    // conflicts: super-voxels sharing a prior neighbourhood -- x-y-z neighbours
    // in the same frame, the same block in adjacent frames
    S->sv_nbr.assign(S->sv_all.size(), {});
    for (int i = 0; i < N_time; i++)
        for (int zg = 0; zg < S->nzg; zg++)
            for (int ty = 0; ty < nty; ty++)
                for (int tx = 0; tx < ntx; tx++) {
                    const int id = cell[cell_of(i, zg, ty, tx)];
                    if (id < 0) continue;
                    for (int dz = -1; dz <= 1; dz++)
                        for (int dy = -1; dy <= 1; dy++)
                            for (int dx = -1; dx <= 1; dx++) {
                                const int z2 = zg + dz, y2 = ty + dy, x2 = tx + dx;
                                if ((dz | dy | dx) == 0 || z2 < 0 || z2 >= S->nzg || y2 < 0 || y2 >= nty || x2 < 0 ||
                                    x2 >= ntx)
                                    continue;
                                const int nb = cell[cell_of(i, z2, y2, x2)];
                                if (nb >= 0) S->sv_nbr[id].push_back(nb);
                            }
                    for (int di = -1; di <= 1; di += 2)
                        if (i + di >= 0 && i + di < N_time) {
                            const int nb = cell[cell_of(i + di, zg, ty, tx)];
                            if (nb >= 0) S->sv_nbr[id].push_back(nb);
                        }
                }
    // full-sweep launch lists, one per phase rotation
    S->sv_rot.assign(nphase, {});
    for (int r = 0; r < nphase; r++) {
        std::vector<int> ids(S->sv_all.size());
        for (size_t q = 0; q < ids.size(); q++) ids[q] = (int)q;
        sv_sort(S, ids, r);
        sv_build_list(S, ids, buf, S->sv_rot[r]);
    }
}

static void sv_schedule(MbirStage *S, const SvParams &sp, int gz, std::vector<int> &buf)
{
    std::string key(reinterpret_cast<const char *>(S->mask.data()), S->mask.size());
    const int dims[7] = {S->st.N_x, S->st.N_y, S->st.N_z, S->sg.N_time, sp.S, gz, S->nzg};
    key.append(reinterpret_cast<const char *>(dims), sizeof(dims));
    std::shared_ptr<const SvScheduleCache> hit;
    {
        std::lock_guard<std::mutex> lock(g_sched_mu);
        for (auto &e : g_sched_cache)
            if (e.first == key) hit = e.second;
    }
    if (!hit) {
        sv_schedule_build(S, sp, gz, buf);
        auto c = std::make_shared<SvScheduleCache>();
        c->all = S->sv_all;
        c->phase = S->sv_all_phase;
        c->rank = S->sv_rank;
        c->nbr = S->sv_nbr;
        c->rot = S->sv_rot;
        c->buf = buf;
        c->nphase = S->sv_nphase;
        std::lock_guard<std::mutex> lock(g_sched_mu);
        g_sched_cache.emplace_back(std::move(key), std::move(c));
        if (g_sched_cache.size() > 8) g_sched_cache.erase(g_sched_cache.begin());
        return;
    }
    S->sv_all = hit->all;
    S->sv_all_phase = hit->phase;
    S->sv_rank = hit->rank;
    S->sv_nbr = hit->nbr;
    S->sv_rot = hit->rot;
    S->sv_nphase = hit->nphase;
    buf = hit->buf;
    for (SvTask &t : S->sv_all) t.mag = S->d_mag + (size_t)t.plane * S->nxy();
}

// dynamic shared memory per CTA: the 227 KB opt-in limit less the kernels' static
// shared memory (at most 1.1 KB: the batched kernel's problem descriptor)
// Lines the NHICD pass selects per plane: nh_fraction of the in-mask lines.
static int sv_upload_nsel(MbirStage *S)
{
    if (!S->d_nh_nsel) return 0;
    size_t in_mask = 0;
    for (uint8_t m : S->mask) in_mask += m == 1;
    S->nh_nsel.assign((size_t)S->sg.N_time * S->nzg, (int)std::floor(S->nh_fraction * (double)in_mask));
    CK(cudaMemcpyAsync(S->d_nh_nsel, S->nh_nsel.data(), S->nh_nsel.size() * sizeof(int), cudaMemcpyHostToDevice,
                       S->stream));
    CK(cudaStreamSynchronize(S->stream));
    return 0;
}

// Over-relaxation and in-flight cap of the super-voxel schedule for `want`
// super-voxels wanted in flight at once (see the concurrency note in
// mbir_set_schedule): alpha = the stage's (1.5 unless set) when the cap of
// each active (frame, z-group) sinogram holds its share, else the largest
// value down to 0.7 that does, as long as the share stays under 12 % of the
// group's super-voxels.  *cap = super-voxels per sinogram, *grid = in total.
static void sv_relaxation(const MbirStage *S, double want, double *alpha_out, int *cap_out, int *grid_out)
{
    const SvParams &sp = S->sp;
    const int N_time = S->sg.N_time;
    const double Rv = S->sg.radius_obj / S->st.delta_xy;
    const double Wv = sp.W * S->sg.delta_r / S->st.delta_xy;
    const double ref_alpha = S->pr.alpha;
    auto cap_for = [&](double alpha) {
        const double crossings = 1.8 * (2.0 / alpha - 1.0) / (2.0 / 1.5 - 1.0);
        return std::max(4, (int)std::floor(crossings * M_PI * Rv / (2.0 * Wv)));
    };
    const long long active = (long long)(N_time > 1 ? (N_time + 1) / 2 : 1) * (S->nzg > 1 ? (S->nzg + 1) / 2 : 1);
    double alpha = S->sv_alpha > 0 ? S->sv_alpha : ref_alpha;
    const double groups = (double)N_time * S->nzg;
    const double per = std::min(want / (double)active,  // in flight per sinogram wanted
                                std::max(1.0, std::floor(0.12 * (double)S->sv_all.size() / groups)));
    if (S->sv_alpha <= 0 && cap_for(ref_alpha) < per) {
        const double g = per / cap_for(ref_alpha) * (2.0 / ref_alpha - 1.0);
        alpha = std::min(ref_alpha, std::max(0.7, 2.0 / (1.0 + g)));
    }
    *alpha_out = alpha;
    *cap_out = cap_for(alpha);
    *grid_out = (int)std::max<double>(1.0, std::min<double>(std::ceil(want), (double)*cap_out * active));
}

static const size_t kSmemLimit = 227 * 1024 - 2048;
static const int kMaxLaunchesPerIter = 64;

// Super-voxel side 0 = choose the largest side (<= 16) whose band for a
// z-group of min(N_z, 32) slices fits shared memory, shrinking the group if
// even side 4 does not fit.
extern "C" int mbir_set_schedule(MbirStage *S, int32_t schedule, int32_t sv_side, int32_t warps_per_slice)
{
    if (schedule == 0) {
        S->schedule = 0;
        return 0;
    }
    if (schedule != 1) return fail("unknown schedule %d", schedule);
    const int Nz = S->st.N_z;
    // the column cache: used when it fits (or always / never, as set)
    {
        const SvParams probe = sv_params(S, 4, 1, 1);
        // FP16 values: full resolution (3 columns, one detector row per slice)
        // and detectors of at most 4096 columns (12-bit column index)
        const bool half = S->acol_mode == 2 && probe.amax == 3 && S->st.m_z == 1 && S->sg.N_r <= 4096;
        const size_t bytes = mbir_acache_bytes(S->g, probe.eq, half);
        size_t fr = 0, tot = 0;
        CK(cudaMemGetInfo(&fr, &tot));
        const bool want = S->acol_mode == 1 || ((S->acol_mode == -1 || S->acol_mode == 2) && bytes <= fr / 3);
        S->acol_half = want && half;
        if (want && bytes != S->acol_bytes) {
            dfree(S->d_acol);
            S->d_acol = nullptr;
            S->acol_bytes = 0;
            if (S->acol_mode == 1 && bytes > fr)
                return fail("A-matrix column cache of %zu bytes does not fit (%zu free)", bytes, fr);
            CK(dalloc(&S->d_acol, bytes / sizeof(int4)));
            S->acol_bytes = bytes;
        } else if (!want) {
            dfree(S->d_acol);
            S->d_acol = nullptr;
            S->acol_bytes = 0;
        }
        S->acol_built = false;
    }
    const bool cached = S->d_acol != nullptr;
    int gz = S->sv_zgroup > 0 ? std::min(S->sv_zgroup, Nz) : std::min(Nz, 32), side = sv_side;
    SvParams sp{};
    for (;;) {
        if (side > 0) {
            sp = sv_params(S, side, gz, warps_per_slice);
            if (mbir_sv_smem_bytes(sp, cached) <= kSmemLimit) break;
        } else {
            int best = 0;
            for (int s = 16; s >= 4; s--) {
                sp = sv_params(S, s, gz, warps_per_slice);
                if (mbir_sv_smem_bytes(sp, cached) <= kSmemLimit) {
                    best = s;
                    break;
                }
            }
            if (best) {
                sp = sv_params(S, best, gz, warps_per_slice);
                break;
            }
        }
        if (gz == 1) return fail("no super-voxel configuration fits shared memory");
        gz = std::max(1, gz / 2);
    }
    if (cached && sp.ahalf) {
        const int vpl = (sp.max_views + 32 * sp.vsplit - 1) / (32 * sp.vsplit);
        const int thr = 32 * sp.max_nz * sp.vsplit;
        if (!((vpl <= 4 && thr <= 512) || (vpl <= 8 && thr <= 256)))
            return fail("the FP16 column cache needs at most 4 views per lane and 512 threads per super-voxel, or "
                        "8 and 256 (%d views per lane, %d threads)", vpl, thr);
    }
    S->sp = sp;
    S->gz = gz;
    S->nzg = (Nz + gz - 1) / gz;
    // the magnitude map holds one plane per (frame, z-group)
    if (S->nzg != S->nblk) {
        dfree(S->d_mag);
        dfree(S->d_filt);
        S->d_mag = S->d_filt = nullptr;
        S->nblk = S->nzg;
        CK(dalloc(&S->d_mag, S->nmag()));
        CK(dalloc(&S->d_filt, S->nmag()));
        CK(cudaMemsetAsync(S->d_mag, 0, S->nmag() * sizeof(float), S->stream));
        S->dv.mag = S->d_mag;
        S->nr.assign((size_t)S->sg.N_time * S->nblk, 0);
        S->nn.assign((size_t)S->sg.N_time * S->nblk, 0);
    }
    if (S->mask.empty()) object_mask(S->sg, S->st, S->mask);
    int dev = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&S->sm_count, cudaDevAttrMultiProcessorCount, dev));
    std::vector<int> buf;
    sv_schedule(S, sp, gz, buf);
    dfree(S->d_sv_all);
    dfree(S->d_sv_done);
    dfree(S->d_sv_lists);
    dfree(S->d_sv_out);
    dfree(S->d_scratch);
    dfree(S->d_queue);
    S->d_sv_all = nullptr;
    S->d_sv_done = S->d_sv_lists = nullptr;
    S->d_sv_out = nullptr;
    S->d_scratch = nullptr;
    S->d_queue = nullptr;
    CK(dalloc(&S->d_sv_all, S->sv_all.size()));
    CK(cudaMemcpyAsync(S->d_sv_all, S->sv_all.data(), S->sv_all.size() * sizeof(SvTask), cudaMemcpyHostToDevice,
                       S->stream));
    CK(dalloc(&S->d_sv_done, S->sv_all.size()));
    CK(cudaMemsetAsync(S->d_sv_done, 0, S->sv_all.size() * sizeof(int), S->stream));
    S->sv_epoch = 0;
    CK(dalloc(&S->d_sv_lists, buf.size()));
    CK(cudaMemcpyAsync(S->d_sv_lists, buf.data(), buf.size() * sizeof(int), cudaMemcpyHostToDevice, S->stream));
    // NHICD selection buffers; n_sel per plane = nh_fraction of the in-mask
    // lines (XT_NHICD.c:171: the lines updated / NHICD iterations)
    {
        const int planes = S->sg.N_time * S->nzg;
        dfree(S->d_nh_sel);
        dfree(S->d_nh_nsel);
        dfree(S->d_nh_count);
        dfree(S->d_nh_pos);
        dfree(S->d_nh_nt);
        dfree(S->d_nh_thresh);
        S->d_nh_sel = nullptr;
        S->d_nh_nsel = S->d_nh_count = S->d_nh_pos = S->d_nh_nt = nullptr;
        S->d_nh_thresh = nullptr;
        CK(dalloc(&S->d_nh_sel, (size_t)planes * S->nxy()));
        CK(dalloc(&S->d_nh_nsel, planes));
        CK(dalloc(&S->d_nh_count, planes));
        CK(dalloc(&S->d_nh_thresh, planes));
        CK(dalloc(&S->d_nh_pos, std::max<size_t>(S->sv_all.size(), 1)));
        CK(dalloc(&S->d_nh_nt, 1));
        if (sv_upload_nsel(S)) return -1;
    }
    // Concurrency.  Super-voxels that run at once each correct the residual of
    // the rays they share as if alone, so their steps add up.  A ray of a
    // (frame, z-group) sinogram crosses on average c = 2 n W / (pi R) of the n
    // super-voxels in flight on it (band width W, object radius R, both in
    // voxels).  With the reference's over-relaxation 1.5 the iteration
    // diverges once c exceeds about 2.1 (measured on 256 x 256 slices, sides
    // 4-10: side 6 converges with 33 in flight, diverges with 48); the limit
    // behaves as (2 / alpha - 1) / 0.16, so a smaller alpha allows more in
    // flight.  The cap keeps c at 1.8 x that limit / 2.1.  The queue runs one
    // colour phase at a time -- one z-group parity and one frame parity -- so
    // half the z-groups and half the frames have super-voxels in flight; it
    // interleaves those groups.  Unless set, alpha is the reference's 1.5
    // when the cap lets every resident CTA work, else the largest value
    // (down to 0.7) that does, as long as the super-voxels in flight stay a
    // small share (12 %) of their group's: measured on the 3-D workload, alpha
    // 0.76 with all 148 CTAs (10 % of the super-voxels) reaches the MAP cost
    // within 1e-5 in 21 iterations and 32 ms, alpha 1.5 with the 30 CTAs it
    // allows in 26 iterations and 156 ms; on a 32 x 32 slice with 64
    // super-voxels, 28 in flight at alpha 0.7 converged far more slowly.
    S->sv_fit = mbir_sv_ctas_per_sm(S->g, sp, cached) * S->sm_count;
    {
        const long long want = std::min<long long>((long long)S->sv_all.size(), (long long)S->sv_fit);
        sv_relaxation(S, (double)want, &S->sv_alpha_eff, &S->sv_cap, &S->sv_grid);
    }
    const size_t ctas = std::min<size_t>(std::max<size_t>(S->sv_all.size(), 1), (size_t)S->sv_fit);
    CK(dalloc(&S->d_sv_out, 2));
    CK(dalloc(&S->d_scratch, ctas * sp.band_floats));
    CK(dalloc(&S->d_queue, kMaxLaunchesPerIter));
    if (!S->d_err) CK(dalloc(&S->d_err, 1));
    CK(cudaMemsetAsync(S->d_err, 0, sizeof(int), S->stream));
    CK(cudaStreamSynchronize(S->stream));
    if (!S->sv_ev[0])
        for (auto &e : S->sv_ev) CK(cudaEventCreate(&e));
    S->stab_events = 0;
    S->have_cost = S->win_open = false;
    S->guard_checks = 0;
    S->schedule = 1;
    return 0;
}

extern "C" int mbir_set_acache(MbirStage *S, int32_t mode)
{
    if (mode < -1 || mode > 2) return fail("column cache mode must be -1, 0, 1 or 2");
    S->acol_mode = mode;
    return 0;
}

extern "C" int mbir_set_sv_ctas(MbirStage *S, int32_t ctas)
{
    if (ctas < 0) return fail("negative CTA count");
    S->sv_ctas = ctas;
    return 0;
}

extern "C" int mbir_set_sv_zgroup(MbirStage *S, int32_t slices)
{
    if (slices < 0) return fail("negative z-group size");
    S->sv_zgroup = slices;
    return 0;
}

extern "C" int mbir_set_sv_relaxation(MbirStage *S, double alpha)
{
    if (!(alpha == 0 || (alpha > 0 && alpha < 2))) return fail("over-relaxation must lie in (0, 2), or be 0");
    S->sv_alpha = alpha;
    return 0;
}

extern "C" int mbir_get_sv_grid(MbirStage *S, int32_t *ctas, int32_t *cap_per_group, int32_t *resident,
                                double *relaxation)
{
    if (ctas) *ctas = S->sv_grid;
    if (cap_per_group) *cap_per_group = S->sv_cap;
    if (resident) *resident = S->sv_fit;
    if (relaxation) *relaxation = S->sv_alpha_eff;
    return 0;
}

extern "C" int mbir_set_sv_nhicd(MbirStage *S, double fraction)
{
    if (!(fraction >= 0.0 && fraction <= 1.0)) return fail("NHICD fraction must lie in [0, 1]");
    S->nh_fraction = fraction;
    return sv_upload_nsel(S);
}

extern "C" int mbir_nhicd_select(const float *mag, int32_t planes, int32_t N_y, int32_t N_x, const int32_t *nsel,
                                 uint8_t *sel, float *thresh)
{
    if (planes <= 0 || N_y <= 0 || N_x <= 0) return fail("non-positive dimensions");
    const size_t n = (size_t)planes * N_y * N_x;
    float *d_mag = nullptr, *d_filt = nullptr, *d_th = nullptr;
    int *d_nsel = nullptr, *d_cnt = nullptr;
    uint8_t *d_sel = nullptr;
    auto release = [&]() {
        dfree(d_mag);
        dfree(d_filt);
        dfree(d_th);
        dfree(d_nsel);
        dfree(d_cnt);
        dfree(d_sel);
    };
    cudaError_t e = dalloc(&d_mag, n);
    if (e == cudaSuccess) e = dalloc(&d_filt, n);
    if (e == cudaSuccess) e = dalloc(&d_th, (size_t)planes);
    if (e == cudaSuccess) e = dalloc(&d_nsel, (size_t)planes);
    if (e == cudaSuccess) e = dalloc(&d_cnt, (size_t)planes);
    if (e == cudaSuccess) e = dalloc(&d_sel, n);
    if (e == cudaSuccess) e = cudaMemcpy(d_mag, mag, n * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_nsel, nsel, planes * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = mbir_launch_vsc_filter(d_mag, d_filt, planes, N_y, N_x, 0);
    if (e == cudaSuccess) e = mbir_launch_vsc_threshold(d_filt, planes, N_y * N_x, d_nsel, d_th, d_sel, d_cnt, 0);
    if (e == cudaSuccess) e = cudaMemcpy(sel, d_sel, n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && thresh) e = cudaMemcpy(thresh, d_th, planes * sizeof(float), cudaMemcpyDeviceToHost);
    release();
    if (e != cudaSuccess) return fail("NHICD selection: %s", cudaGetErrorString(e));
    return 0;
}

extern "C" int mbir_upsample(const float *in, float *out, int32_t n_z, int32_t n_y, int32_t n_x, int32_t z_too)
{
    if (n_z < 1 || n_y < 2 || n_x < 2 || (z_too && n_z < 2)) return fail("up-sampling needs n_y, n_x >= 2 (and n_z >= 2 with z)");
    const size_t ni = (size_t)n_z * n_y * n_x, no = (z_too ? 8 : 4) * ni;
    float *d_in = nullptr, *d_out = nullptr;
    cudaError_t e = dalloc(&d_in, ni);
    if (e == cudaSuccess) e = dalloc(&d_out, no);
    if (e == cudaSuccess) e = cudaMemcpy(d_in, in, ni * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = mbir_launch_upsample(d_in, d_out, n_z, n_y, n_x, z_too != 0, 0);
    if (e == cudaSuccess) e = cudaMemcpy(out, d_out, no * sizeof(float), cudaMemcpyDeviceToHost);
    dfree(d_in);
    dfree(d_out);
    if (e != cudaSuccess) return fail("up-sampling: %s", cudaGetErrorString(e));
    return 0;
}

extern "C" int mbir_set_sv_guard(MbirStage *S, int32_t on)
{
    S->guard = on != 0;
    S->win_open = false;
    return 0;
}

// Times the stability guard of the super-voxel schedule has halved the
// super-voxels in flight since the schedule was set.
extern "C" int mbir_get_sv_adjustments(MbirStage *S) { return S->stab_events; }

extern "C" int mbir_get_acache(MbirStage *S, int32_t *used, int64_t *bytes)
{
    if (used) *used = S->d_acol != nullptr ? (S->acol_half ? 2 : 1) : 0;
    if (bytes) *bytes = (int64_t)S->acol_bytes;
    return 0;
}

// Cached A-matrix columns of one voxel line, [N_p][4 eq] words in the
// stored format (word 0 = j0 | n << 16, then the values' bits).
extern "C" int mbir_get_acache_line(MbirStage *S, int32_t row, int32_t col, int32_t *words)
{
    if (!S->d_acol) return fail("no A-matrix column cache (super-voxel schedule with the cache enabled)");
    if (!S->prepared) return fail("mbir_icd_prepare has not run");
    if (row < 0 || row >= S->st.N_y || col < 0 || col >= S->st.N_x) return fail("line (%d, %d) outside the grid", row, col);
    if (!S->mask[(size_t)row * S->st.N_x + col]) return fail("line (%d, %d) outside the reconstruction mask", row, col);
    if (!S->acol_built) {
        CK(mbir_build_acache(S->g, S->dv, S->sp.amax, S->sp.eq, S->acol_half, S->d_acol, S->d_err, S->stream));
        S->acol_built = true;
    }
    if (S->acol_half) {
        // 8-byte entries, unpacked into the FP32 layout
        std::vector<uint32_t> h((size_t)S->g.N_p * 2);
        CK(cudaMemcpyAsync(h.data(), reinterpret_cast<const uint2 *>(S->d_acol) + ((size_t)row * S->st.N_x + col) * S->g.N_p,
                           h.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, S->stream));
        CK(cudaStreamSynchronize(S->stream));
        auto half_to_float = [](uint32_t b) {
            const uint32_t sgn = (b >> 15) & 1u, ex = (b >> 10) & 31u, man = b & 1023u;
            float v = ex == 0 ? std::ldexp((float)man, -24) : std::ldexp((float)(man | 1024u), (int)ex - 25);
            return sgn ? -v : v;
        };
        for (int p = 0; p < S->g.N_p; p++) {
            const uint32_t w0 = h[2 * p], w1 = h[2 * p + 1];
            const float a[3] = {half_to_float(w0 >> 16), half_to_float(w1 & 0xffffu), half_to_float(w1 >> 16)};
            words[4 * p] = (int32_t)((w0 & 0xfffu) | ((w0 >> 12) & 3u) << 16);
            for (int k = 0; k < 3; k++) std::memcpy(&words[4 * p + 1 + k], &a[k], sizeof(float));
        }
        return 0;
    }
    const size_t n = (size_t)S->g.N_p * S->sp.eq;
    CK(cudaMemcpyAsync(words, S->d_acol + ((size_t)row * S->st.N_x + col) * n, n * sizeof(int4),
                       cudaMemcpyDeviceToHost, S->stream));
    CK(cudaStreamSynchronize(S->stream));
    return 0;
}

extern "C" int mbir_get_schedule(MbirStage *S, int32_t *schedule, int32_t *sv_side, int32_t *z_group,
                                 int32_t *band_width, int32_t *phases, int32_t *warps_per_slice)
{
    if (warps_per_slice) *warps_per_slice = S->sp.vsplit;
    if (schedule) *schedule = S->schedule;
    if (sv_side) *sv_side = S->sp.S;
    if (z_group) *z_group = S->gz;
    if (band_width) *band_width = S->sp.W;
    if (phases) *phases = S->sv_nphase;
    return 0;
}

// One launch of the SV kernel over a launch list at `list` (device) with
// layout meta; no host sync.  subset: the NHICD pass -- queue entries are
// the positions in d_nh_pos, their count in d_nh_nt, and only the lines
// selected in d_nh_sel are visited.
static int sv_launch(MbirStage *S, const int *list, const std::array<size_t, 4> &meta, int iter, uint32_t seed,
                     int qslot, SvTaskOut *acc, bool subset = false, int first = 0, int count = -1, int epoch = 0)
{
    const int n = count >= 0 ? count : (int)meta[0];
    if (n <= 0) return 0;
    const int ctas = std::min(n, S->sv_ctas > 0 ? std::min(S->sv_ctas, S->sv_fit) : S->sv_grid);
    SvACache ac{S->d_acol};
    SvLaunch L{S->d_sv_all, list + meta[1] + first, list + meta[2] + first, list + meta[3], n, S->d_sv_done,
               epoch > 0 ? epoch : ++S->sv_epoch};
    if (subset) {
        L.pos = S->d_nh_pos;
        L.ntasks_dev = S->d_nh_nt;
        L.sel = S->d_nh_sel;
    }
    MbirPrior pr = S->pr;
    pr.alpha = S->sv_alpha_eff;
    CK(mbir_launch_icd_sv(S->g, pr, S->dv, S->sp, ac, L, ctas, S->d_queue + qslot, S->d_scratch, acc, iter,
                          seed, S->d_err, S->stream));
    S->launches++;
    S->icd_launches++;
    return 0;
}

// NHICD selection of schedule 1 on the device, for the sweep of rotation
// `rot`: the VSC filter of the magnitude map, each plane's order statistic
// and selected lines, and the sweep's order compacted to the super-voxels
// holding a selected line (the others marked finished for the pass's epoch).
static int sv_nh_select(MbirStage *S, int rot)
{
    const int planes = S->sg.N_time * S->nzg;
    CK(mbir_launch_vsc_filter(S->d_mag, S->d_filt, planes, S->st.N_y, S->st.N_x, S->stream));
    CK(mbir_launch_vsc_threshold(S->d_filt, planes, (int)S->nxy(), S->d_nh_nsel, S->d_nh_thresh, S->d_nh_sel,
                                 S->d_nh_count, S->stream));
    const auto &m = S->sv_rot[rot];
    CK(mbir_launch_sv_nh_list(S->d_sv_lists + m[1], (int)m[0], S->d_sv_all, S->sp.S, S->st.N_x, S->st.N_y,
                              S->d_nh_sel, S->d_mask, S->sv_epoch + 1, S->d_sv_done, S->d_nh_pos, S->d_nh_nt,
                              S->stream));
    S->launches += 3;
    return 0;
}

// One outer iteration of the super-voxel schedule: a sweep over every SV in
// one launch, colour phase by colour phase (the phase order rotates with the
// iteration; an SV starts as soon as the conflicting SVs before it have
// finished), a ring-offset update, then (from the second iteration) a
// non-homogeneous pass over the SVs whose lines changed most in the sweep,
// another ring-offset update, and the variance update.  Convergence uses the
// reference's criterion, with the ratio of summed |dx| to summed |x'| over
// the sweep scaled by its 10 sub-iterations (XT_ICD_update.c:1066-1103).
static int sv_iterate(MbirStage *S, int iter, int32_t *converged)
{
    const int P = S->sv_nphase;
    // the state at the start of a window of iterations, for the stability
    // guard below
    const size_t nsino = S->nsino(), nvox = S->nvox(), noff = (size_t)S->sg.N_t * S->sg.N_r;
    const int grid_now = S->sv_ctas > 0 ? std::min(S->sv_ctas, S->sv_fit) : S->sv_grid;
    const bool adjustable = S->guard && grid_now > 1;
    if (adjustable && !S->win_open) {
        if (!S->d_snap_x) {
            CK(dalloc(&S->d_snap_x, nvox));
            CK(dalloc(&S->d_snap_e, nsino));
            CK(dalloc(&S->d_snap_w, nsino));
            CK(dalloc(&S->d_snap_d, noff));
        }
        if (!S->have_cost) {
            if (mbir_compute_cost(S, &S->prev_cost, nullptr, nullptr)) return -1;
            S->have_cost = true;
        }
        CK(cudaMemcpyAsync(S->d_snap_x, S->d_x, nvox * sizeof(float), cudaMemcpyDeviceToDevice, S->stream));
        CK(cudaMemcpyAsync(S->d_snap_e, S->d_e, nsino * sizeof(float), cudaMemcpyDeviceToDevice, S->stream));
        CK(cudaMemcpyAsync(S->d_snap_w, S->d_w, nsino * sizeof(float), cudaMemcpyDeviceToDevice, S->stream));
        CK(cudaMemcpyAsync(S->d_snap_d, S->d_d, noff * sizeof(float), cudaMemcpyDeviceToDevice, S->stream));
        S->snap_var = S->var_est;
        S->win_open = true;
        S->win_iters = 0;
    }
    if (S->d_acol && !S->acol_built) {
        CK(mbir_build_acache(S->g, S->dv, S->sp.amax, S->sp.eq, S->acol_half, S->d_acol, S->d_err, S->stream));
        S->acol_built = true;
        S->launches++;
    }
    // queue counters: slot 0 the sweep, slot 1 the NHICD pass
    CK(cudaMemsetAsync(S->d_queue, 0, 2 * sizeof(int), S->stream));
    if (S->debug_skip > 0) {
        CK(cudaMemcpyAsync(S->d_queue, &S->debug_skip, sizeof(int), cudaMemcpyHostToDevice, S->stream));
        CK(cudaStreamSynchronize(S->stream));
        S->debug_skip = 0;
    }
    CK(cudaMemsetAsync(S->d_sv_out, 0, 2 * sizeof(SvTaskOut), S->stream));
    const int rot = iter % P;
    // the sweep: one launch over every super-voxel, then the ring offsets
    const uint32_t sweep_seed = (uint32_t)(S->rng.next() * 4294967295.0);
    CK(cudaEventRecord(S->sv_ev[0], S->stream));
    if (sv_launch(S, S->d_sv_lists, S->sv_rot[rot], iter, sweep_seed, 0, S->d_sv_out)) return -1;
    CK(cudaEventRecord(S->sv_ev[1], S->stream));
    if (S->upd_offset > 1 && offset_update_async(S)) return -1;
    bool nh = false;
    if (iter > 1 && S->nh_fraction > 0) {
        // non-homogeneous pass over the lines the sweep changed most
        // (VSC_based_Voxel_Line_Select, XT_NHICD.c:164-216), chosen on the device
        if (sv_nh_select(S, rot)) return -1;
        nh = true;
        CK(cudaEventRecord(S->sv_ev[2], S->stream));
        if (sv_launch(S, S->d_sv_lists, S->sv_rot[rot], iter, (uint32_t)(S->rng.next() * 4294967295.0), 1,
                      S->d_sv_out + 1, true))
            return -1;
        CK(cudaEventRecord(S->sv_ev[3], S->stream));
        if (S->upd_offset > 1 && offset_update_async(S)) return -1;
    }
    if (S->upd_var == 1 && mbir_update_variance_parameter(S)) return -1;
    SvTaskOut acc[2];
    int err = 0;
    CK(cudaMemcpyAsync(acc, S->d_sv_out, sizeof(acc), cudaMemcpyDeviceToHost, S->stream));
    CK(cudaMemcpyAsync(&err, S->d_err, sizeof(int), cudaMemcpyDeviceToHost, S->stream));
    CK(cudaStreamSynchronize(S->stream));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, S->sv_ev[0], S->sv_ev[1]));
    S->icd_ms += ms;
    if (nh) {
        CK(cudaEventElapsedTime(&ms, S->sv_ev[2], S->sv_ev[3]));
        S->icd_ms += ms;
    }
    if (err & 1) return fail("super-voxel band overflow (A-matrix column outside the staged band)");
    if (err & 2) return fail("A-matrix column wider than 2 mult_xy + 1 detector columns");
    if (err & 4) return fail("super-voxel dependency wait timed out");
    if (err & 16) return fail("ring-offset constraint system is not positive definite");
    // Stability guard.  Super-voxels in flight together over-correct the
    // rays they share; the in-flight cap bounds that for the geometries it
    // was measured on.  Every step of an iteration (the voxel updates with
    // over-relaxation below 2, the offset and variance updates) lowers the
    // MAP cost, so a cost that rose by more than 1e-6 of its value over a
    // window of iterations means the super-voxels in flight diverged: the
    // state at the window's start is restored and this iteration redone with
    // half as many in flight.  The first four windows are one iteration long
    // (divergence from a poor start shows at once), later ones eight (one
    // FP64 cost evaluation per eight iterations).  mbir_set_sv_guard turns
    // it off.
    // summed over the slabs (XT_ICD_update.c:1079-1081)
    double sums[2] = {acc[0].sum_abs_dx, acc[0].sum_abs_x};
    if (slab_sum(S, sums, 2)) return -1;
    const double ax = sums[1];
    const double pct = ax > 0 ? 100.0 * S->K * sums[0] / ax : 0.0;
    if (adjustable && S->win_open && ++S->win_iters >= (S->guard_checks < 4 ? 1 : 8)) {
        double c = 0;
        if (mbir_compute_cost(S, &c, nullptr, nullptr)) return -1;
        S->guard_checks++;
        if (!(c - S->prev_cost <= 1e-6 * std::fabs(S->prev_cost))) {
            CK(cudaMemcpyAsync(S->d_x, S->d_snap_x, nvox * sizeof(float), cudaMemcpyDeviceToDevice, S->stream));
            CK(cudaMemcpyAsync(S->d_e, S->d_snap_e, nsino * sizeof(float), cudaMemcpyDeviceToDevice, S->stream));
            CK(cudaMemcpyAsync(S->d_w, S->d_snap_w, nsino * sizeof(float), cudaMemcpyDeviceToDevice, S->stream));
            CK(cudaMemcpyAsync(S->d_d, S->d_snap_d, noff * sizeof(float), cudaMemcpyDeviceToDevice, S->stream));
            S->var_est = S->snap_var;
            if (S->sv_ctas > 0)
                S->sv_ctas = std::max(1, grid_now / 2);
            else
                S->sv_grid = std::max(1, S->sv_grid / 2);
            S->stab_events++;
            S->win_iters = 0;  // the snapshot is the current state again
            S->guard_checks = 0;
            return sv_iterate(S, iter, converged);
        }
        S->prev_cost = c;
        S->win_open = false;
    }
    for (int q = 0; q < (nh ? 2 : 1); q++) {
        S->updates += acc[q].updates;
        S->zero_skips += acc[q].zero_skips;
    }
    S->last_pct = pct;
    *converged = S->last_pct < S->stop_thresh ? 1 : 0;
    return 0;
}

extern "C" int mbir_update_voxels_time_slices(MbirStage *S, int32_t iter, int32_t *converged)
{
    if (!S->prepared) return fail("mbir_icd_prepare has not run");
    if (S->schedule == 1) return sv_iterate(S, iter, converged);
    if (random_select(S)) return -1;
    double vox = 0;
    for (int j = 0; j < S->K; j++) {
        vox = 0;
        if (run_half(S, j, 0, 0, iter, &vox)) return -1;
        if (S->upd_offset > 1 && mbir_update_sinogram_offset(S)) return -1;
        if (run_half(S, j, 1, 0, iter, &vox)) return -1;
        if (S->upd_offset > 1 && mbir_update_sinogram_offset(S)) return -1;
        if (vsc_select(S)) return -1;
        if (iter > 1) {
            double unused = 0;
            if (run_half(S, j, 0, 1, iter, &unused)) return -1;
            if (S->upd_offset > 1 && mbir_update_sinogram_offset(S)) return -1;
            if (run_half(S, j, 1, 1, iter, &unused)) return -1;
            if (S->upd_offset > 1 && mbir_update_sinogram_offset(S)) return -1;
        }
    }
    if (S->upd_var == 1 && mbir_update_variance_parameter(S)) return -1;
    // convergence (XT_ICD_update.c:1066-1103): summed last-visit magnitudes of
    // the HICD lines over the summed |x'| of the last sub-iteration's HICD updates
    std::vector<float> mag(S->nmag());
    std::vector<int> xs(S->nmag()), ys(S->nmag());
    CK(cudaMemcpy(mag.data(), S->d_mag, mag.size() * sizeof(float), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(xs.data(), S->d_xr, xs.size() * sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(ys.data(), S->d_yr, ys.size() * sizeof(int), cudaMemcpyDeviceToHost));
    double avg = 0;
    const size_t nxy = S->nxy();
    for (int pl = 0; pl < S->sg.N_time * S->nblk; pl++)
        for (int q = 0; q < S->nr[pl]; q++)
            avg += mag[(size_t)pl * nxy + (size_t)ys[(size_t)pl * nxy + q] * S->st.N_x + xs[(size_t)pl * nxy + q]];
    double sums[2] = {avg, vox};
    if (slab_sum(S, sums, 2)) return -1;
    S->last_pct = 100 * sums[0] / sums[1];
    *converged = S->last_pct < S->stop_thresh ? 1 : 0;
    return 0;
}

// MAP cost (computeCost, XT_ICD_update.c:186-319) in FP64.
extern "C" int mbir_compute_cost(MbirStage *S, double *total, double *forward, double *prior)
{
    CK(mbir_launch_cost(S->g, S->pr, S->dv, S->d_partials, S->nparts, S->d_result, S->stream));
    S->launches += 2;
    double r[2];
    CK(cudaMemcpyAsync(r, S->d_result, sizeof(r), cudaMemcpyDeviceToHost, S->stream));
    CK(cudaStreamSynchronize(S->stream));
    // data and prior terms summed over the slabs (XT_ICD_update.c:301-317)
    if (slab_sum(S, r, 2)) return -1;
    const double data = r[0] / 2.0;
    const double fw = data + (double)S->slab_count * (double)S->sg.N_p * (double)S->sg.N_r * (double)S->sg.N_t *
                                 log(S->var_est) / 2;
    if (forward) *forward = fw;
    if (prior) *prior = r[1];
    if (total) *total = fw + r[1];
    return 0;
}

// ---------------------------------------------------------------------------
// State access
// ---------------------------------------------------------------------------
extern "C" int mbir_stage_dims(MbirStage *S, int32_t *d)
{
    d[0] = S->sg.N_p; d[1] = S->sg.N_r; d[2] = S->sg.N_t; d[3] = S->st.N_x; d[4] = S->st.N_y;
    d[5] = S->st.N_z; d[6] = S->sg.N_time; d[7] = S->nblk; d[8] = S->st.m_z;
    return 0;
}

extern "C" int mbir_get_object(MbirStage *S, float *out)
{
    CK(cudaMemcpy(out, S->d_x, S->nvox() * sizeof(float), cudaMemcpyDeviceToHost));
    return 0;
}

extern "C" int mbir_set_object(MbirStage *S, const float *in)
{
    CK(cudaMemcpy(S->d_x, in, S->nvox() * sizeof(float), cudaMemcpyHostToDevice));
    return 0;
}

// Sinogram-shaped arrays come back in the reference's [view][col][row] layout.
static int get_sino(MbirStage *S, const float *dev, float *out)
{
    const ScanGeom &sg = S->sg;
    std::vector<float> tmp(S->nsino());
    CK(cudaMemcpy(tmp.data(), dev, tmp.size() * sizeof(float), cudaMemcpyDeviceToHost));
    for (int t = 0; t < sg.N_t; t++)
        for (int p = 0; p < sg.N_p; p++)
            for (int r = 0; r < sg.N_r; r++)
                out[((size_t)p * sg.N_r + r) * sg.N_t + t] = tmp[((size_t)t * sg.N_p + p) * sg.N_r + r];
    return 0;
}

extern "C" int mbir_get_errorsino(MbirStage *S, float *out) { return get_sino(S, S->d_e, out); }
extern "C" int mbir_get_weight(MbirStage *S, float *out) { return get_sino(S, S->d_w, out); }

extern "C" int mbir_get_offset(MbirStage *S, float *out)
{
    const ScanGeom &sg = S->sg;
    std::vector<float> d((size_t)sg.N_t * sg.N_r);
    CK(cudaMemcpy(d.data(), S->d_d, d.size() * sizeof(float), cudaMemcpyDeviceToHost));
    for (int r = 0; r < sg.N_r; r++)
        for (int t = 0; t < sg.N_t; t++) out[(size_t)r * sg.N_t + t] = d[(size_t)t * sg.N_r + r];
    return 0;
}

extern "C" int mbir_get_magmap(MbirStage *S, float *out)
{
    CK(cudaMemcpy(out, S->d_mag, S->nmag() * sizeof(float), cudaMemcpyDeviceToHost));
    return 0;
}

extern "C" int mbir_get_hr(MbirStage *S, float *out)
{
    if (!S->hr_ready && compute_detector_response(S)) return -1;
    CK(cudaMemcpy(out, S->d_H, (size_t)S->sg.N_p * (MBIR_RESP_BINS + 1) * sizeof(float), cudaMemcpyDeviceToHost));
    return 0;
}

extern "C" int mbir_get_mask(MbirStage *S, uint8_t *out)
{
    std::copy(S->mask.begin(), S->mask.end(), out);
    return 0;
}

extern "C" int mbir_get_lines(MbirStage *S, int32_t kind, int32_t frame, int32_t block, int32_t *xs,
                              int32_t *ys)
{
    const size_t plane = (size_t)frame * S->nblk + block;
    const int n = kind == 0 ? S->nr[plane] : S->nn[plane];
    const int *dx = (kind == 0 ? S->d_xr : S->d_xn) + plane * S->nxy();
    const int *dy = (kind == 0 ? S->d_yr : S->d_yn) + plane * S->nxy();
    if (n > 0) {
        CK(cudaMemcpy(xs, dx, n * sizeof(int), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(ys, dy, n * sizeof(int), cudaMemcpyDeviceToHost));
    }
    return n;
}

extern "C" double mbir_get_var_est(MbirStage *S) { return S->var_est; }
extern "C" double mbir_get_update_percentage(MbirStage *S) { return S->last_pct; }
extern "C" long long mbir_get_update_count(MbirStage *S) { return S->updates; }

// Device-side clock around a span of stage calls: events recorded on the
// stage's stream (all stage calls are synchronous, so the span covers them).
extern "C" int mbir_time_begin(MbirStage *S)
{
    CK(cudaStreamSynchronize(S->stream));
    CK(cudaEventRecord(S->tev0, S->stream));
    return 0;
}

extern "C" int mbir_time_end(MbirStage *S, double *ms)
{
    CK(cudaEventRecord(S->tev1, S->stream));
    CK(cudaEventSynchronize(S->tev1));
    float f = 0;
    CK(cudaEventElapsedTime(&f, S->tev0, S->tev1));
    *ms = f;
    return 0;
}

// Device time of the ICD update kernels (CUDA events on the stage's stream)
// and the number of kernels this stage has launched.
extern "C" int mbir_get_kernel_stats(MbirStage *S, double *icd_ms, long long *icd_launches,
                                     long long *launches)
{
    if (icd_ms) *icd_ms = S->icd_ms;
    if (icd_launches) *icd_launches = S->icd_launches;
    if (launches) *launches = S->launches;
    return 0;
}

// Filtered backprojection of the stage's projections, frame by frame, into
// out [N_time][N_z][N_y][N_x] (host); zero outside the reconstruction mask.
extern "C" int mbir_fbp(MbirStage *S, float *out)
{
    if (S->mask.empty()) object_mask(S->sg, S->st, S->mask);
    CK(cudaMemcpyAsync(S->d_mask, S->mask.data(), S->mask.size(), cudaMemcpyHostToDevice, S->stream));
    float *q = nullptr, *x = nullptr;
    CK(dalloc(&q, S->nsino()));
    CK(dalloc(&x, S->nvox()));
    cudaError_t e = mbir_launch_fbp(S->g, S->d_mask, S->d_y, q, x, S->stream);
    S->launches += 2;
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, x, S->nvox() * sizeof(float), cudaMemcpyDeviceToHost, S->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(S->stream);
    dfree(q);
    dfree(x);
    CK(e);
    return 0;
}

// Forward projection A x of an object [N_time][N_z][N_y][N_x] into a
// sinogram [view][row][col] (the layout reconstruct() takes), with this
// stage's geometry.  Used to synthesise scans of voxelised phantoms.
extern "C" int mbir_forward_project(MbirStage *S, const float *object, float *out)
{
    if (!S->hr_ready && compute_detector_response(S)) return -1;
    CK(cudaMemcpy(S->d_x, object, S->nvox() * sizeof(float), cudaMemcpyHostToDevice));
    CK(mbir_forward_rows(S->g, S->d_fov, S->d_x, nullptr, nullptr, S->d_e, 1, S->amax(), S->stream));
    S->launches++;
    CK(cudaStreamSynchronize(S->stream));
    const ScanGeom &sg = S->sg;
    std::vector<float> tmp(S->nsino());
    CK(cudaMemcpy(tmp.data(), S->d_e, tmp.size() * sizeof(float), cudaMemcpyDeviceToHost));
    for (int t = 0; t < sg.N_t; t++)
        for (int p = 0; p < sg.N_p; p++)
            for (int r = 0; r < sg.N_r; r++)
                out[((size_t)p * sg.N_t + t) * sg.N_r + r] = tmp[((size_t)t * sg.N_p + p) * sg.N_r + r];
    return 0;
}

// ---------------------------------------------------------------------------
// Batched super-voxel ICD: independent problems (stages) in one persistent
// launch per iteration, each iteration one replay of a captured CUDA graph
// ---------------------------------------------------------------------------
struct MbirBatch {
    std::vector<MbirStage *> stages;
    int n = 0, ctas = 1, nrot = 1, ntasks = 0;
    bool half = false;
    size_t smem = 0;  // shared memory per CTA: the largest problem's plan
    size_t scratch_floats = 0;
    cudaStream_t stream = nullptr;
    SvProblem *d_probs = nullptr;
    SvBatchState *d_state = nullptr;
    SvTask *d_tasks = nullptr;
    int *d_lists = nullptr, *d_done = nullptr, *d_queue = nullptr, *d_err = nullptr, *d_ctl = nullptr;
    float *d_scratch = nullptr;
    int *h_ctl = nullptr;  // pinned copy of the control words
    std::vector<cudaGraphExec_t> graphs;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double ms = 0;
    long long replays = 0;
    std::vector<long long> seen;  // updates already added to each stage's count
    // stability guard per problem, as the single stage's (sv_iterate): the
    // problem's state at the start of its current window of iterations and
    // the MAP cost there; a cost that rose restores that state and halves
    // the problem's super-voxels in flight
    struct Guard {
        float *x = nullptr, *e = nullptr;
        double cost = 0;
        int win = 0, checks = 0, last_iters = 0, cap = 1;
        long long upd = 0, zs = 0;
    };
    bool guard = false;
    std::vector<Guard> gd;
    // NHICD passes (stages with a non-zero mbir_set_sv_nhicd fraction): each
    // problem's iteration count when its last pass ran, and the event that
    // orders a pass after the batched sweep
    std::vector<int> nh_iters;
    cudaEvent_t ev_sweep = nullptr;
    ~MbirBatch()
    {
        if (stream) cudaStreamSynchronize(stream);
        if (ev_sweep) cudaEventDestroy(ev_sweep);
        for (auto g : graphs) cudaGraphExecDestroy(g);
        void *bufs[] = {d_probs, d_state, d_tasks, d_lists, d_done, d_queue, d_err, d_ctl, d_scratch};
        for (void *b : bufs) dfree(b);
        for (auto &g : gd) {
            dfree(g.x);
            dfree(g.e);
        }
        if (h_ctl) cudaFreeHost(h_ctl);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }
};

// Launch lists of a batch for phase rotation r, appended to buf as
// [order | dep_off | deps | seq]: each problem's full sweep in its own order
// (its colour phases from phase r), the problems interleaved in proportion
// to their super-voxel counts so that they all advance together; deps are
// the conflicting super-voxels of the same problem earlier in the list, seq
// the position in the problem's own order.
static void batch_build_list(const std::vector<MbirStage *> &st, const std::vector<int> &base, int r,
                             std::vector<int> &buf, std::array<size_t, 5> &meta)
{
    struct Ent {
        double key;
        int prob, k;
    };
    std::vector<std::vector<int>> ids(st.size());
    std::vector<Ent> all;
    for (size_t p = 0; p < st.size(); p++) {
        const MbirStage *S = st[p];
        ids[p].resize(S->sv_all.size());
        for (size_t q = 0; q < ids[p].size(); q++) ids[p][q] = (int)q;
        sv_sort(S, ids[p], r % std::max(1, S->sv_nphase));
        const double n = (double)ids[p].size();
        for (size_t k = 0; k < ids[p].size(); k++) all.push_back({(k + 0.5) / n, (int)p, (int)k});
    }
    std::stable_sort(all.begin(), all.end(), [](const Ent &a, const Ent &b) { return a.key < b.key; });
    const size_t n = all.size();
    meta[0] = n;
    meta[1] = buf.size();
    for (const Ent &e : all) buf.push_back(base[e.prob] + ids[e.prob][e.k]);
    // position of each local id in its problem's order
    std::vector<std::vector<int>> pos(st.size());
    for (size_t p = 0; p < st.size(); p++) {
        pos[p].assign(ids[p].size(), -1);
        for (size_t k = 0; k < ids[p].size(); k++) pos[p][ids[p][k]] = (int)k;
    }
    meta[2] = buf.size();
    buf.resize(buf.size() + n + 1);
    std::vector<int> deps;
    for (size_t t = 0; t < n; t++) {
        const Ent &e = all[t];
        buf[meta[2] + t] = (int)deps.size();
        const int id = ids[e.prob][e.k];
        for (int nb : st[e.prob]->sv_nbr[id])
            if (pos[e.prob][nb] < e.k) deps.push_back(base[e.prob] + nb);
    }
    buf[meta[2] + n] = (int)deps.size();
    meta[3] = buf.size();
    buf.insert(buf.end(), deps.begin(), deps.end());
    meta[4] = buf.size();
    for (const Ent &e : all) buf.push_back(e.k);
}

// MAP cost of a batch problem (as mbir_compute_cost), on the batch's stream.
static int batch_cost(MbirBatch *B, int p, double *total)
{
    MbirStage *S = B->stages[p];
    CK(mbir_launch_cost(S->g, S->pr, S->dv, S->d_partials, S->nparts, S->d_result, B->stream));
    double r[2];
    CK(cudaMemcpyAsync(r, S->d_result, sizeof(r), cudaMemcpyDeviceToHost, B->stream));
    CK(cudaStreamSynchronize(B->stream));
    *total = r[0] / 2.0 + (double)S->sg.N_p * (double)S->sg.N_r * (double)S->sg.N_t * log(S->var_est) / 2 + r[1];
    return 0;
}

// The guard's snapshot of problem p: object and error sinogram, cost (given,
// or evaluated when cost is null), counts.
static int batch_snapshot(MbirBatch *B, int p, const SvBatchState &st, const double *cost = nullptr)
{
    MbirStage *S = B->stages[p];
    MbirBatch::Guard &g = B->gd[p];
    if (!g.x) {
        CK(dalloc(&g.x, S->nvox()));
        CK(dalloc(&g.e, S->nsino()));
    }
    CK(cudaMemcpyAsync(g.x, S->d_x, S->nvox() * sizeof(float), cudaMemcpyDeviceToDevice, B->stream));
    CK(cudaMemcpyAsync(g.e, S->d_e, S->nsino() * sizeof(float), cudaMemcpyDeviceToDevice, B->stream));
    if (cost)
        g.cost = *cost;
    else if (batch_cost(B, p, &g.cost))
        return -1;
    g.upd = st.updates;
    g.zs = st.zero_skips;
    g.win = 0;
    return 0;
}

extern "C" int mbir_batch_create(MbirBatch **out, MbirStage *const *stages, int32_t n, int32_t uncapped)
{
    *out = nullptr;
    if (n <= 0) return fail("a batch needs at least one stage");
    auto B = std::make_unique<MbirBatch>();
    B->stages.assign(stages, stages + n);
    B->n = n;
    for (int p = 0; p < n; p++) {
        MbirStage *S = B->stages[p];
        if (!S->prepared) return fail("batch problem %d: mbir_icd_prepare has not run", p);
        if (S->schedule != 1 || !S->d_acol)
            return fail("batch problem %d: the super-voxel schedule with a column cache is required", p);
        if (S->upd_offset > 1 || S->upd_var == 1)
            return fail("batch problem %d: batched iterations run plain ICD (no ring-offset or variance update)", p);
        if (S->slab_count > 1)
            return fail("batch problem %d: a z-slab of a sharded volume (its sums reduce over ranks)", p);
        const SvParams &sp = S->sp;
        const int vpl = (sp.max_views + 32 * sp.vsplit - 1) / (32 * sp.vsplit);
        if (sp.amax != 3 || S->st.m_z != 1 || vpl > kSvBatchViewsPerLane ||
            32 * sp.max_nz * sp.vsplit > kSvBatchThreads)
            return fail("batch problem %d: needs 3 detector columns per entry, one row per slice, at most %d views "
                        "per lane and %d threads per super-voxel (%d columns, %d rows, %d views per lane, %d "
                        "threads)",
                        p, kSvBatchViewsPerLane, kSvBatchThreads, sp.amax, S->st.m_z, vpl,
                        32 * sp.max_nz * sp.vsplit);
        if (p > 0 && S->acol_half != B->half) return fail("batch problem %d: mixed FP32 and FP16 column caches", p);
        B->half = S->acol_half;
        if (!S->acol_built) {
            CK(mbir_build_acache(S->g, S->dv, sp.amax, sp.eq, S->acol_half, S->d_acol, S->d_err, S->stream));
            S->acol_built = true;
            S->launches++;
        }
        CK(cudaStreamSynchronize(S->stream));
        B->smem = std::max(B->smem, mbir_sv_plan_bytes(mbir_sv_plan(sp, true)));
        B->scratch_floats = std::max(B->scratch_floats, sp.band_floats);
    }
    if (B->smem > kSmemLimit) return fail("a batch problem needs %zu bytes of shared memory", B->smem);
    // problems, tasks, launch lists
    std::vector<SvProblem> probs(n);
    std::vector<SvTask> tasks;
    std::vector<int> base(n);
    for (int p = 0; p < n; p++) {
        MbirStage *S = B->stages[p];
        SvProblem &P = probs[p];
        P.g = S->g;
        P.pr = S->pr;
        P.pr.alpha = S->sv_alpha_eff;
        P.dv = S->dv;
        P.sp = S->sp;
        P.ac = SvACache{S->d_acol};
        P.plan = mbir_sv_plan(S->sp, true);
        P.cap = uncapped ? (1 << 30) : std::max(1, S->sv_grid);
        P.K = S->K;
        P.stop = S->stop_thresh;
        base[p] = (int)tasks.size();
        for (SvTask t : S->sv_all) {
            t.prob = p;
            tasks.push_back(t);
        }
        B->nrot = std::max(B->nrot, S->sv_nphase);
    }
    B->ntasks = (int)tasks.size();
    if (B->ntasks == 0) return fail("the batch has no super-voxels");
    std::vector<int> buf;
    std::vector<std::array<size_t, 5>> meta(B->nrot);
    for (int r = 0; r < B->nrot; r++) batch_build_list(B->stages, base, r, buf, meta[r]);
    CK(cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking));
    CK(cudaEventCreate(&B->ev0));
    CK(cudaEventCreate(&B->ev1));
    int dev = 0, sms = 148;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    B->ctas = std::max(1, std::min(B->ntasks, mbir_sv_batch_ctas_per_sm(B->smem, B->half) * sms));
    CK(dalloc(&B->d_probs, n));
    CK(dalloc(&B->d_state, n));
    CK(dalloc(&B->d_tasks, tasks.size()));
    CK(dalloc(&B->d_lists, buf.size()));
    CK(dalloc(&B->d_done, tasks.size()));
    CK(dalloc(&B->d_queue, 1));
    CK(dalloc(&B->d_err, 1));
    CK(dalloc(&B->d_ctl, 4));
    CK(dalloc(&B->d_scratch, (size_t)B->ctas * B->scratch_floats));
    CK(cudaMallocHost(&B->h_ctl, 4 * sizeof(int)));
    std::vector<SvBatchState> state(n);
    for (auto &s : state) s.active = 1;
    const int ctl[4] = {1, n, 0, 0};
    CK(cudaMemcpyAsync(B->d_probs, probs.data(), n * sizeof(SvProblem), cudaMemcpyHostToDevice, B->stream));
    CK(cudaMemcpyAsync(B->d_state, state.data(), n * sizeof(SvBatchState), cudaMemcpyHostToDevice, B->stream));
    CK(cudaMemcpyAsync(B->d_tasks, tasks.data(), tasks.size() * sizeof(SvTask), cudaMemcpyHostToDevice, B->stream));
    CK(cudaMemcpyAsync(B->d_lists, buf.data(), buf.size() * sizeof(int), cudaMemcpyHostToDevice, B->stream));
    CK(cudaMemcpyAsync(B->d_ctl, ctl, sizeof(ctl), cudaMemcpyHostToDevice, B->stream));
    CK(cudaMemsetAsync(B->d_done, 0, tasks.size() * sizeof(int), B->stream));
    CK(cudaMemsetAsync(B->d_queue, 0, sizeof(int), B->stream));
    CK(cudaMemsetAsync(B->d_err, 0, sizeof(int), B->stream));
    CK(cudaStreamSynchronize(B->stream));
    B->seen.assign(n, 0);
    // the stability guard (not for the autotuner's uncapped timing runs)
    B->guard = !uncapped;
    B->gd.assign(n, MbirBatch::Guard{});
    if (B->guard)
        for (int p = 0; p < n; p++) {
            B->gd[p].cap = probs[p].cap;
            if (batch_snapshot(B.get(), p, state[p])) return -1;
        }
    // one graph per phase rotation: the sweep, then the end of the iteration
    CK(mbir_sv_batch_prepare(B->smem, B->half));
    for (int r = 0; r < B->nrot; r++) {
        SvLaunch L{B->d_tasks, B->d_lists + meta[r][1], B->d_lists + meta[r][2], B->d_lists + meta[r][3],
                   (int)meta[r][0], B->d_done, 0, B->d_probs, B->d_lists + meta[r][4], B->d_state, B->d_ctl};
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e1 = mbir_launch_icd_sv_batch(B->smem, B->half, L, B->ctas, B->d_queue, B->d_scratch,
                                                  B->scratch_floats, 0x2545F491u + 977u * r, B->d_err, B->stream);
        cudaError_t e2 = mbir_launch_sv_batch_end(B->d_probs, B->d_state, n, B->d_ctl, B->d_queue, B->stream);
        cudaError_t e3 = cudaStreamEndCapture(B->stream, &g);
        CK(e1);
        CK(e2);
        CK(e3);
        cudaGraphExec_t ge = nullptr;
        cudaError_t e4 = cudaGraphInstantiate(&ge, g, 0);
        cudaGraphDestroy(g);
        CK(e4);
        B->graphs.push_back(ge);
    }
    *out = B.release();
    return 0;
}

extern "C" void mbir_batch_free(MbirBatch *B) { delete B; }

// After a batched iteration: for every problem that iterated and whose
// window is due (one iteration for its first four checks, then eight, or
// when it has just passed the convergence test), the MAP cost against the
// window's start.  Every step of a problem's iteration lowers its cost, so a
// rise of more than 1e-6 of it means its super-voxels in flight diverged: its
// state and counts at the window's start are restored, it is set iterating
// again, and its in-flight cap halves.
static int batch_guard(MbirBatch *B)
{
    std::vector<SvBatchState> st(B->n);
    CK(cudaMemcpyAsync(st.data(), B->d_state, B->n * sizeof(SvBatchState), cudaMemcpyDeviceToHost, B->stream));
    CK(cudaStreamSynchronize(B->stream));
    bool reactivated = false;
    for (int p = 0; p < B->n; p++) {
        MbirBatch::Guard &g = B->gd[p];
        if (st[p].iters == g.last_iters) continue;  // not iterating
        g.last_iters = st[p].iters;
        if (++g.win < (g.checks < 4 ? 1 : 8) && !st[p].converged) continue;
        double c = 0;
        if (batch_cost(B, p, &c)) return -1;
        MbirStage *S = B->stages[p];
        if (!(c - g.cost <= 1e-6 * std::fabs(g.cost))) {
            CK(cudaMemcpyAsync(S->d_x, g.x, S->nvox() * sizeof(float), cudaMemcpyDeviceToDevice, B->stream));
            CK(cudaMemcpyAsync(S->d_e, g.e, S->nsino() * sizeof(float), cudaMemcpyDeviceToDevice, B->stream));
            g.cap = std::max(1, g.cap / 2);
            CK(cudaMemcpyAsync(reinterpret_cast<char *>(B->d_probs + p) + offsetof(SvProblem, cap), &g.cap,
                               sizeof(int), cudaMemcpyHostToDevice, B->stream));
            reactivated |= !st[p].active;
            st[p].updates = g.upd;
            st[p].zero_skips = g.zs;
            st[p].active = 1;
            st[p].converged = 0;
            st[p].prev_ax = 0;
            st[p].adjustments++;
            CK(cudaMemcpyAsync(B->d_state + p, &st[p], sizeof(SvBatchState), cudaMemcpyHostToDevice, B->stream));
            CK(cudaStreamSynchronize(B->stream));
            S->stab_events++;
            g.win = 0;
            g.checks = 0;
        } else {
            if (batch_snapshot(B, p, st[p], &c)) return -1;
            g.checks++;
        }
    }
    if (reactivated) {  // the control word counts the problems iterating
        int act = 0;
        for (auto &x : st) act += x.active;
        CK(cudaMemcpyAsync(B->d_ctl + 1, &act, sizeof(int), cudaMemcpyHostToDevice, B->stream));
        CK(cudaStreamSynchronize(B->stream));
    }
    return 0;
}

// NHICD pass of every problem that iterated in the replay just launched
// (phase rotation r), from its second iteration, when its stage's NHICD
// fraction is non-zero: the stage's own device selection and subset launch,
// as its single-problem iteration runs them (VSC_based_Voxel_Line_Select,
// XT_NHICD.c:164-216, after the homogeneous sweep, XT_ICD_update.c:1010-1040),
// on the stage's stream after the batch's sweep; the pass's super-voxels in
// flight are capped as the batch caps the problem's.  The convergence test
// stays the sweep's, as in the reference (HICD lines only).
static int batch_nhicd(MbirBatch *B, int r)
{
    bool any = false;
    for (MbirStage *S : B->stages) any |= S->nh_fraction > 0;
    if (!any) return 0;
    if (!B->ev_sweep) CK(cudaEventCreateWithFlags(&B->ev_sweep, cudaEventDisableTiming));
    if (B->nh_iters.empty()) B->nh_iters.assign(B->n, 0);
    std::vector<SvBatchState> st(B->n);
    CK(cudaMemcpyAsync(st.data(), B->d_state, B->n * sizeof(SvBatchState), cudaMemcpyDeviceToHost, B->stream));
    CK(cudaEventRecord(B->ev_sweep, B->stream));
    CK(cudaStreamSynchronize(B->stream));
    std::vector<int> ran;
    for (int p = 0; p < B->n; p++) {
        MbirStage *S = B->stages[p];
        if (S->nh_fraction <= 0 || st[p].iters == B->nh_iters[p]) continue;  // not iterating in this replay
        B->nh_iters[p] = st[p].iters;
        if (st[p].iters < 2) continue;
        CK(cudaStreamWaitEvent(S->stream, B->ev_sweep, 0));
        CK(cudaMemsetAsync(S->d_queue + 1, 0, sizeof(int), S->stream));
        CK(cudaMemsetAsync(S->d_sv_out + 1, 0, sizeof(SvTaskOut), S->stream));
        const int rot = r % std::max(1, S->sv_nphase);
        if (sv_nh_select(S, rot)) return -1;
        const int grid = S->sv_grid, ctas = S->sv_ctas;
        const int cap = B->guard ? B->gd[p].cap : grid;
        S->sv_ctas = 0;
        S->sv_grid = std::max(1, std::min(ctas > 0 ? std::min(ctas, S->sv_fit) : grid, cap));
        const int rc = sv_launch(S, S->d_sv_lists, S->sv_rot[rot], st[p].iters,
                                 (uint32_t)(S->rng.next() * 4294967295.0), 1, S->d_sv_out + 1, true);
        S->sv_grid = grid;
        S->sv_ctas = ctas;
        if (rc) return -1;
        ran.push_back(p);
    }
    for (int p : ran) {
        MbirStage *S = B->stages[p];
        SvTaskOut acc;
        int err = 0;
        CK(cudaMemcpyAsync(&acc, S->d_sv_out + 1, sizeof(acc), cudaMemcpyDeviceToHost, S->stream));
        CK(cudaMemcpyAsync(&err, S->d_err, sizeof(int), cudaMemcpyDeviceToHost, S->stream));
        CK(cudaStreamSynchronize(S->stream));
        if (err & 1) return fail("problem %d NHICD pass: super-voxel band overflow", p);
        if (err & 4) return fail("problem %d NHICD pass: super-voxel dependency wait timed out", p);
        if (err) return fail("problem %d NHICD pass: device error flags 0x%x", p, err);
        S->updates += acc.updates;
        S->zero_skips += acc.zero_skips;
    }
    return 0;
}

extern "C" int mbir_batch_iterate(MbirBatch *B, int32_t max_iters, int32_t check_every, int32_t *active_left)
{
    if (check_every <= 0) check_every = 1;
    CK(cudaEventRecord(B->ev0, B->stream));
    int left = B->n;
    for (int k = 0; k < max_iters; k++) {
        const int r = (int)(B->replays % B->nrot);
        CK(cudaGraphLaunch(B->graphs[r], B->stream));
        B->replays++;
        if (batch_nhicd(B, r)) return -1;
        if (B->guard && batch_guard(B)) return -1;
        if ((k + 1) % check_every == 0 || k + 1 == max_iters) {
            CK(cudaMemcpyAsync(B->h_ctl, B->d_ctl, 4 * sizeof(int), cudaMemcpyDeviceToHost, B->stream));
            CK(cudaStreamSynchronize(B->stream));
            left = B->h_ctl[1];
            if (left == 0) break;
        }
    }
    CK(cudaEventRecord(B->ev1, B->stream));
    CK(cudaEventSynchronize(B->ev1));
    float f = 0;
    CK(cudaEventElapsedTime(&f, B->ev0, B->ev1));
    B->ms += f;
    int err = 0;
    CK(cudaMemcpy(&err, B->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err & 1) return fail("super-voxel band overflow (A-matrix column outside the staged band)");
    if (err & 2) return fail("A-matrix column wider than 2 mult_xy + 1 detector columns");
    if (err & 4) return fail("super-voxel dependency wait timed out");
    if (err & 16) return fail("ring-offset constraint system is not positive definite");
    if (err & 8) return fail("super-voxel in-flight wait timed out");
    // the stages' own counters
    std::vector<SvBatchState> st(B->n);
    CK(cudaMemcpy(st.data(), B->d_state, B->n * sizeof(SvBatchState), cudaMemcpyDeviceToHost));
    for (int p = 0; p < B->n; p++) {
        MbirStage *S = B->stages[p];
        S->updates += st[p].updates - B->seen[p];
        B->seen[p] = st[p].updates;
        S->last_pct = st[p].pct;
    }
    if (active_left) *active_left = left;
    return 0;
}

// Per problem: iterations done, stopped by the convergence test, voxel
// updates, zero-skipped voxels, last convergence ratio (percent).  Any
// pointer may be null.
extern "C" int mbir_batch_stats(MbirBatch *B, int32_t *iters, int32_t *converged, int64_t *updates,
                                int64_t *zero_skips, double *pct)
{
    std::vector<SvBatchState> st(B->n);
    CK(cudaMemcpy(st.data(), B->d_state, B->n * sizeof(SvBatchState), cudaMemcpyDeviceToHost));
    for (int p = 0; p < B->n; p++) {
        if (iters) iters[p] = st[p].iters;
        if (converged) converged[p] = st[p].converged;
        if (updates) updates[p] = st[p].updates;
        if (zero_skips) zero_skips[p] = st[p].zero_skips;
        if (pct) pct[p] = st[p].pct;
    }
    return 0;
}

// Device time of the batch's iterations so far (CUDA events on its stream),
// graph replays, kernels launched (two per replay), persistent CTAs, shared
// memory per CTA.
extern "C" int mbir_batch_info(MbirBatch *B, double *ms, int64_t *replays, int64_t *launches, int32_t *ctas,
                               int64_t *smem_bytes)
{
    if (ms) *ms = B->ms;
    if (replays) *replays = B->replays;
    if (launches) *launches = 2 * B->replays;
    if (ctas) *ctas = B->ctas;
    if (smem_bytes) *smem_bytes = (int64_t)B->smem;
    return 0;
}

// Autotuner: times the batched kernel on this stage alone (no in-flight cap,
// every resident CTA busy) for super-voxel sides 4..8 and 1, 2 or 4 warps
// per slice (with the z-group filling 256 threads), two iterations after one
// warm-up from the stage's prepared state, and keeps the fastest per voxel
// update.  The object and error sinogram are restored afterwards and the
// magnitude map cleared; call after mbir_icd_prepare, before iterating.
extern "C" int mbir_autotune_stage(MbirStage *S, int32_t *side, int32_t *warps_per_slice, int32_t *zgroup,
                                   double *ns_per_update)
{
    if (!S->prepared) return fail("mbir_icd_prepare has not run");
    const int Nz = S->st.N_z;
    float *x0 = nullptr, *e0 = nullptr;
    CK(dalloc(&x0, S->nvox()));
    CK(dalloc(&e0, S->nsino()));
    auto release = [&]() {
        dfree(x0);
        dfree(e0);
    };
    CK(cudaMemcpyAsync(x0, S->d_x, S->nvox() * sizeof(float), cudaMemcpyDeviceToDevice, S->stream));
    CK(cudaMemcpyAsync(e0, S->d_e, S->nsino() * sizeof(float), cudaMemcpyDeviceToDevice, S->stream));
    auto restore = [&]() -> int {
        CK(cudaMemcpyAsync(S->d_x, x0, S->nvox() * sizeof(float), cudaMemcpyDeviceToDevice, S->stream));
        CK(cudaMemcpyAsync(S->d_e, e0, S->nsino() * sizeof(float), cudaMemcpyDeviceToDevice, S->stream));
        CK(cudaMemsetAsync(S->d_mag, 0, S->nmag() * sizeof(float), S->stream));
        CK(cudaStreamSynchronize(S->stream));
        return 0;
    };
    const int zg_saved = S->sv_zgroup;
    double best = 1e300;
    int bs = 0, bv = 0, bz = 0;
    const int warps = kSvBatchThreads / 32;
    for (int s = 4; s <= 8; s++)
        for (int v = 1; v <= 4; v *= 2) {
            const int nz = std::min(warps / v, Nz);
            S->sv_zgroup = nz;
            if (mbir_set_schedule(S, 1, s, v) != 0 || !S->d_acol) continue;
            const SvParams &sp = S->sp;
            if (sp.S != s || sp.vsplit != v || sp.max_nz != nz) continue;
            if (restore()) return release(), -1;
            MbirBatch *B = nullptr;
            if (mbir_batch_create(&B, &S, 1, 1) != 0) continue;
            int32_t left = 0;
            int rc = mbir_batch_iterate(B, 1, 1, &left);
            int64_t u0 = 0, u1 = 0;
            double ms0 = 0, ms1 = 0;
            if (!rc) {
                mbir_batch_stats(B, nullptr, nullptr, &u0, nullptr, nullptr);
                mbir_batch_info(B, &ms0, nullptr, nullptr, nullptr, nullptr);
                rc = mbir_batch_iterate(B, 2, 2, &left);
                mbir_batch_stats(B, nullptr, nullptr, &u1, nullptr, nullptr);
                mbir_batch_info(B, &ms1, nullptr, nullptr, nullptr, nullptr);
            }
            mbir_batch_free(B);
            if (rc) {
                S->sv_zgroup = zg_saved;
                release();
                return -1;
            }
            const double ns = u1 > u0 ? (ms1 - ms0) * 1e6 / (double)(u1 - u0) : 1e300;
            if (ns < best) {
                best = ns;
                bs = s;
                bv = v;
                bz = nz;
            }
        }
    if (!bs) {
        S->sv_zgroup = zg_saved;
        release();
        return fail("no super-voxel configuration of the batched kernel fits this stage");
    }
    S->sv_zgroup = bz;
    if (mbir_set_schedule(S, 1, bs, bv) != 0 || restore()) {
        release();
        return -1;
    }
    // the stage's counters exclude the trial iterations
    S->updates = 0;
    S->zero_skips = 0;
    release();
    *side = bs;
    *warps_per_slice = bv;
    *zgroup = bz;
    *ns_per_update = best;
    return 0;
}
