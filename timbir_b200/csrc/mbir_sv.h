// Super-voxel ICD kernel interface (mbir_sv.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "mbir_internal.h"

// A-column ring slots of the super-voxel kernel
constexpr int kSvRing = 4;

struct SvParams {
    int S;          // super-voxel side (voxel lines)
    int W;          // band width (detector columns per view)
    int amax;       // max A-matrix entries per (line, view): 2 mult_xy + 1
    int eq;         // 16-byte words per A-matrix column entry: ceil((1 + amax) / 4)
    int max_views;  // max views of any frame (shared-memory stride)
    int max_nz;     // slices per CTA
    int max_rows;   // detector rows per CTA: max_nz * m_z
    int vsplit;     // warps per slice (1, 2 or 4; > 1 needs max_nz <= 15)
    int prod_warps; // warps computing the next line's A-matrix column (0 with a column cache)
    int ring;       // A-column ring slots: kSvRing (the cache is read ring - 2 lines ahead)
    int ahalf;      // the column cache holds FP16 values (8-byte entries; full resolution)
    size_t band_floats;  // scratch floats per CTA: sv_scratch_floats()
};

// 16-byte words of e a super-voxel CTA keeps per (detector row, view) pair for
// its band commit: the words the staging loads, at 16-byte-aligned detector
// columns (a band of W columns starting anywhere in a word spans at most
// ceil((W + 3) / 4)), never fewer than the staging's four per pair.
__host__ __device__ inline int sv_scratch_words(int W) { return (W + 6) / 4 > 4 ? (W + 6) / 4 : 4; }
// Scratch floats per CTA: the per-element copy of e (rows x W x views, detector
// rows not a multiple of four columns) or the staged words (rows x views x 4 nw).
inline size_t sv_scratch_floats(int max_rows, int W, int max_views)
{
    const size_t per = (size_t)(4 * sv_scratch_words(W) > W ? 4 * sv_scratch_words(W) : W);
    return (size_t)max_rows * max_views * per;
}

// A-matrix column of one (voxel line, view), as the kernels store it:
// word 0 = j0 | n << 16 (first kept detector column j0, n kept columns, which
// are consecutive), words 1..amax = the values of columns j0 .. j0 + amax - 1
// (0 past n); eq 16-byte words in all.
//
// Column cache: the columns of every in-mask line for every view, laid out
// [N_y * N_x][N_p][eq] (line-major, view next), computed once per stage.
// FP16 variant (full resolution, N_r <= 4096): 8 bytes per entry, word 0 =
// j0 | n << 12 | fp16(a0) << 16, word 1 = fp16(a1) | fp16(a2) << 16.
struct SvACache {
    const int4 *a;  // nullptr: the kernel computes columns itself
};

struct SvTask {
    int frame, k0, j0, z0, nz;
    int nlines;  // in-mask voxel lines (host-side ordering of the work queue)
    float *mag;  // [N_y][N_x] plane of the magnitude map for (frame, z-group)
    int prob;    // problem of a batched launch (0 otherwise)
    int plane;   // index of that plane: frame * z-groups + z-group
};

struct SvTaskOut {
    double sum_abs_dx, sum_abs_x;
    long long updates, zero_skips;
};

// Shared-memory regions of one CTA for one problem, in elements (a batched
// launch carves them per task from its problem's plan, within the largest
// plan's bytes).
struct SvPlan {
    int ring_bytes;    // A-column ring
    int band_pairs;    // (e, sqrt(w)) float2 band entries
    int trig_views;    // views with cos / sin (computed columns only)
    int xb, tb, magl;  // voxel block, temporal neighbours, |dx| per (slice, line)
    int part;          // per-slice theta partials (floats)
    int views;         // view index / band origin entries
    int order;         // step-sequence entries
};
SvPlan mbir_sv_plan(const SvParams &sp, bool cached);
size_t mbir_sv_plan_bytes(const SvPlan &pl);
size_t mbir_sv_smem_bytes(const SvParams &sp, bool cached);
size_t mbir_acache_bytes(const MbirGeom &g, int eq, bool half);
// Fills the column cache (exact bin indices, FP32 values) for the in-mask
// lines.  err |= 2 if a column has more than amax entries.
cudaError_t mbir_build_acache(const MbirGeom &g, const MbirDev &dv, int amax, int eq, bool half, int4 *cache,
                              int *err, cudaStream_t s);
// Forward projection, deterministic (FP32 sums in a fixed order, no
// atomics): mode 0: out = y - A x - d; mode 1: out = A x.  amax: most
// columns per A-matrix entry (2 mult_xy + 1).
cudaError_t mbir_forward_rows(const MbirGeom &g, const int *frame_of_view, const float *x, const float *y,
                              const float *d, float *out, int mode, int amax, cudaStream_t s);

// One launch: the super-voxels order[0 .. ntasks) (ids into tasks[]) in
// that order.  Super-voxel order[k] first waits until done[d] == epoch for
// every id d in deps[dep_off[k] .. dep_off[k + 1]) (the conflicting ones
// earlier in the order), and sets done[order[k]] = epoch when finished.
struct SvProblem;
struct SvBatchState;
struct SvLaunch {
    const SvTask *tasks;
    const int *order, *dep_off, *deps;
    int ntasks;
    int *done;
    int epoch;
    // batched launches only: the problems, the position of each queue entry
    // in its problem's own order (seq), per-problem state, and the control
    // words ctl[0] = iteration number (also the epoch of the done flags)
    const SvProblem *problems;
    const int *seq;
    SvBatchState *state;
    const int *ctl;
    // a pass over a device-chosen subset (NHICD): queue entry k is position
    // pos[k] of the order / dependency lists, *ntasks_dev entries in all,
    // and only the lines with sel[plane][line] != 0 are visited (all three
    // null: every entry of the lists, every in-mask line)
    const int *pos;
    const int *ntasks_dev;
    const uint8_t *sel;
};

// One problem of a batched launch: its stage's geometry, arrays, prior (the
// over-relaxation it uses), schedule parameters and column cache.
struct SvProblem {
    MbirGeom g;
    MbirPrior pr;
    MbirDev dv;
    SvParams sp;
    SvACache ac;
    SvPlan plan;  // shared-memory regions
    int cap;      // super-voxels in flight at most
    int K;        // sub-iterations per iteration (scales the convergence ratio)
    double stop;  // convergence threshold, percent
};

// Per-problem state of a batched run (device).
struct SvBatchState {
    SvTaskOut out;   // this iteration's statistics
    long long updates, zero_skips;
    double pct;      // convergence ratio of the last iteration, percent
    double prev_ax;  // summed |x'| of the previous iteration's updates
    int active;      // still iterating
    int iters;       // iterations done
    int converged;   // stopped by the convergence test
    int fin;         // super-voxels finished in this launch
    int adjustments; // times the in-flight cap was halved
};

// NHICD selection on the device (mbir_nhicd.cu).  Per plane of `filt`
// (planes x n values, the VSC-filtered magnitude map): thresh[plane] = the
// (n - nsel[plane])-th smallest value, sel[plane][q] = filt > thresh,
// count[plane] = lines selected (XT_NHICD.c:164-216).
cudaError_t mbir_launch_vsc_threshold(const float *filt, int planes, int n, const int *nsel, float *thresh,
                                      uint8_t *sel, int *count, cudaStream_t s);
// The positions k of a sweep's order[0 .. n) whose super-voxel holds a
// selected in-mask line, kept in order, into pos[0 .. *ntasks); the others
// get done[id] = epoch.
cudaError_t mbir_launch_sv_nh_list(const int *order, int n, const SvTask *tasks, int S, int N_x, int N_y,
                                   const uint8_t *sel, const uint8_t *mask, int epoch, int *done, int *pos,
                                   int *ntasks, cudaStream_t s);

// CTAs of the super-voxel kernel that fit one SM for this configuration.
int mbir_sv_ctas_per_sm(const MbirGeom &g, const SvParams &sp, bool cached);

// ctas persistent CTAs take the launch's super-voxels from the queue counter
// (zero before the launch); scratch holds ctas * sp.band_floats floats; the
// CTAs add their statistics to *out.  err |= 1: a column outside the band,
// 2: a column wider than amax, 4: a dependency wait gave up.
cudaError_t mbir_launch_icd_sv(const MbirGeom &g, const MbirPrior &pr, const MbirDev &dv, const SvParams &sp,
                               SvACache ac, const SvLaunch &L, int ctas, int *queue, float *scratch, SvTaskOut *out,
                               int iter, uint32_t seed, int *err, cudaStream_t s);

// Batched launches: every problem has a column cache (FP32 values, or FP16
// when half), 3 detector columns per entry and one row per slice, at most
// kSvBatchThreads / 32 warps per super-voxel and kSvBatchViewsPerLane views
// per lane.  The super-voxel of queue entry k starts when its conflicting
// super-voxels have finished (as above) and when at most cap - 1 super-voxels
// of its problem before it are unfinished; super-voxels of problems no
// longer active are skipped.  The CTA statistics go to state[prob].out;
// err |= 8: an in-flight wait gave up.
constexpr int kSvBatchThreads = 256;
constexpr int kSvBatchViewsPerLane = 8;
int mbir_sv_batch_ctas_per_sm(size_t smem_bytes, bool half);
cudaError_t mbir_sv_batch_prepare(size_t smem_bytes, bool half);
cudaError_t mbir_launch_icd_sv_batch(size_t smem_bytes, bool half, const SvLaunch &L, int ctas, int *queue,
                                     float *scratch, size_t scratch_floats, uint32_t seed, int *err, cudaStream_t s);
// End of a batched iteration: per active problem, the iteration's statistics
// into the totals, the convergence test and the stability guard (a summed
// |x'| above 2 x the previous iteration's halves the problem's in-flight
// cap); then the
// statistics, in-flight counters and queue counter are reset, ctl[0] (the
// iteration) advances and ctl[1] = problems still active.
cudaError_t mbir_launch_sv_batch_end(SvProblem *probs, SvBatchState *state, int n, int *ctl, int *queue,
                                     cudaStream_t s);
