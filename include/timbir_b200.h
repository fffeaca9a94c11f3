/*
 * timbir_b200 -- C ABI of the B200 (sm_100a) MBIR ICD/NHICD engine.
 *
 * Two levels:
 *
 *  1. The drop-in library call, declared in mbir4d.h beside this file:
 *     reconstruct(), with the signature, argument meaning, file outputs and
 *     ownership rules of the reference's (TIMBIR v0.0.2
 *     src/include/mbir4d.h:35, src/MBIR_4D/XT_Engine.c:81).
 *
 *  2. Stage-level entry points that reconstruct() is built from.  Each one
 *     replaces the reference function named beside it, operates on one
 *     resolution stage held in device memory, and returns 0 on success or -1
 *     with a message available from mbir_last_error().  Plain pointers and
 *     sizes only; host arrays use the reference's layouts:
 *       projections / weights  float [proj_num][proj_rows][proj_cols]
 *       sinogram-shaped output float [proj_num][proj_cols][proj_rows]
 *                              (the reference's internal [N_p][N_r][N_t])
 *       object                 float [recon_num][N_z][N_y][N_x]
 *       ring offsets           float [proj_cols][proj_rows]
 *       magnitude map          float [recon_num][num_z_blocks][N_y][N_x]
 */
#ifndef TIMBIR_B200_H_
#define TIMBIR_B200_H_

#include <stdint.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct MbirStage MbirStage;
typedef struct MbirBatch MbirBatch;

/* initStatStructures + initDynStructures for one stage whose voxels are
 * mult_xy detector columns wide and mult_z detector rows high
 * (src/MBIR_4D/XT_Init.c:449-669 and 211-445).  The object starts at zero,
 * the ring offsets at zero, the variance estimate at 1.  num_z_blocks plays
 * the role the OpenMP thread count plays in the reference
 * (XT_Init.c:389-398): the number of z-blocks of the checkerboard schedule;
 * it must be even, >= 2 and <= N_z. */
int mbir_init_stage(MbirStage **out, const float *projections, const float *weights,
                    const float *proj_angles, const float *proj_times, const float *recon_times,
                    int32_t proj_rows, int32_t proj_cols, int32_t proj_num, int32_t recon_num,
                    float vox_wid, float rot_center, float sig_s, float sig_t, float c_s, float c_t,
                    float convg_thresh, int32_t remove_rings, int32_t quad_convex, float huber_delta,
                    float huber_T, int32_t mult_xy, int32_t mult_z, int32_t num_z_blocks);

/* freeDynMemory + freeStatMemory (XT_Init.c:672-707). */
void mbir_free_stage(MbirStage *stage);

/* Message of the last failing call on this thread. */
const char *mbir_last_error(void);

/* Stage switches set by initDynStructures from the stage index
 * (updateProjOffset, updateVar; XT_Init.c:236-266) and the variance estimate
 * read from the previous stage (XT_Init.c:290-291, 327-330). */
int mbir_set_stage_switches(MbirStage *stage, int32_t update_proj_offset, int32_t update_var,
                            double var_est);

/* Convergence threshold of the stage's iterations, percent (the convg_thresh
 * of reconstruct(); XT_ICD_update.c:1066-1103). */
int mbir_set_convergence_threshold(MbirStage *stage, double convg_thresh);

/* State of the voxel-line order generator (randlib.c srandom2/random2); one
 * stream runs through a whole reconstruct() call. */
int mbir_set_rng_state(MbirStage *stage, uint32_t state);
uint32_t mbir_get_rng_state(MbirStage *stage);

/* Stage prologue of ICD_BackProject (XT_ICD_update.c:1134-1159): mask,
 * detector response (DetectorResponseProfile, XT_Profile.c:129), initial
 * object / offsets / magnitude map (any may be NULL for zero), and the error
 * sinogram e = y - A x - d (initErrorSinogam, XT_ICD_update.c:655). */
int mbir_icd_prepare(MbirStage *stage, const float *object, const float *offset,
                     const float *magmap);

/* Voxel-update schedule of mbir_update_voxels_time_slices:
 *   0  the reference's (default): checkerboard (frame, z-block) tasks, random
 *      line order, 10 HICD/NHICD sub-iterations, exactly as
 *      updateVoxelsTimeSlices (XT_ICD_update.c:936-1105);
 *   1  super-voxel schedule (no reference counterpart): sv_side x sv_side
 *      blocks of voxel lines updated by one CTA each from a shared-memory copy
 *      of the error-sinogram band they touch, blocks of one colour of a
 *      (x, y, z-group, frame) checkerboard in parallel.  sv_side 0 picks the
 *      largest side (<= 16) whose band fits shared memory; warps_per_slice
 *      (1, 2 or 4; 0 = 2 when a z-group has at most 15 slices) splits each
 *      slice's views over that many warps.
 * The magnitude map of schedule 1 has one plane per (frame, z-group). */
int mbir_set_schedule(MbirStage *stage, int32_t schedule, int32_t sv_side, int32_t warps_per_slice);
int mbir_get_schedule(MbirStage *stage, int32_t *schedule, int32_t *sv_side, int32_t *z_group,
                      int32_t *band_width, int32_t *phases, int32_t *warps_per_slice);

/* A-matrix column cache of schedule 1 (no reference counterpart; the
 * reference recomputes every column at every visit, calcAMatrixColumnforAngle,
 * XT_AMatrix.c:50-110): the exact columns of every in-mask voxel line for
 * every view, 16 bytes per (line, view) at full resolution, built once per
 * stage at its first iteration.  mode -1 (default): used when it takes at
 * most a third of free device memory; 0: never (columns computed in the
 * kernel); 1: always (mbir_set_schedule fails if it cannot be allocated);
 * 2: as -1, with FP16 values (8 bytes per entry; accumulation stays FP32;
 * full-resolution stages of detectors up to 4096 columns, others keep FP32
 * values): the iteration then minimises the cost of the A matrix rounded to
 * FP16.  Takes effect at the next mbir_set_schedule.  mbir_get_acache's
 * *used is 0 (no cache), 1 (FP32 values) or 2 (FP16 values). */
int mbir_set_acache(MbirStage *stage, int32_t mode);
int mbir_get_acache(MbirStage *stage, int32_t *used, int64_t *bytes);
/* Persistent CTAs per launch of schedule 1 (0, the default: automatic, see
 * mbir_get_sv_grid).  With 1 the super-voxels of a launch run one after
 * another, which makes the schedule deterministic (a debugging and testing
 * aid); more than the automatic count can make the iteration diverge. */
int mbir_set_sv_ctas(MbirStage *stage, int32_t ctas);
/* Slices per z-group of schedule 1 (0, the default: automatic); takes
 * effect at the next mbir_set_schedule.  Z-groups have disjoint sinogram
 * rows, so smaller groups allow more super-voxels in flight. */
int mbir_set_sv_zgroup(MbirStage *stage, int32_t slices);
/* Over-relaxation of schedule 1's voxel steps, in (0, 2); 0 (the default)
 * chooses it: the reference's 1.5 (XT_ICD_update.c:134-183) when the GPU can
 * be kept busy with it, else the largest value down to 0.7 that allows enough
 * super-voxels in flight (see mbir_get_sv_grid).  Takes effect at the next
 * mbir_set_schedule.  The reference schedule always uses 1.5. */
int mbir_set_sv_relaxation(MbirStage *stage, double alpha);
/* Times the super-voxel schedule's stability guard has halved the
 * super-voxels in flight since the schedule was set: when the MAP cost rose
 * (by more than 1e-6 of it) over a window of iterations (one iteration for
 * the first four windows, then eight), the state at the window's start is
 * restored and the iteration redone with half as many in flight (the
 * automatic grid, or the CTA count mbir_set_sv_ctas set). */
int mbir_get_sv_adjustments(MbirStage *stage);
/* The stability guard on (1, the default) or off (0). */
int mbir_set_sv_guard(MbirStage *stage, int32_t on);
/* Non-homogeneous pass of schedule 1 (the reference's NHICD, XT_NHICD.c:
 * 164-216, XT_ICD_update.c:1015-1058): from the second iteration, after the
 * sweep, the lines whose 5x5 Hamming-filtered update magnitude is above each
 * (frame, z-group) plane's order statistic -- `fraction` of the plane's
 * in-mask lines (the reference takes 0.1: lines / NHICD iterations) -- are
 * updated once more, chosen on the device.  0, the default, turns the pass
 * off (the sweep alone reached the MAP cost sooner on the measured
 * workloads); reconstruct() reads the fraction from TIMBIR_SV_NHICD. */
int mbir_set_sv_nhicd(MbirStage *stage, double fraction);
/* The NHICD line selection on the device, for testing against the
 * reference's VSC_based_Voxel_Line_Select (XT_NHICD.c:164-216): mag host
 * float [planes][N_y][N_x] magnitude maps, nsel[plane] lines wanted; sel
 * (host, same shape) = 1 where the filtered magnitude (ComputeVSC) exceeds the
 * plane's (N_y N_x - nsel)-th smallest filtered value, thresh[plane] (may be
 * NULL) = that value. */
int mbir_nhicd_select(const float *mag, int32_t planes, int32_t N_y, int32_t N_x, const int32_t *nsel,
                      uint8_t *sel, float *thresh);
/* The x2 up-sampling that hands a stage's object and magnitude map to the
 * next multi-resolution stage on the device (upsample_object_bilinear_2D /
 * _3D, upsample_bilinear_2D / _3D, XT_ICD_update.c:323-498): host float in
 * [n_z][n_y][n_x] -> out [n_z or 2 n_z][2 n_y][2 n_x] (z_too = 1: also along
 * z), computed by the same GPU kernels reconstruct() uses between stages.
 * For testing; n_y, n_x >= 2, n_z >= 2 with z_too. */
int mbir_upsample(const float *in, float *out, int32_t n_z, int32_t n_y, int32_t n_x, int32_t z_too);
/* The automatic launch size of schedule 1: persistent CTAs per launch, the
 * super-voxels allowed in flight per (frame, z-group) sinogram (more of them
 * correct the same rays at once and the iteration diverges), the CTAs that
 * fit the GPU, and the over-relaxation in use. */
int mbir_get_sv_grid(MbirStage *stage, int32_t *ctas, int32_t *cap_per_group, int32_t *resident,
                     double *relaxation);
/* The cached columns of in-mask voxel line (row, col) for every view:
 * N_p x 4 ceil((2 + 2 mult_xy) / 4) words; per view, word 0 = j0 | n << 16
 * (first detector column with a positive entry, number of columns from it),
 * then the n values (float bits), zero-padded. */
int mbir_get_acache_line(MbirStage *stage, int32_t row, int32_t col, int32_t *words);

/* One outer ICD iteration with the reference schedule
 * (updateVoxelsTimeSlices, XT_ICD_update.c:936-1105): random line order,
 * 10 sub-iterations of checkerboard HICD half-sweeps with ring-offset updates,
 * NHICD selection and (iter > 1) NHICD half-sweeps, variance update, and the
 * convergence test; *converged is set to its result. */
int mbir_update_voxels_time_slices(MbirStage *stage, int32_t iter, int32_t *converged);

/* computeCost (XT_ICD_update.c:186-319), FP64 on the GPU. */
int mbir_compute_cost(MbirStage *stage, double *total, double *forward, double *prior);

/* update_Sinogram_Offset (XT_ICD_update.c:919-927), by remove_rings. */
int mbir_update_sinogram_offset(MbirStage *stage);
/* Rectangular-patch constraint windows for ring-offset mode 3 (remove_rings
 * 3): on = 1 builds them as gen_offset_constraint_windows does
 * (XT_OffsetError.c:46-96; overlapping windows of 2 N_r / round(sqrt N_r)
 * columns by 2 N_t / round(sqrt N_t) rows with tent weights), and mode 3
 * then solves the constrained problem of update_d_offset_rect_patch_constraint
 * / constrained_quad_opt (XT_ICD_update.c:753-800, XT_OffsetError.c:99-168):
 * the offsets minimise the data term subject to a zero weighted sum over
 * every window, through an M x M FP64 system solved on the GPU.  on = 0 (the
 * default, and the reference's reconstruct path, which builds no windows)
 * leaves mode 3 unconstrained.  mbir_get_offset_windows = windows built. */
int mbir_set_offset_windows(MbirStage *stage, int32_t on);
int mbir_get_offset_windows(MbirStage *stage);

/* update_variance_parameter (XT_ICD_update.c:720-751). */
int mbir_update_variance_parameter(MbirStage *stage);

/* ---- fault injection, for testing the error paths (no counterpart) ------
 * mbir_set_device_bytes_cap: the library's device allocator refuses an
 * allocation that would take the memory its stages hold above `bytes`, as an
 * exhausted device would (0: no cap); mbir_get_device_bytes: the bytes held.
 * mbir_debug_sv_skip_tasks: the next super-voxel sweep of the stage starts
 * its work queue n entries in, so those super-voxels never run and the ones
 * ordered after them that conflict with them wait for them until the
 * kernel's bounded wait gives up (about half a second); the iteration then
 * returns an error ("dependency wait timed out") and the context stays
 * usable.  The stage's state afterwards is that of an interrupted sweep. */
int mbir_set_device_bytes_cap(int64_t bytes);
int64_t mbir_get_device_bytes(void);
int mbir_debug_sv_skip_tasks(MbirStage *stage, int32_t n);

/* ---- data ingestion (the drivers' readers, before reconstruct()) --------
 * The HDF5 file access is the caller's; these take the datasets' arrays as
 * the file holds them, [frames][rows][cols] in HOST memory, and select the
 * readers' hyperslabs: columns trimmed symmetrically to a multiple of
 * proj_cols (ratio = kept columns / proj_cols, the same along rows), rows
 * datafile_row0 + rank (proj_rows / ranks) ratio onwards (rank / ranks in
 * place of MPI_Comm_rank / MPI_Comm_size), views proj_start ..
 * proj_start + proj_num - 1.  Outputs projections and weights [proj_num]
 * [proj_rows / ranks][proj_cols] (host).  Return 0, or -1 with
 * mbir_ingest_last_error().
 *
 * APS counts (read_data, aps_data/XT_HDFIO.c:46-236): bright and dark
 * stacks averaged over their frames 1 .. n - 2, per output sample over its
 * ratio x ratio raw samples weights = sum |count - dark|, bright =
 * sum |white - dark|, t = log(bright / weights), projection = bh t^2 + t
 * (bh: BH_QUAD_COEF, 0.5 in the APS driver). */
const char *mbir_ingest_last_error(void);
int mbir_normalize_counts(const uint16_t *counts, int32_t n_counts, const uint16_t *whites, int32_t n_whites,
                          const uint16_t *darks, int32_t n_darks, int32_t rows, int32_t cols, int32_t datafile_row0,
                          int32_t proj_rows, int32_t proj_cols, int32_t proj_start, int32_t proj_num, int32_t rank,
                          int32_t ranks, double bh_quad_coef, float *projections, float *weights);
/* Standard-format projections and weights (read_ProjWeightData,
 * std_data/XT_HDFIO.c:41-158): per output sample the mean of the ratio x
 * ratio projections through bh t^2 + t (bh 0 in that driver) and the sum of
 * the weights. */
int mbir_downsample_projections(const float *projs, const float *wts, int32_t n_views, int32_t rows, int32_t cols,
                                int32_t datafile_row0, int32_t proj_rows, int32_t proj_cols, int32_t proj_start,
                                int32_t proj_num, int32_t rank, int32_t ranks, double bh_quad_coef,
                                float *projections, float *weights);
/* The same normalisation on DEVICE arrays (stream: a cudaStream_t, NULL for
 * the default stream; enqueued, not waited for): frame means of a
 * [n_frames][rows][cols] uint16 stack, and projections / weights of
 * counts [views][win_rows][win_cols] against the bright and dark means of
 * the same window. */
int mbir_frame_mean_device(const uint16_t *frames, int32_t n_frames, int32_t rows, int32_t cols, float *out,
                           void *stream);
int mbir_normalize_counts_device(const uint16_t *counts, const float *white_mean, const float *dark_mean,
                                 int32_t views, int32_t win_rows, int32_t win_cols, int32_t ratio, double bh_quad_coef,
                                 float *projections, float *weights, void *stream);
/* gen_interlaced_views_0_to_Inf (aps_data/XT_Views.c:41-80): angles
 * (radians) and times of views proj_start .. proj_start + N_p - 1 of an
 * interlaced scan of K interlaced sub-scans of N_theta / K views per half
 * turn (bit-reversed offsets), views closer than rot_speed x min_acq_time to
 * the last kept one skipped.  Returns the kept views generated, or -1. */
int32_t mbir_gen_interlaced_views(float *views, float *times, int32_t K, int32_t N_theta, int32_t proj_start,
                                  int32_t N_p, float min_acq_time, float rot_speed);

/* ---- z-slab sharding (the reference's MPI decomposition, XT_MPI.c:47-122)
 * A volume split into `ranks` z-slabs, one per process (or GPU): the stage
 * holds slab `rank`, built from that slab's detector rows, as each MPI rank
 * of the reference holds its slab.  The slab's first and last slices take
 * the neighbouring slabs' boundary slices as prior neighbours (halo slices
 * 0 and N_z + 1 of the reference's object, XT_VoxUpdate.c:126-131), and the
 * cost counts the pairs with the slab above (XT_ICD_update.c:207-210).
 * `allreduce(values, count, ctx)` sums `count` doubles over the ranks in
 * place and returns 0 (nonzero: failure); the stage calls it where the
 * reference reduces over MPI_COMM_WORLD: the cost's data and prior sums
 * (XT_ICD_update.c:301-317), the variance's sum (:738-739), and the
 * convergence sums (:1079-1081).  Every rank must make the same calls in the
 * same order, so every rank runs the same stage settings.  Ring-offset mode 3
 * with constraint windows (which reduces its window system over ranks) is
 * refused for a sharded stage; modes 1 and 2 are per slab, as in the
 * reference.  ranks = 1 restores the whole-volume behaviour. */
typedef int (*MbirAllreduceFn)(double *values, int32_t count, void *ctx);
int mbir_set_z_slab(MbirStage *stage, int32_t rank, int32_t ranks, MbirAllreduceFn allreduce, void *ctx);
/* This slab's boundary slices: slice 0 (to the slab below) into lo and
 * slice N_z - 1 (to the slab above) into hi, each [N_time][N_y][N_x] in
 * DEVICE memory; returns when they are written.  Either may be NULL. */
int mbir_get_slab_faces(MbirStage *stage, float *lo, float *hi);
/* The halo slices from DEVICE memory [N_time][N_y][N_x]: lo = the slab
 * below's slice N_z - 1, hi = the slab above's slice 0 (NULL: unchanged).
 * MPI_Send_Recv_Z_Slices' exchange (XT_MPI.c:47-82) is the caller's: the
 * faces of each slab go to its neighbours' halos between iterations. */
int mbir_set_slab_halo(MbirStage *stage, const float *lo, const float *hi);

/* State read-back.  dims: N_p, N_r, N_t, N_x, N_y, N_z, N_time,
 * num_z_blocks, z_overlap_num. */
int mbir_stage_dims(MbirStage *stage, int32_t *dims);
int mbir_get_object(MbirStage *stage, float *out);
int mbir_set_object(MbirStage *stage, const float *in);
int mbir_get_errorsino(MbirStage *stage, float *out);
int mbir_get_weight(MbirStage *stage, float *out);
int mbir_get_offset(MbirStage *stage, float *out);
int mbir_get_magmap(MbirStage *stage, float *out);
int mbir_get_hr(MbirStage *stage, float *out);
int mbir_get_mask(MbirStage *stage, uint8_t *out);
/* kind 0: HICD random order of (frame, block); kind 1: NHICD selection.
 * Returns the number of lines (or -1). */
int mbir_get_lines(MbirStage *stage, int32_t kind, int32_t frame, int32_t block, int32_t *xs,
                   int32_t *ys);
double mbir_get_var_est(MbirStage *stage);
double mbir_get_update_percentage(MbirStage *stage);
long long mbir_get_update_count(MbirStage *stage);
/* Device time of the ICD update kernels, measured with CUDA events on the
 * stage's stream, and the number of kernels the stage has launched (no
 * reference counterpart: instrumentation). */
int mbir_get_kernel_stats(MbirStage *stage, double *icd_ms, long long *icd_launches, long long *launches);
/* Device clock around a span of stage calls: CUDA events recorded on the
 * stage's stream at begin and end (instrumentation; no reference counterpart). */
int mbir_time_begin(MbirStage *stage);
int mbir_time_end(MbirStage *stage, double *ms);

/* Ring-offset update that allocates no device memory.  No counterpart in the
 * reference: it is mbir_update_sinogram_offset's computation (the reference's
 * update_Sinogram_Offset) on device arrays the caller owns, for callers that
 * cannot allocate device memory -- an application or acquisition framework
 * that reserves all of the GPU's memory for its own pool at start-up (so
 * cudaMalloc fails) and forbids libraries to allocate behind its back, or a
 * processing loop that must not take cudaMalloc's implicit device-wide
 * synchronisation.
 *   e  device float [N_t][N_p][N_r]  error sinogram, updated in place
 *   w  device float [N_t][N_p][N_r]  weights
 *   d  device float [N_t][N_r]       ring offsets, updated in place
 * remove_rings 1, 2 or 3 and quad_convex / huber_delta / huber_T as for
 * reconstruct(); stream is a cudaStream_t (NULL for the default stream); the
 * call returns after the stream has run it.  Its scratch is one file-scope
 * device array of MBIR_NOALLOC_MAX_ELEMS detector elements (16 MiB, held by
 * every GPU that loads the library until exit); larger detectors are rejected
 * with an error (-1, message from mbir_noalloc_last_error()).  The first call
 * on a device looks the array's address up and caches it for the process's
 * life, so make that first call before any stream capture, and do not call
 * it on a device after cudaDeviceReset.  All calls share the array: calls
 * that overlap on the GPU (other streams, other host threads) race and must
 * be serialised by the caller.  Nothing in the array needs to start at zero. */
#define MBIR_NOALLOC_MAX_ELEMS (1 << 20)
int mbir_update_sinogram_offset_noalloc(float *e, const float *w, float *d, int32_t N_p, int32_t N_r,
                                        int32_t N_t, int32_t remove_rings, int32_t quad_convex,
                                        float huber_delta, float huber_T, void *stream);
const char *mbir_noalloc_last_error(void);

/* Filtered backprojection (ramp-filtered parallel-beam backprojection of
 * each frame's views) of the stage's projections into out
 * [N_time][N_z][N_y][N_x], zero outside the reconstruction mask: the start
 * image of FBP-initialised ICD.  No counterpart in the reference, whose
 * coarsest stage starts from zero. */
int mbir_fbp(MbirStage *stage, float *out);

/* A x of an object into a sinogram [proj_num][proj_rows][proj_cols], with the
 * forward projector of initErrorSinogam (XT_ForwardProject.c:8-25).  Meant
 * for a fresh stage: it overwrites the stage's object and error sinogram. */
int mbir_forward_project(MbirStage *stage, const float *object, float *out);

/* ---- batched super-voxel ICD (many independent problems per launch) -----
 * No counterpart in the reference, which reconstructs one scan per process;
 * each problem iterates exactly as updateVoxelsTimeSlices' HICD sweep with
 * its convergence test (XT_ICD_update.c:936-1105), without the NHICD pass.
 *
 * mbir_batch_create: the stages must be prepared (mbir_icd_prepare) and use
 * the super-voxel schedule with a column cache (mbir_set_schedule 1), plain
 * ICD (no ring-offset or variance update), full resolution (3 detector
 * columns per entry, one row per slice), at most 8 views per lane and 256
 * threads per super-voxel.  The batch holds the stages' schedules as they are
 * at creation and reads and writes the stages' objects and error sinograms;
 * free it before changing or freeing a stage.  Each problem keeps its own
 * over-relaxation and in-flight cap (uncapped = 1 drops the cap: timing
 * runs only).  Every iteration is one replay of a captured CUDA graph: a
 * persistent launch over every super-voxel of the problems still iterating,
 * then a one-CTA kernel that applies each problem's convergence test
 * (percentage below the stage's convg_thresh) and retires it. */
int mbir_batch_create(MbirBatch **batch, MbirStage *const *stages, int32_t n, int32_t uncapped);
void mbir_batch_free(MbirBatch *batch);
/* Up to max_iters iterations; every check_every iterations the host reads
 * how many problems are still active and stops at 0.  *active_left (may be
 * NULL) = problems still iterating.  Adds the updates to each stage's count.
 * A problem whose stage has a non-zero mbir_set_sv_nhicd fraction also gets
 * its NHICD pass after each batched sweep from its second iteration (the
 * stage's own device selection and launch, on its stream, in flight capped
 * as the batch caps it); its convergence test stays the sweep's. */
int mbir_batch_iterate(MbirBatch *batch, int32_t max_iters, int32_t check_every, int32_t *active_left);
/* Per problem (arrays of n; any may be NULL): iterations done, 1 when the
 * convergence test stopped it, voxel updates, zero-skipped voxels, the last
 * iteration's convergence percentage. */
int mbir_batch_stats(MbirBatch *batch, int32_t *iters, int32_t *converged, int64_t *updates,
                     int64_t *zero_skips, double *pct);
/* Device time of the batch's iterations (CUDA events on its stream), graph
 * replays, kernels launched, persistent CTAs, shared memory per CTA. */
int mbir_batch_info(MbirBatch *batch, double *ms, int64_t *replays, int64_t *launches, int32_t *ctas,
                    int64_t *smem_bytes);
/* Autotuner: times the batched kernel on this stage alone for super-voxel
 * sides 4..8 and 1, 2 or 4 warps per slice (the z-group filling 256
 * threads) and sets the stage's schedule to the fastest per voxel update.
 * Call after mbir_icd_prepare and before iterating: the object and error
 * sinogram are restored, the magnitude map cleared. */
int mbir_autotune_stage(MbirStage *stage, int32_t *sv_side, int32_t *warps_per_slice, int32_t *z_group,
                        double *ns_per_update);

/* ---- learned warm start ------------------------------------------------
 * A 3-D encoder-decoder convolutional network (4 levels, 16-128 channels,
 * 3x3x3 convolutions, average-pool down, nearest up, additive skips; 1.33 M
 * parameters) mapping a frame's filtered backprojection to an ICD start
 * image: out = in + r(s in) / s.  BF16 activations, weights and operands on
 * the tensor cores (tcgen05, FP32 accumulation in tensor memory); FP32 master
 * parameters, Adam state and loss.  Activations read back by
 * mbir_net_get_activation are the BF16 values widened to float.
 * Tensors are device float arrays [B][D][H][W] with D, H, W multiples of 8;
 * stream is a cudaStream_t (NULL: the default stream); calls return after
 * the stream has run them.  No counterpart in the reference. */
typedef struct MbirNet MbirNet;
int mbir_net_create(MbirNet **net, uint32_t seed);
void mbir_net_free(MbirNet *net);
const char *mbir_net_last_error(void);
int64_t mbir_net_param_count(void);
/* host float arrays of mbir_net_param_count() entries: per layer the weights
 * [27 taps][in channels][out channels] (tap = 9 (dz+1) + 3 (dy+1) + dx+1),
 * then the biases */
int mbir_net_get_params(MbirNet *net, float *out);
int mbir_net_set_params(MbirNet *net, const float *in);
int mbir_net_get_grads(MbirNet *net, float *out);
int mbir_net_forward(MbirNet *net, const float *in, float *out, int32_t B, int32_t D, int32_t H, int32_t W,
                     float scale, void *stream);
/* Parameter gradients of the loss mean(wt (s in + r - s target)^2) into the
 * network's gradient array (wt = 1 unless loss weights are set); *loss (may
 * be NULL) = the loss. */
int mbir_net_gradients(MbirNet *net, const float *in, const float *target, int32_t B, int32_t D, int32_t H,
                       int32_t W, float scale, double *loss, void *stream);
/* Per-voxel loss weights for the following mbir_net_gradients calls: a
 * device float array of the input's shape, read by each call (NULL: none). */
int mbir_net_set_loss_weights(MbirNet *net, const float *w);
/* High-pass loss for the following mbir_net_gradients calls: the loss
 * becomes mean(wt ((I - G) d)^2), d = s in + r - s target, G the separable
 * Gaussian low-pass of widths sigma_z (slices) and sigma_xy (voxels) per
 * patch, zeros outside the patch, radius int(4 sigma + 0.5): the network is
 * trained on the frequencies a start keeps under mbir_lowpass_blend.  Widths
 * 0, 0: the plain loss; at most 15.9. */
int mbir_net_set_loss_highpass(MbirNet *net, float sigma_z, float sigma_xy);
/* Layer k's output (which 0; layer -1: the network input) or its gradient
 * (which 1) from the last forward / gradient call, as host float
 * [B][D][H][W][C] at the layer's level; *count (may be NULL) = elements,
 * out may be NULL to ask for the count.  For tests. */
int mbir_net_get_activation(MbirNet *net, int32_t layer, int32_t which, float *out, int64_t *count);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) with the last gradients. */
int mbir_net_adam_step(MbirNet *net, float lr, void *stream);
/* start += G (ref - start) on device float arrays [N][D][H][W], G the
 * separable Gaussian low-pass of widths sigma_z (slices) and sigma_xy (x and
 * y voxels) per volume n (radius int(4 sigma + 0.5), edges mirrored about
 * the half-sample point; a width of 0 skips the axis; widths up to 15.9):
 * the low frequencies of `ref` under the high frequencies of `start`.
 * scratch: device float array of 2 N D H W.  Returns after the stream has
 * run it; errors via mbir_net_last_error().  No counterpart in the reference. */
int mbir_lowpass_blend(const float *ref, float *start, float *scratch, int32_t N, int32_t D, int32_t H, int32_t W,
                       float sigma_z, float sigma_xy, void *stream);

#ifdef __cplusplus
}
#endif
#endif
