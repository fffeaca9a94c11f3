// Internal declarations shared by the host driver (mbir_stage.cu,
// mbir_reconstruct.cpp) and the CUDA kernels (mbir_kernels.cu).
//
// Device layouts (chosen for the access patterns of the kernels, not copied
// from the reference's [view][col][row] layout, which is kept only at the file
// boundary):
//   sinogram-shaped arrays  e, w, y : float [N_t][N_p][N_r]  (slice-major,
//                                      detector column fastest; one slice's
//                                      sinogram is one contiguous plane)
//   ring offset d                   : float [N_t][N_r]
//   object x                        : float [N_time][N_z][N_y][N_x]
//   update-magnitude map            : float [N_time][nblk][N_y][N_x]
//   detector response H_r           : float [N_p][65]
//   cos/sin of view angles          : double [N_p]
//   views of frame i                : int32 view_idx[i*max_views + k]
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define MBIR_RESP_BINS 64
#define MBIR_MAX_STAGES 8

struct MbirGeom {
    // detector
    int N_p, N_r, N_t, m_z;
    double delta_r, R0, RMax, OffsetR;
    // object
    int N_x, N_y, N_z, N_time;
    double x0, y0, delta_xy;
    // views
    int max_views;
    const int *view_idx;   // [N_time][max_views]
    const int *view_num;   // [N_time]
    const double *cosv, *sinv;
    const float *H_r;      // [N_p][65]
};

struct MbirPrior {
    double sSQ, sSQP, sTQ, sTQP, c_s, c_t;
    double SF[27];  // spatial weights, index 9*dz + 3*dy + dx (each 0..2)
    double TF;      // temporal weight
    double alpha;   // over-relaxation
    double hT, hdelta;  // generalized-Huber threshold and slope
};

struct MbirDev {
    float *e, *w, *d, *x, *mag;
    const uint8_t *mask;   // [N_y][N_x]
    // z-slab of a volume sharded over ranks (XT_MPI.c:47-82): the slab
    // below's top slice (halo_lo) and the slab above's bottom slice
    // (halo_hi) of every frame, [2][N_time][N_y][N_x]; they are neighbours
    // of this slab's first and last slices, read but never updated
    const float *halo;
    int halo_lo, halo_hi;
};

#ifdef __CUDACC__
// Does slice zz (-1 .. N_z) exist as a neighbour: the slab's own slices, and
// the halo slices when the neighbouring slab exists (XT_VoxUpdate.c:126-131).
__device__ __forceinline__ bool slab_has_z(const MbirGeom &g, const MbirDev &dv, int zz)
{
    return zz >= (dv.halo_lo ? -1 : 0) && zz < g.N_z + (dv.halo_hi ? 1 : 0);
}

// Plane [N_y][N_x] of slice zz of frame i (zz = -1 and N_z: the halo slices).
__device__ __forceinline__ const float *slab_plane(const MbirGeom &g, const MbirDev &dv, int i, int zz)
{
    const size_t plane = (size_t)g.N_y * g.N_x;
    if (zz < 0) return dv.halo + (size_t)i * plane;
    if (zz >= g.N_z) return dv.halo + ((size_t)g.N_time + i) * plane;
    return dv.x + ((size_t)i * g.N_z + zz) * plane;
}
#endif

// One task of a reference-schedule half-sweep: a (frame, z-block) pair and a
// range of one of its line lists.
struct MbirTask {
    int frame, z0, z1, b0, b1;
    const int *xs, *ys;    // line list (device)
    float *mag;            // [N_y][N_x] plane of the magnitude map
};

struct MbirTaskOut {
    double vox_mag;        // sum of |x'| over updated voxels
    long long updates;     // voxel updates performed
    long long zero_skips;  // voxels skipped by zero skipping
};

// ---- kernel launchers (mbir_kernels.cu) -------------------------------------
// (the forward projection is mbir_forward_rows in mbir_sv.cu)
cudaError_t mbir_launch_icd_ref(const MbirGeom &g, const MbirPrior &pr, const MbirDev &dv,
                                const MbirTask *tasks, int ntasks, MbirTaskOut *out, int iter,
                                int threads, size_t acache_bytes, void *acache_global,
                                cudaStream_t s);
cudaError_t mbir_launch_cost(const MbirGeom &g, const MbirPrior &pr, const MbirDev &dv,
                             double *partials, int nparts, double *result, cudaStream_t s);
// Rectangular-patch constraint windows of offset type 3 (device arrays; the
// element index is q = t N_r + r): per window m its elements win_el /
// weights win_a in [win_off[m], win_off[m+1]); per overlapping window pair
// (pair_i <= pair_j) the shared elements and both weights; per element its
// windows el_m / weights el_a.  D (M x M), y (M), x (nel) are scratch.
struct OffsetWindows {
    int M, nel, npairs;
    const int *win_off, *win_el;
    const float *win_a;
    const int *pair_off, *pair_i, *pair_j, *pair_el;
    const float *pair_ai, *pair_aj;
    const int *el_off, *el_m;
    const float *el_a;
    double *D, *y, *x;
};
// Ring-offset update of the given type; with type 3 and windows (M > 0) the
// constrained solve (err |= 16 if its system is not positive definite).
// With `chunks` (2 mbir_offset_chunks(g) N_t N_r doubles of scratch) the view
// sums are spread over view chunks of kOffsetViewChunk and the sinogram is
// updated by one thread per entry; without, one thread per detector element
// sums all views (the scratch is num, den and the partials only).
constexpr int kOffsetViewChunk = 16;
int mbir_offset_chunks(const MbirGeom &g);
cudaError_t mbir_launch_offset(const MbirGeom &g, const MbirPrior &pr, const MbirDev &dv, int type,
                               double *num, double *den, double *partials, int nparts,
                               cudaStream_t s, const OffsetWindows *win = nullptr, int *err = nullptr,
                               double *chunks = nullptr);
cudaError_t mbir_launch_variance(const MbirGeom &g, const MbirPrior &pr, const MbirDev &dv,
                                 double var_est, double *partials, int nparts, double *result,
                                 cudaStream_t s);
cudaError_t mbir_launch_variance_apply(const MbirGeom &g, const MbirDev &dv, double var_new,
                                       cudaStream_t s);
cudaError_t mbir_launch_vsc_filter(const float *mag, float *filt, int planes, int N_y, int N_x,
                                   cudaStream_t s);
cudaError_t mbir_launch_select_stats(const float *mag, const int *xs, const int *ys,
                                     const int *counts, int planes, int stride, double *out,
                                     cudaStream_t s);
int mbir_amax(double delta_xy, double delta_r);
// x2 up-sampling of n_z coarse [n_y][n_x] slices into [n_z or 2 n_z][2 n_y][2 n_x]
// (z_too: also along z), as the host hand-off between stages computes it.
cudaError_t mbir_launch_upsample(const float *in, float *out, int n_z, int n_y, int n_x, bool z_too, cudaStream_t s);
// [view][row][col] -> [row][view][col].
cudaError_t mbir_launch_to_slice_major(const float *in, float *out, int N_p, int N_t, int N_r, cudaStream_t s);
// Detector response table H_r [N_p][65] from the host-computed trapezoids and beam.
cudaError_t mbir_launch_detector_response(const double *trap, const double *beam, int N_p, double OffsetR,
                                          double delta_xy, double r0, double step, double tc, float *H_r,
                                          cudaStream_t s);
