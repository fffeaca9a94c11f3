// Super-voxel ICD kernel interface (mbir_sv.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "mbir_internal.h"

struct SvParams {
    int S;          // super-voxel side (voxel lines)
    int W;          // band width (detector columns per view)
    int amax;       // max A-matrix entries per (line, view): 2 mult_xy + 1
    int max_views;  // max views of any frame (shared-memory stride)
    int max_nz;     // slices per CTA
    int max_rows;   // detector rows per CTA: max_nz * m_z
    int vsplit;     // warps per slice (1, 2 or 4; > 1 needs max_nz <= 15)
    int prod_warps; // warps computing the next line's A-matrix column
    size_t band_floats;  // scratch floats per CTA: max_rows * W * max_views
};

struct SvTask {
    int frame, k0, j0, z0, nz;
    int nlines;  // in-mask voxel lines (host-side ordering of the work queue)
    float *mag;  // [N_y][N_x] plane of the magnitude map for (frame, z-group)
};

struct SvTaskOut {
    double sum_abs_dx, sum_abs_x;
    long long updates, zero_skips;
};

size_t mbir_sv_smem_bytes(const SvParams &sp);
// ctas persistent CTAs take the ntasks tasks from the queue counter (zero
// before the launch); scratch holds ctas * sp.band_floats floats; the CTAs
// add their statistics to *out.
cudaError_t mbir_launch_icd_sv(const MbirGeom &g, const MbirPrior &pr, const MbirDev &dv, const SvParams &sp,
                               const SvTask *tasks, int ntasks, int ctas, int *queue, float *scratch,
                               SvTaskOut *out, int iter, uint32_t seed, int *err, cudaStream_t s);
