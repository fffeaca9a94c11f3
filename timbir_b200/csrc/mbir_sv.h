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
    int max_nz;     // slices per CTA (one warp each)
    int max_rows;   // detector rows per CTA: max_nz * m_z
    size_t band_floats;  // scratch floats per CTA: max_rows * W * max_views
};

struct SvTask {
    int frame, k0, j0, z0, nz;
    float *mag;  // [N_y][N_x] plane of the magnitude map for (frame, z-group)
};

struct SvTaskOut {
    double sum_abs_dx, sum_abs_x;
    long long updates, zero_skips;
};

size_t mbir_sv_smem_bytes(const SvParams &sp);
cudaError_t mbir_launch_icd_sv(const MbirGeom &g, const MbirPrior &pr, const MbirDev &dv, const SvParams &sp,
                               const SvTask *tasks, int ntasks, float *scratch, SvTaskOut *out, int iter,
                               uint32_t seed, int *err, cudaStream_t s);
