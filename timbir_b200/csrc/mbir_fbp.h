// Filtered backprojection (mbir_fbp.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "mbir_internal.h"

// x [N_time][N_z][N_y][N_x] = the frames' filtered backprojections of the
// slice-major projections y [N_t][N_p][N_r]; scratch holds N_t N_p N_r floats.
cudaError_t mbir_launch_fbp(const MbirGeom &g, const uint8_t *mask, const float *y, float *scratch, float *x,
                            cudaStream_t s);
