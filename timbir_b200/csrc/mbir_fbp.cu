// Filtered backprojection (parallel beam), frame by frame: the start image of
// FBP-initialised ICD and the input of the learned warm start.  No reference
// counterpart (TIMBIR starts its coarsest stage from zero); the geometry is
// the stage's own (detector column j at R0 + (j + 0.5) delta_r, voxel centres
// as in the A matrix, r = x cos(theta) - y sin(theta), XT_AMatrix.c:62-68).
//
//   ramp filter   q(j) = delta_r sum_k p(k) h(j - k), the band-limited
//                 Ram-Lak kernel h(0) = 1 / (4 delta_r^2),
//                 h(n odd) = -1 / (pi^2 n^2 delta_r^2), h(n even) = 0
//                 (Kak and Slaney, Principles of Computerized Tomographic
//                 Imaging, eq. 3.61), over each (detector row, view);
//   backprojection  x = pi / n_f sum over the frame's n_f views of q at r,
//                 linearly interpolated; voxels outside the reconstruction
//                 mask are 0 (ICD never updates them).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "mbir_internal.h"
#include "mbir_fbp.h"

namespace {

__global__ void __launch_bounds__(256) k_ramp(const float *__restrict__ y, float *__restrict__ q, int N_r,
                                              double delta_r)
{
    extern __shared__ float line[];
    const size_t base = (size_t)blockIdx.x * N_r;  // one (row, view) line of [N_t][N_p][N_r]
    for (int j = threadIdx.x; j < N_r; j += blockDim.x) line[j] = y[base + j];
    __syncthreads();
    const double h0 = 1.0 / (4.0 * delta_r * delta_r);
    const double c = -1.0 / (M_PI * M_PI * delta_r * delta_r);
    for (int j = threadIdx.x; j < N_r; j += blockDim.x) {
        double acc = h0 * line[j];
        // odd offsets only; both sides of j
        for (int n = 1; n < N_r; n += 2) {
            const double h = c / ((double)n * n);
            float s = 0.0f;
            if (j - n >= 0) s += line[j - n];
            if (j + n < N_r) s += line[j + n];
            acc += h * s;
        }
        q[base + j] = (float)(delta_r * acc);
    }
}

// One thread per voxel (x, y) of one slice and frame.
__global__ void __launch_bounds__(256) k_backproject(MbirGeom g, const uint8_t *__restrict__ mask,
                                                     const float *__restrict__ q, float *__restrict__ x)
{
    const int xy = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.y, i = blockIdx.z;
    if (xy >= g.N_x * g.N_y) return;
    const int k = xy % g.N_x, j = xy / g.N_x;
    float *out = x + (((size_t)i * g.N_z + z) * g.N_y + j) * g.N_x + k;
    if (!mask[xy]) {
        *out = 0.0f;
        return;
    }
    const double vxp = g.x0 + ((double)k + 0.5) * g.delta_xy;
    const double vyp = g.y0 + ((double)j + 0.5) * g.delta_xy;
    const int nv = g.view_num[i];
    const int *vl = g.view_idx + (size_t)i * g.max_views;
    double acc = 0.0;
    for (int v = 0; v < nv; v++) {
        const int p = vl[v];
        const double r = vxp * g.cosv[p] - vyp * g.sinv[p];
        const double t = (r - g.R0) / g.delta_r - 0.5;
        const int j0 = (int)floor(t);
        const double w = t - j0;
        for (int rr = 0; rr < g.m_z; rr++) {
            const float *ql = q + ((size_t)(z * g.m_z + rr) * g.N_p + p) * g.N_r;
            const double a = j0 >= 0 && j0 < g.N_r ? ql[j0] : 0.0;
            const double b = j0 + 1 >= 0 && j0 + 1 < g.N_r ? ql[j0 + 1] : 0.0;
            acc += (1.0 - w) * a + w * b;
        }
    }
    *out = nv > 0 ? (float)(M_PI / nv * acc / g.m_z) : 0.0f;
}

}  // namespace

cudaError_t mbir_launch_fbp(const MbirGeom &g, const uint8_t *mask, const float *y, float *scratch, float *x,
                            cudaStream_t s)
{
    const int lines = g.N_t * g.N_p;
    k_ramp<<<lines, 256, g.N_r * sizeof(float), s>>>(y, scratch, g.N_r, g.delta_r);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const dim3 grid((g.N_x * g.N_y + 255) / 256, g.N_z, g.N_time);
    k_backproject<<<grid, 256, 0, s>>>(g, mask, scratch, x);
    return cudaGetLastError();
}
