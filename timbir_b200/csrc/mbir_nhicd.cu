// Non-homogeneous ICD (NHICD) selection on the device.
//
// VSC_based_Voxel_Line_Select (XT_NHICD.c:164-216) picks, per (frame,
// z-block) plane of the update-magnitude map, the voxel lines whose 5x5
// Hamming-filtered magnitude (ComputeVSC, XT_NHICD.c:128-162; k_vsc_filter)
// exceeds the plane's (N - n_sel)-th smallest filtered value, N = N_y N_x,
// n_sel = floor(lines updated / NHICD iterations).  The reference finds that
// order statistic with a randomized quickselect (RandomizedSelect,
// XT_NHICD.c:63-84); its value does not depend on the pivots, so here it is
// found by a 4-pass most-significant-digit radix select over the filtered
// values' order-preserving bit patterns, one CTA per plane, and the
// selection is written as a per-line byte map.
//
// The super-voxel schedule then visits only the super-voxels holding a
// selected line: k_sv_nh_list compacts the sweep's launch order (keeping its
// order, so its dependency lists stay valid) and marks the super-voxels left
// out as finished for the pass's epoch, so that no dependency wait names one.
#include <cuda_runtime.h>
#include <stdint.h>

#include "mbir_internal.h"
#include "mbir_sv.h"

namespace {

// order-preserving map of a float's bits to an unsigned key
__device__ __forceinline__ unsigned fkey(float f)
{
    const unsigned b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float fkey_inv(unsigned k)
{
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// One CTA per plane: thresh = the rank-th smallest (1-based) of the plane's
// n values, rank = n - nsel[plane]; sel[q] = filt[q] > thresh; count[plane]
// = lines selected.  nsel <= 0 selects nothing (the threshold is the largest
// value).
__global__ void __launch_bounds__(1024) k_vsc_threshold(const float *__restrict__ filt, int n,
                                                        const int *__restrict__ nsel, float *__restrict__ thresh,
                                                        uint8_t *__restrict__ sel, int *__restrict__ count)
{
    __shared__ unsigned hist[256];
    __shared__ unsigned s_prefix, s_rank;
    __shared__ int s_count;
    const int plane = blockIdx.x;
    const float *f = filt + (size_t)plane * n;
    const int want = nsel[plane];
    if (threadIdx.x == 0) {
        s_prefix = 0u;
        s_rank = (unsigned)(want > 0 ? n - want : n);
        s_count = 0;
    }
    unsigned mask = 0u;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int b = threadIdx.x; b < 256; b += blockDim.x) hist[b] = 0u;
        __syncthreads();
        const unsigned prefix = s_prefix;
        for (int q = threadIdx.x; q < n; q += blockDim.x) {
            const unsigned k = fkey(f[q]);
            if ((k & mask) == prefix) atomicAdd(&hist[(k >> shift) & 255u], 1u);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned r = s_rank, cum = 0u;
            int b = 0;
            for (; b < 255; b++) {
                if (cum + hist[b] >= r) break;
                cum += hist[b];
            }
            s_rank = r - cum;
            s_prefix = prefix | ((unsigned)b << shift);
        }
        mask |= 255u << shift;
        __syncthreads();
    }
    const float th = fkey_inv(s_prefix);
    int mine = 0;
    uint8_t *sp = sel + (size_t)plane * n;
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
        const bool take = f[q] > th;
        sp[q] = take ? 1 : 0;
        mine += take;
    }
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(&s_count, mine);
    __syncthreads();
    if (threadIdx.x == 0) {
        thresh[plane] = th;
        count[plane] = s_count;
    }
}

// One CTA: the positions k of order[0 .. n) whose super-voxel holds a
// selected in-mask line, in order, into pos[0 .. *ntasks); the others get
// done[id] = epoch.
__global__ void __launch_bounds__(1024) k_sv_nh_list(const int *__restrict__ order, int n,
                                                     const SvTask *__restrict__ tasks, int S, int N_x, int N_y,
                                                     const uint8_t *__restrict__ sel, const uint8_t *__restrict__ mask,
                                                     int epoch, int *__restrict__ done, int *__restrict__ pos,
                                                     int *__restrict__ ntasks)
{
    __shared__ int warp_sum[32];
    __shared__ int s_base;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const size_t nxy = (size_t)N_x * N_y;
    if (threadIdx.x == 0) s_base = 0;
    __syncthreads();
    for (int k0 = 0; k0 < n; k0 += blockDim.x) {
        const int k = k0 + threadIdx.x;
        bool take = false;
        int id = -1;
        if (k < n) {
            id = order[k];
            const SvTask t = tasks[id];
            const uint8_t *sp = sel + (size_t)t.plane * nxy;
            for (int y = t.j0; y < min(N_y, t.j0 + S) && !take; y++)
                for (int x = t.k0; x < min(N_x, t.k0 + S); x++) {
                    const size_t l = (size_t)y * N_x + x;
                    if (sp[l] && mask[l] == 1) {
                        take = true;
                        break;
                    }
                }
        }
        const unsigned bal = __ballot_sync(0xffffffffu, take);
        if (lane == 0) warp_sum[warp] = __popc(bal);
        __syncthreads();
        int before = s_base;
        for (int w = 0; w < warp; w++) before += warp_sum[w];
        if (take) pos[before + __popc(bal & ((1u << lane) - 1u))] = k;
        else if (id >= 0) done[id] = epoch;
        __syncthreads();
        if (threadIdx.x == 0) {
            int tot = 0;
            for (int w = 0; w < nw; w++) tot += warp_sum[w];
            s_base += tot;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *ntasks = s_base;
}

}  // namespace

cudaError_t mbir_launch_vsc_threshold(const float *filt, int planes, int n, const int *nsel, float *thresh,
                                      uint8_t *sel, int *count, cudaStream_t s)
{
    if (planes <= 0) return cudaSuccess;
    k_vsc_threshold<<<planes, 1024, 0, s>>>(filt, n, nsel, thresh, sel, count);
    return cudaGetLastError();
}

cudaError_t mbir_launch_sv_nh_list(const int *order, int n, const SvTask *tasks, int S, int N_x, int N_y,
                                   const uint8_t *sel, const uint8_t *mask, int epoch, int *done, int *pos,
                                   int *ntasks, cudaStream_t s)
{
    k_sv_nh_list<<<1, 1024, 0, s>>>(order, n, tasks, S, N_x, N_y, sel, mask, epoch, done, pos, ntasks);
    return cudaGetLastError();
}
