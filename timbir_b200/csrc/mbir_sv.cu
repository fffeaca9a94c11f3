// Super-voxel-parallel ICD kernel (sm_100a).
//
// One CTA owns a super-voxel (SV): an S x S block of voxel lines of one
// frame and a group of nz consecutive slices.  It stages into shared memory
//   * the error-sinogram and weight band the SV touches: for each view of the
//     frame, the W consecutive detector columns [rlo_p, rlo_p + W) that cover
//     every voxel of the block, for each detector row of the slices, as
//     (e, sqrt(w)) pairs;
//   * the block's voxels with a one-voxel halo, and the temporal neighbours;
// then performs exact ICD steps on its voxels -- theta1/theta2 with the
// generalized-Huber weights over the band (XT_VoxUpdate.c:43-115), the
// qGGMRF surrogate step with over-relaxation (XT_ICD_update.c:134-183) --
// and finally adds the band's change back to the global error sinogram with
// atomics, so that SVs running concurrently on other CTAs compose.
//
// Inside the CTA, `vsplit` warps own slice z of the group (each a share of
// the frame's views): they walk the SV's lines one step at a time, and the
// slices of odd parity lag one line behind the even ones, so a voxel's
// z-neighbours are never being updated while it is; lines are ordered by
// their 2x2 (x, y) parity class, so consecutive lines are never x-y
// neighbours (where the last line of one class and the first of the next
// would be, a later line of the class is moved to the front, or failing that
// an idle step separates them).  Only slice z's warps touch slice z's band
// rows, and each view is always handled by the same lane, so error-sinogram
// updates need no synchronisation; the warps of one slice combine theta through shared
// memory and a named barrier; one CTA barrier per line step hands the
// updated voxels and the next line's A-matrix column to all warps.
//
// A-matrix columns reach a ring of R shared-memory slots either from the
// stage's column cache in HBM (cp.async, R - 2 lines ahead, every thread
// copying a share) or, when the cache does not fit, from producer warps that
// compute the next line's column (exact FP64 bin arithmetic) while the
// consumer warps update voxels.
//
// CTAs are persistent: each takes SVs from a device work queue (host-sorted
// by decreasing work) until the queue of the launch is empty.
//
// Concurrent SVs are chosen by the host so that no two share a prior
// neighbourhood (2x2 SV checkerboard, z-group and frame parity); they may
// share error-sinogram entries, whose concurrent changes they see at their
// next visit (the super-voxel ICD scheme of Wang et al., "High performance
// model based image reconstruction", PPoPP 2016).
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>

#include "mbir_internal.h"
#include "mbir_sv.h"

namespace {

__device__ __forceinline__ double vx(const MbirGeom &g, int col)
{
    return __dadd_rn(g.x0, __dmul_rn((double)col + 0.5, g.delta_xy));
}
__device__ __forceinline__ double vy(const MbirGeom &g, int row)
{
    return __dadd_rn(g.y0, __dmul_rn((double)row + 0.5, g.delta_xy));
}

// floor(a / b) for b > 0, bit-exact with the IEEE quotient: the product with
// the reciprocal is exact enough away from integers; near one the true
// quotient decides.
__device__ __forceinline__ int floor_div(double a, double b, double inv_b)
{
    const double q = __dmul_rn(a, inv_b);
    const double f = floor(q);
    const double fr = q - f;
    if (fr < 1e-9 || fr > 1.0 - 1e-9) return (int)floor(__ddiv_rn(a, b));
    return (int)f;
}

// Sums four values over the warp by reduce-scatter (six shuffles): the
// total of value j ends in lanes 8j .. 8j + 7.
__device__ __forceinline__ float warp_reduce_scatter4(float v0, float v1, float v2, float v3, int lane)
{
    const bool h16 = lane & 16, h8 = lane & 8;
    float k0 = h16 ? v2 : v0, k1 = h16 ? v3 : v1;
    const float s0 = h16 ? v0 : v2, s1 = h16 ? v1 : v3;
    k0 += __shfl_xor_sync(0xffffffffu, s0, 16);
    k1 += __shfl_xor_sync(0xffffffffu, s1, 16);
    float k = h8 ? k1 : k0;
    k += __shfl_xor_sync(0xffffffffu, h8 ? k0 : k1, 8);
    k += __shfl_xor_sync(0xffffffffu, k, 4);
    k += __shfl_xor_sync(0xffffffffu, k, 2);
    k += __shfl_xor_sync(0xffffffffu, k, 1);
    return k;
}

__device__ __forceinline__ uint32_t hash32(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

__device__ __forceinline__ void named_barrier(int id, int count)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

__device__ __forceinline__ int ld_acquire(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
// Once one wait of the launch has given up (err bits 4 or 8), the others
// stop waiting too (checked every 1024 polls), so that a broken dependency
// costs one wait limit, not one per super-voxel.
__device__ __forceinline__ bool wait_abandoned(const int *err, int spins)
{
    return (spins & 1023) == 1023 && (*(volatile const int *)err & 12) != 0;
}

__device__ __forceinline__ void st_release(int *p, int v)
{
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// 2^x and 1/x by the SFU approximations (a few ulp; the prior's weights and
// the surrogate step need no more)
__device__ __forceinline__ float ex2_approx(float x)
{
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_approx(float x)
{
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ void red_add_v4(float *p, float a, float b, float c, float d)
{
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(a), "f"(b), "f"(c), "f"(d)
                 : "memory");
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
// waits until at most N of this thread's commit groups are pending
template <int N>
__device__ __forceinline__ void cp_async_wait_upto()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Exact A-matrix column of the voxel line centred at (x, y) for one view
// (calcAMatrixColumnforAngle, XT_AMatrix.c:50-110): detector columns
// floor((r -+ delta_xy - R0) / delta_r) clipped to the detector, value = the
// view's detector response interpolated at |r - r_j| / OffsetR, kept where
// positive.  Kept columns are consecutive (the response decreases with
// distance); the entry records the first, j0, the span n and n values
// (stored format of SvACache).  Returns false if the span exceeds amax.
template <int AMAXC>
__device__ __forceinline__ bool acol_entry(const MbirGeom &g, double x, double y, double c, double s,
                                           const float *__restrict__ H, double inv_dr, double inv_off,
                                           float inv_off_f, int amax, int nwd, int *__restrict__ dst)
{
    const double r = __dsub_rn(__dmul_rn(x, c), __dmul_rn(y, s));
    const double rmin = __dsub_rn(r, g.delta_xy), rmax = __dadd_rn(r, g.delta_xy);
    int j0 = 0, n = 0;
    bool ok = true;
    float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f;
    if (!(rmax < g.R0 || rmin > g.RMax)) {
        int imin = floor_div(__dsub_rn(rmin, g.R0), g.delta_r, inv_dr);
        int imax = floor_div(__dsub_rn(rmax, g.R0), g.delta_r, inv_dr);
        if (imax >= g.N_r) imax = g.N_r - 1;
        if (imin < 0) imin = 0;
        for (int j = imin; j <= imax; j++) {
            const double rc = __dadd_rn(g.R0, __dmul_rn((double)j + 0.5, g.delta_r));
            const double dr = fabs(__dsub_rn(r, rc));
            const int id = floor_div(dr, g.OffsetR, inv_off);
            if (id >= 0 && id < MBIR_RESP_BINS) {
                const double w1 = __dsub_rn(dr, __dmul_rn((double)id, g.OffsetR));
                const double w2 = __dsub_rn(g.OffsetR, w1);
                const double num =
                    __dadd_rn(__dmul_rn(w2, (double)__ldg(H + id)), __dmul_rn(w1, (double)__ldg(H + id + 1)));
                if (num > 0) {
                    if (n == 0) j0 = j;
                    const int k = j - j0;
                    if (k >= amax) {
                        ok = false;
                        break;
                    }
                    const float a = (float)__ddiv_rn(num, g.OffsetR);
                    if constexpr (AMAXC == 3) {
                        if (k == 0) a0 = a;
                        else if (k == 1) a1 = a;
                        else a2 = a;
                    } else {
                        for (; n < k; n++) dst[1 + n] = 0;  // a gap (not produced by a decreasing response)
                        dst[1 + k] = __float_as_int(a);
                    }
                    n = k + 1;
                }
            }
        }
    }
    if constexpr (AMAXC == 3) {
        *reinterpret_cast<int4 *>(dst) =
            make_int4(j0 | (n << 16), __float_as_int(a0), __float_as_int(a1), __float_as_int(a2));
    } else {
        for (int k = n; k < nwd - 1; k++) dst[1 + k] = 0;
        dst[0] = j0 | (n << 16);
    }
    return ok;
}

// theta1/theta2 contribution of one band entry (e, sqrt(w)) with A value a:
// weight w where |e sqrt(w)| < T (ProjSelect), else T delta sqrt(w) / |e|
// (XT_VoxUpdate.c:62-84).
__device__ __forceinline__ void theta_acc(float2 es, float a, float hT, float hTd, float &t1, float &t2)
{
    const float e = es.x, sw = es.y;
    float om = sw * sw;
    if (!(fabsf(e * sw) < hT)) om = __fdividef(hTd * sw, fabsf(e));
    const float ao = a * om;
    t2 = fmaf(a, ao, t2);
    t1 = fmaf(-e, ao, t1);
}

// Fills the column cache: one warp per in-mask line, lanes over views.
// HALF: the full-resolution entries in 8 bytes (see SvACache).
template <int AMAXC, bool HALF>
__global__ void __launch_bounds__(256) k_acache(MbirGeom g, const uint8_t *__restrict__ mask, int amax, int eq,
                                                 int4 *__restrict__ cache, int *err)
{
    const int lane = threadIdx.x & 31;
    const long long line = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (line >= (long long)g.N_y * g.N_x || mask[line] != 1) return;
    const int row = (int)(line / g.N_x), col = (int)(line - (long long)row * g.N_x);
    const double x = vx(g, col), y = vy(g, row);
    const double inv_dr = 1.0 / g.delta_r, inv_off = 1.0 / g.OffsetR;
    const float inv_off_f = (float)inv_off;
    bool ok = true;
    if constexpr (HALF) {
        uint2 *dst = reinterpret_cast<uint2 *>(cache) + (size_t)line * g.N_p;
        for (int p = lane; p < g.N_p; p += 32) {
            int4 e;
            ok &= acol_entry<3>(g, x, y, g.cosv[p], g.sinv[p], g.H_r + (size_t)p * (MBIR_RESP_BINS + 1), inv_dr,
                                inv_off, inv_off_f, 3, 4, reinterpret_cast<int *>(&e));
            const unsigned j0 = (unsigned)e.x & 0xfffu, n = ((unsigned)e.x >> 16) & 3u;
            const unsigned h0 = __half_as_ushort(__float2half_rn(__int_as_float(e.y)));
            const unsigned h1 = __half_as_ushort(__float2half_rn(__int_as_float(e.z)));
            const unsigned h2 = __half_as_ushort(__float2half_rn(__int_as_float(e.w)));
            dst[p] = make_uint2(j0 | n << 12 | h0 << 16, h1 | h2 << 16);
        }
    } else {
        int4 *dst = cache + (size_t)line * g.N_p * eq;
        for (int p = lane; p < g.N_p; p += 32)
            ok &= acol_entry<AMAXC>(g, x, y, g.cosv[p], g.sinv[p], g.H_r + (size_t)p * (MBIR_RESP_BINS + 1), inv_dr,
                                    inv_off, inv_off_f, amax, 4 * eq, reinterpret_cast<int *>(dst + (size_t)p * eq));
    }
    if (!ok) atomicOr(err, 2);
}

// Forward projection (initErrorSinogam / forward_project_voxel_AMat1D,
// XT_ICD_update.c:655-716, XT_ForwardProject.c:8-25), gathered and
// deterministic: a CTA owns one view, a chunk of up to ZC slices and up to
// BPT * Tg detector columns, and walks the image rows (or columns, whichever
// the view's detector direction crosses faster), split over G thread groups
// of Tg threads (rows g, g + G, ...).  For each of its rows a group first
// computes the exact A-matrix column of every voxel with a non-zero value in
// the chunk into its shared buffer, with the voxel values; then each thread
// adds, for each of its detector columns j, a x over the row's voxels whose
// column includes j -- candidates are the voxels whose centre projects within
// delta_xy of column j's extent, widened by one voxel each side; the stored
// column decides.  FP32 sums, as the reference accumulates the projection
// into its float error sinogram (XT_ForwardProject.c:22); the groups' sums
// are added in group order at the end.  No atomics.
template <int AMAXC, int BPT, int ZC>
__global__ void __launch_bounds__(512, 2) k_forward_rows(MbirGeom g, const int *__restrict__ frame_of_view,
                                                       const float *__restrict__ x, const float *__restrict__ y,
                                                       const float *__restrict__ d, float *__restrict__ out, int mode,
                                                       int amax, int eq, int G)
{
    extern __shared__ __align__(16) unsigned char fsm[];
    const int p = blockIdx.x, z0 = blockIdx.y * ZC, nzc = min(ZC, g.N_z - z0);
    const int Tg = blockDim.x / G, grp = threadIdx.x / Tg, tid = threadIdx.x - grp * Tg;
    const int jbase = blockIdx.z * Tg * BPT;
    const double c = g.cosv[p], sn = g.sinv[p];
    const bool rows = fabs(c) >= fabs(sn);
    const int nouter = rows ? g.N_y : g.N_x, ninner = rows ? g.N_x : g.N_y;
    const int nwd = 4 * eq;
    const size_t gbytes = (sizeof(int4) * (size_t)eq + sizeof(float) * ZC) * ninner;  // one group's buffer
    int4 *ent = reinterpret_cast<int4 *>(fsm + grp * gbytes);                     // [ninner][eq]
    float *xsm = reinterpret_cast<float *>(fsm + grp * gbytes + sizeof(int4) * (size_t)eq * ninner);  // [ZC][ninner]
    float acc[BPT][ZC];
#pragma unroll
    for (int b = 0; b < BPT; b++)
#pragma unroll
        for (int s = 0; s < ZC; s++) acc[b][s] = 0.0f;
    const int f = frame_of_view[p];
    if (f >= 0) {
        const size_t plane = (size_t)g.N_y * g.N_x;
        const float *xs = x + ((size_t)f * g.N_z + z0) * plane;
        const double inv_dr = 1.0 / g.delta_r, inv_off = 1.0 / g.OffsetR;
        const float *H = g.H_r + (size_t)p * (MBIR_RESP_BINS + 1);
        for (int o = grp; o < nouter; o += G) {
            const double oc = rows ? vy(g, o) : vx(g, o);
            for (int i = tid; i < ninner; i += Tg) {
                const int line = rows ? o * g.N_x + i : i * g.N_x + o;
                bool any = false;
#pragma unroll
                for (int s = 0; s < ZC; s++) {
                    const float v = s < nzc ? __ldg(xs + s * plane + line) : 0.0f;
                    xsm[s * ninner + i] = v;
                    any |= v != 0.0f;
                }
                int *dst = reinterpret_cast<int *>(ent + (size_t)i * eq);
                if (!any)
                    dst[0] = 0;
                else if (!acol_entry<AMAXC>(g, rows ? vx(g, i) : oc, rows ? oc : vy(g, i), c, sn, H, inv_dr, inv_off,
                                            0.0f, amax, nwd, dst))
                    dst[0] = 0;  // wider than amax: cannot occur for 2 mult_xy + 1 columns
            }
            named_barrier(1 + grp, Tg);
#pragma unroll
            for (int b = 0; b < BPT; b++) {
                const int j = jbase + b * Tg + tid;
                if (j >= g.N_r) continue;
                // rows: xc in [(lo + yc sin) / cos, (hi + yc sin) / cos];
                // columns: yc in [(xc cos - hi) / sin, (xc cos - lo) / sin]
                const double lo = g.R0 + (double)j * g.delta_r - g.delta_xy;
                const double hi = g.R0 + (double)(j + 1) * g.delta_r + g.delta_xy;
                double a0 = rows ? (lo + oc * sn) / c : (oc * c - hi) / sn;
                double a1 = rows ? (hi + oc * sn) / c : (oc * c - lo) / sn;
                if (a0 > a1) {
                    const double t = a0;
                    a0 = a1;
                    a1 = t;
                }
                const double base = rows ? g.x0 : g.y0;
                const int i0 = max((int)floor((a0 - base) / g.delta_xy - 0.5) - 1, 0);
                const int i1 = min((int)ceil((a1 - base) / g.delta_xy - 0.5) + 1, ninner - 1);
                for (int i = i0; i <= i1; i++) {
                    const int *e = reinterpret_cast<const int *>(ent + (size_t)i * eq);
                    const int h = e[0], k = j - (h & 0xffff);
                    if (k < 0 || k >= (h >> 16)) continue;
                    const float a = __int_as_float(e[1 + k]);
#pragma unroll
                    for (int s = 0; s < ZC; s++) acc[b][s] = fmaf(a, xsm[s * ninner + i], acc[b][s]);
                }
            }
            named_barrier(1 + grp, Tg);
        }
    }
    // groups' sums, added in group order
    __syncthreads();
    float *red = reinterpret_cast<float *>(fsm);  // [G][BPT][ZC][Tg]
#pragma unroll
    for (int b = 0; b < BPT; b++)
#pragma unroll
        for (int s = 0; s < ZC; s++) red[((size_t)(grp * BPT + b) * ZC + s) * Tg + tid] = acc[b][s];
    __syncthreads();
    if (grp != 0) return;
#pragma unroll
    for (int b = 0; b < BPT; b++) {
        const int j = jbase + b * Tg + tid;
        if (j >= g.N_r) continue;
#pragma unroll
        for (int s = 0; s < ZC; s++) {
            if (s >= nzc) break;
            float ax = 0.0f;
            for (int q = 0; q < G; q++) ax += red[((size_t)(q * BPT + b) * ZC + s) * Tg + tid];
            for (int rr = 0; rr < g.m_z; rr++) {
                const int t = (z0 + s) * g.m_z + rr;
                const size_t o = ((size_t)t * g.N_p + p) * g.N_r + j;
                if (mode == 0)
                    out[o] = __fsub_rn(__fsub_rn(y[o], ax), d[(size_t)t * g.N_r + j]);
                else
                    out[o] = ax;
            }
        }
    }
}

template <int AMAXC, int BPT, int ZC>
cudaError_t launch_forward_rows(const MbirGeom &g, const int *fov, const float *x, const float *y, const float *d,
                                float *out, int mode, int amax, cudaStream_t s)
{
    const int eq = (1 + amax + 3) / 4;
    const int per = BPT == 2 ? (g.N_r + 1) / 2 : g.N_r;
    const int Tg = std::min(128, std::max(64, (per + 31) / 32 * 32));
    const int ninner = std::max(g.N_x, g.N_y);
    const size_t gbytes = (sizeof(int4) * (size_t)eq + sizeof(float) * ZC) * ninner;
    // up to four groups whose row buffers fit 200 KB; the final sums reuse the space
    const int G = (int)std::max<size_t>(1, std::min<size_t>(4, (200 * 1024) / gbytes));
    const size_t sm = std::max(G * gbytes, sizeof(float) * G * BPT * ZC * Tg);
    cudaError_t e =
        cudaFuncSetAttribute(k_forward_rows<AMAXC, BPT, ZC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    dim3 grid(g.N_p, (g.N_z + ZC - 1) / ZC, (g.N_r + Tg * BPT - 1) / (Tg * BPT));
    k_forward_rows<AMAXC, BPT, ZC><<<grid, G * Tg, sm, s>>>(g, fov, x, y, d, out, mode, amax, eq, G);
    return cudaGetLastError();
}

// AMAXC: entries per (line, view) known at compile time (3 at full
// resolution), 0 = runtime sp.amax.  MZC: detector rows per slice known at
// compile time (1 at full resolution), 0 = runtime m_z.  AC: columns come
// from the column cache (else from producer warps).  MAXT: most threads per
// CTA (512 leaves 128 registers per thread).  AC = 2: the cache holds FP16
// values (8-byte entries, full resolution only).  VU (full-resolution path): a
// lane's views per slice, at most VU, are held in registers from theta to
// the error-sinogram update.
// The problem a task runs on: the launch's own (a kernel parameter) or, in
// a batched launch, the CTA's shared-memory copy of the task's problem.
template <bool B>
__device__ __forceinline__ const SvProblem *pick_problem(const unsigned char *shared_copy, const SvProblem *param)
{
    if constexpr (B)
        return reinterpret_cast<const SvProblem *>(shared_copy);
    else
        return param;
}

template <int AMAXC, int MZC, int AC, int MAXT, int VU, bool BATCH>
__global__ void __launch_bounds__(MAXT) k_icd_sv(const __grid_constant__ SvProblem P0,
                                                  const SvLaunch L, int *queue, float *__restrict__ scratch,
                                                  size_t scratch_floats, SvTaskOut *__restrict__ out, int iter_arg,
                                                  uint32_t seed_arg, int *err)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ __align__(16) unsigned char s_prob[BATCH ? sizeof(SvProblem) : 16];
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nwarps = nthr >> 5;
    constexpr int kHalf = AC == 2;

    __shared__ int s_nlines, s_task, s_bad;
    __shared__ float s_red[32][4];

    // a batched launch's iteration number comes from the device (so that one
    // captured graph serves every iteration); it is also the epoch of the
    // done flags and varies the line order
    const int epoch = BATCH ? __ldcg(L.ctl) : L.epoch;
    const int iter = BATCH ? epoch : iter_arg;
    const uint32_t seed = BATCH ? hash32(seed_arg ^ ((uint32_t)epoch * 0x9E3779B9u)) : seed_arg;
    float sum_abs_dx = 0.0f, sum_abs_x = 0.0f;
    int n_upd = 0, n_skip = 0;
    // statistics of the CTA's updates since the last call (lane 0 of each
    // slice's first warp counts) into *o; every thread calls it
    auto flush_stats = [&](SvTaskOut *o) {
        if (lane == 0) {
            s_red[warp][0] = sum_abs_dx;
            s_red[warp][1] = sum_abs_x;
            s_red[warp][2] = (float)n_upd;
            s_red[warp][3] = (float)n_skip;
        }
        __syncthreads();
        if (tid == 0) {
            double d0 = 0, d1 = 0, d2 = 0, d3 = 0;
            for (int w = 0; w < nwarps; w++) {
                d0 += s_red[w][0];
                d1 += s_red[w][1];
                d2 += s_red[w][2];
                d3 += s_red[w][3];
            }
            atomicAdd(&o->sum_abs_dx, d0);
            atomicAdd(&o->sum_abs_x, d1);
            atomicAdd((unsigned long long *)&o->updates, (unsigned long long)d2);
            atomicAdd((unsigned long long *)&o->zero_skips, (unsigned long long)d3);
        }
        sum_abs_dx = sum_abs_x = 0.0f;
        n_upd = n_skip = 0;
    };
    int cur = -1;  // problem held in s_prob (batched launches)
    // a subset pass takes its length from the device (written by the kernel
    // that chose the subset, earlier on the stream)
    const int ntasks = L.ntasks_dev ? min(*L.ntasks_dev, L.ntasks) : L.ntasks;

    for (;;) {
        __syncthreads();
        if (tid == 0) {
            s_task = atomicAdd(queue, 1);
            s_bad = 0;
        }
        __syncthreads();
        const int tix0 = s_task;
        if (tix0 >= ntasks) break;
        // position in the order / dependency lists
        const int tix = L.pos ? L.pos[tix0] : tix0;
        const int id = L.order[tix];
        const SvTask task = L.tasks[id];
        if constexpr (BATCH) {
            if (task.prob != cur) {
                cur = task.prob;
                const long long *src = reinterpret_cast<const long long *>(L.problems + cur);
                long long *dst = reinterpret_cast<long long *>(s_prob);
                for (int q = tid; q < (int)(sizeof(SvProblem) / sizeof(long long)); q += nthr) dst[q] = src[q];
                __syncthreads();
            }
            // a problem that has stopped iterating: skip its super-voxels
            if (!__ldcg(&L.state[cur].active)) {
                if (tid == 0) st_release(L.done + id, epoch);
                continue;
            }
        }
        const SvProblem &P = *pick_problem<BATCH>(s_prob, &P0);
        const MbirGeom &g = P.g;
        const MbirPrior &pr = P.pr;
        const MbirDev &dv = P.dv;
        const SvParams &sp = P.sp;
        const SvACache ac = P.ac;
        // ---- carve shared memory (the problem's region sizes) ----
        const SvPlan &pl = P.plan;
        unsigned char *p = smraw;
        int4 *ring = reinterpret_cast<int4 *>(p); p += pl.ring_bytes;
        float2 *band = reinterpret_cast<float2 *>(p); p += sizeof(float2) * (size_t)pl.band_pairs;
        double *cs = reinterpret_cast<double *>(p);
        double *sn = cs + pl.trig_views;
        p += 2 * sizeof(double) * pl.trig_views;
        float *xb = reinterpret_cast<float *>(p); p += sizeof(float) * pl.xb;
        float *tb = reinterpret_cast<float *>(p); p += sizeof(float) * pl.tb;
        // |dx| of each (slice, line) at this visit; summed over the slices in
        // slice order at write-back (the line's magnitude-map entry)
        float *magl = reinterpret_cast<float *>(p); p += sizeof(float) * pl.magl;
        float *part = reinterpret_cast<float *>(p); p += sizeof(float) * pl.part;
        int *vidx = reinterpret_cast<int *>(p); p += sizeof(int) * pl.views;
        int *rlo = reinterpret_cast<int *>(p); p += sizeof(int) * pl.views;
        // step sequence: lx | ly << 8 of the line, or -1 for an idle step
        int *order = reinterpret_cast<int *>(p);
        const int S = sp.S, W = sp.W, vsplit = sp.vsplit;
        const int amax = AMAXC > 0 ? AMAXC : sp.amax;
        const int eq = AMAXC > 0 ? (AMAXC + 4) / 4 : sp.eq;
        const int nwd = 4 * eq;  // words per ring entry
        const int mz = MZC > 0 ? MZC : g.m_z;
        const int NpS = sp.max_views;  // smem stride (views)
        const int S2 = S + 2;
        const size_t rowstride = (size_t)W * NpS;  // band entries per detector row
        // ring slots (the host always plans 4) and column prefetch distance (lines)
        constexpr int R = kSvRing, D = kSvRing - 2;
        const double inv_dr = 1.0 / g.delta_r, inv_off = 1.0 / g.OffsetR;
        const float inv_off_f = (float)inv_off;
        const float alpha = (float)pr.alpha, hT = (float)pr.hT, hTd = (float)(pr.hT * pr.hdelta);
        const float sSQ_inv = (float)(1.0 / pr.sSQ), sSQP_inv = (float)(1.0 / pr.sSQP), cS = (float)pr.c_s;
        const float sTQ_inv = (float)(1.0 / pr.sTQ), sTQP_inv = (float)(1.0 / pr.sTQP), cT = (float)pr.c_t;
        // warps [0, ncons) update voxels (vsplit per slice); warps [ncons, nwarps)
        // produce the next line's A-matrix column while they do (or, in a
        // batched launch, idle when the problem needs fewer warps)
        const int ncons = sp.max_nz * vsplit, nprod = nwarps - ncons;
        const bool consumer = warp < ncons;
        const int zl = consumer ? warp / vsplit : 0, vh = consumer ? warp - zl * vsplit : 0;
        // neighbour of lane: spatial (dz, dy, dx) for lanes 0..25, temporal 26, 27
        int ndz = 0, ndy = 0, ndx = 0;
        float bw = 0.0f, qinv = 0.0f, qpinv = 0.0f, cc = 1.0f;
        bool spatial = false, temporal = false;
        int nboff = 0;  // offset of the spatial neighbour in the staged block
        if (lane < 26) {
            const int n = lane < 13 ? lane : lane + 1;  // skip the centre (13)
            ndz = n / 9 - 1;
            ndy = (n / 3) % 3 - 1;
            ndx = n % 3 - 1;
            nboff = (ndz * S2 + ndy) * S2 + ndx;
            bw = (float)pr.SF[n];
            qinv = sSQ_inv;
            qpinv = sSQP_inv;
            cc = cS;
            spatial = true;
        } else if (lane < 28) {
            bw = (float)pr.TF;
            qinv = sTQ_inv;
            qpinv = sTQP_inv;
            cc = cT;
            temporal = true;
        }
        // views of the A-column computation: the producer warps' (all warps
        // for the first line of a task, or when there are no producers)
        const int av_all = (NpS + nwarps - 1) / nwarps;
        const int av_prod = nprod > 0 ? (NpS + nprod - 1) / nprod : 0;

        const int nz = task.nz, rows = nz * mz;
        const int i = task.frame;
        const int Np = g.view_num[i];
        // (row, view) of a band pair index pq < rows Np: pq / Np as a multiply
        // by ceil(2^32 / Np) and the high word, exact while rows Np^2 < 2^32
        // (then pq e < 2^32 for the rounding excess e = m Np - 2^32 < Np)
        const bool np_fast = Np > 1 && (unsigned long long)rows * Np * Np < (1ull << 32);
        const unsigned np_magic = np_fast ? 0xFFFFFFFFu / (unsigned)Np + 1u : 1u;
        auto div_np = [&](int pq) -> int { return np_fast ? (int)__umulhi((unsigned)pq, np_magic) : pq / Np; };
        const int k0 = task.k0, j0 = task.j0, z0 = task.z0;
        const int kx = min(S, g.N_x - k0), ky = min(S, g.N_y - j0);
        const int *vl = g.view_idx + (size_t)i * g.max_views;
        const bool active = consumer && zl < nz;
        const int zg = z0 + zl;

        // ---- views, trig, band origin per view; the band must hold every
        //      column of every line (the corners bound r) ----
        for (int v = tid; v < Np; v += nthr) {
            const int view = vl[v];
            vidx[v] = view;
            const double c = g.cosv[view], s = g.sinv[view];
            if (!AC) {
                cs[v] = c;
                sn[v] = s;
            }
            int lo = 1 << 30, hi = -(1 << 30);
            const double xs[2] = {vx(g, k0), vx(g, k0 + kx - 1)};
            const double ys[2] = {vy(g, j0), vy(g, j0 + ky - 1)};
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const double r = __dsub_rn(__dmul_rn(xs[u & 1], c), __dmul_rn(ys[u >> 1], s));
                lo = min(lo, floor_div(__dsub_rn(__dsub_rn(r, g.delta_xy), g.R0), g.delta_r, inv_dr));
                hi = max(hi, floor_div(__dsub_rn(__dadd_rn(r, g.delta_xy), g.R0), g.delta_r, inv_dr));
            }
            lo = max(lo, 0);
            hi = min(hi, g.N_r - 1);
            rlo[v] = lo;
            if (hi - lo >= W) {
                atomicOr(err, 1);
                s_bad = 1;
            }
        }
        // the views' band origins are read by every warp below
        __syncthreads();
        // Warp 0 waits for the conflicting super-voxels; warp 1 (warp 0
        // after its waits when the CTA has one warp) orders the lines while
        // the other warps, released by warp 0 through barrier 1 (free
        // outside the line steps), stage the band and the voxel block.
        auto order_lines = [&]() {
            // in-mask bit of line q = 32 k + lane in bit k (all loads in flight
            // at once); a subset pass keeps the selected lines only
            const uint8_t *lsel = L.sel ? L.sel + (size_t)task.plane * g.N_y * g.N_x : nullptr;
            unsigned mbits = 0;
            for (int k = 0; 32 * k < S * S; k++) {
                const int q = 32 * k + lane;
                const int lx = q % S, ly = q / S;
                const size_t l = (size_t)(j0 + ly) * g.N_x + k0 + lx;
                if (q < S * S && lx < kx && ly < ky && dv.mask[l] == 1 && (!lsel || lsel[l]))
                    mbits |= 1u << k;
            }
            int n = 0;
            for (int cls = 0; cls < 4; cls++) {
                const int base = n;
                for (int q0 = 0; q0 < S * S; q0 += 32) {
                    const int q = q0 + lane;
                    const int lx = q % S, ly = q / S;
                    const bool take = ((mbits >> (q0 >> 5)) & 1u) &&
                                      ((((k0 + lx) & 1) | (((j0 + ly) & 1) << 1)) == cls);
                    const unsigned bal = __ballot_sync(0xffffffffu, take);
                    if (take) order[n + __popc(bal & ((1u << lane) - 1))] = lx | (ly << 8);
                    n += __popc(bal);
                }
                __syncwarp();
                // random order within the class: each line's rank among the
                // class's per-visit hash keys (ties by position), computed by
                // the whole warp; classes of more than 64 lines (sides above
                // 16) are shuffled by lane 0
                const int m = n - base;
                if (m > 1 && m <= 64) {
                    const int oa = lane < m ? order[base + lane] : 0;
                    const int ob = lane + 32 < m ? order[base + lane + 32] : 0;
                    const uint32_t ka = hash32(seed ^ hash32((uint32_t)tix * 1315423911u + (uint32_t)oa));
                    const uint32_t kb = hash32(seed ^ hash32((uint32_t)tix * 1315423911u + (uint32_t)ob));
                    int ra = 0, rb = 0;
                    for (int j = 0; j < m; j++) {
                        const uint32_t kj = __shfl_sync(0xffffffffu, j < 32 ? ka : kb, j & 31);
                        ra += kj < ka || (kj == ka && j < lane);
                        rb += kj < kb || (kj == kb && j < lane + 32);
                    }
                    __syncwarp();
                    if (lane < m) order[base + ra] = oa;
                    if (lane + 32 < m) order[base + rb] = ob;
                    __syncwarp();
                }
                if (lane == 0 && n > base) {
                    if (m > 64)
                        for (int q = n - 1; q > base; q--) {
                            const uint32_t h = hash32(seed ^ hash32((uint32_t)tix * 1315423911u + (uint32_t)q));
                            const int r = base + (int)(h % (uint32_t)(q - base + 1));
                            const int t = order[q];
                            order[q] = order[r];
                            order[r] = t;
                        }
                    // the odd slices lag one step: keep the previous class's last
                    // line and this class's first line apart
                    auto adjacent = [](int a, int b) {
                        return abs((a & 0xff) - (b & 0xff)) <= 1 && abs((a >> 8) - (b >> 8)) <= 1;
                    };
                    if (base > 0 && adjacent(order[base - 1], order[base])) {
                        int q = base + 1;
                        while (q < n && adjacent(order[base - 1], order[q])) q++;
                        if (q < n) {
                            const int t = order[q];
                            order[q] = order[base];
                            order[base] = t;
                        } else {
                            for (int k = n; k > base; k--) order[k] = order[k - 1];
                            order[base] = -1;
                            n++;
                        }
                    }
                }
                n = __shfl_sync(0xffffffffu, n, 0);
                __syncwarp();
            }
            if (lane == 0) s_nlines = n;
        };
        // ---- A-matrix column of line `li` (of nlines) into ring slot `slot`
        //      from the cache, copied by threads t0, t0 + tn, ... (one commit
        //      group per call and thread) ----
        auto fetch_by = [&](int li, int slot, int nlines, int t0, int tn) {
            if (li < nlines && order[li] >= 0) {
                const int o = order[li];
                const size_t line = (size_t)(j0 + (o >> 8)) * g.N_x + k0 + (o & 0xff);
                if constexpr (kHalf) {
                    uint2 *dst = reinterpret_cast<uint2 *>(ring) + (size_t)slot * NpS;
                    const uint2 *src = reinterpret_cast<const uint2 *>(ac.a) + line * g.N_p;
                    for (int q = t0; q < Np; q += tn) cp_async8(dst + q, src + vidx[q]);
                } else {
                    int4 *dst = ring + (size_t)slot * eq * NpS;
                    for (int q = t0; q < Np * eq; q += tn) {
                        const int v = q / eq, w = q - v * eq;
                        cp_async16(dst + q, ac.a + (line * g.N_p + vidx[v]) * eq + w);
                    }
                }
            }
            cp_async_commit();
        };
        const bool orderer = warp == (nwarps > 1 ? 1 : 0);
        if (warp == 0) {
            // wait for the conflicting super-voxels earlier in this launch
            // (bounded: a wait that gives up flags err and goes on)
            if constexpr (BATCH) {
                // at most cap super-voxels of the problem in flight: those
                // before this one in its order, less the finished ones
                const int need = L.seq[tix] + 1 - P.cap;
                if (lane == 0 && need > 0)
                    for (int spins = 0; ld_acquire(&L.state[cur].fin) < need; spins++) {
                        if (spins > (1 << 22) || wait_abandoned(err, spins)) {
                            atomicOr(err, 8);
                            break;
                        }
                        __nanosleep(100);
                    }
                __syncwarp();
            }
            for (int d = L.dep_off[tix] + lane; d < L.dep_off[tix + 1]; d += 32) {
                const int *flag = L.done + L.deps[d];
                for (int spins = 0; ld_acquire(flag) != epoch; spins++) {
                    if (spins > (1 << 22) || wait_abandoned(err, spins)) {
                        atomicOr(err, 4);
                        break;
                    }
                    __nanosleep(100);
                }
            }
        }
        if (orderer) order_lines();
        // with a column cache and more than one warp, the orderer also starts
        // the first D lines' columns while the others stage (the other
        // threads' later waits find none of these groups of theirs pending)
        const bool early = AC && nwarps > 1 && orderer;
        if (early) {
            __syncwarp();
            const int n0 = s_bad ? 0 : s_nlines;
            for (int q = 0; q < D; q++) fetch_by(q, q, n0, lane, 32);
        }
        for (int q = tid; q < sp.max_nz * S * S; q += nthr) magl[q] = 0.0f;
        // staging warps: all but warp 1 (all of one warp)
        const int sw_n = nwarps > 1 ? nwarps - 1 : 1, sw = warp < 2 ? 0 : warp - 1;
        const int st_n = sw_n * 32;
        const bool stager = nwarps == 1 || !orderer;
        const int st_first = stager ? sw * 32 + lane : (1 << 30);  // past every loop's end: no share
        const int sw_first = stager ? sw : (1 << 30);
        if (nwarps > 1 && !orderer) named_barrier(1, st_n);
        int nl = 0;  // the task's lines, read after the barrier that follows the ordering

        // ---- stage the band: (e, sqrt(w)) pairs, e also to this CTA's
        //      scratch slot.  Four lanes serve a (detector row, view), each
        //      every fourth 16-byte-aligned word of the W columns (rows of
        //      N_r % 4 == 0 are 16-byte aligned; words starting past the row
        //      end stage zeros) ----
        float *__restrict__ scr = scratch + (size_t)blockIdx.x * scratch_floats;
        const bool vec = (g.N_r & 3) == 0;
        const int nw = sv_scratch_words(W);  // 16-byte words of e kept per pair
        const int npairs = rows * Np;
        if (vec) {
            // one 16-byte word of a (row, view): pqc = 4 (row Np + v) + c
            // the scratch keeps each staged word of e as loaded, word c of
            // pair pq at float4 index pq nw + c, for the commit's changes
            auto stage_word = [&](int pq, int c, float4 ev, float4 wv) {
                const int row = div_np(pq), v = pq - row * Np;
                const int sh = rlo[v] & 3;
                const float ee[4] = {ev.x, ev.y, ev.z, ev.w};
                const float ww[4] = {wv.x, wv.y, wv.z, wv.w};
                float2 *bd = band + (size_t)row * rowstride + v;
                reinterpret_cast<float4 *>(scr)[(size_t)pq * nw + c] = ev;
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int off = 4 * c + j - sh;
                    if (off >= 0 && off < W) bd[(size_t)off * NpS] = make_float2(ee[j], sqrtf(ww[j]));
                }
            };
            // global address of word c of pair pq (-1: past the band or the row)
            auto word_at = [&](int pq, int c) -> long long {
                const int row = div_np(pq), v = pq - row * Np;
                const int lo = rlo[v], a0 = lo & ~3;
                if (4 * c >= (lo - a0) + W || a0 + 4 * c >= g.N_r) return -1;
                return (long long)((size_t)(z0 * mz + row) * g.N_p + vidx[v]) * g.N_r + a0 + 4 * c;
            };
            // words 0-3 of every pair, four per thread in flight at once
            constexpr int U = 4;
            const int stride = st_n, total = 4 * npairs;
            for (int b = st_first; b < total; b += U * stride) {
                float4 ev[U], wv[U];
                long long at[U];
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const int pqc = b + u * stride;
                    at[u] = pqc < total ? word_at(pqc >> 2, pqc & 3) : -2;
                    ev[u] = wv[u] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    if (at[u] >= 0) {
                        ev[u] = __ldcg(reinterpret_cast<const float4 *>(dv.e + at[u]));
                        wv[u] = __ldcg(reinterpret_cast<const float4 *>(dv.w + at[u]));
                    }
                }
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const int pqc = b + u * stride;
                    if (at[u] != -2) stage_word(pqc >> 2, pqc & 3, ev[u], wv[u]);
                }
            }
            // words 4 and up (bands wider than 13 columns)
            if (W + 3 > 16)
                for (int pqc = st_first; pqc < total; pqc += stride)
                    for (int c = (pqc & 3) + 4; 4 * c < W + 3; c += 4) {
                        const long long a = word_at(pqc >> 2, c);
                        float4 ev = make_float4(0.0f, 0.0f, 0.0f, 0.0f), wv = ev;
                        if (a >= 0) {
                            ev = __ldcg(reinterpret_cast<const float4 *>(dv.e + a));
                            wv = __ldcg(reinterpret_cast<const float4 *>(dv.w + a));
                        }
                        stage_word(pqc >> 2, c, ev, wv);
                    }
        } else {
            for (int pq = st_first; pq < npairs; pq += st_n) {
                const int row = div_np(pq), v = pq - row * Np;
                const int lo = rlo[v];
                const size_t rbase = ((size_t)(z0 * mz + row) * g.N_p + vidx[v]) * g.N_r;
                float2 *bd = band + (size_t)row * rowstride + v;
                float *sc = scr + (size_t)row * rowstride + v;
                for (int off = 0; off < W; off++) {
                    const int r = lo + off;
                    const float e = r < g.N_r ? __ldcg(dv.e + rbase + r) : 0.0f;
                    const float w = r < g.N_r ? __ldg(dv.w + rbase + r) : 0.0f;
                    bd[(size_t)off * NpS] = make_float2(e, sqrtf(w));
                    sc[(size_t)off * NpS] = e;
                }
            }
        }
        // ---- voxel block with halo, temporal neighbours ----
        const size_t plane = (size_t)g.N_y * g.N_x;
        const float *xf = dv.x + (size_t)i * g.N_z * plane;
        for (int lz = sw_first; lz < nz + 2; lz += sw_n)
            for (int q = lane; q < S2 * S2; q += 32) {
                const int lx = q % S2, ly = q / S2;
                const int xx = k0 + lx - 1, yy = j0 + ly - 1, zz = z0 + lz - 1;
                float v = 0.0f;
                if (xx >= 0 && xx < g.N_x && yy >= 0 && yy < g.N_y) {
                    if (zz >= 0 && zz < g.N_z)
                        v = __ldcg(xf + (size_t)zz * plane + (size_t)yy * g.N_x + xx);
                    else if (slab_has_z(g, dv, zz))
                        v = __ldcg(slab_plane(g, dv, i, zz) + (size_t)yy * g.N_x + xx);
                }
                xb[lz * S2 * S2 + q] = v;
            }
        for (int sz = sw_first; sz < 2 * nz; sz += sw_n) {
            const int side = sz / nz, lz = sz - side * nz;
            const int ti = i + (side == 0 ? -1 : 1);
            for (int q = lane; q < S * S; q += 32) {
                const int lx = q % S, ly = q / S;
                float v = 0.0f;
                if (ti >= 0 && ti < g.N_time && lx < kx && ly < ky)
                    v = __ldcg(dv.x + ((size_t)ti * g.N_z + z0 + lz) * plane + (size_t)(j0 + ly) * g.N_x + k0 + lx);
                tb[sz * S * S + q] = v;
            }
        }

        // ---- A-matrix column of line `li` into ring slot `slot` (li mod R) ----
        // from the cache: every thread copies a share (one commit group per call)
        auto fetch = [&](int li, int slot) { fetch_by(li, slot, nl, tid, nthr); };
        // computed: warps [w0, nwarps), av_lanes views per warp
        auto acol = [&](int li, int slot, int w0, int av_lanes) {
            const int wr = warp - w0;
            const int o = order[li];
            if (wr < 0 || o < 0) return;
            const double x = vx(g, k0 + (o & 0xff)), y = vy(g, j0 + (o >> 8));
            int *rw = reinterpret_cast<int *>(ring + (size_t)slot * eq * NpS);
            for (int l = lane; l < av_lanes; l += 32) {
                const int v = wr * av_lanes + l;
                if (v >= Np) break;
                if (!acol_entry<AMAXC>(g, x, y, cs[v], sn[v], g.H_r + (size_t)vidx[v] * (MBIR_RESP_BINS + 1),
                                       inv_dr, inv_off, inv_off_f, amax, nwd, rw + (size_t)v * nwd)) {
                    atomicOr(err, 2);
                    rw[(size_t)v * nwd] = 0;  // drop the column
                }
            }
        };

        __syncthreads();  // the line order (and the staged band and voxel block)
        nl = s_bad ? 0 : s_nlines;
        if (AC) {
            if (nwarps == 1)
                for (int q = 0; q < D; q++) fetch(q, q);
            cp_async_wait_upto<D - 1>();
        } else if (nl > 0) {
            acol(0, 0, 0, av_all);
        }
        __syncthreads();

        // the neighbour of this lane exists in z (spatial) or time (temporal)
        // for every voxel of the super-voxel; in x and y too when the block
        // keeps one voxel away from the image edges
        const bool nfix = spatial ? slab_has_z(g, dv, zg + ndz)
                                  : temporal && i + (lane == 26 ? -1 : 1) >= 0 && i + (lane == 26 ? -1 : 1) < g.N_time;
        const bool interior = k0 >= 1 && j0 >= 1 && k0 + kx < g.N_x && j0 + ky < g.N_y;
        // full resolution: this lane's views (vh * 32 + lane + 32 vsplit u, u
        // < VU) as a mask of those the frame has, and their band origins
        constexpr int VRL = VU > 0 ? VU : 1;
        int rl[VRL];
        unsigned okm = 0;
#pragma unroll
        for (int u = 0; u < VRL; u++) {
            const int v = vh * 32 + lane + u * 32 * vsplit;
            rl[u] = v < Np ? rlo[v] : 0;
            okm |= v < Np ? 1u << u : 0u;
        }
        for (int step = 0, sl = 0; step <= nl; step++, sl = sl + 1 == R ? 0 : sl + 1) {
            // sl = step mod R: the slot of line `step`; odd slices use line step - 1
            const int li = (zl & 1) ? step - 1 : step;
            const int slot = (zl & 1) ? (sl == 0 ? R - 1 : sl - 1) : sl;
            const int o = li >= 0 && li < nl ? order[li] : -1;
            if (active && o >= 0) {
                const int lx = o & 0xff, ly = o >> 8;
                const int col = k0 + lx, row = j0 + ly;
                float *xc = xb + ((zl + 1) * S2 + ly + 1) * S2 + lx + 1;
                const float V = *xc;
                // ---- prior neighbourhood ----
                float nbv = 0.0f;
                bool valid = nfix;
                if (spatial) {
                    if (!interior) {
                        const int yy = row + ndy, xx = col + ndx;
                        valid = valid && yy >= 0 && yy < g.N_y && xx >= 0 && xx < g.N_x;
                    }
                    if (valid) nbv = xc[nboff];
                } else if (valid) {
                    nbv = tb[((lane - 26) * nz + zl) * S * S + ly * S + lx];
                }
                const unsigned pos = __ballot_sync(0xffffffffu, valid && nbv > 0.0f);
                if (V == 0.0f && iter > 1 && pos == 0u) {
                    if (vh == 0 && lane == 0) n_skip++;
                } else {
                    // ---- data term over this slice's band rows, this warp's views ----
                    float th1 = 0.0f, th2 = 0.0f, th1b = 0.0f, th2b = 0.0f;
                    const int4 *rq = ring + (size_t)slot * eq * NpS;
                    const float2 *bz = band + (size_t)zl * mz * rowstride;
                    // full resolution: per view three consecutive columns from
                    // j0 (clamped into the band; absent ones carry a = 0),
                    // e kept in registers for the update.  Every entry is
                    // first summed with weight w, tracking the largest
                    // |e sqrt(w)|; only when some lane of the warp holds an
                    // entry with |e sqrt(w)| >= T (generalized Huber,
                    // XT_VoxUpdate.c:62-84) are the warp's sums recomputed
                    // with T delta sqrt(w) / |e| for those entries
                    constexpr int VR = VU > 0 ? VU : 1;
                    float ev[VR][3], av[VR][3];
                    int cx[VR][3];
                    if constexpr (AMAXC == 3 && MZC == 1) {
                        const int vstep = 32 * vsplit;
                        float pmax = 0.0f;
#pragma unroll
                        for (int u = 0; u < VR; u++) {
                            const int v = vh * 32 + lane + u * vstep;
                            const bool ok = v < Np;
                            const int vv = ok ? v : 0;
                            int j0c;
                            if constexpr (kHalf) {
                                uint2 A = make_uint2(0u, 0u);
                                if (ok) A = reinterpret_cast<const uint2 *>(ring)[(size_t)slot * NpS + vv];
                                j0c = (int)(A.x & 0xfffu);
                                av[u][0] = __half2float(__ushort_as_half((unsigned short)(A.x >> 16)));
                                av[u][1] = __half2float(__ushort_as_half((unsigned short)(A.y & 0xffffu)));
                                av[u][2] = __half2float(__ushort_as_half((unsigned short)(A.y >> 16)));
                            } else {
                                int4 A = make_int4(0, 0, 0, 0);
                                if (ok) A = rq[vv];
                                j0c = A.x & 0xffff;
                                av[u][0] = __int_as_float(A.y);
                                av[u][1] = __int_as_float(A.z);
                                av[u][2] = __int_as_float(A.w);
                            }
                            const int off0 = max(j0c - rl[u], 0);
                            cx[u][0] = off0 * NpS + vv;
                            cx[u][1] = min(off0 + 1, W - 1) * NpS + vv;
                            cx[u][2] = min(off0 + 2, W - 1) * NpS + vv;
                        }
#pragma unroll
                        for (int u = 0; u < VR; u++)
#pragma unroll
                            for (int k = 0; k < 3; k++) {
                                const float2 es = bz[cx[u][k]];
                                ev[u][k] = es.x;
                                const float pe = es.x * es.y;
                                const float q = av[u][k] * es.y;
                                pmax = fmaxf(pmax, fabsf(pe));
                                if (u & 1) {
                                    th2b = fmaf(q, q, th2b);
                                    th1b = fmaf(-q, pe, th1b);
                                } else {
                                    th2 = fmaf(q, q, th2);
                                    th1 = fmaf(-q, pe, th1);
                                }
                            }
                        if (__any_sync(0xffffffffu, !(pmax < hT))) {
                            // exact sums: w where |e sqrt(w)| < T, else T delta sqrt(w) / |e|
                            th1 = th2 = th1b = th2b = 0.0f;
#pragma unroll
                            for (int u = 0; u < VR; u++)
#pragma unroll
                                for (int k = 0; k < 3; k++)
                                    theta_acc(make_float2(ev[u][k], bz[cx[u][k]].y), av[u][k], hT, hTd,
                                              (u & 1) ? th1b : th1, (u & 1) ? th2b : th2);
                        }
                    } else {
                        const int *rw = reinterpret_cast<const int *>(rq);
                        for (int v = vh * 32 + lane; v < Np; v += 32 * vsplit) {
                            const int h = rw[(size_t)v * nwd];
                            const int n = h >> 16;
                            const float2 *pp = bz + ((h & 0xffff) - rlo[v]) * NpS + v;
                            for (int k = 0; k < n; k++) {
                                const float a = __int_as_float(rw[(size_t)v * nwd + 1 + k]);
                                for (int rr = 0; rr < mz; rr++)
                                    theta_acc(pp[rr * rowstride + k * NpS], a, hT, hTd, th1, th2);
                            }
                        }
                    }
                    th1 += th1b;
                    th2 += th2b;
                    // prior (first warp of the slice): f rho'(D)/D for q = 2, p = 1.2
                    // is (2 - 0.8 t1/t3) / (t3 s^q)
                    float p1 = 0.0f, p2 = 0.0f;
                    if (vh == 0 && valid) {
                        const float ad = fabsf(V - nbv);
                        const float t1 = (ad > 0.0f ? ex2_approx(0.8f * __log2f(ad)) : 0.0f) * qpinv;
                        const float rt3 = rcp_approx(cc + t1);
                        const float b = bw * (2.0f - 0.8f * t1 * rt3) * rt3 * qinv;
                        p1 = b * nbv;
                        p2 = b;
                    }
                    const float red = warp_reduce_scatter4(th1, th2, p1, p2, lane);
                    if (vsplit > 1) {
                        float *pp = part + 4 * vsplit * zl;
                        if ((lane & 7) == 0) pp[vh * 4 + (lane >> 3)] = red;
                        named_barrier(1 + zl, 32 * vsplit);
                        th1 = th2 = 0.0f;
                        for (int h = 0; h < vsplit; h++) {
                            th1 += pp[h * 4 + 0];
                            th2 += pp[h * 4 + 1];
                        }
                        p1 = pp[2];
                        p2 = pp[3];
                    } else {
                        th1 = __shfl_sync(0xffffffffu, red, 0);
                        th2 = __shfl_sync(0xffffffffu, red, 8);
                        p1 = __shfl_sync(0xffffffffu, red, 16);
                        p2 = __shfl_sync(0xffffffffu, red, 24);
                    }
                    const float u = (p1 + th2 * V - th1) * rcp_approx(p2 + th2);
                    const float xn = V + alpha * (u - V);
                    const float dx = xn - V;
                    if (vh == 0) {
                        __syncwarp();
                        if (lane == 0) {
                            *xc = xn;
                            magl[(zl * S + ly) * S + lx] = fabsf(dx);
                            sum_abs_dx += fabsf(dx);
                            sum_abs_x += fabsf(xn);
                            n_upd++;
                        }
                    }
                    // ---- error sinogram: e -= a dx over this slice's rows ----
                    float *bzf = reinterpret_cast<float *>(band + (size_t)zl * mz * rowstride);
                    if constexpr (AMAXC == 3 && MZC == 1) {
                        // absent columns (a = 0) rewrite their own value; a
                        // clamped one can share the slot of a real column of
                        // the same view at a lower k, so the writes go from
                        // k = 2 down to k = 0 and the real column's is last
#pragma unroll
                        for (int u = 0; u < VR; u++)
                            if (okm & (1u << u)) {
#pragma unroll
                                for (int k = 2; k >= 0; k--) bzf[2 * cx[u][k]] = fmaf(-av[u][k], dx, ev[u][k]);
                            }
                    } else {
                        const int *rw = reinterpret_cast<const int *>(rq);
                        for (int v = vh * 32 + lane; v < Np; v += 32 * vsplit) {
                            const int h = rw[(size_t)v * nwd];
                            const int n = h >> 16;
                            float *pe = bzf + 2 * (((h & 0xffff) - rlo[v]) * NpS + v);
                            for (int k = 0; k < n; k++) {
                                const float a = __int_as_float(rw[(size_t)v * nwd + 1 + k]);
                                for (int rr = 0; rr < mz; rr++) {
                                    float *q = pe + 2 * (rr * rowstride + k * NpS);
                                    *q = fmaf(-a, dx, *q);
                                }
                            }
                        }
                    }
                }
            }
            if (AC) {
                fetch(step + D, sl + D >= R ? sl + D - R : sl + D);
                cp_async_wait_upto<D - 1>();
            } else if (step + 1 < nl) {
                const int sn1 = sl + 1 == R ? 0 : sl + 1;
                if (nprod > 0) {
                    if (!consumer) acol(step + 1, sn1, ncons, av_prod);
                } else {
                    acol(step + 1, sn1, 0, av_all);
                }
            }
            __syncthreads();
        }
        if (AC) cp_async_wait0();

        // ---- write back voxels, magnitude map, band change ----
        float *xo = dv.x + (size_t)i * g.N_z * plane;
        for (int lz = warp; lz < nz; lz += nwarps)
            for (int q = lane; q < S * S; q += 32) {
                const int lx = q % S, ly = q / S;
                if (lx < kx && ly < ky)
                    xo[(size_t)(z0 + lz) * plane + (size_t)(j0 + ly) * g.N_x + k0 + lx] =
                        xb[((lz + 1) * S2 + ly + 1) * S2 + lx + 1];
            }
        for (int q = tid; q < nl; q += nthr) {
            const int o = order[q];
            if (o < 0) continue;
            const int lx = o & 0xff, ly = o >> 8;
            float m = 0.0f;
            for (int z = 0; z < nz; z++) m += magl[(z * S + ly) * S + lx];
            task.mag[(size_t)(j0 + ly) * g.N_x + k0 + lx] = m;
        }
        // band change back to e: vector atomics over the same 16-byte words
        // as the staging (zeros outside the band), four lanes per (row, view)
        if (vec) {
            // word c of pair pq: its change (zeros outside the band) and its
            // global address (-1: past the band or the row); the reads of a
            // thread's U words are issued before any of their atomics
            auto commit_word = [&](int pq, int c, float *d) -> long long {
                const int row = div_np(pq), v = pq - row * Np;
                const int lo = rlo[v], a0 = lo & ~3, sh = lo - a0;
                if (4 * c >= sh + W || a0 + 4 * c >= g.N_r) return -1;
                const float2 *bd = band + (size_t)row * rowstride + v;
                const float4 eo = __ldcg(reinterpret_cast<const float4 *>(scr) + (size_t)pq * nw + c);
                const float e0[4] = {eo.x, eo.y, eo.z, eo.w};
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int off = 4 * c + j - sh;
                    d[j] = 0.0f;
                    if (off >= 0 && off < W) d[j] = bd[(size_t)off * NpS].x - e0[j];
                }
                return (long long)((size_t)(z0 * mz + row) * g.N_p + vidx[v]) * g.N_r + a0 + 4 * c;
            };
            constexpr int U = 2;
            const int total = 4 * npairs;
            for (int b = tid; b < total; b += U * nthr) {
                float d[U][4];
                long long at[U];
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const int pqc = b + u * nthr;
                    at[u] = pqc < total ? commit_word(pqc >> 2, pqc & 3, d[u]) : -1;
                }
#pragma unroll
                for (int u = 0; u < U; u++)
                    if (at[u] >= 0 && (d[u][0] != 0.0f || d[u][1] != 0.0f || d[u][2] != 0.0f || d[u][3] != 0.0f))
                        red_add_v4(dv.e + at[u], d[u][0], d[u][1], d[u][2], d[u][3]);
            }
            if (W + 3 > 16)
                for (int pqc = tid; pqc < total; pqc += nthr)
                    for (int c = (pqc & 3) + 4; 4 * c < W + 3; c += 4) {
                        float d[4];
                        const long long a = commit_word(pqc >> 2, c, d);
                        if (a >= 0 && (d[0] != 0.0f || d[1] != 0.0f || d[2] != 0.0f || d[3] != 0.0f))
                            red_add_v4(dv.e + a, d[0], d[1], d[2], d[3]);
                    }
        } else {
            for (int pq = tid; pq < npairs; pq += nthr) {
                const int row = div_np(pq), v = pq - row * Np;
                const int lo = rlo[v];
                const float2 *bd = band + (size_t)row * rowstride + v;
                const float *sc = scr + (size_t)row * rowstride + v;
                float *erow = dv.e + ((size_t)(z0 * mz + row) * g.N_p + vidx[v]) * g.N_r;
                for (int off = 0; off < W; off++) {
                    const int r = lo + off;
                    if (r >= g.N_r) break;
                    const float dnew = bd[(size_t)off * NpS].x - sc[(size_t)off * NpS];
                    if (dnew != 0.0f) atomicAdd(erow + r, dnew);
                }
            }
        }
        // publish: every thread's writes of this super-voxel, then its flag
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            st_release(L.done + id, epoch);
            if constexpr (BATCH) atomicAdd(&L.state[cur].fin, 1);
        }
        if constexpr (BATCH) flush_stats(&L.state[cur].out);
    }
    if constexpr (!BATCH) flush_stats(out);
}

// End of a batched iteration (one CTA).
__global__ void __launch_bounds__(256) k_sv_batch_end(SvProblem *__restrict__ probs, SvBatchState *__restrict__ st,
                                                      int n, int *ctl, int *queue)
{
    __shared__ int s_active;
    if (threadIdx.x == 0) s_active = 0;
    __syncthreads();
    int act = 0;
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
        SvBatchState &b = st[q];
        if (b.active) {
            b.iters++;
            b.updates += b.out.updates;
            b.zero_skips += b.out.zero_skips;
            // the reference's convergence ratio (XT_ICD_update.c:1066-1103)
            const double ax = b.out.sum_abs_x;
            const double pct = ax > 0 ? 100.0 * probs[q].K * b.out.sum_abs_dx / ax : 0.0;
            // (the stability guard is the host's: mbir_batch_iterate
            // compares each problem's MAP cost over a window of iterations)
            b.prev_ax = ax;
            b.pct = pct;
            if (b.pct < probs[q].stop) {
                b.active = 0;
                b.converged = 1;
            }
        }
        act += b.active;
        b.out = SvTaskOut{};
        b.fin = 0;
    }
    if (act) atomicAdd(&s_active, act);
    __syncthreads();
    if (threadIdx.x == 0) {
        ctl[0]++;
        ctl[1] = s_active;
        *queue = 0;
    }
}

template <int AMAXC, int MZC, int AC, int MAXT, int VU, bool BATCH = false>
int occupancy_sv(int threads, size_t sm)
{
    if (cudaFuncSetAttribute(k_icd_sv<AMAXC, MZC, AC, MAXT, VU, BATCH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sm) != cudaSuccess)
        return 1;
    int n = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_icd_sv<AMAXC, MZC, AC, MAXT, VU, BATCH>, threads, sm) !=
        cudaSuccess)
        return 1;
    return n > 0 ? n : 1;
}

template <int AMAXC, int MZC, int AC, int MAXT, int VU, bool BATCH = false>
cudaError_t launch_sv(const SvProblem &P, const SvLaunch &L, int ctas, int threads, size_t sm, int *queue,
                      float *scratch, size_t scratch_floats, SvTaskOut *out, int iter, uint32_t seed, int *err,
                      cudaStream_t s)
{
    cudaError_t e = cudaFuncSetAttribute(k_icd_sv<AMAXC, MZC, AC, MAXT, VU, BATCH>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    k_icd_sv<AMAXC, MZC, AC, MAXT, VU, BATCH>
        <<<ctas, threads, sm, s>>>(P, L, queue, scratch, scratch_floats, out, iter, seed, err);
    return cudaGetLastError();
}

}  // namespace

SvPlan mbir_sv_plan(const SvParams &sp, bool cached)
{
    const int NpS = sp.max_views, S = sp.S, S2 = sp.S + 2;
    SvPlan pl{};
    pl.ring_bytes = (cached && sp.ahalf ? 8 : 16 * sp.eq) * sp.ring * NpS;
    pl.band_pairs = sp.max_rows * sp.W * NpS;
    pl.trig_views = cached ? 0 : NpS;
    pl.xb = (sp.max_nz + 2) * S2 * S2;
    pl.tb = 2 * sp.max_nz * S * S;
    pl.magl = sp.max_nz * S * S;
    pl.part = 4 * 4 * sp.max_nz;
    pl.views = NpS;
    pl.order = S * S + 4;
    return pl;
}

size_t mbir_sv_plan_bytes(const SvPlan &pl)
{
    size_t b = (size_t)pl.ring_bytes + 8 * (size_t)pl.band_pairs + 16 * (size_t)pl.trig_views;
    b += sizeof(float) * ((size_t)pl.xb + pl.tb + pl.magl + pl.part);
    b += sizeof(int) * (2 * (size_t)pl.views + pl.order);
    return (b + 15) & ~(size_t)15;
}

size_t mbir_sv_smem_bytes(const SvParams &sp, bool cached) { return mbir_sv_plan_bytes(mbir_sv_plan(sp, cached)); }

cudaError_t mbir_forward_rows(const MbirGeom &g, const int *frame_of_view, const float *x, const float *y,
                              const float *d, float *out, int mode, int amax, cudaStream_t s)
{
    const bool full = amax == 3;
    if (g.N_z <= 8)
        return full ? launch_forward_rows<3, 2, 8>(g, frame_of_view, x, y, d, out, mode, amax, s)
                    : launch_forward_rows<0, 2, 8>(g, frame_of_view, x, y, d, out, mode, amax, s);
    return full ? launch_forward_rows<3, 2, 16>(g, frame_of_view, x, y, d, out, mode, amax, s)
                : launch_forward_rows<0, 2, 16>(g, frame_of_view, x, y, d, out, mode, amax, s);
}

size_t mbir_acache_bytes(const MbirGeom &g, int eq, bool half)
{
    return (size_t)g.N_y * g.N_x * g.N_p * (half ? 8 : eq * 16);
}

cudaError_t mbir_build_acache(const MbirGeom &g, const MbirDev &dv, int amax, int eq, bool half, int4 *cache,
                              int *err, cudaStream_t s)
{
    const long long lines = (long long)g.N_y * g.N_x;
    const int blocks = (int)((lines + 7) / 8);
    if (half)
        k_acache<3, true><<<blocks, 256, 0, s>>>(g, dv.mask, amax, eq, cache, err);
    else if (amax == 3)
        k_acache<3, false><<<blocks, 256, 0, s>>>(g, dv.mask, amax, eq, cache, err);
    else
        k_acache<0, false><<<blocks, 256, 0, s>>>(g, dv.mask, amax, eq, cache, err);
    return cudaGetLastError();
}

// Instantiation of the super-voxel kernel for a configuration: F is called
// with a tag carrying its template arguments.
template <int A_, int M_, int C_, int T_, int V_>
struct SvInst {
    static constexpr int AMAXC = A_, MZC = M_, AC = C_, MAXT = T_, VU = V_;
};
template <class F>
auto sv_dispatch(const MbirGeom &g, const SvParams &sp, bool cached, int threads, F &&f)
{
    // full resolution (3 columns per entry, one detector row per slice) with
    // at most 4 views per lane and slice has its own instantiations with
    // fixed trip counts; one warp per slice with up to 8 views per lane in
    // registers (the cached path; 256 threads leave 255 registers per thread)
    const int vpl = (sp.max_views + 32 * sp.vsplit - 1) / (32 * sp.vsplit);
    const bool full = sp.amax == 3 && g.m_z == 1 && vpl <= 4;
    // FP16 cache: full resolution with at most 4 views per lane, 512 threads
    // (the host asks for it only then)
    if (cached && sp.ahalf && full && threads <= 512) {
        if (vpl <= 2) return f(SvInst<3, 1, 2, 512, 2>{});
        return f(SvInst<3, 1, 2, 512, 4>{});
    }
    if (cached && threads <= 256 && sp.amax == 3 && g.m_z == 1 && vpl > 4 && vpl <= 8)
        return sp.ahalf ? f(SvInst<3, 1, 2, 256, 8>{}) : f(SvInst<3, 1, 1, 256, 8>{});
#define MBIR_SV_PICK(T)                                                                              \
    if (full && vpl <= 2) return cached ? f(SvInst<3, 1, 1, T, 2>{}) : f(SvInst<3, 1, 0, T, 2>{}); \
    if (full) return cached ? f(SvInst<3, 1, 1, T, 4>{}) : f(SvInst<3, 1, 0, T, 4>{});             \
    return cached ? f(SvInst<0, 0, 1, T, 0>{}) : f(SvInst<0, 0, 0, T, 0>{});
    if (threads <= 512) {
        MBIR_SV_PICK(512)
    }
    MBIR_SV_PICK(1024)
#undef MBIR_SV_PICK
}

int mbir_sv_ctas_per_sm(const MbirGeom &g, const SvParams &sp, bool cached)
{
    const size_t sm = mbir_sv_smem_bytes(sp, cached);
    const int threads = 32 * (sp.max_nz * sp.vsplit + (cached ? 0 : sp.prod_warps));
    return sv_dispatch(g, sp, cached, threads, [&](auto I) {
        using In = decltype(I);
        return occupancy_sv<In::AMAXC, In::MZC, In::AC, In::MAXT, In::VU>(threads, sm);
    });
}

cudaError_t mbir_launch_icd_sv(const MbirGeom &g, const MbirPrior &pr, const MbirDev &dv, const SvParams &sp,
                               SvACache ac, const SvLaunch &L, int ctas, int *queue, float *scratch, SvTaskOut *out,
                               int iter, uint32_t seed, int *err, cudaStream_t s)
{
    if (L.ntasks <= 0) return cudaSuccess;
    const bool cached = ac.a != nullptr;
    SvProblem P{};
    P.g = g;
    P.pr = pr;
    P.dv = dv;
    P.sp = sp;
    P.ac = ac;
    P.plan = mbir_sv_plan(sp, cached);
    const size_t sm = mbir_sv_plan_bytes(P.plan);
    const int threads = 32 * (sp.max_nz * sp.vsplit + (cached ? 0 : sp.prod_warps));
    return sv_dispatch(g, sp, cached, threads, [&](auto I) {
        using In = decltype(I);
        return launch_sv<In::AMAXC, In::MZC, In::AC, In::MAXT, In::VU>(P, L, ctas, threads, sm, queue, scratch,
                                                                       sp.band_floats, out, iter, seed, err, s);
    });
}

int mbir_sv_batch_ctas_per_sm(size_t smem_bytes, bool half)
{
    return half ? occupancy_sv<3, 1, 2, kSvBatchThreads, kSvBatchViewsPerLane, true>(kSvBatchThreads, smem_bytes)
                : occupancy_sv<3, 1, 1, kSvBatchThreads, kSvBatchViewsPerLane, true>(kSvBatchThreads, smem_bytes);
}

cudaError_t mbir_sv_batch_prepare(size_t smem_bytes, bool half)
{
    const int sm = (int)smem_bytes;
    return half ? cudaFuncSetAttribute(k_icd_sv<3, 1, 2, kSvBatchThreads, kSvBatchViewsPerLane, true>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, sm)
                : cudaFuncSetAttribute(k_icd_sv<3, 1, 1, kSvBatchThreads, kSvBatchViewsPerLane, true>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
}

cudaError_t mbir_launch_icd_sv_batch(size_t smem_bytes, bool half, const SvLaunch &L, int ctas, int *queue,
                                     float *scratch, size_t scratch_floats, uint32_t seed, int *err, cudaStream_t s)
{
    // the problems come from L.problems; the parameter copy is unused
    const SvProblem none{};
    if (half)
        k_icd_sv<3, 1, 2, kSvBatchThreads, kSvBatchViewsPerLane, true><<<ctas, kSvBatchThreads, smem_bytes, s>>>(
            none, L, queue, scratch, scratch_floats, nullptr, 0, seed, err);
    else
        k_icd_sv<3, 1, 1, kSvBatchThreads, kSvBatchViewsPerLane, true><<<ctas, kSvBatchThreads, smem_bytes, s>>>(
            none, L, queue, scratch, scratch_floats, nullptr, 0, seed, err);
    return cudaGetLastError();
}

cudaError_t mbir_launch_sv_batch_end(SvProblem *probs, SvBatchState *state, int n, int *ctl, int *queue,
                                     cudaStream_t s)
{
    k_sv_batch_end<<<1, 256, 0, s>>>(probs, state, n, ctl, queue);
    return cudaGetLastError();
}
