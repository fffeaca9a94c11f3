// Super-voxel-parallel ICD kernel (sm_100a).
//
// One CTA owns a super-voxel (SV): an S x S block of voxel lines of one
// frame and a group of nz consecutive slices.  It stages into shared memory
//   * the error-sinogram and weight band the SV touches: for each view of the
//     frame, the W consecutive detector columns [rlo_p, rlo_p + W) that cover
//     every voxel of the block, for each detector row of the slices;
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
// neighbours.  Only slice z's warps touch slice z's band rows, and each view
// is always handled by the same lane, so error-sinogram updates need no
// synchronisation; the warps of one slice combine theta through shared
// memory and a named barrier; one CTA barrier per line step hands the next
// line's A-matrix column (computed cooperatively into a three-slot ring) and
// the updated voxels to all warps.
//
// CTAs are persistent: each takes SVs from a device work queue (host-sorted
// by decreasing work) until the queue of the launch is empty.
//
// Concurrent SVs are chosen by the host so that no two share a prior
// neighbourhood (2x2 SV checkerboard, z-group and frame parity); they may
// share error-sinogram entries, whose concurrent changes they see at their
// next visit (the super-voxel ICD scheme of Wang et al., "High performance
// model based image reconstruction", PPoPP 2016).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

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

// Four independent butterfly all-reductions, interleaved so their shuffle
// latencies overlap.
__device__ __forceinline__ void warp_allsum4(float &a, float &b, float &c, float &d)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float ta = __shfl_xor_sync(0xffffffffu, a, o);
        const float tb = __shfl_xor_sync(0xffffffffu, b, o);
        const float tc = __shfl_xor_sync(0xffffffffu, c, o);
        const float td = __shfl_xor_sync(0xffffffffu, d, o);
        a += ta;
        b += tb;
        c += tc;
        d += td;
    }
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

struct AEnt {
    float a;  // A-matrix value
    int so;   // shared-memory offset of the entry in a band row: off * NpS + v
};

// AMAXC: entries per (line, view) known at compile time (3 at full
// resolution), 0 = runtime sp.amax.  MZC: detector rows per slice known at
// compile time (1 at full resolution), 0 = runtime m_z.
template <int AMAXC, int MZC>
__global__ void __launch_bounds__(1024) k_icd_sv(MbirGeom g, MbirPrior pr, MbirDev dv, SvParams sp,
                                                  const SvTask *__restrict__ tasks, int ntasks,
                                                  int *queue, float *__restrict__ scratch,
                                                  SvTaskOut *__restrict__ out, int iter, uint32_t seed, int *err)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    const int S = sp.S, W = sp.W, vsplit = sp.vsplit;
    const int amax = AMAXC > 0 ? AMAXC : sp.amax;
    const int mz = MZC > 0 ? MZC : g.m_z;
    const int NpS = sp.max_views;  // smem stride (views)
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nwarps = nthr >> 5;
    const int S2 = S + 2;
    const int rowstride = W * NpS;

    // ---- carve shared memory (sizes fixed by the host in sp) ----
    unsigned char *p = smraw;
    double *cs = reinterpret_cast<double *>(p); p += sizeof(double) * NpS;
    double *sn = reinterpret_cast<double *>(p); p += sizeof(double) * NpS;
    AEnt *aring = reinterpret_cast<AEnt *>(p); p += sizeof(AEnt) * 3 * amax * NpS;
    float *eb = reinterpret_cast<float *>(p); p += sizeof(float) * (size_t)sp.max_rows * rowstride;
    float *sb = reinterpret_cast<float *>(p); p += sizeof(float) * (size_t)sp.max_rows * rowstride;
    float *xb = reinterpret_cast<float *>(p); p += sizeof(float) * (sp.max_nz + 2) * S2 * S2;
    float *tb = reinterpret_cast<float *>(p); p += sizeof(float) * 2 * sp.max_nz * S * S;
    float *magl = reinterpret_cast<float *>(p); p += sizeof(float) * S * S;
    float *part = reinterpret_cast<float *>(p); p += sizeof(float) * 4 * 4 * sp.max_nz;
    int *vidx = reinterpret_cast<int *>(p); p += sizeof(int) * NpS;
    int *rlo = reinterpret_cast<int *>(p); p += sizeof(int) * NpS;
    int *order = reinterpret_cast<int *>(p); p += sizeof(int) * S * S;
    __shared__ int s_nlines, s_task;
    __shared__ float s_red[32][4];

    const double inv_dr = 1.0 / g.delta_r, inv_off = 1.0 / g.OffsetR;
    const float inv_off_f = (float)inv_off;
    const float alpha = (float)pr.alpha, hT = (float)pr.hT, hTd = (float)(pr.hT * pr.hdelta);
    const float sSQ_inv = (float)(1.0 / pr.sSQ), sSQP_inv = (float)(1.0 / pr.sSQP), cS = (float)pr.c_s;
    const float sTQ_inv = (float)(1.0 / pr.sTQ), sTQP_inv = (float)(1.0 / pr.sTQP), cT = (float)pr.c_t;
    // warps [0, ncons) update voxels (vsplit per slice); warps [ncons, nwarps)
    // produce the next line's A-matrix column while they do
    const int ncons = sp.max_nz * vsplit, nprod = nwarps - ncons;
    const bool consumer = warp < ncons;
    const int zl = consumer ? warp / vsplit : 0, vh = consumer ? warp - zl * vsplit : 0;
    // neighbour of lane: spatial (dz, dy, dx) for lanes 0..25, temporal 26, 27
    int ndz = 0, ndy = 0, ndx = 0;
    float bw = 0.0f, qinv = 0.0f, qpinv = 0.0f, cc = 1.0f;
    bool spatial = false, temporal = false;
    if (lane < 26) {
        const int n = lane < 13 ? lane : lane + 1;  // skip the centre (13)
        ndz = n / 9 - 1;
        ndy = (n / 3) % 3 - 1;
        ndx = n % 3 - 1;
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
    float sum_abs_dx = 0.0f, sum_abs_x = 0.0f;
    int n_upd = 0, n_skip = 0;

    for (;;) {
        __syncthreads();
        if (tid == 0) s_task = atomicAdd(queue, 1);
        __syncthreads();
        const int tix = s_task;
        if (tix >= ntasks) break;
        const SvTask task = tasks[tix];
        const int nz = task.nz, rows = nz * mz;
        const int i = task.frame;
        const int Np = g.view_num[i];
        const int k0 = task.k0, j0 = task.j0, z0 = task.z0;
        const int kx = min(S, g.N_x - k0), ky = min(S, g.N_y - j0);
        const int *vl = g.view_idx + (size_t)i * g.max_views;
        const bool active = consumer && zl < nz;
        const int zg = z0 + zl;

        // ---- views, trig, band origin per view ----
        for (int v = tid; v < Np; v += nthr) {
            const int view = vl[v];
            vidx[v] = view;
            const double c = g.cosv[view], s = g.sinv[view];
            cs[v] = c;
            sn[v] = s;
            int lo = 1 << 30;
            const double xs[2] = {vx(g, k0), vx(g, k0 + kx - 1)};
            const double ys[2] = {vy(g, j0), vy(g, j0 + ky - 1)};
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const double r = __dsub_rn(__dmul_rn(xs[u & 1], c), __dmul_rn(ys[u >> 1], s));
                lo = min(lo, floor_div(__dsub_rn(__dsub_rn(r, g.delta_xy), g.R0), g.delta_r, inv_dr));
            }
            rlo[v] = max(lo, 0);
        }
        // ---- in-mask lines, ordered by 2x2 parity class then a per-visit hash ----
        if (warp == 0) {
            int n = 0;
            for (int cls = 0; cls < 4; cls++) {
                const int base = n;
                for (int q0 = 0; q0 < S * S; q0 += 32) {
                    const int q = q0 + lane;
                    const int lx = q % S, ly = q / S;
                    bool take = false;
                    if (q < S * S && lx < kx && ly < ky)
                        take = ((((k0 + lx) & 1) | (((j0 + ly) & 1) << 1)) == cls) &&
                               dv.mask[(size_t)(j0 + ly) * g.N_x + k0 + lx] == 1;
                    const unsigned bal = __ballot_sync(0xffffffffu, take);
                    if (take) order[n + __popc(bal & ((1u << lane) - 1))] = q;
                    n += __popc(bal);
                }
                __syncwarp();
                if (lane == 0)
                    for (int q = n - 1; q > base; q--) {
                        const uint32_t h = hash32(seed ^ hash32((uint32_t)tix * 1315423911u + (uint32_t)q));
                        const int r = base + (int)(h % (uint32_t)(q - base + 1));
                        const int t = order[q];
                        order[q] = order[r];
                        order[r] = t;
                    }
                __syncwarp();
            }
            if (lane == 0) s_nlines = n;
        }
        for (int q = tid; q < S * S; q += nthr) magl[q] = 0.0f;
        __syncthreads();
        const int nl = s_nlines;

        // ---- stage bands: e (also to this CTA's scratch slot) and sqrt(w);
        //      four loads in flight per thread before the stores ----
        float *__restrict__ scr = scratch + (size_t)blockIdx.x * sp.band_floats;
        for (int ro = warp; ro < rows * W; ro += nwarps) {
            const int row = ro / W, off = ro - row * W;
            const int t = z0 * mz + row;
            const float *__restrict__ erow = dv.e + (size_t)t * g.N_p * g.N_r;
            const float *__restrict__ wrow = dv.w + (size_t)t * g.N_p * g.N_r;
            for (int v0 = lane; v0 < Np; v0 += 128) {
                float ev[4], wv[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int v = v0 + 32 * u;
                    ev[u] = 0.0f;
                    wv[u] = 0.0f;
                    if (v < Np) {
                        const int r = rlo[v] + off;
                        if (r < g.N_r) {
                            const size_t o = (size_t)vidx[v] * g.N_r + r;
                            ev[u] = __ldcg(erow + o);
                            wv[u] = __ldg(wrow + o);
                        }
                    }
                }
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int v = v0 + 32 * u;
                    if (v < Np) {
                        eb[ro * NpS + v] = ev[u];
                        sb[ro * NpS + v] = sqrtf(wv[u]);
                        scr[ro * NpS + v] = ev[u];
                    }
                }
            }
        }
        // ---- voxel block with halo, temporal neighbours ----
        const size_t plane = (size_t)g.N_y * g.N_x;
        const float *xf = dv.x + (size_t)i * g.N_z * plane;
        for (int lz = warp; lz < nz + 2; lz += nwarps)
            for (int q = lane; q < S2 * S2; q += 32) {
                const int lx = q % S2, ly = q / S2;
                const int xx = k0 + lx - 1, yy = j0 + ly - 1, zz = z0 + lz - 1;
                float v = 0.0f;
                if (xx >= 0 && xx < g.N_x && yy >= 0 && yy < g.N_y && zz >= 0 && zz < g.N_z)
                    v = xf[(size_t)zz * plane + (size_t)yy * g.N_x + xx];
                xb[lz * S2 * S2 + q] = v;
            }
        for (int sz = warp; sz < 2 * nz; sz += nwarps) {
            const int side = sz / nz, lz = sz - side * nz;
            const int ti = i + (side == 0 ? -1 : 1);
            for (int q = lane; q < S * S; q += 32) {
                const int lx = q % S, ly = q / S;
                float v = 0.0f;
                if (ti >= 0 && ti < g.N_time && lx < kx && ly < ky)
                    v = dv.x[((size_t)ti * g.N_z + z0 + lz) * plane + (size_t)(j0 + ly) * g.N_x + k0 + lx];
                tb[sz * S * S + q] = v;
            }
        }

        // ---- A-matrix column of line `li` into ring slot `slot` (exact bins);
        //      unused entries carry a = 0 ----
        auto acol = [&](int li, int slot, int w0, int av_lanes) {
            const int wr = warp - w0;
            if (wr < 0) return;
            const int loc = order[li];
            const int col = k0 + loc % S, row = j0 + loc / S;
            const double x = vx(g, col), y = vy(g, row);
            AEnt *ar = aring + slot * amax * NpS;
            for (int l = lane; l < av_lanes; l += 32) {
                const int v = wr * av_lanes + l;
                if (v >= Np) break;
                const double r = __dsub_rn(__dmul_rn(x, cs[v]), __dmul_rn(y, sn[v]));
                const double rmin = __dsub_rn(r, g.delta_xy), rmax = __dadd_rn(r, g.delta_xy);
                int n = 0;
                if (!(rmax < g.R0 || rmin > g.RMax)) {
                    int imin = floor_div(__dsub_rn(rmin, g.R0), g.delta_r, inv_dr);
                    int imax = floor_div(__dsub_rn(rmax, g.R0), g.delta_r, inv_dr);
                    if (imax >= g.N_r) imax = g.N_r - 1;
                    if (imin < 0) imin = 0;
                    const float *H = g.H_r + (size_t)vidx[v] * (MBIR_RESP_BINS + 1);
                    const int base = rlo[v];
                    for (int j = imin; j <= imax; j++) {
                        const double rc = __dadd_rn(g.R0, __dmul_rn((double)j + 0.5, g.delta_r));
                        const double dr = fabs(__dsub_rn(r, rc));
                        const int id = floor_div(dr, g.OffsetR, inv_off);
                        if (id >= 0 && id < MBIR_RESP_BINS) {
                            const double w1 = __dsub_rn(dr, __dmul_rn((double)id, g.OffsetR));
                            const double w2 = __dsub_rn(g.OffsetR, w1);
                            const double num = __dadd_rn(__dmul_rn(w2, (double)__ldg(H + id)),
                                                         __dmul_rn(w1, (double)__ldg(H + id + 1)));
                            const int off = j - base;
                            if (num > 0) {
                                if (off < 0 || off >= W || n >= amax) {
                                    atomicOr(err, 1);
                                } else {
                                    AEnt en;
                                    en.a = (float)num * inv_off_f;
                                    en.so = off * NpS + v;
                                    ar[n * NpS + v] = en;
                                    n++;
                                }
                            }
                        }
                    }
                }
                for (; n < amax; n++) {
                    AEnt en;
                    en.a = 0.0f;
                    en.so = v;
                    ar[n * NpS + v] = en;
                }
            }
        };

        __syncthreads();
        if (nl > 0) acol(0, 0, 0, av_all);
        __syncthreads();

        for (int step = 0; step <= nl; step++) {
            const int li = (zl & 1) ? step - 1 : step;
            if (active && li >= 0 && li < nl) {
                const int slot = li % 3;
                const int loc = order[li];
                const int lx = loc % S, ly = loc / S;
                const int col = k0 + lx, row = j0 + ly;
                float *xc = xb + ((zl + 1) * S2 + ly + 1) * S2 + lx + 1;
                const float V = *xc;
                // ---- prior neighbourhood ----
                float nbv = 0.0f;
                bool valid = false;
                if (spatial) {
                    const int zz = zg + ndz, yy = row + ndy, xx = col + ndx;
                    valid = zz >= 0 && zz < g.N_z && yy >= 0 && yy < g.N_y && xx >= 0 && xx < g.N_x;
                    if (valid) nbv = xc[(ndz * S2 + ndy) * S2 + ndx];
                } else if (temporal) {
                    const int ti = i + (lane == 26 ? -1 : 1);
                    valid = ti >= 0 && ti < g.N_time;
                    if (valid) nbv = tb[((lane - 26) * nz + zl) * S * S + ly * S + lx];
                }
                const unsigned pos = __ballot_sync(0xffffffffu, valid && nbv > 0.0f);
                if (V == 0.0f && iter > 1 && pos == 0u) {
                    if (vh == 0 && lane == 0) n_skip++;
                } else {
                    // ---- data term over this slice's band rows, this warp's views ----
                    float th1 = 0.0f, th2 = 0.0f, th1b = 0.0f, th2b = 0.0f;
                    const AEnt *ar = aring + slot * amax * NpS;
                    const float *erow = eb + zl * mz * rowstride;
                    const float *srow = sb + zl * mz * rowstride;
                    auto theta_entry = [&](const AEnt &en, int rr, float &t1, float &t2) {
                        const float e = erow[rr * rowstride + en.so];
                        const float sw = srow[rr * rowstride + en.so];
                        float om = sw * sw;
                        if (!(fabsf(e * sw) < hT)) om = __fdividef(hTd * sw, fabsf(e));
                        if (en.a != 0.0f) {
                            t2 = fmaf(en.a * en.a, om, t2);
                            t1 = fmaf(-e * en.a, om, t1);
                        }
                    };
                    if constexpr (AMAXC > 0 && MZC > 0) {
                        int v = vh * 32 + lane;
                        const int vstep = 32 * vsplit;
                        for (; v + vstep < Np; v += 2 * vstep) {
                            AEnt ea[AMAXC], eb2[AMAXC];
#pragma unroll
                            for (int q = 0; q < AMAXC; q++) {
                                ea[q] = ar[q * NpS + v];
                                eb2[q] = ar[q * NpS + v + vstep];
                            }
#pragma unroll
                            for (int q = 0; q < AMAXC; q++)
#pragma unroll
                                for (int rr = 0; rr < MZC; rr++) {
                                    theta_entry(ea[q], rr, th1, th2);
                                    theta_entry(eb2[q], rr, th1b, th2b);
                                }
                        }
                        if (v < Np) {
#pragma unroll
                            for (int q = 0; q < AMAXC; q++) {
                                const AEnt en = ar[q * NpS + v];
#pragma unroll
                                for (int rr = 0; rr < MZC; rr++) theta_entry(en, rr, th1, th2);
                            }
                        }
                    } else {
                        for (int v = vh * 32 + lane; v < Np; v += 32 * vsplit)
                            for (int q = 0; q < amax; q++) {
                                const AEnt en = ar[q * NpS + v];
                                if (en.a == 0.0f) break;
                                for (int rr = 0; rr < mz; rr++) theta_entry(en, rr, th1, th2);
                            }
                    }
                    th1 += th1b;
                    th2 += th2b;
                    // prior (first warp of the slice): f rho'(D)/D for q = 2, p = 1.2
                    // is (2 - 0.8 t1/t3) / (t3 s^q)
                    float p1 = 0.0f, p2 = 0.0f;
                    if (vh == 0 && valid) {
                        const float ad = fabsf(V - nbv);
                        const float t1 = (ad > 0.0f ? exp2f(0.8f * __log2f(ad)) : 0.0f) * qpinv;
                        const float rt3 = __frcp_rn(cc + t1);
                        const float b = bw * (2.0f - 0.8f * t1 * rt3) * rt3 * qinv;
                        p1 = b * nbv;
                        p2 = b;
                    }
                    warp_allsum4(th1, th2, p1, p2);
                    if (vsplit > 1) {
                        float *pp = part + 4 * vsplit * zl;
                        if (lane == 0) {
                            pp[vh * 4 + 0] = th1;
                            pp[vh * 4 + 1] = th2;
                            pp[vh * 4 + 2] = p1;
                            pp[vh * 4 + 3] = p2;
                        }
                        named_barrier(1 + zl, 32 * vsplit);
                        th1 = th2 = 0.0f;
                        for (int h = 0; h < vsplit; h++) {
                            th1 += pp[h * 4 + 0];
                            th2 += pp[h * 4 + 1];
                        }
                        p1 = pp[2];
                        p2 = pp[3];
                    }
                    const float u = (p1 + th2 * V - th1) / (p2 + th2);
                    const float xn = V + alpha * (u - V);
                    const float dx = xn - V;
                    if (vh == 0) {
                        __syncwarp();
                        if (lane == 0) {
                            *xc = xn;
                            magl[loc] += fabsf(dx);
                            sum_abs_dx += fabsf(dx);
                            sum_abs_x += fabsf(xn);
                            n_upd++;
                        }
                    }
                    // ---- error sinogram: e -= a dx over this slice's rows ----
                    float *erw = eb + zl * mz * rowstride;
                    if constexpr (AMAXC > 0 && MZC > 0) {
#pragma unroll 2
                        for (int v = vh * 32 + lane; v < Np; v += 32 * vsplit) {
#pragma unroll
                            for (int q = 0; q < AMAXC; q++) {
                                const AEnt en = ar[q * NpS + v];
                                if (en.a != 0.0f) {
#pragma unroll
                                    for (int rr = 0; rr < MZC; rr++) {
                                        float *pe = erw + rr * rowstride + en.so;
                                        *pe = fmaf(-en.a, dx, *pe);
                                    }
                                }
                            }
                        }
                    } else {
                        for (int v = vh * 32 + lane; v < Np; v += 32 * vsplit)
                            for (int q = 0; q < amax; q++) {
                                const AEnt en = ar[q * NpS + v];
                                if (en.a == 0.0f) break;
                                for (int rr = 0; rr < mz; rr++) {
                                    float *pe = erw + rr * rowstride + en.so;
                                    *pe = fmaf(-en.a, dx, *pe);
                                }
                            }
                    }
                }
            }
            if (step + 1 < nl) {
                if (nprod > 0) {
                    if (!consumer) acol(step + 1, (step + 1) % 3, ncons, av_prod);
                } else {
                    acol(step + 1, (step + 1) % 3, 0, av_all);
                }
            }
            __syncthreads();
        }

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
            const int loc = order[q];
            task.mag[(size_t)(j0 + loc / S) * g.N_x + k0 + loc % S] = magl[loc];
        }
        for (int ro = warp; ro < rows * W; ro += nwarps) {
            const int row = ro / W, off = ro - row * W;
            float *erow = dv.e + (size_t)(z0 * mz + row) * g.N_p * g.N_r;
            for (int v0 = lane; v0 < Np; v0 += 128) {
                float old[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int v = v0 + 32 * u;
                    old[u] = v < Np ? scr[ro * NpS + v] : 0.0f;
                }
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int v = v0 + 32 * u;
                    if (v >= Np) continue;
                    const int r = rlo[v] + off;
                    if (r >= g.N_r) continue;
                    const float dnew = eb[ro * NpS + v] - old[u];
                    if (dnew != 0.0f) atomicAdd(erow + (size_t)vidx[v] * g.N_r + r, dnew);
                }
            }
        }
    }
    // ---- per-CTA statistics (lane 0 of each slice's first warp counts) ----
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
        atomicAdd(&out->sum_abs_dx, d0);
        atomicAdd(&out->sum_abs_x, d1);
        atomicAdd((unsigned long long *)&out->updates, (unsigned long long)d2);
        atomicAdd((unsigned long long *)&out->zero_skips, (unsigned long long)d3);
    }
}

}  // namespace

size_t mbir_sv_smem_bytes(const SvParams &sp)
{
    const size_t NpS = sp.max_views, S = sp.S, S2 = sp.S + 2;
    size_t b = 0;
    b += 2 * sizeof(double) * NpS;
    b += 8 * 3 * (size_t)sp.amax * NpS;  // A ring of (value, offset) pairs
    b += 2 * sizeof(float) * (size_t)sp.max_rows * sp.W * NpS;
    b += sizeof(float) * (sp.max_nz + 2) * S2 * S2;
    b += sizeof(float) * 2 * sp.max_nz * S * S;
    b += sizeof(float) * S * S;
    b += sizeof(float) * 4 * 4 * sp.max_nz;
    b += sizeof(int) * NpS * 2;
    b += sizeof(int) * S * S;
    return (b + 15) & ~(size_t)15;
}

cudaError_t mbir_launch_icd_sv(const MbirGeom &g, const MbirPrior &pr, const MbirDev &dv, const SvParams &sp,
                               const SvTask *tasks, int ntasks, int ctas, int *queue, float *scratch,
                               SvTaskOut *out, int iter, uint32_t seed, int *err, cudaStream_t s)
{
    if (ntasks <= 0) return cudaSuccess;
    const size_t sm = mbir_sv_smem_bytes(sp);
    cudaError_t e = cudaSuccess;
    const int threads = 32 * (sp.max_nz * sp.vsplit + sp.prod_warps);
    // full resolution (3 bins per column, one detector row per slice) has its
    // own instantiation with fixed trip counts
    if (sp.amax == 3 && g.m_z == 1) {
        e = cudaFuncSetAttribute(k_icd_sv<3, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        k_icd_sv<3, 1><<<ctas, threads, sm, s>>>(g, pr, dv, sp, tasks, ntasks, queue, scratch, out, iter, seed, err);
    } else {
        e = cudaFuncSetAttribute(k_icd_sv<0, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        k_icd_sv<0, 0><<<ctas, threads, sm, s>>>(g, pr, dv, sp, tasks, ntasks, queue, scratch, out, iter, seed, err);
    }
    return cudaGetLastError();
}
