// CUDA kernels for the MBIR ICD hot path (sm_100a).
//
// Reference algorithm: TIMBIR v0.0.2, src/MBIR_4D.  Every kernel cites the
// reference function whose arithmetic it reproduces.  Arithmetic that feeds
// an index decision (detector bin of the A-matrix column) or that the
// reference performs in float is written with explicit round-to-nearest
// intrinsics so that no fused multiply-add changes a rounding step.
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>
#include <stdint.h>

#include "mbir_internal.h"

namespace {

constexpr double kP = 1.2;  // qGGMRF p (XT_Constants.h:61)
constexpr double kQ = 2.0;  // qGGMRF q (XT_Constants.h:62)

// ----------------------------------------------------------------------------
// A-matrix column (XT_AMatrix.c:50-110): detector bins within delta_xy of the
// voxel's projected centre r = x cos - y sin, weight = linear interpolation of
// H_r[view] at |r - R_c| / OffsetR, kept if > 0.  Returns the count.
// ----------------------------------------------------------------------------
__device__ __forceinline__ double voxel_x(const MbirGeom &g, int col)
{
    return __dadd_rn(g.x0, __dmul_rn((double)col + 0.5, g.delta_xy));
}
__device__ __forceinline__ double voxel_y(const MbirGeom &g, int row)
{
    return __dadd_rn(g.y0, __dmul_rn((double)row + 0.5, g.delta_xy));
}

// Visits every kept (bin, weight) pair of the column; f(bin, weight).
template <typename F>
__device__ __forceinline__ void acol_visit(const MbirGeom &g, double x, double y, int view, F &&f)
{
    const double r = __dsub_rn(__dmul_rn(x, g.cosv[view]), __dmul_rn(y, g.sinv[view]));
    const double rmin = __dsub_rn(r, g.delta_xy), rmax = __dadd_rn(r, g.delta_xy);
    if (rmax < g.R0 || rmin > g.RMax) return;
    int imin = (int)floor(__ddiv_rn(__dsub_rn(rmin, g.R0), g.delta_r));
    int imax = (int)floor(__ddiv_rn(__dsub_rn(rmax, g.R0), g.delta_r));
    if (imax >= g.N_r) imax = g.N_r - 1;
    if (imin < 0) imin = 0;
    const float *H = g.H_r + (size_t)view * (MBIR_RESP_BINS + 1);
    for (int j = imin; j <= imax; j++) {
        const double rc = __dadd_rn(g.R0, __dmul_rn((double)j + 0.5, g.delta_r));
        const double dr = fabs(__dsub_rn(r, rc));
        const int id = (int)floor(__ddiv_rn(dr, g.OffsetR));
        if (id >= 0 && id < MBIR_RESP_BINS) {
            const double w1 = __dsub_rn(dr, __dmul_rn((double)id, g.OffsetR));
            const double w2 = __dsub_rn(g.OffsetR, w1);
            const double f1 = __ddiv_rn(
                __dadd_rn(__dmul_rn(w2, (double)__ldg(H + id)), __dmul_rn(w1, (double)__ldg(H + id + 1))),
                g.OffsetR);
            if (f1 > 0) f(j, f1);
        }
    }
}

__device__ __forceinline__ int acol_exact(const MbirGeom &g, double x, double y, int view, int *idx,
                                          double *val, int cap)
{
    int n = 0;
    acol_visit(g, x, y, view, [&](int j, double f1) {
        if (n < cap) {
            idx[n] = j;
            val[n] = f1;
            n++;
        }
    });
    return n;
}

// qGGMRF derivative rho'(d) (XT_ICD_update.c:93-128).
__device__ __forceinline__ double qggmrf_deriv(double d, double sQ, double sQP, double c)
{
    const double ad = fabs(d);
    const double t1 = pow(ad, kQ - kP) / sQP;
    const double t2 = ad;  // |d|^(q-1), q = 2
    const double t3 = c + t1;
    const double m = __dsub_rn(kQ, __ddiv_rn(__dmul_rn(kQ - kP, t1), t3));
    const double v = __dmul_rn(t2 / __dmul_rn(t3, sQ), m);
    return d < 0 ? -v : v;
}

// qGGMRF potential rho(d) (XT_ICD_update.c:83-91); pow(|d|, 2) is |d|^2.
__device__ __forceinline__ double qggmrf_value(double d, double sQ, double sQP, double c)
{
    const double ad = fabs(d);
    // |d|^(q - p) as exp((q - p) log |d|) in FP64 (within a few ulp of pow;
    // 0 for d = 0)
    const double pw = ad > 0.0 ? exp((kQ - kP) * log(ad)) : 0.0;
    return (__dmul_rn(ad, ad) / sQ) / (c + pw / sQP);
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// ----------------------------------------------------------------------------
// Reference-schedule ICD (XT_VoxUpdate.c:43-281 inside the half-sweeps of
// XT_ICD_update.c:974-1060).  One CTA per (frame, z-block) task; it walks the
// task's voxel lines in list order and, per line, the slices of the block in
// order, exactly as updateVoxels_Atten does.  Per voxel:
//   * every thread forms theta1/theta2 over its views (generalized-Huber
//     weights; a view is always handled by the same thread, so the error
//     sinogram entries it updates are private to it);
//   * warp 0 gathers the 26+2 neighbourhood, applies zero skipping and forms
//     the surrogate's prior sums;
//   * thread 0 solves the 1-D surrogate with over-relaxation (FP64), stores the
//     voxel and broadcasts the float-rounded change;
//   * every thread subtracts a * change from its error sinogram entries.
// The A column of each (line, view) is computed once per line into a cache
// (shared memory when it fits, else a per-task global slab).
// ----------------------------------------------------------------------------
template <int NT>
__global__ void __launch_bounds__(NT) k_icd_ref(MbirGeom g, MbirPrior pr, MbirDev dv,
                                                 const MbirTask *__restrict__ tasks,
                                                 MbirTaskOut *__restrict__ out, int iter, int amax,
                                                 int acache_smem, char *acache_global,
                                                 size_t acache_bytes)
{
    extern __shared__ __align__(16) char smem_raw[];
    __shared__ double s_t1[NT / 32], s_t2[NT / 32];
    __shared__ double s_pt1, s_pt2, s_V, s_delta;
    __shared__ int s_zs, s_skip;
    constexpr int NW = NT / 32;
    const MbirTask t = tasks[blockIdx.x];
    const int i = t.frame;
    const int nv = g.view_num[i];
    const int *vl = g.view_idx + (size_t)i * g.max_views;
    char *base = acache_smem ? smem_raw : acache_global + (size_t)blockIdx.x * acache_bytes;
    double *aval = reinterpret_cast<double *>(base);
    int *aidx = reinterpret_cast<int *>(aval + (size_t)nv * amax);
    int *acnt = aidx + (size_t)nv * amax;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int N_x = g.N_x, N_y = g.N_y, N_z = g.N_z;
    const size_t plane = (size_t)N_y * N_x;

    double vox_mag = 0.0;
    long long upd = 0, zskips = 0;
    for (int li = t.b0; li <= t.b1; li++) {
        const int k = t.xs[li], j = t.ys[li];
        if (threadIdx.x == 0) t.mag[(size_t)j * N_x + k] = 0.0f;
        const double xc = voxel_x(g, k), yc = voxel_y(g, j);
        for (int v = threadIdx.x; v < nv; v += NT)
            acnt[v] = acol_exact(g, xc, yc, vl[v], aidx + (size_t)v * amax, aval + (size_t)v * amax, amax);
        if (dv.mask[(size_t)j * N_x + k] != 1) continue;
        for (int s = t.z0; s <= t.z1; s++) {
            // ---- data term: theta1, theta2 ----
            double th1 = 0.0, th2 = 0.0;
            for (int v = threadIdx.x; v < nv; v += NT) {
                const int view = vl[v], cnt = acnt[v];
                for (int q = 0; q < cnt; q++) {
                    const int ir = aidx[(size_t)v * amax + q];
                    const double a = aval[(size_t)v * amax + q];
                    for (int rr = 0; rr < g.m_z; rr++) {
                        const size_t o = ((size_t)(s * g.m_z + rr) * g.N_p + view) * g.N_r + ir;
                        const double ed = dv.e[o], wd = dv.w[o];
                        const double sw = sqrt(wd);
                        if (fabs(__dmul_rn(ed, sw)) < pr.hT) {
                            th2 = __dadd_rn(th2, __dmul_rn(__dmul_rn(a, a), wd));
                            th1 = __dadd_rn(th1, -__dmul_rn(__dmul_rn(ed, a), wd));
                        } else {
                            const double tmp = __ddiv_rn(__dmul_rn(__dmul_rn(pr.hT, pr.hdelta), sw), fabs(ed));
                            th2 = __dadd_rn(th2, __dmul_rn(__dmul_rn(a, a), tmp));
                            th1 = __dadd_rn(th1, -__dmul_rn(__dmul_rn(ed, a), tmp));
                        }
                    }
                }
            }
            th1 = warp_sum(th1);
            th2 = warp_sum(th2);
            if (lane == 0) {
                s_t1[warp] = th1;
                s_t2[warp] = th2;
            }
            // ---- prior: 26 spatial + 2 temporal neighbours (warp 0) ----
            if (warp == 0) {
                const float *xf = dv.x + (size_t)i * N_z * plane;
                const double V = xf[(size_t)s * plane + (size_t)j * N_x + k];
                double nb = 0.0, b = 0.0;
                bool valid = false;
                if (lane < 27 && lane != 13) {
                    const int dz = lane / 9 - 1, dy = (lane / 3) % 3 - 1, dx = lane % 3 - 1;
                    const int zz = s + dz, yy = j + dy, xx = k + dx;
                    if (slab_has_z(g, dv, zz) && yy >= 0 && yy < N_y && xx >= 0 && xx < N_x) {
                        valid = true;
                        nb = slab_plane(g, dv, i, zz)[(size_t)yy * N_x + xx];
                    }
                    if (valid) {
                        const double d0 = V - nb;
                        const double prm = d0 != 0 ? qggmrf_deriv(d0, pr.sSQ, pr.sSQP, pr.c_s) / d0
                                                   : kQ / (pr.sSQ * pr.c_s);
                        b = pr.SF[lane] * prm;
                    }
                } else if (lane == 27 || lane == 28) {
                    const int ti = i + (lane == 27 ? -1 : 1);
                    if (ti >= 0 && ti < g.N_time) {
                        valid = true;
                        nb = dv.x[((size_t)ti * N_z + s) * plane + (size_t)j * N_x + k];
                        const double d0 = V - nb;
                        const double prm = d0 != 0 ? qggmrf_deriv(d0, pr.sTQ, pr.sTQP, pr.c_t) / d0
                                                   : kQ / (pr.sTQ * pr.c_t);
                        b = pr.TF * prm;
                    }
                }
                const unsigned pos = __ballot_sync(0xffffffffu, valid && nb > 0.0);
                double p1 = warp_sum(__dmul_rn(b, nb));
                double p2 = warp_sum(b);
                if (lane == 0) {
                    s_pt1 = p1;
                    s_pt2 = p2;
                    s_V = V;
                    s_zs = (V == 0.0 && iter > 1 && pos == 0u) ? 1 : 0;
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                if (s_zs) {
                    s_skip = 1;
                    zskips++;
                } else {
                    double T1 = 0.0, T2 = 0.0;
#pragma unroll
                    for (int w = 0; w < NW; w++) {
                        T1 += s_t1[w];
                        T2 += s_t2[w];
                    }
                    const double V = s_V;
                    const double u = __ddiv_rn(__dsub_rn(__dadd_rn(s_pt1, __dmul_rn(T2, V)), T1),
                                               __dadd_rn(s_pt2, T2));
                    const double xn = __dadd_rn(V, __dmul_rn(pr.alpha, __dsub_rn(u, V)));
                    const float xf = (float)xn;
                    const size_t o = ((size_t)i * N_z + s) * plane + (size_t)j * N_x + k;
                    dv.x[o] = xf;
                    const double dl = (double)xf - V;
                    s_delta = dl;
                    s_skip = 0;
                    float *m = t.mag + (size_t)j * N_x + k;
                    *m = (float)((double)*m + fabs(dl));
                    vox_mag += fabs((double)xf);
                    upd++;
                }
            }
            __syncthreads();
            if (!s_skip) {
                const double dl = s_delta;
                for (int v = threadIdx.x; v < nv; v += NT) {
                    const int view = vl[v], cnt = acnt[v];
                    for (int q = 0; q < cnt; q++) {
                        const int ir = aidx[(size_t)v * amax + q];
                        const double a = aval[(size_t)v * amax + q];
                        for (int rr = 0; rr < g.m_z; rr++) {
                            const size_t o = ((size_t)(s * g.m_z + rr) * g.N_p + view) * g.N_r + ir;
                            dv.e[o] = (float)__dsub_rn((double)dv.e[o], __dmul_rn(a, dl));
                        }
                    }
                }
            }
        }
    }
    if (threadIdx.x == 0) {
        out[blockIdx.x].vox_mag = vox_mag;
        out[blockIdx.x].updates = upd;
        out[blockIdx.x].zero_skips = zskips;
    }
}

// ----------------------------------------------------------------------------
// Deterministic block reduction helpers: each block writes one partial per
// quantity; a single block sums the partials in index order.
// ----------------------------------------------------------------------------
template <int NQ>
__device__ void block_partials(double (&v)[NQ], double *partials, int nparts)
{
    __shared__ double sh[NQ][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int q = 0; q < NQ; q++) {
        double s = warp_sum(v[q]);
        if (lane == 0) sh[q][warp] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NQ; q++) {
            double s = 0.0;
            for (int w = 0; w < nw; w++) s += sh[q][w];
            partials[(size_t)q * nparts + blockIdx.x] = s;
        }
    }
}

__global__ void k_sum_partials(const double *partials, int nparts, int nq, double *result)
{
    __shared__ double sh[32];
    for (int q = 0; q < nq; q++) {
        double s = 0.0;
        for (int b = threadIdx.x; b < nparts; b += blockDim.x) s += partials[(size_t)q * nparts + b];
        s = warp_sum(s);
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double tot = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) tot += sh[w];
            result[q] = tot;
        }
        __syncthreads();
    }
}

// ----------------------------------------------------------------------------
// MAP cost (XT_ICD_update.c:186-319): generalized-Huber data term and the
// prior over the 13 causal spatial pairs plus the forward temporal pair, in
// FP64.  partials[0][b] = data sum, partials[1][b] = prior sum.
// ----------------------------------------------------------------------------
__global__ void k_cost(MbirGeom g, MbirPrior pr, MbirDev dv, double *partials, int nparts)
{
    double v[2] = {0.0, 0.0};
    const size_t ns = (size_t)g.N_t * g.N_p * g.N_r;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t o = (size_t)blockIdx.x * blockDim.x + threadIdx.x; o < ns; o += stride) {
        double t = __dmul_rn((double)dv.e[o], sqrt((double)dv.w[o]));
        if (fabs(t) < pr.hT)
            t = __dmul_rn(t, t);
        else
            t = __dadd_rn(__dmul_rn(__dmul_rn(2.0 * pr.hdelta, pr.hT), fabs(t)),
                          __dmul_rn(__dmul_rn(pr.hT, pr.hT), 1.0 - 2.0 * pr.hdelta));
        v[0] += t;
    }
    const size_t plane = (size_t)g.N_y * g.N_x;
    const size_t nvox = (size_t)g.N_time * g.N_z * plane;
    // causal spatial offsets (dz, dy, dx) and their filter index 9*(dz+1)+3*(dy+1)+(dx+1)
    const int off[13][3] = {{0, 0, 1},  {0, 1, -1}, {0, 1, 0},  {0, 1, 1},  {1, -1, 0},
                            {1, 0, 0},  {1, 1, 0},  {1, -1, -1}, {1, -1, 1}, {1, 0, -1},
                            {1, 1, -1}, {1, 1, 1},  {1, 0, 1}};
    for (size_t o = (size_t)blockIdx.x * blockDim.x + threadIdx.x; o < nvox; o += stride) {
        const int k = (int)(o % g.N_x);
        const int j = (int)((o / g.N_x) % g.N_y);
        const int s = (int)((o / plane) % g.N_z);
        const int i = (int)(o / ((size_t)g.N_z * plane));
        const float xv = dv.x[o];
        for (int n = 0; n < 13; n++) {
            const int zz = s + off[n][0], yy = j + off[n][1], xx = k + off[n][2];
            if (zz < g.N_z + (dv.halo_hi ? 1 : 0) && yy >= 0 && yy < g.N_y && xx >= 0 && xx < g.N_x) {
                // the pair with the slab above's bottom slice is this slab's
                // (computeCost, XT_ICD_update.c:207-210)
                const float nbv = slab_plane(g, dv, i, zz)[(size_t)yy * g.N_x + xx];
                const double dl = (double)__fsub_rn(xv, nbv);
                const int fi = 9 * (off[n][0] + 1) + 3 * (off[n][1] + 1) + (off[n][2] + 1);
                v[1] += pr.SF[fi] * qggmrf_value(dl, pr.sSQ, pr.sSQP, pr.c_s);
            }
        }
        if (i + 1 < g.N_time) {
            const double dl = (double)__fsub_rn(xv, dv.x[o + (size_t)g.N_z * plane]);
            v[1] += pr.TF * qggmrf_value(dl, pr.sTQ, pr.sTQP, pr.c_t);
        }
    }
    block_partials<2>(v, partials, nparts);
}

// ----------------------------------------------------------------------------
// Ring offsets (XT_ICD_update.c:753-927).  Pass 1: per detector element
// (t, r), num and den summed over all views in view order (FP64, with the
// reference's float products), plus block partials of sum(d + num/den) and
// sum(1/den) for the zero-mean gamma.  Pass 2: shift = (num - gamma)/den,
// d += shift, e -= shift over all views (types 1, 2); type 3 (rectangular
// patches with no constraint windows, as on the reference's reconstruct path)
// sets d = b/Lambda and e += d_old - d.
// ----------------------------------------------------------------------------
__global__ void k_offset_terms(MbirGeom g, MbirPrior pr, MbirDev dv, int type, double *num, double *den,
                               double *partials, int nparts)
{
    double v[2] = {0.0, 0.0};
    const size_t nel = (size_t)g.N_t * g.N_r;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < nel; q += stride) {
        const int t = (int)(q / g.N_r), r = (int)(q % g.N_r);
        const float dq = dv.d[q];
        double nm = 0.0, dn = 0.0;
        for (int p = 0; p < g.N_p; p++) {
            const size_t o = ((size_t)t * g.N_p + p) * g.N_r + r;
            const float ef = dv.e[o], wf = dv.w[o];
            const double sw = sqrt((double)wf);
            const double tmp = __dmul_rn(__dmul_rn(pr.hT, pr.hdelta), sw);
            const bool sel = fabs(__dmul_rn((double)ef, sw)) < pr.hT;
            if (type == 3) {
                if (sel) {
                    dn += (double)wf;
                    nm += (double)__fmul_rn(__fadd_rn(ef, dq), wf);
                } else {
                    const double om = __ddiv_rn(tmp, fabs((double)ef));
                    dn += om;
                    nm += __ddiv_rn(__dmul_rn((double)__fadd_rn(ef, dq), tmp), fabs((double)ef));
                }
            } else {
                if (sel) {
                    nm += (double)__fmul_rn(ef, wf);
                    dn += (double)wf;
                } else {
                    const double sg = (double)((ef > 0) - (ef < 0));
                    nm += __dmul_rn(tmp, sg);
                    dn += __ddiv_rn(tmp, fabs((double)ef));
                }
            }
        }
        num[q] = nm;
        den[q] = dn;
        v[0] += (double)dq + nm / dn;
        v[1] += 1.0 / dn;
    }
    block_partials<2>(v, partials, nparts);
}

__global__ void k_offset_apply(MbirGeom g, MbirDev dv, int type, const double *num, const double *den,
                               const double *sums, const double *xw)
{
    const size_t nel = (size_t)g.N_t * g.N_r;
    const double gamma = type == 2 ? sums[0] / sums[1] : 0.0;
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nel) return;
    const int t = (int)(q / g.N_r), r = (int)(q % g.N_r);
    if (type == 3) {
        const float xn = xw ? (float)xw[q] : (float)((num[q] - 0.0) / den[q]);
        const float dd = __fsub_rn(dv.d[q], xn);
        for (int p = 0; p < g.N_p; p++) {
            const size_t o = ((size_t)t * g.N_p + p) * g.N_r + r;
            dv.e[o] = __fadd_rn(dv.e[o], dd);
        }
        dv.d[q] = xn;
    } else {
        const double sh = __ddiv_rn(num[q] - gamma, den[q]);
        dv.d[q] = (float)__dadd_rn((double)dv.d[q], sh);
        for (int p = 0; p < g.N_p; p++) {
            const size_t o = ((size_t)t * g.N_p + p) * g.N_r + r;
            dv.e[o] = (float)__dsub_rn((double)dv.e[o], sh);
        }
    }
}

// The same update spread over the views: k_offset_chunks sums views
// [c VC, (c + 1) VC) of each detector element into partial num / den
// [c][element]; k_offset_combine adds the chunks in chunk order (a fixed
// order: deterministic) and forms the block partials of the zero-mean gamma;
// k_offset_shift turns num / den (and gamma, or the constrained solution)
// into each element's shift and new offset; k_offset_apply_e applies the
// shift to every sinogram entry.
__global__ void k_offset_chunks(MbirGeom g, MbirPrior pr, MbirDev dv, int type, int vc, double *__restrict__ pnum,
                                double *__restrict__ pden)
{
    const int nel = g.N_t * g.N_r;
    const int q = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
    if (q >= nel) return;
    const int t = q / g.N_r, r = q - t * g.N_r;
    const float dq = dv.d[q];
    double nm = 0.0, dn = 0.0;
    const int p1 = min(g.N_p, (c + 1) * vc);
    for (int p = c * vc; p < p1; p++) {
        const size_t o = ((size_t)t * g.N_p + p) * g.N_r + r;
        const float ef = dv.e[o], wf = dv.w[o];
        const double sw = sqrt((double)wf);
        const double tmp = __dmul_rn(__dmul_rn(pr.hT, pr.hdelta), sw);
        const bool sel = fabs(__dmul_rn((double)ef, sw)) < pr.hT;
        if (type == 3) {
            if (sel) {
                dn += (double)wf;
                nm += (double)__fmul_rn(__fadd_rn(ef, dq), wf);
            } else {
                const double om = __ddiv_rn(tmp, fabs((double)ef));
                dn += om;
                nm += __ddiv_rn(__dmul_rn((double)__fadd_rn(ef, dq), tmp), fabs((double)ef));
            }
        } else {
            if (sel) {
                nm += (double)__fmul_rn(ef, wf);
                dn += (double)wf;
            } else {
                const double sg = (double)((ef > 0) - (ef < 0));
                nm += __dmul_rn(tmp, sg);
                dn += __ddiv_rn(tmp, fabs((double)ef));
            }
        }
    }
    pnum[(size_t)c * nel + q] = nm;
    pden[(size_t)c * nel + q] = dn;
}

__global__ void k_offset_combine(MbirGeom g, MbirDev dv, int nchunks, const double *__restrict__ pnum,
                                 const double *__restrict__ pden, double *__restrict__ num, double *__restrict__ den,
                                 double *partials, int nparts)
{
    double v[2] = {0.0, 0.0};
    const size_t nel = (size_t)g.N_t * g.N_r;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < nel; q += stride) {
        double nm = 0.0, dn = 0.0;
        for (int c = 0; c < nchunks; c++) {
            nm += pnum[(size_t)c * nel + q];
            dn += pden[(size_t)c * nel + q];
        }
        num[q] = nm;
        den[q] = dn;
        v[0] += (double)dv.d[q] + nm / dn;
        v[1] += 1.0 / dn;
    }
    block_partials<2>(v, partials, nparts);
}

// per element: the shift of e (types 1, 2: (num - gamma) / den, e -= shift;
// type 3: d_old - x, e += it), into num[q]; the new offset into d
__global__ void k_offset_shift(MbirGeom g, MbirDev dv, int type, double *num, const double *den, const double *sums,
                               const double *xw)
{
    const size_t nel = (size_t)g.N_t * g.N_r;
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nel) return;
    if (type == 3) {
        const float xn = xw ? (float)xw[q] : (float)((num[q] - 0.0) / den[q]);
        num[q] = (double)__fsub_rn(dv.d[q], xn);
        dv.d[q] = xn;
    } else {
        const double gamma = type == 2 ? sums[0] / sums[1] : 0.0;
        const double sh = __ddiv_rn(num[q] - gamma, den[q]);
        dv.d[q] = (float)__dadd_rn((double)dv.d[q], sh);
        num[q] = sh;
    }
}

__global__ void k_offset_apply_e(MbirGeom g, MbirDev dv, int type, const double *__restrict__ shift)
{
    const size_t ns = (size_t)g.N_t * g.N_p * g.N_r;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t o = (size_t)blockIdx.x * blockDim.x + threadIdx.x; o < ns; o += stride) {
        const size_t r = o % g.N_r, t = o / ((size_t)g.N_p * g.N_r);
        const double sh = shift[t * g.N_r + r];
        if (type == 3)
            dv.e[o] = __fadd_rn(dv.e[o], (float)sh);
        else
            dv.e[o] = (float)__dsub_rn((double)dv.e[o], sh);
    }
}

// ----------------------------------------------------------------------------
// Ring offsets of type 3 with rectangular-patch constraint windows
// (constrained_quad_opt, XT_OffsetError.c:99-168): minimise
// sum Lambda (x - b / Lambda)^2 subject to A x = 0 for the M windows A.
// With D = A Lambda^-1 A^T (symmetric positive definite) and
// c = A (b / Lambda): D y = c, x = (b - A^T y) / Lambda.  One CTA, FP64: c per
// window and D per overlapping window pair as fixed-order sums over the
// (host-built) element lists, Cholesky factorisation of D in place
// (column by column), forward and back substitution, then x per element.
// The reference inverts D by LU decomposition; the solution is the same up
// to FP64 rounding.  err |= 16 if D is not positive definite.
// ----------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum_d(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void __launch_bounds__(1024) k_offset_windows(OffsetWindows W, const double *__restrict__ b,
                                                         const double *__restrict__ L, double *__restrict__ xw,
                                                         int *err)
{
    const int M = W.M, tid = threadIdx.x, nthr = blockDim.x, lane = tid & 31, warp = tid >> 5,
              nw = nthr >> 5;
    double *D = W.D, *y = W.y;
    for (int q = tid; q < M * M; q += nthr) D[q] = 0.0;
    __syncthreads();
    for (int m = warp; m < M; m += nw) {
        double s = 0.0;
        for (int k = W.win_off[m] + lane; k < W.win_off[m + 1]; k += 32) {
            const int q = W.win_el[k];
            s += (double)W.win_a[k] * b[q] / L[q];
        }
        s = warp_sum_d(s);
        if (lane == 0) y[m] = s;
    }
    for (int p = warp; p < W.npairs; p += nw) {
        double s = 0.0;
        for (int k = W.pair_off[p] + lane; k < W.pair_off[p + 1]; k += 32) {
            const int q = W.pair_el[k];
            s += (double)W.pair_ai[k] * (double)W.pair_aj[k] / L[q];
        }
        s = warp_sum_d(s);
        if (lane == 0) {
            D[W.pair_i[p] * M + W.pair_j[p]] = s;
            D[W.pair_j[p] * M + W.pair_i[p]] = s;
        }
    }
    __syncthreads();
    // D = L L^T, L in the lower triangle
    for (int k = 0; k < M; k++) {
        if (tid == 0) {
            double v = D[k * M + k];
            if (!(v > 0.0)) {
                atomicOr(err, 16);
                v = 1.0;
            }
            D[k * M + k] = sqrt(v);
        }
        __syncthreads();
        const double dk = D[k * M + k];
        for (int i = k + 1 + tid; i < M; i += nthr) D[i * M + k] /= dk;
        __syncthreads();
        const int n = M - k - 1;
        for (int q = tid; q < n * n; q += nthr) {
            const int i = k + 1 + q / n, j = k + 1 + q % n;
            if (j <= i) D[i * M + j] -= D[i * M + k] * D[j * M + k];
        }
        __syncthreads();
    }
    // L z = c, then L^T y = z (y holds c on entry)
    for (int k = 0; k < M; k++) {
        if (tid == 0) y[k] /= D[k * M + k];
        __syncthreads();
        for (int i = k + 1 + tid; i < M; i += nthr) y[i] -= D[i * M + k] * y[k];
        __syncthreads();
    }
    for (int k = M - 1; k >= 0; k--) {
        if (tid == 0) y[k] /= D[k * M + k];
        __syncthreads();
        for (int i = tid; i < k; i += nthr) y[i] -= D[k * M + i] * y[k];
        __syncthreads();
    }
    for (int q = tid; q < W.nel; q += nthr) {
        double v = 0.0;
        for (int k = W.el_off[q]; k < W.el_off[q + 1]; k++) v += (double)W.el_a[k] * y[W.el_m[k]];
        xw[q] = (b[q] - v) / L[q];
    }
}

// ----------------------------------------------------------------------------
// Multi-resolution hand-off on the device: the x2 up-samplings of the object
// and the update-magnitude map between stages (initObject / upsample_*,
// XT_ICD_update.c:323-651), in the operation order of the host versions
// (mbir_setup.cpp upsample_xy / upsample_xyz), so the results are identical.
// Interior samples are (a + 3 b) / 4 and (3 b + c) / 4 of the two nearest
// coarse ones, edge samples repeat the edge value.
// ----------------------------------------------------------------------------
// x-pass value at fine column X of coarse row r (length n_x), in double
__device__ __forceinline__ double up_x(const float *r, int n_x, int X)
{
    const int ox = 2 * n_x;
    if (X == 0) return (double)r[0];
    if (X == 1) return __ddiv_rn(__dadd_rn(__dmul_rn(3.0, (double)r[0]), (double)r[1]), 4.0);
    if (X == ox - 1) return (double)r[n_x - 1];
    if (X == ox - 2) return __ddiv_rn(__dadd_rn((double)r[n_x - 2], __dmul_rn(3.0, (double)r[n_x - 1])), 4.0);
    const int k = X >> 1;
    if ((X & 1) == 0) return __ddiv_rn(__dadd_rn((double)r[k - 1], __dmul_rn(3.0, (double)r[k])), 4.0);
    return __ddiv_rn(__dadd_rn(__dmul_rn(3.0, (double)r[k]), (double)r[k + 1]), 4.0);
}

// slices up-sampled in x and y only (same slice count)
__global__ void k_upsample_xy(const float *__restrict__ in, float *__restrict__ out, int n_z, int n_y, int n_x)
{
    const int ox = 2 * n_x, oy = 2 * n_y;
    const size_t n = (size_t)n_z * oy * ox;
    const size_t o = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    const int X = (int)(o % ox), Y = (int)((o / ox) % oy), s = (int)(o / ((size_t)ox * oy));
    const float *I = in + (size_t)s * n_y * n_x;
    // the x-pass rows are stored as float
    auto b = [&](int j) { return (float)up_x(I + (size_t)j * n_x, n_x, X); };
    float v;
    if (Y == 0)
        v = b(0);
    else if (Y == 1)
        v = (float)__ddiv_rn(__dadd_rn(__dmul_rn(3.0, (double)b(0)), (double)b(1)), 4.0);
    else if (Y == oy - 1)
        v = b(n_y - 1);
    else if (Y == oy - 2)
        v = (float)__ddiv_rn(__dadd_rn((double)b(n_y - 2), __dmul_rn(3.0, (double)b(n_y - 1))), 4.0);
    else {
        const int j = Y >> 1;
        if ((Y & 1) == 0)
            v = (float)__ddiv_rn(__dadd_rn((double)b(j - 1), __dmul_rn(3.0, (double)b(j))), 4.0);
        else  // float arithmetic for 3 b + c, as the host version
            v = (float)__ddiv_rn((double)__fadd_rn(__fmul_rn(3.0f, b(j)), b(j + 1)), 4.0);
    }
    out[o] = v;
}

// up-sampled in x, y and z (twice the slices); every pass in double
__global__ void k_upsample_xyz(const float *__restrict__ in, float *__restrict__ out, int n_z, int n_y, int n_x)
{
    const int ox = 2 * n_x, oy = 2 * n_y, oz = 2 * n_z;
    const size_t n = (size_t)oz * oy * ox;
    const size_t o = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    const int X = (int)(o % ox), Y = (int)((o / ox) % oy), Z = (int)(o / ((size_t)ox * oy));
    auto b2 = [&](int s, int j) { return up_x(in + ((size_t)s * n_y + j) * n_x, n_x, X); };
    auto b3 = [&](int s) {
        if (Y == 0) return b2(s, 0);
        if (Y == 1) return __ddiv_rn(__dadd_rn(__dmul_rn(3.0, b2(s, 0)), b2(s, 1)), 4.0);
        if (Y == oy - 1) return b2(s, n_y - 1);
        if (Y == oy - 2) return __ddiv_rn(__dadd_rn(b2(s, n_y - 2), __dmul_rn(3.0, b2(s, n_y - 1))), 4.0);
        const int j = Y >> 1;
        if ((Y & 1) == 0) return __ddiv_rn(__dadd_rn(b2(s, j - 1), __dmul_rn(3.0, b2(s, j))), 4.0);
        return __ddiv_rn(__dadd_rn(__dmul_rn(3.0, b2(s, j)), b2(s, j + 1)), 4.0);
    };
    double v;
    if (Z == 0)
        v = b3(0);
    else if (Z == 1)
        v = __ddiv_rn(__dadd_rn(__dmul_rn(3.0, b3(0)), b3(1)), 4.0);
    else if (Z == oz - 1)
        v = b3(n_z - 1);
    else if (Z == oz - 2)
        v = __ddiv_rn(__dadd_rn(__dmul_rn(3.0, b3(n_z - 1)), b3(n_z - 2)), 4.0);
    else {
        const int s = Z >> 1;
        if ((Z & 1) == 0)
            v = __ddiv_rn(__dadd_rn(b3(s - 1), __dmul_rn(3.0, b3(s))), 4.0);
        else
            v = __ddiv_rn(__dadd_rn(__dmul_rn(3.0, b3(s)), b3(s + 1)), 4.0);
    }
    out[o] = (float)v;
}


// ----------------------------------------------------------------------------
// Variance (XT_ICD_update.c:720-751).  Pass 1 restores w_orig = w * sigma^2
// (float) and sums e^2 w_orig (selected, float products) or
// |e| delta T sqrt(w_orig sigma^2) (zingers); pass 2 divides by the new sigma^2.
// ----------------------------------------------------------------------------
__global__ void k_variance(MbirGeom g, MbirPrior pr, MbirDev dv, double var_est, double *partials,
                           int nparts)
{
    double v[1] = {0.0};
    const size_t ns = (size_t)g.N_t * g.N_p * g.N_r;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t o = (size_t)blockIdx.x * blockDim.x + threadIdx.x; o < ns; o += stride) {
        const float ef = dv.e[o], wold = dv.w[o];
        const bool sel = fabs(__dmul_rn((double)ef, sqrt((double)wold))) < pr.hT;
        const float wn = (float)__dmul_rn((double)wold, var_est);
        dv.w[o] = wn;
        if (sel)
            v[0] += (double)__fmul_rn(__fmul_rn(ef, ef), wn);
        else
            v[0] += __dmul_rn(__dmul_rn(__dmul_rn(fabs((double)ef), pr.hdelta), pr.hT),
                              sqrt(__dmul_rn((double)wn, var_est)));
    }
    block_partials<1>(v, partials, nparts);
}

__global__ void k_variance_apply(MbirGeom g, MbirDev dv, double var_new)
{
    const size_t ns = (size_t)g.N_t * g.N_p * g.N_r;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t o = (size_t)blockIdx.x * blockDim.x + threadIdx.x; o < ns; o += stride)
        dv.w[o] = (float)__ddiv_rn((double)dv.w[o], var_new);
}

// ----------------------------------------------------------------------------
// NHICD voxel-selection criterion (XT_NHICD.c:128-162): 5x5 Hamming-weighted
// sum of the update-magnitude map, zero outside the image.
// ----------------------------------------------------------------------------
__constant__ double c_hamming[25] = {0.0064, 0.0432, 0.0800, 0.0432, 0.0064, 0.0432, 0.2916,
                                     0.5400, 0.2916, 0.0432, 0.0800, 0.5400, 1.0000, 0.5400,
                                     0.0800, 0.0432, 0.2916, 0.5400, 0.2916, 0.0432, 0.0064,
                                     0.0432, 0.0800, 0.0432, 0.0064};

__global__ void k_vsc_filter(const float *mag, float *filt, int planes, int N_y, int N_x)
{
    const size_t n = (size_t)planes * N_y * N_x;
    const size_t o = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    const int k = (int)(o % N_x), j = (int)((o / N_x) % N_y);
    const float *m = mag + (o - (size_t)j * N_x - k);
    double acc = 0.0;
    for (int p = -2; p <= 2; p++)
        for (int q = -2; q <= 2; q++)
            if (j + p >= 0 && j + p < N_y && k + q >= 0 && k + q < N_x)
                acc = __dadd_rn(acc, __dmul_rn(c_hamming[(p + 2) * 5 + q + 2], (double)m[(size_t)(j + p) * N_x + k + q]));
    filt[o] = (float)acc;
}

// ----------------------------------------------------------------------------
// Detector response (XT_Profile.c:47-170), GPU half.  One CTA per view: the
// trapezoidal voxel profile sampled at 1536 points (as float, like the
// reference's VoxProfile), then for each of the 64 distances the sum over the
// 512-point beam in the reference's order, FP64 without contraction.
// trap[view][5] = (height, left corner, left near, right near, right corner).
// ----------------------------------------------------------------------------
__global__ void k_detector_response(const double *__restrict__ trap, const double *__restrict__ beam, int N_p,
                                    double OffsetR, double delta_xy, double r0, double step, double tc,
                                    float *__restrict__ H_r)
{
    __shared__ float prof[1536];
    __shared__ double bm[512];
    const int k = blockIdx.x;
    const double *t = trap + (size_t)k * 5;
    const double maxv = t[0], lc = t[1], ln = t[2], rn = t[3], rc = t[4];
    for (int p = threadIdx.x; p < 512; p += blockDim.x) bm[p] = beam[p];
    for (int j = threadIdx.x; j < 1536; j += blockDim.x) {
        const double tt = __ddiv_rn(__dmul_rn(2.0, (double)j), 1536.0);
        float v;
        if (tt <= lc || tt >= rc)
            v = 0.0f;
        else if (tt > rn)
            v = (float)__ddiv_rn(__dmul_rn(maxv, __dsub_rn(rc, tt)), __dsub_rn(rc, rn));
        else if (tt >= ln)
            v = (float)maxv;
        else
            v = (float)__ddiv_rn(__dmul_rn(maxv, __dsub_rn(tt, lc)), __dsub_rn(ln, lc));
        prof[j] = v;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < MBIR_RESP_BINS + 1; i += blockDim.x) {
        if (i == MBIR_RESP_BINS) {
            H_r[(size_t)k * (MBIR_RESP_BINS + 1) + i] = 0.0f;
            continue;
        }
        const double rmin = __dsub_rn(__dmul_rn((double)i, OffsetR), delta_xy);
        double acc = 0.0;
        for (int p = 0; p < 512; p++) {
            const double r = __dadd_rn(r0, __dmul_rn((double)p, step));
            const int pi = (int)floor(__dmul_rn(__dsub_rn(r, rmin), tc));
            if (pi >= 0 && pi <= 1535) acc = __dadd_rn(acc, __dmul_rn((double)prof[pi], bm[p]));
        }
        H_r[(size_t)k * (MBIR_RESP_BINS + 1) + i] = (float)acc;
    }
}

// Reference input layout [view][row][col] -> device layout [row][view][col];
// whole detector rows move, so reads and writes are both coalesced.
__global__ void k_to_slice_major(const float *__restrict__ in, float *__restrict__ out, int N_p, int N_t, int N_r)
{
    const size_t n = (size_t)N_p * N_t * N_r;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t o = (size_t)blockIdx.x * blockDim.x + threadIdx.x; o < n; o += stride) {
        const int r = (int)(o % N_r);
        const size_t pt = o / N_r;
        const int t = (int)(pt % N_t), p = (int)(pt / N_t);
        out[((size_t)t * N_p + p) * N_r + r] = in[o];
    }
}

}  // namespace

cudaError_t mbir_launch_upsample(const float *in, float *out, int n_z, int n_y, int n_x, bool z_too, cudaStream_t s)
{
    const size_t n = (size_t)(z_too ? 2 * n_z : n_z) * 4 * n_y * n_x;
    if (z_too)
        k_upsample_xyz<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(in, out, n_z, n_y, n_x);
    else
        k_upsample_xy<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(in, out, n_z, n_y, n_x);
    return cudaGetLastError();
}

// ---------------------------------------------------------------- launchers --
cudaError_t mbir_launch_detector_response(const double *trap, const double *beam, int N_p, double OffsetR,
                                          double delta_xy, double r0, double step, double tc, float *H_r,
                                          cudaStream_t s)
{
    k_detector_response<<<N_p, 128, 0, s>>>(trap, beam, N_p, OffsetR, delta_xy, r0, step, tc, H_r);
    return cudaGetLastError();
}

int mbir_amax(double delta_xy, double delta_r) { return (int)ceil(3 * delta_xy / delta_r) + 2; }

cudaError_t mbir_launch_to_slice_major(const float *in, float *out, int N_p, int N_t, int N_r, cudaStream_t s)
{
    k_to_slice_major<<<1184, 256, 0, s>>>(in, out, N_p, N_t, N_r);
    return cudaGetLastError();
}

cudaError_t mbir_launch_icd_ref(const MbirGeom &g, const MbirPrior &pr, const MbirDev &dv,
                                const MbirTask *tasks, int ntasks, MbirTaskOut *out, int iter,
                                int threads, size_t acache_bytes, void *acache_global,
                                cudaStream_t s)
{
    if (ntasks <= 0) return cudaSuccess;
    const int amax = mbir_amax(g.delta_xy, g.delta_r);
    const int smem_ok = acache_bytes <= 160 * 1024;
    const size_t sm = smem_ok ? acache_bytes : 0;
    cudaError_t e = cudaSuccess;
#define MBIR_LAUNCH_REF(NT)                                                                        \
    do {                                                                                           \
        e = cudaFuncSetAttribute(k_icd_ref<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,       \
                                 (int)(sm > 0 ? sm : 1));                                          \
        if (e != cudaSuccess) return e;                                                            \
        k_icd_ref<NT><<<ntasks, NT, sm, s>>>(g, pr, dv, tasks, out, iter, amax, smem_ok,           \
                                             (char *)acache_global, acache_bytes);                 \
    } while (0)
    if (threads <= 64)
        MBIR_LAUNCH_REF(64);
    else if (threads <= 128)
        MBIR_LAUNCH_REF(128);
    else
        MBIR_LAUNCH_REF(256);
#undef MBIR_LAUNCH_REF
    return cudaGetLastError();
}

cudaError_t mbir_launch_cost(const MbirGeom &g, const MbirPrior &pr, const MbirDev &dv,
                             double *partials, int nparts, double *result, cudaStream_t s)
{
    k_cost<<<nparts, 1024, 0, s>>>(g, pr, dv, partials, nparts);
    k_sum_partials<<<1, 1024, 0, s>>>(partials, nparts, 2, result);
    return cudaGetLastError();
}

int mbir_offset_chunks(const MbirGeom &g) { return (g.N_p + kOffsetViewChunk - 1) / kOffsetViewChunk; }

cudaError_t mbir_launch_offset(const MbirGeom &g, const MbirPrior &pr, const MbirDev &dv, int type,
                               double *num, double *den, double *partials, int nparts,
                               cudaStream_t s, const OffsetWindows *win, int *err, double *chunks)
{
    if (chunks) {
        const int nel = g.N_t * g.N_r, nc = mbir_offset_chunks(g);
        double *pnum = chunks, *pden = chunks + (size_t)nc * nel;
        k_offset_chunks<<<dim3((nel + 127) / 128, nc), 128, 0, s>>>(g, pr, dv, type, kOffsetViewChunk, pnum, pden);
        k_offset_combine<<<nparts, 128, 0, s>>>(g, dv, nc, pnum, pden, num, den, partials, nparts);
        double *sums = partials + 2 * (size_t)nparts;
        k_sum_partials<<<1, 1024, 0, s>>>(partials, nparts, 2, sums);
        const double *xw = nullptr;
        if (type == 3 && win && win->M > 0) {
            k_offset_windows<<<1, 1024, 0, s>>>(*win, num, den, win->x, err);
            xw = win->x;
        }
        k_offset_shift<<<(nel + 127) / 128, 128, 0, s>>>(g, dv, type, num, den, sums, xw);
        k_offset_apply_e<<<1184, 256, 0, s>>>(g, dv, type, num);
        return cudaGetLastError();
    }
    k_offset_terms<<<nparts, 128, 0, s>>>(g, pr, dv, type, num, den, partials, nparts);
    double *sums = partials + 2 * (size_t)nparts;
    k_sum_partials<<<1, 1024, 0, s>>>(partials, nparts, 2, sums);
    const size_t nel = (size_t)g.N_t * g.N_r;
    const double *xw = nullptr;
    if (type == 3 && win && win->M > 0) {
        k_offset_windows<<<1, 1024, 0, s>>>(*win, num, den, win->x, err);
        xw = win->x;
    }
    k_offset_apply<<<(unsigned)((nel + 127) / 128), 128, 0, s>>>(g, dv, type, num, den, sums, xw);
    return cudaGetLastError();
}

cudaError_t mbir_launch_variance(const MbirGeom &g, const MbirPrior &pr, const MbirDev &dv,
                                 double var_est, double *partials, int nparts, double *result,
                                 cudaStream_t s)
{
    k_variance<<<nparts, 256, 0, s>>>(g, pr, dv, var_est, partials, nparts);
    k_sum_partials<<<1, 1024, 0, s>>>(partials, nparts, 1, result);
    return cudaGetLastError();
}

cudaError_t mbir_launch_variance_apply(const MbirGeom &g, const MbirDev &dv, double var_new,
                                       cudaStream_t s)
{
    k_variance_apply<<<1184, 256, 0, s>>>(g, dv, var_new);
    return cudaGetLastError();
}

cudaError_t mbir_launch_vsc_filter(const float *mag, float *filt, int planes, int N_y, int N_x,
                                   cudaStream_t s)
{
    const size_t n = (size_t)planes * N_y * N_x;
    k_vsc_filter<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(mag, filt, planes, N_y, N_x);
    return cudaGetLastError();
}
