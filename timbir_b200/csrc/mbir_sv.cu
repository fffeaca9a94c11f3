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
// Inside the CTA, warp w owns slice w of the group: it walks the SV's lines
// one step at a time, and the slices of odd parity lag one line behind the
// even ones, so a voxel's z-neighbours are never being updated while it is;
// lines are ordered by their 2x2 (x, y) parity class, so consecutive lines
// are never x-y neighbours.  Only warp w touches slice w's band rows, so the
// error-sinogram updates need no synchronisation; one CTA barrier per line
// step hands the next line's A-matrix column (computed cooperatively into a
// three-slot ring) and the updated voxels to all warps.
//
// Concurrent SVs are chosen by the host so that no two share a prior
// neighbourhood (2x2 SV checkerboard, z-group and frame parity); they may
// share error-sinogram entries, whose concurrent changes they see at the next
// visit (the super-voxel ICD scheme of Wang et al., "High performance model
// based image reconstruction", PPoPP 2016).
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

// First / last detector bin of a voxel's footprint at a view, before
// clamping (XT_AMatrix.c:61-82), exact FP64.
__device__ __forceinline__ void bin_range(const MbirGeom &g, double x, double y, double c, double s,
                                          int &imin, int &imax)
{
    const double r = __dsub_rn(__dmul_rn(x, c), __dmul_rn(y, s));
    imin = (int)floor(__ddiv_rn(__dsub_rn(__dsub_rn(r, g.delta_xy), g.R0), g.delta_r));
    imax = (int)floor(__ddiv_rn(__dsub_rn(__dadd_rn(r, g.delta_xy), g.R0), g.delta_r));
}

__device__ __forceinline__ float warp_allsum(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
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

struct SvSmem {
    float *eb, *wb;          // [rows][W][Np]
    float *xb;               // [nz+2][S+2][S+2]
    float *tb;               // [2][nz][S][S]
    double *cs, *sn;         // [Np]
    int *vidx, *rlo;         // [Np]
    float *aval;             // [3][amax][Np]
    uint8_t *aoff;           // [3][amax][Np]
    uint8_t *acnt;           // [3][Np]
    int *order;              // [S*S] line (local index ly*S+lx) per step
    float *magl;             // [S*S]
};

__global__ void __launch_bounds__(1024) k_icd_sv(MbirGeom g, MbirPrior pr, MbirDev dv, SvParams sp,
                                                  const SvTask *__restrict__ tasks, float *scratch,
                                                  SvTaskOut *__restrict__ out, int iter, uint32_t seed,
                                                  int *err)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    const SvTask task = tasks[blockIdx.x];
    const int S = sp.S, W = sp.W, amax = sp.amax, mz = g.m_z;
    const int nz = task.nz, rows = nz * mz;
    const int i = task.frame;
    const int Np = g.view_num[i];
    const int NpS = sp.max_views;  // smem stride (views)
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int S2 = S + 2;

    // ---- carve shared memory (sizes fixed by the host in sp) ----
    SvSmem m;
    unsigned char *p = smraw;
    m.cs = reinterpret_cast<double *>(p); p += sizeof(double) * NpS;
    m.sn = reinterpret_cast<double *>(p); p += sizeof(double) * NpS;
    m.eb = reinterpret_cast<float *>(p); p += sizeof(float) * (size_t)sp.max_rows * W * NpS;
    m.wb = reinterpret_cast<float *>(p); p += sizeof(float) * (size_t)sp.max_rows * W * NpS;
    m.aval = reinterpret_cast<float *>(p); p += sizeof(float) * 3 * amax * NpS;
    m.xb = reinterpret_cast<float *>(p); p += sizeof(float) * (sp.max_nz + 2) * S2 * S2;
    m.tb = reinterpret_cast<float *>(p); p += sizeof(float) * 2 * sp.max_nz * S * S;
    m.magl = reinterpret_cast<float *>(p); p += sizeof(float) * S * S;
    m.vidx = reinterpret_cast<int *>(p); p += sizeof(int) * NpS;
    m.rlo = reinterpret_cast<int *>(p); p += sizeof(int) * NpS;
    m.order = reinterpret_cast<int *>(p); p += sizeof(int) * S * S;
    m.aoff = p; p += 3 * amax * NpS;
    m.acnt = p; p += 3 * NpS;
    __shared__ int s_nlines;
    __shared__ float s_red[32][4];

    const int k0 = task.k0, j0 = task.j0, z0 = task.z0;
    const int kx = min(S, g.N_x - k0), ky = min(S, g.N_y - j0);
    const int *vl = g.view_idx + (size_t)i * g.max_views;

    // ---- views, trig, band origin per view ----
    for (int v = tid; v < Np; v += nthr) {
        const int view = vl[v];
        m.vidx[v] = view;
        const double c = g.cosv[view], s = g.sinv[view];
        m.cs[v] = c;
        m.sn[v] = s;
        int lo = 1 << 30, a, b;
        const double xs[2] = {vx(g, k0), vx(g, k0 + kx - 1)};
        const double ys[2] = {vy(g, j0), vy(g, j0 + ky - 1)};
#pragma unroll
        for (int u = 0; u < 4; u++) {
            bin_range(g, xs[u & 1], ys[u >> 1], c, s, a, b);
            lo = min(lo, a);
        }
        m.rlo[v] = max(lo, 0);
    }
    // ---- in-mask lines, ordered by 2x2 parity class then a per-visit hash ----
    if (tid == 0) {
        int n = 0;
        for (int cls = 0; cls < 4; cls++) {
            const int base = n;
            for (int ly = 0; ly < ky; ly++)
                for (int lx = 0; lx < kx; lx++)
                    if ((((k0 + lx) & 1) | (((j0 + ly) & 1) << 1)) == cls &&
                        dv.mask[(size_t)(j0 + ly) * g.N_x + k0 + lx] == 1)
                        m.order[n++] = ly * S + lx;
            // shuffle the class with hash keys (Fisher-Yates)
            for (int q = n - 1; q > base; q--) {
                const uint32_t h = hash32(seed ^ hash32(blockIdx.x * 1315423911u + q));
                const int r = base + (int)(h % (uint32_t)(q - base + 1));
                const int t = m.order[q];
                m.order[q] = m.order[r];
                m.order[r] = t;
            }
        }
        s_nlines = n;
    }
    for (int q = tid; q < S * S; q += nthr) m.magl[q] = 0.0f;
    __syncthreads();
    const int nl = s_nlines;

    // ---- stage bands (e also to this CTA's scratch slot for the commit) ----
    float *scr = scratch + (size_t)blockIdx.x * sp.band_floats;
    const size_t bandn = (size_t)rows * W * Np;
    for (size_t q = tid; q < bandn; q += nthr) {
        const int v = (int)(q % Np);
        const int off = (int)((q / Np) % W);
        const int row = (int)(q / ((size_t)Np * W));
        const int r = m.rlo[v] + off;
        const int t = z0 * mz + row;
        float ev = 0.0f, wv = 0.0f;
        if (r < g.N_r) {
            const size_t o = ((size_t)t * g.N_p + m.vidx[v]) * g.N_r + r;
            ev = dv.e[o];
            wv = dv.w[o];
        }
        const size_t so = ((size_t)row * W + off) * NpS + v;
        m.eb[so] = ev;
        m.wb[so] = wv;
        scr[q] = ev;
    }
    // ---- voxel block with halo, temporal neighbours ----
    const size_t plane = (size_t)g.N_y * g.N_x;
    const float *xf = dv.x + (size_t)i * g.N_z * plane;
    const int nb = (nz + 2) * S2 * S2;
    for (int q = tid; q < nb; q += nthr) {
        const int lx = q % S2, ly = (q / S2) % S2, lz = q / (S2 * S2);
        const int xx = k0 + lx - 1, yy = j0 + ly - 1, zz = z0 + lz - 1;
        float v = 0.0f;
        if (xx >= 0 && xx < g.N_x && yy >= 0 && yy < g.N_y && zz >= 0 && zz < g.N_z)
            v = xf[(size_t)zz * plane + (size_t)yy * g.N_x + xx];
        m.xb[q] = v;
    }
    const int nt = 2 * nz * S * S;
    for (int q = tid; q < nt; q += nthr) {
        const int lx = q % S, ly = (q / S) % S, lz = (q / (S * S)) % nz, side = q / (nz * S * S);
        const int ti = i + (side == 0 ? -1 : 1);
        float v = 0.0f;
        if (ti >= 0 && ti < g.N_time && lx < kx && ly < ky)
            v = dv.x[((size_t)ti * g.N_z + z0 + lz) * plane + (size_t)(j0 + ly) * g.N_x + k0 + lx];
        m.tb[q] = v;
    }

    // ---- A-matrix column of line `li` into ring slot `slot` (exact bins) ----
    auto acol = [&](int li, int slot) {
        const int loc = m.order[li];
        const int col = k0 + loc % S, row = j0 + loc / S;
        const double x = vx(g, col), y = vy(g, row);
        float *av = m.aval + (size_t)slot * amax * NpS;
        uint8_t *ao = m.aoff + (size_t)slot * amax * NpS;
        uint8_t *ac = m.acnt + (size_t)slot * NpS;
        for (int v = tid; v < Np; v += nthr) {
            const double r = __dsub_rn(__dmul_rn(x, m.cs[v]), __dmul_rn(y, m.sn[v]));
            const double rmin = __dsub_rn(r, g.delta_xy), rmax = __dadd_rn(r, g.delta_xy);
            int n = 0;
            if (!(rmax < g.R0 || rmin > g.RMax)) {
                int imin = (int)floor(__ddiv_rn(__dsub_rn(rmin, g.R0), g.delta_r));
                int imax = (int)floor(__ddiv_rn(__dsub_rn(rmax, g.R0), g.delta_r));
                if (imax >= g.N_r) imax = g.N_r - 1;
                if (imin < 0) imin = 0;
                const float *H = g.H_r + (size_t)m.vidx[v] * (MBIR_RESP_BINS + 1);
                for (int j = imin; j <= imax; j++) {
                    const double rc = __dadd_rn(g.R0, __dmul_rn((double)j + 0.5, g.delta_r));
                    const double dr = fabs(__dsub_rn(r, rc));
                    const int id = (int)floor(__ddiv_rn(dr, g.OffsetR));
                    if (id >= 0 && id < MBIR_RESP_BINS) {
                        const double w1 = __dsub_rn(dr, __dmul_rn((double)id, g.OffsetR));
                        const double w2 = __dsub_rn(g.OffsetR, w1);
                        const double f1 = __ddiv_rn(__dadd_rn(__dmul_rn(w2, (double)__ldg(H + id)),
                                                              __dmul_rn(w1, (double)__ldg(H + id + 1))),
                                                    g.OffsetR);
                        const int off = j - m.rlo[v];
                        if (f1 > 0) {
                            if (off < 0 || off >= W || n >= amax) {
                                atomicOr(err, 1);
                            } else {
                                av[(size_t)n * NpS + v] = (float)f1;
                                ao[(size_t)n * NpS + v] = (uint8_t)off;
                                n++;
                            }
                        }
                    }
                }
            }
            ac[v] = (uint8_t)n;
        }
    };

    __syncthreads();
    if (nl > 0) acol(0, 0);
    __syncthreads();

    const float alpha = (float)pr.alpha, hT = (float)pr.hT, hTd = (float)(pr.hT * pr.hdelta);
    const float sSQ = (float)pr.sSQ, sSQP_inv = (float)(1.0 / pr.sSQP), cS = (float)pr.c_s;
    const float sTQ = (float)pr.sTQ, sTQP_inv = (float)(1.0 / pr.sTQP), cT = (float)pr.c_t;
    // neighbour of lane: spatial (dz, dy, dx) for lanes 0..25, temporal 26, 27
    int ndz = 0, ndy = 0, ndx = 0;
    float bw = 0.0f;
    bool spatial = false, temporal = false;
    if (lane < 26) {
        const int n = lane < 13 ? lane : lane + 1;  // skip the centre (13)
        ndz = n / 9 - 1;
        ndy = (n / 3) % 3 - 1;
        ndx = n % 3 - 1;
        bw = (float)pr.SF[n];
        spatial = true;
    } else if (lane < 28) {
        bw = (float)pr.TF;
        temporal = true;
    }
    const int zl = warp;  // this warp's slice in the group
    const bool active_warp = zl < nz;
    const int zg = z0 + zl;
    float sum_abs_dx = 0.0f, sum_abs_x = 0.0f;
    int n_upd = 0, n_skip = 0;

    for (int step = 0; step <= nl; step++) {
        const int li = (zl & 1) ? step - 1 : step;
        if (active_warp && li >= 0 && li < nl) {
            const int slot = li % 3;
            const int loc = m.order[li];
            const int lx = loc % S, ly = loc / S;
            const int col = k0 + lx, row = j0 + ly;
            float *xc = m.xb + ((size_t)(zl + 1) * S2 + ly + 1) * S2 + lx + 1;
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
                if (valid) nbv = m.tb[(((size_t)(lane - 26) * nz + zl) * S + ly) * S + lx];
            }
            const unsigned pos = __ballot_sync(0xffffffffu, valid && nbv > 0.0f);
            if (V == 0.0f && iter > 1 && pos == 0u) {
                n_skip++;
            } else {
                float b = 0.0f;
                if (valid) {
                    // f * rho'(D)/D for q = 2, p = 1.2: (2 - 0.8 t1/t3) / (t3 s^q)
                    const float d = V - nbv;
                    const float ad = fabsf(d);
                    const float t1 = (ad > 0.0f ? exp2f(0.8f * log2f(ad)) : 0.0f) * (spatial ? sSQP_inv : sTQP_inv);
                    const float t3 = (spatial ? cS : cT) + t1;
                    b = bw * (2.0f - 0.8f * t1 / t3) / (t3 * (spatial ? sSQ : sTQ));
                }
                float p1 = warp_allsum(b * nbv);
                float p2 = warp_allsum(b);
                // ---- data term over this slice's band rows ----
                float th1 = 0.0f, th2 = 0.0f;
                const float *av = m.aval + (size_t)slot * amax * NpS;
                const uint8_t *ao = m.aoff + (size_t)slot * amax * NpS;
                const uint8_t *ac = m.acnt + (size_t)slot * NpS;
                for (int v = lane; v < Np; v += 32) {
                    const int cnt = ac[v];
                    for (int q = 0; q < cnt; q++) {
                        const float a = av[(size_t)q * NpS + v];
                        const int off = ao[(size_t)q * NpS + v];
                        for (int rr = 0; rr < mz; rr++) {
                            const size_t so = ((size_t)(zl * mz + rr) * W + off) * NpS + v;
                            const float e = m.eb[so], w = m.wb[so];
                            const float sw = sqrtf(w);
                            float om = w;
                            if (!(fabsf(e * sw) < hT)) om = hTd * sw / fabsf(e);
                            th2 = fmaf(a * a, om, th2);
                            th1 = fmaf(-e * a, om, th1);
                        }
                    }
                }
                th1 = warp_allsum(th1);
                th2 = warp_allsum(th2);
                const float u = (p1 + th2 * V - th1) / (p2 + th2);
                const float xn = V + alpha * (u - V);
                const float dx = xn - V;
                __syncwarp();
                if (lane == 0) {
                    *xc = xn;
                    atomicAdd(&m.magl[loc], fabsf(dx));
                }
                sum_abs_dx += fabsf(dx);
                sum_abs_x += fabsf(xn);
                n_upd++;
                // ---- error sinogram: e -= a dx over this slice's rows ----
                for (int v = lane; v < Np; v += 32) {
                    const int cnt = ac[v];
                    for (int q = 0; q < cnt; q++) {
                        const float a = av[(size_t)q * NpS + v];
                        const int off = ao[(size_t)q * NpS + v];
                        for (int rr = 0; rr < mz; rr++) {
                            const size_t so = ((size_t)(zl * mz + rr) * W + off) * NpS + v;
                            m.eb[so] = fmaf(-a, dx, m.eb[so]);
                        }
                    }
                }
            }
        }
        if (step + 1 < nl) acol(step + 1, (step + 1) % 3);
        __syncthreads();
    }

    // ---- write back voxels, magnitude map, band change ----
    float *xo = dv.x + (size_t)i * g.N_z * plane;
    for (int q = tid; q < nz * S * S; q += nthr) {
        const int lx = q % S, ly = (q / S) % S, lz = q / (S * S);
        if (lx < kx && ly < ky)
            xo[(size_t)(z0 + lz) * plane + (size_t)(j0 + ly) * g.N_x + k0 + lx] =
                m.xb[((size_t)(lz + 1) * S2 + ly + 1) * S2 + lx + 1];
    }
    for (int q = tid; q < nl; q += nthr) {
        const int loc = m.order[q];
        task.mag[(size_t)(j0 + loc / S) * g.N_x + k0 + loc % S] = m.magl[loc];
    }
    for (size_t q = tid; q < bandn; q += nthr) {
        const int v = (int)(q % Np);
        const int off = (int)((q / Np) % W);
        const int row = (int)(q / ((size_t)Np * W));
        const int r = m.rlo[v] + off;
        if (r >= g.N_r) continue;
        const float dnew = m.eb[((size_t)row * W + off) * NpS + v] - scr[q];
        if (dnew != 0.0f) {
            const int t = z0 * mz + row;
            atomicAdd(&dv.e[((size_t)t * g.N_p + m.vidx[v]) * g.N_r + r], dnew);
        }
    }
    // ---- per-task statistics ----
    float a0 = warp_allsum(sum_abs_dx), a1 = warp_allsum(sum_abs_x);
    float a2 = warp_allsum((float)n_upd), a3 = warp_allsum((float)n_skip);
    if (lane == 0) {
        s_red[warp][0] = a0;
        s_red[warp][1] = a1;
        s_red[warp][2] = a2;
        s_red[warp][3] = a3;
    }
    __syncthreads();
    if (tid == 0) {
        double d0 = 0, d1 = 0, d2 = 0, d3 = 0;
        for (int w = 0; w < (nthr >> 5); w++) {
            d0 += s_red[w][0];
            d1 += s_red[w][1];
            d2 += s_red[w][2];
            d3 += s_red[w][3];
        }
        out[blockIdx.x].sum_abs_dx = d0;
        out[blockIdx.x].sum_abs_x = d1;
        out[blockIdx.x].updates = (long long)d2;
        out[blockIdx.x].zero_skips = (long long)d3;
    }
}

}  // namespace

size_t mbir_sv_smem_bytes(const SvParams &sp)
{
    const size_t NpS = sp.max_views, S = sp.S, S2 = sp.S + 2;
    size_t b = 0;
    b += 2 * sizeof(double) * NpS;
    b += 2 * sizeof(float) * (size_t)sp.max_rows * sp.W * NpS;
    b += sizeof(float) * 3 * sp.amax * NpS;
    b += sizeof(float) * (sp.max_nz + 2) * S2 * S2;
    b += sizeof(float) * 2 * sp.max_nz * S * S;
    b += sizeof(float) * S * S;
    b += sizeof(int) * NpS * 2;
    b += sizeof(int) * S * S;
    b += 3 * sp.amax * NpS + 3 * NpS;
    return (b + 15) & ~(size_t)15;
}

cudaError_t mbir_launch_icd_sv(const MbirGeom &g, const MbirPrior &pr, const MbirDev &dv, const SvParams &sp,
                               const SvTask *tasks, int ntasks, float *scratch, SvTaskOut *out, int iter,
                               uint32_t seed, int *err, cudaStream_t s)
{
    if (ntasks <= 0) return cudaSuccess;
    const size_t sm = mbir_sv_smem_bytes(sp);
    cudaError_t e = cudaFuncSetAttribute(k_icd_sv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    k_icd_sv<<<ntasks, 32 * sp.max_nz, sm, s>>>(g, pr, dv, sp, tasks, scratch, out, iter, seed, err);
    return cudaGetLastError();
}
