// Learned warm start: a 3-D encoder-decoder convolutional network that maps a
// frame's filtered backprojection to a start image for ICD, with its forward,
// backward and Adam kernels.  No counterpart in the reference (which starts
// its coarsest stage from zero); ICD still runs to its own convergence from
// the network's output, so the answer is the MAP estimate either way.
//
// Network (channels-last FP32 activations [B][D][H][W][C], BF16 weights and
// operands on the tensor cores, FP32 accumulation):
//   level 0 (D x H x W):        conv 16->16, conv 16->16          -> e0
//   level 1 (/2, average pool): conv 16->32, conv 32->32          -> e1
//   level 2 (/4):               conv 32->64, conv 64->64          -> e2
//   level 3 (/8):               conv 64->128, conv 128->128       -> e3
//   up to level 2 (nearest):    conv 128->64 + e2, conv 64->64    -> d2
//   up to level 1:              conv 64->32 + e1, conv 32->32     -> d1
//   up to level 0:              conv 32->16 + e0, conv 16->16     -> d0
//   output: conv 16->16 (channel 0 used): residual r
// Every convolution is 3 x 3 x 3, stride 1, zero padding 1, with a bias, and
// all but the last are followed by ReLU (after the skip addition).  The input
// is s * fbp in channel 0 of 16 (the others zero), the prediction
// s * fbp + r, the loss the mean over voxels of (prediction - s * target)^2;
// s scales attenuation values to order one.
//
// Convolutions are implicit GEMMs on mma.sync m16n8k16 (BF16 in, FP32
// accumulate): forward M = voxels, N = output channels, K = 27 taps x input
// channels, the input block staged in shared memory per 16-channel chunk;
// the input gradient is the same kernel with the flipped, transposed
// weights; the weight gradient is a GEMM over voxels (M = input channels,
// N = output channels, K = voxels) over staged blocks, reduced over CTAs
// with FP32 atomics.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/timbir_b200.h"

namespace {

constexpr int kLayers = 15;
constexpr int kCh[kLayers][2] = {{16, 16},  {16, 16},  {16, 32},  {32, 32}, {32, 64},
                                 {64, 64},  {64, 128}, {128, 128}, {128, 64}, {64, 64},
                                 {64, 32},  {32, 32},  {32, 16},  {16, 16}, {16, 16}};

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

struct Shape {
    int B, D, H, W;
    __host__ __device__ long long voxels() const { return (long long)B * D * H * W; }
};

// voxel m -> (b, z, y, x); false past the end (32-bit arithmetic: tensors
// hold fewer than 2^31 voxels, which net_shape checks)
__device__ __forceinline__ bool decode(const Shape &s, long long m, int &b, int &z, int &y, int &x)
{
    if (m >= s.voxels()) return false;
    unsigned r = (unsigned)m;
    x = (int)(r % (unsigned)s.W);
    r /= (unsigned)s.W;
    y = (int)(r % (unsigned)s.H);
    r /= (unsigned)s.H;
    z = (int)(r % (unsigned)s.D);
    b = (int)(r / (unsigned)s.D);
    return true;
}

// Voxel blocks of the weight gradient: 2 x 4 x 16 voxels, with a one-voxel halo.
constexpr int TZ = 2, TY = 4, TX = 16, HZ = TZ + 2, HY = TY + 2, HX = TX + 2, HV = HZ * HY * HX;

using bf16 = __nv_bfloat16;
__device__ __forceinline__ float b2f(bf16 v) { return __bfloat162float(v); }
__device__ __forceinline__ bf16 f2b(float v) { return __float2bfloat16_rn(v); }

// ---------------------------------------------------------------------------
// Convolution on the 5th-generation tensor cores (tcgen05, accumulators in
// tensor memory).  Implicit GEMM: M = 128 output voxels (8 along x by 16
// along y, one z-plane; ZT planes per CTA, one accumulator each), N = Cout,
// K = 27 taps x Cin, one tcgen05.mma of K = 16 per (tap, 16-channel input
// chunk, plane).
//
// Operands in shared memory, canonical K-major layouts without swizzle
// (8-row core matrices of 16 bytes per row; SBO = byte stride between 8-row
// groups along M or N, LBO = byte stride between the two 8-element halves
// of K = 16):
//   A: the CTA's input block with a one-voxel halo for one 16-channel chunk,
//      [half h][z][y][x][8 channels] BF16 (AZ x 18 x 10 voxels per half),
//      brought in by two TMA tensor copies per chunk (one per channel half;
//      the activations are BF16 channels-last, and a box {8 channels, 10 x,
//      18 y, AZ z, 1 batch} lands exactly in that layout, zeros outside the
//      volume): 8 consecutive x of one (z, y) row are one core matrix, the
//      next y row is SBO = 160 B on, the other channel half LBO = one
//      half-block on.  A tap (dz, dy, dx) is the same layout started
//      (dz, dy, dx) voxels away, so all 27 taps read the one block (no im2col);
//   B: the chunk's weights for all 27 taps, [tap][h][n][8] BF16, packed in
//      global memory in that order by k_pack_umma and brought in by one bulk
//      copy.
// One thread drives the pipeline: per chunk it waits until the MMAs that
// last used the stage's buffers are done, starts the chunk's three copies
// on the stage's mbarrier (byte count), waits for them and issues the
// chunk's MMAs, committed to the stage's MMA mbarrier; the copies of chunk
// k + 1 thus run while the tensor cores work on chunk k (NS = 2 stages; one
// for 128 output channels, whose weights fill most of shared memory).  The
// epilogue reads the accumulators with tcgen05.ld (warp w: rows
// 32w..32w+31), adds bias and skip input, applies ReLU or accumulates, and
// writes BF16 channels-last.  Every wait is bounded (1 s of global time);
// one that runs out sets *err, nothing more is issued, the copies and MMAs
// in flight are waited for (bounded again) and the tensor memory is freed.
constexpr int UX = 8, UY = 16, UZT = 2, UHX = UX + 2, UHY = UY + 2, UAZ = UZT + 2;
constexpr int kUmmaHalf = UAZ * UHY * UHX * 16;  // bytes of one channel half of the staged block

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t gtime()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// wait until the mbarrier's phase of parity `par` has completed; false after 1 s
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t par)
{
    const uint64_t t0 = gtime();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(smem_addr(bar)), "r"(par)
            : "memory");
        if (done) return true;
        if (gtime() - t0 > 1000000000ull) return false;
    }
}

__device__ __forceinline__ uint64_t umma_sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);  // version 1, no swizzle
}

// kind::f16 instruction descriptor: BF16 A and B (K-major), FP32 D, M = 128
__host__ __device__ constexpr uint32_t umma_idesc(int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

// tile copy of a 5-D box of tensor map tm at (c0..c4) into shared memory,
// completion counted in bytes on bar
__device__ __forceinline__ void tma_load_5d(void *dst, const CUtensorMap *tm, int c0, int c1, int c2, int c3, int c4,
                                            uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5, %6}], [%7];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_addr(bar))
        : "memory");
}

template <int N, int NS>
__global__ void __launch_bounds__(128) k_conv_umma(const __grid_constant__ CUtensorMap tmX, int Cin,
                                                   const bf16 *__restrict__ Wu, const float *__restrict__ bias,
                                                   const bf16 *__restrict__ add, int relu, int accumulate,
                                                   bf16 *__restrict__ Y, Shape s, int *__restrict__ err)
{
    constexpr int kBBytes = 27 * N * 32;  // one chunk's weights
    constexpr int kStage = 2 * kUmmaHalf + kBBytes;
    constexpr uint32_t kCols = UZT * N < 32 ? 32 : UZT * N;
    extern __shared__ __align__(128) uint8_t usm_raw[];
    // stages [NS][A halves | B], from a 128-byte aligned base (tensor copies)
    uint8_t *usm = usm_raw + ((128u - (smem_addr(usm_raw) & 127u)) & 127u);
    __shared__ __align__(8) uint64_t bar_full[NS], bar_mma[NS];
    __shared__ uint32_t s_tmem;
    __shared__ int s_ok;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ntx = (s.W + UX - 1) / UX, nty = (s.H + UY - 1) / UY, ntz = (s.D + UZT - 1) / UZT;
    int t = blockIdx.x;
    const int bx = t % ntx;
    t /= ntx;
    const int by = t % nty;
    t /= nty;
    const int bz = t % ntz;
    const int b = t / ntz;
    const int x0 = bx * UX, y0 = by * UY, z0 = bz * UZT;
    const int KC = Cin / 16;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&s_tmem)),
                     "r"(kCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int q = 0; q < NS; q++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar_full[q])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar_mma[q])));
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_ok = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;

    if (tid == 0) {
        constexpr uint32_t idesc = umma_idesc(N);
        bool ok = true;
        int committed = 0, started = 0;  // chunks whose MMAs were committed / copies started
        for (int kc = 0; kc < KC && ok; kc++) {
            const int st = kc % NS;
            const uint32_t use = (uint32_t)(kc / NS);  // earlier chunks on this stage
            // the stage's buffers are free once the MMAs of its last chunk are done
            if (use > 0 && !mbar_wait(&bar_mma[st], (use - 1) & 1)) {
                ok = false;
                break;
            }
            uint8_t *Ab = usm + (size_t)st * kStage, *Bb = Ab + 2 * kUmmaHalf;
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(&bar_full[st])),
                         "r"((uint32_t)kStage)
                         : "memory");
            tma_load_5d(Ab, &tmX, kc * 16, x0 - 1, y0 - 1, z0 - 1, b, &bar_full[st]);
            tma_load_5d(Ab + kUmmaHalf, &tmX, kc * 16 + 8, x0 - 1, y0 - 1, z0 - 1, b, &bar_full[st]);
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    smem_addr(Bb)),
                "l"(Wu + (size_t)kc * 27 * N * 16), "r"((uint32_t)kBBytes), "r"(smem_addr(&bar_full[st]))
                : "memory");
            started = kc + 1;
            if (!mbar_wait(&bar_full[st], use & 1)) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a0 = smem_addr(Ab), b0 = smem_addr(Bb);
            for (int tap = 0; tap < 27; tap++) {
                const int dz = tap / 9, dy = (tap / 3) % 3, dx = tap % 3;
                const uint64_t bd = umma_sdesc(b0 + (uint32_t)tap * N * 32, N * 16, 128);
#pragma unroll
                for (int m = 0; m < UZT; m++) {
                    const uint32_t aoff = (uint32_t)((((m + dz) * UHY + dy) * UHX + dx) * 16);
                    const uint64_t ad = umma_sdesc(a0 + aoff, kUmmaHalf, UHX * 16);
                    const uint32_t acc = (kc > 0 || tap > 0) ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem + m * N),
                        "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
                        : "memory");
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_addr(&bar_mma[st]))
                         : "memory");
            committed = kc + 1;
        }
        // the last committed MMAs (they complete in order); on a failure also
        // the copies of a chunk started but not multiplied, so that nothing
        // writes this CTA's shared memory after it exits
        if (committed > 0) {
            const int c = committed - 1;
            if (!mbar_wait(&bar_mma[c % NS], (uint32_t)(c / NS) & 1)) ok = false;
        }
        if (started > committed) {
            const int c = started - 1;
            mbar_wait(&bar_full[c % NS], (uint32_t)(c / NS) & 1);
        }
        s_ok = ok && committed == KC;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!s_ok) {
        if (tid == 0) atomicOr(err, 32);
    } else {
        // epilogue: thread = accumulator row 32 warp + lane = voxel (x0 + r % 8, y0 + r / 8)
        const int r = warp * 32 + lane;
        const int x = x0 + (r & 7), y = y0 + (r >> 3);
#pragma unroll 1
        for (int m = 0; m < UZT; m++) {
            const int z = z0 + m;
            const bool live = x < s.W && y < s.H && z < s.D;
            const size_t mo = live ? ((((size_t)b * s.D + z) * s.H + y) * s.W + x) : 0;
#pragma unroll 1
            for (int c0 = 0; c0 < N; c0 += 8) {
                uint32_t v[8];
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                      "=r"(v[7])
                    : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(m * N + c0)));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (!live) continue;
                float o[8];
#pragma unroll
                for (int j = 0; j < 8; j++) o[j] = __uint_as_float(v[j]) + (bias ? bias[c0 + j] : 0.0f);
                uint4 *yp = reinterpret_cast<uint4 *>(Y + mo * N + c0);  // 8 BF16 channels
                if (add) {
                    const uint4 a = *reinterpret_cast<const uint4 *>(add + mo * N + c0);
                    const bf16 *ab = reinterpret_cast<const bf16 *>(&a);
#pragma unroll
                    for (int j = 0; j < 8; j++) o[j] += b2f(ab[j]);
                }
                if (relu)
#pragma unroll
                    for (int j = 0; j < 8; j++) o[j] = fmaxf(o[j], 0.0f);
                if (accumulate) {
                    const uint4 pv = *yp;
                    const bf16 *pb = reinterpret_cast<const bf16 *>(&pv);
#pragma unroll
                    for (int j = 0; j < 8; j++) o[j] += b2f(pb[j]);
                }
                uint4 w;
                uint32_t *wv = reinterpret_cast<uint32_t *>(&w);
#pragma unroll
                for (int j = 0; j < 4; j++) wv[j] = pack_bf16(o[2 * j], o[2 * j + 1]);
                *yp = w;
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols));
}

// Weights of a layer in the tensor-core layout of k_conv_umma: per input
// chunk kc, tap, channel half h, output channel n, the 8 input channels
// kc 16 + 8 h + j (j = 0..7), BF16.  Forward: K = cin, N = cout, element
// W[tap][k][n]; input gradient: K = cout, N = cin, element W[26 - tap][n][k]
// (the flipped, transposed kernel).
// All layers in one launch: segment q packs layer layer[q] (flip[q]: the
// input-gradient weights) into out + dst[q]; a thread finds its segment by
// the segments' first element indices (at most 2 kLayers of them).
struct PackPlan {
    int nseg;
    long long first[2 * kLayers + 1];  // segment q: elements [first[q], first[q + 1])
    long long src[2 * kLayers], dst[2 * kLayers];
    int cin[2 * kLayers], cout[2 * kLayers], flip[2 * kLayers];
};

__global__ void k_pack_umma(const float *__restrict__ params, bf16 *__restrict__ out, const PackPlan plan)
{
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= plan.first[plan.nseg]) return;
    int q = 0;
    while (g >= plan.first[q + 1]) q++;
    const long long i = g - plan.first[q];
    const int cin = plan.cin[q], cout = plan.cout[q], flip = plan.flip[q];
    const int N = flip ? cin : cout;
    const float *W = params + plan.src[q];
    const int j = (int)(i % 8);
    long long r = i / 8;
    const int n = (int)(r % N);
    r /= N;
    const int h = (int)(r % 2);
    r /= 2;
    const int tap = (int)(r % 27);
    const int kc = (int)(r / 27);
    const int k = kc * 16 + h * 8 + j;
    const float v = flip ? W[((size_t)(26 - tap) * cin + n) * cout + k] : W[((size_t)tap * cin + k) * cout + n];
    out[plan.dst[q] + i] = f2b(v);
}

// Weight gradient, tiled: a CTA owns one 16-channel input chunk and NT
// output tiles and walks 2 x 4 x 16 voxel blocks; per block it stages the
// input with a one-voxel halo as [channel][voxel] BF16 (twice: aligned and
// shifted by one voxel, so that every tap's pair of consecutive voxels is one
// aligned 32-bit word) and the block's output gradient as [channel][voxel]
// BF16; warp w accumulates taps w, w + 9, w + 18 over the blocks (K = voxels,
// 16 per step), then adds its sums to dW with FP32 atomics.
constexpr int kWgWarps = 9;

template <int NT>
__global__ void __launch_bounds__(32 * kWgWarps) k_wgrad3t(const bf16 *__restrict__ X, int Cin,
                                                          const bf16 *__restrict__ dY, int Cout,
                                                          float *__restrict__ dW, float *__restrict__ part, Shape s)
{
    __shared__ __align__(16) __nv_bfloat16 xs[2][16][HV];
    __shared__ __align__(16) __nv_bfloat16 ys[NT * 8][TZ * TY * TX];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, tq = lane & 3;
    const int ci0 = blockIdx.y * 16, co0 = blockIdx.z * NT * 8;
    const int ntx = (s.W + TX - 1) / TX, nty = (s.H + TY - 1) / TY, ntz = (s.D + TZ - 1) / TZ;
    const int nblocks = s.B * ntz * nty * ntx;
    float acc[3][NT][4];
#pragma unroll
    for (int u = 0; u < 3; u++)
#pragma unroll
        for (int j = 0; j < NT; j++) acc[u][j][0] = acc[u][j][1] = acc[u][j][2] = acc[u][j][3] = 0.0f;
    for (int blk = blockIdx.x; blk < nblocks; blk += gridDim.x) {
        int t = blk;
        const int bx = t % ntx;
        t /= ntx;
        const int by = t % nty;
        t /= nty;
        const int bz = t % ntz;
        const int b = t / ntz;
        const int x0 = bx * TX, y0 = by * TY, z0 = bz * TZ;
        __syncthreads();  // the previous block's tiles are consumed
        for (int q = threadIdx.x; q < HV * 4; q += blockDim.x) {
            const int v = q >> 2, part = q & 3;
            const int lx = v % HX, ly = (v / HX) % HY, lz = v / (HX * HY);
            const int x = x0 + lx - 1, y = y0 + ly - 1, z = z0 + lz - 1;
            uint2 f = make_uint2(0u, 0u);  // four BF16 channels
            if (x >= 0 && x < s.W && y >= 0 && y < s.H && z >= 0 && z < s.D)
                f = __ldg(reinterpret_cast<const uint2 *>(
                    X + ((((size_t)b * s.D + z) * s.H + y) * s.W + x) * Cin + ci0 + part * 4));
            const bf16 *fv = reinterpret_cast<const bf16 *>(&f);
#pragma unroll
            for (int c = 0; c < 4; c++) {
                xs[0][part * 4 + c][v] = fv[c];
                if (v > 0) xs[1][part * 4 + c][v - 1] = fv[c];
            }
            if (v == HV - 1)
#pragma unroll
                for (int c = 0; c < 4; c++) xs[1][part * 4 + c][HV - 1] = __float2bfloat16_rn(0.0f);
        }
        for (int q = threadIdx.x; q < TZ * TY * TX * NT * 2; q += blockDim.x) {
            const int i = q / (NT * 2), part = q % (NT * 2);  // block voxel, 4 output channels
            const int lx = i % TX, ly = (i / TX) % TY, lz = i / (TX * TY);
            const int x = x0 + lx, y = y0 + ly, z = z0 + lz;
            uint2 f = make_uint2(0u, 0u);
            if (x < s.W && y < s.H && z < s.D)
                f = __ldg(reinterpret_cast<const uint2 *>(
                    dY + ((((size_t)b * s.D + z) * s.H + y) * s.W + x) * Cout + co0 + part * 4));
            const bf16 *fv = reinterpret_cast<const bf16 *>(&f);
            ys[part * 4 + 0][i] = fv[0];
            ys[part * 4 + 1][i] = fv[1];
            ys[part * 4 + 2][i] = fv[2];
            ys[part * 4 + 3][i] = fv[3];
        }
        __syncthreads();
        const uint32_t *yw = reinterpret_cast<const uint32_t *>(&ys[0][0]);
#pragma unroll 1
        for (int r = 0; r < TZ * TY; r++) {  // k-step: the 16 voxels of block row r
            const int oz = r / TY, oy = r % TY;
            uint32_t b0[NT], b1[NT];
#pragma unroll
            for (int j = 0; j < NT; j++) {
                const int w0 = ((j * 8 + g) * (TZ * TY * TX) + r * TX + 2 * tq) >> 1;
                b0[j] = yw[w0];
                b1[j] = yw[w0 + 4];
            }
#pragma unroll
            for (int u = 0; u < 3; u++) {
                const int tap = warp + kWgWarps * u;
                const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
                const int v0 = ((oz + 1 + dz) * HY + (oy + 1 + dy)) * HX + 1 + dx;
                const int par = v0 & 1;
                const uint32_t *xw = reinterpret_cast<const uint32_t *>(&xs[par][0][0]);
                const int wa = (g * HV + v0 - par + 2 * tq) >> 1, wb = ((g + 8) * HV + v0 - par + 2 * tq) >> 1;
                const uint32_t a0 = xw[wa], a1 = xw[wb], a2 = xw[wa + 4], a3 = xw[wb + 4];
#pragma unroll
                for (int j = 0; j < NT; j++) mma_bf16(acc[u][j], a0, a1, a2, a3, b0[j], b1[j]);
            }
        }
    }
    // this CTA's sums: into its own slice of `part` (summed over the CTAs
    // by k_wgrad_reduce), or added to dW with atomics when part is null
    float *dst = part ? part + (size_t)blockIdx.x * 27 * Cin * Cout : dW;
#pragma unroll
    for (int u = 0; u < 3; u++) {
        const int tap = warp + kWgWarps * u;
#pragma unroll
        for (int j = 0; j < NT; j++) {
            const int co = co0 + j * 8 + 2 * tq;
            float *w0 = dst + ((size_t)tap * Cin + ci0 + g) * Cout + co;
            float *w1 = w0 + (size_t)8 * Cout;
            if (part) {
                *reinterpret_cast<float2 *>(w0) = make_float2(acc[u][j][0], acc[u][j][1]);
                *reinterpret_cast<float2 *>(w1) = make_float2(acc[u][j][2], acc[u][j][3]);
            } else {
                atomicAdd(w0, acc[u][j][0]);
                atomicAdd(w0 + 1, acc[u][j][1]);
                atomicAdd(w1, acc[u][j][2]);
                atomicAdd(w1 + 1, acc[u][j][3]);
            }
        }
    }
}

// dW[i] += sum over the nx CTA slices of part (each n values), in slice order
__global__ void k_wgrad_reduce(const float *__restrict__ part, int nx, int n, float *__restrict__ dW)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float a0 = 0.0f, a1 = 0.0f;
    int x = 0;
    for (; x + 1 < nx; x += 2) {
        a0 += part[(size_t)x * n + i];
        a1 += part[(size_t)(x + 1) * n + i];
    }
    if (x < nx) a0 += part[(size_t)x * n + i];
    dW[i] += a0 + a1;
}

// db[c] += sum over voxels of dY[m][c]
// (blockDim 256, C <= 256 and dividing 256: the block's lanes of a channel
// are summed in shared memory first, one atomic per channel per block)
__global__ void __launch_bounds__(256) k_bias_grad(const bf16 *__restrict__ dY, int C, long long M, long long chunk,
                                                   float *__restrict__ db)
{
    __shared__ float red[256];
    const int c = threadIdx.x % C;
    const int lanes = blockDim.x / C;
    const int l = threadIdx.x / C;
    const long long start = (long long)blockIdx.x * chunk, end = min(M, start + chunk);
    // four independent sums in flight per thread
    float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f, a3 = 0.0f;
    long long m = start + l;
    for (; m + 3 * lanes < end; m += 4 * lanes) {
        a0 += b2f(dY[(size_t)m * C + c]);
        a1 += b2f(dY[(size_t)(m + lanes) * C + c]);
        a2 += b2f(dY[(size_t)(m + 2 * lanes) * C + c]);
        a3 += b2f(dY[(size_t)(m + 3 * lanes) * C + c]);
    }
    for (; m < end; m += lanes) a0 += b2f(dY[(size_t)m * C + c]);
    float acc = (a0 + a1) + (a2 + a3);
    red[threadIdx.x] = acc;
    __syncthreads();
    if (l == 0) {
        for (int q = 1; q < lanes; q++) acc += red[q * C + c];
        atomicAdd(db + c, acc);
    }
}

// Elementwise kernels over groups of 8 BF16 channels (16 bytes; every
// tensor has a multiple of 16 channels): thread q handles channels
// 8 (q mod C/8) .. + 7 of voxel q / (C/8).
struct V8 {
    float v[8];
};
__device__ __forceinline__ V8 ld8(const bf16 *p)
{
    const uint4 u = *reinterpret_cast<const uint4 *>(p);
    const bf16 *b = reinterpret_cast<const bf16 *>(&u);
    V8 r;
#pragma unroll
    for (int j = 0; j < 8; j++) r.v[j] = b2f(b[j]);
    return r;
}
__device__ __forceinline__ void st8(bf16 *p, const V8 &r)
{
    uint4 u;
    uint32_t *w = reinterpret_cast<uint32_t *>(&u);
#pragma unroll
    for (int j = 0; j < 4; j++) w[j] = pack_bf16(r.v[2 * j], r.v[2 * j + 1]);
    *reinterpret_cast<uint4 *>(p) = u;
}

// dA *= (A > 0): the ReLU's gradient mask (n: elements, a multiple of 8)
__global__ void k_relu_mask(bf16 *__restrict__ dA, const bf16 *__restrict__ A, long long n)
{
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q * 8 >= n) return;
    const V8 a = ld8(A + q * 8);
    V8 d = ld8(dA + q * 8);
#pragma unroll
    for (int j = 0; j < 8; j++)
        if (!(a.v[j] > 0.0f)) d.v[j] = 0.0f;
    st8(dA + q * 8, d);
}

// 2 x 2 x 2 average pooling; forward fine -> coarse, backward coarse -> fine
// (accumulate adds to the fine gradient); FP32 sums of BF16 values
__global__ void k_pool(const bf16 *__restrict__ X, bf16 *__restrict__ Y, Shape c, int C)
{
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int G = C / 8;
    if (q >= c.voxels() * G) return;
    const int ch = (int)(q % G) * 8;
    int b, z, y, x;
    decode(c, q / G, b, z, y, x);
    const Shape f{c.B, 2 * c.D, 2 * c.H, 2 * c.W};
    V8 s{};
    for (int k = 0; k < 8; k++) {
        const int zz = 2 * z + (k >> 2), yy = 2 * y + ((k >> 1) & 1), xx = 2 * x + (k & 1);
        const V8 a = ld8(X + ((((size_t)b * f.D + zz) * f.H + yy) * f.W + xx) * C + ch);
#pragma unroll
        for (int j = 0; j < 8; j++) s.v[j] += a.v[j];
    }
#pragma unroll
    for (int j = 0; j < 8; j++) s.v[j] *= 0.125f;
    st8(Y + q * 8, s);
}

__global__ void k_pool_bwd(const bf16 *__restrict__ dY, bf16 *__restrict__ dX, Shape f, int C, int accumulate)
{
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int G = C / 8;
    if (q >= f.voxels() * G) return;
    const int ch = (int)(q % G) * 8;
    int b, z, y, x;
    decode(f, q / G, b, z, y, x);
    const Shape c{f.B, f.D / 2, f.H / 2, f.W / 2};
    V8 v = ld8(dY + ((((size_t)b * c.D + z / 2) * c.H + y / 2) * c.W + x / 2) * C + ch);
    const V8 o = accumulate ? ld8(dX + q * 8) : V8{};
#pragma unroll
    for (int j = 0; j < 8; j++) v.v[j] = 0.125f * v.v[j] + o.v[j];
    st8(dX + q * 8, v);
}

// nearest-neighbour x2 up-sampling; backward sums the 8 fine gradients
__global__ void k_up(const bf16 *__restrict__ X, bf16 *__restrict__ Y, Shape f, int C)
{
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int G = C / 8;
    if (q >= f.voxels() * G) return;
    const int ch = (int)(q % G) * 8;
    int b, z, y, x;
    decode(f, q / G, b, z, y, x);
    const Shape c{f.B, f.D / 2, f.H / 2, f.W / 2};
    *reinterpret_cast<uint4 *>(Y + q * 8) =
        *reinterpret_cast<const uint4 *>(X + ((((size_t)b * c.D + z / 2) * c.H + y / 2) * c.W + x / 2) * C + ch);
}

__global__ void k_up_bwd(const bf16 *__restrict__ dY, bf16 *__restrict__ dX, Shape c, int C)
{
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int G = C / 8;
    if (q >= c.voxels() * G) return;
    const int ch = (int)(q % G) * 8;
    int b, z, y, x;
    decode(c, q / G, b, z, y, x);
    const Shape f{c.B, 2 * c.D, 2 * c.H, 2 * c.W};
    V8 s{};
    for (int k = 0; k < 8; k++) {
        const int zz = 2 * z + (k >> 2), yy = 2 * y + ((k >> 1) & 1), xx = 2 * x + (k & 1);
        const V8 a = ld8(dY + ((((size_t)b * f.D + zz) * f.H + yy) * f.W + xx) * C + ch);
#pragma unroll
        for (int j = 0; j < 8; j++) s.v[j] += a.v[j];
    }
    st8(dX + q * 8, s);
}

// network input: channel 0 = s * in, channels 1..15 = 0
__global__ void k_input(const float *__restrict__ in, float s, bf16 *__restrict__ X0, long long M)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M * 16) return;
    X0[i] = f2b((i % 16) == 0 ? s * in[i / 16] : 0.0f);
}

// out = in + r / s (r = channel 0 of the last layer)
__global__ void k_output(const float *__restrict__ in, const bf16 *__restrict__ Z, float s, float *__restrict__ out,
                         long long M)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < M) out[i] = in[i] + b2f(Z[(size_t)i * 16]) / s;
}

// loss = mean wt (s in + r - s t)^2 (wt = 1 without weights); dZ channel 0
// = its gradient, others 0; per-block partial sums (FP64) into part
__global__ void __launch_bounds__(256) k_loss(const float *__restrict__ in, const float *__restrict__ t,
                                              const float *__restrict__ wt, const bf16 *__restrict__ Z, float s,
                                              bf16 *__restrict__ dZ, long long M, double *__restrict__ part)
{
    __shared__ double red[256];
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double l = 0.0;
    if (i < M) {
        const float d = s * in[i] + b2f(Z[(size_t)i * 16]) - s * t[i];
        const float wi = wt ? wt[i] : 1.0f;
        l = (double)wi * d * d;
        bf16 *g = dZ + (size_t)i * 16;
        g[0] = f2b(2.0f * wi * d / (float)M);
        for (int c = 1; c < 16; c++) g[c] = f2b(0.0f);
    }
    red[threadIdx.x] = l;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// Adam (Kingma and Ba, 2015) on the FP32 master parameters
__global__ void k_adam(float *__restrict__ p, const float *__restrict__ gr, float *__restrict__ m,
                       float *__restrict__ v, long long n, float lr, float b1, float b2, float eps, float c1,
                       float c2)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = gr[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// He-normal initial weights (Box-Muller on a counter hash), zero biases
__device__ __forceinline__ uint32_t mix32(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

__global__ void k_init(float *__restrict__ W, long long n, float stdv, uint32_t seed)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t h1 = mix32(seed ^ mix32((uint32_t)i * 2u + 1u));
    const uint32_t h2 = mix32(seed ^ mix32((uint32_t)i * 2u + 2u) ^ 0x9e3779b9u);
    const float u1 = ((h1 >> 8) + 1.0f) * (1.0f / 16777217.0f);
    const float u2 = (h2 >> 8) * (1.0f / 16777216.0f);
    W[i] = stdv * sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
}

inline int blocks(long long n, int t = 256) { return (int)((n + t - 1) / t); }

}  // namespace

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
static thread_local char g_net_err[512];

static int net_fail(const char *msg, cudaError_t e = cudaSuccess)
{
    snprintf(g_net_err, sizeof g_net_err, "%s%s%s", msg, e != cudaSuccess ? ": " : "",
             e != cudaSuccess ? cudaGetErrorString(e) : "");
    return -1;
}

#define NK(call)                                                             \
    do {                                                                     \
        cudaError_t _e = (call);                                             \
        if (_e != cudaSuccess) return net_fail(#call, _e);                   \
    } while (0)

// A BF16 channels-last activation or gradient tensor and the tensor map the
// convolutions read it through (box {8 channels, 10 x, 18 y, 4 z, 1 batch})
struct NetTensor {
    bf16 *p = nullptr;
    size_t n = 0;
    int C = 0;
    CUtensorMap tm;
};

struct MbirNet {
    size_t w_off[kLayers], b_off[kLayers], nparams = 0;
    float *params = nullptr, *grads = nullptr, *m = nullptr, *v = nullptr;
    // the weights in the tensor-core layout of k_conv_umma (BF16), forward and
    // input-gradient (flipped, transposed) per layer
    bf16 *upack = nullptr;
    size_t upack_off[kLayers], udpack_off[kLayers], nupack = 0;
    int *d_err = nullptr;  // wait time-outs of the tensor-core convolution (bit 32)
    float *wg_part = nullptr;  // per-CTA weight-gradient sums (kWgPartFloats)
    long long step = 0;
    Shape shape{0, 0, 0, 0};
    // activations: X0 (input), A[k] (layer outputs), P1..P3 (pooled), U0..U2 (up-sampled)
    std::vector<NetTensor> act, grad;
    double *part = nullptr;
    size_t npart = 0;
    // CUDA graph of one gradient evaluation (forward, loss, backward) for the
    // last (shape, input, target, scale), captured on the second call with
    // them and replayed while they repeat (one launch instead of ~130)
    cudaStream_t gstream = nullptr;
    cudaGraphExec_t gexec = nullptr;
    const float *g_in = nullptr, *g_t = nullptr, *g_w = nullptr;
    const float *loss_w = nullptr;  // per-voxel loss weights (device, the input's shape) or null
    // high-pass loss: widths of the Gaussian G in mean(wt ((I - G) d)^2)
    // (0, 0: the plain loss) and its three float work volumes
    float hp_sz = 0.0f, hp_sxy = 0.0f;
    float *hp_buf = nullptr;
    size_t hp_n = 0;
    float g_scale = 0.0f;
    Shape g_shape{0, 0, 0, 0};
    int g_seen = 0;
    ~MbirNet()
    {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (gstream) cudaStreamDestroy(gstream);
        for (void *q : {(void *)params, (void *)grads, (void *)m, (void *)v, (void *)part, (void *)upack,
                        (void *)d_err, (void *)wg_part, (void *)hp_buf})
            if (q) cudaFree(q);
        for (auto &t : act)
            if (t.p) cudaFree(t.p);
        for (auto &t : grad)
            if (t.p) cudaFree(t.p);
    }
};

// tensor slots
enum { T_X0 = 0, T_A0 = 1, /* A0..A14 = 1..15 */ T_P1 = 16, T_P2, T_P3, T_U2, T_U1, T_U0, T_COUNT };

static Shape level_shape(const Shape &s, int lv) { return Shape{s.B, s.D >> lv, s.H >> lv, s.W >> lv}; }

// level and channels of each tensor slot
static void slot_info(int t, int &lv, int &C)
{
    static const int layer_level[kLayers] = {0, 0, 1, 1, 2, 2, 3, 3, 2, 2, 1, 1, 0, 0, 0};
    if (t == T_X0) {
        lv = 0;
        C = 16;
    } else if (t >= T_A0 && t < T_A0 + kLayers) {
        lv = layer_level[t - T_A0];
        C = kCh[t - T_A0][1];
    } else if (t == T_P1 || t == T_P2 || t == T_P3) {
        lv = t - T_P1 + 1;
        C = kCh[2 * (t - T_P1) + 1][1];
    } else {  // U2, U1, U0: up-sampled to levels 2, 1, 0
        lv = 2 - (t - T_U2);
        C = kCh[7 + 2 * (t - T_U2)][1];
    }
}

// cuTensorMapEncodeTiled from the driver (no link against libcuda)
static PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// Tensor map of a BF16 channels-last tensor [B][D][H][W][C] for the
// convolution's input boxes {8 channels, UHX, UHY, UAZ, 1}; zeros outside.
static int make_tmap(CUtensorMap *m, const bf16 *p, const Shape &s, int C)
{
    PFN_cuTensorMapEncodeTiled_v12000 enc = tmap_encoder();
    if (!enc) return net_fail("cuTensorMapEncodeTiled is not available from the driver");
    const cuuint64_t dims[5] = {(cuuint64_t)C, (cuuint64_t)s.W, (cuuint64_t)s.H, (cuuint64_t)s.D, (cuuint64_t)s.B};
    const cuuint64_t e = sizeof(bf16);
    const cuuint64_t strides[4] = {C * e, (cuuint64_t)s.W * C * e, (cuuint64_t)s.H * s.W * C * e,
                                   (cuuint64_t)s.D * s.H * s.W * C * e};
    const cuuint32_t box[5] = {8, UHX, UHY, UAZ, 1};
    const cuuint32_t es[5] = {1, 1, 1, 1, 1};
    const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<bf16 *>(p), dims, strides, box, es,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        snprintf(g_net_err, sizeof g_net_err, "cuTensorMapEncodeTiled failed (%d) for a %d-channel tensor", (int)r, C);
        return -1;
    }
    return 0;
}

static int net_shape(MbirNet *N, const Shape &s, bool train)
{
    if (s.B == N->shape.B && s.D == N->shape.D && s.H == N->shape.H && s.W == N->shape.W &&
        (!train || !N->grad.empty()))
        return 0;
    if (s.D % 8 || s.H % 8 || s.W % 8 || s.B < 1)
        return net_fail("network input sides must be multiples of 8");
    if (s.voxels() >= (1LL << 31)) return net_fail("network input above 2^31 voxels");
    // the captured gradient evaluation refers to the buffers freed here
    if (N->gexec) cudaGraphExecDestroy(N->gexec);
    N->gexec = nullptr;
    N->g_seen = 0;
    N->g_in = N->g_t = nullptr;
    for (auto &t : N->act)
        if (t.p) cudaFree(t.p);
    for (auto &t : N->grad)
        if (t.p) cudaFree(t.p);
    N->act.assign(T_COUNT, {});
    N->grad.clear();
    if (train) N->grad.assign(T_COUNT, {});
    for (int t = 0; t < T_COUNT; t++) {
        int lv, C;
        slot_info(t, lv, C);
        const Shape ls = level_shape(s, lv);
        const size_t n = (size_t)ls.voxels() * C;
        for (int g = 0; g < (train ? 2 : 1); g++) {
            NetTensor &x = g ? N->grad[t] : N->act[t];
            NK(cudaMalloc(&x.p, n * sizeof(bf16)));
            x.n = n;
            x.C = C;
            if (make_tmap(&x.tm, x.p, ls, C)) return -1;
        }
    }
    const size_t np = (size_t)blocks(s.voxels());
    if (np > N->npart) {
        if (N->part) cudaFree(N->part);
        NK(cudaMalloc(&N->part, np * sizeof(double)));
        N->npart = np;
    }
    N->shape = s;
    return 0;
}

template <int N, int NS>
static cudaError_t conv_umma_launch(const NetTensor &X, const bf16 *Wu, const float *bias, const bf16 *add, int relu,
                                    int accumulate, bf16 *Y, const Shape &s, int *err, cudaStream_t st)
{
    // as the kernel carves it: min(chunks, NS) stages of (two A halves, B), a
    // 128-byte alignment margin
    const int kc = X.C / 16;
    const size_t stage = (size_t)2 * kUmmaHalf + (size_t)27 * N * 32;
    const size_t smem = (size_t)std::min(kc, NS) * stage + 128;
    static bool attr = false;
    if (!attr) {  // the largest size this instantiation launches with
        cudaError_t e = cudaFuncSetAttribute(k_conv_umma<N, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)(NS * stage + 128));
        if (e != cudaSuccess) return e;
        attr = true;
    }
    const long long tiles =
        (long long)s.B * ((s.D + UZT - 1) / UZT) * ((s.H + UY - 1) / UY) * ((s.W + UX - 1) / UX);
    k_conv_umma<N, NS><<<(unsigned)tiles, 128, smem, st>>>(X.tm, X.C, Wu, bias, add, relu, accumulate, Y, s, err);
    return cudaGetLastError();
}

// Y = conv(X) (+ bias, + add, ReLU), or Y += conv(X); X at shape s
static cudaError_t conv(const NetTensor &X, const bf16 *Wu, int cout, const float *bias, const bf16 *add, int relu,
                        int accumulate, bf16 *Y, const Shape &s, int *err, cudaStream_t st)
{
    switch (cout) {
    case 16: return conv_umma_launch<16, 2>(X, Wu, bias, add, relu, accumulate, Y, s, err, st);
    case 32: return conv_umma_launch<32, 2>(X, Wu, bias, add, relu, accumulate, Y, s, err, st);
    case 64: return conv_umma_launch<64, 2>(X, Wu, bias, add, relu, accumulate, Y, s, err, st);
    case 128: return conv_umma_launch<128, 1>(X, Wu, bias, add, relu, accumulate, Y, s, err, st);
    default: return cudaErrorInvalidValue;
    }
}

// Weight gradient: CTAs along x split the voxel blocks; each writes its sums
// to its own slice of `part` (kWgPartFloats floats: as many x-CTAs as fit,
// up to four per SM) and k_wgrad_reduce adds them to dW.
constexpr size_t kWgPartFloats = 4u << 20;

static cudaError_t wgrad(const bf16 *X, int cin, const bf16 *dY, int cout, float *dW, float *db, const Shape &s,
                         float *part, cudaStream_t st)
{
    const int NT = std::min(cout / 8, 4);
    const long long blocks_ = (long long)s.B * ((s.D + TZ - 1) / TZ) * ((s.H + TY - 1) / TY) * ((s.W + TX - 1) / TX);
    const long long n = 27LL * cin * cout;
    const long long nx = std::max(1LL, std::min({blocks_, (long long)(kWgPartFloats / n), 4LL * 148}));
    const dim3 grid((unsigned)nx, (unsigned)(cin / 16), (unsigned)(cout / 8 / NT));
    switch (NT) {
    case 1: k_wgrad3t<1><<<grid, 32 * kWgWarps, 0, st>>>(X, cin, dY, cout, dW, part, s); break;
    case 2: k_wgrad3t<2><<<grid, 32 * kWgWarps, 0, st>>>(X, cin, dY, cout, dW, part, s); break;
    default: k_wgrad3t<4><<<grid, 32 * kWgWarps, 0, st>>>(X, cin, dY, cout, dW, part, s); break;
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (part) {
        k_wgrad_reduce<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(part, (int)nx, (int)n, dW);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    const long long M = s.voxels();
    const long long bch = std::max(1LL, std::min(M / 256, 4096LL));
    const long long bchunk = (M + bch - 1) / bch;
    k_bias_grad<<<(unsigned)bch, 256, 0, st>>>(dY, cout, M, bchunk, db);
    return cudaGetLastError();
}

static int pack_all(MbirNet *N, cudaStream_t st)
{
    PackPlan plan{};
    long long first = 0;
    int q = 0;
    for (int k = 0; k < kLayers; k++)
        for (int flip = 0; flip < (k > 0 ? 2 : 1); flip++, q++) {
            plan.first[q] = first;
            plan.src[q] = (long long)N->w_off[k];
            plan.dst[q] = (long long)(flip ? N->udpack_off[k] : N->upack_off[k]);
            plan.cin[q] = kCh[k][0];
            plan.cout[q] = kCh[k][1];
            plan.flip[q] = flip;
            first += 27LL * kCh[k][0] * kCh[k][1];
        }
    plan.nseg = q;
    plan.first[q] = first;
    k_pack_umma<<<blocks(first), 256, 0, st>>>(N->params, N->upack, plan);
    NK(cudaGetLastError());
    return 0;
}

static int forward(MbirNet *N, const float *in, float scale, cudaStream_t st)
{
    const Shape s = N->shape;
    auto &A = N->act;
    const long long M = s.voxels();
    k_input<<<blocks(M * 16), 256, 0, st>>>(in, scale, A[T_X0].p, M);
    NK(cudaGetLastError());
    // layer k from input slot x (with skip input add, ReLU or not) into A[k]
    auto L = [&](int k, int x, const bf16 *add, int relu, const Shape &sh) {
        return conv(A[x], N->upack + N->upack_off[k], kCh[k][1], N->params + N->b_off[k], add, relu, 0,
                    A[T_A0 + k].p, sh, N->d_err, st);
    };
    const Shape s1 = level_shape(s, 1), s2 = level_shape(s, 2), s3 = level_shape(s, 3);
    NK(L(0, T_X0, nullptr, 1, s));
    NK(L(1, T_A0 + 0, nullptr, 1, s));
    k_pool<<<blocks(s1.voxels() * 2), 256, 0, st>>>(A[T_A0 + 1].p, A[T_P1].p, s1, 16);
    NK(L(2, T_P1, nullptr, 1, s1));
    NK(L(3, T_A0 + 2, nullptr, 1, s1));
    k_pool<<<blocks(s2.voxels() * 4), 256, 0, st>>>(A[T_A0 + 3].p, A[T_P2].p, s2, 32);
    NK(L(4, T_P2, nullptr, 1, s2));
    NK(L(5, T_A0 + 4, nullptr, 1, s2));
    k_pool<<<blocks(s3.voxels() * 8), 256, 0, st>>>(A[T_A0 + 5].p, A[T_P3].p, s3, 64);
    NK(L(6, T_P3, nullptr, 1, s3));
    NK(L(7, T_A0 + 6, nullptr, 1, s3));
    k_up<<<blocks(s2.voxels() * 16), 256, 0, st>>>(A[T_A0 + 7].p, A[T_U2].p, s2, 128);
    NK(L(8, T_U2, A[T_A0 + 5].p, 1, s2));
    NK(L(9, T_A0 + 8, nullptr, 1, s2));
    k_up<<<blocks(s1.voxels() * 8), 256, 0, st>>>(A[T_A0 + 9].p, A[T_U1].p, s1, 64);
    NK(L(10, T_U1, A[T_A0 + 3].p, 1, s1));
    NK(L(11, T_A0 + 10, nullptr, 1, s1));
    k_up<<<blocks(s.voxels() * 4), 256, 0, st>>>(A[T_A0 + 11].p, A[T_U0].p, s, 32);
    NK(L(12, T_U0, A[T_A0 + 1].p, 1, s));
    NK(L(13, T_A0 + 12, nullptr, 1, s));
    NK(L(14, T_A0 + 13, nullptr, 0, s));
    return 0;
}

// Gradients of the loss with respect to every parameter into N->grads
// (zeroed here); dZ of the last layer must already be in grad[A14].
static int backward(MbirNet *N, cudaStream_t st)
{
    const Shape s = N->shape, s1 = level_shape(s, 1), s2 = level_shape(s, 2), s3 = level_shape(s, 3);
    auto &A = N->act;
    auto &G = N->grad;
    NK(cudaMemsetAsync(N->grads, 0, N->nparams * sizeof(float), st));
    // layer k: weight and bias gradients from its input x and output
    // gradient dz; the input gradient (into dx, optionally accumulated)
    auto layer = [&](int k, const bf16 *x, const Shape &sh, bf16 *dx, int acc) -> int {
        const NetTensor &dz = G[T_A0 + k];
        NK(wgrad(x, kCh[k][0], dz.p, kCh[k][1], N->grads + N->w_off[k], N->grads + N->b_off[k], sh, N->wg_part,
                 st));
        if (dx)
            NK(conv(dz, N->upack + N->udpack_off[k], kCh[k][0], nullptr, nullptr, 0, acc, dx, sh, N->d_err, st));
        return 0;
    };
    auto mask = [&](int t) -> int {  // dA -> dZ of a ReLU output
        k_relu_mask<<<blocks((long long)A[t].n / 8), 256, 0, st>>>(G[t].p, A[t].p, (long long)A[t].n);
        NK(cudaGetLastError());
        return 0;
    };
    if (layer(14, A[T_A0 + 13].p, s, G[T_A0 + 13].p, 0) || mask(T_A0 + 13)) return -1;
    if (layer(13, A[T_A0 + 12].p, s, G[T_A0 + 12].p, 0) || mask(T_A0 + 12)) return -1;
    // layer 12: input U0, skip from A1 (its gradient seeds dA1)
    if (layer(12, A[T_U0].p, s, G[T_U0].p, 0)) return -1;
    NK(cudaMemcpyAsync(G[T_A0 + 1].p, G[T_A0 + 12].p, A[T_A0 + 1].n * sizeof(bf16), cudaMemcpyDeviceToDevice, st));
    k_up_bwd<<<blocks(s1.voxels() * 4), 256, 0, st>>>(G[T_U0].p, G[T_A0 + 11].p, s1, 32);
    NK(cudaGetLastError());
    if (mask(T_A0 + 11)) return -1;
    if (layer(11, A[T_A0 + 10].p, s1, G[T_A0 + 10].p, 0) || mask(T_A0 + 10)) return -1;
    if (layer(10, A[T_U1].p, s1, G[T_U1].p, 0)) return -1;
    NK(cudaMemcpyAsync(G[T_A0 + 3].p, G[T_A0 + 10].p, A[T_A0 + 3].n * sizeof(bf16), cudaMemcpyDeviceToDevice, st));
    k_up_bwd<<<blocks(s2.voxels() * 8), 256, 0, st>>>(G[T_U1].p, G[T_A0 + 9].p, s2, 64);
    NK(cudaGetLastError());
    if (mask(T_A0 + 9)) return -1;
    if (layer(9, A[T_A0 + 8].p, s2, G[T_A0 + 8].p, 0) || mask(T_A0 + 8)) return -1;
    if (layer(8, A[T_U2].p, s2, G[T_U2].p, 0)) return -1;
    NK(cudaMemcpyAsync(G[T_A0 + 5].p, G[T_A0 + 8].p, A[T_A0 + 5].n * sizeof(bf16), cudaMemcpyDeviceToDevice, st));
    k_up_bwd<<<blocks(s3.voxels() * 16), 256, 0, st>>>(G[T_U2].p, G[T_A0 + 7].p, s3, 128);
    NK(cudaGetLastError());
    if (mask(T_A0 + 7)) return -1;
    if (layer(7, A[T_A0 + 6].p, s3, G[T_A0 + 6].p, 0) || mask(T_A0 + 6)) return -1;
    if (layer(6, A[T_P3].p, s3, G[T_P3].p, 0)) return -1;
    k_pool_bwd<<<blocks(s2.voxels() * 8), 256, 0, st>>>(G[T_P3].p, G[T_A0 + 5].p, s2, 64, 1);
    NK(cudaGetLastError());
    if (mask(T_A0 + 5)) return -1;
    if (layer(5, A[T_A0 + 4].p, s2, G[T_A0 + 4].p, 0) || mask(T_A0 + 4)) return -1;
    if (layer(4, A[T_P2].p, s2, G[T_P2].p, 0)) return -1;
    k_pool_bwd<<<blocks(s1.voxels() * 4), 256, 0, st>>>(G[T_P2].p, G[T_A0 + 3].p, s1, 32, 1);
    NK(cudaGetLastError());
    if (mask(T_A0 + 3)) return -1;
    if (layer(3, A[T_A0 + 2].p, s1, G[T_A0 + 2].p, 0) || mask(T_A0 + 2)) return -1;
    if (layer(2, A[T_P1].p, s1, G[T_P1].p, 0)) return -1;
    k_pool_bwd<<<blocks(s.voxels() * 2), 256, 0, st>>>(G[T_P1].p, G[T_A0 + 1].p, s, 16, 1);
    NK(cudaGetLastError());
    if (mask(T_A0 + 1)) return -1;
    if (layer(1, A[T_A0 + 0].p, s, G[T_A0 + 0].p, 0) || mask(T_A0 + 0)) return -1;
    if (layer(0, A[T_X0].p, s, nullptr, 0)) return -1;
    return 0;
}

// time-outs recorded by the tensor-core convolutions since the last check
static int net_err_check(MbirNet *N, cudaStream_t st)
{
    int e = 0;
    NK(cudaMemcpyAsync(&e, N->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    NK(cudaStreamSynchronize(st));
    if (e) {
        cudaMemsetAsync(N->d_err, 0, sizeof(int), st);
        return net_fail("tensor-core convolution: a wait for its operands or MMAs timed out");
    }
    return 0;
}

// ---- high-pass loss: mean(wt ((I - G) d)^2), d = s in + r - s t ----
__global__ void k_loss_residual(const float *__restrict__ in, const float *__restrict__ t,
                                const bf16 *__restrict__ Z, float s, float *__restrict__ d, long long M)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < M) d[i] = s * in[i] + b2f(Z[(size_t)i * 16]) - s * t[i];
}

// h = d - G d; u = wt h (in place of d); per-block sums of wt h^2 into part
__global__ void __launch_bounds__(256) k_hp_loss(float *__restrict__ du, const float *__restrict__ gd,
                                                 const float *__restrict__ wt, long long M, double *__restrict__ part)
{
    __shared__ double red[256];
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double l = 0.0;
    if (i < M) {
        const float h = du[i] - gd[i];
        const float wi = wt ? wt[i] : 1.0f;
        du[i] = wi * h;
        l = (double)wi * h * h;
    }
    red[threadIdx.x] = l;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// dZ channel 0 = 2 (I - G) u / M (G symmetric: zero edges), others 0
__global__ void k_hp_grad(const float *__restrict__ u, const float *__restrict__ gu, bf16 *__restrict__ dZ,
                          long long M)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M) return;
    bf16 *g = dZ + (size_t)i * 16;
    g[0] = f2b(2.0f * (u[i] - gu[i]) / (float)M);
    for (int c = 1; c < 16; c++) g[c] = f2b(0.0f);
}

// ---- low-frequency blend of two starts ----
// Gaussian taps of one axis: radius int(4 sigma + 0.5), exp(-x^2 / (2 sigma^2))
// normalised to sum 1 (the truncation and normalisation of scipy.ndimage's
// gaussian_filter); edges mirrored about the half-sample point (d c b a | a b
// c d | d c b a).
constexpr int kBlurMaxRadius = 64;
struct BlurTaps {
    int r;
    float w[2 * kBlurMaxRadius + 1];
};

__global__ void k_blend_diff(const float *__restrict__ a, const float *__restrict__ b, float *__restrict__ d,
                             long long n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) d[i] = a[i] - b[i];
}

// out = in filtered along one axis (length len, element stride stride);
// mirrored edges, or zeros outside (zero_edge: the filter is then a symmetric
// matrix, its own transpose)
__global__ void k_blur_axis(const float *__restrict__ in, float *__restrict__ out, long long n, long long stride,
                            int len, BlurTaps t, int zero_edge)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = (int)((i / stride) % len);
    const float *base = in + (i - (long long)c * stride);
    float acc = 0.0f;
    for (int k = -t.r; k <= t.r; k++) {
        int q = c + k;
        if (zero_edge) {
            if (q < 0 || q >= len) continue;
        } else {
            while (q < 0 || q >= len) q = q < 0 ? -q - 1 : 2 * len - q - 1;
        }
        acc = fmaf(t.w[k + t.r], base[(long long)q * stride], acc);
    }
    out[i] = acc;
}

static BlurTaps blur_taps(float sigma)
{
    BlurTaps t{};
    t.r = (int)(4.0 * sigma + 0.5);
    double w[2 * kBlurMaxRadius + 1], sum = 0.0;
    for (int k = -t.r; k <= t.r; k++) sum += w[k + t.r] = std::exp(-0.5 * k * k / ((double)sigma * sigma));
    for (int k = 0; k <= 2 * t.r; k++) t.w[k] = (float)(w[k] / sum);
    return t;
}

// G x of a float volume [B][D][H][W] into one of the two work buffers
// (a, b; x may be either); returns the buffer holding the result
static float *blur3(const float *x, float *a, float *b, const Shape &s, float sz, float sxy, int zero_edge,
                    cudaStream_t st)
{
    const long long n = s.voxels();
    const unsigned nb = (unsigned)((n + 255) / 256);
    const struct {
        float sigma;
        long long stride;
        int len;
    } axes[3] = {{sxy, 1, s.W}, {sxy, s.W, s.H}, {sz, (long long)s.H * s.W, s.D}};
    const float *cur = x;
    float *dst = (x == a) ? b : a;
    for (const auto &ax : axes) {
        if (ax.sigma <= 0.0f) continue;
        k_blur_axis<<<nb, 256, 0, st>>>(cur, dst, n, ax.stride, ax.len, blur_taps(ax.sigma), zero_edge);
        cur = dst;
        dst = (dst == a) ? b : a;
    }
    return const_cast<float *>(cur);
}

__global__ void k_blend_add(float *__restrict__ start, const float *__restrict__ d, long long n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) start[i] += d[i];
}


extern "C" {

const char *mbir_net_last_error(void) { return g_net_err; }

int mbir_lowpass_blend(const float *ref, float *start, float *scratch, int32_t N, int32_t D, int32_t H, int32_t W,
                       float sigma_z, float sigma_xy, void *stream)
{
    if (N < 1 || D < 1 || H < 1 || W < 1) return net_fail("blend: empty volume");
    if (!(sigma_z >= 0.0f && sigma_xy >= 0.0f) || 4.0f * sigma_z + 0.5f > (float)kBlurMaxRadius ||
        4.0f * sigma_xy + 0.5f > (float)kBlurMaxRadius)
        return net_fail("blend: Gaussian widths must be in [0, 15.9]");
    cudaStream_t st = (cudaStream_t)stream;
    const long long n = (long long)N * D * H * W;
    const unsigned nb = (unsigned)((n + 255) / 256);
    float *a = scratch, *b = scratch + n;
    k_blend_diff<<<nb, 256, 0, st>>>(ref, start, a, n);
    NK(cudaGetLastError());
    // x (stride 1), y (stride W), z (stride H W); a zero width skips the axis
    const struct {
        float sigma;
        long long stride;
        int len;
    } axes[3] = {{sigma_xy, 1, W}, {sigma_xy, W, H}, {sigma_z, (long long)H * W, D}};
    for (const auto &ax : axes) {
        if (ax.sigma <= 0.0f) continue;
        k_blur_axis<<<nb, 256, 0, st>>>(a, b, n, ax.stride, ax.len, blur_taps(ax.sigma), 0);
        NK(cudaGetLastError());
        std::swap(a, b);
    }
    k_blend_add<<<nb, 256, 0, st>>>(start, a, n);
    NK(cudaGetLastError());
    NK(cudaStreamSynchronize(st));
    return 0;
}

int64_t mbir_net_param_count(void)
{
    int64_t n = 0;
    for (int k = 0; k < kLayers; k++) n += 27LL * kCh[k][0] * kCh[k][1] + kCh[k][1];
    return n;
}

int mbir_net_create(MbirNet **out, uint32_t seed)
{
    *out = nullptr;
    auto N = std::make_unique<MbirNet>();
    size_t off = 0;
    for (int k = 0; k < kLayers; k++) {
        const int ci = kCh[k][0], co = kCh[k][1];
        N->w_off[k] = off;
        off += 27 * (size_t)ci * co;
        N->b_off[k] = off;
        off += co;
        N->upack_off[k] = N->nupack;
        N->nupack += 27 * (size_t)ci * co;
        N->udpack_off[k] = N->nupack;
        if (k > 0) N->nupack += 27 * (size_t)ci * co;
    }
    N->nparams = off;
    NK(cudaMalloc(&N->params, off * sizeof(float)));
    NK(cudaMalloc(&N->grads, off * sizeof(float)));
    NK(cudaMalloc(&N->m, off * sizeof(float)));
    NK(cudaMalloc(&N->v, off * sizeof(float)));
    NK(cudaMalloc(&N->upack, N->nupack * sizeof(bf16)));
    NK(cudaMalloc(&N->d_err, sizeof(int)));
    NK(cudaMalloc(&N->wg_part, kWgPartFloats * sizeof(float)));
    NK(cudaMemset(N->d_err, 0, sizeof(int)));
    NK(cudaMemset(N->params, 0, off * sizeof(float)));
    NK(cudaMemset(N->grads, 0, off * sizeof(float)));
    NK(cudaMemset(N->m, 0, off * sizeof(float)));
    NK(cudaMemset(N->v, 0, off * sizeof(float)));
    for (int k = 0; k < kLayers; k++) {
        const long long n = 27LL * kCh[k][0] * kCh[k][1];
        // He initialisation for ReLU layers; the output layer starts small
        // so that the untrained network returns about its input
        const float stdv = k == kLayers - 1 ? 1e-3f : sqrtf(2.0f / (27.0f * kCh[k][0]));
        k_init<<<blocks(n), 256>>>(N->params + N->w_off[k], n, stdv, seed * 2654435761u + (uint32_t)k);
        NK(cudaGetLastError());
    }
    if (pack_all(N.get(), 0)) return -1;
    NK(cudaDeviceSynchronize());
    *out = N.release();
    return 0;
}

void mbir_net_free(MbirNet *net) { delete net; }

int mbir_net_get_params(MbirNet *N, float *out)
{
    NK(cudaMemcpy(out, N->params, N->nparams * sizeof(float), cudaMemcpyDeviceToHost));
    return 0;
}

int mbir_net_set_params(MbirNet *N, const float *in)
{
    NK(cudaMemcpy(N->params, in, N->nparams * sizeof(float), cudaMemcpyHostToDevice));
    if (pack_all(N, 0)) return -1;
    NK(cudaDeviceSynchronize());
    return 0;
}

int mbir_net_get_grads(MbirNet *N, float *out)
{
    NK(cudaMemcpy(out, N->grads, N->nparams * sizeof(float), cudaMemcpyDeviceToHost));
    return 0;
}

// Activation (which = 0) or its gradient (which = 1) of layer k (0..14;
// -1: the network input) from the last forward / gradient call, host
// float [B][D][H][W][C] at the layer's level; *count = its elements.
int mbir_net_get_activation(MbirNet *N, int32_t layer, int32_t which, float *out, int64_t *count)
{
    const int t = layer < 0 ? T_X0 : T_A0 + layer;
    if (layer < -1 || layer >= kLayers || N->act.empty()) return net_fail("no such activation");
    if (which == 1 && N->grad.empty()) return net_fail("no gradients computed");
    const NetTensor &x = which == 1 ? N->grad[t] : N->act[t];
    if (count) *count = (int64_t)x.n;
    if (out) {  // BF16 on the device; widened to float here
        std::vector<uint16_t> h(x.n);
        NK(cudaMemcpy(h.data(), x.p, x.n * sizeof(bf16), cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < x.n; i++) {
            const uint32_t u = (uint32_t)h[i] << 16;
            memcpy(out + i, &u, sizeof u);
        }
    }
    return 0;
}

int mbir_net_forward(MbirNet *N, const float *in, float *out, int32_t B, int32_t D, int32_t H, int32_t W,
                     float scale, void *stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (net_shape(N, Shape{B, D, H, W}, false) || forward(N, in, scale, st)) return -1;
    const long long M = N->shape.voxels();
    k_output<<<blocks(M), 256, 0, st>>>(in, N->act[T_A0 + 14].p, scale, out, M);
    NK(cudaGetLastError());
    NK(cudaStreamSynchronize(st));
    if (net_err_check(N, st)) return -1;
    return 0;
}

int mbir_net_gradients(MbirNet *N, const float *in, const float *target, int32_t B, int32_t D, int32_t H, int32_t W,
                       float scale, double *loss, void *stream)
{
    cudaStream_t caller = (cudaStream_t)stream;
    const Shape sh{B, D, H, W};
    if (net_shape(N, sh, true)) return -1;
    const bool same = N->g_in == in && N->g_t == target && N->g_w == N->loss_w && N->g_scale == scale &&
                      N->g_shape.B == B && N->g_shape.D == D && N->g_shape.H == H && N->g_shape.W == W;
    if (!same) {  // a new key: the graph of the old one is dropped
        if (N->gexec) cudaGraphExecDestroy(N->gexec);
        N->gexec = nullptr;
        N->g_in = in;
        N->g_t = target;
        N->g_w = N->loss_w;
        N->g_scale = scale;
        N->g_shape = sh;
        N->g_seen = 0;
    }
    const long long M = N->shape.voxels();
    const int nb = blocks(M);
    const bool hp = N->hp_sz > 0.0f || N->hp_sxy > 0.0f;
    if (hp && N->hp_n < 3 * (size_t)M) {  // work volumes of the high-pass loss
        if (N->gexec) cudaGraphExecDestroy(N->gexec);
        N->gexec = nullptr;
        N->g_seen = 0;
        if (N->hp_buf) cudaFree(N->hp_buf);
        N->hp_buf = nullptr;
        N->hp_n = 0;
        NK(cudaMalloc(&N->hp_buf, 3 * (size_t)M * sizeof(float)));
        N->hp_n = 3 * (size_t)M;
    }
    auto enqueue = [&](cudaStream_t st) -> int {
        if (forward(N, in, scale, st)) return -1;
        if (hp) {
            float *du = N->hp_buf, *a = du + M, *b = a + M;
            k_loss_residual<<<nb, 256, 0, st>>>(in, target, N->act[T_A0 + 14].p, scale, du, M);
            const float *gd = blur3(du, a, b, N->shape, N->hp_sz, N->hp_sxy, 1, st);
            k_hp_loss<<<nb, 256, 0, st>>>(du, gd, N->loss_w, M, N->part);
            const float *gu = blur3(du, a, b, N->shape, N->hp_sz, N->hp_sxy, 1, st);
            k_hp_grad<<<nb, 256, 0, st>>>(du, gu, N->grad[T_A0 + 14].p, M);
        } else {
            k_loss<<<nb, 256, 0, st>>>(in, target, N->loss_w, N->act[T_A0 + 14].p, scale, N->grad[T_A0 + 14].p, M,
                                       N->part);
        }
        NK(cudaGetLastError());
        return backward(N, st);
    };
    cudaStream_t st = caller;
    if (!N->gexec && N->g_seen >= 1) {
        // second call with this key: capture on a stream of our own (the
        // caller's may be the legacy default stream, which cannot capture)
        if (!N->gstream) NK(cudaStreamCreateWithFlags(&N->gstream, cudaStreamNonBlocking));
        NK(cudaStreamSynchronize(caller));
        NK(cudaStreamBeginCapture(N->gstream, cudaStreamCaptureModeThreadLocal));
        const int rc = enqueue(N->gstream);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(N->gstream, &g);
        if (rc || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return rc ? -1 : net_fail("capturing the gradient evaluation", e);
        }
        const cudaError_t ei = cudaGraphInstantiate(&N->gexec, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) {
            N->gexec = nullptr;
            return net_fail("instantiating the gradient evaluation's graph", ei);
        }
    }
    if (N->gexec) {
        NK(cudaStreamSynchronize(caller));  // the caller's work on the parameters (Adam, packing)
        NK(cudaGraphLaunch(N->gexec, N->gstream));
        st = N->gstream;
    } else {
        if (enqueue(caller)) return -1;
        N->g_seen++;
    }
    std::vector<double> part(nb);
    NK(cudaMemcpyAsync(part.data(), N->part, nb * sizeof(double), cudaMemcpyDeviceToHost, st));
    NK(cudaStreamSynchronize(st));
    if (net_err_check(N, st)) return -1;
    double l = 0;
    for (double v : part) l += v;
    if (loss) *loss = l / (double)M;
    return 0;
}

int mbir_net_set_loss_weights(MbirNet *N, const float *w)
{
    if (!N) return net_fail("null network");
    N->loss_w = w;
    return 0;
}

int mbir_net_set_loss_highpass(MbirNet *N, float sigma_z, float sigma_xy)
{
    if (!N) return net_fail("null network");
    if (!(sigma_z >= 0.0f && sigma_xy >= 0.0f) || 4.0f * sigma_z + 0.5f > (float)kBlurMaxRadius ||
        4.0f * sigma_xy + 0.5f > (float)kBlurMaxRadius)
        return net_fail("high-pass loss: Gaussian widths must be in [0, 15.9]");
    if (sigma_z != N->hp_sz || sigma_xy != N->hp_sxy) {  // another loss: the captured evaluation is dropped
        if (N->gexec) cudaGraphExecDestroy(N->gexec);
        N->gexec = nullptr;
        N->g_seen = 0;
        N->g_in = nullptr;
    }
    N->hp_sz = sigma_z;
    N->hp_sxy = sigma_xy;
    return 0;
}

int mbir_net_adam_step(MbirNet *N, float lr, void *stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    const float b1 = 0.9f, b2 = 0.999f;
    N->step++;
    const float c1 = 1.0f - powf(b1, (float)N->step), c2 = 1.0f - powf(b2, (float)N->step);
    k_adam<<<blocks((long long)N->nparams), 256, 0, st>>>(N->params, N->grads, N->m, N->v, (long long)N->nparams, lr,
                                                          b1, b2, 1e-8f, c1, c2);
    NK(cudaGetLastError());
    if (pack_all(N, st)) return -1;
    return 0;
}

}  // extern "C"
