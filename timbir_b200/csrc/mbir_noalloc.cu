// Ring-offset update without device allocation.
//
// mbir_update_sinogram_offset_noalloc() runs the same kernels as the
// stage-level ring-offset update, on device arrays the caller owns, with its
// scratch (per-detector-element numerators and denominators and the partial
// sums of the zero-mean constraint) in a file-scope device array instead of
// memory from cudaMalloc.  It is meant for callers that cannot allocate
// device memory: a host application or acquisition framework that reserves
// all of the GPU's memory for its own pool at start-up (cudaMalloc would then
// fail) and forbids libraries to allocate behind its back, or a processing
// loop that must not take cudaMalloc's implicit device-wide synchronisation.
//
// The array's device address is looked up once per device (the first call
// with that device current) and cached for the life of the process; after
// cudaDeviceReset the cached address is stale, so a process that resets a
// device must not call this entry point on it again.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/timbir_b200.h"
#include "mbir_internal.h"

namespace {

constexpr int kParts = 592;  // partial sums, as the stage-level update uses

// Scratch shared by every call on a device: 2 doubles per detector element
// (numerator, denominator) plus 4 * kParts partial sums.  MBIR_NOALLOC_MAX_ELEMS
// detector elements (rows x columns) at most: 1 Mi elements, 16 MiB, held by
// every GPU that loads the library until the process exits.
constexpr size_t kScratchDoubles = 2 * (size_t)MBIR_NOALLOC_MAX_ELEMS + 4 * kParts;
__device__ __align__(256) double g_offset_scratch[kScratchDoubles];

// Device address of g_offset_scratch per device, looked up once per device
// with that device current (in host code the symbol is only a host-side
// stand-in; its address must come from the runtime).
constexpr int kMaxDevices = 64;
double *g_scratch_addr[kMaxDevices];
std::mutex g_scratch_mu;

thread_local char g_msg[256];

}  // namespace

extern "C" const char *mbir_noalloc_last_error(void) { return g_msg; }

extern "C" int mbir_update_sinogram_offset_noalloc(float *e, const float *w, float *d, int32_t N_p,
                                                   int32_t N_r, int32_t N_t, int32_t remove_rings,
                                                   int32_t quad_convex, float huber_delta, float huber_T,
                                                   void *stream)
{
    if (N_p <= 0 || N_r <= 0 || N_t <= 0) {
        snprintf(g_msg, sizeof(g_msg), "non-positive dimensions");
        return -1;
    }
    if ((size_t)N_r * N_t > (size_t)MBIR_NOALLOC_MAX_ELEMS) {
        snprintf(g_msg, sizeof(g_msg),
                 "detector of %d x %d elements exceeds the no-allocation limit of %d elements",
                 (int)N_t, (int)N_r, (int)MBIR_NOALLOC_MAX_ELEMS);
        return -1;
    }
    if (remove_rings < 1 || remove_rings > 3) {
        snprintf(g_msg, sizeof(g_msg), "remove_rings must be 1, 2 or 3");
        return -1;
    }
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        snprintf(g_msg, sizeof(g_msg), "no usable CUDA device (%s)", cudaGetErrorString(err));
        return -1;
    }
    double *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_scratch_mu);
        if (!g_scratch_addr[dev]) {
            err = cudaGetSymbolAddress((void **)&g_scratch_addr[dev], g_offset_scratch);
            if (err != cudaSuccess) {
                g_scratch_addr[dev] = nullptr;
                snprintf(g_msg, sizeof(g_msg), "cudaGetSymbolAddress: %s", cudaGetErrorString(err));
                return -1;
            }
        }
        scratch = g_scratch_addr[dev];
    }
    MbirGeom g{};
    g.N_p = N_p;
    g.N_r = N_r;
    g.N_t = N_t;
    MbirPrior pr{};
    pr.hT = quad_convex == 0 ? (double)huber_T : 100000.0;
    pr.hdelta = quad_convex == 0 ? (double)huber_delta : 1.0;
    MbirDev dv{};
    dv.e = e;
    dv.w = const_cast<float *>(w);
    dv.d = d;
    const size_t nel = (size_t)N_r * N_t;
    // every word of the scratch that the kernels read is written earlier in
    // the same call, so nothing needs clearing between calls
    err = mbir_launch_offset(g, pr, dv, remove_rings, scratch, scratch + nel, scratch + 2 * nel, kParts,
                             (cudaStream_t)stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize((cudaStream_t)stream);
    if (err != cudaSuccess) {
        snprintf(g_msg, sizeof(g_msg), "ring-offset kernels: %s", cudaGetErrorString(err));
        return -1;
    }
    return 0;
}
