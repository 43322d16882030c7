// og_noalloc.cu -- og_segment_sum_noalloc: the fixed-order segmented sum of og_segment_sum for
// callers that cannot allocate device memory at call time.
//
// Who needs it: code whose process has handed all free device memory to another allocator (a
// framework memory pool sized to the whole GPU), where even a small cudaMalloc / cudaMallocAsync
// fails, and code on a latency-critical path where an allocation call is not acceptable.  Those
// callers still pass their own input and output buffers; this entry point only avoids the
// scratch allocation of og_segment_sum.
//
// The scratch is the file-scope array below (512 KiB on every GPU that loads this library,
// held until the process exits).  Host code cannot pass the array's name to a kernel: on the
// host it is only a stand-in symbol, not a device address.  The device address is obtained
// once per device with cudaGetSymbolAddress, with that device current, on the first call made
// while that device is current; that first call should therefore come before any stream
// capture.  The address belongs to the device's primary context (the one the CUDA runtime
// uses): call this only from that context, and not after a cudaDeviceReset of the device,
// which unloads the module and leaves the looked-up address stale.  Every used scratch entry
// is written before it is read in the same call, so nothing needs clearing; all calls share
// the array, so calls that overlap on the GPU (different streams, or different host threads)
// race and must be serialised by the caller.
//
// Limits: n_seg <= 65535 (one grid row per segment) and n_seg * ceil(max_seg_len / 4096) <=
// 65536 (the scratch holds one partial sum per 4096-item chunk of every segment); beyond
// either the call returns OG_ERR_CAPACITY without launching anything.  A CUDA error already
// pending on the calling thread when the call starts is reported as OG_ERR_CUDA and left
// pending for its owner; nothing is launched then either.
#include <mutex>

#include "../../include/omegagene_b200.h"
#include "og_internal.cuh"

namespace og {
template <int NV>
__global__ void k_part(const double *, int, int, const int *, int, double *);
template <int NV>
__global__ void k_part_final(const double *, int, double *, int, int, const float *, int);
}  // namespace og

#define OG_NOALLOC_SCRATCH_DOUBLES 65536  // n_seg * ceil(max_seg_len / 4096) must not exceed this

static __device__ __align__(256) double og_noalloc_scratch[OG_NOALLOC_SCRATCH_DOUBLES];

namespace {
std::mutex g_scratch_mu;
double *g_scratch_ptr[256] = {};  // device address of og_noalloc_scratch, per device ordinal
}  // namespace

extern "C" og_status og_segment_sum_noalloc(const double *d_values, int32_t stride, const int32_t *d_seg_base,
                                            int32_t n_seg, int32_t max_seg_len, double *d_out, void *cuda_stream) {
    if (!d_values || !d_seg_base || !d_out || n_seg <= 0 || stride <= 0 || max_seg_len < 0) return OG_ERR_INVALID;
    const long long max_chunks = max_seg_len > 0 ? ((long long)max_seg_len + 4095) / 4096 : 1;
    if (n_seg > OG_SEGMENT_SUM_MAX_SEGMENTS) return OG_ERR_CAPACITY;
    if ((long long)n_seg * max_chunks > OG_NOALLOC_SCRATCH_DOUBLES) return OG_ERR_CAPACITY;
    if (cudaPeekAtLastError() != cudaSuccess) return OG_ERR_CUDA;  // the caller's error, left pending
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return OG_ERR_CUDA;
    if (dev < 0 || dev >= 256) return OG_ERR_INVALID;
    double *part = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_scratch_mu);
        if (!g_scratch_ptr[dev]) {
            double *p = nullptr;
            if (cudaGetSymbolAddress((void **)&p, og_noalloc_scratch) != cudaSuccess || !p) return OG_ERR_CUDA;
            g_scratch_ptr[dev] = p;
        }
        part = g_scratch_ptr[dev];
    }
    cudaStream_t st = (cudaStream_t)cuda_stream;
    dim3 grid((unsigned)max_chunks, (unsigned)n_seg);
    og::k_part<1><<<grid, 256, 0, st>>>(d_values, stride, 0, d_seg_base, (int)max_chunks, part);
    og::k_part_final<1><<<n_seg, 256, 0, st>>>(part, (int)max_chunks, d_out, 1, 0, nullptr, 0);
    return cudaGetLastError() == cudaSuccess ? OG_OK : OG_ERR_CUDA;  // only this call's launches
}
