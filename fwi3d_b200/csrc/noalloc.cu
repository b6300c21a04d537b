// noalloc.cu -- misfit residual whose scratch lives in a fixed device array.
//
// Who needs it: some callers cannot let a library call cudaMalloc.  A host
// program that evaluates the misfit inside a latency-critical loop cannot
// afford cudaMalloc's implicit device-wide synchronisation, which stalls
// every other stream on the GPU; an application that hands out all device
// memory from its own pool allocator forbids libraries to allocate behind its
// back.  fwi_residual_dev needs a context, and a context allocates; this entry
// point needs none.  It computes the same thing (res = obs - cal in FP32, the
// sum of res^2 in FP64) and keeps its per-block partial sums in
// g_noalloc_partials below instead of in memory obtained from cudaMalloc.
//
// Limits and sharing:
//   - n may not exceed FWI_NOALLOC_MAX_N (one partial per 65536 elements,
//     4096 partials: 32 KiB of scratch, held by every GPU that loads the
//     library until the process exits); larger n is rejected with
//     FWI_ERR_ARG before anything runs.
//   - Every call on a device uses the same array.  Each call overwrites the
//     partials it reads, so nothing has to start at zero, but two calls whose
//     kernels overlap on the GPU (different streams, or host threads racing)
//     corrupt each other's sums: serialise them.
//   - The first call on each device looks up the array's device address with
//     cudaGetSymbolAddress (in host code the array's name is only a host-side
//     stand-in, not a device address).  Make that first call before any stream
//     capture begins.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/fwi3d.h"

namespace {

constexpr int kNoAllocChunk = 65536;   // elements reduced by one block
constexpr int kNoAllocPartials = 4096;  // capacity of the scratch array
constexpr int kNoAllocThreads = 256;
static_assert((long long)kNoAllocChunk * kNoAllocPartials == FWI_NOALLOC_MAX_N, "limit mismatch");

static __device__ __align__(256) double g_noalloc_partials[kNoAllocPartials];

__device__ __forceinline__ double noalloc_block_sum(double v)
{
    __shared__ double red[kNoAllocThreads / 32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kNoAllocThreads / 32; ++w) s += red[w];
    return s;
}

// Block b reduces elements [b*chunk, min(n, (b+1)*chunk)) into partial[b].
__global__ void __launch_bounds__(kNoAllocThreads)
    noalloc_partial_kernel(const float *__restrict__ obs, const float *__restrict__ cal, long long n,
                           float *__restrict__ res, double *__restrict__ partial)
{
    const long long begin = (long long)blockIdx.x * kNoAllocChunk;
    const long long end = begin + kNoAllocChunk < n ? begin + kNoAllocChunk : n;
    double acc = 0.0;
    for (long long c = begin + threadIdx.x; c < end; c += kNoAllocThreads) {
        const float r = obs[c] - cal[c];
        if (res) res[c] = r;
        acc += (double)r * (double)r;
    }
    const double s = noalloc_block_sum(acc);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// One block adds the np partials in a fixed order and writes the total.
__global__ void __launch_bounds__(kNoAllocThreads)
    noalloc_finish_kernel(const double *__restrict__ partial, int np, double *__restrict__ out)
{
    double acc = 0.0;
    for (int c = threadIdx.x; c < np; c += kNoAllocThreads) acc += partial[c];
    const double s = noalloc_block_sum(acc);
    if (threadIdx.x == 0) *out = s;
}

// Device address of g_noalloc_partials, looked up once per device.
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
double *g_noalloc_addr[kMaxDevices] = {};

int noalloc_scratch(double **out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return FWI_ERR_NODEV;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_partials) != cudaSuccess || !p) {
            cudaGetLastError();
            return FWI_ERR_CUDA;
        }
        g_noalloc_addr[dev] = static_cast<double *>(p);
    }
    *out = g_noalloc_addr[dev];
    return FWI_OK;
}

}  // namespace

extern "C" int fwi_residual_noalloc(const float *d_obs, const float *d_cal, int64_t n, float *d_res,
                                    double *d_sum_sq, void *stream)
{
    if (!d_obs || !d_cal || !d_sum_sq || n < 0) return FWI_ERR_ARG;
    // a non-sticky error left by an earlier call (this library's or another's)
    // must not be reported as this call's launch failure
    cudaGetLastError();
    if (n > FWI_NOALLOC_MAX_N) {
        fprintf(stderr,
                "fwi_residual_noalloc: n = %lld exceeds the no-alloc scratch limit of %lld samples "
                "(FWI_NOALLOC_MAX_N); use fwi_residual_dev or split the call\n",
                (long long)n, (long long)FWI_NOALLOC_MAX_N);
        return FWI_ERR_ARG;
    }
    double *partial = nullptr;
    const int st = noalloc_scratch(&partial);
    if (st != FWI_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int nblocks = (int)((n + kNoAllocChunk - 1) / kNoAllocChunk);
    if (nblocks > 0)
        noalloc_partial_kernel<<<nblocks, kNoAllocThreads, 0, s>>>(d_obs, d_cal, n, d_res, partial);
    noalloc_finish_kernel<<<1, kNoAllocThreads, 0, s>>>(partial, nblocks, d_sum_sq);
    return cudaGetLastError() == cudaSuccess ? FWI_OK : FWI_ERR_CUDA;
}
