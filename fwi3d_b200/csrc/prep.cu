// prep.cu -- RTM input preprocessing on the GPU (run/generate_input_data.py:
// 28-46 of the reference): every shot gather is scaled by 1/max|d|, then each
// trace is tapered before its direct-wave time
//     t_r = int((|x_r - x_s| / velocity + time_delay) / dt)
//     d[t, r] *= exp(-0.5 ((t - t_r) / gstd)^2)   for t < t_r.
// The arithmetic follows the reference's numpy dtypes: the scale factor is
// rounded to FP32 before the multiply, t_r is computed in FP32 and truncated,
// the taper is FP64 and the product is rounded to FP32.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>

#include "../../include/fwi3d.h"

namespace {

__global__ void maxabs_bits_kernel(const float *__restrict__ d, long long n, unsigned int *__restrict__ out)
{
    float m = 0.0f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(d[i]));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

// One block per receiver trace (Fortran [nt, nrec]: trace r is contiguous).
__global__ void mute_kernel(const float *__restrict__ in, float *__restrict__ out, int nt, int nrec,
                            const float *__restrict__ rx, const float *__restrict__ ry, float sx, float sy,
                            float velocity, float delay, float dt, double gstd,
                            const unsigned int *__restrict__ maxbits)
{
    const int r = blockIdx.x;
    if (r >= nrec) return;
    const float scale = (float)(1.0 / (double)__uint_as_float(*maxbits));
    const float dx = __fsub_rn(rx[r], sx), dy = __fsub_rn(ry[r], sy);
    const float dist = __fsqrt_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)));
    const float tf = __fdiv_rn(__fadd_rn(__fdiv_rn(dist, velocity), delay), dt);
    const int tr = (int)tf;
    for (int t = threadIdx.x; t < nt; t += blockDim.x) {
        float v = __fmul_rn(in[(long long)r * nt + t], scale);
        if (t < tr) {
            const double a = ((double)(t - tr)) / gstd;
            v = (float)((double)v * exp(-0.5 * (a * a)));
        }
        out[(long long)r * nt + t] = v;
    }
}

}  // namespace

extern "C" int fwi_prepare_rtm_input(const float *seis, float *out, int nt, int nrec, const float *rx,
                                     const float *ry, float sx, float sy, float velocity, float time_delay,
                                     float dt, float gstd)
{
    if (!seis || !out || !rx || !ry || nt < 1 || nrec < 1 || !(velocity > 0) || !(dt > 0) || !(gstd > 0))
        return FWI_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return FWI_ERR_NODEV;
    }
    const size_t n = (size_t)nt * nrec;
    float *d_in = nullptr, *d_out = nullptr, *d_rx = nullptr, *d_ry = nullptr;
    unsigned int *d_max = nullptr;
    cudaError_t e = cudaMalloc(&d_in, n * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&d_out, n * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&d_rx, nrec * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&d_ry, nrec * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&d_max, sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMemcpy(d_in, seis, n * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_rx, rx, nrec * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_ry, ry, nrec * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(d_max, 0, sizeof(unsigned int));
    if (e == cudaSuccess) {
        maxabs_bits_kernel<<<592, 256>>>(d_in, (long long)n, d_max);
        mute_kernel<<<nrec, 256>>>(d_in, d_out, nt, nrec, d_rx, d_ry, sx, sy, velocity, time_delay, dt,
                                   (double)gstd, d_max);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, d_out, n * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(d_in);
    cudaFree(d_out);
    cudaFree(d_rx);
    cudaFree(d_ry);
    cudaFree(d_max);
    if (e != cudaSuccess) {
        fprintf(stderr, "fwi_prepare_rtm_input: %s\n", cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? FWI_ERR_ALLOC : FWI_ERR_CUDA;
    }
    return FWI_OK;
}
