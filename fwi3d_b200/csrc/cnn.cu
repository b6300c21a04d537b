// cnn.cu -- the learned gradient preconditioner (no counterpart in the
// reference): a 4-layer 3-D CNN (3 -> 16 -> 16 -> 16 -> 1 channels, 3^3
// kernels, zero "same" padding, ReLU between layers) that maps the raw
// gradient, the velocity and the illumination of an FWI iteration to a model
// update.  Forward and backward run on BF16 tensor cores with FP32
// accumulation; master weights, Adam moments and the loss are FP32 / FP64.
//
// Layout: activations are [V][16] BF16 (voxel v = i + nz*(j + nx*k), z fastest
// like the model volumes, 16 channels per voxel, unused channels zero), so the
// 16 channels of a voxel are one 32-byte row: the K dimension of each
// implicit-GEMM tap.  Weights are [27 taps][16 co][16 ci]; tap t = (dz+1) +
// 3 (dx+1) + 9 (dy+1).
//
// Implicit GEMM per tap: out[v][co] += in[v + off_t][ci] * W[t][co][ci].  A warp
// owns 16 consecutive z voxels of one (x, y) column and all 16 output
// channels: per tap two m16n8k16 BF16 MMAs (M = voxels, N = 8 channels,
// K = 16 channels) accumulate in FP32 registers over the 27 taps.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/fwi3d.h"

namespace {

constexpr int CH = 16;     // channels per voxel row
constexpr int NL = 4;      // layers
constexpr int TAPS = 27;
constexpr int WSZ = TAPS * CH * CH;  // weights per layer
constexpr int CIN[NL] = {3, 16, 16, 16};
constexpr int COUT[NL] = {16, 16, 16, 1};
constexpr int WARPS = 8;   // warps per CTA in the conv kernels

struct Geo {
    int nz, nx, ny;
    long long V;
};

__device__ __forceinline__ uint32_t ld_b32(const __nv_bfloat16 *p) { return *reinterpret_cast<const uint32_t *>(p); }

__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
    __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&h);
}

// ---------------------------------------------------------------------------
// Convolution over all 27 taps.  SIGN = +1: forward (out[v] = sum in[v+off] W);
// SIGN = -1: data gradient (dx[v] = sum dy[v-off] W^T, W given transposed).
// MODE 0: BF16 [V][16] output with bias and ReLU; 1: BF16 [V][16] output times
// the ReLU mask of `mask` (data gradient through the previous activation);
// 2: FP32 channel-0 output with bias (last layer, no activation).
// ---------------------------------------------------------------------------
template <int SIGN, int MODE>
__global__ void __launch_bounds__(WARPS * 32)
    conv_kernel(Geo g, const __nv_bfloat16 *__restrict__ in, const __nv_bfloat16 *__restrict__ w,
                const float *__restrict__ bias, const __nv_bfloat16 *__restrict__ mask,
                __nv_bfloat16 *__restrict__ out, float *__restrict__ out32)
{
    __shared__ __align__(16) __nv_bfloat16 ws[WSZ];
    for (int i = threadIdx.x; i < WSZ / 8; i += blockDim.x)
        reinterpret_cast<uint4 *>(ws)[i] = reinterpret_cast<const uint4 *>(w)[i];
    __syncthreads();

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int grp = lane >> 2, q = lane & 3;
    const int nzt = (g.nz + 15) / 16;
    const long long ntiles = (long long)nzt * g.nx * g.ny;
    for (long long tile = (long long)blockIdx.x * WARPS + warp; tile < ntiles; tile += (long long)gridDim.x * WARPS) {
        const int zt = (int)(tile % nzt);
        const long long col = tile / nzt;
        const int j = (int)(col % g.nx), k = (int)(col / g.nx);
        const int z0 = zt * 16;
        float acc0[4] = {0, 0, 0, 0}, acc1[4] = {0, 0, 0, 0};
        for (int dy = -1; dy <= 1; ++dy) {
            const int kk = k + SIGN * dy;
            if (kk < 0 || kk >= g.ny) continue;
            for (int dx = -1; dx <= 1; ++dx) {
                const int jj = j + SIGN * dx;
                if (jj < 0 || jj >= g.nx) continue;
                const long long cbase = ((long long)kk * g.nx + jj) * g.nz;
#pragma unroll
                for (int dz = -1; dz <= 1; ++dz) {
                    const int t = (dz + 1) + 3 * (dx + 1) + 9 * (dy + 1);
                    const int za = z0 + grp + SIGN * dz, zb = za + 8;
                    const bool va = za >= 0 && za < g.nz, vb = zb >= 0 && zb < g.nz;
                    const __nv_bfloat16 *ra = in + (cbase + za) * CH + 2 * q;
                    const __nv_bfloat16 *rb = in + (cbase + zb) * CH + 2 * q;
                    const uint32_t a0 = va ? ld_b32(ra) : 0u, a2 = va ? ld_b32(ra + 8) : 0u;
                    const uint32_t a1 = vb ? ld_b32(rb) : 0u, a3 = vb ? ld_b32(rb + 8) : 0u;
                    const __nv_bfloat16 *wt = ws + t * CH * CH + grp * CH + 2 * q;
                    mma_bf16(acc0, a0, a1, a2, a3, ld_b32(wt), ld_b32(wt + 8));
                    mma_bf16(acc1, a0, a1, a2, a3, ld_b32(wt + 8 * CH), ld_b32(wt + 8 * CH + 8));
                }
            }
        }
        const long long base = ((long long)k * g.nx + j) * g.nz;
        const int za = z0 + grp, zb = za + 8;
        if constexpr (MODE == 2) {
            // last layer: only output channel 0 is real (thread q == 0 of n-tile 0)
            if (q == 0) {
                if (za < g.nz) out32[base + za] = acc0[0] + bias[0];
                if (zb < g.nz) out32[base + zb] = acc0[2] + bias[0];
            }
        } else {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int z = h ? zb : za;
            if (z >= g.nz) continue;
            const long long v = base + z;
#pragma unroll
            for (int nt = 0; nt < 2; ++nt) {
                const float *acc = nt ? acc1 : acc0;
                const int co = nt * 8 + 2 * q;
                float x0 = acc[2 * h], x1 = acc[2 * h + 1];
                if (MODE == 0) {
                    x0 = fmaxf(x0 + bias[co], 0.0f);
                    x1 = fmaxf(x1 + bias[co + 1], 0.0f);
                } else {
                    const __nv_bfloat162 m = *reinterpret_cast<const __nv_bfloat162 *>(mask + v * CH + co);
                    if (!(__bfloat162float(m.x) > 0.0f)) x0 = 0.0f;
                    if (!(__bfloat162float(m.y) > 0.0f)) x1 = 0.0f;
                }
                *reinterpret_cast<uint32_t *>(out + v * CH + co) = pack_bf16(x0, x1);
            }
        }
        }
    }
}

// ---------------------------------------------------------------------------
// Weight gradient: dW[t][co][ci] = sum_v dy[v][co] x[v + off_t][ci], as
// M = co (16) x N = ci (16) x K = voxels MMAs.  Warp w of a CTA owns taps
// 3w..3w+2 over the CTA's columns, so every partial is written by one warp
// (no atomics); partials [cta][27][16][16] are summed in a fixed order by
// reduce_partials_kernel.  Bias gradient partials ride along in warp 0.
// ---------------------------------------------------------------------------
constexpr int WG_WARPS = 9;

__global__ void __launch_bounds__(WG_WARPS * 32)
    conv_wgrad_kernel(Geo g, const __nv_bfloat16 *__restrict__ x, const __nv_bfloat16 *__restrict__ dy,
                      int cols_per_cta, float *__restrict__ partial, float *__restrict__ bpartial)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int grp = lane >> 2, q = lane & 3;
    const long long ncols = (long long)g.nx * g.ny;
    const long long c0 = (long long)blockIdx.x * cols_per_cta;
    const long long c1 = c0 + cols_per_cta < ncols ? c0 + cols_per_cta : ncols;
    float acc[3][2][4];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.0f;
    float bacc = 0.0f;
    const int tdy = warp / 3 - 1, tdx = warp % 3 - 1;  // taps (dz, tdx, tdy), dz = -1..1
    for (long long col = c0; col < c1; ++col) {
        const int j = (int)(col % g.nx), k = (int)(col / g.nx);
        const long long base = ((long long)k * g.nx + j) * g.nz;
        const int jj = j + tdx, kk = k + tdy;
        const bool cin = jj >= 0 && jj < g.nx && kk >= 0 && kk < g.ny;
        const long long xbase = ((long long)kk * g.nx + jj) * g.nz;
        for (int z0 = 0; z0 < g.nz; z0 += 16) {
            // A (m = co, k = voxel): rows grp, grp+8; voxels 2q, 2q+1, 2q+8, 2q+9
            uint32_t a[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int co = grp + (r & 1) * 8;
                const int zv = z0 + 2 * q + (r >> 1) * 8;
                const float lo = zv < g.nz ? __bfloat162float(dy[(base + zv) * CH + co]) : 0.0f;
                const float hi = zv + 1 < g.nz ? __bfloat162float(dy[(base + zv + 1) * CH + co]) : 0.0f;
                a[r] = pack_bf16(lo, hi);
            }
            if (!cin) continue;
#pragma unroll
            for (int dz = -1; dz <= 1; ++dz) {
#pragma unroll
                for (int nt = 0; nt < 2; ++nt) {
                    // B (k = voxel, n = ci): voxels 2q, 2q+1 (+8), channel nt*8 + grp
                    const int ci = nt * 8 + grp;
                    uint32_t b[2];
#pragma unroll
                    for (int r = 0; r < 2; ++r) {
                        // K index z (voxel of dy) reads x at z + dz of the shifted column
                        float vals[2];
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const int z = z0 + 2 * q + r * 8 + h, zx = z + dz;
                            vals[h] = (z < g.nz && zx >= 0 && zx < g.nz)
                                          ? __bfloat162float(x[(xbase + zx) * CH + ci]) : 0.0f;
                        }
                        b[r] = pack_bf16(vals[0], vals[1]);
                    }
                    mma_bf16(acc[dz + 1][nt], a[0], a[1], a[2], a[3], b[0], b[1]);
                }
            }
        }
        if (warp == 0) {
            // bias gradient: lane l sums channel l & 15 over half of the column
            const int co = lane & 15;
            for (int z = lane >> 4; z < g.nz; z += 2) bacc += __bfloat162float(dy[(base + z) * CH + co]);
        }
    }
    float *P = partial + (long long)blockIdx.x * WSZ;
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz) {
        const int t = (dz + 1) + 3 * (tdx + 1) + 9 * (tdy + 1);
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) {
            const float *c = acc[dz + 1][nt];
            const int ci = nt * 8 + 2 * q;
            P[t * CH * CH + grp * CH + ci] = c[0];
            P[t * CH * CH + grp * CH + ci + 1] = c[1];
            P[t * CH * CH + (grp + 8) * CH + ci] = c[2];
            P[t * CH * CH + (grp + 8) * CH + ci + 1] = c[3];
        }
    }
    if (warp == 0) {
        bacc += __shfl_down_sync(0xffffffffu, bacc, 16);
        if (lane < 16) bpartial[(long long)blockIdx.x * CH + lane] = bacc;
    }
}

// Fixed-order sum of per-CTA partials: out[i] = sum_b part[b][i].
__global__ void reduce_partials_kernel(const float *__restrict__ part, int nb, int n, float *__restrict__ out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float s = 0.0f;
        for (int b = 0; b < nb; ++b) s += part[(long long)b * n + i];
        out[i] = s;
    }
}

// Pack three FP32 channel volumes into the BF16 [V][16] input rows.
__global__ void pack_input_kernel(long long V, const float *__restrict__ c0, const float *__restrict__ c1,
                                  const float *__restrict__ c2, __nv_bfloat16 *__restrict__ out)
{
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V; v += (long long)gridDim.x * blockDim.x) {
        uint4 r0, r1;
        r0.x = pack_bf16(c0[v], c1[v]);
        r0.y = pack_bf16(c2[v], 0.0f);
        r0.z = r0.w = 0u;
        r1.x = r1.y = r1.z = r1.w = 0u;
        reinterpret_cast<uint4 *>(out + v * CH)[0] = r0;
        reinterpret_cast<uint4 *>(out + v * CH)[1] = r1;
    }
}

// Loss 0.5 * mean (pred - target)^2 (FP64 partials) and its gradient,
// scaled by `gscale`, into channel 0 of a BF16 [V][16] buffer.
__global__ void mse_kernel(long long V, const float *__restrict__ pred, const float *__restrict__ target,
                           float gscale, __nv_bfloat16 *__restrict__ grad, double *__restrict__ partial)
{
    __shared__ double red[8];
    double acc = 0.0;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V; v += (long long)gridDim.x * blockDim.x) {
        const float d = pred[v] - target[v];
        acc += (double)d * d;
        uint4 r0;
        r0.x = pack_bf16(d * gscale, 0.0f);
        r0.y = r0.z = r0.w = 0u;
        reinterpret_cast<uint4 *>(grad + v * CH)[0] = r0;
        reinterpret_cast<uint4 *>(grad + v * CH)[1] = make_uint4(0u, 0u, 0u, 0u);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        partial[blockIdx.x] = s;
    }
}

__global__ void sum_f64_kernel(const double *__restrict__ p, int n, double *__restrict__ out)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < n; ++i) s += p[i];
        *out = s;
    }
}

// Adam on the FP32 master weights (Kingma & Ba, 2015), then the BF16 copies:
// forward layout [t][co][ci] and the data-gradient layout [t][ci][co].  The
// mask keeps the padding channels of the first and last layer at zero.
__global__ void adam_kernel(int n, float *__restrict__ w, const float *__restrict__ gw, float *__restrict__ m,
                            float *__restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2,
                            const float *__restrict__ mask, __nv_bfloat16 *__restrict__ wb,
                            __nv_bfloat16 *__restrict__ wt)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float g = gw[i] * mask[i];
        const float mi = b1 * m[i] + (1.0f - b1) * g;
        const float vi = b2 * v[i] + (1.0f - b2) * g * g;
        m[i] = mi;
        v[i] = vi;
        const float wi = (w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps)) * mask[i];
        w[i] = wi;
        if (wb) {
            wb[i] = __float2bfloat16_rn(wi);
            const int t = i / (CH * CH), co = (i / CH) % CH, ci = i % CH;
            wt[t * CH * CH + ci * CH + co] = __float2bfloat16_rn(wi);
        }
    }
}

__global__ void bias_adam_kernel(int n, float *__restrict__ b, const float *__restrict__ gb, float *__restrict__ m,
                                 float *__restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2,
                                 int nreal)
{
    const int i = threadIdx.x;
    if (i < n) {
        const float g = i < nreal ? gb[i] : 0.0f;
        m[i] = b1 * m[i] + (1.0f - b1) * g;
        v[i] = b2 * v[i] + (1.0f - b2) * g * g;
        b[i] = i < nreal ? b[i] - lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps) : 0.0f;
    }
}

template <class T>
struct Buf {
    T *p = nullptr;
    size_t n = 0;
    cudaError_t ensure(size_t want)
    {
        if (want <= n) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMalloc((void **)&p, want * sizeof(T));
        if (e == cudaSuccess) n = want;
        return e;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

}  // namespace

struct fwi_cnn {
    Geo g{};
    cudaStream_t stream = nullptr;
    Buf<float> w32[NL], gw[NL], mw[NL], vw[NL], mask[NL];
    Buf<float> b32[NL], gb[NL], mb[NL], vb[NL];
    Buf<__nv_bfloat16> wb[NL], wt[NL];
    Buf<__nv_bfloat16> act[NL];  // act[0] input, act[l] = output of layer l-1 (l = 1..3)
    Buf<__nv_bfloat16> dg[2];    // data gradients, ping-pong
    Buf<float> pred, partial, bpartial;
    Buf<double> lpart, lsum;
    int adam_step = 0;
    std::string err;
};

namespace {

#define CNN_CK(call)                                                            \
    do {                                                                        \
        cudaError_t e_ = (call);                                                \
        if (e_ != cudaSuccess) {                                                \
            n->err = std::string(#call) + ": " + cudaGetErrorString(e_);        \
            return e_ == cudaErrorMemoryAllocation ? FWI_ERR_ALLOC : FWI_ERR_CUDA; \
        }                                                                       \
    } while (0)

int conv_blocks(const Geo &g)
{
    const long long tiles = (long long)((g.nz + 15) / 16) * g.nx * g.ny;
    long long b = (tiles + WARPS - 1) / WARPS;
    return (int)std::min<long long>(std::max<long long>(b, 1), 148LL * 8);
}

int forward_impl(fwi_cnn *n)
{
    const Geo &g = n->g;
    const int blocks = conv_blocks(g);
    for (int l = 0; l < NL; ++l) {
        if (l < NL - 1) {
            conv_kernel<1, 0><<<blocks, WARPS * 32, 0, n->stream>>>(g, n->act[l].p, n->wb[l].p, n->b32[l].p, nullptr,
                                                                    n->act[l + 1].p, nullptr);
        } else {
            conv_kernel<1, 2><<<blocks, WARPS * 32, 0, n->stream>>>(g, n->act[l].p, n->wb[l].p, n->b32[l].p, nullptr,
                                                                    nullptr, n->pred.p);
        }
    }
    CNN_CK(cudaGetLastError());
    return FWI_OK;
}

int ensure_volume(fwi_cnn *n, int nz, int nx, int ny)
{
    if (nz < 1 || nx < 1 || ny < 1) return FWI_ERR_ARG;
    n->g = Geo{nz, nx, ny, (long long)nz * nx * ny};
    const size_t V = n->g.V;
    for (int l = 0; l < NL; ++l) CNN_CK(n->act[l].ensure(V * CH));
    for (int k = 0; k < 2; ++k) CNN_CK(n->dg[k].ensure(V * CH));
    CNN_CK(n->pred.ensure(V));
    const long long ncols = (long long)nx * ny;
    const int cpc = (int)std::max<long long>(1, (ncols + 2047) / 2048);
    const int nblk = (int)((ncols + cpc - 1) / cpc);
    CNN_CK(n->partial.ensure((size_t)nblk * WSZ));
    CNN_CK(n->bpartial.ensure((size_t)nblk * CH));
    CNN_CK(n->lpart.ensure(1024));
    CNN_CK(n->lsum.ensure(1));
    return FWI_OK;
}

int upload_bf16(fwi_cnn *n, int l)
{
    std::vector<float> w(WSZ);
    CNN_CK(cudaMemcpy(w.data(), n->w32[l].p, WSZ * sizeof(float), cudaMemcpyDeviceToHost));
    std::vector<__nv_bfloat16> b(WSZ), t(WSZ);
    for (int i = 0; i < WSZ; ++i) {
        const int tap = i / (CH * CH), co = (i / CH) % CH, ci = i % CH;
        b[i] = __float2bfloat16_rn(w[i]);
        t[tap * CH * CH + ci * CH + co] = b[i];
    }
    CNN_CK(cudaMemcpy(n->wb[l].p, b.data(), WSZ * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice));
    CNN_CK(cudaMemcpy(n->wt[l].p, t.data(), WSZ * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice));
    return FWI_OK;
}

}  // namespace

extern "C" {

int fwi_cnn_create(uint64_t seed, fwi_cnn **out)
{
    if (!out) return FWI_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return FWI_ERR_NODEV;
    }
    fwi_cnn *n = new fwi_cnn();
    std::mt19937_64 rng(seed);
    int st = FWI_OK;
    for (int l = 0; l < NL && st == FWI_OK; ++l) {
        // He initialisation over the real fan-in, zero on padding channels
        std::normal_distribution<float> N(0.0f, std::sqrt(2.0f / (TAPS * CIN[l])));
        std::vector<float> w(WSZ, 0.0f), mk(WSZ, 0.0f);
        for (int t = 0; t < TAPS; ++t)
            for (int co = 0; co < COUT[l]; ++co)
                for (int ci = 0; ci < CIN[l]; ++ci) {
                    const int i = t * CH * CH + co * CH + ci;
                    w[i] = N(rng) * (l == NL - 1 ? 0.1f : 1.0f);
                    mk[i] = 1.0f;
                }
        for (auto *b : {&n->w32[l], &n->gw[l], &n->mw[l], &n->vw[l], &n->mask[l]})
            if (b->ensure(WSZ) != cudaSuccess) st = FWI_ERR_ALLOC;
        for (auto *b : {&n->b32[l], &n->gb[l], &n->mb[l], &n->vb[l]})
            if (b->ensure(CH) != cudaSuccess) st = FWI_ERR_ALLOC;
        for (auto *b : {&n->wb[l], &n->wt[l]})
            if (b->ensure(WSZ) != cudaSuccess) st = FWI_ERR_ALLOC;
        if (st != FWI_OK) break;
        cudaMemcpy(n->w32[l].p, w.data(), WSZ * sizeof(float), cudaMemcpyHostToDevice);
        cudaMemcpy(n->mask[l].p, mk.data(), WSZ * sizeof(float), cudaMemcpyHostToDevice);
        cudaMemset(n->mw[l].p, 0, WSZ * sizeof(float));
        cudaMemset(n->vw[l].p, 0, WSZ * sizeof(float));
        cudaMemset(n->b32[l].p, 0, CH * sizeof(float));
        cudaMemset(n->mb[l].p, 0, CH * sizeof(float));
        cudaMemset(n->vb[l].p, 0, CH * sizeof(float));
        st = upload_bf16(n, l);
    }
    if (st != FWI_OK) {
        fwi_cnn_destroy(n);
        return st;
    }
    *out = n;
    return FWI_OK;
}

int fwi_cnn_destroy(fwi_cnn *n)
{
    if (!n) return FWI_ERR_ARG;
    for (int l = 0; l < NL; ++l) {
        for (auto *b : {&n->w32[l], &n->gw[l], &n->mw[l], &n->vw[l], &n->mask[l], &n->b32[l], &n->gb[l], &n->mb[l],
                        &n->vb[l]})
            b->release();
        n->wb[l].release();
        n->wt[l].release();
        n->act[l].release();
    }
    n->dg[0].release();
    n->dg[1].release();
    n->pred.release();
    n->partial.release();
    n->bpartial.release();
    n->lpart.release();
    n->lsum.release();
    delete n;
    return FWI_OK;
}

int fwi_cnn_last_error(fwi_cnn *n, char *buf, int cap)
{
    if (!n || !buf || cap <= 0) return FWI_ERR_ARG;
    snprintf(buf, cap, "%s", n->err.c_str());
    return FWI_OK;
}

int fwi_cnn_set_stream(fwi_cnn *n, void *stream)
{
    if (!n) return FWI_ERR_ARG;
    n->stream = (cudaStream_t)stream;
    return FWI_OK;
}

// Weights [layer][27][16 co][16 ci] FP32 and biases [layer][16] (host).
int fwi_cnn_get_weights(fwi_cnn *n, float *w, float *b)
{
    if (!n) return FWI_ERR_ARG;
    CNN_CK(cudaStreamSynchronize(n->stream));
    for (int l = 0; l < NL; ++l) {
        if (w) CNN_CK(cudaMemcpy(w + (size_t)l * WSZ, n->w32[l].p, WSZ * sizeof(float), cudaMemcpyDeviceToHost));
        if (b) CNN_CK(cudaMemcpy(b + (size_t)l * CH, n->b32[l].p, CH * sizeof(float), cudaMemcpyDeviceToHost));
    }
    return FWI_OK;
}

int fwi_cnn_set_weights(fwi_cnn *n, const float *w, const float *b)
{
    if (!n || !w || !b) return FWI_ERR_ARG;
    CNN_CK(cudaStreamSynchronize(n->stream));
    for (int l = 0; l < NL; ++l) {
        std::vector<float> wl(w + (size_t)l * WSZ, w + (size_t)(l + 1) * WSZ), mk(WSZ);
        CNN_CK(cudaMemcpy(mk.data(), n->mask[l].p, WSZ * sizeof(float), cudaMemcpyDeviceToHost));
        for (int i = 0; i < WSZ; ++i) wl[i] *= mk[i];
        std::vector<float> bl(b + (size_t)l * CH, b + (size_t)(l + 1) * CH);
        for (int c = COUT[l]; c < CH; ++c) bl[c] = 0.0f;
        CNN_CK(cudaMemcpy(n->w32[l].p, wl.data(), WSZ * sizeof(float), cudaMemcpyHostToDevice));
        CNN_CK(cudaMemcpy(n->b32[l].p, bl.data(), CH * sizeof(float), cudaMemcpyHostToDevice));
        const int st = upload_bf16(n, l);
        if (st != FWI_OK) return st;
    }
    return FWI_OK;
}

// Forward pass.  d_in: three FP32 device volumes [3][V] (already normalised);
// d_out: FP32 device volume [V].
int fwi_cnn_forward(fwi_cnn *n, int nz, int nx, int ny, const float *d_in, float *d_out)
{
    if (!n || !d_in || !d_out) return FWI_ERR_ARG;
    int st = ensure_volume(n, nz, nx, ny);
    if (st != FWI_OK) return st;
    const long long V = n->g.V;
    pack_input_kernel<<<1184, 256, 0, n->stream>>>(V, d_in, d_in + V, d_in + 2 * V, n->act[0].p);
    st = forward_impl(n);
    if (st != FWI_OK) return st;
    CNN_CK(cudaMemcpyAsync(d_out, n->pred.p, V * sizeof(float), cudaMemcpyDeviceToDevice, n->stream));
    CNN_CK(cudaStreamSynchronize(n->stream));
    return FWI_OK;
}

// Gradients of the loss 0.5 mean (f(x) - target)^2 w.r.t. every weight and
// bias (FP32, [layer][27][16][16] and [layer][16], host), plus the loss.  With
// lr > 0 an Adam step (beta 0.9 / 0.999) follows.
int fwi_cnn_train_step(fwi_cnn *n, int nz, int nx, int ny, const float *d_in, const float *d_target, float lr,
                       double *loss, float *grad_w, float *grad_b)
{
    if (!n || !d_in || !d_target) return FWI_ERR_ARG;
    int st = ensure_volume(n, nz, nx, ny);
    if (st != FWI_OK) return st;
    const Geo &g = n->g;
    const long long V = g.V;
    pack_input_kernel<<<1184, 256, 0, n->stream>>>(V, d_in, d_in + V, d_in + 2 * V, n->act[0].p);
    st = forward_impl(n);
    if (st != FWI_OK) return st;
    // loss gradient d(0.5 mean d^2)/dpred = d / V, carried in BF16 scaled up
    // by V (loss scaling) and scaled back in the weight gradients
    const int lblk = 1024;
    mse_kernel<<<lblk, 256, 0, n->stream>>>(V, n->pred.p, d_target, 1.0f, n->dg[0].p, n->lpart.p);
    sum_f64_kernel<<<1, 32, 0, n->stream>>>(n->lpart.p, lblk, n->lsum.p);
    const long long ncols = (long long)g.nx * g.ny;
    const int cpc = (int)std::max<long long>(1, (ncols + 2047) / 2048);
    const int nblk = (int)((ncols + cpc - 1) / cpc);
    const int blocks = conv_blocks(g);
    int cur = 0;
    for (int l = NL - 1; l >= 0; --l) {
        // weight and bias gradients of layer l: input act[l], output gradient dg[cur]
        conv_wgrad_kernel<<<nblk, WG_WARPS * 32, 0, n->stream>>>(g, n->act[l].p, n->dg[cur].p, cpc, n->partial.p,
                                                                  n->bpartial.p);
        reduce_partials_kernel<<<(WSZ + 255) / 256, 256, 0, n->stream>>>(n->partial.p, nblk, WSZ, n->gw[l].p);
        reduce_partials_kernel<<<1, 32, 0, n->stream>>>(n->bpartial.p, nblk, CH, n->gb[l].p);
        if (l > 0) {
            // data gradient through layer l, masked by the ReLU of act[l]
            conv_kernel<-1, 1><<<blocks, WARPS * 32, 0, n->stream>>>(g, n->dg[cur].p, n->wt[l].p, nullptr,
                                                                     n->act[l].p, n->dg[1 - cur].p, nullptr);
            cur = 1 - cur;
        }
    }
    CNN_CK(cudaGetLastError());
    double lsum = 0.0;
    CNN_CK(cudaMemcpyAsync(&lsum, n->lsum.p, sizeof(double), cudaMemcpyDeviceToHost, n->stream));
    CNN_CK(cudaStreamSynchronize(n->stream));
    if (loss) *loss = 0.5 * lsum / (double)V;
    // the loss gradient was d (not d/V): scale the parameter gradients by 1/V
    const float inv = 1.0f / (float)V;
    std::vector<float> tmp(WSZ), tb(CH);
    for (int l = 0; l < NL; ++l) {
        if (grad_w || lr > 0) {
            CNN_CK(cudaMemcpy(tmp.data(), n->gw[l].p, WSZ * sizeof(float), cudaMemcpyDeviceToHost));
            for (auto &x : tmp) x *= inv;
            if (grad_w) memcpy(grad_w + (size_t)l * WSZ, tmp.data(), WSZ * sizeof(float));
            CNN_CK(cudaMemcpy(n->gw[l].p, tmp.data(), WSZ * sizeof(float), cudaMemcpyHostToDevice));
        }
        if (grad_b || lr > 0) {
            CNN_CK(cudaMemcpy(tb.data(), n->gb[l].p, CH * sizeof(float), cudaMemcpyDeviceToHost));
            for (auto &x : tb) x *= inv;
            if (grad_b) memcpy(grad_b + (size_t)l * CH, tb.data(), CH * sizeof(float));
            CNN_CK(cudaMemcpy(n->gb[l].p, tb.data(), CH * sizeof(float), cudaMemcpyHostToDevice));
        }
    }
    if (lr > 0) {
        ++n->adam_step;
        const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
        const float c1 = 1.0f - powf(b1, (float)n->adam_step), c2 = 1.0f - powf(b2, (float)n->adam_step);
        for (int l = 0; l < NL; ++l) {
            adam_kernel<<<(WSZ + 255) / 256, 256, 0, n->stream>>>(WSZ, n->w32[l].p, n->gw[l].p, n->mw[l].p,
                                                                  n->vw[l].p, lr, b1, b2, eps, c1, c2, n->mask[l].p,
                                                                  n->wb[l].p, n->wt[l].p);
            bias_adam_kernel<<<1, CH, 0, n->stream>>>(CH, n->b32[l].p, n->gb[l].p, n->mb[l].p, n->vb[l].p, lr, b1,
                                                      b2, eps, c1, c2, COUT[l]);
        }
        CNN_CK(cudaGetLastError());
        CNN_CK(cudaStreamSynchronize(n->stream));
    }
    return FWI_OK;
}

}  // extern "C"
