// aux_kernels.cuh -- the small kernels around the two stencil kernels:
// padding, source start, adjoint injection, seismogram transposes, image and
// gradient post-processing, FP64 reductions and the random boundary.
#pragma once

#include "device.cuh"

namespace fwi {

// ---------------------------------------------------------------------------
// Edge-replication padding of an unpadded [nz,nx,ny] model into a pitched
// padded field: every padded cell copies the nearest model cell
// (same result as expand_boundary, src/modeling/modeling.cu:181-228).
// ---------------------------------------------------------------------------
__global__ void pad_edges_kernel(const float *__restrict__ in, int nz, int nx, int ny, int nb,
                                 int nzz, int nxx, int nyy, int ldz, float *__restrict__ out)
{
    const long long n = (long long)ldz * nxx * nyy;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % ldz);
        const long long r = c / ldz;
        const int j = (int)(r % nxx), k = (int)(r / nxx);
        if (i >= nzz) {
            out[c] = 0.0f;
            continue;
        }
        const int is = min(max(i - nb, 0), nz - 1);
        const int js = min(max(j - nb, 0), nx - 1);
        const int ks = min(max(k - nb, 0), ny - 1);
        out[c] = in[is + (long long)js * nz + (long long)ks * nx * nz];
    }
}

// Dense padded [nzz,nxx,nyy] <-> pitched [nyy][nxx][ldz].
__global__ void dense_to_pitched_kernel(const float *__restrict__ in, int nzz, int nxx, int nyy,
                                        int ldz, float *__restrict__ out)
{
    const long long n = (long long)ldz * nxx * nyy;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % ldz);
        const long long r = c / ldz;
        out[c] = i < nzz ? in[i + r * nzz] : 0.0f;
    }
}

__global__ void pitched_to_dense_kernel(const float *__restrict__ in, int nzz, int nxx, int nyy,
                                        int ldz, float *__restrict__ out)
{
    const long long n = (long long)nzz * nxx * nyy;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % nzz);
        const long long r = c / nzz;
        out[c] = in[i + r * ldz];
    }
}

// Crop the pad of a pitched field into [nz,nx,ny] (reduce_boundary,
// src/modeling/modeling.cu:230-241).
__global__ void crop_kernel(const float *__restrict__ in, int nz, int nx, int ny, int nb, int nxx,
                            int ldz, float *__restrict__ out)
{
    const long long n = (long long)nz * nx * ny;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % nz);
        const long long r = c / nz;
        const int j = (int)(r % nx), k = (int)(r / nx);
        out[c] = in[(i + nb) + (long long)(j + nb) * ldz + (long long)(k + nb) * ldz * nxx];
    }
}

// Sum the accumulator slots of a batch into slot 0.
__global__ void sum_slots_kernel(float *__restrict__ acc, long long vol, int nslot)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < vol;
         c += (long long)gridDim.x * blockDim.x) {
        float s = acc[c];
        for (int k = 1; k < nslot; ++k) {
            s += acc[c + k * vol];
            acc[c + k * vol] = 0.0f;
        }
        acc[c] = s;
    }
}

// First source sample of every shot: A[src] = idh3 * w[0]
// (src/modeling/modeling.cu:347-348 at t = 0).
__global__ void start_source_kernel(float *__restrict__ A, long long vol, int ldz, int nxx,
                                    const BatchInfo *__restrict__ bi, const float *__restrict__ w,
                                    float idh3)
{
    const int s = threadIdx.x;
    if (s < bi->nshot) {
        const long long c = (long long)s * vol + bi->src[s][0] + (long long)bi->src[s][1] * ldz +
                            (long long)bi->src[s][2] * ldz * nxx;
        A[c] += idh3 * w[0];
    }
}

// ---------------------------------------------------------------------------
// Adjoint injection: Pr[cell] += idh3 * d(receiver) for every receiver on the
// cell, time-reversed (inject_seismogram / inject_residuo,
// src/migration/migration.cu:119-132, src/inversion/inversion.cu:385-398).
// Receivers sharing a cell are added one after another in receiver order,
// which keeps the sum deterministic where the reference uses atomicAdd.
// ---------------------------------------------------------------------------
__global__ void inject_adjoint_kernel(float *__restrict__ Pr, const BatchInfo *__restrict__ bi,
                                      const long long *__restrict__ cell,
                                      const int *__restrict__ first, const int *__restrict__ rid,
                                      const float *__restrict__ data_tm, int sample, float idh3)
{
    const int ncell = bi->ncell, R = bi->R;
    for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < ncell; u += gridDim.x * blockDim.x) {
        float v = Pr[cell[u]];
        for (int k = first[u]; k < first[u + 1]; ++k)
            v += idh3 * data_tm[(long long)sample * R + rid[k]];
        Pr[cell[u]] = v;
    }
}

// [rows][cols] -> [cols][rows], 32x32 tiles through shared memory.
__global__ void transpose_kernel(const float *__restrict__ in, long long rows, long long cols,
                                 float *__restrict__ out)
{
    __shared__ float t[32][33];
    const long long r0 = (long long)blockIdx.y * 32, c0 = (long long)blockIdx.x * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const long long r = r0 + k, c = c0 + threadIdx.x;
        if (r < rows && c < cols) t[k][threadIdx.x] = in[r * cols + c];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const long long c = c0 + k, r = r0 + threadIdx.x;
        if (r < rows && c < cols) out[c * rows + r] = t[threadIdx.x][k];
    }
}

// ---------------------------------------------------------------------------
// RTM image: crop, divide by illumination, -d2/dz2 * idh2 with the first and
// last depth sample 0 (Migration::export_seismic,
// src/migration/migration.cu:90-117), FP32 like the reference.
// ---------------------------------------------------------------------------
// Image or gradient over illumination.  A cell the source field never
// reached has illumination 0 and no image either; the reference's 0/0 there
// is NaN (src/migration/migration.cu:100, src/inversion/inversion.cu:150), the
// project defines it as 0.
__device__ __forceinline__ float ratio(float a, float ill) { return ill != 0.0f ? a / ill : 0.0f; }

__global__ void rtm_image_kernel(const float *__restrict__ img, const float *__restrict__ ill,
                                 int nz, int nx, int ny, int nb, int nxx, int ldz, float idh2,
                                 float *__restrict__ out)
{
    const long long n = (long long)nz * nx * ny;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % nz);
        const long long r = c / nz;
        const int j = (int)(r % nx), k = (int)(r / nx);
        float v = 0.0f;
        if (i > 0 && i < nz - 1) {
            const long long p = (i + nb) + (long long)(j + nb) * ldz + (long long)(k + nb) * ldz * nxx;
            const float sm = ratio(img[p - 1], ill[p - 1]);
            const float s0 = ratio(img[p], ill[p]);
            const float sp = ratio(img[p + 1], ill[p + 1]);
            v = -1.0f * (sm - 2.0f * s0 + sp) * idh2;
        }
        out[c] = v;
    }
}

// Gradient post-processing, first pass: crop, divide, -d2/dz2 below the mask
// and the running max |g| (src/inversion/inversion.cu:142-165).  max|g| of
// non-negative floats is taken with an integer atomicMax on their bits, which
// is exact and order independent.
__global__ void grad_post_kernel(const float *__restrict__ g, const float *__restrict__ ill, int nz,
                                 int nx, int ny, int nb, int nxx, int ldz, float idh2, int imask,
                                 float *__restrict__ out, unsigned int *__restrict__ gmax_bits)
{
    const long long n = (long long)nz * nx * ny;
    float lmax = 0.0f;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % nz);
        const long long r = c / nz;
        const int j = (int)(r % nx), k = (int)(r / nx);
        float v = 0.0f;
        if (i > imask && i < nz - 1) {
            const long long p = (i + nb) + (long long)(j + nb) * ldz + (long long)(k + nb) * ldz * nxx;
            const float sm = ratio(g[p - 1], ill[p - 1]);
            const float s0 = ratio(g[p], ill[p]);
            const float sp = ratio(g[p + 1], ill[p + 1]);
            v = -1.0f * (sm - 2.0f * s0 + sp) * idh2;
        }
        out[c] = v;
        lmax = fmaxf(lmax, fabsf(v));
    }
    for (int o = 16; o > 0; o >>= 1) lmax = fmaxf(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
    if ((threadIdx.x & 31) == 0) atomicMax(gmax_bits, __float_as_uint(lmax));
}

// Second pass: g *= 1/gmax (src/inversion/inversion.cu:167-169).
__global__ void scale_by_inverse_kernel(float *__restrict__ g, long long n,
                                        const unsigned int *__restrict__ gmax_bits)
{
    const float m = __uint_as_float(*gmax_bits);
    const float s = m > 0.0f ? 1.0f / m : 0.0f;  // an all-zero gradient stays zero
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x)
        g[c] *= s;
}

// ---------------------------------------------------------------------------
// FP64 reductions.  Stage 1 writes one partial per block in a fixed order;
// stage 2 adds the partials in a fixed order: the result does not depend on
// scheduling.
// ---------------------------------------------------------------------------
template <int NT>
__device__ __forceinline__ double block_sum(double v)
{
    __shared__ double red[NT / 32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < NT / 32; ++w) s += red[w];
    return s;
}

// res = obs - cal (FP32, as the reference stores it) and sum(res^2) in FP64
// (src/inversion/inversion.cu:194-198).
template <int NT>
__global__ void __launch_bounds__(NT)
    residual_partial_kernel(const float *__restrict__ obs, const float *__restrict__ cal,
                            long long n, float *__restrict__ res, double *__restrict__ partial)
{
    double acc = 0.0;
    for (long long c = blockIdx.x * (long long)NT + threadIdx.x; c < n; c += (long long)gridDim.x * NT) {
        const float r = obs[c] - cal[c];
        if (res) res[c] = r;
        acc += (double)r * (double)r;
    }
    const double s = block_sum<NT>(acc);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

template <int NT>
__global__ void __launch_bounds__(NT)
    dot_partial_kernel(const float *__restrict__ a, const float *__restrict__ b, long long n,
                       double *__restrict__ partial)
{
    double acc = 0.0;
    for (long long c = blockIdx.x * (long long)NT + threadIdx.x; c < n; c += (long long)gridDim.x * NT)
        acc += (double)a[c] * (double)b[c];
    const double s = block_sum<NT>(acc);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

template <int NT>
__global__ void __launch_bounds__(NT)
    finish_sum_kernel(const double *__restrict__ partial, int n, double *__restrict__ out)
{
    double acc = 0.0;
    for (int c = threadIdx.x; c < n; c += NT) acc += partial[c];
    const double s = block_sum<NT>(acc);
    if (threadIdx.x == 0) *out = s;
}

// ---------------------------------------------------------------------------
// Deterministic random boundary.
// Counter-based generator: the SplitMix64 output function (Steele, Lea and
// Flood, "Fast splittable pseudorandom number generators", OOPSLA 2014)
// applied to (seed, stream, counter); uniforms take the top 24 bits and
// normals come from the Box-Muller transform.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

__device__ __forceinline__ float uniform01(uint64_t seed, uint64_t stream, uint64_t ctr)
{
    const uint64_t h = splitmix64(seed ^ splitmix64(stream * 0x632BE59BD9B4E019ull + ctr));
    return ((float)(h >> 40) + 0.5f) * (1.0f / 16777216.0f);
}

// Box-Muller in FP64, rounded once to FP32: the deviate is then the FP32
// rounding of a value any FP64 restatement computes to within a few FP64
// ulps, so a host restatement reproduces it bit for bit.
__device__ __forceinline__ float normal01(uint64_t seed, uint64_t stream, uint64_t ctr)
{
    const double u1 = (double)uniform01(seed, stream, 2 * ctr);
    const double u2 = (double)uniform01(seed, stream, 2 * ctr + 1);
    return (float)(sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2));
}

// Pad background.  For every pad cell take the nearest model-edge value, then
//   kind 0: add ramp_a * varVp * N(0,1) for every axis a in the pad, with
//           ramp_a = 1 - depth_a/nb  (random_boundary_bg,
//           src/modeling/modeling.cu:617-666)
//   kind 1: scale by 1 + ratio * ramp * U(-1,1), ramp = max_a ramp_a
// and clamp to [vlo, vhi].
__global__ void rbc_background_kernel(float *__restrict__ vp, int nzz, int nxx, int nyy, int ldz,
                                      int nb, int kind, float ratio, float varVp, float vlo,
                                      float vhi, uint64_t seed)
{
    const long long n = (long long)ldz * nxx * nyy;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % ldz);
        const long long r = c / ldz;
        const int j = (int)(r % nxx), k = (int)(r / nxx);
        if (i >= nzz) continue;
        const bool inside = i >= nb && i < nzz - nb && j >= nb && j < nxx - nb && k >= nb && k < nyy - nb;
        if (inside) continue;
        const int ii = min(max(i, nb), nzz - nb - 1);
        const int jj = min(max(j, nb), nxx - nb - 1);
        const int kk = min(max(k, nb), nyy - nb - 1);
        float v = vp[ii + (long long)jj * ldz + (long long)kk * ldz * nxx];
        const int dz = pad_depth(i, nzz, nb), dx = pad_depth(j, nxx, nb), dy = pad_depth(k, nyy, nb);
        const uint64_t cell = (uint64_t)i + (uint64_t)nzz * ((uint64_t)j + (uint64_t)nxx * k);
        const float fnb = (float)nb;
        // every product and sum rounded on its own (no contraction), so that
        // FP32 arithmetic on the host reproduces the pad exactly
        if (kind == 0) {
            if (dx >= 0) v = __fadd_rn(v, __fmul_rn(__fmul_rn(1.0f - dx / fnb, varVp), normal01(seed, 1, cell)));
            if (dy >= 0) v = __fadd_rn(v, __fmul_rn(__fmul_rn(1.0f - dy / fnb, varVp), normal01(seed, 2, cell)));
            if (dz >= 0) v = __fadd_rn(v, __fmul_rn(__fmul_rn(1.0f - dz / fnb, varVp), normal01(seed, 3, cell)));
        } else {
            float ramp = 0.0f;
            if (dx >= 0) ramp = fmaxf(ramp, 1.0f - dx / fnb);
            if (dy >= 0) ramp = fmaxf(ramp, 1.0f - dy / fnb);
            if (dz >= 0) ramp = fmaxf(ramp, 1.0f - dz / fnb);
            const float u = __fsub_rn(__fmul_rn(2.0f, uniform01(seed, 4, cell)), 1.0f);
            v = __fmul_rn(v, __fadd_rn(1.0f, __fmul_rn(__fmul_rn(ratio, ramp), u)));
        }
        vp[c] = fminf(fmaxf(v, vlo), vhi);
    }
}

// Gaussian blobs (random_boundary_gp, src/modeling/modeling.cu:594-615): every
// cell outside the strict inner box visits, in order, the blobs binned near it
// and applies v += s A exp(-|x-c|^2 / (2 r^2)) followed by the clamp.  Blobs
// are truncated at 5 r (the omitted tail is below 4e-6 A).
struct Blob {
    float x, y, z, r, amp;  // centre [m], radius [m], signed amplitude [m/s]
};

__global__ void rbc_blobs_kernel(float *__restrict__ vp, int nzz, int nxx, int nyy, int ldz, int nb,
                                 float dh, const Blob *__restrict__ blobs,
                                 const int *__restrict__ bin_first, const int *__restrict__ bin_list,
                                 int nbz, int nbx, int nby, float bin_size, float vlo, float vhi)
{
    const long long n = (long long)ldz * nxx * nyy;
    const float fnb = nb * dh;
    const float xmax = (nxx - 1) * dh, ymax = (nyy - 1) * dh, zmax = (nzz - 1) * dh;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % ldz);
        const long long r = c / ldz;
        const int j = (int)(r % nxx), k = (int)(r / nxx);
        if (i >= nzz) continue;
        const float X = j * dh, Y = k * dh, Z = i * dh;
        if (X > fnb && X < xmax - fnb && Y > fnb && Y < ymax - fnb && Z > fnb && Z < zmax - fnb)
            continue;
        const int bz = min((int)(Z / bin_size), nbz - 1);
        const int bx = min((int)(X / bin_size), nbx - 1);
        const int by = min((int)(Y / bin_size), nby - 1);
        const int b = bz + nbz * (bx + nbx * by);
        float v = vp[c];
        for (int q = bin_first[b]; q < bin_first[b + 1]; ++q) {
            const Blob bl = blobs[bin_list[q]];
            const float ir = 1.0f / bl.r;
            const float ex = (X - bl.x) * ir, ey = (Y - bl.y) * ir, ez = (Z - bl.z) * ir;
            const float e2 = ex * ex + ey * ey + ez * ez;
            if (e2 > 25.0f) continue;
            v += bl.amp * expf(-0.5f * e2);
            v = fminf(fmaxf(v, vlo), vhi);
        }
        vp[c] = v;
    }
}

// Stencil coefficient dt^2 v^2 / dh^2 of every cell, evaluated as
// (v * v) * cvel exactly as the stencil kernels would, so reading it instead
// of the velocity changes no result bit.
__global__ void coeff_kernel(const float *__restrict__ vp, float *__restrict__ out, long long n, float cvel)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        const float v = vp[c];
        out[c] = v * v * cvel;
    }
}

// Largest |v| in a pitched field restricted to the real cells (CFL check).
__global__ void max_abs_kernel(const float *__restrict__ v, long long n, int ldz, int nzz,
                               unsigned int *__restrict__ out_bits)
{
    float m = 0.0f;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x)
        if ((int)(c % ldz) < nzz) m = fmaxf(m, fabsf(v[c]));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out_bits, __float_as_uint(m));
}

}  // namespace fwi
