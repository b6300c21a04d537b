// device.cuh -- PTX helpers (TMA, mbarrier), constants and argument structs
// shared by the stencil kernels.  sm_100a only.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace fwi {

// 8th-order second-derivative weights, FP32 images of the reference's double
// literals (src/modeling/modeling.cuh:9-13): centre, then taps m = 1..4.
// The operator is  -W0 f0 + W1 (f1+f-1) - W2 (f2+f-2) + W3 (f3+f-3) - W4 (f4+f-4).
constexpr float W0 = 2.847222222222f;
constexpr float W1 = 1.600000000000f;
constexpr float W2 = 0.200000000000f;
constexpr float W3 = 0.025396825396f;
constexpr float W4 = 0.001785714285f;

constexpr int kMaxBatch = 64;      // shots per launch
constexpr int kMaxPad = 1024;      // largest pad width the damper table holds
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s cap on any device wait

// Error bits the kernels raise in g_status (read back by the host).
constexpr unsigned kErrTimeout = 1u;

// Per-batch shot description, device resident so that a captured time loop
// can be replayed for any batch of shots without re-capture.
struct BatchInfo {
    int nshot;                    // shots in this batch
    int R;                        // receivers of all shots together
    int ncell;                    // distinct receiver cells of all shots together
    int pad_;
    int src[kMaxBatch][3];        // source cell (i=z, j=x, k=y), padded indices
};

// Forward step arguments (one leapfrog step of every shot of a batch).
struct FwdArgs {
    int nzz, nxx, nyy, ldz;
    long long vol;                // device elements of one shot's field (pitched)
    int ntz, ntx, ylen;           // z tiles, x tiles, planes per y chunk
    int t, nt, tlag;              // step index, wavelet length, recording lag
    float cvel;                   // dt^2 / dh^2
    float idh3;                   // source / adjoint scaling 1/dh^3
    int nb;                       // pad width (damper tables)
    int vel_slots;                // 1: every shot reads velocity slot 0; B: shot s reads slot s
    float *Q;                     // field written this step (batch base)
    const float *A;               // field read with the stencil (batch base)
    const float *b1d;             // Cerjan 1-D table (ABC only)
    const float *wavelet;         // [nt]
    const BatchInfo *binfo;
    const long long *rec_cell;    // [R] batch-flat cell index of each receiver
    const float *rec_damp;        // [R] damping at the receiver (1 without ABC)
    float *seis_tm;               // [nt][R] time-major seismograms
};

// Fused backward step arguments (source rebuild + adjoint + imaging).
struct BwdArgs {
    int nzz, nxx, nyy, ldz;
    long long vol;
    int ntz, ntx, ylen;
    int t, nt, nsteps;            // backward step index, wavelet length, N = nt + tlag
    float cvel;                   // dt^2 / dh^2
    float gscale;                 // dt / dh^2 (gradient imaging condition)
    float idh3;
    int subtract_src;             // remove the source while rebuilding Ps
    int vel_slots;                // 1: every shot reads velocity slot 0; B: shot s reads slot s
    int acc_z0, acc_z1;           // box [acc_z0, acc_z1) x [acc_x0, acc_x1) x [acc_y0, acc_y1)
    int acc_x0, acc_x1;           // of the cells whose image and illumination accumulate;
    int acc_y0, acc_y1;           // the accumulators of every other cell are neither read nor written
    int acc_zbox;                 // z extent of the accumulator tiles, from z = floor4(max(z0, acc_z0))
    float *Ps;                    // rebuilt source field (written)
    const float *Psold;           // source field read with the stencil
    float *Prold;                 // adjoint field written
    const float *Pr;              // adjoint field read with the stencil
    float *image;                 // image or gradient accumulator (batch base)
    float *illum;                 // illumination accumulator (batch base)
    const float *wavelet;
    const BatchInfo *binfo;
};

// ---------------------------------------------------------------------------
// PTX wrappers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait for phase `parity` of an mbarrier, giving up after limit_ns.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint64_t limit_ns = kWaitLimitNs)
{
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (;;) {
#pragma unroll 1
        for (int i = 0; i < 32; ++i)
            if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > limit_ns) return false;
    }
}

// 4-D tiled TMA load (z, x, y, shot) into shared memory, completing on bar.
// No multicast: every CTA fetches its own tiles from this GPU's memory.
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, uint64_t *bar,
                                            int c0, int c1, int c2, int c3)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5, %6}], [%2];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_addr(bar)), "r"(c0), "r"(c1), "r"(c2),
        "r"(c3)
        : "memory");
}

// 3-D tiled TMA load, completing on bar.  No multicast.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1,
                                            int c2)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_addr(bar)), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}

// 2-D tiled TMA load, completing on bar.  No multicast.
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_addr(bar)), "r"(c0), "r"(c1)
        : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// ---------------------------------------------------------------------------
// tcgen05 (5th-generation tensor core) wrappers, cta_group::1.
// ---------------------------------------------------------------------------
// Tensor-memory allocation by one full warp; the address lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor.  Bit 46 is the tcgen05 descriptor version.
// No swizzle: core matrices are 128 contiguous bytes.  K-major: 8 M/N rows x
// 16 bytes of K; lbo = byte stride between K halves, sbo = byte stride
// between 8-row groups.  MN-major: 8 K rows x 16 bytes of M/N; lbo = byte
// stride between 8-row K groups, sbo = byte stride between 8-element M/N
// groups.
// 32-byte swizzle (the pattern a SWIZZLE_32B TMA load writes: the 16-byte
// half of each 32-byte row flips with address bit 7): rows of 32 bytes.
// K-major (K = 16 BF16 per row): sbo = stride between 8-row groups, lbo
// unused.  MN-major (16 M/N elements per row, K along rows): lbo = stride
// between 16-element M/N groups, sbo = stride between 8-row K groups.
constexpr uint64_t kSwizzleNone = 0, kSwizzle32B = 6;  // layout type, bits 61..63

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo,
                                              uint64_t layout = kSwizzleNone)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46) | (layout << 61);
}

// Instruction descriptor of kind::f16: D FP32, A and B BF16; a_mn / b_mn
// select the MN-major operand layout (bits 15 / 16), K-major otherwise.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int m, int n, bool a_mn = false, bool b_mn = false)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
           ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread.
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// Arrive on bar once every tcgen05 operation this thread issued has completed.
__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_addr(bar))
                 : "memory");
}

// 16 consecutive FP32 columns of the calling thread's TMEM lane; the
// registers are valid after tmem_wait_ld().
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr)
        : "memory");
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Named barrier over `count` threads that also ANDs a predicate across them.
__device__ __forceinline__ bool bar_and(int id, int count, bool pred)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.and.pred q, %2, %3, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)pred), "r"(id), "r"(count)
        : "memory");
    return r != 0;
}

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap *map)
{
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

__device__ __forceinline__ float4 lds4(const float *p) { return *reinterpret_cast<const float4 *>(p); }

__device__ __forceinline__ float comp(const float4 &v, int e)
{
    return e == 0 ? v.x : (e == 1 ? v.y : (e == 2 ? v.z : v.w));
}

__device__ __forceinline__ void set_comp(float4 &v, int e, float s)
{
    if (e == 0) v.x = s;
    else if (e == 1) v.y = s;
    else if (e == 2) v.z = s;
    else v.w = s;
}

// Distance into the pad along one axis, -1 inside (src/modeling/modeling.cu:408-431).
__device__ __forceinline__ int pad_depth(int i, int n, int nb)
{
    return i < nb ? i : (i >= n - nb ? n - 1 - i : -1);
}

// Cerjan factor of a cell from the 1-D table, bit-identical to the reference's
// b2d/b3d tables (src/modeling/modeling.cu:101-127): the 2-D entry is
// (b1[a] + b1[b]) - 1 and the 3-D entry ((B(z,x) + B(x,y)) + B(z,y)) - 5 with
// B(p,q) = b1[p] + b1[q], all in FP32 in that order.
__device__ __forceinline__ float cerjan(const float *b1, int dz, int dx, int dy)
{
    const int n = (dz >= 0) + (dx >= 0) + (dy >= 0);
    if (n == 0) return 1.0f;
    if (n == 1) return b1[dz >= 0 ? dz : (dx >= 0 ? dx : dy)];
    if (n == 2) {
        const int u = dz >= 0 ? dz : dx;
        const int v = dy >= 0 ? dy : dx;
        return __fsub_rn(__fadd_rn(b1[u], b1[v]), 1.0f);
    }
    const float bzx = __fadd_rn(b1[dz], b1[dx]);
    const float bxy = __fadd_rn(b1[dx], b1[dy]);
    const float bzy = __fadd_rn(b1[dz], b1[dy]);
    return __fsub_rn(__fadd_rn(__fadd_rn(bzx, bxy), bzy), 5.0f);
}

}  // namespace fwi
