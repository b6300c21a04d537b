// cnn.cu -- the learned gradient preconditioner (no counterpart in the
// reference): a 4-layer 3-D CNN (3 -> 16 -> 16 -> 16 -> 1 channels, 3^3
// kernels, zero "same" padding, ReLU between layers) that maps the raw
// gradient, the velocity and the illumination of an FWI iteration to a model
// update.  Forward and backward run on BF16 tensor cores with FP32
// accumulation; master weights, Adam moments and the loss are FP32 / FP64.
//
// Layout: activations are BF16 rows of 16 channels (32 bytes, the K of one
// implicit-GEMM tap) over the volume padded by one zero voxel on every side:
// row r = zp + NZ2 (xp + NX2 yp) with NZ2 = nz + 2, NX2 = nx + 2, z fastest
// like the model volumes.  The zero halo is the convolution's "same" padding,
// so the input rows of tap (dz, dx, dy) for output rows r0..r0+127 are the
// contiguous rows r0 + dz + NZ2 dx + NZ2 NX2 dy + (0..127).  Weights are
// [27 taps][16 out][16 in]; tap t = (dz+1) + 3 (dx+1) + 9 (dy+1).
//
// Forward and data-gradient convolutions are tcgen05 kernels (conv_tc_kernel):
// per tile of 128 output rows, TMA brings one 130-row block per (dx, dy) into
// a shared-memory ring, and the three z taps of that block are three
// MMAs whose weights hold the three z taps side by side (N = 48).  The weight
// gradient (wgrad_tc_kernel) is a tcgen05 reduction over rows into tensor
// memory.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "../../include/fwi3d.h"
#include "device.cuh"

namespace {

using fwi::mbar_arrive;
using fwi::mbar_expect_tx;
using fwi::mbar_init;
using fwi::mbar_wait;
using fwi::smem_addr;

constexpr int CH = 16;     // channels per voxel row
constexpr int NL = 4;      // layers
constexpr int TAPS = 27;
constexpr int WSZ = TAPS * CH * CH;  // weights per layer
constexpr int CIN[NL] = {3, 16, 16, 16};
constexpr int kMaxPartials = 1024;  // per-CTA weight-gradient partials held
constexpr int kMaxDevices = 64;     // devices one process can drive
constexpr int COUT[NL] = {16, 16, 16, 1};

// Division by a run-time invariant d (1 <= d < 2^31) of dividends n < 2^31,
// by multiplication (Granlund & Montgomery, "Division by invariant integers
// using multiplication", PLDI 1994): with s = ceil(log2 d) and
// m = floor(2^32 (2^s - d) / d) + 1, n / d = (umulhi(n, m) + n) >> s.
struct FastDiv {
    uint32_t d = 1, m = 1, s = 0;
};

FastDiv make_fastdiv(uint32_t d)
{
    FastDiv f;
    f.d = d;
    while ((1ull << f.s) < d) ++f.s;
    f.m = (uint32_t)(((1ull << 32) * ((1ull << f.s) - d)) / d + 1);
    return f;
}

__device__ __forceinline__ uint32_t fdiv(uint32_t n, const FastDiv &f) { return (__umulhi(n, f.m) + n) >> f.s; }

struct Geo {
    int nz, nx, ny;
    long long V;      // interior voxels
    int NZ2, NX2;     // padded z and x extents
    long long R;      // padded rows (nz+2)(nx+2)(ny+2), below 2^31
    FastDiv fz, fx;   // division by NZ2 and NX2
};

// Interior voxel of padded row r, or -1 on the halo.
__device__ __forceinline__ long long interior_of(const Geo &g, long long r)
{
    const uint32_t rr = (uint32_t)r;
    const uint32_t rest = fdiv(rr, g.fz), yp = fdiv(rest, g.fx);
    const int zp = (int)(rr - rest * (uint32_t)g.NZ2), xp = (int)(rest - yp * (uint32_t)g.NX2);
    if (zp < 1 || zp > g.nz || xp < 1 || xp > g.nx || yp < 1 || (int)yp > g.ny) return -1;
    return (zp - 1) + (long long)g.nz * ((xp - 1) + (long long)g.nx * ((int)yp - 1));
}

__device__ unsigned int g_cnn_status;  // bit 0: a bounded wait gave up

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
    __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&h);
}

// ---------------------------------------------------------------------------
// tcgen05 convolution over all 27 taps.
// SIGN = +1: forward, out[r] = sum_t in[r + off_t] W_t;
// SIGN = -1: data gradient, dx[r] = sum_t dy[r - off_t] W_t^T (w = W transposed).
// MODE 0: BF16 rows with bias and ReLU; 1: BF16 rows times the ReLU mask of
// `mask` (data gradient through the previous activation); 2: FP32 channel 0
// with bias into the unpadded volume (last layer, no activation).  Halo rows
// of BF16 outputs are written as zeros, so every output is again a padded
// input.
//
// A tile is 120 output rows r0..r0+119, four warp segments of 30.  For each
// (dx, dy) one 128-row MMA block (M = 128, N = 48, K = 16 channels) multiplies
// input rows by the weights of the three z taps side by side: column group k
// holds z tap dz = SIGN (k - 1).  Block row 32 q + i (q = 0..3, i = 0..31) is
// input row r0 - 1 + 30 q + i + SIGN (dx NZ2 + dy NZ2 NX2): four 32-row TMA
// segments that overlap by two rows, so that output row r0 + 30 q + j
// (j < 30) only needs accumulator rows 32 q + j .. 32 q + j + 2, all in the
// TMEM lanes of epilogue warp q:
//     out = D[32q+j][group 0] + D[32q+j+1][group 1] + D[32q+j+2][group 2].
// Nine MMAs per tile; the epilogue adds the three groups with warp shuffles.
//
// Tiles stream along y: tile (pos, k) covers rows pos*120 + k*P + m, P = NZ2
// NX2 the rows of one y plane, m < 120 and pos*120 + m < P.  Its nine blocks
// are three x offsets in each of the planes k-1, k, k+1, so a CTA walking k
// upwards loads one new plane (three TMA copies) per tile and keeps the other
// two in a ring of PS plane slots, like the stencil kernels' y queue.  Each
// CTA owns a contiguous range of tiles in (pos, k) order; a run restarts the
// plane stream where pos changes.
//
// Warp 0 issues the TMA loads, warp 1 allocates tensor memory and issues the
// MMAs, warps 2..5 drain the accumulators (warp w reads TMEM lanes 32 (w%4)..).
// Two accumulators alternate, so the epilogue of one tile overlaps the MMAs of
// the next, and three CTAs share an SM's tensor pipe.  Every wait is bounded;
// a wait that gives up sets g_cnn_status, and the kernel drains its copies and
// MMAs, frees its tensor memory and returns.
// ---------------------------------------------------------------------------
namespace tc {
constexpr int BM = 128;                       // rows per MMA block (M)
constexpr int SEG = 32;                       // rows per TMA segment = TMEM lanes per epilogue warp
constexpr int OSEG = SEG - 2;                 // output rows per segment
constexpr int TM = 4 * OSEG;                  // output rows per tile
constexpr int BLK = BM * CH * 2;              // one block: 128 swizzled 32-byte rows
constexpr int PSLOT = 3 * BLK;                // one plane: blocks for x offsets -1, 0, +1
constexpr int PS = 4;                         // plane slots (a tile reads 3)
constexpr int NG = 3 * CH;                    // MMA N: (z tap, channel)
constexpr int BJ = NG * CH * 2;               // bytes of the B operand of one (dx, dy)
constexpr int WBYTES = 9 * BJ;
constexpr int THREADS = 192;
constexpr int CTAS_PER_SM = 3;
constexpr uint32_t ACC_STRIDE = 64;           // TMEM columns between the two accumulators
constexpr uint32_t TMEM_COLS = 128;
constexpr uint32_t LOAD_BYTES = PSLOT;
constexpr int BAR_BYTES = (2 * PS + 5) * 8;
constexpr int SMEM = PS * PSLOT + WBYTES + BAR_BYTES + 16 + CH * 4;
constexpr uint32_t IDESC = fwi::umma_idesc_bf16(BM, NG);
static_assert(PS >= 4 && PS < 32, "plane slots");
static_assert(4 * SEG == BM, "four segments per block");
static_assert(NG <= (int)ACC_STRIDE, "accumulator columns");
}  // namespace tc

struct ConvArgs {
    Geo g;
    long long P;                // rows of one y plane, NZ2 * NX2
    int ny2;                    // y planes, ny + 2
    int ntiles;                 // tiles: ceil(P / 126) positions x ny2 planes
    int tiles_per_cta;
    const __nv_bfloat16 *w;     // [27][16 n][16 k]: B operand rows n, K = k
    const float *bias;          // [16] (MODE 0, 2)
    const __nv_bfloat16 *mask;  // padded rows (MODE 1)
    __nv_bfloat16 *out;         // padded rows (MODE 0, 1)
    float *out32;               // unpadded volume (MODE 2)
};

__device__ __forceinline__ void cnn_fail(volatile int *abort_flag)
{
    *abort_flag = 1;
    atomicOr(&g_cnn_status, 1u);
}

template <int SIGN, int MODE>
__global__ void __launch_bounds__(tc::THREADS, tc::CTAS_PER_SM)
    conv_tc_kernel(const __grid_constant__ CUtensorMap map, const ConvArgs a)
{
    using namespace tc;
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *ring = smem;
    unsigned char *wsm = smem + PS * PSLOT;
    uint64_t *full = reinterpret_cast<uint64_t *>(wsm + WBYTES);
    uint64_t *empty = full + PS;
    uint64_t *accf = empty + PS;  // [2] accumulator ready
    uint64_t *acce = accf + 2;    // [2] accumulator drained
    uint64_t *done = acce + 2;    // every MMA of this CTA completed
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);
    float *bsm = reinterpret_cast<float *>(wsm + WBYTES + BAR_BYTES + 16);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if ((smem_addr(smem) & 127u) != 0u) {  // TMA destinations need 128-byte alignment
        if (threadIdx.x == 0) atomicOr(&g_cnn_status, 2u);
        return;
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < PS; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&accf[b], 1);
            mbar_init(&acce[b], 4);
        }
        mbar_init(done, 1);
        *abort_flag = 0;
        fwi::fence_mbar_init();
    }
    // B operand of (dx, dy) = j: rows n = 16 k + c_out, k = z-tap group, from
    // w[t][c_out][:] with t = (dz+1) + 3 (dx+1) + 9 (dy+1), dz = SIGN (k-1);
    // stored [j][K half][n][8]: K-major core matrices of 8 rows x 16 bytes,
    // the two K halves NG*16 bytes apart
    for (int i = threadIdx.x; i < 9 * NG * 2; i += blockDim.x) {
        const int j = i / (NG * 2), n = (i >> 1) % NG, c = i & 1;
        const int k = n / CH, co = n % CH;
        const int dz = SIGN * (k - 1), dx = j % 3 - 1, dy = j / 3 - 1;
        const int t = (dz + 1) + 3 * (dx + 1) + 9 * (dy + 1);
        const uint4 v = *reinterpret_cast<const uint4 *>(a.w + (t * CH + co) * CH + c * 8);
        *reinterpret_cast<uint4 *>(wsm + j * BJ + c * (NG * 16) + n * 16) = v;
    }
    if (threadIdx.x < CH) bsm[threadIdx.x] = a.bias ? a.bias[threadIdx.x] : 0.0f;
    fwi::fence_proxy_async();  // the tensor core reads what the threads wrote
    if (warp == 1) fwi::tmem_alloc(tmem_slot, TMEM_COLS);
    fwi::tc_fence_before();
    __syncthreads();
    fwi::tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const int T0 = blockIdx.x * a.tiles_per_cta;
    const int T1 = min(T0 + a.tiles_per_cta, a.ntiles);

    if (warp == 0) {
        if (lane == 0) {
            // producer: plane k' of a run = three 128-row blocks at x offsets
            // -1, 0, +1; rows outside the tensor read as zeros
            fwi::prefetch_tmap(&map);
            uint32_t used = 0, phases = 0;
            unsigned g = 0;  // planes issued
            bool stop = false;
            for (int T = T0; T < T1 && !stop;) {
                const int pos = T / a.ny2, ks = T % a.ny2;
                const int te = min(T1, (pos + 1) * a.ny2);
                const long long rb = (long long)pos * TM - 1;
                for (int j = 0; j < te - T + 2; ++j, ++g) {
                    const int slot = (int)(g % PS);
                    const uint32_t ph = (g / PS) & 1u;
                    if (*abort_flag || !mbar_wait(&empty[slot], ph ^ 1u)) {
                        cnn_fail(abort_flag);
                        stop = true;
                        break;
                    }
                    mbar_expect_tx(&full[slot], LOAD_BYTES);
                    const long long r = rb + (long long)(ks - 1 + j) * a.P;
#pragma unroll
                    for (int bx = 0; bx < 3; ++bx)
#pragma unroll
                        for (int sg = 0; sg < 4; ++sg)
                            fwi::tma_load_2d(ring + slot * PSLOT + bx * BLK + sg * SEG * CH * 2, &map, &full[slot],
                                             0, (int)(r + (bx - 1) * (long long)a.g.NZ2 + sg * OSEG));
                    used |= 1u << slot;
                    phases = (phases & ~(1u << slot)) | (ph << slot);
                }
                T = te;
            }
            // no copy may land after the CTA has gone
            for (int s = 0; s < PS; ++s)
                if ((used >> s) & 1u)
                    if (!mbar_wait(&full[s], (phases >> s) & 1u)) atomicOr(&g_cnn_status, 1u);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // MMA issuer
            const uint32_t ring_a = smem_addr(ring), w_a = smem_addr(wsm);
            unsigned g = 0;  // planes consumed
            int it = 0;
            bool stop = false;
            for (int T = T0; T < T1 && !stop;) {
                const int pos = T / a.ny2;
                const int te = min(T1, (pos + 1) * a.ny2);
                const int n = te - T;
                for (int i = 0; i < n; ++i, ++it) {
                    const int buf = it & 1;
                    bool ok = !*abort_flag && mbar_wait(&acce[buf], (((uint32_t)it >> 1) & 1u) ^ 1u);
                    // planes i, i+1, i+2 of the run (i, i+1 already waited unless i == 0)
                    for (int jp = (i == 0 ? 0 : 2); ok && jp <= 2; ++jp) {
                        const unsigned pl = g + i + jp;
                        ok = mbar_wait(&full[pl % PS], (pl / PS) & 1u);
                    }
                    if (!ok) {
                        cnn_fail(abort_flag);
                        stop = true;
                        break;
                    }
                    fwi::tc_fence_after();
                    const uint32_t d = tmem + (uint32_t)buf * ACC_STRIDE;
#pragma unroll
                    for (int j = 0; j < 9; ++j) {
                        const int dx = j % 3 - 1, dy = j / 3 - 1;
                        const unsigned pl = g + i + 1 + SIGN * dy;
                        const uint32_t blk = ring_a + (pl % PS) * PSLOT + (1 + SIGN * dx) * BLK;
                        const uint64_t ad = fwi::umma_desc(blk, 16, 256, fwi::kSwizzle32B);
                        const uint64_t bd = fwi::umma_desc(w_a + j * BJ, NG * 16, 128);
                        fwi::umma_bf16(d, ad, bd, IDESC, j > 0 ? 1u : 0u);
                    }
                    fwi::umma_commit(&accf[buf]);
                    // plane i is not read again; at the end of the run neither are i+1, i+2
                    fwi::umma_commit(&empty[(g + i) % PS]);
                    if (i == n - 1) {
                        fwi::umma_commit(&empty[(g + i + 1) % PS]);
                        fwi::umma_commit(&empty[(g + i + 2) % PS]);
                    }
                }
                g += n + 2;
                T = te;
            }
            fwi::umma_commit(done);
            if (!mbar_wait(done, 0)) atomicOr(&g_cnn_status, 1u);
        }
    } else {
        // epilogue: warp q drains TMEM lanes 32 q .. 32 q + 31 and writes
        // output rows 30 q .. 30 q + 29 of the tile; waits and exits are
        // warp-uniform (tcgen05.ld is warp-collective)
        const int q = warp & 3;
        int it = 0;
        for (int T = T0; T < T1; ++T, ++it) {
            const int buf = it & 1;
            bool ok = *abort_flag == 0 && mbar_wait(&accf[buf], ((uint32_t)it >> 1) & 1u);
            if (!__all_sync(0xffffffffu, ok)) {
                if (lane == 0) cnn_fail(abort_flag);
                break;
            }
            fwi::tc_fence_after();
            uint32_t v0[16], v1[16], v2[16];
            const uint32_t t0 = tmem + (uint32_t)buf * ACC_STRIDE + ((uint32_t)(32 * q) << 16);
            fwi::tmem_ld16(t0, v0);
            fwi::tmem_ld16(t0 + CH, v1);
            fwi::tmem_ld16(t0 + 2 * CH, v2);
            fwi::tmem_wait_ld();
            fwi::tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acce[buf]);
            // output row j = lane: group 0 of lane j, group 1 of lane j+1, group 2 of lane j+2
            float o[CH];
#pragma unroll
            for (int c = 0; c < CH; ++c) {
                const float b1 = __shfl_down_sync(0xffffffffu, __uint_as_float(v1[c]), 1);
                const float b2 = __shfl_down_sync(0xffffffffu, __uint_as_float(v2[c]), 2);
                o[c] = (__uint_as_float(v0[c]) + b1) + b2;
            }
            const int pos = T / a.ny2, k = T % a.ny2;
            const long long zx = (long long)pos * TM + OSEG * q + lane;  // row within the y plane
            if (lane >= OSEG || zx >= a.P) continue;
            const long long r = zx + (long long)k * a.P;
            const long long vox = interior_of(a.g, r);
            if constexpr (MODE == 2) {
                if (vox >= 0) a.out32[vox] = o[0] + bsm[0];
            } else {
                uint32_t pk[8];
                if (vox < 0) {
#pragma unroll
                    for (int c = 0; c < 8; ++c) pk[c] = 0u;
                } else {
                    uint32_t mk[8];
                    if constexpr (MODE == 1) {
                        const uint4 m0 = reinterpret_cast<const uint4 *>(a.mask + r * CH)[0];
                        const uint4 m1 = reinterpret_cast<const uint4 *>(a.mask + r * CH)[1];
                        mk[0] = m0.x; mk[1] = m0.y; mk[2] = m0.z; mk[3] = m0.w;
                        mk[4] = m1.x; mk[5] = m1.y; mk[6] = m1.z; mk[7] = m1.w;
                    }
#pragma unroll
                    for (int c = 0; c < 8; ++c) {
                        float x0 = o[2 * c], x1 = o[2 * c + 1];
                        if constexpr (MODE == 0) {
                            x0 = fmaxf(x0 + bsm[2 * c], 0.0f);
                            x1 = fmaxf(x1 + bsm[2 * c + 1], 0.0f);
                        } else {
                            __nv_bfloat162 mm;
                            *reinterpret_cast<uint32_t *>(&mm) = mk[c];
                            if (!(__bfloat162float(mm.x) > 0.0f)) x0 = 0.0f;
                            if (!(__bfloat162float(mm.y) > 0.0f)) x1 = 0.0f;
                        }
                        pk[c] = pack_bf16(x0, x1);
                    }
                }
                uint4 *dst = reinterpret_cast<uint4 *>(a.out + r * CH);
                dst[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                dst[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
            }
        }
    }
    fwi::tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        fwi::tc_fence_after();
        fwi::tmem_dealloc(tmem, TMEM_COLS);
    }
}

// ---------------------------------------------------------------------------
// tcgen05 weight gradient.
//   dW[t][co][ci] = sum_v dy[v][co] x[v + off_t][ci]
//                 = sum_u dy[u - dz][co] x[u + NZ2 dx + NZ2 NX2 dy][ci]   (u = v + dz)
// over every padded row (halo rows of dy are zero).  Rows are addressed as
// (row within a y plane, plane) through 3-D tensor maps of extent (P, ny+2),
// P = NZ2 NX2, so that a 128-row block never runs into the next plane (rows
// past P read as zeros) and every u is counted once.
//
// Blocks of u stream along y like the convolution's tiles: block (pos, k) is
// rows pos*128 .. pos*128+127 of plane k, and a CTA owns a contiguous range of
// blocks in (pos, k) order.  The x rows of block k come from planes k-1, k,
// k+1 (dy = -1, 0, +1), each plane three blocks at x offsets -1, 0, +1, held
// in a ring of plane slots: one new plane per block.  Per block, TMA also
// brings the dy rows shifted by dz = -1, 0, +1.  All operands are 32-byte
// swizzled rows, MN-major with K = the row.
//   - A (per plane dy): [x block dx=-1][dx=0][dx=+1][ones in channel 0] and
//     four more blocks of whatever follows in shared memory, whose rows are not
//     used: M rows 16 (dx+1) + ci, and row 48 = the ones.
//   - B: the three dy blocks side by side (N = 3 dz x 16 co).
// Each 16-row K step is three MMAs (M = 128, N = 48, K = 16), one per plane,
// into three accumulators that live in tensor memory for the CTA's whole
// range.  Row 48 of the dy = 0 accumulator against the dz = 0 columns is
// sum_u dy[u][co], the bias gradient.  The epilogue writes per-CTA partials
// [cta][27][16 co][16 ci] and [cta][16], summed in a fixed order by
// reduce_partials_kernel.
// ---------------------------------------------------------------------------
namespace wg {
constexpr int BK = 128;                        // rows of u per block (K)
constexpr int BLK = BK * CH * 2;               // one block: 128 swizzled 32-byte rows
constexpr int PSLOT = 4 * BLK;                 // plane slot: x blocks dx = -1, 0, +1 and the ones block
constexpr int PS = 4;                          // plane slots (a block reads 3)
constexpr int TAIL = 4 * BLK;                  // read, never used, by the last slot's MMA (M spans 8 blocks)
constexpr int DSTAGE = 3 * BLK;                // dy blocks dz = -1, 0, +1
constexpr int ND = 2;                          // dy stages
constexpr int OFF_DY = PS * PSLOT + TAIL;
constexpr int THREADS = 192;
constexpr int CTAS_PER_SM = 2;
constexpr int NG = 3 * CH;                     // MMA N: (z tap, c_out)
constexpr uint32_t TMEM_COLS = 256;            // three 48-column accumulators
constexpr int BAR_BYTES = (2 * PS + 2 * ND + 1) * 8;
constexpr int SMEM = OFF_DY + ND * DSTAGE + BAR_BYTES + 16;
constexpr uint32_t IDESC = fwi::umma_idesc_bf16(128, NG, true, true);
static_assert(PSLOT % 1024 == 0 && DSTAGE % 1024 == 0, "swizzle atom alignment");
static_assert(3 * NG <= (int)TMEM_COLS, "accumulator columns");
static_assert(PS >= 4 && PS < 32 && ND < 32, "slot bitmasks");
}  // namespace wg

struct WgradArgs {
    Geo g;
    int ny2;           // y planes
    int ntiles;        // blocks of u: ceil(P / 128) positions x ny2 planes
    int tiles_per_cta;
    float *partial;    // [gridDim.x][27][16][16]
    float *bpartial;   // [gridDim.x][16]
};

__global__ void __launch_bounds__(wg::THREADS, wg::CTAS_PER_SM)
    wgrad_tc_kernel(const __grid_constant__ CUtensorMap mx, const __grid_constant__ CUtensorMap mdy,
                    const WgradArgs a)
{
    using namespace wg;
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *ring = smem;
    unsigned char *dyb = smem + OFF_DY;
    uint64_t *pfull = reinterpret_cast<uint64_t *>(smem + OFF_DY + ND * DSTAGE);
    uint64_t *pempty = pfull + PS;
    uint64_t *dfull = pempty + PS;
    uint64_t *dempty = dfull + ND;
    uint64_t *done = dempty + ND;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if ((smem_addr(smem) & 127u) != 0u) {
        if (threadIdx.x == 0) atomicOr(&g_cnn_status, 2u);
        return;
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < PS; ++s) {
            mbar_init(&pfull[s], 1);
            mbar_init(&pempty[s], 1);
        }
        for (int s = 0; s < ND; ++s) {
            mbar_init(&dfull[s], 1);
            mbar_init(&dempty[s], 1);
        }
        mbar_init(done, 1);
        *abort_flag = 0;
        fwi::fence_mbar_init();
    }
    // the ones block of every plane slot: channel 0 = 1 in every row.  In the
    // 32-byte swizzle, the 16-byte half h of row r sits at half h ^ (r/4 % 2).
    for (int i = threadIdx.x; i < PS * BK * 2; i += blockDim.x) {
        const int sl = i / (BK * 2), r = (i >> 1) % BK, h = i & 1;
        const int logical = h ^ ((r >> 2) & 1);
        const uint4 v = make_uint4(logical == 0 ? 0x3F80u : 0u, 0u, 0u, 0u);  // BF16 1.0 in channel 0
        *reinterpret_cast<uint4 *>(ring + sl * PSLOT + 3 * BLK + r * 32 + h * 16) = v;
    }
    fwi::fence_proxy_async();
    if (warp == 1) fwi::tmem_alloc(tmem_slot, TMEM_COLS);
    fwi::tc_fence_before();
    __syncthreads();
    fwi::tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const int T0 = blockIdx.x * a.tiles_per_cta;
    const int T1 = min(T0 + a.tiles_per_cta, a.ntiles);

    if (warp == 0) {
        if (lane == 0) {
            fwi::prefetch_tmap(&mx);
            fwi::prefetch_tmap(&mdy);
            uint32_t pused = 0, pph = 0, dused = 0, dph = 0;
            unsigned g = 0, d = 0;  // planes and dy stages issued
            bool stop = false;
            auto issue_plane = [&](int pos, int kp) {
                const int slot = (int)(g % PS);
                const uint32_t ph = (g / PS) & 1u;
                if (*abort_flag || !mbar_wait(&pempty[slot], ph ^ 1u)) return false;
                mbar_expect_tx(&pfull[slot], 3 * BLK);
#pragma unroll
                for (int bx = 0; bx < 3; ++bx)
                    fwi::tma_load_3d(ring + slot * PSLOT + bx * BLK, &mx, &pfull[slot], 0,
                                     pos * BK + (bx - 1) * a.g.NZ2, kp);
                pused |= 1u << slot;
                pph = (pph & ~(1u << slot)) | (ph << slot);
                ++g;
                return true;
            };
            auto issue_dy = [&](int pos, int k) {
                const int st = (int)(d % ND);
                const uint32_t ph = (d / ND) & 1u;
                if (*abort_flag || !mbar_wait(&dempty[st], ph ^ 1u)) return false;
                mbar_expect_tx(&dfull[st], DSTAGE);
#pragma unroll
                for (int kk = 0; kk < 3; ++kk)  // dy rows u - dz, dz = kk - 1
                    fwi::tma_load_3d(dyb + st * DSTAGE + kk * BLK, &mdy, &dfull[st], 0, pos * BK - (kk - 1), k);
                dused |= 1u << st;
                dph = (dph & ~(1u << st)) | (ph << st);
                ++d;
                return true;
            };
            for (int T = T0; T < T1 && !stop;) {
                const int pos = T / a.ny2, ks = T % a.ny2;
                const int te = min(T1, (pos + 1) * a.ny2);
                stop = !issue_plane(pos, ks - 1) || !issue_plane(pos, ks);
                for (int i = 0; i < te - T && !stop; ++i)
                    stop = !issue_plane(pos, ks + i + 1) || !issue_dy(pos, ks + i);
                T = te;
            }
            if (stop) cnn_fail(abort_flag);
            // no copy may land after the CTA has gone
            for (int s = 0; s < PS; ++s)
                if ((pused >> s) & 1u)
                    if (!mbar_wait(&pfull[s], (pph >> s) & 1u)) atomicOr(&g_cnn_status, 1u);
            for (int s = 0; s < ND; ++s)
                if ((dused >> s) & 1u)
                    if (!mbar_wait(&dfull[s], (dph >> s) & 1u)) atomicOr(&g_cnn_status, 1u);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t ring_a = smem_addr(ring), dy_a = smem_addr(dyb);
            unsigned g = 0, d = 0;
            bool first = true, stop = false;
            for (int T = T0; T < T1 && !stop;) {
                const int pos = T / a.ny2;
                const int te = min(T1, (pos + 1) * a.ny2);
                const int n = te - T;
                for (int i = 0; i < n; ++i, ++d) {
                    // planes i, i+1, i+2 of the run (i, i+1 already waited unless i == 0)
                    bool ok = !*abort_flag;
                    for (int jp = (i == 0 ? 0 : 2); ok && jp <= 2; ++jp) {
                        const unsigned pl = g + i + jp;
                        ok = mbar_wait(&pfull[pl % PS], (pl / PS) & 1u);
                    }
                    const int st = (int)(d % ND);
                    ok = ok && mbar_wait(&dfull[st], (d / ND) & 1u);
                    if (!ok) {
                        cnn_fail(abort_flag);
                        stop = true;
                        break;
                    }
                    fwi::tc_fence_after();
#pragma unroll 1
                    for (int s = 0; s < BK / 16; ++s) {
                        const uint32_t koff = s * 512;  // 16 rows of 32 bytes
                        const uint64_t bd =
                            fwi::umma_desc(dy_a + st * DSTAGE + koff, BLK, 256, fwi::kSwizzle32B);
#pragma unroll
                        for (int p = 0; p < 3; ++p) {  // plane k - 1 + p, i.e. dy = p - 1
                            const unsigned pl = g + i + p;
                            const uint64_t ad =
                                fwi::umma_desc(ring_a + (pl % PS) * PSLOT + koff, BLK, 256, fwi::kSwizzle32B);
                            fwi::umma_bf16(tmem + (uint32_t)(p * NG), ad, bd, IDESC, (first && s == 0) ? 0u : 1u);
                        }
                    }
                    first = false;
                    fwi::umma_commit(&dempty[st]);
                    // plane i is not read again; at the end of the run neither are i+1, i+2
                    fwi::umma_commit(&pempty[(g + i) % PS]);
                    if (i == n - 1) {
                        fwi::umma_commit(&pempty[(g + i + 1) % PS]);
                        fwi::umma_commit(&pempty[(g + i + 2) % PS]);
                    }
                }
                g += n + 2;
                T = te;
            }
            fwi::umma_commit(done);
        }
    } else {
        // epilogue: wait for the last MMA, then TMEM lanes 32 q .. 32 q + 31
        const int q = warp & 3;
        const bool ok = __all_sync(0xffffffffu, mbar_wait(done, 0));
        if (ok) {
            fwi::tc_fence_after();
            const bool empty_range = T0 >= T1;
            const int m = 32 * q + lane;  // accumulator row: 16 (dx+1) + ci, or 48 for the ones
            float *P = a.partial + (long long)blockIdx.x * WSZ;
#pragma unroll 1
            for (int acc = 0; acc < 9; ++acc) {
                // plane p = acc / 3 (dy = p - 1), columns of z tap dz = acc % 3 - 1
                uint32_t v[16];
                fwi::tmem_ld16(tmem + (uint32_t)acc * CH + ((uint32_t)(32 * q) << 16), v);
                fwi::tmem_wait_ld();
                const int p = acc / 3, dz = acc % 3 - 1;
                if (m < NG) {
                    const int dx = m / CH - 1, ci = m % CH;
                    const int t = (dz + 1) + 3 * (dx + 1) + 9 * p;
#pragma unroll
                    for (int co = 0; co < CH; ++co)
                        P[(t * CH + co) * CH + ci] = empty_range ? 0.0f : __uint_as_float(v[co]);
                } else if (m == NG && p == 1 && dz == 0) {
#pragma unroll
                    for (int co = 0; co < CH; ++co)
                        a.bpartial[(long long)blockIdx.x * CH + co] = empty_range ? 0.0f : __uint_as_float(v[co]);
                }
            }
        } else if (lane == 0) {
            cnn_fail(abort_flag);
        }
    }
    fwi::tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        fwi::tc_fence_after();
        fwi::tmem_dealloc(tmem, TMEM_COLS);
    }
}

// Fixed-order sum of per-CTA partials: out[i] = sum_b part[b][i].  A block
// is 32 entries x 8 slices of b; slice y sums b = y, y+8, ... in order, then
// the eight slice sums are added in order.
constexpr int RED_X = 32, RED_Y = 8;

__global__ void __launch_bounds__(RED_X * RED_Y)
    reduce_partials_kernel(const float *__restrict__ part, int nb, int n, float *__restrict__ out)
{
    __shared__ float red[RED_Y][RED_X];
    const int x = threadIdx.x % RED_X, y = threadIdx.x / RED_X;
    const int i = blockIdx.x * RED_X + x;
    float s = 0.0f;
    if (i < n)
        for (int b = y; b < nb; b += RED_Y) s += part[(long long)b * n + i];
    red[y][x] = s;
    __syncthreads();
    if (y == 0 && i < n) {
        float t = red[0][x];
        for (int k = 1; k < RED_Y; ++k) t += red[k][x];
        out[i] = t;
    }
}

// Pack three FP32 channel volumes into the BF16 input rows (zero halo).
__global__ void pack_input_kernel(Geo g, const float *__restrict__ c0, const float *__restrict__ c1,
                                  const float *__restrict__ c2, __nv_bfloat16 *__restrict__ out)
{
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < g.R; r += (long long)gridDim.x * blockDim.x) {
        const long long v = interior_of(g, r);
        uint4 r0 = make_uint4(0u, 0u, 0u, 0u);
        if (v >= 0) {
            r0.x = pack_bf16(c0[v], c1[v]);
            r0.y = pack_bf16(c2[v], 0.0f);
        }
        reinterpret_cast<uint4 *>(out + r * CH)[0] = r0;
        reinterpret_cast<uint4 *>(out + r * CH)[1] = make_uint4(0u, 0u, 0u, 0u);
    }
}

// Loss 0.5 * mean (pred - target)^2 (FP64 partials) and its gradient, scaled
// by `gscale`, into channel 0 of BF16 rows (zero halo).
__global__ void mse_kernel(Geo g, const float *__restrict__ pred, const float *__restrict__ target,
                           float gscale, __nv_bfloat16 *__restrict__ grad, double *__restrict__ partial)
{
    __shared__ double red[8];
    double acc = 0.0;
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < g.R; r += (long long)gridDim.x * blockDim.x) {
        const long long v = interior_of(g, r);
        uint4 r0 = make_uint4(0u, 0u, 0u, 0u);
        if (v >= 0) {
            const float d = pred[v] - target[v];
            acc += (double)d * d;
            r0.x = pack_bf16(d * gscale, 0.0f);
        }
        reinterpret_cast<uint4 *>(grad + r * CH)[0] = r0;
        reinterpret_cast<uint4 *>(grad + r * CH)[1] = make_uint4(0u, 0u, 0u, 0u);
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

// One warp: lane l sums p[l], p[l+32], ... in order, then a fixed shuffle tree.
__global__ void sum_f64_kernel(const double *__restrict__ p, int n, double *__restrict__ out)
{
    if (blockIdx.x != 0 || threadIdx.x >= 32) return;
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += 32) s += p[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) *out = s;
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

// Rows map over a padded BF16 activation buffer: (16 channels, row), box of
// `box_rows` whole 32-byte rows, 32-byte swizzle (the SW32 operand layout of
// the tensor-core descriptors).  Rows outside [0, R) read as zeros.
// The driver's tensor-map encoder, looked up once.
PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess && p)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    }
    return fn;
}

int rows_map(fwi_cnn *n, const __nv_bfloat16 *base, int box_rows, CUtensorMap *m)
{
    const PFN_cuTensorMapEncodeTiled_v12000 fn = tmap_encoder();
    if (!fn) {
        n->err = "cuTensorMapEncodeTiled unavailable";
        return FWI_ERR_CUDA;
    }
    cuuint64_t dims[2] = {CH, (cuuint64_t)n->g.R};
    cuuint64_t strides[1] = {CH * 2};
    cuuint32_t box[2] = {CH, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void *)base, dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        n->err = "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")";
        return FWI_ERR_CUDA;
    }
    return FWI_OK;
}

// Plane map over a padded BF16 activation buffer: (16 channels, row within a
// y plane, plane) with extents (16, NZ2 NX2, ny + 2), box (16, 128, 1),
// 32-byte swizzle.  Rows past the end of a plane, and planes outside the
// volume, read as zeros.
int plane_map(fwi_cnn *n, const __nv_bfloat16 *base, CUtensorMap *m)
{
    const PFN_cuTensorMapEncodeTiled_v12000 fn = tmap_encoder();
    if (!fn) {
        n->err = "cuTensorMapEncodeTiled unavailable";
        return FWI_ERR_CUDA;
    }
    const cuuint64_t P = (cuuint64_t)n->g.NZ2 * n->g.NX2;
    cuuint64_t dims[3] = {CH, P, (cuuint64_t)(n->g.ny + 2)};
    cuuint64_t strides[2] = {CH * 2, P * CH * 2};
    cuuint32_t box[3] = {CH, (cuuint32_t)wg::BK, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, (void *)base, dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        n->err = "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")";
        return FWI_ERR_CUDA;
    }
    return FWI_OK;
}

// CTAs of a persistent tensor-core kernel that are resident at once: per SM
// the fewest of `want`, what shared memory holds and what tensor memory (512
// columns) holds.
int resident_ctas(fwi_cnn *n, int smem_bytes, uint32_t tmem_cols, int want)
{
    int dev = 0, sms = 0, smem_sm = 0, reserved = 0;
    CNN_CK(cudaGetDevice(&dev));
    CNN_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CNN_CK(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    CNN_CK(cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev));
    int per_sm = std::min(want, smem_sm / (smem_bytes + reserved));
    per_sm = std::min(per_sm, (int)(512u / tmem_cols));
    return sms * std::max(per_sm, 1);
}

template <int SIGN, int MODE>
int launch_conv(fwi_cnn *n, const __nv_bfloat16 *in, const __nv_bfloat16 *w, const float *bias,
                const __nv_bfloat16 *mask, __nv_bfloat16 *out, float *out32)
{
    // kernel attributes are per device: set them, and size the grid, once per
    // device; host threads that drive the same device take the lock first
    static int ctas_of[kMaxDevices] = {};
    static std::mutex lock_of[kMaxDevices];
    int dev = 0;
    CNN_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        n->err = "device ordinal beyond the supported count";
        return FWI_ERR_ARG;
    }
    int ctas = 0;  // resident CTAs on the whole GPU
    {
        std::lock_guard<std::mutex> guard(lock_of[dev]);
        if (!ctas_of[dev]) {
        CNN_CK(cudaFuncSetAttribute(conv_tc_kernel<SIGN, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    tc::SMEM));
        // the whole unified L1 as shared memory, so that four CTAs fit
        CNN_CK(cudaFuncSetAttribute(conv_tc_kernel<SIGN, MODE>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                    (int)cudaSharedmemCarveoutMaxShared));
            const int c = resident_ctas(n, tc::SMEM, tc::TMEM_COLS, tc::CTAS_PER_SM);
            if (c <= 0) return FWI_ERR_CUDA;
            ctas_of[dev] = c;
        }
        ctas = ctas_of[dev];
    }
    CUtensorMap m;
    const int st = rows_map(n, in, tc::SEG, &m);
    if (st != FWI_OK) return st;
    const long long P = (long long)n->g.NZ2 * n->g.NX2;
    const int ny2 = n->g.ny + 2;
    const int ntiles = (int)((P + tc::TM - 1) / tc::TM) * ny2;
    const int tpc = (ntiles + ctas - 1) / ctas;
    ConvArgs a{n->g, P, ny2, ntiles, tpc, w, bias, mask, out, out32};
    const int blocks = (ntiles + tpc - 1) / tpc;
    conv_tc_kernel<SIGN, MODE><<<blocks, tc::THREADS, tc::SMEM, n->stream>>>(m, a);
    CNN_CK(cudaGetLastError());
    return FWI_OK;
}

int forward_impl(fwi_cnn *n)
{
    for (int l = 0; l < NL; ++l) {
        const int st = l < NL - 1
                           ? launch_conv<1, 0>(n, n->act[l].p, n->wb[l].p, n->b32[l].p, nullptr, n->act[l + 1].p,
                                               nullptr)
                           : launch_conv<1, 2>(n, n->act[l].p, n->wb[l].p, n->b32[l].p, nullptr, nullptr,
                                               n->pred.p);
        if (st != FWI_OK) return st;
    }
    return FWI_OK;
}

// Weight and bias gradients of one layer into gw / gb: x = the layer's input
// rows, dy = the gradient rows of its output.
int launch_wgrad(fwi_cnn *n, const __nv_bfloat16 *x, const __nv_bfloat16 *dy, float *gw, float *gb)
{
    static int ctas_of[kMaxDevices] = {};  // per device, under a lock, as in launch_conv
    static std::mutex lock_of[kMaxDevices];
    int dev = 0;
    CNN_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        n->err = "device ordinal beyond the supported count";
        return FWI_ERR_ARG;
    }
    int ctas = 0;
    {
        std::lock_guard<std::mutex> guard(lock_of[dev]);
        if (!ctas_of[dev]) {
            CNN_CK(cudaFuncSetAttribute(wgrad_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, wg::SMEM));
            CNN_CK(cudaFuncSetAttribute(wgrad_tc_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                        (int)cudaSharedmemCarveoutMaxShared));
            const int c = std::min(resident_ctas(n, wg::SMEM, wg::TMEM_COLS, wg::CTAS_PER_SM), kMaxPartials);
            if (c <= 0) return FWI_ERR_CUDA;
            ctas_of[dev] = c;
        }
        ctas = ctas_of[dev];
    }
    CUtensorMap mx, mdy;
    int st = plane_map(n, x, &mx);
    if (st == FWI_OK) st = plane_map(n, dy, &mdy);
    if (st != FWI_OK) return st;
    const long long P = (long long)n->g.NZ2 * n->g.NX2;
    const int ny2 = n->g.ny + 2;
    WgradArgs a{n->g, ny2, (int)((P + wg::BK - 1) / wg::BK) * ny2, 0, n->partial.p, n->bpartial.p};
    a.tiles_per_cta = (a.ntiles + ctas - 1) / ctas;
    const int grid = (a.ntiles + a.tiles_per_cta - 1) / a.tiles_per_cta;
    wgrad_tc_kernel<<<grid, wg::THREADS, wg::SMEM, n->stream>>>(mx, mdy, a);
    CNN_CK(cudaGetLastError());
    reduce_partials_kernel<<<(WSZ + RED_X - 1) / RED_X, RED_X * RED_Y, 0, n->stream>>>(n->partial.p, grid, WSZ, gw);
    reduce_partials_kernel<<<1, RED_X * RED_Y, 0, n->stream>>>(n->bpartial.p, grid, CH, gb);
    CNN_CK(cudaGetLastError());
    return FWI_OK;
}

// After a synchronised run: a bounded wait that gave up in a tensor-core
// kernel becomes FWI_ERR_TIMEOUT (and the flag is cleared).
int check_cnn_status(fwi_cnn *n)
{
    unsigned st = 0;
    CNN_CK(cudaMemcpyFromSymbol(&st, g_cnn_status, sizeof st));
    if (st) {
        const unsigned z = 0;
        CNN_CK(cudaMemcpyToSymbol(g_cnn_status, &z, sizeof z));
        n->err = st & 2u ? "convolution kernel: shared memory not 128-byte aligned"
                         : "convolution kernel: a bounded wait gave up";
        return st & 2u ? FWI_ERR_CUDA : FWI_ERR_TIMEOUT;
    }
    return FWI_OK;
}

int ensure_volume(fwi_cnn *n, int nz, int nx, int ny)
{
    if (nz < 1 || nx < 1 || ny < 1) return FWI_ERR_ARG;
    Geo g{nz, nx, ny, (long long)nz * nx * ny, nz + 2, nx + 2, (long long)(nz + 2) * (nx + 2) * (ny + 2),
          make_fastdiv((uint32_t)(nz + 2)), make_fastdiv((uint32_t)(nx + 2))};
    // TMA row coordinates are 32-bit
    if (g.R + (long long)g.NZ2 * g.NX2 + 2 * tc::BM >= 0x7FFFFFFFLL) {
        n->err = "volume too large for the convolution kernels";
        return FWI_ERR_ARG;
    }
    n->g = g;
    for (int l = 0; l < NL; ++l) CNN_CK(n->act[l].ensure(g.R * CH));
    for (int k = 0; k < 2; ++k) CNN_CK(n->dg[k].ensure(g.R * CH));
    CNN_CK(n->pred.ensure(g.V));
    CNN_CK(n->partial.ensure((size_t)kMaxPartials * WSZ));
    CNN_CK(n->bpartial.ensure((size_t)kMaxPartials * CH));
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
    pack_input_kernel<<<1184, 256, 0, n->stream>>>(n->g, d_in, d_in + V, d_in + 2 * V, n->act[0].p);
    st = forward_impl(n);
    if (st != FWI_OK) return st;
    CNN_CK(cudaMemcpyAsync(d_out, n->pred.p, V * sizeof(float), cudaMemcpyDeviceToDevice, n->stream));
    CNN_CK(cudaStreamSynchronize(n->stream));
    return check_cnn_status(n);
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
    pack_input_kernel<<<1184, 256, 0, n->stream>>>(g, d_in, d_in + V, d_in + 2 * V, n->act[0].p);
    st = forward_impl(n);
    if (st != FWI_OK) return st;
    // loss gradient d(0.5 mean d^2)/dpred = d / V, carried in BF16 scaled up
    // by V (loss scaling) and scaled back in the weight gradients
    const int lblk = 1024;
    mse_kernel<<<lblk, 256, 0, n->stream>>>(g, n->pred.p, d_target, 1.0f, n->dg[0].p, n->lpart.p);
    sum_f64_kernel<<<1, 32, 0, n->stream>>>(n->lpart.p, lblk, n->lsum.p);
    int cur = 0;
    for (int l = NL - 1; l >= 0; --l) {
        // weight and bias gradients of layer l: input act[l], output gradient dg[cur]
        st = launch_wgrad(n, n->act[l].p, n->dg[cur].p, n->gw[l].p, n->gb[l].p);
        if (st != FWI_OK) return st;
        if (l > 0) {
            // data gradient through layer l, masked by the ReLU of act[l]
            st = launch_conv<-1, 1>(n, n->dg[cur].p, n->wt[l].p, nullptr, n->act[l].p, n->dg[1 - cur].p, nullptr);
            if (st != FWI_OK) return st;
            cur = 1 - cur;
        }
    }
    CNN_CK(cudaGetLastError());
    double lsum = 0.0;
    CNN_CK(cudaMemcpyAsync(&lsum, n->lsum.p, sizeof(double), cudaMemcpyDeviceToHost, n->stream));
    CNN_CK(cudaStreamSynchronize(n->stream));
    st = check_cnn_status(n);
    if (st != FWI_OK) return st;
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
