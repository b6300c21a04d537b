// stencil.cuh -- the two hot kernels of the wave-propagation path.
//
//   fd_forward_kernel   one leapfrog step of every shot of a batch:
//                       Q <- d (dt^2 v^2 lap(A) + 2 A - d Q)   [+ source]
//                       and the receiver samples of A
//                       (reference: compute_pressure + compute_seismogram,
//                        src/modeling/modeling.cu:324-393)
//   fd_backward_kernel  the fused back-propagation step:
//                       Ps    <- dt^2 v^2 lap(Psold) + 2 Psold - Ps  (source rebuilt)
//                       Prold <- dt^2 v^2 lap(Pr) + 2 Pr - Prold      (adjoint)
//                       illum += Ps^2 ; image += Ps Pr  or  the gradient term
//                       (reference: cross_correlation, src/migration/migration.cu:134-202;
//                        build_gradient, src/inversion/inversion.cu:400-468)
//
// Data layout in HBM: every field of one shot is a pitched [nyy][nxx][ldz] FP32
// array (z fastest, ldz = nzz rounded up to 8); the shots of a batch follow
// one another at a stride of `vol` elements.  Cells with an index < 4 or >= n-4
// on any axis are never written and stay 0 (the reference's stencil guard,
// src/modeling/modeling.cu:350).
//
// Tiling: a CTA owns a TZ x TX (z, x) column of one shot and walks a chunk of
// y planes.  Thread (lz, lx) owns 4 consecutive z cells of row lx.
//   - Stencil fields arrive plane by plane as (TZ+8) x (TX+8) halo tiles,
//     TMA-loaded into a ring of SH shared-memory slots (plane y needs slots
//     y..y+4 resident; the rest is prefetch).  z and x neighbours come from the
//     tile of plane y, y neighbours from a 9-deep register queue fed with the
//     centre of plane y+4.
//   - Centre-only fields (old time level, velocity, accumulators) arrive as
//     TZ x TX tiles in a second ring of SC slots; the accumulators only
//     where the tile meets the box of accumulated cells, and then only over
//     the z range that meets it.
//   - One elected thread issues every TMA copy; completion is tracked with
//     mbarriers whose waits are bounded (kWaitLimitNs) and report through
//     g_status instead of hanging.
#pragma once

#include "device.cuh"

namespace fwi {

__device__ unsigned int g_status;

template <int TZ4_, int TX_>
struct Tile {
    static constexpr int TZ4 = TZ4_, TX = TX_;
    static constexpr int NT = TZ4 * TX;          // threads
    static constexpr int TZ = 4 * TZ4;           // z cells
    static constexpr int HZ = TZ + 8, HX = TX + 8;
    static constexpr int HALO_BYTES = HZ * HX * 4;
    static constexpr int HSLOT = (HALO_BYTES + 127) / 128 * 128;
    static constexpr int CTR_BYTES = TZ * TX * 4;
    static constexpr int CSLOT = (CTR_BYTES + 127) / 128 * 128;
    static_assert((HZ * 4) % 16 == 0, "TMA inner box must be a multiple of 16 bytes");
    static_assert(HZ <= 256 && HX <= 256, "TMA box dimension limit");
};

// Second derivative along one axis, without the 1/dh^2 factor, summed from the
// outer taps inwards like the reference (src/modeling/modeling.cu:354-358).
__device__ __forceinline__ float d2(float c, float m1, float p1, float m2, float p2, float m3,
                                    float p3, float m4, float p4)
{
    float acc = -W4 * (m4 + p4);
    acc = fmaf(W3, m3 + p3, acc);
    acc = fmaf(-W2, m2 + p2, acc);
    acc = fmaf(W1, m1 + p1, acc);
    acc = fmaf(-W0, c, acc);
    return acc;
}

// Per-axis second derivatives of 4 consecutive z cells of one thread.
// H: halo tile of the plane (row stride HZ); q: register queue (q[4] = centre).
template <class T>
__device__ __forceinline__ void axis_d2(const float *H, int ro, int zo, const float4 (&q)[9],
                                        float (&ax)[4], float (&ay)[4], float (&az)[4])
{
    const float4 zm = lds4(H + ro + zo - 4);
    const float4 zp = lds4(H + ro + zo + 4);
    const float4 c = q[4];
    const float w[12] = {zm.x, zm.y, zm.z, zm.w, c.x, c.y, c.z, c.w, zp.x, zp.y, zp.z, zp.w};
    float4 xm[4], xp[4];
#pragma unroll
    for (int m = 1; m <= 4; ++m) {
        xm[m - 1] = lds4(H + ro - m * T::HZ + zo);
        xp[m - 1] = lds4(H + ro + m * T::HZ + zo);
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const float c0 = w[4 + e];
        ax[e] = d2(c0, comp(xm[0], e), comp(xp[0], e), comp(xm[1], e), comp(xp[1], e),
                   comp(xm[2], e), comp(xp[2], e), comp(xm[3], e), comp(xp[3], e));
        ay[e] = d2(c0, comp(q[3], e), comp(q[5], e), comp(q[2], e), comp(q[6], e), comp(q[1], e),
                   comp(q[7], e), comp(q[0], e), comp(q[8], e));
        az[e] = d2(c0, w[3 + e], w[5 + e], w[2 + e], w[6 + e], w[1 + e], w[7 + e], w[e], w[8 + e]);
    }
}

__device__ __forceinline__ void raise_status(unsigned bits) { atomicOr(&g_status, bits); }

// A launch after a failed wait does no work: a time loop whose copies stopped
// completing ends after one bounded wait instead of one per step.
__device__ __forceinline__ bool status_failed() { return *(volatile unsigned int *)&g_status != 0; }

// Exercises the bounded-wait path without any fault: an mbarrier that expects
// two arrivals gets one, so its phase never completes; the wait gives up after
// limit_ns and reports through g_status exactly like the stencil kernels.
__global__ void bounded_wait_probe_kernel(uint64_t limit_ns)
{
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 2);
        fence_mbar_init();
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&bar)) : "memory");
        if (!mbar_wait(&bar, 0, limit_ns)) raise_status(kErrTimeout);
    }
}

// ---------------------------------------------------------------------------
// Forward leapfrog step.
//   mh: halo-box map over A (the field read with the stencil)
//   mq: centre-box map over Q (the field overwritten)
//   mv: centre-box map over the velocity slots (one slot shared by every
//       shot, or one slot per shot when every shot has its own random pad)
// ---------------------------------------------------------------------------
template <class T, int SH, int SC, bool ABC>
__global__ void __launch_bounds__(T::NT)
    fd_forward_kernel(const __grid_constant__ CUtensorMap mh, const __grid_constant__ CUtensorMap mq,
                      const __grid_constant__ CUtensorMap mv, const FwdArgs a)
{
    static_assert(SH >= 5, "plane y needs halo slots y..y+4");
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char *hring = smem;
    unsigned char *cring = smem + SH * T::HSLOT;
    uint64_t *hbar = reinterpret_cast<uint64_t *>(cring + SC * 2 * T::CSLOT);
    uint64_t *cbar = hbar + SH;
    __shared__ float b1s[ABC ? kMaxPad : 1];
    __shared__ int abort_flag;

    const int tid = threadIdx.x;
    const int shot = blockIdx.y;
    if (status_failed()) return;

    // Receiver samples of A at this step (before the guard below, so that
    // every launched thread takes part).  The reference records P after its
    // in-place damping, i.e. d * A (src/modeling/modeling.cu:378, 391-392).
    if (a.t > a.tlag) {
        const int R = a.binfo->R;
        const long long total = (long long)gridDim.x * gridDim.y * T::NT;
        for (long long g = ((long long)blockIdx.y * gridDim.x + blockIdx.x) * T::NT + tid; g < R;
             g += total)
            a.seis_tm[(long long)(a.t - a.tlag) * R + g] = a.rec_damp[g] * a.A[a.rec_cell[g]];
    }

    int b = blockIdx.x;
    const int zt = b % a.ntz;
    b /= a.ntz;
    const int xt = b % a.ntx;
    const int ch = b / a.ntx;
    const int z0 = 4 + zt * T::TZ, x0 = 4 + xt * T::TX;
    const int ya = 4 + ch * a.ylen;
    const int yb = min(ya + a.ylen, a.nyy - 4);
    if (ya >= yb || shot >= a.binfo->nshot) return;  // uniform per CTA

    const int lz = tid % T::TZ4, lx = tid / T::TZ4;
    const int zc = z0 + 4 * lz, xc = x0 + lx;
    const int vshot = a.vel_slots > 1 ? shot : 0;

    if constexpr (ABC) {
        for (int i = tid; i < a.nb; i += T::NT) b1s[i] = a.b1d[i];
    }
    if (tid == 0) {
        abort_flag = 0;
        prefetch_tmap(&mh);
        prefetch_tmap(&mq);
        prefetch_tmap(&mv);
        for (int s = 0; s < SH; ++s) mbar_init(&hbar[s], 1);
        for (int s = 0; s < SC; ++s) mbar_init(&cbar[s], 1);
        fence_mbar_init();
    }
    __syncthreads();

    const int pf = ya - 4, pl = yb + 3;  // halo planes loaded: [pf, pl]
    int h_issued = pf - 1, c_issued = ya - 1;  // meaningful in thread 0 only
    auto issue_h = [&](int p) {
        const int s = (p - pf) % SH;
        mbar_expect_tx(&hbar[s], T::HALO_BYTES);
        tma_load_4d(hring + s * T::HSLOT, &mh, &hbar[s], z0 - 4, x0 - 4, p, shot);
        h_issued = p;
    };
    auto issue_c = [&](int y) {
        const int s = (y - ya) % SC;
        mbar_expect_tx(&cbar[s], 2 * T::CTR_BYTES);
        tma_load_4d(cring + (2 * s) * T::CSLOT, &mq, &cbar[s], z0, x0, y, shot);
        tma_load_4d(cring + (2 * s + 1) * T::CSLOT, &mv, &cbar[s], z0, x0, y, vshot);
        c_issued = y;
    };
    if (tid == 0) {
        for (int p = pf; p < pf + SH && p <= pl; ++p) issue_h(p);
        for (int y = ya; y < ya + SC && y < yb; ++y) issue_c(y);
    }

    const int3 src = make_int3(a.binfo->src[shot][0], a.binfo->src[shot][1], a.binfo->src[shot][2]);
    const int ro = (lx + 4) * T::HZ, zo = 4 + 4 * lz;
    const bool row_ok = xc < a.nxx - 4 && zc < a.nzz - 4;
    const int dx = ABC ? pad_depth(xc, a.nxx, a.nb) : -1;
    float *Qshot = a.Q + (long long)shot * a.vol;
    const long long plane = (long long)a.ldz * a.nxx;

    float4 q[9];
#pragma unroll
    for (int m = 0; m < 9; ++m) q[m] = make_float4(0.f, 0.f, 0.f, 0.f);

    for (int p = pf; p <= pl; ++p) {
        const int y = p - 4;
        bool ok = mbar_wait(&hbar[(p - pf) % SH], ((p - pf) / SH) & 1);
        if (y >= ya) ok = mbar_wait(&cbar[(y - ya) % SC], ((y - ya) / SC) & 1) && ok;
        if (!ok) abort_flag = 1;

        const float *Hp = reinterpret_cast<const float *>(hring + ((p - pf) % SH) * T::HSLOT);
#pragma unroll
        for (int m = 0; m < 8; ++m) q[m] = q[m + 1];
        q[8] = lds4(Hp + ro + zo);

        if (y >= ya) {
            const float *Hy = reinterpret_cast<const float *>(hring + ((y - pf) % SH) * T::HSLOT);
            const int cs = (y - ya) % SC;
            const float *Cq = reinterpret_cast<const float *>(cring + (2 * cs) * T::CSLOT);
            const float *Cv = reinterpret_cast<const float *>(cring + (2 * cs + 1) * T::CSLOT);
            float ax[4], ay[4], az[4];
            axis_d2<T>(Hy, ro, zo, q, ax, ay, az);
            const float4 qo = lds4(Cq + lx * T::TZ + 4 * lz);
            const float4 vv = lds4(Cv + lx * T::TZ + 4 * lz);
            const int dy = ABC ? pad_depth(y, a.nyy, a.nb) : -1;
            float4 out;
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const float v = comp(vv, e);
                const float cv = v * v * a.cvel;
                const float lap = ax[e] + ay[e] + az[e];
                const float p0 = comp(q[4], e);
                float old = comp(qo, e);
                float d = 1.0f;
                if constexpr (ABC) {
                    d = cerjan(b1s, pad_depth(zc + e, a.nzz, a.nb), dx, dy);
                    old = __fmul_rn(d, old);
                }
                float nv = fmaf(cv, lap, 2.0f * p0 - old);
                if constexpr (ABC) nv = __fmul_rn(d, nv);
                if (zc + e >= a.nzz - 4) nv = comp(qo, e);
                set_comp(out, e, nv);
            }
            // Source sample t+1 goes into the new field, which is exactly where
            // the reference adds it at the start of the next step
            // (src/modeling/modeling.cu:347-348).
            if (y == src.z && xc == src.y) {
                const int e = src.x - zc;
                if (e >= 0 && e < 4 && a.t + 1 < a.nt)
                    set_comp(out, e, comp(out, e) + a.idh3 * a.wavelet[a.t + 1]);
            }
            if (row_ok)
                *reinterpret_cast<float4 *>(Qshot + y * plane + (long long)xc * a.ldz + zc) = out;
        }
        __syncthreads();
        if (abort_flag) break;
        if (tid == 0) {
            fence_proxy_async();
            if (p < ya) {
                if (p + SH <= pl) issue_h(p + SH);
            } else if (y >= ya) {
                if (y + SH <= pl) issue_h(y + SH);
                if (y + SC < yb) issue_c(y + SC);
            }
        }
    }

    if (abort_flag && tid == 0) {
        raise_status(kErrTimeout);
        // Drain copies still in flight into this CTA's shared memory.
        // (only the newest use of each slot can still be in flight)
        for (int p = max(pf, h_issued - SH + 1); p <= h_issued; ++p)
            mbar_wait(&hbar[(p - pf) % SH], ((p - pf) / SH) & 1);
        for (int y = max(ya, c_issued - SC + 1); y <= c_issued; ++y)
            mbar_wait(&cbar[(y - ya) % SC], ((y - ya) / SC) & 1);
    }
}

// ---------------------------------------------------------------------------
// Fused backward step.
//   mhs, mhr: halo maps over Psold and Pr
//   mcs, mcr: centre maps over Ps and Prold (old time levels, overwritten)
//   mv:       centre map over the velocity slots (shared, or one per shot);
//             with the image condition over their stencil coefficient
//             dt^2 v^2 / dh^2 instead (the gradient condition also needs v^2)
//   mim, mil: maps over the image/gradient and illumination slots, with a box
//             of acc_zbox x TX cells (the widest z range of a tile that meets
//             the accumulated box)
// GRAD: gradient imaging condition (with GRAD_DY the d2y term is kept).
// ---------------------------------------------------------------------------
template <class T, int SH, int SC, bool GRAD, bool GRAD_DY>
__global__ void __launch_bounds__(T::NT)
    fd_backward_kernel(const __grid_constant__ CUtensorMap mhs, const __grid_constant__ CUtensorMap mhr,
                       const __grid_constant__ CUtensorMap mcs, const __grid_constant__ CUtensorMap mcr,
                       const __grid_constant__ CUtensorMap mv, const __grid_constant__ CUtensorMap mim,
                       const __grid_constant__ CUtensorMap mil, const BwdArgs a)
{
    static_assert(SH >= 5, "plane y needs halo slots y..y+4");
    constexpr int NCF = 5;  // centre fields: Ps, Prold, v, image, illum
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char *hring = smem;                            // SH x {Psold, Pr}
    unsigned char *cring = smem + SH * 2 * T::HSLOT;        // SC x {Ps, Prold, v, img, ill}
    uint64_t *hbar = reinterpret_cast<uint64_t *>(cring + SC * NCF * T::CSLOT);
    uint64_t *cbar = hbar + SH;
    __shared__ int abort_flag;

    const int tid = threadIdx.x;
    const int shot = blockIdx.y;
    if (status_failed()) return;
    int b = blockIdx.x;
    const int zt = b % a.ntz;
    b /= a.ntz;
    const int xt = b % a.ntx;
    const int ch = b / a.ntx;
    const int z0 = 4 + zt * T::TZ, x0 = 4 + xt * T::TX;
    const int ya = 4 + ch * a.ylen;
    const int yb = min(ya + a.ylen, a.nyy - 4);
    if (ya >= yb || shot >= a.binfo->nshot) return;

    const int lz = tid % T::TZ4, lx = tid / T::TZ4;
    const int zc = z0 + 4 * lz, xc = x0 + lx;
    const int vshot = a.vel_slots > 1 ? shot : 0;
    // Accumulator box: a CTA whose tile misses it in z or x, and every plane
    // outside it in y, moves no accumulator bytes at all.
    const bool acc_tile = z0 < a.acc_z1 && z0 + T::TZ > a.acc_z0 && x0 < a.acc_x1 && x0 + T::TX > a.acc_x0;
    const bool acc_row = xc >= a.acc_x0 && xc < a.acc_x1 && zc < a.acc_z1 && zc + 4 > a.acc_z0;
    auto acc_plane = [&](int y) { return acc_tile && y >= a.acc_y0 && y < a.acc_y1; };
    // Accumulator tiles cover z in [za, za + acc_zbox) only: the part of the
    // tile's z range that reaches the box, widened to float4 boundaries (the
    // TMA start stays 16-byte aligned).
    const int za = max(z0, a.acc_z0) & ~3;
    const int acc_bytes = a.acc_zbox * T::TX * 4;

    if (tid == 0) {
        abort_flag = 0;
        prefetch_tmap(&mhs);
        prefetch_tmap(&mhr);
        for (int s = 0; s < SH; ++s) mbar_init(&hbar[s], 1);
        for (int s = 0; s < SC; ++s) mbar_init(&cbar[s], 1);
        fence_mbar_init();
    }
    __syncthreads();

    const int pf = ya - 4, pl = yb + 3;
    int h_issued = pf - 1, c_issued = ya - 1;
    auto issue_h = [&](int p, int s) {
        mbar_expect_tx(&hbar[s], 2 * T::HALO_BYTES);
        tma_load_4d(hring + (2 * s) * T::HSLOT, &mhs, &hbar[s], z0 - 4, x0 - 4, p, shot);
        tma_load_4d(hring + (2 * s + 1) * T::HSLOT, &mhr, &hbar[s], z0 - 4, x0 - 4, p, shot);
        h_issued = p;
    };
    auto issue_c = [&](int y, int s) {
        unsigned char *base = cring + s * NCF * T::CSLOT;
        const bool acc = acc_plane(y);
        mbar_expect_tx(&cbar[s], (NCF - 2) * T::CTR_BYTES + (acc ? 2 * acc_bytes : 0));
        tma_load_4d(base + 0 * T::CSLOT, &mcs, &cbar[s], z0, x0, y, shot);
        tma_load_4d(base + 1 * T::CSLOT, &mcr, &cbar[s], z0, x0, y, shot);
        tma_load_4d(base + 2 * T::CSLOT, &mv, &cbar[s], z0, x0, y, vshot);
        if (acc) {
            tma_load_4d(base + 3 * T::CSLOT, &mim, &cbar[s], za, x0, y, shot);
            tma_load_4d(base + 4 * T::CSLOT, &mil, &cbar[s], za, x0, y, shot);
        }
        c_issued = y;
    };
    if (tid == 0) {
        for (int p = pf; p < pf + SH && p <= pl; ++p) issue_h(p, p - pf);
        for (int y = ya; y < ya + SC && y < yb; ++y) issue_c(y, y - ya);
    }

    const int3 src = make_int3(a.binfo->src[shot][0], a.binfo->src[shot][1], a.binfo->src[shot][2]);
    // Stored field A_{N-t} carried source sample N-t; the exact rebuild adds it back.
    const float scorr = (a.subtract_src && a.nsteps - a.t < a.nt)
                            ? a.idh3 * a.wavelet[a.nsteps - a.t] : 0.0f;
    const int ro = (lx + 4) * T::HZ, zo = 4 + 4 * lz;
    const bool row_ok = xc < a.nxx - 4 && zc < a.nzz - 4;
    const long long plane = (long long)a.ldz * a.nxx;
    const long long sh_off = (long long)shot * a.vol;

    float4 qs[9], qr[9];
#pragma unroll
    for (int m = 0; m < 9; ++m) {
        qs[m] = make_float4(0.f, 0.f, 0.f, 0.f);
        qr[m] = qs[m];
    }

    // Ring positions as counters (no division by the ring depths per plane):
    // hs, hph = slot and phase parity of halo plane p; hy = slot of plane
    // y = p - 4; cs, cph = slot and phase parity of centre plane y.
    int hs = 0, hph = 0, cs = 0, cph = 0;
    for (int p = pf; p <= pl; ++p) {
        const int y = p - 4;
        const int hy = hs >= 4 ? hs - 4 : hs + SH - 4;
        bool ok = mbar_wait(&hbar[hs], hph);
        if (y >= ya) ok = mbar_wait(&cbar[cs], cph) && ok;
        if (!ok) abort_flag = 1;

        const float *Hs = reinterpret_cast<const float *>(hring + (2 * hs) * T::HSLOT);
        const float *Hr = reinterpret_cast<const float *>(hring + (2 * hs + 1) * T::HSLOT);
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            qs[m] = qs[m + 1];
            qr[m] = qr[m + 1];
        }
        qs[8] = lds4(Hs + ro + zo);
        qr[8] = lds4(Hr + ro + zo);

        if (y >= ya) {
            const float *Hys = reinterpret_cast<const float *>(hring + (2 * hy) * T::HSLOT);
            const float *Hyr = reinterpret_cast<const float *>(hring + (2 * hy + 1) * T::HSLOT);
            const float *C = reinterpret_cast<const float *>(cring + cs * NCF * T::CSLOT);
            constexpr int CF = T::CSLOT / 4;  // floats per centre slot
            const int co = lx * T::TZ + 4 * lz;
            const float4 ps_old = lds4(C + 0 * CF + co);
            const float4 pr_old = lds4(C + 1 * CF + co);
            const float4 vv = lds4(C + 2 * CF + co);
            const bool acc = acc_plane(y);
            float4 img = make_float4(0.f, 0.f, 0.f, 0.f), ill = img;
            if (acc && acc_row) {  // then za <= zc and zc + 4 <= za + acc_zbox
                const int ao = lx * a.acc_zbox + (zc - za);
                img = lds4(C + 3 * CF + ao);
                ill = lds4(C + 4 * CF + ao);
            }

            float sx[4], sy[4], sz[4];
            axis_d2<T>(Hys, ro, zo, qs, sx, sy, sz);
            float4 ps_new, pr_new;
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const float v = comp(vv, e);
                const float cv = GRAD ? v * v * a.cvel : v;
                float s = fmaf(cv, sx[e] + sy[e] + sz[e], 2.0f * comp(qs[4], e) - comp(ps_old, e));
                set_comp(ps_new, e, s);
            }
            if (y == src.z && xc == src.y) {
                const int e = src.x - zc;
                if (e >= 0 && e < 4) set_comp(ps_new, e, comp(ps_new, e) + scorr);
            }
            float rx[4], ry[4], rz[4];
            axis_d2<T>(Hyr, ro, zo, qr, rx, ry, rz);
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const float v = comp(vv, e);
                const float v2 = v * v;  // used by the gradient condition only
                const float cv = GRAD ? v2 * a.cvel : v;
                const float prc = comp(qr[4], e);
                set_comp(pr_new, e, fmaf(cv, rx[e] + ry[e] + rz[e], 2.0f * prc - comp(pr_old, e)));
                const float psn = comp(ps_new, e);
                const int ze = zc + e;
                if (ze >= a.nzz - 4) {
                    set_comp(ps_new, e, comp(ps_old, e));
                    set_comp(pr_new, e, comp(pr_old, e));
                }
                // (the box lies inside the updated cells: acc_z1 <= nzz - 4)
                if (acc && acc_row && ze >= a.acc_z0 && ze < a.acc_z1) {
                    float im = comp(img, e), il = comp(ill, e);
                    il = fmaf(psn, psn, il);
                    if constexpr (GRAD) {
                        const float lz2 = GRAD_DY ? (sx[e] + sz[e] + sy[e]) : (sx[e] + sz[e]);
                        im += a.gscale * prc * lz2 * v2;
                    } else {
                        im = fmaf(psn, prc, im);
                    }
                    set_comp(img, e, im);
                    set_comp(ill, e, il);
                }
            }
            if (row_ok) {
                const long long off = sh_off + y * plane + (long long)xc * a.ldz + zc;
                *reinterpret_cast<float4 *>(a.Ps + off) = ps_new;
                *reinterpret_cast<float4 *>(a.Prold + off) = pr_new;
                if (acc && acc_row) {
                    *reinterpret_cast<float4 *>(a.image + off) = img;
                    *reinterpret_cast<float4 *>(a.illum + off) = ill;
                }
            }
        }
        __syncthreads();
        if (abort_flag) break;
        if (tid == 0) {
            fence_proxy_async();
            if (p < ya) {
                if (p + SH <= pl) issue_h(p + SH, hs);
            } else if (y >= ya) {
                if (y + SH <= pl) issue_h(y + SH, hy);
                if (y + SC < yb) issue_c(y + SC, cs);
            }
        }
        if (++hs == SH) {
            hs = 0;
            hph ^= 1;
        }
        if (y >= ya && ++cs == SC) {
            cs = 0;
            cph ^= 1;
        }
    }

    if (abort_flag && tid == 0) {
        raise_status(kErrTimeout);
        // (only the newest use of each slot can still be in flight)
        for (int p = max(pf, h_issued - SH + 1); p <= h_issued; ++p)
            mbar_wait(&hbar[(p - pf) % SH], ((p - pf) / SH) & 1);
        for (int y = max(ya, c_issued - SC + 1); y <= c_issued; ++y)
            mbar_wait(&cbar[(y - ya) % SC], ((y - ya) / SC) & 1);
    }
}

}  // namespace fwi
