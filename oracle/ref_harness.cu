// ref_harness.cu -- TEST INFRASTRUCTURE ONLY.
//
// Drives the reference's own CUDA code (phbastosa/FWI3D, compiled from its
// sources by oracle/Makefile into oracle/_ref/) on injected inputs, so that
// tests and bench.py can compare against, and time, the reference build.
//
// Setup goes through the reference's own Modeling::set_parameters()
// (src/modeling/modeling.cu:3-15) from a parameters file written by the
// caller; the forward pass is its own Modeling::initialization() +
// forward_solver() (src/modeling/modeling.cu:264-322).  The padded velocity
// is injected into d_Vp after setup: the reference's random boundary is
// seeded from clock64()/std::random_device and its generator kernels have
// unguarded tail threads (src/modeling/modeling.cu:594-666), so they are not
// run.  The backward pass repeats the five-line time loop of
// Migration::backward_propagation (src/migration/migration.cu:72-80) or
// Inversion::backward_propagation (src/inversion/inversion.cu:244-252) around
// the reference's kernels inject_seismogram + cross_correlation or
// inject_residuo + build_gradient.
#include <cuda_runtime.h>
#include <curand_kernel.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "admin/admin.cpp"
#include "geometry/geometry.cpp"
#include "modeling/modeling.cu"
#include "migration/migration.cu"
#include "inversion/inversion.cu"

namespace {

int check(const char *where)
{
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "ref_harness: %s: %s\n", where, cudaGetErrorString(e));
        return 2;
    }
    return 0;
}

struct Harness : public Modeling {
    // The reference never frees its buffers; the harness does, so that many
    // runs fit in one process.
    void release()
    {
        cudaFree(d_P);
        cudaFree(d_Pold);
        cudaFree(d_Vp);
        cudaFree(d_b1d);
        cudaFree(d_b2d);
        cudaFree(d_b3d);
        cudaFree(d_wavelet);
        cudaFree(d_seismogram);
        cudaFree(d_rIdx);
        cudaFree(d_rIdy);
        cudaFree(d_rIdz);
        delete[] Vp;
        delete[] seismogram;
        if (geometry) {
            delete[] geometry->xsrc;
            delete[] geometry->ysrc;
            delete[] geometry->zsrc;
            delete[] geometry->xrec;
            delete[] geometry->yrec;
            delete[] geometry->zrec;
            delete geometry;
            geometry = nullptr;
        }
    }

    int dims_of(const char *params, int *dims)
    {
    try {
        parameters = params;
        set_parameters();
        dims[0] = nzz;
        dims[1] = nxx;
        dims[2] = nyy;
        dims[3] = nb;
        dims[4] = nt;
        dims[5] = geometry->nrec;
        dims[6] = tlag;
        release();
        return check("ref_dims");
    } catch (const std::exception &e) {
        fprintf(stderr, "ref_harness: %s\n", e.what());
        return 1;
    }
    }

    int run(const char *params, const float *vp_padded, int shot, int abc, int backward, const float *adj,
            float *seis, float *p_cur, float *p_old, float *image, float *illum, float *ms)
    {
    try {
        parameters = params;
        set_parameters();
        ABC = abc != 0;
        const size_t vol = (size_t)volsize;
        const size_t ns = (size_t)nt * geometry->nrec;
        cudaMemcpy(d_Vp, vp_padded, vol * sizeof(float), cudaMemcpyHostToDevice);
        cudaMemset(d_seismogram, 0, ns * sizeof(float));
        srcId = shot;
        initialization();
        cudaEvent_t e[4];
        for (auto &x : e) cudaEventCreate(&x);
        cudaEventRecord(e[0]);
        forward_solver();
        cudaEventRecord(e[1]);
        int st = check("forward");
        if (st) return st;
        if (seis) cudaMemcpy(seis, d_seismogram, ns * sizeof(float), cudaMemcpyDeviceToHost);
        if (p_cur) cudaMemcpy(p_cur, d_P, vol * sizeof(float), cudaMemcpyDeviceToHost);
        if (p_old) cudaMemcpy(p_old, d_Pold, vol * sizeof(float), cudaMemcpyDeviceToHost);
        float fms = 0, bms = 0;
        cudaEventElapsedTime(&fms, e[0], e[1]);
        if (backward) {
            float *Pr, *Prold, *img, *ill;
            cudaMalloc(&Pr, vol * sizeof(float));
            cudaMalloc(&Prold, vol * sizeof(float));
            cudaMalloc(&img, vol * sizeof(float));
            cudaMalloc(&ill, vol * sizeof(float));
            cudaMemset(Pr, 0, vol * sizeof(float));
            cudaMemset(Prold, 0, vol * sizeof(float));
            cudaMemset(img, 0, vol * sizeof(float));
            cudaMemset(ill, 0, vol * sizeof(float));
            cudaMemcpy(d_seismogram, adj, ns * sizeof(float), cudaMemcpyHostToDevice);
            float *Ps = d_P, *Psold = d_Pold;
            const int nrec = geometry->nrec;
            cudaEventRecord(e[2]);
            for (int t = 0; t < nt + tlag; ++t) {
                if (backward == 1) {
                    inject_seismogram<<<sBlocks, NTHREADS>>>(Pr, d_rIdx, d_rIdy, d_rIdz, d_seismogram,
                                                               nrec, t, nt, nxx, nzz, idh3);
                    cross_correlation<<<nBlocks, NTHREADS>>>(Ps, Psold, Pr, Prold, d_Vp, img, ill, nxx,
                                                               nyy, nzz, nt, idh2, dt);
                } else {
                    inject_residuo<<<sBlocks, NTHREADS>>>(Pr, d_rIdx, d_rIdy, d_rIdz, d_seismogram, nrec,
                                                            t, nt, nxx, nzz, idh3);
                    build_gradient<<<nBlocks, NTHREADS>>>(Ps, Psold, Pr, Prold, d_Vp, img, ill, nxx, nyy,
                                                            nzz, nt, dt, idh2);
                }
                std::swap(Ps, Psold);
                std::swap(Pr, Prold);
            }
            cudaEventRecord(e[3]);
            st = check("backward");
            if (!st) {
                cudaEventElapsedTime(&bms, e[2], e[3]);
                if (image) cudaMemcpy(image, img, vol * sizeof(float), cudaMemcpyDeviceToHost);
                if (illum) cudaMemcpy(illum, ill, vol * sizeof(float), cudaMemcpyDeviceToHost);
            }
            cudaFree(Pr);
            cudaFree(Prold);
            cudaFree(img);
            cudaFree(ill);
            if (st) return st;
        }
        for (auto &x : e) cudaEventDestroy(x);
        if (ms) {
            ms[0] = fms;
            ms[1] = bms;
        }
        release();
        return check("release");
    } catch (const std::exception &e) {
        fprintf(stderr, "ref_harness: %s\n", e.what());
        return 1;
    }
    }
};

}  // namespace

extern "C" {

// dims[0..6] = nzz, nxx, nyy, nb, nt, nrec, tlag of the setup the parameters
// file describes (the abc_length key fixes nb).
int ref_dims(const char *params, int *dims)
{
    Harness h{};  // value-initialised, like `new Modeling()` in the mains
    return h.dims_of(params, dims);
}

// One shot through the reference.
//   abc       1 = Cerjan sponge on (modeling.exe), 0 = off (migration/inversion)
//   backward  0 = forward only, 1 = RTM imaging, 2 = FWI gradient
//   adj       [nt, nrec] data injected time-reversed in the backward pass
//   seis      [nt, nrec] recorded seismogram (sample 0 zeroed beforehand)
//   p_cur, p_old  padded wavefields after the last forward step (or NULL)
//   image, illum  padded accumulators after the backward pass (or NULL)
//   ms        device time of the forward and backward time loops
int ref_run(const char *params, const float *vp_padded, int shot, int abc, int backward,
            const float *adj, float *seis, float *p_cur, float *p_old, float *image, float *illum,
            float *ms)
{
    Harness h{};  // value-initialised, like `new Modeling()` in the mains
    return h.run(params, vp_padded, shot, abc, backward, adj, seis, p_cur, p_old, image, illum, ms);
}

}  // extern "C"
