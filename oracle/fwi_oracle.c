/*
 * fwi_oracle.c -- CPU FP64 restatement of FWI3D's wave-propagation hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library in
 * fwi3d_b200/csrc and the timed CPU baseline of bench.py.  Nothing in the
 * product links or calls it; only tests/, __graft_entry__.smoke() and bench.py
 * (its cpu_baseline leg and its `--impl reference` fallback) load it.
 *
 * Every routine restates, in double precision, one piece of the reference
 * (phbastosa/FWI3D); the citation above each routine is `file:line` inside
 * that project.  State and arithmetic are FP64 throughout (the reference stores
 * FP32 wavefields and evaluates its stencil in FP64 because its FD coefficients
 * are double literals, src/modeling/modeling.cuh:9-13).
 *
 * Where the reference is racy or leaves memory undefined, the oracle fixes the
 * deterministic meaning used by the whole project:
 *   - the source is added to P before any stencil reads P
 *     (src/modeling/modeling.cu:347-348);
 *   - the stencil reads P before it is damped; damping then scales both P and
 *     the new field (src/modeling/modeling.cu:372-380);
 *   - seismogram sample 0 is never recorded by the reference
 *     (src/modeling/modeling.cu:391); the oracle leaves it at 0.
 *
 * Parity pins: tests/golden/ holds outputs of the reference's own CUDA kernels
 * (built from source by oracle/Makefile into oracle/_ref and run on a B200);
 * tests/test_golden.py checks this file against them, tests/test_reference_build.py
 * and tests/test_fullsize_parity.py against the live reference build, and
 * tests/test_known_answers.py against analytic known answers (eighth-order
 * stencil symbol, constant-velocity Green's function, finite-difference
 * gradient) and the dot-product identity of the imaging operator with
 * orc_image_adjoint.
 *
 * Build: oracle/Makefile -> oracle/liboracle.so (gcc -O3 -fopenmp).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* FD coefficients exactly as the reference's double literals
 * (src/modeling/modeling.cuh:9-13).  Tap m=1..4 and centre. */
static const double ORC_C[5] = {
    2.847222222222,  /* centre, FDM5 */
    1.600000000000,  /* m = 1, FDM4 */
    0.200000000000,  /* m = 2, FDM3 */
    0.025396825396,  /* m = 3, FDM2 */
    0.001785714285,  /* m = 4, FDM1 */
};
/* sign of tap m in the second-derivative operator: + for m=1,3; - for m=2,4 */
static const double ORC_S[5] = {-1.0, +1.0, -1.0, +1.0, -1.0};

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------------------------ */
/* Ricker wavelet: src/modeling/modeling.cu:36-59.                           */
/* Peak frequency is fmax/3; delay t0 = 2 sqrt(pi)/fmax; tlag = int(t0/dt)+1 */
/* ------------------------------------------------------------------------ */
void orc_wavelet(int nt, double dt, double fmax, double *w, int *tlag)
{
    const double pi = 3.14159265358979323846;
    double t0 = 2.0 * sqrt(pi) / fmax;
    double fc = fmax / (3.0 * sqrt(pi));
    *tlag = (int)(t0 / dt) + 1;
    for (int n = 0; n < nt; ++n) {
        double td = n * dt - t0;
        double a = pi * pi * pi * fc * fc * td * td;
        w[n] = 1e5 * (1.0 - 2.0 * a) * exp(-a);
    }
}

/* ------------------------------------------------------------------------ */
/* Cerjan damper tables: src/modeling/modeling.cu:83-140.                     */
/*   b1d[i] = exp(-(f (nb - i))^2)                                           */
/*   b2d[p + q nb] = b1d[p] + b1d[q] - 1                                     */
/*   b3d[i + j nb + k nb^2] = 2 (b1d[i] + b1d[j] + b1d[k]) - 5               */
/* ------------------------------------------------------------------------ */
void orc_damper_tables(int nb, double factor, double *b1d, double *b2d, double *b3d)
{
    for (int i = 0; i < nb; ++i) {
        double a = factor * (double)(nb - i);
        b1d[i] = exp(-a * a);
    }
    for (int q = 0; q < nb; ++q)
        for (int p = 0; p < nb; ++p)
            b2d[p + (size_t)q * nb] = b1d[p] + b1d[q] - 1.0;
    if (b3d)
        for (int k = 0; k < nb; ++k)
            for (int j = 0; j < nb; ++j)
                for (int i = 0; i < nb; ++i)
                    b3d[i + (size_t)j * nb + (size_t)k * nb * nb] =
                        2.0 * (b1d[i] + b1d[j] + b1d[k]) - 5.0;
}

/* Distance into the pad along one axis, or -1 for the inner region.
 * Low side uses the index itself, high side counts back from the last cell
 * (src/modeling/modeling.cu:408-431). */
static inline int pad_depth(int i, int n, int nb)
{
    if (i < nb) return i;
    if (i >= n - nb) return n - 1 - i;
    return -1;
}

/* Damping factor of cell (i,j,k): src/modeling/modeling.cu:395-520.  The
 * reference's 27-way branch reduces to: count the axes in the pad and read the
 * 1-D, 2-D or 3-D table with the per-axis pad depths (z, x, y order). */
double orc_damper_at(const double *b1d, const double *b2d, const double *b3d, int nb,
                     int nzz, int nxx, int nyy, int i, int j, int k)
{
    int dz = pad_depth(i, nzz, nb), dx = pad_depth(j, nxx, nb), dy = pad_depth(k, nyy, nb);
    int n = (dz >= 0) + (dx >= 0) + (dy >= 0);
    if (n == 0) return 1.0;
    if (n == 1) return b1d[dz >= 0 ? dz : (dx >= 0 ? dx : dy)];
    if (n == 2) {
        int a = dz >= 0 ? dz : dx;
        int b = dy >= 0 ? dy : dx;
        return b2d[a + (size_t)b * nb];
    }
    return b3d[dz + (size_t)dx * nb + (size_t)dy * nb * nb];
}

/* ------------------------------------------------------------------------ */
/* Edge-replication padding: src/modeling/modeling.cu:181-228.               */
/* Layout z fastest: idx = i + j nzz + k nxx nzz.                            */
/* ------------------------------------------------------------------------ */
void orc_expand(const double *in, int nz, int nx, int ny, int nb, double *out)
{
    int nzz = nz + 2 * nb, nxx = nx + 2 * nb, nyy = ny + 2 * nb;
#pragma omp parallel for
    for (int k = 0; k < nyy; ++k) {
        int ks = k < nb ? 0 : (k >= ny + nb ? ny - 1 : k - nb);
        for (int j = 0; j < nxx; ++j) {
            int js = j < nb ? 0 : (j >= nx + nb ? nx - 1 : j - nb);
            const double *src = in + (size_t)js * nz + (size_t)ks * nx * nz;
            double *dst = out + (size_t)j * nzz + (size_t)k * nxx * nzz;
            for (int i = 0; i < nzz; ++i) {
                int is = i < nb ? 0 : (i >= nz + nb ? nz - 1 : i - nb);
                dst[i] = src[is];
            }
        }
    }
}

/* Crop the pad: src/modeling/modeling.cu:230-241. */
void orc_reduce(const double *in, int nz, int nx, int ny, int nb, double *out)
{
    int nzz = nz + 2 * nb, nxx = nx + 2 * nb;
#pragma omp parallel for
    for (int k = 0; k < ny; ++k)
        for (int j = 0; j < nx; ++j)
            for (int i = 0; i < nz; ++i)
                out[i + (size_t)j * nz + (size_t)k * nx * nz] =
                    in[(i + nb) + (size_t)(j + nb) * nzz + (size_t)(k + nb) * nxx * nzz];
}

/* Grid index of a coordinate: src/modeling/modeling.cu:270-288, evaluated in
 * FP32 like the reference (coordinates are float there). */
int orc_grid_index(float coord, float dh, int nb)
{
    return (int)((coord + 0.5f * dh) / dh) + nb;
}

/* ------------------------------------------------------------------------ */
/* Second derivatives of one field at cell c (interior cell only).           */
/* The reference writes each axis as a 9-point sum in FP64                   */
/* (src/modeling/modeling.cu:354-370).                                       */
/* ------------------------------------------------------------------------ */
static inline double d2_axis(const double *f, size_t c, size_t s)
{
    double acc = -ORC_C[0] * f[c];
    for (int m = 1; m <= 4; ++m)
        acc += ORC_S[m] * ORC_C[m] * (f[c - m * s] + f[c + m * s]);
    return acc;
}

typedef struct {
    int nzz, nxx, nyy;
    double idh2, dt;
} orc_dims;

/* ------------------------------------------------------------------------ */
/* One leapfrog step over the interior (4 <= i < n-4 on every axis):          */
/*   Pold <- dt^2 v^2 lap(P) + 2 P - Pold            (modeling.cu:350-372)     */
/* then, with Cerjan damping on, P and Pold are both scaled (modeling.cu:374- */
/* 380) -- after the sweep, so the stencil read the undamped P.              */
/* ------------------------------------------------------------------------ */
static void step_forward(const orc_dims *g, const double *vp, double *P, double *Pold,
                         const double *b1d, const double *b2d, const double *b3d, int nb, int abc)
{
    const size_t sz = 1, sx = (size_t)g->nzz, sy = (size_t)g->nzz * g->nxx;
    const double dt2 = g->dt * g->dt;
#pragma omp parallel for
    for (int k = 4; k < g->nyy - 4; ++k)
        for (int j = 4; j < g->nxx - 4; ++j)
            for (int i = 4; i < g->nzz - 4; ++i) {
                size_t c = i + j * sx + k * sy;
                double lap = (d2_axis(P, c, sx) + d2_axis(P, c, sy) + d2_axis(P, c, sz)) * g->idh2;
                Pold[c] = dt2 * vp[c] * vp[c] * lap + 2.0 * P[c] - Pold[c];
            }
    if (!abc) return;
#pragma omp parallel for
    for (int k = 4; k < g->nyy - 4; ++k)
        for (int j = 4; j < g->nxx - 4; ++j)
            for (int i = 4; i < g->nzz - 4; ++i) {
                size_t c = i + j * sx + k * sy;
                double d = orc_damper_at(b1d, b2d, b3d, nb, g->nzz, g->nxx, g->nyy, i, j, k);
                P[c] *= d;
                Pold[c] *= d;
            }
}

/* ------------------------------------------------------------------------ */
/* Forward modeling of one shot: src/modeling/modeling.cu:309-322 (time loop) */
/* with compute_pressure (:324-382) and compute_seismogram (:384-393).        */
/*                                                                           */
/* vp        padded velocity, nzz*nxx*nyy                                    */
/* w         wavelet, nt samples (injected for t < nt, scaled by idh3)       */
/* src       flat padded index of the source cell                            */
/* rec       flat padded indices of the nrec receivers                       */
/* seis      [nt, nrec] Fortran order (t + r nt); sample 0 left at 0         */
/* P, Pold   in: ignored (zeroed); out: the two wavefields after the last    */
/*           swap (P = u^N, Pold = u^{N-1}), ready for back-propagation      */
/* abc       1 = Cerjan sponge (b1d/b2d/b3d, nb), 0 = no damping (RBC runs)  */
/* ------------------------------------------------------------------------ */
void orc_forward(int nzz, int nxx, int nyy, double dh, double dt, int nt, int tlag,
                 const double *vp, const double *w, long src, int nrec, const long *rec,
                 int abc, int nb, const double *b1d, const double *b2d, const double *b3d,
                 double *seis, double *P, double *Pold)
{
    orc_dims g = {nzz, nxx, nyy, 1.0 / (dh * dh), dt};
    const double idh3 = 1.0 / (dh * dh * dh);
    size_t vol = (size_t)nzz * nxx * nyy;
    memset(P, 0, vol * sizeof(double));
    memset(Pold, 0, vol * sizeof(double));
    if (seis) memset(seis, 0, (size_t)nt * nrec * sizeof(double));
    double *a = P, *b = Pold;
    for (int t = 0; t < tlag + nt; ++t) {
        if (t < nt) a[src] += idh3 * w[t];
        step_forward(&g, vp, a, b, b1d, b2d, b3d, nb, abc);
        if (seis && t > tlag)
            for (int r = 0; r < nrec; ++r) seis[(t - tlag) + (size_t)r * nt] = a[rec[r]];
        double *tmp = a; a = b; b = tmp;
    }
    /* After an odd number of steps the roles end swapped (a == Pold); hand the
     * pair back as (current, previous) in the caller's arrays. */
    if (a != P) {
        double *tmp = (double *)malloc(vol * sizeof(double));
        memcpy(tmp, Pold, vol * sizeof(double));
        memcpy(Pold, P, vol * sizeof(double));
        memcpy(P, tmp, vol * sizeof(double));
        free(tmp);
    }
}

/* ------------------------------------------------------------------------ */
/* Adjoint source: src/migration/migration.cu:119-132 and                     */
/* src/inversion/inversion.cu:385-398 -- time-reversed data added at the     */
/* receiver cells, scaled by idh3, for t < nt.                               */
/* ------------------------------------------------------------------------ */
static void inject_reversed(double *Pr, int nt, int t, int nrec, const long *rec,
                            const double *data, double idh3)
{
    if (t >= nt) return;
    for (int r = 0; r < nrec; ++r) Pr[rec[r]] += idh3 * data[(nt - t - 1) + (size_t)r * nt];
}

/* ------------------------------------------------------------------------ */
/* Back-propagation of one shot through a non-damping (random) boundary.     */
/*   mode 0 (RTM)      src/migration/migration.cu:61-81 + 134-202            */
/*       Ps    <- dt^2 v^2 lap(Psold) + 2 Psold - Ps     (source rebuilt)    */
/*       Prold <- dt^2 v^2 lap(Pr) + 2 Pr - Prold        (adjoint field)     */
/*       illum += Ps^2 ; image += Ps Pr                                       */
/*   mode 1 (gradient) src/inversion/inversion.cu:235-253 + 400-468          */
/*       same two updates; illum += Ps^2 ;                                   */
/*       image += dt Pr (d2x Psold + d2z Psold [+ d2y Psold]) v^2            */
/*       The reference omits d2y (inversion.cu:466); with_dy=1 restores it.  */
/* subtract_src = 1 removes the source term while rebuilding Ps (the        */
/* reference does not, migration.cu:195); w, src and tlag give that term.    */
/* Ps, Psold in: the forward pair (u^N, u^{N-1}); out: rebuilt fields.       */
/* ------------------------------------------------------------------------ */
void orc_backward(int nzz, int nxx, int nyy, double dh, double dt, int nt, int tlag,
                  const double *vp, int nrec, const long *rec, const double *data,
                  int mode, int with_dy, int subtract_src, const double *w, long src,
                  double *Ps, double *Psold, double *image, double *illum)
{
    const size_t sz = 1, sx = (size_t)nzz, sy = (size_t)nzz * nxx;
    const size_t vol = (size_t)nzz * nxx * nyy;
    const double idh2 = 1.0 / (dh * dh), idh3 = 1.0 / (dh * dh * dh), dt2 = dt * dt;
    const int N = nt + tlag;
    double *Pr = (double *)calloc(vol, sizeof(double));
    double *Prold = (double *)calloc(vol, sizeof(double));
    double *ps = Ps, *pso = Psold, *pr = Pr, *pro = Prold;
    for (int t = 0; t < N; ++t) {
        inject_reversed(pr, nt, t, nrec, rec, data, idh3);
        /* the stored field being replaced, A_{N-t}, carried source sample N-t */
        const double scorr = (subtract_src && (N - t) < nt) ? idh3 * w[N - t] : 0.0;
#pragma omp parallel for
        for (int k = 4; k < nyy - 4; ++k)
            for (int j = 4; j < nxx - 4; ++j)
                for (int i = 4; i < nzz - 4; ++i) {
                    size_t c = i + j * sx + k * sy;
                    double v2 = vp[c] * vp[c];
                    double sxx = d2_axis(pso, c, sx) * idh2;
                    double syy = d2_axis(pso, c, sy) * idh2;
                    double szz = d2_axis(pso, c, sz) * idh2;
                    double rl = (d2_axis(pr, c, sx) + d2_axis(pr, c, sy) + d2_axis(pr, c, sz)) * idh2;
                    double psn = dt2 * v2 * (sxx + syy + szz) + 2.0 * pso[c] - ps[c];
                    if ((long)c == src) psn += scorr;
                    ps[c] = psn;
                    pro[c] = dt2 * v2 * rl + 2.0 * pr[c] - pro[c];
                    illum[c] += psn * psn;
                    if (mode == 0)
                        image[c] += psn * pr[c];
                    else
                        image[c] += dt * pr[c] * (sxx + szz + (with_dy ? syy : 0.0)) * v2;
                }
        double *tmp = ps; ps = pso; pso = tmp;
        tmp = pr; pr = pro; pro = tmp;
    }
    /* hand the rebuilt pair back in (current, previous) order */
    if (ps != Ps) {
        double *tmp = (double *)malloc(vol * sizeof(double));
        memcpy(tmp, Ps, vol * sizeof(double));
        memcpy(Ps, Psold, vol * sizeof(double));
        memcpy(Psold, tmp, vol * sizeof(double));
        free(tmp);
    }
    free(Pr);
    free(Prold);
}

/* ------------------------------------------------------------------------ */
/* Adjoint of the imaging operator of orc_backward (mode 0) for fixed source  */
/* fields: the image is sum_t S_t . u_t, where S_t is the rebuilt source     */
/* field of back-propagation step t and u_t the adjoint field after the      */
/* injection of step t, with                                                  */
/*     u_{t+1} = (2 + V L) u_t - u_{t-1} + J_{t+1} d,   V = dt^2 v^2,         */
/* L the interior Laplacian (zero outer shell) and J_t the injection of      */
/* idh3 d[r, nt-1-t] at the receiver cells (src/migration/migration.cu:       */
/* 61-81, 119-202).  Its adjoint runs                                         */
/*     lambda_t = (2 + L V) lambda_{t+1} - lambda_{t+2} + S_t . m            */
/* from t = N-1 down to 0 and reads data[r, nt-1-t] = idh3 lambda_t(rec r):  */
/* Born modelling of the model m scattering the source field.  Ps0, Psold0   */
/* are the forward pair handed to orc_backward; subtract_src, w and src as   */
/* there.  For the dot-product test <image(d), m> = <d, adjoint(m)>; keeps   */
/* all N source fields in memory (small grids only).                          */
/* ------------------------------------------------------------------------ */
int orc_image_adjoint(int nzz, int nxx, int nyy, double dh, double dt, int nt, int tlag,
                      const double *vp, int nrec, const long *rec, int subtract_src, const double *w,
                      long src, const double *Ps0, const double *Psold0, const double *m, double *data)
{
    const size_t sz = 1, sx = (size_t)nzz, sy = (size_t)nzz * nxx;
    const size_t vol = (size_t)nzz * nxx * nyy;
    const double idh2 = 1.0 / (dh * dh), idh3 = 1.0 / (dh * dh * dh), dt2 = dt * dt;
    const int N = nt + tlag;
    double *S = (double *)calloc((size_t)N * vol, sizeof(double));
    double *ps = (double *)malloc(vol * sizeof(double));
    double *pso = (double *)malloc(vol * sizeof(double));
    double *l0 = (double *)calloc(vol, sizeof(double));  /* lambda_{t+1} */
    double *l1 = (double *)calloc(vol, sizeof(double));  /* lambda_{t+2} */
    double *vl = (double *)calloc(vol, sizeof(double));  /* V lambda_{t+1} */
    if (!S || !ps || !pso || !l0 || !l1 || !vl) {
        free(S); free(ps); free(pso); free(l0); free(l1); free(vl);
        return 1;
    }
    memcpy(ps, Ps0, vol * sizeof(double));
    memcpy(pso, Psold0, vol * sizeof(double));
    /* the source fields exactly as orc_backward rebuilds them */
    for (int t = 0; t < N; ++t) {
        const double scorr = (subtract_src && (N - t) < nt) ? idh3 * w[N - t] : 0.0;
        double *St = S + (size_t)t * vol;
#pragma omp parallel for
        for (int k = 4; k < nyy - 4; ++k)
            for (int j = 4; j < nxx - 4; ++j)
                for (int i = 4; i < nzz - 4; ++i) {
                    size_t c = i + j * sx + k * sy;
                    double lap = (d2_axis(pso, c, sx) + d2_axis(pso, c, sy) + d2_axis(pso, c, sz)) * idh2;
                    double psn = dt2 * vp[c] * vp[c] * lap + 2.0 * pso[c] - ps[c];
                    if ((long)c == src) psn += scorr;
                    St[c] = psn;
                }
        for (size_t c = 0; c < vol; ++c) ps[c] = St[c];
        double *tmp = ps; ps = pso; pso = tmp;
    }
    memset(data, 0, (size_t)nrec * nt * sizeof(double));
    for (int t = N - 1; t >= 0; --t) {
        const double *St = S + (size_t)t * vol;
#pragma omp parallel for
        for (int k = 4; k < nyy - 4; ++k)
            for (int j = 4; j < nxx - 4; ++j)
                for (int i = 4; i < nzz - 4; ++i) {
                    size_t c = i + j * sx + k * sy;
                    vl[c] = dt2 * vp[c] * vp[c] * l0[c];
                }
        /* lambda_t overwrites lambda_{t+2} */
#pragma omp parallel for
        for (int k = 4; k < nyy - 4; ++k)
            for (int j = 4; j < nxx - 4; ++j)
                for (int i = 4; i < nzz - 4; ++i) {
                    size_t c = i + j * sx + k * sy;
                    double lap = (d2_axis(vl, c, sx) + d2_axis(vl, c, sy) + d2_axis(vl, c, sz)) * idh2;
                    l1[c] = 2.0 * l0[c] + lap - l1[c] + St[c] * m[c];
                }
        if (t < nt)
            for (int r = 0; r < nrec; ++r) data[(nt - 1 - t) + (size_t)r * nt] += idh3 * l1[rec[r]];
        double *tmp = l0; l0 = l1; l1 = tmp;
    }
    free(S); free(ps); free(pso); free(l0); free(l1); free(vl);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* RTM image post-processing: src/migration/migration.cu:90-117.             */
/* Crop image and illumination, divide, then -d2/dz2 scaled by idh2 with the  */
/* first and last depth sample set to 0.                                     */
/* ------------------------------------------------------------------------ */
void orc_rtm_post(const double *image_pad, const double *illum_pad, int nz, int nx, int ny,
                  int nb, double dh, double *out)
{
    size_t n = (size_t)nz * nx * ny;
    double *a = (double *)malloc(n * sizeof(double));
    double *s = (double *)malloc(n * sizeof(double));
    orc_reduce(image_pad, nz, nx, ny, nb, a);
    orc_reduce(illum_pad, nz, nx, ny, nb, s);
    /* 0 where the illumination is 0: the reference's 0/0 is NaN there; the
     * project defines it as 0 */
    for (size_t c = 0; c < n; ++c) s[c] = s[c] != 0.0 ? a[c] / s[c] : 0.0;
    double idh2 = 1.0 / (dh * dh);
#pragma omp parallel for
    for (long c = 0; c < (long)n; ++c) {
        int i = (int)(c % nz);
        out[c] = (i > 0 && i < nz - 1) ? -(s[c - 1] - 2.0 * s[c] + s[c + 1]) * idh2 : 0.0;
    }
    free(a);
    free(s);
}

/* ------------------------------------------------------------------------ */
/* FWI gradient post-processing: src/inversion/inversion.cu:142-169.         */
/* Crop, divide by illumination, -d2/dz2 below the depth mask               */
/* (i > int(zmask/dh) and i < nz-1), normalise by max |g|.  Returns max|g|.  */
/* ------------------------------------------------------------------------ */
double orc_gradient_post(const double *grad_pad, const double *illum_pad, int nz, int nx, int ny,
                         int nb, double dh, double zmask, double *out)
{
    size_t n = (size_t)nz * nx * ny;
    double *g = (double *)malloc(n * sizeof(double));
    double *s = (double *)malloc(n * sizeof(double));
    orc_reduce(grad_pad, nz, nx, ny, nb, g);
    orc_reduce(illum_pad, nz, nx, ny, nb, s);
    for (size_t c = 0; c < n; ++c) s[c] = s[c] != 0.0 ? g[c] / s[c] : 0.0;  /* as orc_rtm_post */
    double idh2 = 1.0 / (dh * dh);
    int imask = (int)(zmask / dh);
    double gmax = 0.0;
    for (size_t c = 0; c < n; ++c) {
        int i = (int)(c % nz);
        double v = (i > imask && i < nz - 1) ? -(s[c - 1] - 2.0 * s[c] + s[c + 1]) * idh2 : 0.0;
        out[c] = v;
        if (fabs(v) > gmax) gmax = fabs(v);
    }
    if (gmax > 0.0)
        for (size_t c = 0; c < n; ++c) out[c] *= 1.0 / gmax;
    free(g);
    free(s);
    return gmax;
}

/* ------------------------------------------------------------------------ */
/* Residual and L2 misfit: src/inversion/inversion.cu:190-201.               */
/* res = obs - cal ; returns sum(res^2) (the reference sums in FP32).        */
/* ------------------------------------------------------------------------ */
double orc_residual(const double *obs, const double *cal, long n, double *res)
{
    double acc = 0.0;
    for (long c = 0; c < n; ++c) {
        double r = obs[c] - cal[c];
        if (res) res[c] = r;
        acc += r * r;
    }
    return acc;
}

/* Same sum with single-precision inputs (seismograms are FP32 on disk). */
double orc_residual_f32(const float *obs, const float *cal, long n)
{
    double acc = 0.0;
#pragma omp parallel for reduction(+ : acc)
    for (long c = 0; c < n; ++c) {
        double r = (double)obs[c] - (double)cal[c];
        acc += r * r;
    }
    return acc;
}

/* ------------------------------------------------------------------------ */
/* Parabolic line search: src/inversion/inversion.cu:291-313.                */
/* Fit f(a) through (a0,f0),(a1,f1),(a2,f2) and return the vertex.           */
/* ------------------------------------------------------------------------ */
double orc_parabola_step(double a0, double a1, double a2, double f0, double f1, double f2)
{
    double num = (a1 * a1 - a2 * a2) * f0 + (a2 * a2 - a0 * a0) * f1 + (a0 * a0 - a1 * a1) * f2;
    double den = (a1 - a2) * f0 + (a2 - a0) * f1 + (a0 - a1) * f2;
    return 0.5 * num / den;
}

/* Trial / updated velocity in slowness-squared: inversion.cu:315-321, 349-356.
 * m = 1/v^2 ; v' = 1/sqrt(m - alpha g). */
void orc_model_step(const double *m, const double *g, long n, double alpha, double *v_out)
{
#pragma omp parallel for
    for (long c = 0; c < n; ++c) v_out[c] = 1.0 / sqrt(m[c] - alpha * g[c]);
}

/* ------------------------------------------------------------------------ */
/* A single forward step on FP64 arrays, exposed for unit tests of the       */
/* stencil (plane-wave dispersion, Green's function).                        */
/* ------------------------------------------------------------------------ */
void orc_step(int nzz, int nxx, int nyy, double dh, double dt, const double *vp, double *P,
              double *Pold)
{
    orc_dims g = {nzz, nxx, nyy, 1.0 / (dh * dh), dt};
    step_forward(&g, vp, P, Pold, NULL, NULL, NULL, 0, 0);
}

/* Laplacian operator alone (no time update), for the adjoint identity test. */
void orc_laplacian(int nzz, int nxx, int nyy, double dh, const double *f, double *out)
{
    const size_t sx = (size_t)nzz, sy = (size_t)nzz * nxx;
    const double idh2 = 1.0 / (dh * dh);
    memset(out, 0, (size_t)nzz * nxx * nyy * sizeof(double));
#pragma omp parallel for
    for (int k = 4; k < nyy - 4; ++k)
        for (int j = 4; j < nxx - 4; ++j)
            for (int i = 4; i < nzz - 4; ++i) {
                size_t c = i + j * sx + k * sy;
                out[c] = (d2_axis(f, c, sx) + d2_axis(f, c, sy) + d2_axis(f, c, 1)) * idh2;
            }
}
