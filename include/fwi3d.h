/*
 * fwi3d.h -- C ABI of the B200 wave-propagation library (libfwi3d.so).
 *
 * The library replaces the device side of FWI3D's three workflows:
 *   src/modeling  (class Modeling:  forward_solver / get_seismogram)
 *   src/migration (class Migration: forward_propagation / backward_propagation /
 *                  export_seismic)
 *   src/inversion (class Inversion: compute_gradient / optimization /
 *                  update_model)
 * All paths in citations are inside phbastosa/FWI3D.
 *
 * Conventions
 *   - Volumes are float32, z fastest, then x, then y (Fortran [nz, nx, ny]),
 *     as read by src/modeling/modeling.cu:160-162 and written by
 *     src/migration/migration.cu:115-116.
 *   - Seismograms are float32 Fortran [nt, nrec] (sample t of receiver r at
 *     t + r*nt), as written by src/modeling/modeling.cu:302-307.
 *   - Host buffers are owned by the caller; device buffers by the library.
 *     Entry points ending in _dev take device pointers instead.
 *   - Every call returns an int status (FWI_OK = 0).  No C++ exception crosses
 *     the ABI.  fwi_last_error() returns the message of the last failure.
 *   - One context per host thread; calls on one context are not re-entrant.
 *     Each context owns one CUDA stream (or uses the one set with
 *     fwi_set_stream) and its captured time-loop graphs.
 *   - The library keeps per-device state for the life of the process (kernel
 *     attributes, grid sizes, the no-alloc scratch address); cudaDeviceReset
 *     while it is loaded is not supported.
 */
#ifndef FWI3D_H
#define FWI3D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define FWI_OK 0
#define FWI_ERR_ARG 1       /* bad argument or size */
#define FWI_ERR_CUDA 2      /* CUDA runtime / driver error */
#define FWI_ERR_ALLOC 3     /* device allocation failed */
#define FWI_ERR_TIMEOUT 4   /* a bounded device wait gave up */
#define FWI_ERR_STATE 5     /* call out of order (e.g. no velocity yet) */
#define FWI_ERR_IO 6        /* file could not be opened (host helpers) */
#define FWI_ERR_NUMERIC 7   /* CFL violated or non-finite result */
#define FWI_ERR_NODEV 8     /* no CUDA device */

/* boundary treatment of the padded grid */
#define FWI_BOUNDARY_ABC 0  /* Cerjan sponge, src/modeling/modeling.cu:83-140, 395-520 */
#define FWI_BOUNDARY_RBC 1  /* random velocity pad, no damping, modeling.cu:558-673 */

/* behaviour flags (fwi_params.flags) */
#define FWI_FLAG_GRAD_DY 0x1        /* include d2/dy2 in the gradient (reference omits it,
                                       src/inversion/inversion.cu:466) */
#define FWI_FLAG_SUBTRACT_SOURCE 0x2 /* remove the source while rebuilding the forward field
                                       backwards (reference does not, migration.cu:195) */
#define FWI_FLAG_PAD_ACCUMULATE 0x4  /* accumulate the image / gradient and the illumination
                                       in the pad as well, as the reference does
                                       (migration.cu:134-202, inversion.cu:400-468).  Without
                                       it only the physical box [nb, nb+n) accumulates: the
                                       only cells that the reference's post-processing reads
                                       (reduce_boundary in migration.cu:90-97 and
                                       inversion.cu:142-146), so the image and the gradient
                                       are the same bit for bit, and the pad accumulators
                                       keep their values (zero after a reset) */

typedef struct fwi_ctx fwi_ctx;

/* Grid: the unpadded model plus the pad width.
 * Replaces Modeling::set_main_parameters / set_properties
 * (src/modeling/modeling.cu:17-34, 142-179) and Migration/Inversion's
 * nb = int(length/dh)+1 (src/migration/migration.cu:13, inversion.cu:57, 84). */
typedef struct {
    int nz, nx, ny;   /* z_samples, x_samples, y_samples */
    int nb;           /* pad cells on every side */
    float dh;         /* model_spacing [m] */
} fwi_grid;

/* Time axis and boundary. fmax is max_frequency: the Ricker peak is fmax/3
 * (src/modeling/modeling.cu:36-59). */
typedef struct {
    int nt;            /* time_samples */
    float dt;          /* time_spacing [s] */
    float fmax;        /* max_frequency [Hz] */
    int boundary;      /* FWI_BOUNDARY_ABC or FWI_BOUNDARY_RBC */
    float abc_factor;  /* abc_factor (used with FWI_BOUNDARY_ABC) */
    int max_batch;     /* shots propagated together in one launch (>= 1) */
    int flags;         /* FWI_FLAG_* */
} fwi_params;

/* Random-boundary recipe. kind 0 follows the reference
 * (src/modeling/modeling.cu:558-673: ramped Gaussian noise per pad axis plus
 * Gaussian blobs on Poisson-disk points, clamped to [vmin-varVp, vmax+varVp]);
 * kind 1 is a ramped uniform relative perturbation (|dv/v| <= ratio at the
 * outer face).  Both are deterministic functions of the seed and both cap the
 * pad at cfl_cap * the leapfrog stability velocity. */
typedef struct {
    int kind;          /* 0 = reference recipe, 1 = uniform relative */
    float ratio;       /* kind 0: blob radius scale [m] (rbc_ratio); kind 1: max |dv/v| */
    float varVp;       /* kind 0: velocity spread [m/s] (rbc_varVp) */
    float cfl_cap;     /* fraction of the stability limit (<= 0: 0.98) */
} fwi_rbc;

/* ---- lifetime ---------------------------------------------------------- */
int fwi_create(const fwi_grid *grid, const fwi_params *params, fwi_ctx **out);
int fwi_destroy(fwi_ctx *ctx);
const char *fwi_status_string(int status);
int fwi_last_error(fwi_ctx *ctx, char *buf, int buflen);
/* Run the context's work on a caller stream (cudaStream_t as void*). */
int fwi_set_stream(fwi_ctx *ctx, void *stream);
/* Padded dims, device pitch and time lag the context uses. */
int fwi_get_dims(fwi_ctx *ctx, int *nzz, int *nxx, int *nyy, int *ldz, int *tlag);

/* ---- model ------------------------------------------------------------- */
/* Unpadded model [nz,nx,ny]; padded on the GPU by edge replication
 * (replaces expand_boundary, src/modeling/modeling.cu:181-228). */
int fwi_set_velocity(fwi_ctx *ctx, const float *vp);
/* Padded model [nzz,nxx,nyy] as is (parity harnesses inject identical pads). */
int fwi_set_padded_velocity(fwi_ctx *ctx, const float *vp_padded);
int fwi_get_padded_velocity(fwi_ctx *ctx, float *vp_padded);
/* Overwrite the pad with a random boundary (replaces set_random_boundary,
 * src/modeling/modeling.cu:558-592).  Deterministic in (seed). */
int fwi_apply_random_boundary(fwi_ctx *ctx, const fwi_rbc *rbc, uint64_t seed);
/* A new random boundary for every shot, as the reference builds one per shot
 * (Migration::forward_propagation, src/migration/migration.cu:49-59;
 * Inversion::update_RBC, src/inversion/inversion.cu:204-216).  From this call
 * on, every modeling, migration or gradient call rebuilds the velocity of each
 * shot s of a batch from the clean padded model with the pad of seed
 * base_seed + s.  With max_batch > 1 each batch slot reads its own velocity
 * slot, so shots with different pads propagate in one launch and the result
 * of a shot does not depend on the batch it runs in.  rbc == NULL turns it
 * off and restores the clean padded model. */
int fwi_set_shot_random_boundary(fwi_ctx *ctx, const fwi_rbc *rbc, uint64_t base_seed);
/* The recipe behind fwi_apply_random_boundary for one seed, for checking it
 * (no counterpart in the reference, whose pads come from clock seeds): the
 * clamp bounds and the Gaussian blobs in the order the blob pass adds them,
 * five floats each (x, y, z centre [m], radius [m], signed amplitude [m/s];
 * src/modeling/modeling.cu:558-615).  At most cap blobs are written; *nblobs
 * receives the total.  The context's state does not change. */
int fwi_random_boundary_recipe(fwi_ctx *ctx, const fwi_rbc *rbc, uint64_t seed, float *vlo, float *vhi,
                               float *blobs, int cap, int *nblobs);

/* ---- geometry ---------------------------------------------------------- */
/* Source and receiver coordinates in metres (SPS/RPS, src/geometry/
 * geometry.cpp:3-47); grid index = int((c + dh/2)/dh) + nb
 * (src/modeling/modeling.cu:264-300).  rec_first/rec_count give each shot
 * its receiver range inside rx/ry/rz; NULL means every shot uses all nrec. */
int fwi_set_geometry(fwi_ctx *ctx, int nsrc, const float *sx, const float *sy, const float *sz,
                     int nrec, const float *rx, const float *ry, const float *rz,
                     const int *rec_first, const int *rec_count);
int fwi_shot_nrec(fwi_ctx *ctx, int shot, int *nrec);

/* ---- modeling ---------------------------------------------------------- */
/* Forward-model shots; seismograms are written one after another, shot s as
 * Fortran [nt, nrec_s].  Replaces Modeling::forward_solver + get_seismogram
 * (src/modeling/modeling.cu:302-322, 324-393). */
int fwi_model_shots(fwi_ctx *ctx, const int *shots, int nshots, float *seis);
int fwi_model_shots_dev(fwi_ctx *ctx, const int *shots, int nshots, float *d_seis);

/* ---- migration --------------------------------------------------------- */
/* Forward through the current (random-boundary) model, then the fused pass:
 * rebuild the source field backwards, propagate the time-reversed data and
 * accumulate image += Ps*Pr, illum += Ps^2.  data holds each shot's
 * [nt, nrec_s] seismogram one after another.  Replaces
 * Migration::forward_propagation + backward_propagation
 * (src/migration/migration.cu:49-81, 119-202). */
int fwi_rtm_shots(fwi_ctx *ctx, const int *shots, int nshots, const float *data);
int fwi_rtm_shots_dev(fwi_ctx *ctx, const int *shots, int nshots, const float *d_data);
/* Zero the padded image / gradient and illumination accumulators. */
int fwi_reset_accumulators(fwi_ctx *ctx);
/* Zero only the image / gradient accumulator and keep the illumination: the
 * reference zeroes its gradient for every gradient (inversion.cu:119) but never
 * its illumination (d_sumPs_rbc, inversion.cu:51, 145). */
int fwi_zero_image(fwi_ctx *ctx);
/* Raw padded accumulators [nzz,nxx,nyy] (either pointer may be NULL). */
int fwi_get_accumulators(fwi_ctx *ctx, float *image_padded, float *illum_padded);
/* Same, into caller device buffers [nzz,nxx,nyy] (for a cross-GPU sum of
 * shot-sharded images before the post-processing). */
int fwi_get_accumulators_dev(fwi_ctx *ctx, float *d_image_padded, float *d_illum_padded);
/* Replace the accumulators by caller device buffers [nzz,nxx,nyy] (after
 * such a sum, or to resume from a saved image). */
int fwi_set_accumulators_dev(fwi_ctx *ctx, const float *d_image_padded, const float *d_illum_padded);
/* Final image [nz,nx,ny]: crop, divide by illumination, -d2/dz2
 * (replaces Migration::export_seismic, src/migration/migration.cu:90-117). */
int fwi_rtm_image(fwi_ctx *ctx, float *image);

/* ---- inversion --------------------------------------------------------- */
/* Same fused pass with the gradient imaging condition
 * grad += dt*Pr*(d2x+d2z[+d2y])Ps*v^2 (src/inversion/inversion.cu:400-468);
 * residual holds each shot's [nt, nrec_s] obs-cal one after another. */
int fwi_gradient_shots(fwi_ctx *ctx, const int *shots, int nshots, const float *residual);
int fwi_gradient_shots_dev(fwi_ctx *ctx, const int *shots, int nshots, const float *d_residual);
/* Gradient post-processing [nz,nx,ny]: crop, divide by illumination, -d2/dz2
 * below int(zmask/dh), divide by max|g| (src/inversion/inversion.cu:142-169).
 * gmax receives max|g| before normalisation (may be NULL). */
int fwi_gradient_post(fwi_ctx *ctx, float zmask, float *grad, float *gmax);
/* Residual obs - cal and its sum of squares, accumulated in FP64 on the GPU
 * (replaces the FP32 host loop of src/inversion/inversion.cu:190-201).
 * res may be NULL. */
int fwi_residual(fwi_ctx *ctx, const float *obs, const float *cal, int64_t n, float *res,
                 double *sum_sq);
int fwi_residual_dev(fwi_ctx *ctx, const float *d_obs, const float *d_cal, int64_t n,
                     float *d_res, double *sum_sq);
/* No counterpart in the reference.  The residual and FP64 sum of squares of
 * fwi_residual_dev for callers that cannot let a library allocate device
 * memory (a latency-critical loop that cannot absorb cudaMalloc's implicit
 * device synchronisation, or an application whose own pool owns all device
 * memory).  Needs no context: d_obs, d_cal, d_res (may be NULL) and d_sum_sq
 * (one double) are caller device buffers; stream may be NULL.  The scratch is
 * a fixed 32 KiB device array inside the library, so n <= FWI_NOALLOC_MAX_N
 * (larger n returns FWI_ERR_ARG); every call on a device shares it, so calls
 * that overlap on the GPU race.  The first call on a device looks the array up
 * and should come before any stream capture. */
#define FWI_NOALLOC_MAX_N 268435456LL
int fwi_residual_noalloc(const float *d_obs, const float *d_cal, int64_t n, float *d_res,
                         double *d_sum_sq, void *stream);
/* FP64 dot product of two device vectors (gradient dot products). */
int fwi_dot_dev(fwi_ctx *ctx, const float *d_a, const float *d_b, int64_t n, double *out);

/* ---- learned preconditioner (no counterpart in the reference) ----------- */
/* A 4-layer 3-D CNN, 3 -> 16 -> 16 -> 16 -> 1 channels, 3^3 kernels, ReLU,
 * BF16 tensor-core forward/backward with FP32 accumulation and FP32 Adam.
 * Inputs are three normalised FP32 device volumes [3][nz*nx*ny] (raw
 * gradient, velocity, illumination); the output is one FP32 device volume
 * (the predicted model update).  Weights: [4][27][16 co][16 ci] FP32,
 * tap t = (dz+1) + 3(dx+1) + 9(dy+1); biases [4][16]. */
typedef struct fwi_cnn fwi_cnn;
int fwi_cnn_create(uint64_t seed, fwi_cnn **out);
int fwi_cnn_destroy(fwi_cnn *cnn);
int fwi_cnn_last_error(fwi_cnn *cnn, char *buf, int cap);
int fwi_cnn_set_stream(fwi_cnn *cnn, void *stream);
int fwi_cnn_get_weights(fwi_cnn *cnn, float *weights, float *biases);
int fwi_cnn_set_weights(fwi_cnn *cnn, const float *weights, const float *biases);
int fwi_cnn_forward(fwi_cnn *cnn, int nz, int nx, int ny, const float *d_in, float *d_out);
/* Loss 0.5 mean (f(x) - target)^2; its weight/bias gradients (host, may be
 * NULL); an Adam step with learning rate lr when lr > 0. */
int fwi_cnn_train_step(fwi_cnn *cnn, int nz, int nx, int ny, const float *d_in, const float *d_target, float lr,
                       double *loss, float *grad_w, float *grad_b);

/* ---- pipeline preprocessing -------------------------------------------- */
/* RTM input data of one shot (run/generate_input_data.py:28-46): scale the
 * Fortran [nt, nrec] gather by 1/max|d|, then taper each trace before its
 * direct-wave sample int((|x_r - x_s|/velocity + time_delay)/dt) with
 * exp(-0.5 ((t - t_r)/gstd)^2).  Host buffers; the reference script uses
 * velocity 3600 m/s, time_delay 0.18 s, gstd 30 samples. */
int fwi_prepare_rtm_input(const float *seis, float *out, int nt, int nrec, const float *rx, const float *ry,
                          float sx, float sy, float velocity, float time_delay, float dt, float gstd);

/* ---- reference file formats (host only, no device needed) --------------- */
/* catch_parameter (src/admin/admin.cpp:53-88): value of the first line that
 * starts with `key` and not with '#' or ' ' -- a prefix match -- taken from two
 * characters after '=' up to '#', spaces removed.  Missing key: empty value. */
int fwi_catch_parameter(const char *parameters_file, const char *key, char *value, int cap);
/* SPS/RPS "x,y,z" lines in metres, '#' lines skipped (src/geometry/geometry.cpp:
 * 3-47).  x == NULL returns only the count in *n. */
int fwi_read_points(const char *file, float *x, float *y, float *z, int cap, int *n);
/* Raw float32 files (import/export_binary_float, src/admin/admin.cpp:13-37). */
int fwi_read_binary(const char *file, float *buf, int64_t n);
int fwi_write_binary(const char *file, const float *buf, int64_t n);

/* ---- diagnostics ------------------------------------------------------- */
/* Runs one wait that nothing completes, bounded by limit_ms (1..2000): the
 * kernels' timeout path end to end.  Returns FWI_ERR_TIMEOUT and leaves the
 * context usable. */
int fwi_selftest_bounded_wait(fwi_ctx *ctx, int limit_ms);
/* Device time [ms] of the last call's forward and backward time loops. */
int fwi_last_timing(fwi_ctx *ctx, float *fwd_ms, float *bwd_ms);
/* Kernel launches issued by the library since creation (graph nodes count
 * once per replay). */
int fwi_launch_count(fwi_ctx *ctx, int64_t *count);
/* Stencil tile chosen by the autotuner for the forward and backward kernels
 * (index into the compiled tile table; -1 = not tuned yet). */
int fwi_get_tiles(fwi_ctx *ctx, int *fwd_tile, int *bwd_tile);
int fwi_set_tiles(fwi_ctx *ctx, int fwd_tile, int bwd_tile);
int fwi_autotune(fwi_ctx *ctx);
int fwi_num_tiles(int *n);
int fwi_tile_shape(int tile, int *tz, int *tx);

#ifdef __cplusplus
}
#endif
#endif /* FWI3D_H */
