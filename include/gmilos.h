/*
 * gmilos.h -- C ABI of the B200 Milne-Eddington inversion engine.
 *
 * The engine is a drop-in for the two device paths of G-MILOS: the per-pixel
 * Levenberg-Marquardt inversion (the __global__ lm_mils / lm_mils_11 kernels,
 * milosUtils.cuh:54-60, launched at gmilos.cu:1233-1240) and the single-model
 * synthesis with response functions (kernel_synthesis, gmilos.cu:71-84,
 * launched at gmilos.cu:557-562).  The reference passes its configuration
 * through ~20 __constant__ symbols uploaded at gmilos.cu:1184-1198; here it is
 * one gm_config struct handed to gm_configure.
 *
 * Conventions
 *  - every call returns a gm_status and never exits the process;
 *  - handles are opaque; the caller owns every buffer it passes;
 *  - pointers may be host (pageable or pinned) or device memory: the engine
 *    checks with cudaPointerGetAttributes and copies host data itself;
 *  - `stream` is a cudaStream_t passed as void* (NULL = the context's stream);
 *    calls on host buffers return after the results are in host memory,
 *    calls on device buffers are stream-ordered and return after launch;
 *  - one context per host thread, or serialise calls on a shared context
 *    (the serving entry points gm_submit / gm_poll / gm_cancel are
 *    internally locked and may be called from any thread); inversions of a
 *    context on different streams run one after another on the device, as
 *    they share its scratch.
 *
 * Layouts (all float32 unless stated; pixel-major like the reference's
 * spectroImagen, gmilos.cu:1200):
 *   Stokes cube  iquv [P][4][nl]     (I, Q, U, V rows per pixel)
 *   model        [P][11]             eta0, B [G], vlos [km/s], dopp [A],
 *                                    damping, gamma [deg], phi [deg], S0, S1,
 *                                    vmac [km/s], alpha (filling factor)
 *   response fn  rf [P][4][nterms][nl]
 */
#ifndef GMILOS_H
#define GMILOS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GM_MAX_NL 64          /* wavelength samples per pixel (reference: MAX_LAMBDA 50) */
#define GM_NPAR 11
#define GM_ABI_VERSION 3

typedef enum {
    GM_OK = 0,
    GM_ERR_INVALID = 1,       /* bad argument or configuration */
    GM_ERR_CUDA = 2,          /* CUDA runtime error (see gm_last_error) */
    GM_ERR_NOMEM = 3,         /* allocation failed or request exceeds the HBM budget */
    GM_ERR_NOT_CONFIGURED = 4,
    GM_ERR_UNSUPPORTED = 5,   /* feature not available in this build / configuration */
    GM_ERR_TIMEOUT = 6,       /* gm_poll waited its full timeout */
    GM_ERR_CANCELLED = 7,
    GM_ERR_IO = 8             /* file could not be read or written */
} gm_status;

/* per-pixel status bits written by gm_invert */
#define GM_PIX_INIT_NAN      0x01u  /* a classical estimate was NaN and was replaced
                                       (milosUtils.cu:621-628) */
#define GM_PIX_MAXITER       0x02u  /* stopped at the iteration limit */
#define GM_PIX_LAMBDA_EXIT   0x04u  /* stopped because lambda_LM left [1e-25, 1e7] */
#define GM_PIX_CHI2_EXIT     0x08u  /* stopped by the relative-chi2 or chi2 < 1e-4 rule */
#define GM_PIX_NONFINITE     0x10u  /* final chi2 not finite */
#define GM_PIX_BAD_INPUT     0x20u  /* no valid continuum sample in Stokes I */
#define GM_PIX_LEARNED_INIT  0x40u  /* the start model came from the learned initial guess
                                       (its chi2 beat the classical start's) */

typedef enum {
    GM_INIT_CLASSICAL = 0,    /* reference: guess model + classical estimates of B, vlos,
                                 gamma, phi (milosUtils.cu:616-628) */
    GM_INIT_GIVEN = 1,        /* guess model as given, no estimates */
    GM_INIT_PER_PIXEL = 2,    /* caller supplies init_models [P][11] to gm_invert_ex */
    GM_INIT_LEARNED = 3       /* per pixel the better (lower chi2) of the classical start
                                 and the learned initial guess gm_config.mlp; no
                                 counterpart in the reference */
} gm_init_mode;

/* Learned initial guess: a multilayer perceptron 4 nl -> 256 -> 256 -> 9
 * (GELU, tanh form), nl <= 32 (120 inputs on the 30-sample grid), that maps a pixel's
 * Stokes profiles to a start model.  Inputs are the profiles [4][nl] in the
 * cube's order, standardised per feature (x' = (x - in_mean) * in_scale,
 * zero past 4 nl).  The 9 outputs, standardised the same way (y = y' *
 * out_scale + out_mean), are eta0, vlos [km/s], Doppler width [A], damping,
 * S0, S1, and the field as B cos gamma, B sin gamma cos 2 phi,
 * B sin gamma sin 2 phi [G] (continuous across the 180-degree azimuth
 * ambiguity).  The parameters are kept in FP32 here; the engine's kernels
 * compute with BF16 copies of the weights and FP32 accumulation on the
 * tensor cores.  No counterpart in the reference. */
#define GM_MLP_IN 128
#define GM_MLP_HIDDEN 256
#define GM_MLP_OUT 9
#define GM_MLP_OUT_PAD 16
typedef struct {
    int abi_version;                              /* GM_ABI_VERSION */
    int nl;                                       /* samples per Stokes parameter read */
    int64_t steps;                                /* optimiser steps taken */
    float in_mean[GM_MLP_IN], in_scale[GM_MLP_IN];
    float out_mean[GM_MLP_OUT_PAD], out_scale[GM_MLP_OUT_PAD];
    float w1[GM_MLP_HIDDEN][GM_MLP_IN];           /* [out][in], inputs past 4 nl unused */
    float b1[GM_MLP_HIDDEN];
    float w2[GM_MLP_HIDDEN][GM_MLP_HIDDEN];
    float b2[GM_MLP_HIDDEN];
    float w3[GM_MLP_OUT][GM_MLP_HIDDEN];
    float b3[GM_MLP_OUT_PAD];
} gm_mlp;

/* Zeeman pattern of the line (Cuantic, defines.h:108-123) */
typedef struct {
    int n_pi, n_sig;
    float nub[10], nup[10], nur[10];
    float web[10], wep[10], wer[10];
    float gl, gu, geff, fo;
} gm_zeeman;

/* Everything the reference's __constant__ symbols carry (gmilos.cu:46-68). */
typedef struct {
    int abi_version;              /* GM_ABI_VERSION */
    int nl;                       /* wavelength samples, 1..GM_MAX_NL */
    double lambda0;               /* line centre [A] (d_wlines_const[1]) */
    double lambda[GM_MAX_NL];     /* absolute wavelengths [A] (d_lambda_const) */
    gm_zeeman zeeman;             /* d_cuantic_const */
    int use_psf;                  /* d_use_convolution_const */
    double psf[GM_MAX_NL];        /* nl taps centred at nl/2 (d_psfFunction_const) */
    float mu;                     /* d_ah_const */
    float weight[4];              /* d_weight_const */
    float noise;                  /* sigma^2, d_sigma_const */
    int fix[GM_NPAR];             /* 1 = free (d_fix_const) */
    double init_model[GM_NPAR];   /* d_initModel_const */
    int init_mode;                /* gm_init_mode */
    int miter;                    /* d_miter_const */
    float ilambda;                /* d_ilambda_const */
    double toplim;                /* d_toplim_const */
    int logclambda;               /* d_logclambda_const */
    double stop_dchi2;            /* >0: extra per-pixel stop when the accepted
                                     chi2 improves by less than this (absolute);
                                     0 = reference stop rule only */
    int use_slight;               /* stray-light mixing on */
    int slight_per_pixel;         /* 0: one profile slight[4][nl]; 1: map [P][4][nl] */
    const float *slight;          /* profile (copied at gm_configure when global) */
    int reference_quirks;         /* 1 (default): reproduce the reference's numerics
                                     exactly where it deviates from the textbook
                                     derivative (alpha RF of the mixed profile after
                                     an accepted step, milosUtils.cu:675) */
    int numerics;                 /* GM_NUMERICS_REFERENCE (default) or
                                     GM_NUMERICS_ACCURATE */
    int lambda_per_pixel;         /* 0: every pixel on `lambda`; 1: pixel p on
                                     lambda_map[p][0..nl) (read at each call, like
                                     the per-pixel stray map).  The PSF taps stay
                                     those of `psf`.  The reference's per-pixel
                                     wavelength FITS (utilsFits.c:1488-1500). */
    const double *lambda_map;     /* [P][nl] absolute wavelengths [A], host or device */
    int kernel;                   /* GM_KERNEL_AUTO (default): the fused kernel
                                     for calls of fewer than 16384 pixels (32768
                                     without a PSF), else the wave-synchronous
                                     kernels where they cover the call;
                                     GM_KERNEL_FUSED: the fused persistent kernel
                                     for every call (the kernel of
                                     gm_invert_noalloc); GM_KERNEL_WAVES: the
                                     wave kernels wherever they cover the call */
    const gm_mlp *mlp;            /* network of GM_INIT_LEARNED (host memory, copied
                                     at gm_configure; its nl must be the grid's) */
} gm_config;

/* Inversion kernels (gm_config.kernel).  Both execute the same LM arithmetic;
 * compiled as different kernels they round differently at the float level. */
#define GM_KERNEL_AUTO 0
#define GM_KERNEL_FUSED 1
#define GM_KERNEL_WAVES 2

/* Trigonometry of the 10x10 Jacobi solve and of the field angles.
 * REFERENCE uses the hardware approximations the reference uses
 * (__sincosf, __fdividef; svdcordic.cu:38,97); their absolute error of a few
 * 1e-7 is amplified by the badly scaled normal matrix into step differences
 * of ~1e-3, so only this mode follows the reference's LM trajectories.
 * ACCURATE uses correctly rounded sincosf/atanf and IEEE division there. */
#define GM_NUMERICS_REFERENCE 0
#define GM_NUMERICS_ACCURATE 1

typedef struct gm_ctx gm_ctx;

/* ---------------- lifecycle ---------------------------------------------- */
gm_status gm_create(int device, size_t hbm_budget, gm_ctx **out);
gm_status gm_destroy(gm_ctx *ctx);
const char *gm_last_error(gm_ctx *ctx);
const char *gm_status_string(gm_status s);
void gm_config_defaults(gm_config *cfg);

/* ---------------- configuration ------------------------------------------ */
gm_status gm_configure(gm_ctx *ctx, const gm_config *cfg);

/* ---------------- the two reference paths -------------------------------- */
/* Invert P pixels (replaces lm_mils / lm_mils_11).  fitted (optional) receives
 * the last trial synthesis per pixel, as the reference's spectraAdjusted
 * (milosUtils.cu:658).  status (optional) receives GM_PIX_* bits.
 *
 * Kernels: inversions run wave-synchronously -- per LM trial, one kernel for the
 * trials of every pixel still iterating and one for the response functions and
 * normal equations of the accepted ones, over chunks of up to 2^20 pixels
 * whose LM state (about 4 KB per pixel at nl <= 32, 7.4 KB above) the
 * context keeps in device memory within its HBM budget.  First-step outputs
 * (gm_lm_step), in-kernel classical estimates (gm_invert_noalloc), calls of
 * fewer than 16384 pixels (32768 without a PSF; GM_KERNEL_AUTO) and calls
 * whose budget leaves room for fewer than 16384 pixels of state run one fused
 * persistent kernel.  Both execute the same LM arithmetic; compiled
 * as different kernels they round differently at the float level, so their
 * trajectories agree to rounding.  gm_config.kernel = GM_KERNEL_FUSED
 * selects the fused kernel for every call (for comparisons). */
gm_status gm_invert(gm_ctx *ctx, const float *iquv, int64_t npix, int nl,
                    float *model, float *chi2, int *iters, float *fitted,
                    uint32_t *status, void *stream);

/* Extended form: per-pixel initial models, FP64 model output in the
 * reference's Init_Model layout, accepted-step counts. Any pointer may be NULL. */
gm_status gm_invert_ex(gm_ctx *ctx, const float *iquv, int64_t npix, int nl,
                       const double *init_models, float *model, double *model_f64,
                       float *chi2, int *iters, int *accepted, float *fitted,
                       uint32_t *status, void *stream);

/* Inversion for callers that cannot allocate device memory (the fused kernel,
 * its results those of gm_invert with gm_config.kernel = GM_KERNEL_FUSED).  No
 * counterpart in the reference.  Some callers cannot call cudaMalloc while
 * they run: a real-time pipeline (a telescope's on-line reduction loop, say)
 * that must not stall on the allocator, which can synchronise the device and
 * take milliseconds, or a host framework that owns every device byte through
 * its own pool and whose accounting would break if the library allocated
 * behind its back.  This entry point allocates nothing: it takes the
 * configuration directly (no gm_ctx) and only device pointers (inputs
 * [P][4][nl], outputs as in gm_invert; fitted, chi2, iters, status may be
 * NULL; a per-pixel stray map must be device memory, a single stray profile
 * may be host or device memory and is copied on `stream` by every call).
 * Its scratch -- the work-stealing counters and the single stray-light
 * profile -- lives in one file-scope device array of GM_NOALLOC_SCRATCH_BYTES
 * that every GPU loading the library keeps until the process exits; requests
 * needing more are rejected with GM_ERR_INVALID.  The first call on a device
 * (with that device current) looks up that array's address and loads the
 * inversion kernels; later calls do neither.  Every call clears the counters
 * it needs before its launch.  All calls share the array and it keeps the
 * last call's contents: calls that overlap on the GPU race, so serialise them
 * (one stream, or events).  Errors are reported by status only:
 * GM_ERR_INVALID (bad configuration, host pointer, or scratch over the
 * maximum), GM_ERR_UNSUPPORTED (per-pixel wavelength grids), GM_ERR_CUDA. */
#define GM_NOALLOC_SCRATCH_BYTES 4096
gm_status gm_invert_noalloc(const gm_config *cfg, const float *iquv, int64_t npix, int nl,
                            float *model, float *chi2, int *iters, float *fitted,
                            uint32_t *status, void *stream);

/* One Levenberg-Marquardt iteration from explicit per-pixel states
 * (models [P][11], damping flambda): the step delta [P][nterms] (10, or 11
 * when v_mac and alpha are both free) from the damped
 * normal equations, the trial model [P][11] after step limits and range
 * checks, and chi2 of the start and trial models (milosUtils.cu:645-660).
 * Any output may be NULL. */
gm_status gm_lm_step(gm_ctx *ctx, const float *iquv, int64_t npix, int nl,
                     const double *models, float flambda, float *delta, double *trial,
                     float *chi2_start, float *chi2_trial, void *stream);

/* Synthesis with optional response functions for P models [P][11] (float or
 * the FP64 Init_Model layout via gm_synthesize_f64); rf [P][4][nterms][nl]
 * with nterms = 10 (11 when both vmac and alpha are free). */
gm_status gm_synthesize(gm_ctx *ctx, const float *models, int64_t npix, float *iquv,
                        float *rf, void *stream);
/* Classical estimates only (the reference's NumberOfCycles < 0 mode,
 * gmilos.cu:309-431): models [P][11] (Init_Model layout) = the configured
 * guess model with B, vlos, gamma, phi from the weak-field and
 * centre-of-gravity estimates (estimacionesClasicas, milosUtils.cu:386-563,
 * non-initialisation use) and S0 = the longitudinal field. */
gm_status gm_classical(gm_ctx *ctx, const float *iquv, int64_t npix, int nl, double *models,
                       void *stream);
gm_status gm_synthesize_f64(gm_ctx *ctx, const double *models, int64_t npix, float *iquv,
                            float *rf, void *stream);

/* ME profiles without PSF or stray light on an arbitrary grid of offsets from
 * lambda0 (any length); used for data generation on fine grids. */
gm_status gm_synthesize_grid(gm_ctx *ctx, const double *models, int64_t npix,
                             const double *offsets_A, int ngrid, float *iquv, void *stream);

/* ---------------- ragged batches ------------------------------------------ */
/* A batch of regions of interest, each with its own size and wavelength
 * grid, inverted by one persistent wave-synchronous launch sequence per
 * samples-per-lane class (grids of <= 32 samples, grids of 33..64; the two
 * run concurrently): every pixel carries its grid's index and its profiles'
 * offset, and a warp reloads the grid's constants (offsets, PSF taps) when
 * it moves to a pixel of another grid, so ROIs of any size and grid share
 * the work-stealing waves and pixels that converge early leave them.  The
 * context's configuration supplies everything but the grids and PSF taps
 * (classical start models; no stray light, no learned guess, no per-pixel
 * grids).  The reference inverts one cube on one grid per run
 * (gmilos.cu:1008-1249); no counterpart. */
typedef struct {
    const float *iquv;            /* [P][4][nl] host or device */
    int64_t npix;
    int nl;                       /* 2..GM_MAX_NL */
    const double *lambda;         /* [nl] absolute wavelengths [A] (host) */
    const double *psf;            /* [nl] taps centred at nl/2 (host), or NULL: no PSF */
    float *model;                 /* [P][11] */
    float *chi2;                  /* [P] (optional) */
    int *iters;                   /* [P] (optional) */
    uint32_t *status;             /* [P] (optional) */
} gm_roi;

typedef struct {
    int use_graph;                /* capture the device work of a batch in a CUDA
                                     graph and replay it for later batches of the
                                     same layout (sizes, grids) */
    int autotune;                 /* on the first batch of a layout, time the
                                     resident-block limits of the two wave kernels
                                     (full, 3/4, 1/2) and keep the fastest */
} gm_batch_opts;

typedef struct {
    int64_t pixels;
    int grids;                    /* distinct wavelength grids (with their taps) */
    int launches;                 /* engine kernels launched (inside the graph too) */
    int graph_replayed;           /* 1: the device work was a replayed graph */
    int cap_trial, cap_accept;    /* resident blocks per SM used (tuned or full) */
    float device_ms;              /* device time of the batch's kernels */
    double lane_occupancy;        /* wavelength samples over lane slots, weighted by
                                     each pixel's trials (sum nl (it + 1) over
                                     sum 32 LPL (it + 1)) */
} gm_batch_stats;

gm_status gm_invert_rois(gm_ctx *ctx, const gm_roi *rois, int nroi, const gm_batch_opts *opts,
                         gm_batch_stats *stats, void *stream);

/* ---------------- serving (continuous batching) --------------------------- */
/* Requests (frames or ROIs of any size) are admitted in arrival order as
 * slots and device memory free up: at most max_active at a time, their
 * staging within the context's HBM budget.  Admitted requests are cut into
 * chunks of chunk_pixels; `streams` lanes each keep one chunk on the device,
 * taken from the admitted requests by the serving policy (below), so the
 * work of requests that arrive while others run overlaps on the device.
 * Each lane keeps one chunk of wave-kernel state and classical start models
 * on the device (about 270 MB per lane at the default chunk and
 * nl <= 32), so a served pixel runs the kernels of gm_invert and its result
 * is the one gm_invert gives, whatever the mix.  Requests share
 * the configured stray-light profile and wavelength grid: a configuration
 * with per-pixel stray maps or per-pixel grids is refused with
 * GM_ERR_UNSUPPORTED.  No counterpart in the reference (its main inverts one
 * cube per process run). */
typedef uint64_t gm_ticket;
typedef struct {
    const float *iquv;            /* [P][4][nl] host or device */
    int64_t npix;
    int nl;
    float *model;                 /* [P][11] */
    float *chi2;                  /* [P] (optional) */
    int *iters;                   /* [P] (optional) */
    uint32_t *status;             /* [P] (optional) */
    const int *fix;               /* optional per-request free mask [11] */
    double *latency_ms;           /* optional out: submit -> results in place */
    double *queue_ms;             /* optional out: submit -> first chunk launched */
} gm_request;

/* before the first gm_submit: lanes (1..32, default 4), pixels per chunk
 * (default 65536), admitted requests at a time (default 16) */
gm_status gm_serving_options(gm_ctx *ctx, int streams, int64_t chunk_pixels, int max_active);
/* Which admitted request a free lane serves next (any time):
 * GM_SERVE_ROUND_ROBIN -- the admitted requests in turn, so each
 *   progresses at the same rate and a request's latency grows with its size;
 * GM_SERVE_FIFO -- the earliest submitted first, so requests finish in
 *   arrival order and under load every request waits about as long;
 * GM_SERVE_SHORTEST_FIRST -- the fewest pixels left first (the lowest mean
 *   latency; large requests wait behind small ones);
 * GM_SERVE_RESPONSE_RATIO (default) -- the highest ratio of time since
 *   submission to the request's pixels first (highest response ratio next):
 *   small requests go first as with shortest-first, but a request's
 *   priority grows while it waits, so large requests are not starved. */
#define GM_SERVE_ROUND_ROBIN 0
#define GM_SERVE_FIFO 1
#define GM_SERVE_SHORTEST_FIRST 2
#define GM_SERVE_RESPONSE_RATIO 3
gm_status gm_serving_policy(gm_ctx *ctx, int policy);
gm_status gm_submit(gm_ctx *ctx, const gm_request *req, gm_ticket *ticket);
/* wait for a request (timeout_us < 0: no limit); consumes the ticket */
gm_status gm_poll(gm_ctx *ctx, gm_ticket ticket, int timeout_us);
/* cancel a request that has not been admitted yet */
gm_status gm_cancel(gm_ctx *ctx, gm_ticket ticket);

/* ---------------- host helpers mirroring the reference's set-up ---------- */
/* Zeeman pattern from LS quantum numbers (create_cuantic.c:31-215) */
gm_status gm_zeeman_from_levels(double sl, double ll, double jl, double su, double lu,
                                double ju, double fos, gm_zeeman *out);
/* Gaussian PSF of FWHM [mA] on the grid, centred at lambda[nl/2] (fgaussC.c:14-87) */
gm_status gm_psf_gaussian(double fwhm_mA, const double *lambda, int nl, double *psf);
/* Tabulated PSF (offsets [mA], values) linearly interpolated at the grid
 * offsets [mA] and centred at nl/2 (gmilos.cu:246-296, interpolLineal.c:46-98) */
gm_status gm_psf_from_table(const double *x_mA, const double *y, int ntab,
                            const double *offsets_mA, int nl, double step_mA, double *psf);

/* ---------------- introspection ------------------------------------------ */
typedef struct {
    int64_t pixels;               /* pixels of the last gm_invert */
    int64_t iterations;           /* sum of LM trials */
    int64_t accepted;             /* sum of accepted steps */
    float kernel_ms;              /* device time of the last inversion kernel */
    int grid_blocks, block_threads, warps_per_block;
    int kernel_launches;          /* engine kernels launched by the last call */
} gm_stats;
gm_status gm_get_stats(gm_ctx *ctx, gm_stats *out);

/* Measured arithmetic peaks of this device (FFMA and DFMA issue-bound
 * microbenchmarks, TFLOP/s counting an FMA as 2 flops) -- the denominators of
 * the engine's roofline fraction.  Measurement helper, no reference
 * counterpart. */
gm_status gm_measure_peaks(gm_ctx *ctx, double *fp32_tflops, double *fp64_tflops);
/* Special-function-unit throughput (MUFU operations, G ops/s) from chains of
 * the PTX base-2 exponential; the SFU side of the roofline.  No counterpart
 * in the reference. */
gm_status gm_measure_sfu_peak(gm_ctx *ctx, double *gops);

/* Device bytes of wave-synchronous inversion state for a chunk of `pixels`
 * pixels on a grid of nl samples with at most miter iterations: what an
 * inversion of that many pixels (one chunk) adds to its cube and outputs,
 * and what a context's HBM budget must leave room for (at least 16384 pixels'
 * worth, else the fused kernel runs).  0 for nl outside 1..GM_MAX_NL or a
 * negative count.  No counterpart in the reference; needs no device. */
size_t gm_wave_state_bytes(int nl, int miter, int64_t pixels);

/* ---------------- learned initial guess (no reference counterpart) -------- */
/* A fresh network for grids of nl samples (nl <= 32): identity
 * standardisation, weights drawn from `seed` (uniform, variance 2 / fan-in),
 * zero biases.  Host only, needs no device. */
gm_status gm_mlp_init(gm_mlp *net, int nl, uint64_t seed);

typedef struct {
    int epochs;                   /* passes over the training set (default 8) */
    int batch;                    /* pixels per optimiser step, a multiple of 128
                                     (default 16384) */
    float lr;                     /* peak Adam learning rate, cosine decay to 0
                                     (default 2e-3) */
    float weight_decay;           /* decoupled (AdamW) decay (default 0) */
    uint64_t seed;                /* shuffling */
} gm_mlp_train_opts;
void gm_mlp_train_defaults(gm_mlp_train_opts *o);

/* Train `net` in place on n pixels: Stokes profiles iquv [n][4][nl] and the
 * models that made them, truth [n][11] (Init_Model layout); host or device
 * memory.  Every forward and backward pass runs on the device in the
 * engine's own tensor-core kernels (BF16 operands, FP32 accumulation, Adam on
 * FP32 parameters).  An untrained net (steps == 0) first takes its
 * standardisation from the data.  loss_per_epoch (optional, [epochs]): mean
 * squared error of the standardised outputs over each epoch.  n must be at
 * least one batch.  Profiles in device memory must start on a 16-byte
 * boundary (the kernels read them in 16-byte vectors), as must the cube of
 * an inversion that starts from the learned guess (GM_INIT_LEARNED);
 * otherwise the call fails before the network runs (GM_ERR_INVALID here and
 * in gm_mlp_predict, GM_ERR_CUDA "invalid argument" from an inversion). */
gm_status gm_mlp_train(gm_ctx *ctx, gm_mlp *net, const float *iquv, const double *truth,
                       int64_t n, const gm_mlp_train_opts *opts, float *loss_per_epoch);

/* Loss and gradients of one batch (n a multiple of 128) without an update,
 * in `grads` (same layout as the network; its weight and bias arrays are
 * written).  For checks of the training kernels. */
gm_status gm_mlp_gradients(gm_ctx *ctx, const gm_mlp *net, const float *iquv, const double *truth,
                           int64_t n, gm_mlp *grads, float *loss);

/* Start models [n][11] (Init_Model layout) predicted by `net` for the
 * profiles iquv [n][4][nl]: the 9 outputs mapped back to the model
 * parameters within the reference's ranges (milosUtils.cu:160-238); v_mac
 * and the filling factor from the configured guess model.  The context must
 * be configured on a grid of net->nl samples. */
gm_status gm_mlp_predict(gm_ctx *ctx, const gm_mlp *net, const float *iquv, int64_t n,
                         double *models, void *stream);

#ifdef __cplusplus
}
#endif
#endif
