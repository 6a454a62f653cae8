/* gmref.h -- C interface of the two comparison builds of the reference's own
 * per-pixel routines (test and benchmark infrastructure, never the product):
 *
 *   libgmref_cpu.so  the reference's device routines (lm_mils,
 *                    milosUtils.cu:574-710, and everything it calls) compiled
 *                    as host C++, one pixel per OpenMP task;
 *   libgmref_gpu.so  the same routines compiled for sm_100a with the
 *                    reference's launch geometry, streams and device heap
 *                    (gmilos.cu:1008-1249), child launches run in-thread.
 *
 * Both are built by oracle/build_ref.py from the reference's sources. */
#ifndef GMREF_H
#define GMREF_H

#ifdef __cplusplus
extern "C" {
#endif

#define GMREF_MAX_NL 50 /* MAX_LAMBDA, definesCuda.cuh */

typedef struct gmref_setup {
  int nl;                       /* wavelength samples */
  double lambda[GMREF_MAX_NL];  /* absolute wavelengths [A] (d_lambda_const) */
  double lambda0;               /* central wavelength [A] (d_wlines_const[1]) */
  double quantum[6];            /* sl, ll, jl, su, lu, ju of the line (create_cuantic input) */
  int use_psf;                  /* ConvolveWithPSF */
  double psf[GMREF_MAX_NL];     /* PSF sampled on the grid, centred at nl/2 */
  float weight[4];              /* WeightForStokes */
  float noise;                  /* noise (sigma^2 in the reference's naming) */
  float mu;                     /* heliocentric angle cosine (ah) */
  float ilambda;                /* InitialDiagonalElement */
  double toplim;
  int miter;                    /* NumberOfCycles */
  int logclambda;
  int fix[11];
  double init[11];              /* Init_Model: eta0 B vlos dopp aa gm az S0 S1 mac alfa */
} gmref_setup;

/* ---- host (OpenMP) build ---- */

/* Invert npix pixels of iquv [P][4][nl] with lm_mils, or lm_mils_11 when
 * fix[9] and fix[10] are both set.  slight: NULL, one profile [4][nl]
 * or, with slight_per_pixel, a map [P][4][nl].  Outputs: model [P][11]
 * (Init_Model layout), chi2 [P], iters [P], fitted [P][4][nl] (may be NULL).
 * nthreads <= 0 uses every OpenMP thread.  Returns 0 on success. */
int gmref_cpu_invert(const gmref_setup* s, const float* iquv, long long npix,
                     const float* slight, int slight_per_pixel, double* model,
                     float* chi2, int* iters, float* fitted, int nthreads);

/* Synthesis of one model (kernel_synthesis, gmilos.cu:71-84): profiles
 * [4][nl] and, when rf != NULL, response functions [4][nterms][nl]
 * (nterms 10 or 11). */
int gmref_cpu_synth(const gmref_setup* s, const double* model, const float* slight,
                    float* iquv, float* rf, int nterms);

/* The Zeeman pattern create_cuantic builds for the setup's quantum numbers:
 * out[0..1] = N_PI, N_SIG; out[2..61] = NUB, NUP, NUR, WEB, WEP, WER (10
 * each); out[62..65] = GL, GU, GEFF, FO. */
int gmref_cpu_cuantic(const gmref_setup* s, float* out);

int gmref_cpu_max_threads(void);

/* ---- sm_100a build ---- */

typedef struct gmref_gpu_report {
  float kernel_ms;          /* event-timed launches of all streams (gmilos.cu:1196-1220) */
  float e2e_ms;             /* H2D of the cube + launches + D2H of every output */
  int num_blocks;           /* occupancy-derived blocks per stream */
  int threads_per_block;    /* 32 */
  int n_rte_parallel;       /* num_blocks * threads_per_block */
  int nstreams;
  unsigned long long heap_bytes;
  unsigned long long stack_bytes;
  unsigned long long local_bytes;   /* per-thread local memory of lm_mils */
  int regs;                 /* registers per thread of lm_mils */
  unsigned malloc_failures; /* device-heap allocations that failed (run invalid if > 0) */
  int cuda_error;
  char msg[256];
} gmref_gpu_report;

/* Invert npix pixels with the reference's kernel on the current device.
 * Host buffers in and out, as the reference's main does. */
int gmref_gpu_invert(const gmref_setup* s, const float* iquv, long long npix,
                     const float* slight, int slight_per_pixel, int nstreams,
                     double* model, float* chi2, int* iters, float* fitted,
                     gmref_gpu_report* rep);

#ifdef __cplusplus
}
#endif
#endif
