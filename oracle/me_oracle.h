/*
 * me_oracle.h -- CPU oracle for the Milne-Eddington inversion path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA engine
 * is compared against; only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference legs may load it.  The engine never calls it.
 *
 * It restates, in plain C, the per-pixel arithmetic of the reference G-MILOS
 * code (file:line citations on each function in me_core.inc / me_oracle.c).
 * Two numeric modes are compiled from the same source:
 *   *_d : everything in IEEE double (the FP64 oracle),
 *   *_f : "reference-faithful" single precision: REAL=float where the
 *         reference uses float, double where it uses PRECISION=double
 *         (Voigt polynomial, convolution accumulators, model parameters).
 *
 * Parity is pinned by the reference's only shipped known-answer vector
 * (data/synthesis_gpu.per, a 30-sample synthesis with the CRISP PSF) and by
 * the reference's own per-pixel routines compiled host-side (oracle/_ref).
 */
#ifndef ME_ORACLE_H
#define ME_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAXNL 128   /* wavelength samples per pixel supported by the oracle */
#define ORC_NPAR 11     /* eta0 B vlos dopp aa gm az S0 S1 mac alfa */

/* parameter slots, same order as Init_Model (defines.h:94-106) */
enum { ORC_ETA0 = 0, ORC_B, ORC_VLOS, ORC_DOPP, ORC_AA, ORC_GM, ORC_AZ,
       ORC_S0, ORC_S1, ORC_MAC, ORC_ALFA };

/* Zeeman pattern of one line (Cuantic, defines.h:108-123) */
typedef struct {
    int n_pi, n_sig;
    double nub[10], nup[10], nur[10];   /* splittings (units of the Larmor shift) */
    double web[10], wep[10], wer[10];   /* normalised component strengths */
    double gl, gu, geff, fo;
} orc_zeeman;

/* Everything one inversion / synthesis needs (the reference keeps this in
 * __constant__ symbols, gmilos.cu:46-68). */
typedef struct {
    int nl;                        /* wavelength samples */
    int nterms;                    /* 10 (FP32 solve) or 11 (FP64 solve) */
    double lambda[ORC_MAXNL];      /* absolute wavelengths [A] */
    double lambda0;                /* line centre [A] */
    orc_zeeman z;
    int use_psf;
    double psf[ORC_MAXNL];         /* nl taps, centred at nl/2 */
    double mu;                     /* cos(theta) */
    double weight[4];              /* Stokes weights */
    double noise;                  /* sigma^2 */
    int fix[ORC_NPAR];             /* 1 = free parameter */
    double init[ORC_NPAR];         /* guess model */
    int miter;
    double ilambda;                /* initial LM diagonal factor */
    double toplim;                 /* relative chi2 stop threshold */
    int logclambda;
    int classical_init;            /* 1: classical estimates override B, vlos, gm, az */
    int alpha_rf_mixed;            /* 1: reproduce the mixed-spectrum alpha response
                                      function after an accepted step (milosUtils.cu:675) */
    double stop_dchi2;             /* > 0: also stop when an accepted step lowers chi2 by
                                      less than this (the engine's optional early stop;
                                      0 = the reference's stop rules only) */
} orc_cfg;

/* ---------------- host-side atomic / instrument helpers ----------------- */
void orc_cuanten(double sl, double ll, double jl, double su, double lu, double ju,
                 double fos, orc_zeeman *z);
int orc_psf_gauss(double fwhm_mA, double step_A, double lambda_first,
                  double lambda_central, int n, double *out);
double orc_psf_center_shift(const double *offsets_mA, int n, double step_A);
int orc_psf_linear(const double *x_mA, const double *y, int npsf,
                   const double *offsets_mA, int n, double shift_mA, double *out);

/* ---------------- forward model ---------------------------------------- */
/* spec: [4][nl]; rf (optional): [4][nterms][nl]; slight (optional): [4][nl] */
void orc_synth_d(const orc_cfg *c, const double *model, const double *slight,
                 double *spec, double *rf);
void orc_synth_f(const orc_cfg *c, const double *model, const float *slight,
                 float *spec, float *rf);

/* ---------------- pieces of the LM step -------------------------------- */
void orc_classical(double lambda0, const double *lambda, int nl, const float *spectro,
                   double *model, int for_init, double geff);
void orc_svdcordic_f(const float *a, float *w, float *v);
void orc_svdcordic_d(const double *a, double *w, double *v);
void orc_solve_f(const float *h, const float *beta, float *delta);
void orc_svdcmp(double *a, int m, int n, double *w, double *v);

/* normal equations of one state: alpha [nterms*nterms], beta [nterms], chi2 */
void orc_normal_f(const orc_cfg *c, const double *model, const float *obs,
                  const float *slight, float *alpha, float *beta, float *chi2);

/* one LM iteration from an explicit state (model, lambda_LM); delta holds
 * nterms entries (10, or 11 for the FP64 11-term step) */
void orc_lm_step_f(const orc_cfg *c, const double *model, const float *obs,
                   const float *slight, float flambda, float *delta,
                   double *model_trial, float *chi2_trial, float *chi2_model);

/* full per-pixel inversion (lm_mils / lm_mils_11) */
void orc_lm_f(const orc_cfg *c, const float *obs, const float *slight,
              double *model_out, float *chi2, int *iters, int *accepted, float *fitted);
void orc_lm_d(const orc_cfg *c, const float *obs, const float *slight,
              double *model_out, double *chi2, int *iters, int *accepted, double *fitted);

/* batch over pixels (OpenMP when built with it); obs/fitted [P][4][nl],
 * slight either [4][nl] (slight_per_pixel=0) or [P][4][nl] */
void orc_lm_batch_f(const orc_cfg *c, long P, const float *obs, const float *slight,
                    int slight_per_pixel, double *model_out, float *chi2, int *iters,
                    int *accepted, float *fitted, int nthreads);
void orc_synth_batch_f(const orc_cfg *c, long P, const double *models, const float *slight,
                       int slight_per_pixel, float *spec, int nthreads);
int orc_max_threads(void);
/* test hook: scale of the magneto-optical profile derivatives (1 = reference) */
void orc_set_mo_scale(double s);

#ifdef __cplusplus
}
#endif
#endif
