// gmref_cpu.cpp -- host driver of the reference's per-pixel routines compiled
// as host C++ (test and benchmark infrastructure).
//
// The reference keeps its configuration in __constant__ symbols defined in
// gmilos.cu:46-68 and filled at gmilos.cu:213-239, 532-547 and 636-641; in
// this build they are ordinary globals defined here and filled from a
// gmref_setup.  lm_mils (milosUtils.cu:574-710) is then called once per
// pixel, as a one-thread "launch" whose pixel slice is that one pixel, so the
// pixels can be spread over OpenMP threads with a dynamic schedule.
#include <omp.h>

#include <mutex>

#include "definesCuda.cuh"
#include "milosUtils.cuh"
#include "gmref.h"

// ---- the reference's configuration symbols (gmilos.cu:46-68)
int d_fix_const[11];
PRECISION d_lambda_const[MAX_LAMBDA];
PRECISION d_psfFunction_const[MAX_LAMBDA];
REAL d_weight_const[4];
REAL d_weight_sigma_const[4];
PRECISION d_wlines_const[2];
Cuantic d_cuantic_const;
Init_Model d_initModel_const;
int d_nlambda_const;
PRECISION d_toplim_const;
int d_miter_const;
REAL d_sigma_const;
REAL d_ilambda_const;
int d_use_convolution_const;
REAL d_ah_const;
int d_logclambda_const;
cuDoubleComplex d_zdenV[7];
cuDoubleComplex d_zdivV[7];
int cordicPosFila[TAMANIO_SVD * TAMANIO_SVD];
int cordicPosCol[TAMANIO_SVD * TAMANIO_SVD];
PRECISION LIMITE_INFERIOR_PRECISION_SVD;
PRECISION LIMITE_INFERIOR_PRECISION_TRIG;
PRECISION LIMITE_INFERIOR_PRECISION_SINCOS;

thread_local uint3 gm_shim_threadIdx = {0, 0, 0};
thread_local uint3 gm_shim_blockIdx = {0, 0, 0};
thread_local dim3 gm_shim_blockDim = dim3(1, 1, 1);

namespace {

std::mutex g_mu;  // the symbols above are process-wide

// The round-robin order of the parallel Jacobi sweep: row r of the 10x10
// working matrix moves to row kPerm[r] after each step (the tables uploaded
// at gmilos.cu:636-637 are this permutation, by row and by column).
const int kPerm[TAMANIO_SVD] = {0, 2, 4, 1, 6, 3, 8, 5, 9, 7};

Init_Model to_model(const double* m) {
  Init_Model r;
  r.eta0 = m[0]; r.B = m[1]; r.vlos = m[2]; r.dopp = m[3]; r.aa = m[4];
  r.gm = m[5]; r.az = m[6]; r.S0 = m[7]; r.S1 = m[8]; r.mac = m[9]; r.alfa = m[10];
  return r;
}

void from_model(const Init_Model& r, double* m) {
  m[0] = r.eta0; m[1] = r.B; m[2] = r.vlos; m[3] = r.dopp; m[4] = r.aa;
  m[5] = r.gm; m[6] = r.az; m[7] = r.S0; m[8] = r.S1; m[9] = r.mac; m[10] = r.alfa;
}

int make_cuantic(const gmref_setup* s, Cuantic* out) {
  PRECISION dat[8] = {1, s->quantum[0], s->quantum[1], s->quantum[2],
                      s->quantum[3], s->quantum[4], s->quantum[5], 1};
  Cuantic* c = create_cuantic(dat, 0);
  if (!c) return -1;
  *out = c[0];
  free(c);
  return 0;
}

int upload(const gmref_setup* s) {
  if (!s || s->nl < 2 || s->nl > MAX_LAMBDA) return -1;
  const int nl = s->nl;
  for (int i = 0; i < nl; ++i) {
    d_lambda_const[i] = s->lambda[i];
    d_psfFunction_const[i] = s->psf[i];
  }
  d_wlines_const[0] = 1;
  d_wlines_const[1] = s->lambda0;
  for (int k = 0; k < 4; ++k) {
    d_weight_const[k] = s->weight[k];
    d_weight_sigma_const[k] = s->weight[k] / s->noise;
  }
  if (make_cuantic(s, &d_cuantic_const)) return -1;
  d_initModel_const = to_model(s->init);
  for (int i = 0; i < 11; ++i) d_fix_const[i] = s->fix[i];
  d_nlambda_const = nl;
  d_toplim_const = s->toplim;
  d_miter_const = s->miter;
  d_sigma_const = s->noise;
  d_ilambda_const = s->ilambda;
  d_use_convolution_const = s->use_psf;
  d_ah_const = s->mu;
  d_logclambda_const = s->logclambda;
  // Voigt rational coefficients, highest power first (gmilos.cu:220-239)
  for (int k = 0; k < 7; ++k) {
    d_zdenV[k] = make_cuDoubleComplex(a_fvoigt[6 - k], 0);
    d_zdivV[k] = make_cuDoubleComplex(b_fvoigt[6 - k], 0);
  }
  for (int r = 0; r < TAMANIO_SVD; ++r)
    for (int c = 0; c < TAMANIO_SVD; ++c) {
      cordicPosFila[r * TAMANIO_SVD + c] = kPerm[r];
      cordicPosCol[r * TAMANIO_SVD + c] = kPerm[c];
    }
  LIMITE_INFERIOR_PRECISION_SVD = pow(2.0, -39);
  LIMITE_INFERIOR_PRECISION_TRIG = pow(2.0, -39);
  LIMITE_INFERIOR_PRECISION_SINCOS = pow(2.0, -39);
  return 0;
}

}  // namespace

extern "C" int gmref_cpu_max_threads(void) { return omp_get_max_threads(); }

extern "C" int gmref_cpu_cuantic(const gmref_setup* s, float* out) {
  Cuantic c;
  if (make_cuantic(s, &c)) return -1;
  out[0] = (float)c.N_PI;
  out[1] = (float)c.N_SIG;
  for (int k = 0; k < 10; ++k) {
    out[2 + k] = c.NUB[k];
    out[12 + k] = c.NUP[k];
    out[22 + k] = c.NUR[k];
    out[32 + k] = c.WEB[k];
    out[42 + k] = c.WEP[k];
    out[52 + k] = c.WER[k];
  }
  out[62] = c.GL;
  out[63] = c.GU;
  out[64] = c.GEFF;
  out[65] = c.FO;
  return 0;
}

extern "C" int gmref_cpu_invert(const gmref_setup* s, const float* iquv, long long npix,
                                const float* slight, int slight_per_pixel, double* model,
                                float* chi2, int* iters, float* fitted, int nthreads) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (upload(s)) return -1;
  if (npix < 0 || !iquv || !model || !chi2 || !iters) return -1;
  const int nl = s->nl;
  const long long stride = 4LL * nl;
  if (stride * npix > 0x7fffffffLL) return -1;  // the reference's offsets are int
  float* trash = nullptr;  // lm_mils always writes the fitted profiles
  if (!fitted) {
    trash = (float*)malloc(sizeof(float) * stride * (npix > 0 ? npix : 1));
    if (!trash) return -1;
  }
  float* fit = fitted ? fitted : trash;
  Init_Model* out = (Init_Model*)malloc(sizeof(Init_Model) * (npix > 0 ? npix : 1));
  if (!out) { free(trash); return -1; }
  const int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
  for (long long p = 0; p < npix; ++p) {
    // a one-thread launch whose slice is pixel p: every offset the kernel
    // reads is relative to the pixel, so pass shifted base pointers
    const int displ_spectro = 0, count = 1, displ_pixel = 0;
    REAL* sl = nullptr;
    if (slight) sl = (REAL*)(slight_per_pixel ? slight + p * stride : slight);
    // the reference's main picks the 11-term kernel when both macroturbulence
    // and the filling factor are free (gmilos.cu:1016-1021, 1233-1240)
    if (s->fix[9] && s->fix[10])
      lm_mils_11(iquv + p * stride, out + p, chi2 + p, sl, iters + p, fit + p * stride,
                 &displ_spectro, &count, &displ_pixel, 1, 0, slight_per_pixel ? 1 : 0);
    else
      lm_mils(iquv + p * stride, out + p, chi2 + p, sl, iters + p, fit + p * stride,
              &displ_spectro, &count, &displ_pixel, 1, 0, slight_per_pixel ? 1 : 0);
  }
  for (long long p = 0; p < npix; ++p) from_model(out[p], model + p * 11);
  free(out);
  free(trash);
  return 0;
}

extern "C" int gmref_cpu_synth(const gmref_setup* s, const double* model_in, const float* slight,
                               float* iquv, float* rf, int nterms) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (upload(s) || !model_in || !iquv || (nterms != NTERMS && nterms != NTERMS_11)) return -1;
  const int nl = s->nl;
  Init_Model m = to_model(model_in);
  ProfilesMemory* pM = (ProfilesMemory*)malloc(sizeof(ProfilesMemory));
  InitProfilesMemoryFromDevice(nl, pM, d_cuantic_const, nterms);
  REAL cosi, sinis, sina, cosa, sinda, cosda, sindi, cosdi, cosis_2;
  int uuGlobal, FGlobal, HGlobal;
  REAL* spectra = (REAL*)calloc(4 * nl, sizeof(REAL));
  mil_sinrf(d_cuantic_const, &m, d_wlines_const, nl, spectra, d_ah_const, (const REAL*)slight,
            pM->spectra_mac, pM->spectra_slight, d_use_convolution_const, pM, &cosi, &sinis,
            &sina, &cosa, &sinda, &cosda, &sindi, &cosdi, &cosis_2, &uuGlobal, &FGlobal,
            &HGlobal);
  for (int i = 0; i < 4 * nl; ++i) iquv[i] = spectra[i];
  if (rf) {
    me_der(&d_cuantic_const, &m, d_wlines_const, nl, pM->d_spectra, pM->spectra_mac,
           pM->spectra_slight, d_ah_const, (const REAL*)slight, d_use_convolution_const, pM,
           d_fix_const, cosi, sinis, sina, cosa, sinda, cosda, sindi, cosdi, cosis_2, &uuGlobal,
           &FGlobal, &HGlobal, nterms);
    for (int i = 0; i < 4 * nterms * nl; ++i) rf[i] = pM->d_spectra[i];
  }
  free(spectra);
  FreeProfilesMemoryFromDevice(pM, d_cuantic_const);
  free(pM);
  return 0;
}
