// gm_setup.cpp -- host-side set-up helpers of the C ABI: the Zeeman pattern
// of a line and the instrumental profile (PSF) sampled on the grid.
#include <cmath>
#include <cstring>

#include "gmilos.h"

extern "C" {

// Zeeman pattern from the LS quantum numbers of the lower (sl, ll, jl) and
// upper (su, lu, ju) levels: Lande factors, effective Lande factor, the pi,
// sigma_b (M_u - M_l = +1) and sigma_r (-1) components with shifts
// g_l M_l - g_u M_u and relative strengths, each group normalised to unit
// sum (Cuanten, create_cuantic.c:31-215).  Magnetic quantum numbers run over
// i - (int)J as in the reference.
gm_status gm_zeeman_from_levels(double sl, double ll, double jl, double su, double lu, double ju,
                                double fos, gm_zeeman* z) {
  if (!z || jl < 0 || ju < 0 || jl > 20 || ju > 20) return GM_ERR_INVALID;
  float g1 = 0.f, g2 = 0.f;
  if (jl != 0) g1 = (float)((3.0 * jl * (jl + 1) + sl * (sl + 1) - ll * (ll + 1)) / (2 * jl * (jl + 1)));
  if (ju != 0) g2 = (float)((3.0 * ju * (ju + 1.0) + su * (su + 1.0) - lu * (lu + 1.0)) / (2.0 * ju * (ju + 1.0)));
  std::memset(z, 0, sizeof(*z));
  const int n1 = (int)(2 * jl + 1), n2 = (int)(2 * ju + 1), dj = (int)(ju - jl);
  const int n_pi = (int)(2 * (jl < ju ? jl : ju)) + 1, n_sig = (int)(jl + ju);
  if (n_pi > 10 || n_sig > 10 || n_sig < 1) return GM_ERR_INVALID;
  int ip = 0, ib = 0, ir = 0;
  for (int a = 0; a < n1; ++a) {
    const int ml = a - (int)jl;
    for (int b = 0; b < n2; ++b) {
      const int mu = b - (int)ju;
      const float shift = g1 * ml - g2 * mu;
      switch (mu - ml) {
        case 0:
          if (ip >= 10) break;
          z->wep[ip] = (float)(dj == -1 ? jl * jl - ml * ml : dj == 0 ? (double)ml * ml
                                                                      : (jl + 1) * (jl + 1) - ml * ml);
          z->nup[ip++] = shift;
          break;
        case 1:
          if (ib >= 10) break;
          z->web[ib] = (float)(dj == -1 ? (jl - ml) * (jl - ml - 1) / 4
                               : dj == 0 ? (jl - ml) * (jl + ml + 1) / 4
                                         : (jl + ml + 1) * (jl + ml + 2) / 4);
          z->nub[ib++] = shift;
          break;
        case -1:
          if (ir >= 10) break;
          z->wer[ir] = (float)(dj == -1 ? (jl + ml) * (jl + ml - 1) / 4
                               : dj == 0 ? (jl + ml) * (jl - ml + 1) / 4
                                         : (jl - ml + 1) * (jl - ml + 2) / 4);
          z->nur[ir++] = shift;
          break;
        default:
          break;
      }
    }
  }
  float sp = 0.f, sb = 0.f, sr = 0.f;
  for (int i = 0; i < n_pi; ++i) sp += z->wep[i];
  for (int i = 0; i < n_sig; ++i) sb += z->web[i];
  for (int i = 0; i < n_sig; ++i) sr += z->wer[i];
  for (int i = 0; i < n_pi; ++i) z->wep[i] /= sp;
  for (int i = 0; i < n_sig; ++i) {
    z->web[i] /= sb;
    z->wer[i] /= sr;
  }
  z->n_pi = n_pi;
  z->n_sig = n_sig;
  z->gl = g1;
  z->gu = g2;
  z->geff = (float)((g1 + g2) / 2 + (g1 - g2) * (jl * (jl + 1.) - ju * (ju + 1.)) / 4);
  z->fo = (float)fos;
  return GM_OK;
}

// Gaussian instrumental profile of FWHM [mA] on the grid spacing, centred on
// lambda[nl/2], normalised to unit sum (fgauss_WL, fgaussC.c:14-87).
gm_status gm_psf_gaussian(double fwhm_mA, const double* lambda, int nl, double* psf) {
  if (!lambda || !psf || nl < 2 || fwhm_mA <= 0) return GM_ERR_INVALID;
  const double sigma = fwhm_mA * 0.42466090 / 1000.0;
  const double step = lambda[1] - lambda[0], centre = lambda[nl / 2];
  double sum = 0;
  for (int i = 0; i < nl; ++i) {
    const double t = ((lambda[0] + i * step) - centre) / sigma;
    const double term = t * t / 2;
    psf[i] = term < 1e30 ? std::exp(-term) : 0.0;
  }
  for (int i = 0; i < nl; ++i) sum += psf[i];
  for (int i = 0; i < nl; ++i) psf[i] /= sum;
  return GM_OK;
}

// Tabulated PSF (ascending offsets [mA], values) sampled by linear
// interpolation at the grid offsets, shifted so that the line-centre sample
// falls on index nl/2, zero outside the table, normalised to unit sum
// (gmilos.cu:246-296 with interpolationLinearPSF, interpolLineal.c:46-98).
gm_status gm_psf_from_table(const double* x, const double* y, int ntab, const double* offsets_mA,
                            int nl, double step_mA, double* psf) {
  if (!x || !y || !offsets_mA || !psf || ntab < 2 || nl < 2) return GM_ERR_INVALID;
  int pos = 0;
  for (int i = 0; i < nl && !pos; ++i)
    if (std::fabs(std::trunc(offsets_mA[i])) == 0) pos = i;
  const double shift = (pos != nl / 2) ? (((nl / 2) - pos) * (step_mA / 1000.0)) * 1000 : 0.0;
  double sum = 0;
  for (int i = 0; i < nl; ++i) {
    const double q = offsets_mA[i] - shift;
    double v = 0.0;
    if (q >= x[0] && q <= x[ntab - 1]) {
      int lo = 0, hi = ntab - 1;
      while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        if (x[mid] > q) hi = mid; else lo = mid;
      }
      v = y[lo] + (q - x[lo]) / (x[hi] - x[lo]) * (y[hi] - y[lo]);
    }
    psf[i] = v;
    sum += v;
  }
  if (!(sum > 0)) return GM_ERR_INVALID;
  for (int i = 0; i < nl; ++i) psf[i] /= sum;
  return GM_OK;
}

}  // extern "C"
