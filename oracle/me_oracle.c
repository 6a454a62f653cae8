/*
 * me_oracle.c -- CPU oracle for the Milne-Eddington inversion path.
 * TEST INFRASTRUCTURE ONLY (see me_oracle.h): the checker, never the product.
 */
#include "me_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_MAXCOMP 30
#define ORC_PI 3.14159265358979323846264338327950288419716939937510
#define ORC_VLIGHT 2.99792458e+5       /* km/s (defines.h:83) */
#define ORC_CTE4_6_13 4.6686411e-13    /* e/(4 pi m c^2) in A^-1 G^-1 (defines.h:85) */
#define ORC_RR 0.5641895836            /* 1/sqrt(pi) as used by me_der.cu:64 */

/* Hui, Armstrong & Wray (1978) coefficients, lowest order first (the
 * published values also tabulated in definesCuda.cuh:88-111). */
static const double hui_p[7] = {122.607931777104326, 214.382388694706425,
                                181.928533092181549, 93.155580458138441,
                                30.180142196210589, 5.912626209773153,
                                0.564189583562615};
static const double hui_q[7] = {122.60793177387535, 352.730625110963558,
                                457.334478783897737, 348.703917719495792,
                                170.354001821091472, 53.992906912940207,
                                10.479857114260399};

/* Round-robin relabelling applied after every parallel Jacobi step: index i
 * moves to orc_rr_perm[i] (the rows of cordicPosFila, gmilos.cu:108-118). */
static const int orc_rr_perm[10] = {0, 2, 4, 1, 6, 3, 8, 5, 9, 7};

/* Scale applied to the dispersion-profile derivatives.  The reference's
 * d_funcionComponentFor (me_der.cu:71-74) differentiates F where the
 * synthesis uses 2F (mil_sinrf.cu:326), so its magneto-optical response
 * functions are half the true derivative; 1.0 reproduces that.  Tests set 2.0
 * to check the rest of the response functions against finite differences. */
static double orc_mo_scale = 1.0;
void orc_set_mo_scale(double s) { orc_mo_scale = s; }

/* Parameter range enforcement after a step (check, milosUtils.cu:160-238). */
static void orc_check(double *m)
{
    if (m[ORC_B] < 0) {
        m[ORC_B] = -m[ORC_B];
        m[ORC_GM] = 180.0 - m[ORC_GM];
    }
    if (m[ORC_B] > 5000) m[ORC_B] = 5000;
    if (m[ORC_GM] < 0) m[ORC_GM] = -m[ORC_GM];
    if (m[ORC_GM] > 180) m[ORC_GM] = 360.0 - m[ORC_GM];
    if (m[ORC_AZ] < 0) m[ORC_AZ] = 180 + m[ORC_AZ];
    if (m[ORC_AZ] > 180) m[ORC_AZ] = m[ORC_AZ] - 180.0;
    if (m[ORC_ETA0] < 1) m[ORC_ETA0] = 1;
    if (m[ORC_ETA0] > 2500) m[ORC_ETA0] = 2500;
    if (m[ORC_VLOS] < -20) m[ORC_VLOS] = -20;
    if (m[ORC_VLOS] > 20) m[ORC_VLOS] = 20;
    if (m[ORC_DOPP] < 0.0001) m[ORC_DOPP] = 0.0001;
    if (m[ORC_DOPP] > 0.6) m[ORC_DOPP] = 0.6;
    if (m[ORC_AA] < 0.0001) m[ORC_AA] = 0.0001;
    if (m[ORC_AA] > 10.0) m[ORC_AA] = 10.0;
    if (m[ORC_S0] < 0.0001) m[ORC_S0] = 0.0001;
    if (m[ORC_S0] > 2.00) m[ORC_S0] = 2.00;
    if (m[ORC_S1] < 0.0001) m[ORC_S1] = 0.0001;
    if (m[ORC_S1] > 2.00) m[ORC_S1] = 2.00;
    if (m[ORC_MAC] < 0) m[ORC_MAC] = 0;
    if (m[ORC_MAC] > 4) m[ORC_MAC] = 4;
    if (m[ORC_ALFA] < 0) m[ORC_ALFA] = 0.0;
    if (m[ORC_ALFA] > 1.0) m[ORC_ALFA] = 1.0;
}

/* Macroturbulence kernel: a Gaussian in wavelength of width
 * sigma = lambda0 * mac / c, sampled on the grid about its central sample
 * nl/2 and normalised to unit sum (fgauss, fgauss.cu:16-63). */
static void orc_fgauss(const orc_cfg *c, double mac, double *g)
{
    const int nl = c->nl;
    const double ild = (c->lambda0 * mac) / 2.99792458e5;
    const double lc = c->lambda[nl / 2];
    double sum = 0;
    for (int i = 0; i < nl; i++) {
        const double x = (c->lambda[i] - lc) / ild;
        const double term = (x * x) / 2;
        g[i] = term < 1e30 ? exp(-term) : 0;
    }
    for (int i = 0; i < nl; i++) sum += g[i];
    for (int i = 0; i < nl; i++) g[i] /= sum;
}

/* Derivative of the macroturbulence kernel with respect to mac,
 * g / mac * (x^2 - 1) (me_der.cu:122-129). */
static void orc_fgauss_deriv(const orc_cfg *c, double mac, const double *g, double *gd)
{
    const int nl = c->nl;
    const double ild = (c->lambda0 * mac) / 2.99792458e5;
    const double lc = c->lambda[nl / 2];
    for (int i = 0; i < nl; i++) {
        const double x = (c->lambda[i] - lc) / ild;
        gd[i] = g[i] / mac * ((x * x) - 1.0);
    }
}

/* In-place same-size correlation of a double vector with the nl-tap PSF
 * centred at nl/2, zero padded (direct_convolution_double,
 * convolution.cu:120-151): used to fold the PSF into the macroturbulence
 * kernels. */
static void orc_conv_double(double *x, int nl, const double *h)
{
    double pad[3 * ORC_MAXNL];
    const int c = nl / 2;
    for (int k = 0; k < 2 * nl; k++) pad[k] = 0;
    for (int k = 0; k < nl; k++) pad[k + c] = x[k];
    for (int k = 0; k < nl; k++) {
        double a = 0;
        for (int j = 0; j < nl; j++) a += h[j] * pad[j + k];
        x[k] = a;
    }
}

/* ---------------- reference-faithful single precision ------------------ */
#define R float
#define SFX(n) n##_f
#define SINCOS_R(x, s, c) sincosf((x), (s), (c))
#define ATAN_R atanf
#define FABS_R fabsf
#define LOG10_R log10f
#include "me_core.inc"
#undef R
#undef SFX
#undef SINCOS_R
#undef ATAN_R
#undef FABS_R
#undef LOG10_R

/* ---------------- FP64 oracle ------------------------------------------- */
#define R double
#define SFX(n) n##_d
#define SINCOS_R(x, s, c) sincos((x), (s), (c))
#define ATAN_R atan
#define FABS_R fabs
#define LOG10_R log10
#include "me_core.inc"
#undef R
#undef SFX
#undef SINCOS_R
#undef ATAN_R
#undef FABS_R
#undef LOG10_R

/* Zeeman pattern from the LS-coupling quantum numbers of the two levels:
 * Lande factors, effective Lande factor, pi / sigma_b / sigma_r components
 * with shifts g_l M_l - g_u M_u and Condon-Shortley relative strengths,
 * each group normalised to unit sum (Cuanten, create_cuantic.c:31-215).
 * Values are rounded to float where the reference stores REAL. */
void orc_cuanten(double sl, double ll, double jl, double su, double lu, double ju,
                 double fos, orc_zeeman *z)
{
    float g1 = 0, g2 = 0;
    if (jl != 0) g1 = (float)((3.0 * jl * (jl + 1) + sl * (sl + 1) - ll * (ll + 1)) / (2 * jl * (jl + 1)));
    if (ju != 0) g2 = (float)((3.0 * ju * (ju + 1.0) + su * (su + 1.0) - lu * (lu + 1.0)) / (2.0 * ju * (ju + 1.0)));
    const float geff = (float)((g1 + g2) / 2 + (g1 - g2) * (jl * (jl + 1.) - ju * (ju + 1.)) / 4);
    memset(z, 0, sizeof(*z));
    const int n1 = (int)(2 * jl + 1), n2 = (int)(2 * ju + 1);
    const int dj = (int)(ju - jl);
    int ip = 0, ib = 0, ir = 0;
    float wep[10] = {0}, web[10] = {0}, wer[10] = {0}, nup[10] = {0}, nub[10] = {0}, nur[10] = {0};
    for (int a = 0; a < n1; a++) {
        const int ml = a - (int)jl;
        for (int b = 0; b < n2; b++) {
            const int mu = b - (int)ju;
            const int dm = mu - ml;
            const float shift = g1 * ml - g2 * mu;
            if (dm == 0 && ip < 10) {
                if (dj == -1) wep[ip] = (float)(jl * jl - ml * ml);
                else if (dj == 0) wep[ip] = (float)(ml * ml);
                else if (dj == 1) wep[ip] = (float)((jl + 1) * (jl + 1) - ml * ml);
                nup[ip++] = shift;
            } else if (dm == 1 && ib < 10) {
                if (dj == -1) web[ib] = (float)((jl - ml) * (jl - ml - 1) / 4);
                else if (dj == 0) web[ib] = (float)((jl - ml) * (jl + ml + 1) / 4);
                else if (dj == 1) web[ib] = (float)((jl + ml + 1) * (jl + ml + 2) / 4);
                nub[ib++] = shift;
            } else if (dm == -1 && ir < 10) {
                if (dj == -1) wer[ir] = (float)((jl + ml) * (jl + ml - 1) / 4);
                else if (dj == 0) wer[ir] = (float)((jl + ml) * (jl - ml + 1) / 4);
                else if (dj == 1) wer[ir] = (float)((jl - ml + 1) * (jl - ml + 2) / 4);
                nur[ir++] = shift;
            }
        }
    }
    const int n_pi = (int)(2 * (jl < ju ? jl : ju)) + 1;
    const int n_sig = (int)(jl + ju);
    float sp = 0, sb = 0, sr = 0;
    for (int i = 0; i < n_pi; i++) sp = sp + wep[i];
    for (int i = 0; i < n_sig; i++) sb = sb + web[i];
    for (int i = 0; i < n_sig; i++) sr = sr + wer[i];
    for (int i = 0; i < 10; i++) {
        z->wep[i] = (i < n_pi) ? (double)(wep[i] / sp) : 0.0;
        z->web[i] = (i < n_sig) ? (double)(web[i] / sb) : 0.0;
        z->wer[i] = (i < n_sig) ? (double)(wer[i] / sr) : 0.0;
        z->nup[i] = nup[i];
        z->nub[i] = nub[i];
        z->nur[i] = nur[i];
    }
    z->n_pi = n_pi;
    z->n_sig = n_sig;
    z->gl = g1;
    z->gu = g2;
    z->geff = geff;
    z->fo = (float)fos;
}

/* Gaussian instrumental profile of the given FWHM [mA] sampled on the
 * observed step and centred on lambda_central, normalised to unit sum
 * (fgauss_WL, fgaussC.c:14-87). */
int orc_psf_gauss(double fwhm_mA, double step_A, double lambda_first,
                  double lambda_central, int n, double *out)
{
    const double sigma = fwhm_mA * 0.42466090 / 1000.0;
    double cte = 0;
    for (int i = 0; i < n; i++) {
        const double x = lambda_first + i * step_A;
        const double t = ((x - lambda_central) / sigma);
        const double term = t * t / 2;
        out[i] = (term < 1e30) ? exp(-term) : 0.0;
    }
    for (int i = 0; i < n; i++) cte += out[i];
    for (int i = 0; i < n; i++) out[i] /= cte;
    return 1;
}

/* Shift [mA] that moves the line-centre sample of the grid to index n/2 so
 * the tabulated PSF can be sampled as an n-tap kernel centred there
 * (gmilos.cu:278-288: first sample whose truncated offset is zero). */
double orc_psf_center_shift(const double *offsets_mA, int n, double step_A)
{
    int pos = 0;
    for (int i = 0; i < n && !pos; i++)
        if (fabs(trunc(offsets_mA[i])) == 0) pos = i;
    if (pos != n / 2) return (((n / 2) - pos) * step_A) * 1000;
    return 0.0;
}

/* Piecewise-linear interpolation of a tabulated PSF (x ascending, mA) at the
 * grid offsets minus the centring shift, zero outside the table, normalised
 * to unit sum (interpolationLinearPSF, interpolLineal.c:46-98; GSL's
 * gsl_interp_linear is plain two-point linear interpolation). */
int orc_psf_linear(const double *x, const double *y, int npsf,
                   const double *offsets_mA, int n, double shift_mA, double *out)
{
    for (int i = 0; i < n; i++) {
        const double q = offsets_mA[i] - shift_mA;
        double v = 0.0;
        if (npsf >= 2 && q >= x[0] && q <= x[npsf - 1]) {
            int lo = 0, hi = npsf - 1;
            while (hi - lo > 1) {
                const int mid = (lo + hi) / 2;
                if (x[mid] > q) hi = mid; else lo = mid;
            }
            const double t = (q - x[lo]) / (x[hi] - x[lo]);
            v = y[lo] + t * (y[hi] - y[lo]);
        }
        out[i] = v;
    }
    double cte = 0;
    for (int i = 0; i < n; i++) cte += out[i];
    for (int i = 0; i < n; i++) out[i] /= cte;
    return 1;
}

/* Weak-field / centre-of-gravity estimates of B, vlos, inclination and
 * azimuth from the observed Stokes profiles (estimacionesClasicas,
 * milosUtils.cu:386-563).  Leading and trailing samples with negative I are
 * skipped; the continuum is the last valid I sample. */
void orc_classical(double l0, const double *lam, int nl, const float *sp,
                   double *m, int for_init, double geff)
{
    const float *I = sp, *Q = sp + nl, *U = sp + 2 * nl, *V = sp + 3 * nl;
    int b = 0, e = nl;
    for (int i = 0; i < nl && I[i] < 0; i++) b++;
    for (int i = nl - 1; i >= 0 && I[i] < 0; i--) e--;
    const double Ic = (e > 0) ? (double)sp[e - 1] : NAN;
    double x = 0, y = 0, xv = 0, yv = 0;
    for (int i = b; i < e - 1; i++) {
        if (I[i] > -1 && V[i] > -1) {
            const double aux = Ic - (double)(I[i] + V[i]);
            const double avl = Ic - (double)I[i];
            x += aux * (lam[i] - l0);
            xv += avl * (lam[i] - l0);
            y += aux;
            yv += avl;
        }
    }
    const double lp = (fabs(y) > 1e-15) ? x / y : 0;
    x = 0;
    y = 0;
    for (int i = b; i < e - 1; i++) {
        if (I[i] > -1 && V[i] > -1) {
            const double aux = Ic - (double)(I[i] - V[i]);
            x += aux * (lam[i] - l0);
            y += aux;
        }
    }
    const double lm = (fabs(y) > 1e-15) ? x / y : 0;
    const double C = (ORC_CTE4_6_13 * (l0 * l0) * geff);
    const double Blos = (1 / C) * ((lp - lm) / 2);
    double Vlos = (ORC_VLIGHT / l0) * ((xv / yv) / 2);
    x = 0;
    y = 0;
    for (int i = b; i < e - 1; i++) {
        if (Q[i] > -1 && U[i] > -1 && V[i] > -1) {
            const double L = (double)fabsf(sqrtf(Q[i] * Q[i] + U[i] * U[i]));
            const double mm = fabs((4 * (lam[i] - l0) * L));
            x = x + (double)fabsf(V[i]) * mm;
            y = y + (double)(fabsf(V[i]) * fabsf(V[i]));
        }
    }
    y = y * fabs((3 * C * Blos));
    const double tg = fabs(sqrt(x / y));
    double grad = atan(tg);
    double gamma = grad * (180 / ORC_PI);
    if (for_init) {
        if (gamma >= 85 && gamma <= 90) grad = 85 * (ORC_PI / 180);
        if (gamma > 90 && gamma <= 95) grad = 95 * (ORC_PI / 180);
    }
    if (Blos < 0) gamma = 180 - gamma;
    double su = 0.0, sq = 0.0;
    for (int i = 0; i < nl; i++) {
        if (U[i] > -1 && Q[i] > -1) {
            if (fabs(U[i]) > 0.0001 || fabs(Q[i]) > 0.0001) {
                su += U[i];
                sq += Q[i];
            }
        }
    }
    double phi = (atan(su / sq) * 180 / ORC_PI) / 2;
    if (su > 0 && sq > 0) {
    } else if (su < 0 && sq > 0) {
        phi = phi + 180;
    } else if (su < 0 && sq < 0) {
        phi = phi + 90;
    } else if (su > 0 && sq < 0) {
        phi = phi + 90;
    }
    const double Baux = fabs(Blos / cos(grad));
    if (Vlos < -4) Vlos = -4;
    if (Vlos > 4) Vlos = 4;
    m[ORC_B] = (Baux > 4000 ? 4000 : Baux);
    m[ORC_VLOS] = Vlos;
    m[ORC_GM] = gamma;
    m[ORC_AZ] = phi;
    if (!for_init) m[ORC_S0] = Blos;
}

/* Singular value decomposition a = U diag(w) V^T of an m x n (m >= n)
 * row-major matrix by one-sided (Hestenes) Jacobi rotations in double; on
 * return a holds U.  The reference uses Golub-Reinsch (svdcmp.cu:37-234); for
 * the symmetric positive semi-definite damped normal matrix both yield the
 * same pseudo-inverse V diag(1/w) V^T up to rounding. */
void orc_svdcmp(double *a, int m, int n, double *w, double *v)
{
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) v[i * n + j] = (i == j) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 60; sweep++) {
        double off = 0.0;
        for (int p = 0; p < n - 1; p++)
            for (int q = p + 1; q < n; q++) {
                double alpha = 0, beta = 0, gamma = 0;
                for (int i = 0; i < m; i++) {
                    alpha += a[i * n + p] * a[i * n + p];
                    beta += a[i * n + q] * a[i * n + q];
                    gamma += a[i * n + p] * a[i * n + q];
                }
                if (gamma == 0.0) continue;
                const double r = fabs(gamma) / sqrt(alpha * beta);
                if (r > off) off = r;
                if (r < 1e-15) continue;
                const double zeta = (beta - alpha) / (2 * gamma);
                const double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1 + zeta * zeta));
                const double c = 1 / sqrt(1 + t * t), s = c * t;
                for (int i = 0; i < m; i++) {
                    const double x = a[i * n + p], y = a[i * n + q];
                    a[i * n + p] = c * x - s * y;
                    a[i * n + q] = s * x + c * y;
                }
                for (int i = 0; i < n; i++) {
                    const double x = v[i * n + p], y = v[i * n + q];
                    v[i * n + p] = c * x - s * y;
                    v[i * n + q] = s * x + c * y;
                }
            }
        if (off < 1e-15) break;
    }
    for (int j = 0; j < n; j++) {
        double s = 0;
        for (int i = 0; i < m; i++) s += a[i * n + j] * a[i * n + j];
        w[j] = sqrt(s);
        if (w[j] > 0)
            for (int i = 0; i < m; i++) a[i * n + j] /= w[j];
    }
}

/* ---------------- public entry points ----------------------------------- */
void orc_synth_d(const orc_cfg *c, const double *model, const double *slight,
                 double *spec, double *rf)
{
    ws_d *w = (ws_d *)malloc(sizeof(ws_d));
    synth_ws_d(c, model, slight, spec, w);
    if (rf) rf_ws_d(c, model, w->pure, slight, rf, w);
    free(w);
}

void orc_synth_f(const orc_cfg *c, const double *model, const float *slight,
                 float *spec, float *rf)
{
    ws_f *w = (ws_f *)malloc(sizeof(ws_f));
    synth_ws_f(c, model, slight, spec, w);
    if (rf) rf_ws_f(c, model, w->pure, slight, rf, w);
    free(w);
}

void orc_svdcordic_f(const float *a, float *w, float *v) { svdcordic_f(a, w, v); }
void orc_svdcordic_d(const double *a, double *w, double *v) { svdcordic_d(a, w, v); }
void orc_solve_f(const float *h, const float *beta, float *delta) { solve10_f(h, beta, delta); }

void orc_normal_f(const orc_cfg *c, const double *model, const float *obs,
                  const float *slight, float *alpha, float *beta, float *chi2)
{
    ws_f *w = (ws_f *)malloc(sizeof(ws_f));
    float *rf = (float *)malloc(sizeof(float) * 4 * 11 * ORC_MAXNL);
    float syn[4 * ORC_MAXNL];
    synth_ws_f(c, model, slight, syn, w);
    rf_ws_f(c, model, w->pure, slight, rf, w);
    fix_zero_f(c, rf);
    normal_f(c, rf, syn, obs, alpha, beta);
    *chi2 = chisqr_f(c, syn, obs);
    free(rf);
    free(w);
}

void orc_lm_step_f(const orc_cfg *c, const double *model, const float *obs,
                   const float *slight, float flambda, float *delta,
                   double *model_trial, float *chi2_trial, float *chi2_model)
{
    float alpha[121], beta[11], covar[121], d10[10];
    double dd[11];
    orc_normal_f(c, model, obs, slight, alpha, beta, chi2_model);
    if (c->nterms == 11) {
        /* the 11-term step in double (milosUtils.cu:787-792) */
        double cv[121], b11[11];
        for (int i = 0; i < 121; i++) cv[i] = (double)alpha[i];
        for (int j = 0; j < 11; j++) cv[j * 12] = (double)alpha[j * 12] * (1.0 + (double)flambda);
        for (int j = 0; j < 11; j++) b11[j] = (double)beta[j];
        solve11_f(cv, b11, dd);
        for (int j = 0; j < 11; j++) delta[j] = (float)dd[j];
    } else {
        for (int i = 0; i < 100; i++) covar[i] = alpha[i];
        for (int j = 0; j < 10; j++) covar[j * 11] = (float)((double)alpha[j * 11] * (1.0 + (double)flambda));
        solve10_f(covar, beta, d10);
        for (int j = 0; j < 10; j++) {
            delta[j] = d10[j];
            dd[j] = d10[j];
        }
        dd[10] = 0;
    }
    for (int i = 0; i < ORC_NPAR; i++) model_trial[i] = model[i];
    apply_delta_f(c, model, dd, model_trial);
    orc_check(model_trial);
    float syn[4 * ORC_MAXNL];
    ws_f *w = (ws_f *)malloc(sizeof(ws_f));
    synth_ws_f(c, model_trial, slight, syn, w);
    *chi2_trial = chisqr_f(c, syn, obs);
    free(w);
}

void orc_lm_f(const orc_cfg *c, const float *obs, const float *slight,
              double *model_out, float *chi2, int *iters, int *accepted, float *fitted)
{
    lm_core_f(c, obs, slight, model_out, chi2, iters, accepted, fitted);
}

void orc_lm_d(const orc_cfg *c, const float *obs, const float *slight,
              double *model_out, double *chi2, int *iters, int *accepted, double *fitted)
{
    double sl[4 * ORC_MAXNL];
    if (slight)
        for (int i = 0; i < 4 * c->nl; i++) sl[i] = slight[i];
    lm_core_d(c, obs, slight ? sl : NULL, model_out, chi2, iters, accepted, fitted);
}

int orc_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_lm_batch_f(const orc_cfg *c, long P, const float *obs, const float *slight,
                    int slight_per_pixel, double *model_out, float *chi2, int *iters,
                    int *accepted, float *fitted, int nthreads)
{
    const long stride = 4L * c->nl;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4)
#endif
    for (long p = 0; p < P; p++) {
        const float *sl = slight ? (slight_per_pixel ? slight + p * stride : slight) : NULL;
        lm_core_f(c, obs + p * stride, sl, model_out + p * ORC_NPAR, chi2 + p, iters + p,
                  accepted ? accepted + p : NULL, fitted ? fitted + p * stride : NULL);
    }
    (void)nthreads;
}

void orc_synth_batch_f(const orc_cfg *c, long P, const double *models, const float *slight,
                       int slight_per_pixel, float *spec, int nthreads)
{
    const long stride = 4L * c->nl;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
#endif
    for (long p = 0; p < P; p++) {
        const float *sl = slight ? (slight_per_pixel ? slight + p * stride : slight) : NULL;
        orc_synth_f(c, models + p * ORC_NPAR, sl, spec + p * stride, NULL);
    }
    (void)nthreads;
}
