// gm_device.cuh -- device building blocks of the Milne-Eddington engine.
//
// Mapping: one warp inverts one pixel; lane l owns wavelength samples
// l, l+32 (LPL = samples per lane, 1 for nl <= 32, 2 for nl <= 64).  All
// per-pixel scalars (model, LM state) are warp-uniform.  The arithmetic
// follows the reference's precision choices: FP32 with the same fast
// intrinsics (__fdividef, __sincosf), FP64 for the Voigt polynomials and
// wherever the reference keeps PRECISION=double (model parameters,
// classical estimates, the PSF convolution).  The PSF convolution of the
// staged rows runs on the FP64 tensor cores (mma.sync m8n8k4); the normal
// equations are FP32 sums with warp-level reductions, as the reference
// forms them in FP32.  file:line citations name the reference code each
// piece reproduces.
#pragma once

#include <cstdint>
#include <utility>
#include <cuda_runtime.h>

#include "gmilos.h"

namespace gm {

constexpr int kMaxNl = 64;
constexpr unsigned kFull = 0xffffffffu;
constexpr double kPi = 3.14159265358979323846264338327950288419716939937510;
constexpr double kVlight = 2.99792458e+5;      // km/s
constexpr double kLarmor = 4.6686411e-13;      // A^-1 G^-1
constexpr double kRR = 0.5641895836;           // 1/sqrt(pi) as the reference rounds it

enum { ETA0 = 0, BFLD, VLOS, DOPP, AA, GM, AZ, S0, S1, MAC, ALFA };

// Per-configuration constants, passed by value as a kernel parameter (lives
// in the constant bank: uniform reads are free).
struct DevCfg {
  int nl, nterms;
  int use_psf, use_slight, slight_per_pixel;
  int init_mode, miter, logclambda, quirks;
  int numerics;          // 0: reference intrinsics, 1: accurate trigonometry
  int n_pi, n_sig;
  int fix[11];
  float dl[kMaxNl];      // (float)(lambda - lambda0), the reference's sub_aux
  double dld[kMaxNl];    // lambda - lambda0 in double (classical estimates)
  double psfd[kMaxNl];   // PSF taps (double, as the reference's psfFunction)
  double lam[kMaxNl];    // absolute wavelengths (macroturbulence kernel)
  float nup[10], nub[10], wep[10], web[10], wer[10];
  float geff, fo, mu, ilambda, noise;
  float weight[4];
  float wsig[4];         // weight / noise (gmilos.cu:1126-1129)
  double lambda0, toplim, stop_dchi2;
  double init[11];
  const float* slight;   // device [4][nl] or [P][4][nl]
  int lambda_per_pixel;  // 1: pixel p's absolute wavelengths are lam_map[p][0..nl)
  const double* lam_map; // device [P][nl] (per-pixel grids) or null
};

// --------------------------------------------------------------- warp utils
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}
__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

// sin and cos as the reference takes them (__sincosf, absolute error of a few
// 1e-7) or correctly rounded (accurate numerics)
__device__ __forceinline__ void sincos_mode(float x, float* s, float* c, bool accurate) {
  if (accurate) sincosf(x, s, c);
  else __sincosf(x, s, c);
}

// --------------------------------------------------------------- Voigt
// Hui, Armstrong & Wray (1978) rational approximation of the complex
// probability function w = P(z)/Q(z), z = a + i v, evaluated by Horner's rule
// in double; H = Re w and F = -Im w / 2 are formed in float with the
// reference's fast division (d_fvoigt, mil_sinrf.cu:172-332).
__device__ __forceinline__ void voigt(double a, float v, float& H, float& F) {
  const double zr = a, zi = (double)v;
  double nr = -0.564189583562615, ni = 0.0;
  const double p[6] = {122.607931777104326, 214.382388694706425, 181.928533092181549,
                       93.155580458138441, 30.180142196210589, 5.912626209773153};
#pragma unroll
  for (int k = 5; k >= 0; --k) {
    const double t = nr * zr - ni * zi - p[k];
    ni = nr * zi + ni * zr;
    nr = t;
  }
  const double q[7] = {122.60793177387535, 352.730625110963558, 457.334478783897737,
                       348.703917719495792, 170.354001821091472, 53.992906912940207,
                       10.479857114260399};
  double dr = 1.0, di = 0.0;
#pragma unroll
  for (int k = 6; k >= 0; --k) {
    const double t = dr * zr - di * zi + q[k];
    di = dr * zi + di * zr;
    dr = t;
  }
  const float den = (float)(dr * dr + di * di);
  const float re = (float)(nr * dr + ni * di);
  const float im = (float)(ni * dr - nr * di);
  H = -__fdividef(re, den);
  F = __fdividef(im, den) * 0.5f;
}

// --------------------------------------------------------------- state
struct Angles {
  float cosi, sinis, sina, cosa, sinda, cosda, sindi, cosdi, cosis_2;
};

// Kernel variants.  V = 0: the reference's 10-term path without
// macroturbulence; V = 1: 10 terms with the macroturbulence convolution
// (a fixed v_mac > 0, or per-pixel start models); V = 2: the 11-term path
// (v_mac and alpha both free: lm_mils_11, milosUtils.cu:713-850) with its
// FP64 solve.  V = 0 solves the 10x10 system for two dampings at once, one
// per half-warp (the second is the damping a rejected trial moves to).
template <int V>
struct Variant {
  static constexpr int NT = (V == 2) ? 11 : 10;         // terms of the normal equations
  static constexpr bool MAC = V != 0;                    // macroturbulence-capable
  static constexpr int ROWS = MAC ? 36 : 32;             // staged rows (+4 for the v_mac RF)
  static constexpr int SOLVES = (V == 0) ? 2 : 1;        // 10x10 systems solved per call
};

// Per-lane results of a synthesis that the response functions reuse:
// absorption / dispersion profiles of the pi, blue and red groups and the
// last component's H, F, v of each group (the reference's profile
// derivatives keep only the last component of a group, me_der.cu:66-74);
// with macroturbulence also the profile before any convolution (the
// reference's spectra_mc, mil_sinrf.cu:425-430).
template <int LPL, int V>
struct Lane {
  float fi[LPL][3], shi[LPL][3];
  float lh[LPL][3], lf[LPL][3], lu[LPL][3];
  float mc[Variant<V>::MAC ? LPL : 1][4];
};

// Rows staged for the PSF: Stokes s x RF slot {eta0, B, vlos, dopp, damping,
// gamma, azimuth, S1} (S0's RF is constant, alpha's is never convolved);
// macroturbulence variants add the v_mac RF of Stokes s at row 32 + s.
constexpr int kRows = 32;
__host__ __device__ constexpr int rf_row(int s, int t) { return s * 8 + (t == 8 ? 7 : t); }
__host__ __device__ constexpr int mac_row(int s) { return kRows + s; }
// A staged row holds samples [0, 32 LPL) (zero past nl); its pitch of
// 32 LPL + 4 floats puts the 8 rows of a tensor-core fragment in distinct
// shared-memory banks.
template <int LPL>
__host__ __device__ constexpr int row_pitch() { return 32 * LPL + 4; }

// Dynamic shared memory of the inversion and synthesis kernels: the block's
// PSF taps (block_taps), then one WarpSmem per warp.
extern __shared__ __align__(16) unsigned char gm_dyn_smem[];

// The PSF taps in double, zero padded, shared by the warps of a block: tap j
// of the nl-tap PSF at index tap_off + j of tap_span doubles.  The padding
// lets every lane read its Toeplitz element of the convolution matrix with one
// load and no bounds test.
template <int LPL>
__host__ __device__ constexpr int tap_span() { return 96 * LPL; }
template <int LPL>
__host__ __device__ constexpr int tap_off() { return 32 * LPL; }
template <int LPL>
__host__ __device__ constexpr size_t tap_bytes() { return sizeof(double) * tap_span<LPL>(); }
__device__ __forceinline__ double* block_taps() { return reinterpret_cast<double*>(gm_dyn_smem); }

// Extra rows of the normal equations' operand: per Stokes the column of
// alpha's slot (asrc - slight) and the residual syn - obs, then a row of ones
// (S0's RF of Stokes I) and a row of zeros, all zero past nl.
constexpr int kXAlpha = 0, kXRes = 4, kXOne = 8, kXZero = 9, kXRows = 10;

// The 11-term solve's FP64 Jacobi matrix (12x12, double-buffered) and its
// accumulated rotations; the elimination uses the first matrix.
template <bool S11>
struct Jacobi11 {
  double A[S11 ? 2 : 1][S11 ? 144 : 1];
  double V[S11 ? 2 : 1][S11 ? 144 : 1];
};

// Warp-private shared memory.
template <int LPL, int V>
struct WarpSmem {
  static constexpr int NR = Variant<V>::ROWS;
  static constexpr bool S11 = V == 2;
  double m[11];          // current (last accepted) model: the reference's initModel
  double t[11];          // trial model, persistent like the reference's `model`
  static constexpr int NS = Variant<V>::SOLVES;
  // Jacobi working matrix per damping, double-buffered, in 2x2 blocks of
  // the upper triangle (solve10's layout: damping h, buffer b at
  // h * kSolveH + b * kSolveB)
  alignas(16) float A[NS == 2 ? 272 : 200];
  float alpha[68];       // undamped normal matrix, packed upper triangle (55 or 66)
  float beta[12];
  float vec[NS][2][12];  // rotated beta per damping, double-buffered; a step lands in vec[d][0]
  float cs[NS][18][5], sn[NS][18][5];
  float ic[NR];          // continuum about which each staged I row is reflected
  double gk[Variant<V>::MAC ? kMaxNl : 1];   // macroturbulence kernel (PSF folded in)
  double gd[Variant<V>::MAC ? kMaxNl : 1];   // its derivative with respect to v_mac
  double dd[12];         // FP64 step of the 11-term solve
  double b11[S11 ? 12 : 1], z11[S11 ? 12 : 1];
  double c11[S11 ? 6 : 1], s11[S11 ? 6 : 1]; // the step's rotations
  // staged rows (PSF, macroturbulence, RFs), sharing their space with the
  // 11-term solve's matrices: a trial solves before its synthesis stages
  // any row, the accept half never solves, and the response functions are
  // consumed by the normal equations before the next solve
  union {
    float rows[NR][row_pitch<LPL>()];
    Jacobi11<S11> j11;
  };
  // the normal equations' operand rows (kX*), right after `rows` with the
  // same pitch: row NR + x of the combined array is xrows[x]
  float xrows[kXRows][row_pitch<LPL>()];
  // offsets of the normal equations' operand rows per Stokes parameter and
  // term (jrow times the pitch; 12 per parameter, the last unused)
  alignas(16) int nero[4][12];
};

template <int LPL>
__host__ __device__ constexpr int warps_per_block() { return LPL == 1 ? 4 : 2; }

// --------------------------------------------------------------- PSF
// Stage one row (LPL samples per lane) in shared memory; I rows are
// reflected about their continuum max(first, last) (direct_convolution_ic,
// convolution.cu:200-241).
template <int LPL, int V>
__device__ __forceinline__ void put_row(WarpSmem<LPL, V>& sm, int r, const float (&x)[LPL], int nl,
                                        int lane, bool reflect) {
  float ic = 0.f;
  if (reflect) {
    const float first = __shfl_sync(kFull, x[0], 0);
    const int kl = (nl - 1) >> 5, ll = (nl - 1) & 31;
    float lastv = x[0];
#pragma unroll
    for (int k = 1; k < LPL; ++k)
      if (k == kl) lastv = x[k];
    const float last = __shfl_sync(kFull, lastv, ll);
    ic = first > last ? first : last;
    if (lane == 0) sm.ic[r] = ic;
  }
#pragma unroll
  for (int k = 0; k < LPL; ++k) {
    const int l = lane + 32 * k;
    sm.rows[r][l] = (l < nl) ? (reflect ? ic - x[k] : x[k]) : 0.f;
  }
}

// Load the block's padded PSF taps (all threads of the block, once).
template <int LPL>
__device__ __forceinline__ void load_taps(const DevCfg& c) {
  double* taps = block_taps();
  for (int i = threadIdx.x; i < tap_span<LPL>(); i += blockDim.x) {
    const int j = i - tap_off<LPL>();
    taps[i] = (c.use_psf && j >= 0 && j < c.nl) ? c.psfd[j] : 0.0;
  }
  __syncthreads();
}

// D += A B on the FP64 tensor cores: an 8x8 tile from an 8x4 by 4x8 product.
// Lane l holds A[l / 4][l % 4], B[l % 4][l / 4] and D[l / 4][2 (l % 4) + i].
__device__ __forceinline__ void dmma_884(double& d0, double& d1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

// In-place same-size correlation of the staged rows in `mask` with the
// nl-tap PSF centred at nl/2, zero padded, in double -- the reference's
// direct_convolution{,_ic} (convolution.cu:153-241), whose taps, padded row
// and sums are double and whose result is rounded to float once.  Rows in
// `reflect` are reflected back about sm.ic in double as there.  The
// correlation is the product out = X T of the staged rows X (8-row tiles) and
// the Toeplitz matrix T[n][m] = h[n - m + nl/2] (zero outside the taps, which
// is the zero padding), on the FP64 tensor cores; only the order of the double
// additions differs from the reference.  A tile holding a row outside `mask`
// computes it but stores only the rows in `mask`.  The caller syncs the warp
// after staging.
template <int LPL, int V>
__device__ __forceinline__ void psf_rows(WarpSmem<LPL, V>& sm, const DevCfg& c, uint32_t mask,
                                         uint32_t reflect, int lane) {
  constexpr int S = 32 * LPL;                 // samples per row: the K and N extents
  const int nl = c.nl, half = nl >> 1;
  const int gr = lane >> 2, gc = lane & 3;   // fragment row group, column group
  // this lane's B element of step (k0, n0): T[k0 + gc][n0 + gr]
  const double* tb = block_taps() + tap_off<LPL>() + half + gc - gr;
  while (mask) {
    const int mt = (__ffs(mask) - 1) >> 3;    // 8-row tile of the next staged row
    const uint32_t tile = (mask >> (8 * mt)) & 0xffu;
    mask &= ~(0xffu << (8 * mt));
    const int r = 8 * mt + gr;
    const float* arow = sm.rows[r];
    const bool mine = (tile >> gr) & 1u;
    const bool refl = (reflect >> r) & 1u;
    const double ic = refl ? (double)sm.ic[r] : 0.0;
    float res[LPL][4][2];
#pragma unroll
    for (int p = 0; p < LPL; ++p) {           // output columns in passes of 32
      double acc[4][2];
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q][0] = acc[q][1] = 0.0;
#pragma unroll 2
      for (int k0 = 0; k0 < S; k0 += 4) {
        const double a = (double)arow[k0 + gc];
#pragma unroll
        for (int q = 0; q < 4; ++q) dmma_884(acc[q][0], acc[q][1], a, tb[k0 - 8 * (4 * p + q)]);
      }
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int i = 0; i < 2; ++i) res[p][q][i] = (float)(refl ? ic - acc[q][i] : acc[q][i]);
    }
    __syncwarp();
    if (mine) {
#pragma unroll
      for (int p = 0; p < LPL; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
          for (int i = 0; i < 2; ++i) {
            const int m = 32 * p + 8 * q + 2 * gc + i;
            sm.rows[r][m] = (m < nl) ? res[p][q][i] : 0.f;
          }
    }
  }
  __syncwarp();
}

// --------------------------------------------------------------- macroturbulence
// The macroturbulence kernel: a Gaussian in wavelength of width
// lambda0 * v_mac / c sampled on the grid about sample nl/2 and normalised to
// unit sum (fgauss, fgauss.cu:16-63), in sm.gk; with `deriv` also its
// derivative with respect to v_mac, g / v_mac * (x^2 - 1) (me_der.cu:122-129),
// in sm.gd.  With a PSF both are then correlated with it in double, zero
// padded about nl/2 (direct_convolution_double, convolution.cu:120-151;
// mil_sinrf.cu:105-107, me_der.cu:131-136).  lamp: the pixel's own
// wavelengths, or null for the configured grid.
template <int LPL, int V>
__device__ __forceinline__ void mac_kernels(const DevCfg& c, WarpSmem<LPL, V>& sm, double mac,
                                            int lane, bool deriv, const double* lamp) {
  const int nl = c.nl, half = nl >> 1;
  const double ild = (c.lambda0 * mac) / kVlight;
  const double lc = lamp ? lamp[half] : c.lam[half];
  double g[LPL], x2[LPL], part = 0.0;
#pragma unroll
  for (int k = 0; k < LPL; ++k) {
    const int l = lane + 32 * k;
    g[k] = 0.0;
    x2[k] = 0.0;
    if (l < nl) {
      const double x = ((lamp ? lamp[l] : c.lam[l]) - lc) / ild;
      const double term = (x * x) / 2;
      g[k] = term < 1e30 ? exp(-term) : 0.0;
      x2[k] = x * x;
      part += g[k];
    }
  }
  const double sum = warp_sum_d(part);
#pragma unroll
  for (int k = 0; k < LPL; ++k) {
    const int l = lane + 32 * k;
    if (l < nl) {
      const double gn = g[k] / sum;
      sm.gk[l] = gn;
      if (deriv) sm.gd[l] = gn / mac * (x2[k] - 1.0);
    }
  }
  __syncwarp();
  if (!c.use_psf) return;
  double og[LPL], od[LPL];
#pragma unroll
  for (int k = 0; k < LPL; ++k) {
    const int l = lane + 32 * k;
    double a = 0.0, b = 0.0;
    if (l < nl) {
      for (int j = 0; j < nl; ++j) {
        const int idx = l + j - half;
        if (idx < 0 || idx >= nl) continue;
        a += c.psfd[j] * sm.gk[idx];
        if (deriv) b += c.psfd[j] * sm.gd[idx];
      }
    }
    og[k] = a;
    od[k] = b;
  }
  __syncwarp();
#pragma unroll
  for (int k = 0; k < LPL; ++k) {
    const int l = lane + 32 * k;
    if (l < nl) {
      sm.gk[l] = og[k];
      if (deriv) sm.gd[l] = od[k];
    }
  }
  __syncwarp();
}

// In-place circular convolution of the staged rows in `mask` with the nl-tap
// kernel h, accumulated in double with kernel sample j at lag j, the result
// rotated so that sample nl/2 is the zero lag (convCircular,
// convolution.cu:251-279): output m takes the circular sum at index
// (m + nl/2) mod nl.  The caller syncs the warp after staging.
template <int LPL, int V>
__device__ __forceinline__ void circ_rows(WarpSmem<LPL, V>& sm, const DevCfg& c, uint64_t mask,
                                          const double* h, int lane) {
  const int nl = c.nl, half = nl >> 1;
  while (mask) {
    const int r = __ffsll((long long)mask) - 1;
    mask &= mask - 1;
    const float* x = sm.rows[r];
    float out[LPL];
#pragma unroll
    for (int k = 0; k < LPL; ++k) {
      const int mo = lane + 32 * k;
      double a = 0.0;
      if (mo < nl) {
        int idx = mo + half;
        if (idx >= nl) idx -= nl;
        for (int j = 0; j < nl; ++j) {
          a += h[j] * (double)x[idx];
          idx = (idx == 0) ? nl - 1 : idx - 1;
        }
      }
      out[k] = (float)a;
    }
    __syncwarp();
#pragma unroll
    for (int k = 0; k < LPL; ++k) {
      const int mo = lane + 32 * k;
      if (mo < nl) sm.rows[r][mo] = out[k];
    }
  }
  __syncwarp();
}

// --------------------------------------------------------------- synthesis
// ME synthesis of this lane's samples (mil_sinrf.cu:27-142 with
// mil_sinrf_kernel :334-433): Zeeman components through the Voigt
// profiles, Unno-Rachkovsky solution, PSF, stray-light mix.
template <int LPL, int V>
__device__ __forceinline__ void synth_lane(const DevCfg& c, const double* m, const float (&dlv)[LPL],
                                           int lane, Lane<LPL, V>& st, Angles& an,
                                           float (&spec)[LPL][4], float (&pure)[LPL][4],
                                           const float (&sl)[LPL][4], WarpSmem<LPL, V>& sm,
                                           const double* lamp = nullptr) {
  const float CC = (float)(kPi / 180.0), CC2 = (float)((kPi / 180.0) * 2);
  const double azi = m[AZ] * (double)CC, gmr = m[GM] * (double)CC;
  float sgm, cgm;
  const bool acc = c.numerics != 0;
  sincos_mode((float)gmr, &sgm, &cgm, acc);
  an.cosi = cgm;
  an.sinis = sgm * sgm;
  const float cosis = cgm * cgm;
  an.cosis_2 = __fdividef(1.f + cosis, 2.f);
  sincos_mode((float)(2 * azi), &an.sina, &an.cosa, acc);
  an.sinda = an.cosa * CC2;
  an.cosda = -an.sina * CC2;
  an.sindi = cgm * sgm * CC2;
  an.cosdi = -sgm * CC;
  const float sinis_cosa = an.sinis * an.cosa, sinis_sina = an.sinis * an.sina;
  const double E0 = m[ETA0] * (double)c.fo;
  const float ulos = __fdividef((float)(m[VLOS] * c.lambda0), (float)(kVlight * m[DOPP]));
  const float parcial = (float)((c.lambda0 * c.lambda0 / m[DOPP]) * kLarmor);
  const float doppf = (float)m[DOPP];
  const double aa = m[AA];

  // every Zeeman component in one rolled loop (one copy of the Voigt code):
  // group g of component ci, its index kk within the group
  const int ncomp = c.n_pi + 2 * c.n_sig;
#pragma unroll 1
  for (int ci = 0; ci < ncomp; ++ci) {
    const int g = ci < c.n_pi ? 0 : (ci < c.n_pi + c.n_sig ? 1 : 2);
    const int kk = g == 0 ? ci : (g == 1 ? ci - c.n_pi : ci - c.n_pi - c.n_sig);
    float nu, wex;
    if (g == 0) { nu = parcial * c.nup[kk]; wex = c.wep[kk]; }
    else if (g == 1) { nu = parcial * c.nub[kk]; wex = c.web[kk]; }
    else { nu = -(parcial * c.nub[c.n_sig - 1 - kk]); wex = c.wer[kk]; }
    const float rnu = (float)((double)nu * m[BFLD]);
#pragma unroll
    for (int k = 0; k < LPL; ++k) {
      float v = __fdividef(dlv[k], doppf);
      v = v - ulos;
      v = v - rnu;
      float h, f;
      voigt(aa, v, h, f);
      const float fh = wex * h, fs = wex * f * 2.f;
#pragma unroll
      for (int gg = 0; gg < 3; ++gg) {
        if (gg != g) continue;
        st.fi[k][gg] = kk == 0 ? fh : st.fi[k][gg] + fh;
        st.shi[k][gg] = kk == 0 ? fs : st.shi[k][gg] + fs;
        st.lh[k][gg] = h;
        st.lf[k][gg] = f;
        st.lu[k][gg] = v;
      }
    }
  }

  const float E0_2 = __fdividef((float)E0, 2.f);
  const double s1mu = -(m[S1] * (double)c.mu);
#pragma unroll
  for (int k = 0; k < LPL; ++k) {
    const float fp = st.fi[k][0], fb = st.fi[k][1], fr = st.fi[k][2];
    const float sp = st.shi[k][0], sb = st.shi[k][1], sr = st.shi[k][2];
    const float p1 = fb + fr;
    const float p2 = E0_2 * (fp - __fdividef(p1, 2.f));
    const float p3 = E0_2 * (sp - __fdividef(sb + sr, 2.f));
    const float ein = E0_2 * (fp * an.sinis + p1 * an.cosis_2);
    const float eq = p2 * sinis_cosa, eu = p2 * sinis_sina, ev = (fr - fb) * (E0_2 * an.cosi);
    const float rq = p3 * sinis_cosa, ru = p3 * sinis_sina, rv = (sr - sb) * (E0_2 * an.cosi);
    const float ei = 1.f + ein;
    const float ei2 = ei * ei;
    const float q2 = rq * rq, u2 = ru * ru, v2 = rv * rv;
    const float gp1 = ei2 - eq * eq - eu * eu - ev * ev + q2 + u2 + v2;
    const float gp3 = ei2 + q2 + u2 + v2;
    const float gp2 = eq * rq + eu * ru + ev * rv;
    const float dt = ei2 * gp1 - gp2 * gp2;
    const float dti = __fdividef(1.f, dt);
    const float gp4 = ei2 * eq + ei * (ev * ru - eu * rv);
    const float gp5 = ei2 * eu + ei * (eq * rv - ev * rq);
    const float gp6 = ei2 * ev + ei * (eu * rq - eq * ru);
    const float dtiaux = (float)((double)dti * s1mu);
    spec[k][0] = (float)(m[S0] - (double)(dtiaux * ei * gp3));
    spec[k][1] = dtiaux * (gp4 + rq * gp2);
    spec[k][2] = dtiaux * (gp5 + ru * gp2);
    spec[k][3] = dtiaux * (gp6 + rv * gp2);
  }

  bool mac_on = false;
  if constexpr (Variant<V>::MAC) {
#pragma unroll
    for (int k = 0; k < LPL; ++k)
#pragma unroll
      for (int s = 0; s < 4; ++s) st.mc[k][s] = spec[k][s];
    mac_on = m[MAC] > 0.0001;
  }
  if (mac_on) {
    // macroturbulence with the PSF folded into its kernel; the PSF is not
    // applied again (mil_sinrf.cu:101-130)
    mac_kernels<LPL, V>(c, sm, m[MAC], lane, false, lamp);
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      float row[LPL];
#pragma unroll
      for (int k = 0; k < LPL; ++k) row[k] = spec[k][s];
      put_row<LPL, V>(sm, s, row, c.nl, lane, false);
    }
    __syncwarp();
    circ_rows<LPL, V>(sm, c, 0xfull, sm.gk, lane);
#pragma unroll
    for (int k = 0; k < LPL; ++k)
#pragma unroll
      for (int s = 0; s < 4; ++s) spec[k][s] = sm.rows[s][lane + 32 * k];
    __syncwarp();
  } else if (c.use_psf) {
    __syncwarp();
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      float row[LPL];
#pragma unroll
      for (int k = 0; k < LPL; ++k) row[k] = spec[k][s];
      put_row<LPL, V>(sm, s, row, c.nl, lane, s == 0);
    }
    __syncwarp();
    psf_rows<LPL, V>(sm, c, 0xfu, 0x1u, lane);
#pragma unroll
    for (int k = 0; k < LPL; ++k)
#pragma unroll
      for (int s = 0; s < 4; ++s) spec[k][s] = sm.rows[s][lane + 32 * k];
    __syncwarp();
  }
#pragma unroll
  for (int k = 0; k < LPL; ++k)
#pragma unroll
    for (int s = 0; s < 4; ++s) pure[k][s] = spec[k][s];
  if (c.use_slight) {
    const double a = m[ALFA];
#pragma unroll
    for (int k = 0; k < LPL; ++k)
#pragma unroll
      for (int s = 0; s < 4; ++s)
        spec[k][s] = (float)((double)spec[k][s] * a + (double)sl[k][s] * (1.0 - a));
  }
}

// --------------------------------------------------------------- response functions
// Staged rows of the free response functions that go through the PSF: every
// free parameter but S0 (the azimuth RF of I and V is identically zero).
__device__ __forceinline__ uint32_t rf_row_mask(const DevCfg& c) {
  uint32_t mk = 0;
#pragma unroll
  for (int t = 0; t < 9; ++t) {
    if (t == 7 || !c.fix[t]) continue;
#pragma unroll
    for (int s = 0; s < 4; ++s)
      if (!(t == 6 && (s == 0 || s == 3))) mk |= 1u << rf_row(s, t);
  }
  return mk;
}

// Analytic derivatives of the last synthesis (me_der.cu:81-376): profile
// derivatives of each group's last component (d_funcionComponentFor
// :53-77), their Zeeman combination and the RTE derivative (me_der_kernel
// :218-376), then the PSF of every free RF except S0's (:162-189), I rows
// reflected about max(first, last).  The results stay in the staged rows
// of sm (rf_row); gather_rf adds S0, alpha, the stray-light scaling
// (:191-211) and the zeros of fixed parameters
// (FijaACeroDerivadasNoNecesarias, milosUtils.cu:243-271).
template <int LPL, int V>
__device__ __forceinline__ void rf_rows(const DevCfg& c, const double* m, const Lane<LPL, V>& st,
                                        const Angles& an, int lane, WarpSmem<LPL, V>& sm,
                                        const double* lamp = nullptr) {
  const float auxCte = __fdividef((float)(-c.lambda0), (float)(kVlight * m[DOPP]));
  const double aa = m[AA], dopp = m[DOPP];
  // last component of each group: its scaled splitting and strength
  const float parcial = (float)((c.lambda0 * c.lambda0 / m[DOPP]) * kLarmor);
  float nul[3], wel[3];
  nul[0] = parcial * c.nup[c.n_pi - 1];
  wel[0] = c.wep[c.n_pi - 1];
  nul[1] = parcial * c.nub[c.n_sig - 1];
  wel[1] = c.web[c.n_sig - 1];
  nul[2] = -(parcial * c.nub[0]);
  wel[2] = c.wer[c.n_sig - 1];

  const float E0f = (float)(m[ETA0] * (double)c.fo);
  const double E0dd = m[ETA0] * (double)c.fo;
  const float sc = __fdividef(E0f * (an.sinis * an.cosa), 2.f);
  const float ss = __fdividef(E0f * (an.sinis * an.sina), 2.f);
  const float E0_2 = __fdividef(E0f, 2.f);
  const float sindi_cosa = an.sindi * an.cosa, sindi_sina = an.sindi * an.sina;
  const float cosdi_E0_2 = E0_2 * an.cosdi;
  const float cosi_2_E0 = __fdividef(E0f * an.cosi, 2.f);
  const float cosis_2_E0_2 = an.cosis_2 * E0_2;
  const float sinis_E0_2 = an.sinis * E0_2;
  const float cosi_cosdi = an.cosi * an.cosdi * E0_2, sindi_E0_2 = an.sindi * E0_2;
  const float sinis_cosda = an.sinis * an.cosda, sinis_sinda = an.sinis * an.sinda;
  const float sinis_cosa = an.sinis * an.cosa, sinis_sina = an.sinis * an.sina;
  const float s1mu_f = (float)(-(m[S1] * (double)c.mu));
  const float muf = c.mu;
  const uint32_t mask = rf_row_mask(c);
  const int nl = c.nl;

#pragma unroll
  for (int k = 0; k < LPL; ++k) {
    const int l = lane + 32 * k;
    float dfi[3][4], dshi[3][4];
#pragma unroll
    for (int g = 0; g < 3; ++g) {
      const float u = st.lu[k][g], h = st.lh[k][g], f = st.lf[k][g];
      const float dH = (float)((4 * aa * (double)f - (double)(2.f * u * h)) * (double)wel[g]);
      const float dF = (float)((kRR - aa * (double)h - (double)(2.f * u * f)) * (double)wel[g]);
      const float su = (float)(-(double)u / dopp);
      dfi[g][0] = dH * (-nul[g]);
      dfi[g][1] = dH * auxCte;
      dfi[g][2] = dH * su;
      dfi[g][3] = -2.f * dF;
      dshi[g][0] = dF * (-nul[g]);
      dshi[g][1] = dF * auxCte;
      dshi[g][2] = dF * su;
      dshi[g][3] = dH * 0.5f;
    }
    // RTE quantities of this sample (recomputed from the stored profiles;
    // identical to the synthesis' values)
    const float fp = st.fi[k][0], fb = st.fi[k][1], fr = st.fi[k][2];
    const float sp = st.shi[k][0], sb = st.shi[k][1], sr = st.shi[k][2];
    const float p1 = fb + fr;
    const float p2 = E0_2 * (fp - __fdividef(p1, 2.f));
    const float p3 = E0_2 * (sp - __fdividef(sb + sr, 2.f));
    const float ein = E0_2 * (fp * an.sinis + p1 * an.cosis_2);
    const float eq = p2 * sinis_cosa, eu = p2 * sinis_sina, ev = (fr - fb) * (E0_2 * an.cosi);
    const float rq = p3 * sinis_cosa, ru = p3 * sinis_sina, rv = (sr - sb) * (E0_2 * an.cosi);
    const float ei = 1.f + ein;
    const float ei2 = ei * ei;
    const float gp1 = ei2 - eq * eq - eu * eu - ev * ev + rq * rq + ru * ru + rv * rv;
    const float gp3 = ei2 + rq * rq + ru * ru + rv * rv;
    const float gp2 = eq * rq + eu * ru + ev * rv;
    const float dt = ei2 * gp1 - gp2 * gp2;
    const float g4 = (ei2 * eq + ei * (ev * ru - eu * rv)) + rq * gp2;
    const float g5 = (ei2 * eu + ei * (eq * rv - ev * rq)) + ru * gp2;
    const float g6 = (ei2 * ev + ei * (eu * rq - eq * ru)) + rv * gp2;
    const float dtaux = __fdividef(s1mu_f, dt * dt);
    const float eigp3 = ei * gp3;
    const float a2 = 2.f * ei;
    const float ext1 = a2 * eq + ev * ru - eu * rv;
    const float ext2 = a2 * eu + eq * rv - ev * rq;
    const float ext3 = a2 * ev + eu * rq - eq * ru;
    const float ext4 = a2 * gp1;

#pragma unroll
    for (int il = 0; il < 9; ++il) {
      if (il == 7) continue;
      float de = 0.f, dq = 0.f, du = 0.f, dv = 0.f, drq = 0.f, dru = 0.f, drv = 0.f;
      if (il == 0) {
        de = (float)((double)ein / E0dd);
        dq = __fdividef(eq, (float)E0dd);
        du = __fdividef(eu, (float)E0dd);
        dv = __fdividef(ev, (float)E0dd);
        drq = __fdividef(rq, (float)E0dd);
        dru = __fdividef(ru, (float)E0dd);
        drv = __fdividef(rv, (float)E0dd);
      } else if (il < 5) {
        const int j = il - 1;
        const float dsum = dfi[1][j] + dfi[2][j];
        de = dfi[0][j] * sinis_E0_2 + dsum * cosis_2_E0_2;
        const float aux = dfi[0][j] - __fdividef(dsum, 2.f);
        dq = aux * sc;
        du = aux * ss;
        dv = (dfi[2][j] - dfi[1][j]) * cosi_2_E0;
        const float s1 = dshi[1][j], s2 = dshi[2][j];
        const float aux2 = dshi[0][j] - __fdividef(s1 + s2, 2.f);
        drq = aux2 * sc;
        dru = aux2 * ss;
        drv = (s2 - s1) * cosi_2_E0;
      } else if (il == 5) {
        de = fp * sindi_E0_2 + p1 * cosi_cosdi;
        dq = p2 * sindi_cosa;
        du = p2 * sindi_sina;
        dv = (fr - fb) * cosdi_E0_2;
        drq = p3 * sindi_cosa;
        dru = p3 * sindi_sina;
        drv = (sr - sb) * cosdi_E0_2;
      } else if (il == 6) {
        dq = p2 * sinis_cosda;
        du = p2 * sinis_sinda;
        drq = p3 * sinis_cosda;
        dru = p3 * sinis_sinda;
      }
      float o[4];
      if (il == 8) {   // source-function gradient
        const float dti = -(__fdividef(1.f, dt) * muf);
        o[0] = -dti * eigp3;
        o[1] = dti * g4;
        o[2] = dti * g5;
        o[3] = dti * g6;
      } else {
        const float dgp1 = 2.f * (ei * de - eq * dq - eu * du - ev * dv + rq * drq + ru * dru + rv * drv);
        const float dgp2 = rq * dq + eq * drq + ru * du + eu * dru + rv * dv + ev * drv;
        const float ddt = ext4 * de + ei2 * dgp1 - 2.f * gp2 * dgp2;
        const float dgp3 = 2.f * (ei * de + rq * drq + ru * dru + rv * drv);
        const float dgp4 = de * ext1 + ei2 * dq + ei * (ru * dv + ev * dru - rv * du - eu * drv);
        const float dgp5 = de * ext2 + ei2 * du + ei * (rv * dq + eq * drv - rq * dv - ev * drq);
        const float dgp6 = de * ext3 + ei2 * dv + ei * (rq * du + eu * drq - ru * dq - eq * dru);
        o[0] = -(((de * gp3 + ei * dgp3) * dt - ddt * eigp3) * dtaux);
        o[1] = ((dgp4 + drq * gp2 + rq * dgp2) * dt - ddt * g4) * dtaux;
        o[2] = ((dgp5 + dru * gp2 + ru * dgp2) * dt - ddt * g5) * dtaux;
        o[3] = ((dgp6 + drv * gp2 + rv * dgp2) * dt - ddt * g6) * dtaux;
      }
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const int r = rf_row(s, il);
        if ((mask >> r) & 1u) sm.rows[r][l] = (l < nl) ? o[s] : 0.f;
      }
    }
  }
  __syncwarp();

  bool mac_on = false;
  if constexpr (Variant<V>::MAC) mac_on = m[MAC] > 0.0001;
  if (mac_on) {
    if constexpr (Variant<V>::MAC) {
      // macroturbulence (me_der.cu:117-156): the v_mac RF is the profile
      // before convolution through the kernel's derivative; every other
      // staged RF goes through the kernel (PSF folded into both)
      mac_kernels<LPL, V>(c, sm, m[MAC], lane, true, lamp);
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        float row[LPL];
#pragma unroll
        for (int k = 0; k < LPL; ++k) row[k] = st.mc[k][s];
        put_row<LPL, V>(sm, mac_row(s), row, nl, lane, false);
      }
      __syncwarp();
      circ_rows<LPL, V>(sm, c, 0xfull << kRows, sm.gd, lane);
      circ_rows<LPL, V>(sm, c, (uint64_t)mask, sm.gk, lane);
    }
  } else if (c.use_psf) {
    // reflect the I rows about max(first, last) (me_der.cu:167-176)
    uint32_t refl = 0;
    float icv[8];
#pragma unroll
    for (int tt = 0; tt < 8; ++tt) {
      const int r = rf_row(0, tt == 7 ? 8 : tt);
      icv[tt] = 0.f;
      if (!((mask >> r) & 1u)) continue;
      refl |= 1u << r;
      const float f0 = sm.rows[r][0];
      const float f1 = sm.rows[r][nl - 1];
      icv[tt] = f0 > f1 ? f0 : f1;
      if (lane == 0) sm.ic[r] = icv[tt];
    }
    __syncwarp();   // every lane has read the end samples before any is overwritten
#pragma unroll
    for (int tt = 0; tt < 8; ++tt) {
      const int r = rf_row(0, tt == 7 ? 8 : tt);
      if (!((refl >> r) & 1u)) continue;
#pragma unroll
      for (int k = 0; k < LPL; ++k) {
        const int l = lane + 32 * k;
        if (l < nl) sm.rows[r][l] = icv[tt] - sm.rows[r][l];
      }
    }
    __syncwarp();
    psf_rows<LPL, V>(sm, c, mask, refl, lane);
  }
}

// Response function of sample l, Stokes s, slot t in the reference's layout
// after the PSF: 10 terms (slot 7 = S0, slot 9 = alpha) or 11 terms (slot 9
// = v_mac, slot 10 = alpha).  Stray-light scaling, alpha's RF from the
// unscaled profile (me_der.cu:191-211), zero for fixed parameters
// (FijaACeroDerivadasNoNecesarias, milosUtils.cu:243-271; in the 10-term
// layout slot 9 follows alpha's flag).  mac_on: the v_mac RF rows hold the
// derivative of the macroturbulence convolution.
template <int LPL, int V>
__device__ __forceinline__ float gather_rf(const DevCfg& c, const WarpSmem<LPL, V>& sm, double alfa,
                                           float asrc, float sl, int l, int s, int t, bool mac_on) {
  constexpr int NT = Variant<V>::NT;
  const int key = (NT == 10 && t == 9) ? 10 : t;
  if (!c.fix[key]) return 0.f;
  float v = 0.f;
  if (t == NT - 1) {
    // alpha's slot; without stray light the 10-term slot keeps the v_mac RF
    // me_der wrote there (me_der.cu:140-143)
    if (c.use_slight) return asrc - sl;
    if constexpr (Variant<V>::MAC && NT == 10) {
      if (mac_on) return sm.rows[mac_row(s)][l];
    }
    return 0.f;
  }
  if (t == 9) {
    if constexpr (Variant<V>::MAC) {
      if (mac_on) v = sm.rows[mac_row(s)][l];
    }
  } else if (t == 7) {
    v = (s == 0) ? 1.f : 0.f;
  } else if (t == 6 && (s == 0 || s == 3)) {
    v = 0.f;
  } else {
    v = sm.rows[rf_row(s, t)][l];
  }
  if (c.use_slight) v = (float)((double)v * alfa);
  return v;
}

// packed index of (i <= h) in the upper triangle of an n x n matrix
template <int NT>
__host__ __device__ constexpr int upk(int i, int h) { return i * NT - (i * (i - 1)) / 2 + (h - i); }

// Row of the operand J' of the normal equations for term t and Stokes s,
// as an index into the staged rows followed by the operand rows (NR + kX*):
// the response function of parameter t < NT as gather_rf defines it (a
// staged RF row, alpha's column, S0's constant RF, or zeros for fixed
// parameters, FijaACeroDerivadasNoNecesarias, milosUtils.cu:243-271), the
// residual syn - obs for t = NT, zeros beyond; `scaled` tells whether the
// stray-light factor alpha applies (me_der.cu:191-211).  t differs between
// the lanes of a warp, so this is written with selects and the free-
// parameter bitmask `fixmask` rather than branches and indexed constants.
template <int LPL, int V>
__device__ __forceinline__ int jrow(const DevCfg& c, uint32_t fixmask, int t, int s, bool mac_on,
                                   bool& scaled) {
  constexpr int NT = Variant<V>::NT, NR = WarpSmem<LPL, V>::NR;
  const int zero = NR + kXZero;
  const int key = (NT == 10 && t == 9) ? 10 : t;
  const bool free_t = t < NT && ((fixmask >> key) & 1u);
  int mac_r = zero;
  if constexpr (Variant<V>::MAC) mac_r = mac_on ? mac_row(s) : zero;
  const int alpha_r = c.use_slight ? NR + kXAlpha + s : ((Variant<V>::MAC && NT == 10) ? mac_r : zero);
  const int tt = t < 8 ? t : 7;   // rf_row's slot of a staged parameter (t = 8 is S1's)
  int r = (t == 6 && (s == 0 || s == 3)) ? zero : rf_row(s, t == 8 ? 8 : tt);
  if (t == 7) r = s == 0 ? NR + kXOne : zero;
  if (NT == 11 && t == 9) r = mac_r;
  if (t == NT - 1) r = alpha_r;
  if (!free_t) r = zero;
  if (t == NT) r = NR + kXRes + s;
  scaled = c.use_slight && t < NT - 1;
  return r;
}

// Entry e of the normal equations in the order they are summed and stored:
// alpha's packed upper triangle (e < NT (NT + 1) / 2, row-major, as upk),
// then beta (column NT of J' W J'^T).  Returns a * 16 + b for operand rows
// a <= b (b = NT: the residual).
template <int NT>
__host__ __device__ constexpr int ne_entry(int e) {
  int a = 0, len = NT;
  while (a < NT && e >= len) {
    e -= len;
    ++a;
    len = NT - a;
  }
  return a < NT ? a * 16 + a + e : e * 16 + NT;
}
template <int NT>
__host__ __device__ constexpr int ne_entries() { return NT * (NT + 1) / 2 + NT; }

// Factors of the stray-light fraction alpha in entry e (0, 1 or 2: one per
// operand row that me_der.cu:191-211 scales, every RF but alpha's own), two
// bits per entry, 32 entries per word.
template <int NT>
__host__ __device__ constexpr uint64_t ne_alfa_bits(int word) {
  uint64_t w = 0;
  for (int i = 0; i < 32; ++i) {
    const int e = 32 * word + i;
    if (e >= ne_entries<NT>()) break;
    const int ab = ne_entry<NT>(e), a = ab >> 4, b = ab & 15;
    w |= (uint64_t)((a < NT - 1 ? 1 : 0) + (b < NT - 1 ? 1 : 0)) << (2 * i);
  }
  return w;
}

// Reduce-scatter of N per-lane partial sums (N a power of two, <= 32) over
// the warp by a shuffle butterfly: at each of the five steps a lane keeps
// half of its values and adds its partner's copy of them, so every step
// halves the values a lane holds; once a lane holds one value the rest of
// the steps are plain butterfly sums.  Returns, in every lane, the warp sum
// of entry lane >> (5 - log2 N).
template <int N>
__device__ __forceinline__ float warp_reduce_scatter(float (&v)[N], int lane) {
  static_assert(N >= 1 && N <= 32 && (N & (N - 1)) == 0, "N must be a power of two <= 32");
#pragma unroll
  for (int st = 0; st < 5; ++st) {
    const int m = 16 >> st, h = (N >> st) / 2;
    if (h >= 1) {
      const bool up = (lane & m) != 0;
#pragma unroll
      for (int j = 0; j < h; ++j) {
        const float send = up ? v[j] : v[j + h];
        const float keep = up ? v[j + h] : v[j];
        v[j] = keep + __shfl_xor_sync(kFull, send, m);
      }
    } else {
      v[0] += __shfl_xor_sync(kFull, v[0], m);
    }
  }
  return v[0];
}

// acc[i] += w x_a x_b for entry P0 + i = (a, b) of every i in I..., the
// operand rows of each entry fixed at compile time.
template <int NT, int E>
__device__ __forceinline__ void ne_product(float& acc, const float (&x)[NT + 1], float w) {
  if constexpr (E < ne_entries<NT>()) {
    constexpr int ab = ne_entry<NT>(E), a = ab >> 4, b = ab & 15;
    acc = fmaf(w * x[a], x[b], acc);
  }
}
template <int NT, int P0, int N, int... I>
__device__ __forceinline__ void ne_products(float (&acc)[N], const float (&x)[NT + 1], float w,
                                            std::integer_sequence<int, I...>) {
  (ne_product<NT, P0 + I>(acc[I], x, w), ...);
}

// This lane's samples l of the operand rows of term t = 0 .. NT (NT: the
// residual) for one Stokes parameter, whose row offsets are ro[0 .. 11].
template <int LPL, int V>
__device__ __forceinline__ void ne_operands(const int* ro, const float* rows0, int l,
                                            float (&x)[Variant<V>::NT + 1]) {
  constexpr int NT = Variant<V>::NT;
  int o[12];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const int4 v = reinterpret_cast<const int4*>(ro)[q];
    o[4 * q] = v.x;
    o[4 * q + 1] = v.y;
    o[4 * q + 2] = v.z;
    o[4 * q + 3] = v.w;
  }
#pragma unroll
  for (int t = 0; t <= NT; ++t) x[t] = rows0[o[t] + l];
}

// Entries [P0, P0 + N) of the normal equations (ne_entry order; entries past
// the last are zero): each lane sums w_s x_a x_b over its own samples and
// the four Stokes parameters in FP32, then warp_reduce_scatter adds the
// lanes' sums.  The operand rows are read unscaled by alpha.
template <int LPL, int V, int P0, int N>
__device__ __forceinline__ float ne_pass(const DevCfg& c, const WarpSmem<LPL, V>& sm, int lane) {
  constexpr int NT = Variant<V>::NT;
  float acc[N];
#pragma unroll
  for (int i = 0; i < N; ++i) acc[i] = 0.f;
#pragma unroll 1
  for (int s = 0; s < 4; ++s) {
    const float w = c.wsig[s];
#pragma unroll
    for (int k = 0; k < LPL; ++k) {
      float x[NT + 1];
      ne_operands<LPL, V>(sm.nero[s], &sm.rows[0][0], lane + 32 * k, x);
      ne_products<NT, P0>(acc, x, w, std::make_integer_sequence<int, N>{});
    }
  }
  return warp_reduce_scatter<N>(acc, lane);
}

// Entries [0, 64) in one pass (the operand rows are read once): the
// butterfly's first step leaves 32 values per lane, the remaining four
// halve them as in warp_reduce_scatter, and lane L ends with entries 2L and
// 2L + 1.
template <int LPL, int V>
__device__ __forceinline__ float2 ne_pass64(const DevCfg& c, const WarpSmem<LPL, V>& sm, int lane) {
  constexpr int NT = Variant<V>::NT;
  float acc[64];
#pragma unroll
  for (int i = 0; i < 64; ++i) acc[i] = 0.f;
#pragma unroll 1
  for (int s = 0; s < 4; ++s) {
    const float w = c.wsig[s];
#pragma unroll
    for (int k = 0; k < LPL; ++k) {
      float x[NT + 1];
      ne_operands<LPL, V>(sm.nero[s], &sm.rows[0][0], lane + 32 * k, x);
      ne_products<NT, 0>(acc, x, w, std::make_integer_sequence<int, 64>{});
    }
  }
  // a lane keeps entries [0, 32) (lane bit 4 clear) or [32, 64) and adds
  // its partner's sums of them
  float v[32];
  const bool up = (lane & 16) != 0;
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    const float send = up ? acc[j] : acc[32 + j];
    v[j] = (up ? acc[32 + j] : acc[j]) + __shfl_xor_sync(kFull, send, 16);
  }
#pragma unroll
  for (int st = 1; st < 5; ++st) {
    const int m = 16 >> st, h = 32 >> st;
    const bool u = (lane & m) != 0;
#pragma unroll
    for (int j = 0; j < h; ++j) {
      const float send = u ? v[j] : v[j + h];
      const float keep = u ? v[j + h] : v[j];
      v[j] = keep + __shfl_xor_sync(kFull, send, m);
    }
  }
  return make_float2(v[0], v[1]);
}

// Store entry e of the normal equations: times alpha once per scaled operand
// row (me_der.cu:191-211; in FP64, then rounded to float), into sm.alpha
// (packed) or sm.beta.
template <int LPL, int V>
__device__ __forceinline__ void ne_store(const DevCfg& c, double alfa, int e, float v, WarpSmem<LPL, V>& sm) {
  constexpr int NT = Variant<V>::NT, NA = NT * (NT + 1) / 2;
  constexpr uint64_t w0 = ne_alfa_bits<NT>(0), w1 = ne_alfa_bits<NT>(1), w2 = ne_alfa_bits<NT>(2);
  if (c.use_slight) {
    const uint64_t w = e < 32 ? w0 : e < 64 ? w1 : w2;
    const int f = (int)((w >> (2 * (e & 31))) & 3u);
    if (f) v = (float)((double)v * (f == 2 ? alfa * alfa : alfa));
  }
  if (e < NA) sm.alpha[e] = v;
  else sm.beta[e - NA] = v;
}

// Normal equations alpha = sum_s w_s/sigma^2 J^T J and beta = sum_s w_s J^T
// (syn - obs) / sigma^2 (covarmf, lib.cu:65-118; covarm, lib.cu:12-63 for
// 11 terms) in FP32 with warp-level reductions, as the reference sums them
// in FP32: J' holds the NT response functions and, as row NT, the residual,
// over the 4 nl columns of the Stokes profiles.  Each lane forms the
// weighted products of its own samples for the first 64 entries and a
// shuffle butterfly sums them over the warp, then the last 1 (10 terms) or
// 13 (11 terms) entries the same way.  The reference sums each Stokes
// parameter sequentially and then the four in order; here every entry is
// one FP32 sum over the weighted products, in the order of a lane's
// samples, then a tree over the lanes.  The stray-light factor alpha of the
// scaled rows (me_der.cu:191-211) is applied to the sums in FP64.  alpha's
// RF is taken from the mixed profile `syn` when alpha_mixed
// (milosUtils.cu:675), else from the unmixed `pure`.  Results land in
// sm.alpha (packed) and sm.beta.
template <int LPL, int V>
__device__ __forceinline__ void normal_eq(const DevCfg& c, const double* m, bool alpha_mixed,
                                          const float (&pure)[LPL][4], const float (&sl)[LPL][4],
                                          const float (&syn)[LPL][4], const float (&ob)[LPL][4],
                                          const bool (&valid)[LPL], int lane, WarpSmem<LPL, V>& sm) {
  constexpr int NT = Variant<V>::NT, NE = ne_entries<NT>();
  static_assert(NE > 64 && NE <= 80, "64 entries, then up to 16");
  const double alfa = m[ALFA];
  bool mac_on = false;
  if constexpr (Variant<V>::MAC) mac_on = m[MAC] > 0.0001;
  // stage alpha's column and the residual of this lane's samples
#pragma unroll
  for (int k = 0; k < LPL; ++k) {
    const int l = lane + 32 * k;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const float asrc = alpha_mixed ? syn[k][s] : pure[k][s];
      sm.xrows[kXAlpha + s][l] = valid[k] ? asrc - sl[k][s] : 0.f;
      sm.xrows[kXRes + s][l] = valid[k] ? syn[k][s] - ob[k][s] : 0.f;
    }
  }
  uint32_t fixmask = 0;
#pragma unroll
  for (int i = 0; i < 11; ++i) fixmask |= (c.fix[i] ? 1u : 0u) << i;
  // the operand rows' offsets: one (Stokes, term) pair per lane
  for (int i = lane; i < 48; i += 32) {
    const int s = i / 12, t = i - 12 * s;
    bool scaled;
    sm.nero[s][t] = t <= NT ? jrow<LPL, V>(c, fixmask, t, s, mac_on, scaled) * row_pitch<LPL>() : 0;
  }
  __syncwarp();
  const float2 v01 = ne_pass64<LPL, V>(c, sm, lane);
  ne_store<LPL, V>(c, alfa, 2 * lane, v01.x, sm);
  ne_store<LPL, V>(c, alfa, 2 * lane + 1, v01.y, sm);
  constexpr int R = NE - 64, NL = R <= 1 ? 1 : R <= 2 ? 2 : R <= 4 ? 4 : R <= 8 ? 8 : 16;
  const float v2 = ne_pass<LPL, V, 64, NL>(c, sm, lane);
  constexpr int sh = NL == 1 ? 5 : NL == 2 ? 4 : NL == 4 ? 3 : NL == 8 ? 2 : 1;
  const int e2 = 64 + (lane >> sh);
  if ((lane & ((1 << sh) - 1)) == 0 && e2 < NE) ne_store<LPL, V>(c, alfa, e2, v2, sm);
  __syncwarp();
}

template <int LPL>
__device__ __forceinline__ float chisq(const DevCfg& c, const float (&syn)[LPL][4],
                                       const float (&ob)[LPL][4], const bool (&valid)[LPL]) {
  float acc = 0.f;
#pragma unroll
  for (int k = 0; k < LPL; ++k) {
    if (!valid[k]) continue;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const float d = syn[k][s] - ob[k][s];
      acc += __fdividef((d * d) * c.weight[s], c.noise);
    }
  }
  const float nfree = (float)(c.nl * 4 - c.nterms);
  return warp_sum(acc) / nfree;
}

// --------------------------------------------------------------- 10x10 solve
// delta = V diag(1/w) V^T beta where (w, V) come from 18 steps of the
// reference's parallel Jacobi (svdcordicf, svdcordic.cu:423-536; mil_svdf,
// milosUtils.cu:328-365).  A group of lanes owns the 15 2x2 blocks of the
// upper triangle; after every step the rotated blocks are written to the
// round-robin relabelled positions.  V is never formed: the step rotations
// are applied to beta on the way in and replayed transposed, in reverse, on
// the way out.  The matrix and the vector are double-buffered so a step
// needs one warp barrier, and every lane runs the same instruction stream
// (lanes past 14 of a group shadow block (0, 0) and store nothing).  With
// two solves per call each half-warp is a group with its own damping;
// otherwise the group is the warp.  The step loops stay rolled: the kernel
// is bound by instruction fetch, and a rolled loop keeps the solve's code
// small.
//
// Layout: block (p, q) occupies four consecutive floats (entries (2p, 2q),
// (2p, 2q + 1), (2p + 1, 2q), (2p + 1, 2q + 1); a diagonal block leaves its
// lower entry unused) at 4 solve_slot(block), so a lane reads its block
// with one 16-byte load; entry (i, j), i <= j, lives at solve_addr(i, j).
// The slot order and the dampings' offset kSolveH were chosen by a search
// over slot orders on the host, counting the bank conflicts of the step's
// accesses: they take 13 shared-memory wavefronts (4 for the block loads, 9
// for the four scattered stores) instead of 21 with row-major 10 x 11
// matrices.
constexpr int kSolveH = 68, kSolveB = 2 * kSolveH;   // damping and buffer strides (floats)
__host__ __device__ constexpr int solve_block(int p, int q) {   // p <= q: index in the lanes' order
  return p == q ? p : (p == 0 ? 4 + q : (p == 1 ? 7 + q : (p == 2 ? 9 + q : 14)));
}
// slots of the 15 blocks, 4 bits each (10, 15, 5, 11, 12, 8, 6, 1, 3, 9, 4,
// 14, 7, 0, 13): a shift, not a table that device code would build in
// local memory at every call
__host__ __device__ constexpr int solve_slot(int b) { return (int)((0xd07e493168cb5faull >> (4 * b)) & 0xfu); }
__host__ __device__ constexpr int solve_addr(int i, int j) {
  return i > j ? solve_addr(j, i) : 4 * solve_slot(solve_block(i / 2, j / 2)) + 2 * (i & 1) + (j & 1);
}

struct SolvePlan {
  int src;                      // offset of this lane's block in the working matrix
  int d00, d01, d10, d11;       // offsets its four entries move to
  int p, q;                     // block row / column (rotation pair), as group lanes
  int vin, vout0, vout1;        // beta pair read / relabelled write positions
  int base;                     // first lane of this lane's group
  int wdiag;                    // offset of diagonal entry g (lanes g < 10)
  // packed-triangle entries g + e * (32 / NS) (e < 2 NS, g the group lane)
  // this lane copies in: byte e holds the working-matrix offset, bit 7
  // marking a diagonal entry, 0xff none
  unsigned initpack;
};

template <int NS>
__host__ __device__ constexpr SolvePlan make_solve_plan(int lane) {
  constexpr int G = 32 / NS;
  const int g = lane & (G - 1);
  SolvePlan s{};
  const int bp[15] = {0, 1, 2, 3, 4, 0, 0, 0, 0, 1, 1, 1, 2, 2, 3};
  const int bq[15] = {0, 1, 2, 3, 4, 1, 2, 3, 4, 2, 3, 4, 3, 4, 4};
  const int pr[10] = {0, 2, 4, 1, 6, 3, 8, 5, 9, 7};
  s.base = lane - g;
  s.p = g < 15 ? bp[g] : 0;
  s.q = g < 15 ? bq[g] : 0;
  const int r0 = 2 * s.p, c0 = 2 * s.q;
  s.src = 4 * solve_slot(solve_block(s.p, s.q));
  s.wdiag = g < 10 ? solve_addr(g, g) : 0;
  auto dst = [&](int r, int c) { return solve_addr(pr[r], pr[c]); };
  s.d00 = dst(r0, c0);
  s.d01 = dst(r0, c0 + 1);
  s.d10 = dst(r0 + 1, c0);
  s.d11 = dst(r0 + 1, c0 + 1);
  s.vin = r0;
  s.vout0 = pr[r0];
  s.vout1 = pr[r0 + 1];
  // packed upper-triangle index i -> (row, col)
  s.initpack = 0xffffffffu;
  int i = 0;
  for (int r = 0; r < 10; ++r)
    for (int c = r; c < 10; ++c, ++i) {
      if (i >= g && (i - g) % G == 0 && (i - g) / G < 2 * NS) {
        const int e = (i - g) / G;
        const unsigned b = (unsigned)solve_addr(r, c) | (r == c ? 0x80u : 0u);
        s.initpack = (s.initpack & ~(0xffu << (8 * e))) | (b << (8 * e));
      }
    }
  return s;
}

// Every lane's plan for one and for two solves per call, built by the
// compiler: a kernel loads its lane's plan instead of deriving it (a
// prologue that a warp inverting one pixel per launch would pay in full).
struct SolvePlans {
  SolvePlan lane[32];
};
template <int NS>
__host__ __device__ constexpr SolvePlans solve_plans() {
  SolvePlans t{};
  for (int l = 0; l < 32; ++l) t.lane[l] = make_solve_plan<NS>(l);
  return t;
}
static __device__ const SolvePlans g_solve_plans[2] = {solve_plans<1>(), solve_plans<2>()};

// Solves for damping 1 + flambda into sm.vec[0][0] and, with two solves per
// call, for 1 + flambda2 into sm.vec[1][0].  `accurate` (the numerics mode)
// is a template parameter and the solve an out-of-line function: a runtime
// mode flag put three branches into every step, and inlined the solve adds
// to the register pressure of the whole LM loop (together 7.6 % of the
// kernel's time).
template <int LPL, int V, bool accurate>
__device__ __noinline__ void solve10(WarpSmem<LPL, V>& sm, const SolvePlan& pl, float flambda,
                                        float flambda2, int lane) {
  constexpr int NS = Variant<V>::SOLVES, G = 32 / NS;
  // The plan's indices (all below 256) packed one byte each into three
  // registers: read through the reference, every store to the shared-memory
  // blocks might alias the plan and each step would reload it from local
  // memory, and unpacked the eleven values spill (+3.6 % pixels/s packed).
  const unsigned w0 = (unsigned)pl.src | (unsigned)pl.d00 << 8 | (unsigned)pl.d01 << 16 | (unsigned)pl.d10 << 24;
  const unsigned w1 = (unsigned)pl.d11 | (unsigned)pl.vin << 8 | (unsigned)pl.vout0 << 16 | (unsigned)pl.vout1 << 24;
  const unsigned w2 = (unsigned)pl.p | (unsigned)(pl.base + pl.p) << 8 | (unsigned)(pl.base + pl.q) << 16 |
                     (unsigned)pl.wdiag << 24;
  const unsigned initpack = pl.initpack;
  auto at = [](unsigned w, int i) { return (int)((w >> (8 * i)) & 0xffu); };
  const int h = NS == 2 ? lane >> 4 : 0;
  const int g = lane & (G - 1);
  // damped matrix (diagonal x (1 + lambda), milosUtils.cu:648-652)
  const double damp = 1.0 + (double)(h ? flambda2 : flambda);
  float* A = &sm.A[h * kSolveH];
  float* B = A + kSolveB;
#pragma unroll
  for (int e = 0; e < 2 * NS; ++e) {
    const unsigned b = (initpack >> (8 * e)) & 0xffu;
    if (b != 0xffu) {
      const float a = sm.alpha[g + e * G];
      A[b & 0x7fu] = (b & 0x80u) ? (float)((double)a * damp) : a;
    }
  }
  float* va = &sm.vec[h][0][0];
  float* vb = &sm.vec[h][1][0];
  if (g < 10) va[g] = sm.beta[g];
  __syncwarp();

  const float quarter = (float)(kPi / 4);
  const float qclamp = __fdividef((float)kPi, 4.f);
  const bool diag = g < 5, active = g < 15;
#pragma unroll 1
  for (int step = 0; step < 18; ++step) {
    const float4 blk = *reinterpret_cast<const float4*>(A + at(w0, 0));
    const float m00 = blk.x, m01 = blk.y, m11 = blk.w;
    const float m10 = diag ? m01 : blk.z;
    const float b0 = va[at(w1, 1)], b1 = va[at(w1, 1) + 1];
    float th;
    if (m00 == m11) {
      th = quarter;
    } else {
      const float arc = accurate ? (2.f * m01) / (m11 - m00) : __fdividef(2.f * m01, m11 - m00);
      th = accurate ? atanf(arc) / 2.f : __fdividef(atanf(arc), 2.f);
      th = fminf(fmaxf(th, -qclamp), qclamp);
    }
    float sn, cs;
    sincos_mode(th, &sn, &cs, accurate);
    if (diag) {
      sm.cs[h][step][g] = cs;
      sm.sn[h][step][g] = sn;
    }
    const float cr = __shfl_sync(kFull, cs, at(w2, 1)), sr = __shfl_sync(kFull, sn, at(w2, 1));
    const float cc = __shfl_sync(kFull, cs, at(w2, 2)), sc = __shfl_sync(kFull, sn, at(w2, 2));
    const float t0 = m00 * cr - m10 * sr, t1 = m00 * sr + m10 * cr;
    const float u0 = m01 * cr - m11 * sr, u1 = m01 * sr + m11 * cr;
    const float n00 = t0 * cc - u0 * sc, n11 = t1 * sc + u1 * cc;
    const float n01 = diag ? 0.f : t0 * sc + u0 * cc;
    const float n10 = diag ? 0.f : t1 * cc - u1 * sc;
    if (active) {
      B[at(w0, 1)] = n00;
      B[at(w0, 2)] = n01;
      if (!diag) B[at(w0, 3)] = n10;   // a diagonal block's two off-diagonal entries are one
      B[at(w1, 0)] = n11;
    }
    if (diag) {
      vb[at(w1, 2)] = cs * b0 - sn * b1;
      vb[at(w1, 3)] = sn * b0 + cs * b1;
    }
    __syncwarp();
    float* tA = A; A = B; B = tA;
    float* tv = va; va = vb; vb = tv;
  }
  // 18 steps: the final matrix and vector are back in the first buffers, in
  // the original index order.  z = (V^T beta) / w with the |w| <= 1e-12 cut,
  // component g in group lane g's register.
  float y = 0.f;
  if (g < 10) {
    const float w = A[at(w2, 3)];
    const float inv = ((double)fabsf(w) > 1e-12) ? (1.f / w) : 0.f;
    y = va[g] * inv;
  }
  // delta = V z: undo the steps in reverse order.  Step `step` rotated
  // components (2k, 2k + 1) of pair k and relabelled them to positions
  // (r[2k], r[2k + 1]) of the round-robin permutation r = {0, 2, 4, 1, 6, 3,
  // 8, 5, 9, 7}; undoing it, component g takes pair k = g / 2's two
  // relabelled components from their lanes (shuffles; positions packed one
  // nibble per pair) and that pair's rotation, transposed.
  const int k = g < 10 ? g >> 1 : 4, base = lane - g;
  const int y0_lane = base + (int)((0x98640u >> (4 * k)) & 0xfu);
  const int y1_lane = base + (int)((0x75312u >> (4 * k)) & 0xfu);
  const bool second = (g & 1) != 0;
#pragma unroll 1
  for (int step = 17; step >= 0; --step) {
    const float y0 = __shfl_sync(kFull, y, y0_lane), y1 = __shfl_sync(kFull, y, y1_lane);
    const float cs = sm.cs[h][step][k], sn = sm.sn[h][step][k];
    y = second ? -sn * y0 + cs * y1 : cs * y0 + sn * y1;
  }
  if (g < 10) sm.vec[h][0][g] = y;
  __syncwarp();
}

// --------------------------------------------------------------- 11x11 solve (FP64)
// delta = V diag(1/w) V^T beta for the damped 11x11 normal matrix in double
// with the |w| <= 1e-12 cut (mil_svd, milosUtils.cu:280-325).  The reference
// takes (w, V) from a converged Golub-Reinsch SVD (svdcmp, svdcmp.cu:37-234);
// for this symmetric positive semi-definite matrix the same decomposition is
// reached by cyclic two-sided Jacobi rotations run to convergence.  The
// matrix is padded to 12x12 with a zero row and column (eigenvalue 0, cut).
// Lanes 0..20 own the 21 2x2 blocks of the upper triangle and write each
// rotated block to its round-robin relabelled position (a 12-index
// tournament: every index pair meets once in 11 steps); V's columns follow
// the same relabelling while its rows stay in parameter order.  Sweeps
// repeat until one leaves every off-diagonal entry at or below 1e-15 of the
// geometric mean of its diagonal pair, at most 16.
struct Solve11Plan {
  int src;                 // this lane's block (row-major 12x12 offset)
  int d00, d01, d10, d11;  // where its entries move
  int p, q;                // block row / column (rotation pair)
  int vrow, vpair;         // V update: row and first of three pairs (lanes < 24)
};

__device__ __forceinline__ int perm12(int i) {
  const int pr[12] = {0, 2, 4, 1, 6, 3, 8, 5, 10, 7, 11, 9};
  return pr[i];
}

__device__ __forceinline__ Solve11Plan make_solve11_plan(int lane) {
  Solve11Plan s;
  int p = 0, q = 0;
  if (lane < 6) {
    p = q = lane;
  } else if (lane < 21) {
    int k = 6;
    for (int a = 0; a < 6; ++a)
      for (int b = a + 1; b < 6; ++b, ++k)
        if (k == lane) { p = a; q = b; }
  }
  s.p = p;
  s.q = q;
  const int r0 = 2 * p, c0 = 2 * q;
  s.src = r0 * 12 + c0;
  auto dst = [](int r, int c) {
    const int a = perm12(r), b = perm12(c);
    return (a < b ? a : b) * 12 + (a < b ? b : a);
  };
  s.d00 = dst(r0, c0);
  s.d01 = dst(r0, c0 + 1);
  s.d10 = dst(r0 + 1, c0);
  s.d11 = dst(r0 + 1, c0 + 1);
  s.vrow = lane % 12;
  s.vpair = (lane / 12) * 3;
  return s;
}

template <int LPL, int V>
__device__ __forceinline__ void solve11(WarpSmem<LPL, V>& sm, const Solve11Plan& pl, float flambda,
                                        int lane) {
  static_assert(V == 2, "the FP64 solve belongs to the 11-term variant");
  // damped matrix in double (milosUtils.cu:787-791), padded to 12x12
  const double damp = 1.0 + (double)flambda;
  double* A = sm.j11.A[0];
  double* B = sm.j11.A[1];
  double* Va = sm.j11.V[0];
  double* Vb = sm.j11.V[1];
  for (int i = lane; i < 144; i += 32) {
    const int r = i / 12, c = i - 12 * (i / 12);
    double v = 0.0;
    if (r < 11 && c < 11) {
      const int a = r < c ? r : c, b = r < c ? c : r;
      v = (double)sm.alpha[upk<11>(a, b)];
      if (r == c) v = v * damp;
    }
    A[i] = v;
    Va[i] = (r == c) ? 1.0 : 0.0;
  }
  if (lane < 12) sm.b11[lane] = lane < 11 ? (double)sm.beta[lane] : 0.0;
  __syncwarp();

  const bool diag = lane < 6, active = lane < 21, vlane = lane < 24;
  bool sweep_moved = false;
  for (int step = 0; step < 16 * 11; ++step) {
    const double m00 = A[pl.src], m01 = A[pl.src + 1], m11 = A[pl.src + 13];
    const double m10 = diag ? m01 : A[pl.src + 12];
    bool moved = false;
    if (diag) {
      double cs = 1.0, sn = 0.0;
      if (m01 != 0.0) {
        moved = fabs(m01) > 1e-15 * sqrt(fabs(m00)) * sqrt(fabs(m11));
        const double tau = (m11 - m00) / (2.0 * m01);
        const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
        cs = 1.0 / sqrt(1.0 + t * t);
        sn = t * cs;
      }
      sm.c11[lane] = cs;
      sm.s11[lane] = sn;
    }
    sweep_moved |= __any_sync(kFull, moved);
    __syncwarp();
    const double cr = sm.c11[pl.p], sr = sm.s11[pl.p];
    const double cc = sm.c11[pl.q], sc = sm.s11[pl.q];
    const double t0 = m00 * cr - m10 * sr, t1 = m00 * sr + m10 * cr;
    const double u0 = m01 * cr - m11 * sr, u1 = m01 * sr + m11 * cr;
    const double n00 = t0 * cc - u0 * sc, n11 = t1 * sc + u1 * cc;
    const double n01 = diag ? 0.0 : t0 * sc + u0 * cc;
    const double n10 = diag ? 0.0 : t1 * cc - u1 * sc;
    if (active) {
      B[pl.d00] = n00;
      B[pl.d01] = n01;
      B[pl.d10] = n10;
      B[pl.d11] = n11;
    }
    if (vlane) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const int pp = pl.vpair + k;
        const double c2 = sm.c11[pp], s2 = sm.s11[pp];
        const double v0 = Va[pl.vrow * 12 + 2 * pp], v1 = Va[pl.vrow * 12 + 2 * pp + 1];
        Vb[pl.vrow * 12 + perm12(2 * pp)] = v0 * c2 - v1 * s2;
        Vb[pl.vrow * 12 + perm12(2 * pp + 1)] = v0 * s2 + v1 * c2;
      }
    }
    __syncwarp();
    double* tA = A; A = B; B = tA;
    double* tV = Va; Va = Vb; Vb = tV;
    if (step % 11 == 10) {
      if (!sweep_moved) break;
      sweep_moved = false;
    }
  }
  // z = V^T beta / w with the cut, then delta = V z
  if (lane < 12) {
    double z = 0.0;
    for (int r = 0; r < 11; ++r) z += sm.b11[r] * Va[r * 12 + lane];
    const double w = A[lane * 13];
    sm.z11[lane] = z * ((fabs(w) > 1e-12) ? (1 / w) : 0.0);
  }
  __syncwarp();
  if (lane < 11) {
    double d = 0.0;
    for (int k = 0; k < 12; ++k) d += Va[lane * 12 + k] * sm.z11[k];
    sm.dd[lane] = d;
  }
  __syncwarp();
}

// The same step by Gaussian elimination in double.  The damped normal
// matrix is symmetric and positive definite on the parameters whose response
// functions are not zero, and exactly zero in the rows and columns of the
// others (fixed parameters): there the SVD's cut (|w| <= 1e-12) gives a zero
// step, and so does skipping a pivot that is exactly zero; on the rest both
// give the inverse.  A pivot that is positive but below 1e-10 of its
// diagonal, where the cut might act on a nearly singular direction, makes
// the function return false and the caller takes the Jacobi solve above.
// 11 elimination steps over a 12 x 12 working copy instead of up to 16
// sweeps of 11 rotation steps.
template <int LPL, int V>
__device__ __forceinline__ bool solve11_elim(WarpSmem<LPL, V>& sm, float flambda, int lane) {
  static_assert(V == 2, "the FP64 solve belongs to the 11-term variant");
  const double damp = 1.0 + (double)flambda;
  double* A = sm.j11.A[0];
  for (int i = lane; i < 144; i += 32) {
    const int r = i / 12, c = i - 12 * (i / 12);
    double v = 0.0;
    if (r < 11 && c < 11) {
      const int a = r < c ? r : c, b = r < c ? c : r;
      v = (double)sm.alpha[upk<11>(a, b)];
      if (r == c) v = v * damp;
    }
    A[i] = v;
  }
  if (lane < 12) sm.b11[lane] = lane < 11 ? (double)sm.beta[lane] : 0.0;
  __syncwarp();
  for (int k = 0; k < 11; ++k) {
    const double piv = A[k * 13];
    if (piv == 0.0) continue;   // a zero row and column: zero step
    if (!(piv > 1e-10 * fabs((double)sm.alpha[upk<11>(k, k)] * damp))) return false;
    const double inv = 1.0 / piv;
    const int m = 10 - k;       // rows / columns after k
    for (int e = lane; e < m * m; e += 32) {
      const int i = k + 1 + e / m, j = k + 1 + e % m;
      A[i * 12 + j] -= A[i * 12 + k] * inv * A[k * 12 + j];
    }
    if (lane > k && lane < 11) sm.b11[lane] -= A[lane * 12 + k] * inv * sm.b11[k];
    __syncwarp();
  }
  if (lane == 0) {
    for (int k = 10; k >= 0; --k) {
      const double piv = A[k * 13];
      double x = 0.0;
      if (piv != 0.0) {
        double s = sm.b11[k];
        for (int j = k + 1; j < 11; ++j) s -= A[k * 12 + j] * sm.dd[j];
        x = s / piv;
      }
      sm.dd[k] = x;
    }
  }
  __syncwarp();
  return true;
}

// --------------------------------------------------------------- model updates
// model -= delta on free parameters with the reference's step limits
// (AplicaDeltaf, milosUtils.cu:93-159, float delta; AplicaDelta, :30-91,
// double delta for 11 terms), then range checks (check, :160-238).  The
// filling factor's step is slot 9 of 10 or slot 10 of 11.
template <int NT, typename T>
__device__ __forceinline__ void apply_delta_check(const DevCfg& c, const double* m, const T* d,
                                                  double* t) {
  T aux;
  if (c.fix[ETA0]) t[ETA0] = m[ETA0] - d[0];
  if (c.fix[BFLD]) {
    aux = d[1];
    if (aux < -300) aux = -300; else if (aux > 300) aux = 300;
    t[BFLD] = m[BFLD] - aux;
  }
  if (c.fix[VLOS]) t[VLOS] = m[VLOS] - d[2];
  if (c.fix[DOPP]) t[DOPP] = m[DOPP] - d[3];
  if (c.fix[AA]) t[AA] = m[AA] - d[4];
  if (c.fix[GM]) {
    aux = d[5];
    if (aux < -30) aux = -30; else if (aux > 30) aux = 30;
    t[GM] = m[GM] - aux;
  }
  if (c.fix[AZ]) {
    aux = d[6];
    if (aux < -30) aux = -30; else if (aux > 30) aux = 30;
    t[AZ] = m[AZ] - aux;
  }
  if (c.fix[S0]) t[S0] = m[S0] - d[7];
  if (c.fix[S1]) t[S1] = m[S1] - d[8];
  if (c.fix[MAC]) t[MAC] = m[MAC] - d[9];
  if (c.fix[ALFA]) t[ALFA] = m[ALFA] - d[NT == 11 ? 10 : 9];
  if (t[BFLD] < 0) { t[BFLD] = -t[BFLD]; t[GM] = 180.0 - t[GM]; }
  if (t[BFLD] > 5000) t[BFLD] = 5000;
  if (t[GM] < 0) t[GM] = -t[GM];
  if (t[GM] > 180) t[GM] = 360.0 - t[GM];
  if (t[AZ] < 0) t[AZ] = 180 + t[AZ];
  if (t[AZ] > 180) t[AZ] = t[AZ] - 180.0;
  if (t[ETA0] < 1) t[ETA0] = 1;
  if (t[ETA0] > 2500) t[ETA0] = 2500;
  if (t[VLOS] < -20) t[VLOS] = -20;
  if (t[VLOS] > 20) t[VLOS] = 20;
  if (t[DOPP] < 0.0001) t[DOPP] = 0.0001;
  if (t[DOPP] > 0.6) t[DOPP] = 0.6;
  if (t[AA] < 0.0001) t[AA] = 0.0001;
  if (t[AA] > 10.0) t[AA] = 10.0;
  if (t[S0] < 0.0001) t[S0] = 0.0001;
  if (t[S0] > 2.00) t[S0] = 2.00;
  if (t[S1] < 0.0001) t[S1] = 0.0001;
  if (t[S1] > 2.00) t[S1] = 2.00;
  if (t[MAC] < 0) t[MAC] = 0;
  if (t[MAC] > 4) t[MAC] = 4;
  if (t[ALFA] < 0) t[ALFA] = 0.0;
  if (t[ALFA] > 1.0) t[ALFA] = 1.0;
}

// Weak-field and centre-of-gravity estimates of B, vlos, gamma, phi
// (estimacionesClasicas, milosUtils.cu:386-563).  Sums are warp reductions in
// double.  Lane 0 writes m.  for_init (the LM start): gamma in (85, 95]
// degrees is moved off 90 before B is formed, and lm_mils' NaN fallbacks
// follow (:621-628); otherwise (the classical-estimates mode,
// gmilos.cu:383-404) S0 receives the longitudinal field.
template <int LPL>
__device__ __forceinline__ uint32_t classical_warp(const DevCfg& c, const float (&ob)[LPL][4],
                                                   const double (&dld)[LPL], const bool (&valid)[LPL],
                                                   int lane, double* m, bool for_init = true) {
  const int nl = c.nl;
  int bmin = nl, emax = 0;
#pragma unroll
  for (int k = 0; k < LPL; ++k) {
    const int l = lane + 32 * k;
    if (valid[k] && !(ob[k][0] < 0.f)) {
      bmin = min(bmin, l);
      emax = max(emax, l + 1);
    }
  }
  const int b = __reduce_min_sync(kFull, bmin);
  const int e = __reduce_max_sync(kFull, emax);
  uint32_t st = 0;
  double Ic;
  {
    const int l = e - 1;
    float v = 0.f;
#pragma unroll
    for (int k = 0; k < LPL; ++k)
      if (l >= 0 && (l >> 5) == k) v = ob[k][0];
    const float icf = __shfl_sync(kFull, v, l >= 0 ? (l & 31) : 0);
    Ic = (e > 0) ? (double)icf : __longlong_as_double(0x7ff8000000000000ll);
    if (e <= 0) st |= 0x20u;
  }
  double x = 0, y = 0, xv = 0, yv = 0, x2 = 0, y2 = 0, x3 = 0, y3 = 0, su = 0, sq = 0;
#pragma unroll
  for (int k = 0; k < LPL; ++k) {
    if (!valid[k]) continue;
    const int l = lane + 32 * k;
    const float I = ob[k][0], Q = ob[k][1], U = ob[k][2], V = ob[k][3];
    const double d = dld[k];
    if (l >= b && l < e - 1) {
      if (I > -1 && V > -1) {
        const double aux = Ic - (double)(I + V);
        const double avl = Ic - (double)I;
        x += aux * d;
        xv += avl * d;
        y += aux;
        yv += avl;
        const double aux2 = Ic - (double)(I - V);
        x2 += aux2 * d;
        y2 += aux2;
      }
      if (Q > -1 && U > -1 && V > -1) {
        const double L = (double)fabsf(sqrtf(Q * Q + U * U));
        const double mm = fabs((4 * d * L));
        x3 += (double)fabsf(V) * mm;
        y3 += (double)(fabsf(V) * fabsf(V));
      }
    }
    if (U > -1 && Q > -1) {
      if (fabs((double)U) > 0.0001 || fabs((double)Q) > 0.0001) {
        su += U;
        sq += Q;
      }
    }
  }
  x = warp_sum_d(x); y = warp_sum_d(y); xv = warp_sum_d(xv); yv = warp_sum_d(yv);
  x2 = warp_sum_d(x2); y2 = warp_sum_d(y2); x3 = warp_sum_d(x3); y3 = warp_sum_d(y3);
  su = warp_sum_d(su); sq = warp_sum_d(sq);
  const double lp = (fabs(y) > 1e-15) ? x / y : 0;
  const double lmn = (fabs(y2) > 1e-15) ? x2 / y2 : 0;
  const double C = (kLarmor * (c.lambda0 * c.lambda0) * (double)c.geff);
  const double Blos = (1 / C) * ((lp - lmn) / 2);
  double Vlos = (kVlight / (c.lambda0)) * ((xv / yv) / 2);
  y3 = y3 * fabs((3 * C * Blos));
  const double tg = fabs(sqrt(x3 / y3));
  double grad = atan(tg);
  double gamma = grad * (180 / kPi);
  if (for_init) {
    if (gamma >= 85 && gamma <= 90) grad = 85 * (kPi / 180);
    if (gamma > 90 && gamma <= 95) grad = 95 * (kPi / 180);
  }
  if (Blos < 0) gamma = (180) - gamma;
  double phi = (atan(su / sq) * 180 / kPi) / 2;
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
  double B = (Baux > 4000 ? 4000 : Baux);
  if (for_init) {
    if (isnan(B)) { B = 1; st |= 0x01u; }
    if (isnan(Vlos)) { Vlos = 1e-3; st |= 0x01u; }
    if (isnan(gamma)) { gamma = 1; st |= 0x01u; }
    if (isnan(phi)) { phi = 1; st |= 0x01u; }
  }
  if (lane == 0) {
    m[BFLD] = B;
    m[VLOS] = Vlos;
    m[GM] = gamma;
    m[AZ] = phi;
    if (!for_init) m[S0] = Blos;
  }
  return st;
}

}  // namespace gm
