// gm_kernels.cu -- persistent LM inversion kernel, synthesis kernels.
#include <cstddef>

#include "gm_kernels.cuh"

namespace gm {

// Load this lane's observed samples (zero past nl).
template <int LPL>
__device__ __forceinline__ void load_pixel(const float* __restrict__ p, int nl, int lane,
                                           float (&ob)[LPL][4]) {
#pragma unroll
  for (int k = 0; k < LPL; ++k) {
    const int l = lane + 32 * k;
#pragma unroll
    for (int s = 0; s < 4; ++s) ob[k][s] = (l < nl) ? __ldg(p + s * nl + l) : 0.f;
  }
}

// Per-pixel wavelength grids: this pixel's offsets from row pix of the map
// (the same double difference and float rounding the host applies to the
// configured grid) and its absolute wavelengths; null with the configured grid.
template <int LPL>
__device__ __forceinline__ const double* pixel_grid(const DevCfg& c, unsigned long long pix, int lane,
                                                    float (&dlv)[LPL], double (&dld)[LPL]) {
  if (!c.lambda_per_pixel) return nullptr;
  const double* lp = c.lam_map + pix * (unsigned long long)c.nl;
#pragma unroll
  for (int k = 0; k < LPL; ++k) {
    const int l = lane + 32 * k;
    if (l < c.nl) {
      const double d = __ldg(lp + l) - c.lambda0;
      dld[k] = d;
      dlv[k] = (float)d;
    }
  }
  return lp;
}

// Staged rows start at zero (rows that no phase stages then hold zeros in
// the tensor-core tiles); the normal equations' row of ones is 1 up to nl.
template <int LPL, int V>
__device__ __forceinline__ void init_rows(const DevCfg& c, WarpSmem<LPL, V>& sm, int lane) {
  for (int i = lane; i < WarpSmem<LPL, V>::NR * row_pitch<LPL>(); i += 32) (&sm.rows[0][0])[i] = 0.f;
  for (int i = lane; i < kXRows * row_pitch<LPL>(); i += 32) {
    const int r = i / row_pitch<LPL>(), l = i - r * row_pitch<LPL>();
    (&sm.xrows[0][0])[i] = (r == kXOne && l < c.nl) ? 1.f : 0.f;
  }
  __syncwarp();
}

// Warp-private shared memory lives in the dynamic allocation (the larger
// variants exceed the 48 KB static limit), after the block's PSF taps.
template <int LPL, int V>
__device__ __forceinline__ WarpSmem<LPL, V>& warp_smem() {
  return reinterpret_cast<WarpSmem<LPL, V>*>(gm_dyn_smem + tap_bytes<LPL>())[threadIdx.x >> 5];
}

template <int LPL, int V>
constexpr int min_blocks() { return LPL == 1 ? (V == 2 ? 3 : 4) : 5; }

// One warp per pixel, pixels taken from a global cursor until the cube is
// done (lm_mils, milosUtils.cu:574-710, and lm_mils_11, :713-850, with their
// per-thread contiguous pixel slices replaced by work stealing).  The
// initial point is handled as an accepted step of the same loop, so the
// synthesis and the response functions each appear once in the code.
template <int LPL, int V>
__global__ void __launch_bounds__(warps_per_block<LPL>() * 32, min_blocks<LPL, V>())
invert_kernel(const DevCfg c, const InvertArgs a) {
  constexpr int NT = Variant<V>::NT;
  const int lane = threadIdx.x & 31;
  load_taps<LPL>(c);
  WarpSmem<LPL, V>& sm = warp_smem<LPL, V>();
  init_rows<LPL, V>(c, sm, lane);

  const int nl = c.nl;
  float dlv[LPL];
  double dld[LPL];
  bool valid[LPL];
#pragma unroll
  for (int k = 0; k < LPL; ++k) {
    const int l = lane + 32 * k;
    valid[k] = l < nl;
    dlv[k] = valid[k] ? c.dl[l] : 0.f;
    dld[k] = valid[k] ? c.dld[l] : 0.0;
  }
  float slg[LPL][4];
  if (c.use_slight && !c.slight_per_pixel) load_pixel<LPL>(c.slight, nl, lane, slg);
  else {
#pragma unroll
    for (int k = 0; k < LPL; ++k)
#pragma unroll
      for (int s = 0; s < 4; ++s) slg[k][s] = 0.f;
  }

  const SolvePlan plan = g_solve_plans[Variant<V>::SOLVES - 1].lane[lane];
  Solve11Plan plan11;
  if constexpr (NT == 11) plan11 = make_solve11_plan(lane);
  unsigned long long my_iter = 0, my_acc = 0;
  while (true) {
    unsigned long long pix = 0;
    if (lane == 0) pix = atomicAdd(&a.work->next_pixel, 1ull);
    pix = __shfl_sync(kFull, pix, 0);
    if (pix >= (unsigned long long)a.npix) break;
    const size_t off = (size_t)pix * 4 * nl;

    float ob[LPL][4];
    load_pixel<LPL>(a.iquv + off, nl, lane, ob);
    if (c.use_slight && c.slight_per_pixel) load_pixel<LPL>(c.slight + off, nl, lane, slg);
    const double* lamp = pixel_grid<LPL>(c, pix, lane, dlv, dld);

    // initial model
    if (lane < 11) sm.m[lane] = a.init_models ? a.init_models[pix * 11 + lane] : c.init[lane];
    __syncwarp();
    uint32_t st = a.init_status ? a.init_status[pix] : 0u;
    if (c.init_mode == 0) st |= classical_warp<LPL>(c, ob, dld, valid, lane, sm.m);
    __syncwarp();

    Lane<LPL, V> ln;
    Angles an;
    float syn[LPL][4], pure[LPL][4];
    float flambda = c.ilambda, pbf = 1.f, ochisqr = 0.f, chisqr0 = 0.f;
    int iter = 0, acc = 0;
    bool stop = false, first = true;
    // sm.vec[1][0] holds the step for the damping that the last trial's
    // rejection moved to (solved beside the trial's own step)
    bool have_next = false, solved = false;
    while (true) {
      if (!first) {
        if constexpr (NT == 10) {
          const bool reuse = Variant<V>::SOLVES == 2 && have_next;
          if (!reuse) {
            if (c.numerics) solve10<LPL, V, true>(sm, plan, flambda, flambda * 10.f * pbf, lane);
            else solve10<LPL, V, false>(sm, plan, flambda, flambda * 10.f * pbf, lane);
          }
          solved = !reuse;
          if (lane == 0) apply_delta_check<10>(c, sm.m, sm.vec[reuse ? 1 : 0][0], sm.t);
        } else {
          if (!solve11_elim<LPL, V>(sm, flambda, lane)) solve11<LPL, V>(sm, plan11, flambda, lane);
          if (lane == 0) apply_delta_check<11>(c, sm.m, sm.dd, sm.t);
        }
        __syncwarp();
      }
      synth_lane<LPL, V>(c, first ? sm.m : sm.t, dlv, lane, ln, an, syn, pure, slg, sm, lamp);
      const float chisqr = chisq<LPL>(c, syn, ob, valid);
      bool accept = first;
      if (!first) {
        if (iter == 0) {
          if (a.step_delta && lane < NT)
            a.step_delta[pix * NT + lane] = (NT == 10) ? sm.vec[0][0][lane] : (float)sm.dd[lane];
          if (a.step_trial && lane < 11) a.step_trial[pix * 11 + lane] = sm.t[lane];
          if (lane == 0 && a.step_chi2_start) a.step_chi2_start[pix] = chisqr0;
          if (lane == 0 && a.step_chi2_trial) a.step_chi2_trial[pix] = chisqr;
        }
        // stop rules and damping schedule (milosUtils.cu:667-696)
        if ((double)fabsf(((ochisqr) - (chisqr)) * 100 / (chisqr)) < c.toplim || (chisqr) < 0.0001f) {
          stop = true;
          st |= GM_PIX_CHI2_EXIT;
        }
        accept = (chisqr) - (ochisqr) < 0.f;
        if (accept) {
          flambda = flambda / (5.f * pbf);
          if (c.stop_dchi2 > 0.0 && (double)(ochisqr - chisqr) < c.stop_dchi2) stop = true;
          if (lane < 11) sm.m[lane] = sm.t[lane];
          __syncwarp();
          ++acc;
        } else {
          flambda = flambda * 10.f * pbf;
        }
        if (flambda > 1e+7f || flambda < 1e-25f) {
          stop = true;
          st |= GM_PIX_LAMBDA_EXIT;
        }
        ++iter;
        // the rejection damping above is the second one the solve just took
        have_next = !accept && solved;
        if (c.logclambda) pbf = log10f(chisqr) / log10f(chisqr0);
      }
      if (accept) {
        // response functions and normal equations at the accepted model; the
        // alpha RF uses the mixed profile after the first step (milosUtils.cu:675)
        rf_rows<LPL, V>(c, sm.m, ln, an, lane, sm, lamp);
        normal_eq<LPL, V>(c, sm.m, !first && c.quirks, pure, slg, syn, ob, valid, lane, sm);
        ochisqr = chisqr;
      }
      if (first) {
        chisqr0 = ochisqr;
        if (lane < 11) sm.t[lane] = sm.m[lane];
        __syncwarp();
        first = false;
        continue;
      }
      if (iter >= c.miter || stop) break;
    }
    if (!stop) st |= GM_PIX_MAXITER;
    if (!isfinite(ochisqr)) st |= GM_PIX_NONFINITE;

    // outputs: last accepted model and chi2, trial count, last trial synthesis
    if (lane < 11) {
      if (a.model) a.model[pix * 11 + lane] = (float)sm.m[lane];
      if (a.model_f64) a.model_f64[pix * 11 + lane] = sm.m[lane];
    }
    if (lane == 0) {
      if (a.chi2) a.chi2[pix] = ochisqr;
      if (a.iters) a.iters[pix] = iter;
      if (a.accepted) a.accepted[pix] = acc;
      if (a.status) a.status[pix] = st;
    }
    if (a.fitted) {
#pragma unroll
      for (int k = 0; k < LPL; ++k) {
        const int l = lane + 32 * k;
        if (l < nl)
#pragma unroll
          for (int s = 0; s < 4; ++s) a.fitted[off + s * nl + l] = syn[k][s];
      }
    }
    my_iter += iter;
    my_acc += acc;
    __syncwarp();
  }
  if (lane == 0 && (my_iter | my_acc)) {
    atomicAdd(&a.work->iterations, my_iter);
    atomicAdd(&a.work->accepted, my_acc);
  }
}

// ------------------------------------------------- wave-synchronous inversion
// The same LM iteration as invert_kernel (lm_mils, milosUtils.cu:574-710,
// and lm_mils_11, :713-850), split at its two halves and run for every pixel
// of a chunk in lockstep waves.  Wave w launches trial_kernel over the
// pixels still iterating -- the step solve, the step limits, the trial
// synthesis with PSF and stray light, chi2 and the damping schedule -- then
// accept_kernel over the pixels whose trial was accepted: response
// functions, their PSF and the normal equations.  Each kernel executes
// about a third of invert_kernel's code, so the warps of an SM share one hot
// instruction working set, and each has its own register budget (at nl <=
// 32 the trial half runs 28 warps per SM, the accept half 20).  A pixel's
// LM state lives in a PixLM record between the kernels; the per-lane Voigt
// and Zeeman terms, angles and profiles of an accepted trial reach the
// accept kernel through a staging row block, so nothing is recomputed: each
// pixel runs invert_kernel's operations in its order (compiled as other
// kernels, the multiply-adds the compiler fuses differ, so results agree
// with invert_kernel's to rounding, not bit for bit).

// Resident blocks per SM: registers for the 10-term variants; the 11-term
// variant's FP64 Jacobi matrices make shared memory the limit.
template <int LPL, int V>
constexpr int trial_min_blocks() { return V == 2 ? (LPL == 1 ? 5 : 8) : (LPL == 1 ? 7 : 10); }
template <int LPL, int V>
constexpr int accept_min_blocks() { return V == 2 ? (LPL == 1 ? 5 : 5) : 5; }

// The trial half touches the warp's shared memory only up to the first
// 8-row tile of staged rows (the synthesis PSF stages rows 0-3) -- or, in
// the 11-term variant, up to the end of the solve's matrices that share the
// rows' space -- so its warps are packed at that stride: half the
// footprint, more warps per SM.
template <int LPL, int V>
__host__ __device__ constexpr size_t trial_warp_bytes() {
  using WS = WarpSmem<LPL, V>;
  constexpr size_t tile = 8 * row_pitch<LPL>() * sizeof(float);
  constexpr size_t solve = V == 2 ? sizeof(Jacobi11<true>) : 0;   // the 11-term solve's matrices
  return (offsetof(WS, rows) + (tile > solve ? tile : solve) + 15) & ~(size_t)15;
}
template <int LPL, int V>
constexpr bool xrows_follow_rows() {
  using WS = WarpSmem<LPL, V>;
  return offsetof(WS, xrows) == offsetof(WS, rows) + sizeof(WS::rows);
}
static_assert(xrows_follow_rows<1, 0>() && xrows_follow_rows<1, 1>() && xrows_follow_rows<1, 2>() &&
                  xrows_follow_rows<2, 0>() && xrows_follow_rows<2, 1>() && xrows_follow_rows<2, 2>(),
              "the operand rows must follow the staged rows");
template <int LPL, int V>
__device__ __forceinline__ WarpSmem<LPL, V>& trial_smem() {
  return *reinterpret_cast<WarpSmem<LPL, V>*>(gm_dyn_smem + tap_bytes<LPL>() +
                                               (threadIdx.x >> 5) * trial_warp_bytes<LPL, V>());
}

// Staged rows of an accepted trial (one float per lane each): per sample
// slot k the 15 Lane terms, syn and pure, and with macroturbulence the
// profile before its convolution; the last row holds the angles.
template <int LPL, int V>
__device__ __forceinline__ void stage_put(float* __restrict__ q, const Lane<LPL, V>& ln, const Angles& an,
                                          const float (&syn)[LPL][4], const float (&pure)[LPL][4], int lane) {
  constexpr int R = stage_rows_per_slot(Variant<V>::MAC);
#pragma unroll
  for (int k = 0; k < LPL; ++k) {
    float* r = q + k * R * 32 + lane;
#pragma unroll
    for (int g = 0; g < 3; ++g) {
      r[(0 + g) * 32] = ln.fi[k][g];
      r[(3 + g) * 32] = ln.shi[k][g];
      r[(6 + g) * 32] = ln.lh[k][g];
      r[(9 + g) * 32] = ln.lf[k][g];
      r[(12 + g) * 32] = ln.lu[k][g];
    }
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      r[(15 + s) * 32] = syn[k][s];
      r[(19 + s) * 32] = pure[k][s];
      if constexpr (Variant<V>::MAC) r[(23 + s) * 32] = ln.mc[k][s];
    }
  }
  if (lane == 0) {
    float* r = q + LPL * R * 32;
    r[0] = an.cosi; r[1] = an.sinis; r[2] = an.sina; r[3] = an.cosa; r[4] = an.sinda;
    r[5] = an.cosda; r[6] = an.sindi; r[7] = an.cosdi; r[8] = an.cosis_2;
  }
}

template <int LPL, int V>
__device__ __forceinline__ void stage_get(const float* __restrict__ q, Lane<LPL, V>& ln, Angles& an,
                                          float (&syn)[LPL][4], float (&pure)[LPL][4], int lane) {
  constexpr int R = stage_rows_per_slot(Variant<V>::MAC);
#pragma unroll
  for (int k = 0; k < LPL; ++k) {
    const float* r = q + k * R * 32 + lane;
#pragma unroll
    for (int g = 0; g < 3; ++g) {
      ln.fi[k][g] = r[(0 + g) * 32];
      ln.shi[k][g] = r[(3 + g) * 32];
      ln.lh[k][g] = r[(6 + g) * 32];
      ln.lf[k][g] = r[(9 + g) * 32];
      ln.lu[k][g] = r[(12 + g) * 32];
    }
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      syn[k][s] = r[(15 + s) * 32];
      pure[k][s] = r[(19 + s) * 32];
      if constexpr (Variant<V>::MAC) ln.mc[k][s] = r[(23 + s) * 32];
    }
  }
  const float* r = q + LPL * R * 32;
  an.cosi = r[0]; an.sinis = r[1]; an.sina = r[2]; an.cosa = r[3]; an.sinda = r[4];
  an.cosda = r[5]; an.sindi = r[6]; an.cosdi = r[7]; an.cosis_2 = r[8];
}

// Outputs of a pixel that stopped (as invert_kernel writes them).
template <int LPL, bool MG>
__device__ __forceinline__ void finish_pixel(const InvertArgs& a, const double* m, float ochisqr, int iter,
                                             int acc, uint32_t st, const float (&syn)[LPL][4],
                                             uint64_t pix, int nl, int lane, const MultiGrid& mg) {
  if (lane < 11) {
    if (a.model) a.model[pix * 11 + lane] = (float)m[lane];
    if (a.model_f64) a.model_f64[pix * 11 + lane] = m[lane];
  }
  if (lane == 0) {
    if (a.chi2) a.chi2[pix] = ochisqr;
    if (a.iters) a.iters[pix] = iter;
    if (a.accepted) a.accepted[pix] = acc;
    if (a.status) a.status[pix] = st;
  }
  if (a.fitted) {
    const size_t off = MG ? (size_t)mg.off[pix] : (size_t)pix * 4 * nl;
#pragma unroll
    for (int k = 0; k < LPL; ++k) {
      const int l = lane + 32 * k;
      if (l < nl)
#pragma unroll
        for (int s = 0; s < 4; ++s) a.fitted[off + s * nl + l] = syn[k][s];
    }
  }
}

// The configuration a pixel runs on: the launch's own or, in a ragged
// batch, its grid's (device memory).
template <bool MG>
__device__ __forceinline__ const DevCfg& pixel_cfg(const DevCfg& c0, const DevCfg* cp) {
  if constexpr (MG) return *cp;
  else return c0;
}

// Per-lane constants of a grid: samples held, offsets from the line centre,
// the single stray-light profile (zero without one).
template <int LPL>
__device__ __forceinline__ void grid_lanes(const DevCfg& c, int lane, int& nl, float (&dlv)[LPL],
                                           double (&dld)[LPL], bool (&valid)[LPL], float (&slg)[LPL][4]) {
  nl = c.nl;
#pragma unroll
  for (int k = 0; k < LPL; ++k) {
    const int l = lane + 32 * k;
    valid[k] = l < nl;
    dlv[k] = valid[k] ? c.dl[l] : 0.f;
    dld[k] = valid[k] ? c.dld[l] : 0.0;
  }
  if (c.use_slight && !c.slight_per_pixel) load_pixel<LPL>(c.slight, nl, lane, slg);
  else {
#pragma unroll
    for (int k = 0; k < LPL; ++k)
#pragma unroll
      for (int s = 0; s < 4; ++s) slg[k][s] = 0.f;
  }
}

// Blocks of the wave kernels: warps_per_block warps, or one warp in a ragged
// batch (its PSF taps, shared by a block's warps, follow the warp's grid).
template <int LPL, bool MG>
constexpr int wave_warps() { return MG ? 1 : warps_per_block<LPL>(); }

// One trial of every pixel in the wave's active list (wave 0: the start
// models, every pixel of the chunk).  The body is invert_kernel's loop
// body from the solve to the damping schedule (milosUtils.cu:630-700).
template <int LPL, int V, bool MG>
__global__ void __launch_bounds__(wave_warps<LPL, MG>() * 32,
                                  trial_min_blocks<LPL, V>() * warps_per_block<LPL>() / wave_warps<LPL, MG>())
trial_kernel(const DevCfg c0, const InvertArgs a, const WaveArgs w, int wave, const MultiGrid mg) {
  constexpr int NS = Variant<V>::SOLVES, NT = Variant<V>::NT, NA = NT * (NT + 1) / 2;
  const int lane = threadIdx.x & 31;
  if constexpr (!MG) load_taps<LPL>(c0);
  WarpSmem<LPL, V>& sm = trial_smem<LPL, V>();
  for (int i = lane; i < 8 * row_pitch<LPL>(); i += 32) (&sm.rows[0][0])[i] = 0.f;
  __syncwarp();
  int nl = c0.nl;
  float dlv[LPL];
  double dld[LPL];
  bool valid[LPL];
#pragma unroll
  for (int k = 0; k < LPL; ++k) {
    const int l = lane + 32 * k;
    valid[k] = l < nl;
    dlv[k] = valid[k] ? c0.dl[l] : 0.f;
    dld[k] = valid[k] ? c0.dld[l] : 0.0;
  }
  float slg[LPL][4];
  if (c0.use_slight && !c0.slight_per_pixel) load_pixel<LPL>(c0.slight, nl, lane, slg);
  else {
#pragma unroll
    for (int k = 0; k < LPL; ++k)
#pragma unroll
      for (int s = 0; s < 4; ++s) slg[k][s] = 0.f;
  }
  int cur = -1;   // grid whose constants are loaded (ragged batches)
  const SolvePlan plan = g_solve_plans[NS - 1].lane[lane];
  Solve11Plan plan11;
  if constexpr (NT == 11) plan11 = make_solve11_plan(lane);
  const uint32_t n = wave == 0 ? (uint32_t)a.npix : w.cnt[wave - 1].n_next;
  const uint32_t* in = (wave & 1) ? w.act1 : w.act0;
  uint32_t* next = (wave & 1) ? w.act0 : w.act1;
  unsigned long long my_iter = 0, my_acc = 0;
  while (true) {
    uint32_t j = 0;
    if (lane == 0) j = atomicAdd(&w.cnt[wave].cur_trial, 1u);
    j = __shfl_sync(kFull, j, 0);
    if (j >= n) break;
    const uint32_t pix = wave == 0 ? j : in[j];
    const DevCfg* cp = nullptr;
    if constexpr (MG) {
      const int gi = mg.grid[pix];
      cp = mg.cfgs + gi;
      if (gi != cur) {
        cur = gi;
        load_taps<LPL>(*cp);
        grid_lanes<LPL>(*cp, lane, nl, dlv, dld, valid, slg);
      }
    }
    const DevCfg& c = pixel_cfg<MG>(c0, cp);
    PixLM& P = w.state[pix];
    const size_t off = MG ? (size_t)mg.off[pix] : (size_t)pix * 4 * nl;
    float ob[LPL][4];
    load_pixel<LPL>(a.iquv + off, nl, lane, ob);
    if (c.use_slight && c.slight_per_pixel) load_pixel<LPL>(c.slight + off, nl, lane, slg);
    const double* lamp = pixel_grid<LPL>(c, pix, lane, dlv, dld);

    float flambda, pbf, ochisqr, chisqr0;
    int iter, acc;
    uint32_t st;
    bool solved = false;
    if (wave == 0) {
      if (lane < 11) sm.m[lane] = a.init_models ? a.init_models[(size_t)pix * 11 + lane] : c.init[lane];
      st = a.init_status ? a.init_status[pix] : 0u;
      flambda = c.ilambda;
      pbf = 1.f;
      ochisqr = chisqr0 = 0.f;
      iter = acc = 0;
      __syncwarp();
    } else {
      const bool reuse = NS == 2 && (P.flags & 1u);
      if (lane < 11) {
        sm.m[lane] = P.m[lane];
        sm.t[lane] = P.t[lane];
      }
      flambda = P.flambda;
      pbf = P.pbf;
      ochisqr = P.ochisqr;
      chisqr0 = P.chisqr0;
      iter = P.iter;
      acc = P.acc;
      st = P.st;
      if (reuse) {
        if (lane < 10) sm.vec[1][0][lane] = P.vnext[lane];
      } else {
        for (int i = lane; i < NA; i += 32) sm.alpha[i] = P.alpha[i];
        if (lane < NT) sm.beta[lane] = P.beta[lane];
      }
      __syncwarp();
      if constexpr (NT == 11) {
        if (!solve11_elim<LPL, V>(sm, flambda, lane)) solve11<LPL, V>(sm, plan11, flambda, lane);
        if (lane == 0) apply_delta_check<11>(c, sm.m, sm.dd, sm.t);
      } else {
        if (!reuse) {
          if (c.numerics) solve10<LPL, V, true>(sm, plan, flambda, flambda * 10.f * pbf, lane);
          else solve10<LPL, V, false>(sm, plan, flambda, flambda * 10.f * pbf, lane);
        }
        if (lane == 0) apply_delta_check<10>(c, sm.m, sm.vec[reuse ? 1 : 0][0], sm.t);
      }
      solved = !reuse;
      __syncwarp();
    }
    Lane<LPL, V> ln;
    Angles an;
    float syn[LPL][4], pure[LPL][4];
    synth_lane<LPL, V>(c, wave == 0 ? sm.m : sm.t, dlv, lane, ln, an, syn, pure, slg, sm, lamp);
    const float chisqr = chisq<LPL>(c, syn, ob, valid);
    bool accept = true, stop = false, have_next = false;
    if (wave == 0) {
      ochisqr = chisqr;
      chisqr0 = chisqr;
      if (lane < 11) sm.t[lane] = sm.m[lane];
    } else {
      // stop rules and damping schedule (milosUtils.cu:667-696), as in
      // invert_kernel; written out in both kernels because a shared helper
      // changed this kernel's register allocation (+16 B of spills, -0.5 %)
      if ((double)fabsf(((ochisqr) - (chisqr)) * 100 / (chisqr)) < c.toplim || (chisqr) < 0.0001f) {
        stop = true;
        st |= GM_PIX_CHI2_EXIT;
      }
      accept = (chisqr) - (ochisqr) < 0.f;
      if (accept) {
        flambda = flambda / (5.f * pbf);
        if (c.stop_dchi2 > 0.0 && (double)(ochisqr - chisqr) < c.stop_dchi2) stop = true;
        if (lane < 11) sm.m[lane] = sm.t[lane];
        ++acc;
      } else {
        flambda = flambda * 10.f * pbf;
      }
      if (flambda > 1e+7f || flambda < 1e-25f) {
        stop = true;
        st |= GM_PIX_LAMBDA_EXIT;
      }
      ++iter;
      have_next = NS == 2 && !accept && solved;
      if (c.logclambda) pbf = log10f(chisqr) / log10f(chisqr0);
      if (accept) ochisqr = chisqr;
    }
    __syncwarp();
    if (wave > 0 && (iter >= c.miter || stop)) {
      if (!stop) st |= GM_PIX_MAXITER;
      if (!isfinite(ochisqr)) st |= GM_PIX_NONFINITE;
      finish_pixel<LPL, MG>(a, sm.m, ochisqr, iter, acc, st, syn, pix, nl, lane, mg);
      my_iter += iter;
      my_acc += acc;
    } else {
      if (lane < 11) {
        P.m[lane] = sm.m[lane];
        P.t[lane] = sm.t[lane];
      }
      if (NS == 2 && solved && lane < 10) P.vnext[lane] = sm.vec[NS - 1][0][lane];
      uint32_t slot = 0, aslot = 0;
      if (lane == 0) {
        P.flambda = flambda;
        P.pbf = pbf;
        P.ochisqr = ochisqr;
        P.chisqr0 = chisqr0;
        P.iter = iter;
        P.acc = acc;
        P.st = st;
        P.flags = have_next ? 1u : 0u;
        slot = atomicAdd(&w.cnt[wave].n_next, 1u);
        if (accept) aslot = atomicAdd(&w.cnt[wave].n_acc, 1u);
      }
      slot = __shfl_sync(kFull, slot, 0);
      aslot = __shfl_sync(kFull, aslot, 0);
      if (lane == 0) next[slot] = pix;
      if (accept) {
        stage_put<LPL, V>(w.stage + (size_t)pix * stage_floats<LPL>(), ln, an, syn, pure, lane);
        if (lane == 0) w.accl[aslot] = pix;
      }
    }
    __syncwarp();
  }
  if (lane == 0 && (my_iter | my_acc)) {
    atomicAdd(&a.work->iterations, my_iter);
    atomicAdd(&a.work->accepted, my_acc);
  }
}

// Response functions and normal equations of every pixel whose trial of
// this wave was accepted (the accept branch of invert_kernel's loop).
template <int LPL, int V, bool MG>
__global__ void __launch_bounds__(wave_warps<LPL, MG>() * 32,
                                  accept_min_blocks<LPL, V>() * warps_per_block<LPL>() / wave_warps<LPL, MG>())
accept_kernel(const DevCfg c0, const InvertArgs a, const WaveArgs w, int wave, const MultiGrid mg) {
  const int lane = threadIdx.x & 31;
  WarpSmem<LPL, V>& sm = warp_smem<LPL, V>();
  if constexpr (!MG) {
    load_taps<LPL>(c0);
    init_rows<LPL, V>(c0, sm, lane);
  }
  int nl = c0.nl;
  float dlv[LPL];
  double dld[LPL];
  bool valid[LPL];
#pragma unroll
  for (int k = 0; k < LPL; ++k) {
    valid[k] = lane + 32 * k < nl;
    dlv[k] = 0.f;
    dld[k] = 0.0;
  }
  float slg[LPL][4];
  if (c0.use_slight && !c0.slight_per_pixel) load_pixel<LPL>(c0.slight, nl, lane, slg);
  else {
#pragma unroll
    for (int k = 0; k < LPL; ++k)
#pragma unroll
      for (int s = 0; s < 4; ++s) slg[k][s] = 0.f;
  }
  int cur = -1;   // grid whose constants are loaded (ragged batches)
  const uint32_t n = w.cnt[wave].n_acc;
  const bool alpha_mixed = wave > 0 && c0.quirks;
  while (true) {
    uint32_t j = 0;
    if (lane == 0) j = atomicAdd(&w.cnt[wave].cur_acc, 1u);
    j = __shfl_sync(kFull, j, 0);
    if (j >= n) break;
    const uint32_t pix = w.accl[j];
    const DevCfg* cp = nullptr;
    if constexpr (MG) {
      const int gi = mg.grid[pix];
      cp = mg.cfgs + gi;
      if (gi != cur) {
        cur = gi;
        load_taps<LPL>(*cp);
        init_rows<LPL, V>(*cp, sm, lane);
        grid_lanes<LPL>(*cp, lane, nl, dlv, dld, valid, slg);
      }
    }
    const DevCfg& c = pixel_cfg<MG>(c0, cp);
    PixLM& P = w.state[pix];
    const size_t off = MG ? (size_t)mg.off[pix] : (size_t)pix * 4 * nl;
    float ob[LPL][4];
    load_pixel<LPL>(a.iquv + off, nl, lane, ob);
    if (c.use_slight && c.slight_per_pixel) load_pixel<LPL>(c.slight + off, nl, lane, slg);
    const double* lamp = pixel_grid<LPL>(c, pix, lane, dlv, dld);
    if (lane < 11) sm.m[lane] = P.m[lane];
    Lane<LPL, V> ln;
    Angles an;
    float syn[LPL][4], pure[LPL][4];
    stage_get<LPL, V>(w.stage + (size_t)pix * stage_floats<LPL>(), ln, an, syn, pure, lane);
    __syncwarp();
    rf_rows<LPL, V>(c, sm.m, ln, an, lane, sm, lamp);
    normal_eq<LPL, V>(c, sm.m, alpha_mixed, pure, slg, syn, ob, valid, lane, sm);
    constexpr int NT = Variant<V>::NT;
    for (int i = lane; i < NT * (NT + 1) / 2; i += 32) P.alpha[i] = sm.alpha[i];
    if (lane < NT) P.beta[lane] = sm.beta[lane];
    __syncwarp();
  }
}

// Synthesis (+ response functions) of one model per warp
// (kernel_synthesis, gmilos.cu:71-84, batched).
template <int LPL, int V>
__global__ void __launch_bounds__(warps_per_block<LPL>() * 32)
synth_kernel(const DevCfg c, const SynthArgs a) {
  constexpr int NT = Variant<V>::NT;
  const int WPB = warps_per_block<LPL>();
  const int lane = threadIdx.x & 31;
  load_taps<LPL>(c);
  WarpSmem<LPL, V>& sm = warp_smem<LPL, V>();
  init_rows<LPL, V>(c, sm, lane);
  const int nl = c.nl;
  float dlv[LPL];
  double dld[LPL];
#pragma unroll
  for (int k = 0; k < LPL; ++k) {
    const int l = lane + 32 * k;
    dlv[k] = (l < nl) ? c.dl[l] : 0.f;
    dld[k] = 0.0;
  }
  float slg[LPL][4];
  if (c.use_slight && !c.slight_per_pixel) load_pixel<LPL>(c.slight, nl, lane, slg);
  else {
#pragma unroll
    for (int k = 0; k < LPL; ++k)
#pragma unroll
      for (int s = 0; s < 4; ++s) slg[k][s] = 0.f;
  }
  const int64_t wid = (int64_t)blockIdx.x * WPB + (threadIdx.x >> 5);
  const int64_t nw = (int64_t)gridDim.x * WPB;
  for (int64_t pix = wid; pix < a.npix; pix += nw) {
    const size_t off = (size_t)pix * 4 * nl;
    if (c.use_slight && c.slight_per_pixel) load_pixel<LPL>(c.slight + off, nl, lane, slg);
    if (lane < 11) sm.m[lane] = a.models_f64 ? a.models_f64[pix * 11 + lane] : (double)a.models_f32[pix * 11 + lane];
    __syncwarp();
    const double* lamp = pixel_grid<LPL>(c, (unsigned long long)pix, lane, dlv, dld);
    Lane<LPL, V> ln;
    Angles an;
    float syn[LPL][4], pure[LPL][4];
    synth_lane<LPL, V>(c, sm.m, dlv, lane, ln, an, syn, pure, slg, sm, lamp);
#pragma unroll
    for (int k = 0; k < LPL; ++k) {
      const int l = lane + 32 * k;
      if (l < nl)
#pragma unroll
        for (int s = 0; s < 4; ++s) a.iquv[off + s * nl + l] = syn[k][s];
    }
    if (a.rf) {
      rf_rows<LPL, V>(c, sm.m, ln, an, lane, sm, lamp);
      bool mac_on = false;
      if constexpr (Variant<V>::MAC) mac_on = sm.m[MAC] > 0.0001;
      const size_t roff = (size_t)pix * 4 * NT * nl;
#pragma unroll
      for (int k = 0; k < LPL; ++k) {
        const int l = lane + 32 * k;
        if (l < nl)
#pragma unroll
          for (int s = 0; s < 4; ++s)
#pragma unroll
            for (int t = 0; t < NT; ++t)
              a.rf[roff + ((size_t)s * NT + t) * nl + l] =
                  gather_rf<LPL, V>(c, sm, sm.m[ALFA], pure[k][s], slg[k][s], l, s, t, mac_on);
      }
    }
    __syncwarp();
  }
}

// Classical estimates only, one warp per pixel: the configured guess model
// with B, vlos, gamma, phi from the weak-field / centre-of-gravity estimates.
// FOR_INIT = false: the reference's classical-estimates mode, S0 = B_los
// (gmilos.cu:383-404).  FOR_INIT = true: the start models of an inversion,
// exactly as the inversion kernel forms them in place (milosUtils.cu:616-628),
// with their status bits in `status` -- a pre-pass that keeps this code out
// of the inversion kernel's instruction stream.
template <int LPL, bool FOR_INIT, bool MG>
__global__ void __launch_bounds__(128) classical_kernel(const DevCfg c0, const float* __restrict__ iquv,
                                                        int64_t npix, double* __restrict__ models,
                                                        uint32_t* __restrict__ status, const MultiGrid mg) {
  __shared__ double ms[4][11];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int nl = c0.nl;
  double dld[LPL];
  bool valid[LPL];
#pragma unroll
  for (int k = 0; k < LPL; ++k) {
    const int l = lane + 32 * k;
    valid[k] = l < nl;
    dld[k] = valid[k] ? c0.dld[l] : 0.0;
  }
  const int64_t nw = (int64_t)gridDim.x * 4;
  for (int64_t pix = (int64_t)blockIdx.x * 4 + w; pix < npix; pix += nw) {
    const DevCfg* cp = nullptr;
    if constexpr (MG) {
      cp = mg.cfgs + mg.grid[pix];
      nl = cp->nl;
#pragma unroll
      for (int k = 0; k < LPL; ++k) {
        const int l = lane + 32 * k;
        valid[k] = l < nl;
        dld[k] = valid[k] ? cp->dld[l] : 0.0;
      }
    }
    const DevCfg& c = pixel_cfg<MG>(c0, cp);
    float ob[LPL][4], dlv[LPL];
    load_pixel<LPL>(iquv + (MG ? (size_t)mg.off[pix] : (size_t)pix * 4 * nl), nl, lane, ob);
    pixel_grid<LPL>(c, (unsigned long long)pix, lane, dlv, dld);
    if (lane < 11) ms[w][lane] = c.init[lane];
    __syncwarp();
    const uint32_t st = classical_warp<LPL>(c, ob, dld, valid, lane, ms[w], FOR_INIT);
    __syncwarp();
    if (lane < 11) models[pix * 11 + lane] = ms[w][lane];
    if (FOR_INIT && lane == 0) status[pix] = st;
    __syncwarp();
  }
}

static int classical_blocks(int64_t npix) {
  int64_t blocks = (npix + 3) / 4;
  if (blocks > 148 * 32) blocks = 148 * 32;
  return blocks < 1 ? 1 : (int)blocks;
}

cudaError_t launch_classical(const DevCfg& cfg, const float* iquv, int64_t npix, double* models,
                             uint32_t* status, bool for_init, cudaStream_t s) {
  const int blocks = classical_blocks(npix);
  const bool l1 = cfg.nl <= 32;
  const MultiGrid none{};
  if (for_init) {
    if (l1) classical_kernel<1, true, false><<<blocks, 128, 0, s>>>(cfg, iquv, npix, models, status, none);
    else classical_kernel<2, true, false><<<blocks, 128, 0, s>>>(cfg, iquv, npix, models, status, none);
  } else {
    if (l1) classical_kernel<1, false, false><<<blocks, 128, 0, s>>>(cfg, iquv, npix, models, status, none);
    else classical_kernel<2, false, false><<<blocks, 128, 0, s>>>(cfg, iquv, npix, models, status, none);
  }
  return cudaGetLastError();
}

cudaError_t launch_classical_mg(const DevCfg& cfg, const MultiGrid& mg, const float* iquv, int64_t npix,
                                double* models, uint32_t* status, cudaStream_t s) {
  if (npix <= 0) return cudaSuccess;
  const int blocks = classical_blocks(npix);
  if (cfg.nl <= 32) classical_kernel<1, true, true><<<blocks, 128, 0, s>>>(cfg, iquv, npix, models, status, mg);
  else classical_kernel<2, true, true><<<blocks, 128, 0, s>>>(cfg, iquv, npix, models, status, mg);
  return cudaGetLastError();
}

// Start models of a learned-guess inversion, one warp per pixel: the
// classical start (models, from the pre-pass) and the learned guess
// (learned) are each synthesised with the inversion's forward model (PSF,
// stray light) and the one with the lower chi2 is kept in models; a learned
// win sets GM_PIX_LEARNED_INIT in status.  Ties and non-finite chi2 keep the
// classical start, the reference's own (milosUtils.cu:616-628).
template <int LPL, int V>
__global__ void __launch_bounds__(warps_per_block<LPL>() * 32)
select_init_kernel(const DevCfg c, const float* __restrict__ iquv, int64_t npix, double* models,
                   const double* __restrict__ learned, uint32_t* status) {
  const int WPB = warps_per_block<LPL>();
  const int lane = threadIdx.x & 31;
  load_taps<LPL>(c);
  WarpSmem<LPL, V>& sm = warp_smem<LPL, V>();
  init_rows<LPL, V>(c, sm, lane);
  const int nl = c.nl;
  float dlv[LPL];
  double dld[LPL];
  bool valid[LPL];
#pragma unroll
  for (int k = 0; k < LPL; ++k) {
    const int l = lane + 32 * k;
    valid[k] = l < nl;
    dlv[k] = valid[k] ? c.dl[l] : 0.f;
    dld[k] = 0.0;
  }
  float slg[LPL][4];
  if (c.use_slight && !c.slight_per_pixel) load_pixel<LPL>(c.slight, nl, lane, slg);
  else {
#pragma unroll
    for (int k = 0; k < LPL; ++k)
#pragma unroll
      for (int s = 0; s < 4; ++s) slg[k][s] = 0.f;
  }
  const int64_t wid = (int64_t)blockIdx.x * WPB + (threadIdx.x >> 5);
  const int64_t nw = (int64_t)gridDim.x * WPB;
  for (int64_t pix = wid; pix < npix; pix += nw) {
    const size_t off = (size_t)pix * 4 * nl;
    float ob[LPL][4];
    load_pixel<LPL>(iquv + off, nl, lane, ob);
    if (c.use_slight && c.slight_per_pixel) load_pixel<LPL>(c.slight + off, nl, lane, slg);
    float chi[2];
#pragma unroll 1
    for (int k = 0; k < 2; ++k) {
      if (lane < 11) sm.m[lane] = (k == 0 ? models : learned)[pix * 11 + lane];
      __syncwarp();
      Lane<LPL, V> ln;
      Angles an;
      float syn[LPL][4], pure[LPL][4];
      synth_lane<LPL, V>(c, sm.m, dlv, lane, ln, an, syn, pure, slg, sm);
      chi[k] = chisq<LPL>(c, syn, ob, valid);
      __syncwarp();
    }
    if (isfinite(chi[1]) && (!isfinite(chi[0]) || chi[1] < chi[0])) {
      if (lane < 11) models[pix * 11 + lane] = learned[pix * 11 + lane];
      if (lane == 0) status[pix] |= GM_PIX_LEARNED_INIT;
    }
    __syncwarp();
  }
}

template <int LPL, int V>
cudaError_t launch_select_t(const DevCfg& cfg, const float* iquv, int64_t npix, double* models,
                            const double* learned, uint32_t* status, cudaStream_t s) {
  const size_t bytes = tap_bytes<LPL>() + sizeof(WarpSmem<LPL, V>) * warps_per_block<LPL>();
  cudaError_t e = cudaFuncSetAttribute(select_init_kernel<LPL, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)bytes);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t need = (npix + warps_per_block<LPL>() - 1) / warps_per_block<LPL>();
  const int grid = (int)(need < (int64_t)sms * 16 ? (need < 1 ? 1 : need) : (int64_t)sms * 16);
  select_init_kernel<LPL, V><<<grid, warps_per_block<LPL>() * 32, bytes, s>>>(cfg, iquv, npix, models, learned,
                                                                             status);
  return cudaGetLastError();
}

cudaError_t launch_select_init(const DevCfg& cfg, const float* iquv, int64_t npix, double* models,
                               const double* learned, uint32_t* status, cudaStream_t s) {
  if (npix <= 0) return cudaSuccess;
  const int v = kernel_variant(cfg, false);
  if (cfg.nl <= 32) {
    if (v == 0) return launch_select_t<1, 0>(cfg, iquv, npix, models, learned, status, s);
    if (v == 1) return launch_select_t<1, 1>(cfg, iquv, npix, models, learned, status, s);
    return launch_select_t<1, 2>(cfg, iquv, npix, models, learned, status, s);
  }
  if (v == 0) return launch_select_t<2, 0>(cfg, iquv, npix, models, learned, status, s);
  if (v == 1) return launch_select_t<2, 1>(cfg, iquv, npix, models, learned, status, s);
  return launch_select_t<2, 2>(cfg, iquv, npix, models, learned, status, s);
}

// Pure ME profiles (no PSF, no stray light) on an arbitrary offset grid, one
// thread per (pixel, sample): used to synthesise observations on fine grids.
__global__ void synth_grid_kernel(const DevCfg c, const double* __restrict__ models, int64_t npix,
                                  const double* __restrict__ offs, int ngrid, float* __restrict__ out) {
  const int64_t total = npix * ngrid;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t pix = i / ngrid;
    const int l = (int)(i - pix * ngrid);
    const double* m = models + pix * 11;
    const float CC = (float)(kPi / 180.0);
    float sgm, cgm, sina, cosa;
    __sincosf((float)(m[GM] * (double)CC), &sgm, &cgm);
    __sincosf((float)(2 * m[AZ] * (double)CC), &sina, &cosa);
    const float sinis = sgm * sgm, cosis_2 = __fdividef(1.f + cgm * cgm, 2.f);
    const float ulos = __fdividef((float)(m[VLOS] * c.lambda0), (float)(kVlight * m[DOPP]));
    const float parcial = (float)((c.lambda0 * c.lambda0 / m[DOPP]) * kLarmor);
    const float v0 = __fdividef((float)offs[l], (float)m[DOPP]) - ulos;
    float fi[3] = {0, 0, 0}, shi[3] = {0, 0, 0};
    for (int g = 0; g < 3; ++g) {
      const int n = (g == 0) ? c.n_pi : c.n_sig;
      for (int kk = 0; kk < n; ++kk) {
        float nu, wex;
        if (g == 0) { nu = parcial * c.nup[kk]; wex = c.wep[kk]; }
        else if (g == 1) { nu = parcial * c.nub[kk]; wex = c.web[kk]; }
        else { nu = -(parcial * c.nub[c.n_sig - 1 - kk]); wex = c.wer[kk]; }
        const float v = v0 - (float)((double)nu * m[BFLD]);
        float h, f;
        voigt(m[AA], v, h, f);
        fi[g] += wex * h;
        shi[g] += wex * f * 2.f;
      }
    }
    const float E0_2 = __fdividef((float)(m[ETA0] * (double)c.fo), 2.f);
    const float p1 = fi[1] + fi[2];
    const float p2 = E0_2 * (fi[0] - 0.5f * p1);
    const float p3 = E0_2 * (shi[0] - 0.5f * (shi[1] + shi[2]));
    const float ein = E0_2 * (fi[0] * sinis + p1 * cosis_2);
    const float eq = p2 * sinis * cosa, eu = p2 * sinis * sina, ev = (fi[2] - fi[1]) * (E0_2 * cgm);
    const float rq = p3 * sinis * cosa, ru = p3 * sinis * sina, rv = (shi[2] - shi[1]) * (E0_2 * cgm);
    const float ei = 1.f + ein, ei2 = ei * ei;
    const float gp1 = ei2 - eq * eq - eu * eu - ev * ev + rq * rq + ru * ru + rv * rv;
    const float gp3 = ei2 + rq * rq + ru * ru + rv * rv;
    const float gp2 = eq * rq + eu * ru + ev * rv;
    const float dt = ei2 * gp1 - gp2 * gp2;
    const float dtiaux = (float)((double)__fdividef(1.f, dt) * (-(m[S1] * (double)c.mu)));
    const int64_t o = pix * 4 * ngrid + l;
    out[o] = (float)(m[S0] - (double)(dtiaux * ei * gp3));
    out[o + ngrid] = dtiaux * (ei2 * eq + ei * (ev * ru - eu * rv) + rq * gp2);
    out[o + 2 * ngrid] = dtiaux * (ei2 * eu + ei * (eq * rv - ev * rq) + ru * gp2);
    out[o + 3 * ngrid] = dtiaux * (ei2 * ev + ei * (eu * rq - eq * ru) + rv * gp2);
  }
}

template <typename T>
__global__ void peak_kernel(int iters, T* sink) {
  T a[kPeakChains];
  const T x = (T)1.0000001, y = (T)1e-7;
#pragma unroll
  for (int c = 0; c < kPeakChains; ++c) a[c] = (T)(threadIdx.x + c);
  for (int i = 0; i < iters; ++i)
#pragma unroll
    for (int c = 0; c < kPeakChains; ++c) a[c] = fma(a[c], x, y);
  T s = 0;
#pragma unroll
  for (int c = 0; c < kPeakChains; ++c) s += a[c];
  if (s == (T)-1) sink[(blockIdx.x * blockDim.x + threadIdx.x) & 1023] = s;
}

// Special-function-unit issue bound: kPeakChains independent chains of the
// base-2 exponential (one MUFU operation each, the PTX ex2.approx), each
// mapping (0, 1] into [0.5, 1).
__global__ void mufu_peak_kernel(int iters, float* sink) {
  float a[kPeakChains];
#pragma unroll
  for (int c = 0; c < kPeakChains; ++c) a[c] = 0.5f + 1e-3f * (float)((threadIdx.x + c) & 255);
  for (int i = 0; i < iters; ++i)
#pragma unroll
    for (int c = 0; c < kPeakChains; ++c) {
      const float x = -a[c];
      asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(a[c]) : "f"(x));
    }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < kPeakChains; ++c) s += a[c];
  if (s == -1.f) sink[(blockIdx.x * blockDim.x + threadIdx.x) & 1023] = s;
}

cudaError_t launch_peak(int kind, int blocks, int threads, int iters, void* sink, cudaStream_t s) {
  if (kind == 0) peak_kernel<float><<<blocks, threads, 0, s>>>(iters, (float*)sink);
  else if (kind == 1) peak_kernel<double><<<blocks, threads, 0, s>>>(iters, (double*)sink);
  else mufu_peak_kernel<<<blocks, threads, 0, s>>>(iters, (float*)sink);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- launchers
template <int LPL, int V>
constexpr size_t smem_bytes() { return tap_bytes<LPL>() + sizeof(WarpSmem<LPL, V>) * warps_per_block<LPL>(); }

// The wave kernels' launch bounds assume their blocks per SM; their shared
// memory (plus the 1 KB the SM reserves per block) must fit those too.
constexpr size_t kSmemPerSm = 228 * 1024;
template <int LPL, int V>
constexpr bool wave_blocks_fit() {
  return (tap_bytes<LPL>() + trial_warp_bytes<LPL, V>() * warps_per_block<LPL>() + 1024) *
                 trial_min_blocks<LPL, V>() <= kSmemPerSm &&
         (smem_bytes<LPL, V>() + 1024) * accept_min_blocks<LPL, V>() <= kSmemPerSm;
}
static_assert(wave_blocks_fit<1, 0>() && wave_blocks_fit<1, 1>() && wave_blocks_fit<1, 2>(), "nl <= 32");
static_assert(wave_blocks_fit<2, 0>() && wave_blocks_fit<2, 1>() && wave_blocks_fit<2, 2>(), "nl <= 64");

template <int LPL, int V>
cudaError_t prepare_invert() {
  return cudaFuncSetAttribute(invert_kernel<LPL, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)smem_bytes<LPL, V>());
}

template <int LPL, int V>
InvertGeometry geometry_t() {
  // one pixel per warp
  InvertGeometry g{0, warps_per_block<LPL>() * 32, warps_per_block<LPL>(), V};
  if (prepare_invert<LPL, V>() != cudaSuccess) return g;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&g.blocks_per_sm, invert_kernel<LPL, V>, g.threads,
                                                smem_bytes<LPL, V>());
  return g;
}

int kernel_variant(const DevCfg& cfg, bool per_pixel_init) {
  if (cfg.nterms == 11) return 2;
  return (cfg.init[MAC] > 0.0001 || per_pixel_init) ? 1 : 0;
}

InvertGeometry invert_geometry(const DevCfg& cfg, bool per_pixel_init) {
  const int v = kernel_variant(cfg, per_pixel_init);
  if (cfg.nl <= 32) {
    if (v == 0) return geometry_t<1, 0>();
    if (v == 1) return geometry_t<1, 1>();
    return geometry_t<1, 2>();
  }
  if (v == 0) return geometry_t<2, 0>();
  if (v == 1) return geometry_t<2, 1>();
  return geometry_t<2, 2>();
}

template <int LPL, int V>
cudaError_t launch_invert_t(const DevCfg& cfg, const InvertArgs& a, int grid, cudaStream_t s) {
  cudaError_t e = prepare_invert<LPL, V>();
  if (e != cudaSuccess) return e;
  invert_kernel<LPL, V><<<grid, warps_per_block<LPL>() * 32, smem_bytes<LPL, V>(), s>>>(cfg, a);
  return cudaGetLastError();
}

cudaError_t launch_invert(const DevCfg& cfg, const InvertArgs& a, int grid, cudaStream_t s) {
  const int v = kernel_variant(cfg, a.init_models != nullptr && !a.init_status);
  if (cfg.nl <= 32) {
    if (v == 0) return launch_invert_t<1, 0>(cfg, a, grid, s);
    if (v == 1) return launch_invert_t<1, 1>(cfg, a, grid, s);
    return launch_invert_t<1, 2>(cfg, a, grid, s);
  }
  if (v == 0) return launch_invert_t<2, 0>(cfg, a, grid, s);
  if (v == 1) return launch_invert_t<2, 1>(cfg, a, grid, s);
  return launch_invert_t<2, 2>(cfg, a, grid, s);
}

// ---------------------------------------------- wave-synchronous launcher
size_t wave_buffer_bytes(int nl, int miter, int64_t chunk) {
  const int lpl = nl <= 32 ? 1 : 2;
  const int waves = 1 + (miter > 1 ? miter : 1);
  return (size_t)chunk * (sizeof(PixLM) + sizeof(float) * stage_floats_for(lpl) + 3 * sizeof(uint32_t)) +
         sizeof(WaveCounters) * (size_t)waves + 256;
}

WaveBuffers wave_buffers(void* base, int nl, int miter, int64_t chunk) {
  const int lpl = nl <= 32 ? 1 : 2;
  const int waves = 1 + (miter > 1 ? miter : 1);
  char* p = static_cast<char*>(base);
  WaveBuffers b{};
  b.chunk = chunk;
  b.w.state = reinterpret_cast<PixLM*>(p);
  p += sizeof(PixLM) * (size_t)chunk;
  b.w.stage = reinterpret_cast<float*>(p);
  p += sizeof(float) * stage_floats_for(lpl) * (size_t)chunk;
  b.w.cnt = reinterpret_cast<WaveCounters*>(p);
  p += (sizeof(WaveCounters) * (size_t)waves + 255) & ~(size_t)255;
  b.w.act0 = reinterpret_cast<uint32_t*>(p);
  b.w.act1 = b.w.act0 + chunk;
  b.w.accl = b.w.act1 + chunk;
  return b;
}

bool waves_cover(const DevCfg& cfg, const InvertArgs& a) {
  return cfg.init_mode != 0 && !a.step_delta && !a.step_trial && !a.step_chi2_start && !a.step_chi2_trial;
}

// Shared memory of the wave kernels: the block's taps and its warps' blocks
// (the trial kernel packs its warps at trial_warp_bytes).
template <int LPL, int V, bool MG>
constexpr size_t wave_trial_smem() { return tap_bytes<LPL>() + trial_warp_bytes<LPL, V>() * wave_warps<LPL, MG>(); }
template <int LPL, int V, bool MG>
constexpr size_t wave_accept_smem() { return tap_bytes<LPL>() + sizeof(WarpSmem<LPL, V>) * wave_warps<LPL, MG>(); }

// Attributes of both wave kernels and their resident blocks per SM.
template <int LPL, int V, bool MG>
cudaError_t wave_occupancy(int* bt, int* ba) {
  const size_t tsmem = wave_trial_smem<LPL, V, MG>(), smem = wave_accept_smem<LPL, V, MG>();
  cudaError_t e =
      cudaFuncSetAttribute(trial_kernel<LPL, V, MG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(accept_kernel<LPL, V, MG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int threads = wave_warps<LPL, MG>() * 32;
  *bt = *ba = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(bt, trial_kernel<LPL, V, MG>, threads, tsmem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(ba, accept_kernel<LPL, V, MG>, threads, smem);
  return (*bt < 1 || *ba < 1) ? cudaErrorInvalidConfiguration : cudaSuccess;
}

// The waves of one chunk: a pre-zeroed counter block, then per wave the
// trial kernel over the pixels still iterating and the accept kernel over
// those accepted.
template <int LPL, int V, bool MG>
cudaError_t run_waves(const DevCfg& dc, const InvertArgs& c, const WaveBuffers& b, const MultiGrid& mg, int gt,
                      int ga, cudaStream_t s, int* count) {
  const int waves = 1 + (dc.miter > 1 ? dc.miter : 1);
  const int threads = wave_warps<LPL, MG>() * 32;
  cudaError_t e = cudaMemsetAsync(b.w.cnt, 0, sizeof(WaveCounters) * (size_t)waves, s);
  if (e != cudaSuccess) return e;
  for (int wv = 0; wv < waves; ++wv) {
    trial_kernel<LPL, V, MG><<<gt, threads, wave_trial_smem<LPL, V, MG>(), s>>>(dc, c, b.w, wv, mg);
    ++*count;
    // the last wave's pixels all stop: nothing to accept
    if (wv + 1 < waves) {
      accept_kernel<LPL, V, MG><<<ga, threads, wave_accept_smem<LPL, V, MG>(), s>>>(dc, c, b.w, wv, mg);
      ++*count;
    }
  }
  return cudaGetLastError();
}

template <int LPL, int V>
cudaError_t launch_waves_t(const DevCfg& cfg, const InvertArgs& a, const WaveBuffers& b, cudaStream_t s,
                           int* launches) {
  int dev = 0, sms = 0, bt = 0, ba = 0;
  cudaError_t e = wave_occupancy<LPL, V, false>(&bt, &ba);
  if (e != cudaSuccess) return e;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int count = 0;
  for (int64_t first = 0; first < a.npix; first += b.chunk) {
    const int64_t n = a.npix - first < b.chunk ? a.npix - first : b.chunk;
    const DevCfg dc = offset_cfg(cfg, first);
    const InvertArgs c = offset_args(a, first, n, cfg.nl, cfg.nterms);
    const int64_t need = (n + warps_per_block<LPL>() - 1) / warps_per_block<LPL>();
    const int gt = (int)(need < (int64_t)bt * sms ? need : (int64_t)bt * sms);
    const int ga = (int)(need < (int64_t)ba * sms ? need : (int64_t)ba * sms);
    e = run_waves<LPL, V, false>(dc, c, b, MultiGrid{}, gt, ga, s, &count);
    if (e != cudaSuccess) return e;
  }
  if (launches) *launches = count;
  return cudaSuccess;
}

// Ragged batches: chunks of the batch's pixel list; profiles and fitted
// profiles are addressed through mg.off, so only the per-pixel outputs,
// start models and tables move with the chunk.
template <int LPL, int V>
cudaError_t launch_waves_mg_t(const DevCfg& cfg, const MultiGrid& mg, const InvertArgs& a, const WaveBuffers& b,
                              int cap_t, int cap_a, cudaStream_t s, int* launches) {
  int dev = 0, sms = 0, bt = 0, ba = 0;
  cudaError_t e = wave_occupancy<LPL, V, true>(&bt, &ba);
  if (e != cudaSuccess) return e;
  if (cap_t > 0 && cap_t < bt) bt = cap_t;
  if (cap_a > 0 && cap_a < ba) ba = cap_a;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int count = 0;
  for (int64_t first = 0; first < a.npix; first += b.chunk) {
    const int64_t n = a.npix - first < b.chunk ? a.npix - first : b.chunk;
    InvertArgs c = offset_args(a, first, n, cfg.nl, cfg.nterms);
    c.iquv = a.iquv;
    c.fitted = a.fitted;
    MultiGrid m = mg;
    m.grid = mg.grid + first;
    m.off = mg.off + first;
    const int gt = (int)(n < (int64_t)bt * sms ? n : (int64_t)bt * sms);
    const int ga = (int)(n < (int64_t)ba * sms ? n : (int64_t)ba * sms);
    e = run_waves<LPL, V, true>(cfg, c, b, m, gt, ga, s, &count);
    if (e != cudaSuccess) return e;
  }
  if (launches) *launches = count;
  return cudaSuccess;
}

cudaError_t launch_invert_waves_mg(const DevCfg& cfg, const MultiGrid& mg, const InvertArgs& a,
                                   const WaveBuffers& b, int cap_t, int cap_a, cudaStream_t s, int* launches) {
  if (!waves_cover(cfg, a) || !a.init_status || b.chunk < 1 || b.chunk > 0x7fffffff || cfg.lambda_per_pixel ||
      (cfg.use_slight && cfg.slight_per_pixel))
    return cudaErrorInvalidValue;
  const int v = kernel_variant(cfg, false);
  if (cfg.nl <= 32) {
    if (v == 0) return launch_waves_mg_t<1, 0>(cfg, mg, a, b, cap_t, cap_a, s, launches);
    if (v == 1) return launch_waves_mg_t<1, 1>(cfg, mg, a, b, cap_t, cap_a, s, launches);
    return launch_waves_mg_t<1, 2>(cfg, mg, a, b, cap_t, cap_a, s, launches);
  }
  if (v == 0) return launch_waves_mg_t<2, 0>(cfg, mg, a, b, cap_t, cap_a, s, launches);
  if (v == 1) return launch_waves_mg_t<2, 1>(cfg, mg, a, b, cap_t, cap_a, s, launches);
  return launch_waves_mg_t<2, 2>(cfg, mg, a, b, cap_t, cap_a, s, launches);
}

void waves_mg_occupancy(const DevCfg& cfg, int* bt, int* ba) {
  const int v = kernel_variant(cfg, false);
  cudaError_t e;
  if (cfg.nl <= 32)
    e = v == 0 ? wave_occupancy<1, 0, true>(bt, ba) : v == 1 ? wave_occupancy<1, 1, true>(bt, ba)
                                                             : wave_occupancy<1, 2, true>(bt, ba);
  else
    e = v == 0 ? wave_occupancy<2, 0, true>(bt, ba) : v == 1 ? wave_occupancy<2, 1, true>(bt, ba)
                                                             : wave_occupancy<2, 2, true>(bt, ba);
  if (e != cudaSuccess) *bt = *ba = 0;
}

cudaError_t launch_invert_waves(const DevCfg& cfg, const InvertArgs& a, const WaveBuffers& b, cudaStream_t s,
                                int* launches) {
  if (!waves_cover(cfg, a) || b.chunk < 1 || b.chunk > 0x7fffffff) return cudaErrorInvalidValue;
  const int v = kernel_variant(cfg, a.init_models != nullptr && !a.init_status);
  if (cfg.nl <= 32) {
    if (v == 0) return launch_waves_t<1, 0>(cfg, a, b, s, launches);
    if (v == 1) return launch_waves_t<1, 1>(cfg, a, b, s, launches);
    return launch_waves_t<1, 2>(cfg, a, b, s, launches);
  }
  if (v == 0) return launch_waves_t<2, 0>(cfg, a, b, s, launches);
  if (v == 1) return launch_waves_t<2, 1>(cfg, a, b, s, launches);
  return launch_waves_t<2, 2>(cfg, a, b, s, launches);
}

template <int LPL, int V>
cudaError_t launch_synth_t(const DevCfg& cfg, const SynthArgs& a, int grid, cudaStream_t s) {
  const size_t bytes = tap_bytes<LPL>() + sizeof(WarpSmem<LPL, V>) * warps_per_block<LPL>();
  cudaError_t e = cudaFuncSetAttribute(synth_kernel<LPL, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)bytes);
  if (e != cudaSuccess) return e;
  synth_kernel<LPL, V><<<grid, warps_per_block<LPL>() * 32, bytes, s>>>(cfg, a);
  return cudaGetLastError();
}

cudaError_t launch_synth(const DevCfg& cfg, const SynthArgs& a, cudaStream_t s) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int64_t need = (a.npix + warps_for_nl(cfg.nl) - 1) / warps_for_nl(cfg.nl);
  int grid = (int)(need < (int64_t)sms * 16 ? need : (int64_t)sms * 16);
  if (grid < 1) grid = 1;
  // the synthesis of arbitrary models always takes the macroturbulence-capable code
  const bool v2 = cfg.nterms == 11;
  if (cfg.nl <= 32) return v2 ? launch_synth_t<1, 2>(cfg, a, grid, s) : launch_synth_t<1, 1>(cfg, a, grid, s);
  return v2 ? launch_synth_t<2, 2>(cfg, a, grid, s) : launch_synth_t<2, 1>(cfg, a, grid, s);
}

cudaError_t launch_synth_grid(const DevCfg& cfg, const double* models, int64_t npix,
                              const double* offsets, int ngrid, float* out, cudaStream_t s) {
  const int64_t total = npix * ngrid;
  int64_t blocks = (total + 255) / 256;
  if (blocks > 148 * 64) blocks = 148 * 64;
  if (blocks < 1) blocks = 1;
  synth_grid_kernel<<<(int)blocks, 256, 0, s>>>(cfg, models, npix, offsets, ngrid, out);
  return cudaGetLastError();
}

}  // namespace gm
