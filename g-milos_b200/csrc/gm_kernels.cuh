// gm_kernels.cuh -- the engine's kernels and their host-side launchers.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "gm_device.cuh"

namespace gm {

// warps per block of the inversion and synthesis kernels for a grid of nl samples
inline int warps_for_nl(int nl) { return nl <= 32 ? warps_per_block<1>() : warps_per_block<2>(); }

// Work counters shared by the warps of one persistent launch.
struct WorkCounters {
  unsigned long long next_pixel;   // work-stealing cursor
  unsigned long long iterations;   // sum of LM trials
  unsigned long long accepted;     // sum of accepted steps
  unsigned long long pad;
};

struct InvertArgs {
  const float* iquv;          // [P][4][nl]
  int64_t npix;
  const double* init_models;  // [P][11] or null
  const uint32_t* init_status; // [P] status bits of a classical pre-pass that
                               // made init_models (its v_mac is the configured
                               // one), or null
  float* model;               // [P][11] or null
  double* model_f64;          // [P][11] or null
  float* chi2;                // [P] or null
  int* iters;                 // [P] or null
  int* accepted;              // [P] or null
  float* fitted;              // [P][4][nl] or null
  uint32_t* status;           // [P] or null
  float* step_delta;          // [P][nterms] first-iteration step, or null
  double* step_trial;         // [P][11] first-iteration trial model, or null
  float* step_chi2_start;     // [P] chi2 of the starting model, or null
  float* step_chi2_trial;     // [P] chi2 of the first trial, or null
  WorkCounters* work;         // zeroed before the launch
};

// Wave-synchronous inversion (launch_invert_waves): the LM state of one
// pixel between the trial and the accept kernel of a wave.
struct PixLM {
  double m[11], t[11];         // accepted and trial models
  float alpha[68], beta[12];   // normal equations of the accepted model (packed alpha, 55 or 66)
  float vnext[12];             // step for the damping a rejection moves to (10 terms)
  float flambda, pbf, ochisqr, chisqr0;
  int iter, acc;
  uint32_t st, flags;          // status bits; flags bit 0: vnext holds the next step
};
static_assert(sizeof(PixLM) == 576, "PixLM is one 576-byte record");

// Per wave: the trial kernel's cursor, the pixels it passes to the next wave
// and to the accept kernel, and the accept kernel's cursor.
struct WaveCounters {
  unsigned int cur_trial, n_next, n_acc, cur_acc;
};

// Floats of one pixel's staged trial (accepted trial -> accept kernel): 23
// rows of 32 lanes per sample slot (27 with macroturbulence) and a row of
// angles; every variant's block is sized for the larger.
__host__ __device__ constexpr int stage_rows_per_slot(bool mac) { return mac ? 27 : 23; }
__host__ __device__ constexpr int stage_floats_for(int lpl) { return (stage_rows_per_slot(true) * lpl + 1) * 32; }
template <int LPL>
__host__ __device__ constexpr int stage_floats() { return stage_floats_for(LPL); }

struct WaveArgs {
  PixLM* state;                // [chunk]
  float* stage;                // [chunk][stage_floats]
  uint32_t* act0;              // pixels iterating in even / odd waves
  uint32_t* act1;
  uint32_t* accl;              // pixels accepted in the current wave
  WaveCounters* cnt;           // [waves], zeroed per chunk
};

// Device memory of a wave-synchronous inversion, carved from one buffer.
struct WaveBuffers {
  WaveArgs w;
  int64_t chunk;               // pixels per chunk
};
size_t wave_buffer_bytes(int nl, int miter, int64_t chunk);
WaveBuffers wave_buffers(void* base, int nl, int miter, int64_t chunk);
// Whether the wave path covers a launch: every variant, with start models
// given or configured (no in-kernel classical estimates) and no first-step
// outputs.
bool waves_cover(const DevCfg& cfg, const InvertArgs& a);

// Arguments of the pixels [first, first + n) of a launch.
inline InvertArgs offset_args(const InvertArgs& ia, int64_t first, int64_t n, int nl, int nterms) {
  const size_t row = 4 * (size_t)nl;
  InvertArgs c = ia;
  c.iquv = ia.iquv + first * row;
  c.npix = n;
  if (ia.init_models) c.init_models = ia.init_models + first * 11;
  if (ia.init_status) c.init_status = ia.init_status + first;
  if (ia.model) c.model = ia.model + first * 11;
  if (ia.model_f64) c.model_f64 = ia.model_f64 + first * 11;
  if (ia.chi2) c.chi2 = ia.chi2 + first;
  if (ia.iters) c.iters = ia.iters + first;
  if (ia.accepted) c.accepted = ia.accepted + first;
  if (ia.fitted) c.fitted = ia.fitted + first * row;
  if (ia.status) c.status = ia.status + first;
  if (ia.step_delta) c.step_delta = ia.step_delta + first * nterms;
  if (ia.step_trial) c.step_trial = ia.step_trial + first * 11;
  if (ia.step_chi2_start) c.step_chi2_start = ia.step_chi2_start + first;
  if (ia.step_chi2_trial) c.step_chi2_trial = ia.step_chi2_trial + first;
  return c;
}
inline DevCfg offset_cfg(const DevCfg& d, int64_t first) {
  DevCfg dc = d;
  if (d.use_slight && d.slight_per_pixel) dc.slight = d.slight + first * 4 * (int64_t)d.nl;
  if (d.lambda_per_pixel) dc.lam_map = d.lam_map + first * (int64_t)d.nl;
  return dc;
}

// Ragged batches: pixels of many wavelength grids in one launch.  Pixel p
// runs on configuration cfgs[grid[p]] (its grid, PSF taps and stray profile;
// everything else shared) and its profiles start at iquv + off[p] (floats),
// its fitted profiles (when asked for) at fitted + off[p].  A launch holds
// grids of one samples-per-lane class (all <= 32 or all 33..64 samples).
struct MultiGrid {
  const DevCfg* cfgs;          // device [grids]
  const uint16_t* grid;        // [P] configuration index per pixel
  const uint64_t* off;         // [P] offset of the pixel's [4][nl] block
};

struct SynthArgs {
  const float* models_f32;    // [P][11] (one of the two)
  const double* models_f64;
  int64_t npix;
  float* iquv;                // [P][4][nl]
  float* rf;                  // [P][4][nterms][nl] or null (nterms 10 or 11)
};

// launchers (gm_kernels.cu); return the CUDA error of the launch
cudaError_t launch_invert(const DevCfg& cfg, const InvertArgs& a, int grid, cudaStream_t s);
// The wave-synchronous inversion of a.npix pixels in chunks of b.chunk on
// stream s (waves_cover must hold); *launches receives the kernel count.
cudaError_t launch_invert_waves(const DevCfg& cfg, const InvertArgs& a, const WaveBuffers& b, cudaStream_t s,
                                int* launches);
// The same for a ragged batch (one warp per block, the grid's constants
// reloaded when a warp moves to a pixel of another grid): cfg is any of the
// batch's configurations (they share everything but the grid, taps and stray
// profile); a.init_models / a.init_status come from launch_classical_mg.
// cap: resident blocks per SM of the trial / accept kernels (0: as many as fit).
cudaError_t launch_invert_waves_mg(const DevCfg& cfg, const MultiGrid& mg, const InvertArgs& a,
                                   const WaveBuffers& b, int cap_trial, int cap_accept, cudaStream_t s,
                                   int* launches);
cudaError_t launch_classical_mg(const DevCfg& cfg, const MultiGrid& mg, const float* iquv, int64_t npix,
                                double* models, uint32_t* status, cudaStream_t s);
// resident blocks per SM of the ragged-batch wave kernels (the autotuner's range)
void waves_mg_occupancy(const DevCfg& cfg, int* trial_blocks, int* accept_blocks);
cudaError_t launch_synth(const DevCfg& cfg, const SynthArgs& a, cudaStream_t s);
// classical estimates: for_init false -> the classical-estimates mode
// (S0 = B_los); true -> start models of an inversion plus status bits
cudaError_t launch_classical(const DevCfg& cfg, const float* iquv, int64_t npix, double* models,
                             uint32_t* status, bool for_init, cudaStream_t s);
cudaError_t launch_synth_grid(const DevCfg& cfg, const double* models, int64_t npix,
                              const double* offsets, int ngrid, float* out, cudaStream_t s);
// learned-guess inversions: per pixel the start model with the lower chi2 of
// models (classical, in/out) and learned; GM_PIX_LEARNED_INIT in status when
// the learned one is kept
cudaError_t launch_select_init(const DevCfg& cfg, const float* iquv, int64_t npix, double* models,
                               const double* learned, uint32_t* status, cudaStream_t s);
// kernel variant for a configuration (0: 10 terms, 1: 10 terms with
// macroturbulence, 2: 11 terms); per_pixel_init: start models given per pixel
int kernel_variant(const DevCfg& cfg, bool per_pixel_init);
// launch geometry of the inversion kernel for a configuration
struct InvertGeometry {
  int blocks_per_sm;      // resident blocks per SM (0: the kernel cannot be resident)
  int threads;            // threads per block
  int pixels_per_block;   // pixels in flight per block
  int variant;
};
InvertGeometry invert_geometry(const DevCfg& cfg, bool per_pixel_init);

// Issue-bound microbenchmarks (kind 0: FP32 FMA, 1: FP64 FMA, 2: MUFU
// exponential); each thread runs kPeakChains independent chains of `iters`
// steps.
constexpr int kPeakChains = 8;
cudaError_t launch_peak(int kind, int blocks, int threads, int iters, void* sink, cudaStream_t s);

}  // namespace gm
