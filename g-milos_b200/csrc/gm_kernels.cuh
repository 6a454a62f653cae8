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

struct SynthArgs {
  const float* models_f32;    // [P][11] (one of the two)
  const double* models_f64;
  int64_t npix;
  float* iquv;                // [P][4][nl]
  float* rf;                  // [P][4][nterms][nl] or null (nterms 10 or 11)
};

// launchers (gm_kernels.cu); return the CUDA error of the launch
cudaError_t launch_invert(const DevCfg& cfg, const InvertArgs& a, int grid, cudaStream_t s);
cudaError_t launch_synth(const DevCfg& cfg, const SynthArgs& a, cudaStream_t s);
// classical estimates: for_init false -> the classical-estimates mode
// (S0 = B_los); true -> start models of an inversion plus status bits
cudaError_t launch_classical(const DevCfg& cfg, const float* iquv, int64_t npix, double* models,
                             uint32_t* status, bool for_init, cudaStream_t s);
cudaError_t launch_synth_grid(const DevCfg& cfg, const double* models, int64_t npix,
                              const double* offsets, int ngrid, float* out, cudaStream_t s);
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
