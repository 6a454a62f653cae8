// gm_mlp.cuh -- the learned initial guess: a 4 nl -> 256 -> 256 -> 9 GELU
// network evaluated and trained on the tensor cores (tcgen05.mma, BF16
// operands staged by TMA in 128-byte-swizzled shared memory, FP32
// accumulators in tensor memory).  Host-side interface of gm_mlp.cu.
#pragma once

#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

#include "gmilos.h"

namespace gm {
namespace mlp {

constexpr int kIn = GM_MLP_IN;          // padded input features (K of layer 1)
constexpr int kHid = GM_MLP_HIDDEN;     // hidden width (N of layers 1-2, K of 2-3)
constexpr int kOut = GM_MLP_OUT;        // outputs
constexpr int kOut16 = GM_MLP_OUT_PAD;  // N of layer 3
constexpr int kG = 64;                  // K of the output-gradient product (9 padded)
constexpr int kTile = 128;              // pixels per tile (M of every product)

// A network on the device: its FP32 parameters (a gm_mlp), the BF16
// operand copies of its weights, and the TMA descriptors of those copies.
struct DevNet {
  gm_mlp* p = nullptr;        // device copy of the parameters
  uint16_t* pack = nullptr;   // BF16 operands (w1b, w2b, w3b, w2tb, w3tb)
  CUtensorMap mw1{}, mw2{}, mw3{}, mw2t{}, mw3t{};
  int nl = 0;
};

// Offsets (elements) of the BF16 operand copies inside DevNet::pack.
constexpr size_t kW1b = 0;                                  // [256][128]
constexpr size_t kW2b = kW1b + (size_t)kHid * kIn;          // [256][256]
constexpr size_t kW3b = kW2b + (size_t)kHid * kHid;         // [16][256]  (rows >= 9 zero)
constexpr size_t kW2tb = kW3b + (size_t)kOut16 * kHid;      // [256][256] transposed w2
constexpr size_t kW3tb = kW2tb + (size_t)kHid * kHid;       // [256][64]  transposed w3 (cols >= 9 zero)
constexpr size_t kPackElems = kW3tb + (size_t)kHid * kG;

// Set up / release a device network from host parameters (copy, BF16 pack,
// descriptors); stream-ordered.
cudaError_t devnet_create(DevNet* d, const gm_mlp* host, cudaStream_t s);
void devnet_destroy(DevNet* d);

// Start models [n][11] for the profiles iquv [n][4][nl] (device memory):
// free parameters (fix[i] != 0, i < 9) from the network, the others and
// v_mac / the filling factor from guess.  err: a device word, zero before
// the call, that a kernel which gave up waiting sets non-zero.
cudaError_t predict(const DevNet& d, const float* iquv, int64_t n, int nl, const double* guess, const int* fix,
                    double* models, int* err, cudaStream_t s);

// Training on device-resident data; net (host) in/out.  loss (optional):
// per-epoch mean loss.  grads_only: one batch of n pixels, no update; its
// gradients into *grads (host) and its loss into loss[0].  err as for
// predict; why (optional) receives a reason on failure.
struct TrainArgs {
  const float* iquv;      // [n][4][nl] device
  const double* truth;    // [n][11] device
  int64_t n;
  int nl;
  int epochs, batch;
  float lr, weight_decay;
  uint64_t seed;
  bool grads_only;
};
cudaError_t train(gm_mlp* net, const TrainArgs& a, float* loss, gm_mlp* grads, int* err, cudaStream_t s,
                  const char** why);

// Host helpers (no device): the 9 standardised-output targets of a model,
// and a fresh network.
void targets_of(const double* m, float* y9);
void init_net(gm_mlp* net, int nl, uint64_t seed);

}  // namespace mlp
}  // namespace gm
