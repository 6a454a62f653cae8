// gm_capi.cu -- the C ABI (include/gmilos.h): contexts, configuration,
// host/device buffer handling and kernel launches.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "gm_kernels.cuh"
#include "gm_mlp.cuh"
#include "gmilos.h"

namespace {

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

using Clock = std::chrono::steady_clock;

// One inversion request of the serving path: its configuration snapshot, its
// device buffers (the caller's when it passed device memory), and how far its
// chunks have been launched and completed.
struct Request {
  gm_request req;
  gm::DevCfg dev{};
  gm_status result = GM_OK;
  bool done = false;
  bool cancelled = false;
  bool admitted = false;
  // device views: input cube and outputs (owned when the caller's are host memory)
  float* d_in = nullptr;
  float* d_model = nullptr;
  float* d_chi2 = nullptr;
  int* d_iters = nullptr;
  uint32_t* d_status = nullptr;
  std::vector<void*> owned;
  size_t bytes = 0;          // device memory charged to the HBM budget
  int64_t next = 0;          // first pixel not yet launched
  int outstanding = 0;       // launched chunks not yet complete
  Clock::time_point t_submit, t_start;
  bool started = false;
};

// A serving lane: a stream with its own work counters and one chunk in flight.
struct ServeLane {
  cudaStream_t stream = nullptr;
  gm::WorkCounters* work = nullptr;
  cudaEvent_t done = nullptr;
  // one chunk's wave-kernel state, then its classical start models and
  // status bits (null: the fused kernel serves this lane)
  void* scratch = nullptr;
  size_t wave_bytes = 0;
  int nl = 0, miter = 0;
  int64_t chunk = 0;
  std::shared_ptr<Request> req;
  bool busy = false;
};

}  // namespace

struct gm_ctx {
  int device = 0;
  size_t budget = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int sms = 0;
  bool configured = false;
  gm_config cfg{};
  gm::DevCfg dev{};
  gm::WorkCounters* work = nullptr;   // device scratch of the persistent launch
  // pipelined host-memory inversions: a second stream and its work counters
  cudaStream_t aux = nullptr;
  cudaEvent_t evx0 = nullptr, evx1 = nullptr;
  gm::WorkCounters* work2 = nullptr;
  // the device scratch (work counters, pre-pass output, wave state) is
  // reused by every inversion: the next one, on whatever stream, waits for
  // the last one's work
  cudaEvent_t ev_scratch = nullptr;
  bool scratch_pending = false;
  DevBuf slight;                      // global stray-light profile (device copy)
  std::map<std::string, DevBuf> bufs; // staging buffers for host-memory calls
  std::string err;
  gm_stats stats{};
  // serving: continuous batching over `serve_streams` lanes
  std::mutex mu;
  std::condition_variable cv, done_cv;
  std::deque<gm_ticket> queue;        // submitted, not yet admitted
  std::map<gm_ticket, std::shared_ptr<Request>> reqs;
  std::vector<std::shared_ptr<Request>> active;   // admitted, chunks pending or in flight
  std::vector<ServeLane> lanes;
  size_t serve_bytes = 0;             // device memory held by admitted requests
  int serve_streams = 4;
  int64_t serve_chunk = 65536;        // pixels per launch
  int serve_max_active = 16;
  int serve_policy = GM_SERVE_RESPONSE_RATIO;   // which admitted request a free lane takes
  size_t rr = 0;                      // round-robin cursor over active requests
  gm_ticket next_ticket = 1;
  std::thread worker;
  bool stopping = false;
  std::mutex call_mu;                 // serialises the synchronous entry points
  // learned initial guess (GM_INIT_LEARNED): the configured network on the
  // device, and the error word its kernels set when a wait gives up
  gm::mlp::DevNet net;
  bool learned = false;
  int* mlp_err = nullptr;
  // ragged batches: the layout of the last batch, its captured device work
  // and its resident-block limits per samples-per-lane class
  std::string batch_key;
  cudaGraphExec_t batch_exec = nullptr;
  int batch_cap[2][2] = {{0, 0}, {0, 0}};
  bool batch_tuned = false;
};

namespace {

gm_status fail(gm_ctx* ctx, gm_status s, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return s;
}

gm_status cuda_fail(gm_ctx* ctx, cudaError_t e, const char* what) {
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  return fail(ctx, GM_ERR_CUDA, m);
}

bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes at{};
  cudaError_t e = cudaPointerGetAttributes(&at, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

gm_status ensure_buf(gm_ctx* ctx, const std::string& name, size_t bytes, void** out) {
  DevBuf& b = ctx->bufs[name];
  if (b.bytes < bytes) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
    cudaError_t e = cudaMalloc(&b.p, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(ctx, GM_ERR_NOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed");
    }
    b.bytes = bytes;
  }
  *out = b.p;
  return GM_OK;
}

// A host- or device-side argument staged onto the device.
struct Arg {
  void* dev = nullptr;      // pointer the kernel uses
  void* host = nullptr;     // user host pointer to copy back to (outputs)
  size_t bytes = 0;
};

gm_status stage_in(gm_ctx* ctx, const char* name, const void* p, size_t bytes, Arg* a,
                   cudaStream_t s) {
  a->bytes = bytes;
  if (!p) return GM_OK;
  if (is_device_ptr(p)) {
    a->dev = const_cast<void*>(p);
    return GM_OK;
  }
  gm_status st = ensure_buf(ctx, name, bytes, &a->dev);
  if (st != GM_OK) return st;
  cudaError_t e = cudaMemcpyAsync(a->dev, p, bytes, cudaMemcpyHostToDevice, s);
  return e == cudaSuccess ? GM_OK : cuda_fail(ctx, e, "host-to-device copy");
}

gm_status stage_out(gm_ctx* ctx, const char* name, void* p, size_t bytes, Arg* a) {
  a->bytes = bytes;
  if (!p) return GM_OK;
  if (is_device_ptr(p)) {
    a->dev = p;
    return GM_OK;
  }
  a->host = p;
  return ensure_buf(ctx, name, bytes, &a->dev);
}

gm_status copy_back(gm_ctx* ctx, const Arg& a, cudaStream_t s) {
  if (!a.host || !a.dev) return GM_OK;
  cudaError_t e = cudaMemcpyAsync(a.host, a.dev, a.bytes, cudaMemcpyDeviceToHost, s);
  return e == cudaSuccess ? GM_OK : cuda_fail(ctx, e, "device-to-host copy");
}

gm_status build_devcfg(gm_ctx* ctx, const gm_config& c, gm::DevCfg* d) {
  if (c.abi_version != GM_ABI_VERSION) return fail(ctx, GM_ERR_INVALID, "gm_config.abi_version mismatch");
  if (c.nl < 2 || c.nl > GM_MAX_NL) return fail(ctx, GM_ERR_INVALID, "nl must be in [2, 64]");
  const gm_zeeman& z = c.zeeman;
  if (z.n_pi < 1 || z.n_pi > 10 || z.n_sig < 1 || z.n_sig > 10)
    return fail(ctx, GM_ERR_INVALID, "Zeeman pattern needs 1..10 pi and sigma components");
  if (c.noise <= 0.f) return fail(ctx, GM_ERR_INVALID, "noise must be > 0");
  std::memset(d, 0, sizeof(*d));
  d->nl = c.nl;
  // the reference switches to its 11-term kernel when v_mac and alpha are
  // both free (gmilos.cu:1016-1021)
  d->nterms = (c.fix[9] && c.fix[10]) ? 11 : 10;
  d->use_psf = c.use_psf ? 1 : 0;
  d->use_slight = c.use_slight ? 1 : 0;
  d->slight_per_pixel = c.slight_per_pixel ? 1 : 0;
  d->lambda_per_pixel = c.lambda_per_pixel ? 1 : 0;
  d->lam_map = nullptr;   // bound per call
  if (c.init_mode < GM_INIT_CLASSICAL || c.init_mode > GM_INIT_LEARNED)
    return fail(ctx, GM_ERR_INVALID, "unknown init_mode");
  // the learned guess competes with the classical start: both need the pre-pass
  d->init_mode = (c.init_mode == GM_INIT_CLASSICAL || c.init_mode == GM_INIT_LEARNED) ? 0 : 1;
  d->miter = c.miter;
  d->logclambda = c.logclambda;
  d->quirks = c.reference_quirks;
  if (c.numerics != GM_NUMERICS_REFERENCE && c.numerics != GM_NUMERICS_ACCURATE)
    return fail(ctx, GM_ERR_INVALID, "numerics must be GM_NUMERICS_REFERENCE or GM_NUMERICS_ACCURATE");
  if (c.kernel != GM_KERNEL_AUTO && c.kernel != GM_KERNEL_FUSED && c.kernel != GM_KERNEL_WAVES)
    return fail(ctx, GM_ERR_INVALID, "kernel must be GM_KERNEL_AUTO, GM_KERNEL_FUSED or GM_KERNEL_WAVES");
  d->numerics = c.numerics;
  d->n_pi = z.n_pi;
  d->n_sig = z.n_sig;
  for (int i = 0; i < GM_NPAR; ++i) d->fix[i] = c.fix[i] ? 1 : 0;
  for (int l = 0; l < c.nl; ++l) {
    const double off = c.lambda[l] - c.lambda0;
    d->dl[l] = (float)off;
    d->dld[l] = off;
    d->psfd[l] = c.psf[l];
    d->lam[l] = c.lambda[l];
  }
  for (int i = 0; i < 10; ++i) {
    d->nup[i] = z.nup[i];
    d->nub[i] = z.nub[i];
    d->wep[i] = z.wep[i];
    d->web[i] = z.web[i];
    d->wer[i] = z.wer[i];
  }
  d->geff = z.geff;
  d->fo = z.fo;
  d->mu = c.mu;
  d->ilambda = c.ilambda;
  d->noise = c.noise;
  for (int s = 0; s < 4; ++s) {
    d->weight[s] = c.weight[s];
    d->wsig[s] = c.weight[s] / c.noise;
  }
  d->lambda0 = c.lambda0;
  d->toplim = c.toplim;
  d->stop_dchi2 = c.stop_dchi2;
  for (int i = 0; i < GM_NPAR; ++i) d->init[i] = c.init_model[i];
  return GM_OK;
}

// Blocks of a persistent inversion launch: every resident slot of every SM,
// but no more blocks than the pixels need.
int64_t invert_grid(const gm::DevCfg& d, bool per_pixel_init, int sms, int64_t npix,
                    gm::InvertGeometry* out) {
  const gm::InvertGeometry g = gm::invert_geometry(d, per_pixel_init);
  if (out) *out = g;
  int64_t grid = (int64_t)std::max(1, g.blocks_per_sm) * sms;
  const int64_t needed = (npix + g.pixels_per_block - 1) / g.pixels_per_block;
  if (grid > needed) grid = needed;
  return grid < 1 ? 1 : grid;
}

void serve_loop(gm_ctx* ctx);

}  // namespace

extern "C" {

const char* gm_status_string(gm_status s) {
  switch (s) {
    case GM_OK: return "ok";
    case GM_ERR_INVALID: return "invalid argument";
    case GM_ERR_CUDA: return "CUDA error";
    case GM_ERR_NOMEM: return "out of memory / over budget";
    case GM_ERR_NOT_CONFIGURED: return "context not configured";
    case GM_ERR_UNSUPPORTED: return "unsupported";
    case GM_ERR_TIMEOUT: return "timeout";
    case GM_ERR_CANCELLED: return "cancelled";
    case GM_ERR_IO: return "I/O error";
  }
  return "unknown";
}

const char* gm_last_error(gm_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

// Defaults of loadInitialValues (readConfig.c:704-744): unit weights,
// noise 1e-6, lambda_LM 0.1, toplim 1e-12, mu 1.
void gm_config_defaults(gm_config* c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->abi_version = GM_ABI_VERSION;
  for (int s = 0; s < 4; ++s) c->weight[s] = 1.f;
  c->noise = 1e-6f;
  c->mu = 1.f;
  c->ilambda = 0.1f;
  c->toplim = 1e-12;
  c->miter = 50;
  c->init_mode = GM_INIT_CLASSICAL;
  c->reference_quirks = 1;
  // the values of the reference's run/guess.mod (eta_0 40, B 1000 G, ...)
  const double guess[GM_NPAR] = {40.0, 1000.0, 0.2, 0.03, 0.05, 150.0, 110.0, 0.35, 0.5, 0.0, 1.0};
  for (int i = 0; i < GM_NPAR; ++i) c->init_model[i] = guess[i];
}

gm_status gm_create(int device, size_t hbm_budget, gm_ctx** out) {
  if (!out) return GM_ERR_INVALID;
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    return GM_ERR_CUDA;
  }
  if (device < 0 || device >= n) return GM_ERR_INVALID;
  std::unique_ptr<gm_ctx> ctx(new gm_ctx());
  ctx->device = device;
  if ((e = cudaSetDevice(device)) != cudaSuccess) return GM_ERR_CUDA;
  cudaDeviceProp prop{};
  cudaGetDeviceProperties(&prop, device);
  ctx->sms = prop.multiProcessorCount;
  ctx->budget = hbm_budget ? hbm_budget : (size_t)prop.totalGlobalMem;
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) return GM_ERR_CUDA;
  cudaEventCreate(&ctx->ev0);
  cudaEventCreate(&ctx->ev1);
  if (cudaMalloc(&ctx->work, sizeof(gm::WorkCounters)) != cudaSuccess) return GM_ERR_NOMEM;
  if (cudaMalloc(&ctx->work2, sizeof(gm::WorkCounters)) != cudaSuccess) return GM_ERR_NOMEM;
  if (cudaMalloc(&ctx->mlp_err, sizeof(int) * 4) != cudaSuccess) return GM_ERR_NOMEM;
  cudaMemset(ctx->mlp_err, 0, sizeof(int) * 4);
  if (cudaStreamCreateWithFlags(&ctx->aux, cudaStreamNonBlocking) != cudaSuccess) return GM_ERR_CUDA;
  cudaEventCreateWithFlags(&ctx->evx0, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&ctx->evx1, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&ctx->ev_scratch, cudaEventDisableTiming);
  *out = ctx.release();
  return GM_OK;
}

gm_status gm_destroy(gm_ctx* ctx) {
  if (!ctx) return GM_ERR_INVALID;
  {
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->stopping = true;
  }
  ctx->cv.notify_all();
  if (ctx->worker.joinable()) ctx->worker.join();
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (auto& kv : ctx->bufs)
    if (kv.second.p) cudaFree(kv.second.p);
  if (ctx->slight.p) cudaFree(ctx->slight.p);
  if (ctx->aux) cudaStreamSynchronize(ctx->aux);
  if (ctx->work) cudaFree(ctx->work);
  if (ctx->work2) cudaFree(ctx->work2);
  gm::mlp::devnet_destroy(&ctx->net);
  if (ctx->mlp_err) cudaFree(ctx->mlp_err);
  if (ctx->batch_exec) cudaGraphExecDestroy(ctx->batch_exec);
  cudaEventDestroy(ctx->ev0);
  cudaEventDestroy(ctx->ev1);
  if (ctx->evx0) cudaEventDestroy(ctx->evx0);
  if (ctx->evx1) cudaEventDestroy(ctx->evx1);
  if (ctx->ev_scratch) cudaEventDestroy(ctx->ev_scratch);
  if (ctx->aux) cudaStreamDestroy(ctx->aux);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
  return GM_OK;
}

gm_status gm_configure(gm_ctx* ctx, const gm_config* cfg) {
  if (!ctx || !cfg) return GM_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->call_mu);
  cudaSetDevice(ctx->device);
  gm::DevCfg d;
  gm_status st = build_devcfg(ctx, *cfg, &d);
  if (st != GM_OK) return st;
  if (cfg->use_slight && !cfg->slight_per_pixel) {
    if (!cfg->slight) return fail(ctx, GM_ERR_INVALID, "use_slight set but slight is NULL");
    const size_t bytes = sizeof(float) * 4 * cfg->nl;
    if (ctx->slight.bytes < bytes) {
      if (ctx->slight.p) cudaFree(ctx->slight.p);
      ctx->slight.p = nullptr;
      if (cudaMalloc(&ctx->slight.p, bytes) != cudaSuccess) return fail(ctx, GM_ERR_NOMEM, "stray-light buffer");
      ctx->slight.bytes = bytes;
    }
    cudaError_t e = cudaMemcpy(ctx->slight.p, cfg->slight, bytes,
                               is_device_ptr(cfg->slight) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "stray-light upload");
    d.slight = (const float*)ctx->slight.p;
  }
  if (cfg->init_mode == GM_INIT_LEARNED) {
    const gm_mlp* net = cfg->mlp;
    if (!net) return fail(ctx, GM_ERR_INVALID, "GM_INIT_LEARNED needs gm_config.mlp");
    if (net->abi_version != GM_ABI_VERSION) return fail(ctx, GM_ERR_INVALID, "gm_mlp.abi_version mismatch");
    if (net->nl != cfg->nl || 4 * cfg->nl > GM_MLP_IN)
      return fail(ctx, GM_ERR_INVALID, "the network was made for another grid (its nl differs, or nl > 32)");
    if (cfg->lambda_per_pixel)
      return fail(ctx, GM_ERR_UNSUPPORTED, "the learned guess reads one grid, not per-pixel grids");
    cudaError_t e = gm::mlp::devnet_create(&ctx->net, net, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "learned initial guess upload");
    ctx->learned = true;
  } else {
    gm::mlp::devnet_destroy(&ctx->net);
    ctx->learned = false;
  }
  ctx->cfg = *cfg;
  ctx->cfg.mlp = nullptr;                                  // the network now lives on the device
  if (!cfg->slight_per_pixel) ctx->cfg.slight = nullptr;   // the global profile now lives on the device
  ctx->dev = d;
  ctx->configured = true;
  return GM_OK;
}

struct StepOut {
  float* delta = nullptr;
  double* trial = nullptr;
  float* chi2_start = nullptr;
  float* chi2_trial = nullptr;
};

// Smallest pipelined host-memory inversion: two chunks of kPipeChunk pixels.
constexpr int64_t kPipeChunk = 131072;
// Pixels per chunk of the wave-synchronous inversion (its LM state and
// staging take about 4.2 KB per pixel at nl <= 32, 7.6 KB above,
// gm_wave_state_bytes): large chunks make each wave's launches long against
// their tails.  Below
// kWaveMinChunk pixels within the budget the fused kernel runs instead.
constexpr int64_t kWaveChunk = 1 << 20;
constexpr int64_t kWaveMinChunk = 16384;

// Calls (or served requests) of fewer pixels than this run the fused
// persistent kernel under GM_KERNEL_AUTO: there the wave kernels' ~100 short
// launches cost more than their split saves (measured on B200 at 30
// samples: 4096 pixels with a PSF invert 1.4x faster fused, without one
// 1.9x; the two are even at 16384 pixels with a PSF and at ~32768 without).
static int64_t fused_below(const gm::DevCfg& d) { return d.use_psf ? 16384 : 32768; }

// Which kernels invert a call of npix pixels: the wave-synchronous kernels
// where they cover the configuration, unless the configuration selects the
// single persistent kernel (GM_KERNEL_FUSED: the two agree to rounding; the
// choice serves comparisons and the bit-for-bit tests against
// gm_invert_noalloc) or, under GM_KERNEL_AUTO, the call is small.  A served
// request decides by its whole size, as the lone gm_invert of it does.
static bool want_waves(const gm_ctx* ctx, const gm::DevCfg& d, const gm::InvertArgs& ia, int64_t npix) {
  if (ctx->cfg.kernel == GM_KERNEL_FUSED) return false;
  if (ctx->cfg.kernel == GM_KERNEL_AUTO && npix < fused_below(d)) return false;
  return gm::waves_cover(d, ia);
}

// Pixels per wave chunk for a call of npix pixels that already needs `need`
// bytes of the budget, with `sets` chunks in flight; 0: the fused kernel.
static int64_t wave_chunk_for(const gm_ctx* ctx, const gm::DevCfg& d, size_t need, int64_t npix, int sets) {
  int64_t ch = std::min<int64_t>(npix, kWaveChunk);
  while (ch > 0 && need + sets * gm::wave_buffer_bytes(d.nl, d.miter, ch) > ctx->budget) ch /= 2;
  return ch > 0 && ch >= std::min<int64_t>(npix, kWaveMinChunk) ? ch : 0;
}

static gm_status wave_buffers(gm_ctx* ctx, const char* name, const gm::DevCfg& d, int64_t chunk,
                              gm::WaveBuffers* out) {
  void* p = nullptr;
  gm_status st = ensure_buf(ctx, name, gm::wave_buffer_bytes(d.nl, d.miter, chunk), &p);
  if (st == GM_OK) *out = gm::wave_buffers(p, d.nl, d.miter, chunk);
  return st;
}

// The chunked inversion of a host-memory cube: chunk k is copied up,
// inverted and its outputs copied back on stream k % 2 (the caller's stream
// or ctx->aux), with per-stream work counters whose cursor is reset per
// chunk; iteration sums accumulate over the chunks.  The auxiliary stream
// starts after the caller's prior work and the caller's stream waits for it
// at the end, so the call stays ordered on the caller's stream.  outs[0..n)
// are the per-pixel outputs (per-pixel size = bytes / npix).
// Start models of a learned-guess inversion (after the classical pre-pass
// wrote `models` and `status`): the network's guesses into `scratch`, then
// per pixel the one with the lower chi2.
static cudaError_t learned_starts(gm_ctx* ctx, const gm::DevCfg& d, const float* iquv, int64_t n, double* models,
                                  double* scratch, uint32_t* status, cudaStream_t s) {
  int fix[GM_NPAR];
  for (int i = 0; i < GM_NPAR; ++i) fix[i] = d.fix[i];
  cudaError_t e = gm::mlp::predict(ctx->net, iquv, n, d.nl, ctx->cfg.init_model, fix, scratch, ctx->mlp_err, s);
  if (e == cudaSuccess) e = gm::launch_select_init(d, iquv, n, models, scratch, status, s);
  return e;
}

// After a synchronised call that ran the learned guess: did one of its
// kernels give up waiting?
static gm_status learned_check(gm_ctx* ctx) {
  int code = 0;
  if (cudaMemcpy(&code, ctx->mlp_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess || code != 0) {
    cudaMemset(ctx->mlp_err, 0, sizeof(int));
    return fail(ctx, GM_ERR_CUDA, "a learned-guess kernel gave up waiting for its tensor-core work");
  }
  return GM_OK;
}

static gm_status invert_chunks(gm_ctx* ctx, const gm::DevCfg& d, const gm::InvertArgs& ia,
                               const float* iquv, const Arg& a_in, const Arg* const* outs, int nouts,
                               int64_t npix, int nl, bool prepass, double* learned, size_t need, cudaStream_t s) {
  const size_t row = 4 * (size_t)nl;
  // a short first chunk (kPipeChunk pixels), so that the device starts
  // while the rest of the cube is still arriving, then one to seven equal
  // chunks of up to about four times kPipeChunk (the wave kernels prefer
  // long launches).  Below four times kPipeChunk, two equal halves.
  const int64_t first = npix >= 4 * kPipeChunk ? kPipeChunk : npix / 2;
  const int rest =
      (int)std::max<int64_t>(1, std::min<int64_t>(7, (npix - first + 4 * kPipeChunk - 1) / (4 * kPipeChunk)));
  const int nch = rest + 1;
  auto cut = [&](int k) { return k == 0 ? (int64_t)0 : first + (npix - first) * (k - 1) / rest; };
  gm::DevCfg d1 = d;
  if (prepass) d1.init_mode = 1;
  const int64_t most = std::max<int64_t>(first, (npix - first + rest - 1) / rest);
  // one wave chunk per pipeline chunk and stream
  const bool waves = want_waves(ctx, d1, ia, npix) && wave_chunk_for(ctx, d1, need, most, 2) == most;
  gm::WaveBuffers wb[2];
  if (waves) {
    gm_status st = wave_buffers(ctx, "waves0", d1, most, &wb[0]);
    if (st == GM_OK) st = wave_buffers(ctx, "waves1", d1, most, &wb[1]);
    if (st != GM_OK) return st;
  }
  int launches = 0;
  cudaError_t e = cudaMemsetAsync(ctx->work, 0, sizeof(gm::WorkCounters), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(ctx->work2, 0, sizeof(gm::WorkCounters), s);
  if (e == cudaSuccess) e = cudaEventRecord(ctx->evx0, s);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->aux, ctx->evx0, 0);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "pipeline set-up");
  cudaEventRecord(ctx->ev0, s);
  for (int k = 0; k < nch && e == cudaSuccess; ++k) {
    const int64_t a = cut(k), b = cut(k + 1), n = b - a;
    cudaStream_t q = (k & 1) ? ctx->aux : s;
    gm::WorkCounters* w = (k & 1) ? ctx->work2 : ctx->work;
    e = cudaMemcpyAsync((float*)a_in.dev + a * row, iquv + a * row, sizeof(float) * row * n,
                        cudaMemcpyHostToDevice, q);
    if (e == cudaSuccess) e = cudaMemsetAsync(&w->next_pixel, 0, sizeof(w->next_pixel), q);
    if (e != cudaSuccess) break;
    gm::DevCfg dc = gm::offset_cfg(d, a);
    gm::InvertArgs c = gm::offset_args(ia, a, n, nl, d.nterms);
    c.work = w;
    gm::InvertGeometry geo;
    if (prepass) {
      e = gm::launch_classical(dc, c.iquv, n, const_cast<double*>(c.init_models),
                               const_cast<uint32_t*>(c.init_status), true, q);
      if (e == cudaSuccess && learned)
        e = learned_starts(ctx, dc, c.iquv, n, const_cast<double*>(c.init_models), learned + a * 11,
                           const_cast<uint32_t*>(c.init_status), q);
      if (e != cudaSuccess) break;
      dc.init_mode = 1;
    }
    const int64_t grid = invert_grid(dc, c.init_models != nullptr && !c.init_status, ctx->sms, n, &geo);
    if (waves) {
      int nk = 0;
      e = gm::launch_invert_waves(dc, c, wb[k & 1], q, &nk);
      launches += nk + (prepass ? 1 : 0) + (learned ? 2 : 0);
    } else {
      e = gm::launch_invert(dc, c, (int)grid, q);
      launches += 1 + (prepass ? 1 : 0) + (learned ? 2 : 0);
    }
    ctx->stats.grid_blocks = (int)grid;
    ctx->stats.block_threads = geo.threads;
    ctx->stats.warps_per_block = geo.threads / 32;
    for (int o = 0; o < nouts && e == cudaSuccess; ++o) {
      const Arg& x = *outs[o];
      if (!x.host || !x.dev) continue;
      const size_t unit = x.bytes / (size_t)npix;
      e = cudaMemcpyAsync((char*)x.host + a * unit, (const char*)x.dev + a * unit, unit * n,
                          cudaMemcpyDeviceToHost, q);
    }
  }
  if (e == cudaSuccess) e = cudaEventRecord(ctx->evx1, ctx->aux);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(s, ctx->evx1, 0);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "pipelined inversion");
  cudaEventRecord(ctx->ev1, s);
  ctx->stats.kernel_launches = launches;
  ctx->stats.pixels = npix;
  // the cube came from host memory: the call returns with its results in place
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "pipelined inversion");
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  ctx->stats.kernel_ms = ms;
  gm::WorkCounters w0{}, w1{};
  cudaMemcpy(&w0, ctx->work, sizeof(w0), cudaMemcpyDeviceToHost);
  cudaMemcpy(&w1, ctx->work2, sizeof(w1), cudaMemcpyDeviceToHost);
  ctx->stats.iterations = (int64_t)(w0.iterations + w1.iterations);
  ctx->stats.accepted = (int64_t)(w0.accepted + w1.accepted);
  return GM_OK;
}

static gm_status invert_impl(gm_ctx* ctx, const gm::DevCfg& dcfg, const float* iquv, int64_t npix,
                             int nl, const double* init_models, const float* slight_map,
                             const double* lambda_map, float* model, double* model_f64, float* chi2, int* iters,
                             int* accepted, float* fitted, uint32_t* status, void* stream,
                             const StepOut* so = nullptr) {
  if (!ctx->configured) return fail(ctx, GM_ERR_NOT_CONFIGURED, "gm_configure first");
  if (!iquv || npix < 0) return fail(ctx, GM_ERR_INVALID, "iquv is NULL or npix < 0");
  if (nl != dcfg.nl) return fail(ctx, GM_ERR_INVALID, "nl differs from the configured grid");
  if (npix == 0) return GM_OK;
  cudaSetDevice(ctx->device);
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  if (ctx->scratch_pending) cudaStreamWaitEvent(s, ctx->ev_scratch, 0);
  const size_t cube = sizeof(float) * 4 * (size_t)nl * npix;
  // classical estimates of the start models in a pre-pass kernel, so that
  // their code stays out of the inversion kernel's instruction stream
  const bool prepass = dcfg.init_mode == 0 && !init_models;
  const bool learned = prepass && ctx->learned && !so;
  size_t need = cube + (fitted ? cube : 0) + (size_t)npix * (11 * 12 + 16) +
                (dcfg.lambda_per_pixel ? sizeof(double) * (size_t)nl * npix : 0) +
                (prepass ? (size_t)npix * (11 * 8 + 4) : 0) + (learned ? (size_t)npix * 11 * 8 : 0);
  if (need > ctx->budget) return fail(ctx, GM_ERR_NOMEM, "request exceeds the context's HBM budget");
  Arg a_in, a_init, a_sl, a_lam, a_model, a_m64, a_chi, a_it, a_acc, a_fit, a_st;
  gm_status st;
  // A large cube in host memory goes up in chunks on two alternating
  // streams, each chunk inverted by its own launch as soon as it has
  // arrived: the copies overlap the inversion, and a chunk's launch fills
  // the SMs that the previous one's last pixels leave free.
  const bool pipeline = !so && npix >= 2 * kPipeChunk && !is_device_ptr(iquv);
  if (pipeline) {
    if ((st = ensure_buf(ctx, "iquv", cube, &a_in.dev)) != GM_OK) return st;
    a_in.bytes = cube;
  } else if ((st = stage_in(ctx, "iquv", iquv, cube, &a_in, s)) != GM_OK) {
    return st;
  }
  if ((st = stage_in(ctx, "init", init_models, sizeof(double) * 11 * npix, &a_init, s)) != GM_OK) return st;
  gm::DevCfg d = dcfg;
  if (d.use_slight && d.slight_per_pixel) {
    if (!slight_map) return fail(ctx, GM_ERR_INVALID, "per-pixel stray light needs a map");
    if ((st = stage_in(ctx, "slight", slight_map, cube, &a_sl, s)) != GM_OK) return st;
    d.slight = (const float*)a_sl.dev;
  }
  if (d.lambda_per_pixel) {
    if (!lambda_map) return fail(ctx, GM_ERR_INVALID, "per-pixel wavelength grids need lambda_map");
    if ((st = stage_in(ctx, "lammap", lambda_map, sizeof(double) * (size_t)nl * npix, &a_lam, s)) != GM_OK)
      return st;
    d.lam_map = (const double*)a_lam.dev;
  }
  if ((st = stage_out(ctx, "model", model, sizeof(float) * 11 * npix, &a_model)) != GM_OK) return st;
  if ((st = stage_out(ctx, "model64", model_f64, sizeof(double) * 11 * npix, &a_m64)) != GM_OK) return st;
  if ((st = stage_out(ctx, "chi2", chi2, sizeof(float) * npix, &a_chi)) != GM_OK) return st;
  if ((st = stage_out(ctx, "iters", iters, sizeof(int) * npix, &a_it)) != GM_OK) return st;
  if ((st = stage_out(ctx, "acc", accepted, sizeof(int) * npix, &a_acc)) != GM_OK) return st;
  if ((st = stage_out(ctx, "fitted", fitted, cube, &a_fit)) != GM_OK) return st;
  if ((st = stage_out(ctx, "status", status, sizeof(uint32_t) * npix, &a_st)) != GM_OK) return st;
  Arg a_sd, a_strial, a_sc0, a_sc1;
  if (so) {
    if ((st = stage_out(ctx, "sdelta", so->delta, sizeof(float) * d.nterms * npix, &a_sd)) != GM_OK) return st;
    if ((st = stage_out(ctx, "strial", so->trial, sizeof(double) * 11 * npix, &a_strial)) != GM_OK) return st;
    if ((st = stage_out(ctx, "sc0", so->chi2_start, sizeof(float) * npix, &a_sc0)) != GM_OK) return st;
    if ((st = stage_out(ctx, "sc1", so->chi2_trial, sizeof(float) * npix, &a_sc1)) != GM_OK) return st;
  }

  gm::InvertArgs ia{};
  ia.iquv = (const float*)a_in.dev;
  ia.npix = npix;
  ia.init_models = (const double*)a_init.dev;
  ia.model = (float*)a_model.dev;
  ia.model_f64 = (double*)a_m64.dev;
  ia.chi2 = (float*)a_chi.dev;
  ia.iters = (int*)a_it.dev;
  ia.accepted = (int*)a_acc.dev;
  ia.fitted = (float*)a_fit.dev;
  ia.status = (uint32_t*)a_st.dev;
  ia.step_delta = (float*)a_sd.dev;
  ia.step_trial = (double*)a_strial.dev;
  ia.step_chi2_start = (float*)a_sc0.dev;
  ia.step_chi2_trial = (float*)a_sc1.dev;
  ia.work = ctx->work;
  if (prepass) {
    void *mp = nullptr, *sp = nullptr;
    if ((st = ensure_buf(ctx, "cinit", sizeof(double) * 11 * npix, &mp)) != GM_OK) return st;
    if ((st = ensure_buf(ctx, "cstat", sizeof(uint32_t) * npix, &sp)) != GM_OK) return st;
    ia.init_models = (const double*)mp;
    ia.init_status = (const uint32_t*)sp;
  }
  double* lguess = nullptr;
  if (learned) {
    void* lp = nullptr;
    if ((st = ensure_buf(ctx, "linit", sizeof(double) * 11 * npix, &lp)) != GM_OK) return st;
    lguess = (double*)lp;
    cudaMemsetAsync(ctx->mlp_err, 0, sizeof(int), s);
  }
  const Arg* outs[] = {&a_model, &a_m64, &a_chi, &a_it, &a_acc, &a_fit, &a_st,
                       &a_sd, &a_strial, &a_sc0, &a_sc1};
  if (pipeline) {
    st = invert_chunks(ctx, d, ia, iquv, a_in, outs, 7, npix, nl, prepass, lguess, need, s);
    return (st == GM_OK && learned) ? learned_check(ctx) : st;
  }
  cudaError_t e = cudaMemsetAsync(ctx->work, 0, sizeof(gm::WorkCounters), s);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "work counter reset");
  if (prepass) {
    e = gm::launch_classical(d, ia.iquv, npix, const_cast<double*>(ia.init_models),
                             const_cast<uint32_t*>(ia.init_status), true, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "classical-estimates pre-pass");
    if (learned) {
      e = learned_starts(ctx, d, ia.iquv, npix, const_cast<double*>(ia.init_models), lguess,
                         const_cast<uint32_t*>(ia.init_status), s);
      if (e != cudaSuccess) return cuda_fail(ctx, e, "learned initial guess");
    }
    d.init_mode = 1;
  }
  gm::InvertGeometry geo;
  const int64_t grid = invert_grid(d, ia.init_models != nullptr && !ia.init_status, ctx->sms, npix, &geo);
  const int64_t wchunk = want_waves(ctx, d, ia, npix) ? wave_chunk_for(ctx, d, need, npix, 1) : 0;
  const bool waves = wchunk > 0;
  gm::WaveBuffers wb{};
  if (waves && (st = wave_buffers(ctx, "waves0", d, wchunk, &wb)) != GM_OK) return st;
  int launches = 1;
  cudaEventRecord(ctx->ev0, s);
  e = waves ? gm::launch_invert_waves(d, ia, wb, s, &launches) : gm::launch_invert(d, ia, (int)grid, s);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "inversion kernel launch");
  cudaEventRecord(ctx->ev1, s);
  ctx->stats.grid_blocks = (int)grid;
  ctx->stats.block_threads = geo.threads;
  ctx->stats.warps_per_block = geo.threads / 32;
  ctx->stats.kernel_launches = launches + (prepass ? 1 : 0) + (learned ? 2 : 0);
  ctx->stats.pixels = npix;
  bool any_host = false;
  for (const Arg* o : outs) {
    if ((st = copy_back(ctx, *o, s)) != GM_OK) return st;
    any_host |= (o->host != nullptr);
  }
  any_host |= (a_in.dev != (void*)iquv);
  cudaEventRecord(ctx->ev_scratch, s);
  ctx->scratch_pending = true;
  if (any_host || !stream) {
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "inversion");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    ctx->stats.kernel_ms = ms;
    gm::WorkCounters wc{};
    cudaMemcpy(&wc, ctx->work, sizeof(wc), cudaMemcpyDeviceToHost);
    ctx->stats.iterations = (int64_t)wc.iterations;
    ctx->stats.accepted = (int64_t)wc.accepted;
    if (learned) return learned_check(ctx);
  }
  return GM_OK;
}

gm_status gm_invert_ex(gm_ctx* ctx, const float* iquv, int64_t npix, int nl,
                       const double* init_models, float* model, double* model_f64, float* chi2,
                       int* iters, int* accepted, float* fitted, uint32_t* status, void* stream) {
  if (!ctx) return GM_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->call_mu);
  gm::DevCfg d = ctx->dev;
  if (init_models) d.init_mode = 1;
  const float* map = (ctx->cfg.use_slight && ctx->cfg.slight_per_pixel) ? ctx->cfg.slight : nullptr;
  return invert_impl(ctx, d, iquv, npix, nl, init_models, map, ctx->cfg.lambda_map, model, model_f64, chi2, iters,
                     accepted, fitted, status, stream);
}

gm_status gm_invert(gm_ctx* ctx, const float* iquv, int64_t npix, int nl, float* model,
                    float* chi2, int* iters, float* fitted, uint32_t* status, void* stream) {
  return gm_invert_ex(ctx, iquv, npix, nl, nullptr, model, nullptr, chi2, iters, nullptr, fitted,
                      status, stream);
}

gm_status gm_lm_step(gm_ctx* ctx, const float* iquv, int64_t npix, int nl, const double* models,
                     float flambda, float* delta, double* trial, float* chi2_start,
                     float* chi2_trial, void* stream) {
  if (!ctx) return GM_ERR_INVALID;
  if (!models) return fail(ctx, GM_ERR_INVALID, "gm_lm_step needs the starting models");
  std::lock_guard<std::mutex> lk(ctx->call_mu);
  gm::DevCfg d = ctx->dev;
  d.init_mode = 1;
  d.miter = 1;
  d.ilambda = flambda;
  StepOut so;
  so.delta = delta;
  so.trial = trial;
  so.chi2_start = chi2_start;
  so.chi2_trial = chi2_trial;
  const float* map = (ctx->cfg.use_slight && ctx->cfg.slight_per_pixel) ? ctx->cfg.slight : nullptr;
  return invert_impl(ctx, d, iquv, npix, nl, models, map, ctx->cfg.lambda_map, nullptr, nullptr, nullptr, nullptr, nullptr,
                     nullptr, nullptr, stream, &so);
}

static gm_status synth_impl(gm_ctx* ctx, const float* m32, const double* m64, int64_t npix,
                            float* iquv, float* rf, void* stream) {
  if (!ctx) return GM_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->call_mu);
  if (!ctx->configured) return fail(ctx, GM_ERR_NOT_CONFIGURED, "gm_configure first");
  if ((!m32 && !m64) || !iquv || npix < 0) return fail(ctx, GM_ERR_INVALID, "null argument");
  if (npix == 0) return GM_OK;
  cudaSetDevice(ctx->device);
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  const int nl = ctx->dev.nl, nt = ctx->dev.nterms;
  Arg a_m, a_out, a_rf, a_sl, a_lam;
  gm_status st;
  if (m32) st = stage_in(ctx, "smodels", m32, sizeof(float) * 11 * npix, &a_m, s);
  else st = stage_in(ctx, "smodels", m64, sizeof(double) * 11 * npix, &a_m, s);
  if (st != GM_OK) return st;
  if ((st = stage_out(ctx, "siquv", iquv, sizeof(float) * 4 * nl * npix, &a_out)) != GM_OK) return st;
  if ((st = stage_out(ctx, "srf", rf, sizeof(float) * 4 * nt * nl * npix, &a_rf)) != GM_OK) return st;
  gm::DevCfg d = ctx->dev;
  // the synthesis path returns every response function (kernel_synthesis
  // calls me_der without zeroing fixed parameters, gmilos.cu:71-84)
  for (int i = 0; i < GM_NPAR; ++i) d.fix[i] = 1;
  if (d.use_slight && d.slight_per_pixel) {
    if ((st = stage_in(ctx, "sslight", ctx->cfg.slight, sizeof(float) * 4 * nl * npix, &a_sl, s)) != GM_OK) return st;
    d.slight = (const float*)a_sl.dev;
  }
  if (d.lambda_per_pixel) {
    if (!ctx->cfg.lambda_map) return fail(ctx, GM_ERR_INVALID, "per-pixel wavelength grids need lambda_map");
    if ((st = stage_in(ctx, "slammap", ctx->cfg.lambda_map, sizeof(double) * (size_t)nl * npix, &a_lam, s)) != GM_OK)
      return st;
    d.lam_map = (const double*)a_lam.dev;
  }
  gm::SynthArgs sa{};
  sa.models_f32 = m32 ? (const float*)a_m.dev : nullptr;
  sa.models_f64 = m64 ? (const double*)a_m.dev : nullptr;
  sa.npix = npix;
  sa.iquv = (float*)a_out.dev;
  sa.rf = (float*)a_rf.dev;
  cudaError_t e = gm::launch_synth(d, sa, s);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "synthesis kernel launch");
  if ((st = copy_back(ctx, a_out, s)) != GM_OK) return st;
  if ((st = copy_back(ctx, a_rf, s)) != GM_OK) return st;
  if (a_out.host || a_rf.host || a_m.dev != (m32 ? (const void*)m32 : (const void*)m64) || !stream) {
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "synthesis");
  }
  return GM_OK;
}

gm_status gm_synthesize(gm_ctx* ctx, const float* models, int64_t npix, float* iquv, float* rf,
                        void* stream) {
  return synth_impl(ctx, models, nullptr, npix, iquv, rf, stream);
}

gm_status gm_synthesize_f64(gm_ctx* ctx, const double* models, int64_t npix, float* iquv, float* rf,
                            void* stream) {
  return synth_impl(ctx, nullptr, models, npix, iquv, rf, stream);
}

gm_status gm_synthesize_grid(gm_ctx* ctx, const double* models, int64_t npix, const double* offsets,
                             int ngrid, float* iquv, void* stream) {
  if (!ctx) return GM_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->call_mu);
  if (!ctx->configured) return fail(ctx, GM_ERR_NOT_CONFIGURED, "gm_configure first");
  if (!models || !offsets || !iquv || npix < 0 || ngrid < 1) return fail(ctx, GM_ERR_INVALID, "bad argument");
  if (npix == 0) return GM_OK;
  cudaSetDevice(ctx->device);
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  Arg a_m, a_o, a_out;
  gm_status st;
  if ((st = stage_in(ctx, "gmodels", models, sizeof(double) * 11 * npix, &a_m, s)) != GM_OK) return st;
  if ((st = stage_in(ctx, "goffs", offsets, sizeof(double) * ngrid, &a_o, s)) != GM_OK) return st;
  if ((st = stage_out(ctx, "giquv", iquv, sizeof(float) * 4 * (size_t)ngrid * npix, &a_out)) != GM_OK) return st;
  cudaError_t e = gm::launch_synth_grid(ctx->dev, (const double*)a_m.dev, npix, (const double*)a_o.dev,
                                        ngrid, (float*)a_out.dev, s);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "grid synthesis launch");
  if ((st = copy_back(ctx, a_out, s)) != GM_OK) return st;
  if (a_out.host || a_m.dev != (const void*)models || !stream) {
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "grid synthesis");
  }
  return GM_OK;
}

gm_status gm_classical(gm_ctx* ctx, const float* iquv, int64_t npix, int nl, double* models,
                       void* stream) {
  if (!ctx) return GM_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->call_mu);
  if (!ctx->configured) return fail(ctx, GM_ERR_NOT_CONFIGURED, "gm_configure first");
  if (!iquv || !models || npix < 0) return fail(ctx, GM_ERR_INVALID, "bad argument");
  if (nl != ctx->dev.nl) return fail(ctx, GM_ERR_INVALID, "nl differs from the configured grid");
  if (npix == 0) return GM_OK;
  cudaSetDevice(ctx->device);
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  Arg a_in, a_out, a_lam;
  gm_status st;
  if ((st = stage_in(ctx, "iquv", iquv, sizeof(float) * 4 * (size_t)nl * npix, &a_in, s)) != GM_OK) return st;
  if ((st = stage_out(ctx, "cmodels", models, sizeof(double) * 11 * npix, &a_out)) != GM_OK) return st;
  gm::DevCfg d = ctx->dev;
  if (d.lambda_per_pixel) {
    if (!ctx->cfg.lambda_map) return fail(ctx, GM_ERR_INVALID, "per-pixel wavelength grids need lambda_map");
    if ((st = stage_in(ctx, "lammap", ctx->cfg.lambda_map, sizeof(double) * (size_t)nl * npix, &a_lam, s)) != GM_OK)
      return st;
    d.lam_map = (const double*)a_lam.dev;
  }
  cudaError_t e = gm::launch_classical(d, (const float*)a_in.dev, npix, (double*)a_out.dev, nullptr, false, s);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "classical-estimates launch");
  if ((st = copy_back(ctx, a_out, s)) != GM_OK) return st;
  if (a_out.host || a_in.dev != (const void*)iquv || !stream) {
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "classical estimates");
  }
  return GM_OK;
}

gm_status gm_get_stats(gm_ctx* ctx, gm_stats* out) {
  if (!ctx || !out) return GM_ERR_INVALID;
  *out = ctx->stats;
  return GM_OK;
}

gm_status gm_measure_peaks(gm_ctx* ctx, double* fp32_tflops, double* fp64_tflops) {
  if (!ctx) return GM_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->call_mu);
  cudaSetDevice(ctx->device);
  void* sink = nullptr;
  gm_status st = ensure_buf(ctx, "peaksink", sizeof(double) * 1024 * 1024, &sink);
  if (st != GM_OK) return st;
  const int blocks = ctx->sms * 8, threads = 256;
  double best32 = 0, best64 = 0;
  for (int rep = 0; rep < 4; ++rep) {
    for (int kind = 0; kind < 2; ++kind) {
      const int iters = kind == 0 ? 4096 : 1024;
      cudaEventRecord(ctx->ev0, ctx->stream);
      cudaError_t e = gm::launch_peak(kind, blocks, threads, iters, sink, ctx->stream);
      if (e != cudaSuccess) return cuda_fail(ctx, e, "peak kernel");
      cudaEventRecord(ctx->ev1, ctx->stream);
      e = cudaEventSynchronize(ctx->ev1);
      if (e != cudaSuccess) return cuda_fail(ctx, e, "peak kernel");
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
      const double flops = 2.0 * gm::kPeakChains * (double)iters * blocks * threads;
      const double tf = flops / (ms * 1e-3) / 1e12;
      if (kind == 0) best32 = std::max(best32, tf); else best64 = std::max(best64, tf);
    }
  }
  if (fp32_tflops) *fp32_tflops = best32;
  if (fp64_tflops) *fp64_tflops = best64;
  return GM_OK;
}

size_t gm_wave_state_bytes(int nl, int miter, int64_t pixels) {
  if (nl < 1 || nl > GM_MAX_NL || pixels < 0) return 0;
  return gm::wave_buffer_bytes(nl, miter, pixels);
}

gm_status gm_measure_sfu_peak(gm_ctx* ctx, double* gops) {
  if (!ctx || !gops) return GM_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->call_mu);
  cudaSetDevice(ctx->device);
  void* sink = nullptr;
  gm_status st = ensure_buf(ctx, "peaksink", sizeof(double) * 1024 * 1024, &sink);
  if (st != GM_OK) return st;
  const int blocks = ctx->sms * 8, threads = 256, iters = 1024;
  double best = 0;
  for (int rep = 0; rep < 4; ++rep) {
    cudaEventRecord(ctx->ev0, ctx->stream);
    cudaError_t e = gm::launch_peak(2, blocks, threads, iters, sink, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "SFU peak kernel");
    cudaEventRecord(ctx->ev1, ctx->stream);
    e = cudaEventSynchronize(ctx->ev1);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "SFU peak kernel");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    const double ops = (double)gm::kPeakChains * iters * blocks * threads;
    best = std::max(best, ops / (ms * 1e-3) / 1e9);
  }
  *gops = best;
  return GM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- serving
// Continuous batching.  Submitted requests wait in a FIFO until they fit:
// at most serve_max_active admitted at a time and their device memory
// within the context's HBM budget.  Admitted requests are cut into chunks
// of serve_chunk pixels; a dispatcher thread keeps each of serve_streams
// lanes (a stream with its own work counters) busy with the next chunk of
// the admitted request the serving policy picks, so chunks of different
// requests overlap on the device (with round robin a newly admitted request
// starts within one chunk time).  Pixels are independent, so every result
// is the same whatever the mix it ran in.
namespace {

size_t request_bytes(const gm_request& q) {
  const size_t P = (size_t)q.npix;
  size_t b = 0;
  if (!is_device_ptr(q.iquv)) b += sizeof(float) * 4 * (size_t)q.nl * P;
  if (!is_device_ptr(q.model)) b += sizeof(float) * 11 * P;
  if (q.chi2 && !is_device_ptr(q.chi2)) b += sizeof(float) * P;
  if (q.iters && !is_device_ptr(q.iters)) b += sizeof(int) * P;
  if (q.status && !is_device_ptr(q.status)) b += sizeof(uint32_t) * P;
  return b;
}

template <typename T>
bool device_view(Request& r, T* user, size_t bytes, T** out) {
  if (!user) {
    *out = nullptr;
    return true;
  }
  if (is_device_ptr(user)) {
    *out = user;
    return true;
  }
  void* p = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  r.owned.push_back(p);
  *out = (T*)p;
  return true;
}

void release(Request& r) {
  for (void* p : r.owned) cudaFree(p);
  r.owned.clear();
}

void serve_loop(gm_ctx* ctx);

}  // namespace

extern "C" {

gm_status gm_serving_options(gm_ctx* ctx, int streams, int64_t chunk_pixels, int max_active) {
  if (!ctx || streams < 1 || streams > 32 || chunk_pixels < 1 || max_active < 1) return GM_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!ctx->lanes.empty()) return fail(ctx, GM_ERR_INVALID, "serving already started");
  ctx->serve_streams = streams;
  ctx->serve_chunk = chunk_pixels;
  ctx->serve_max_active = max_active;
  return GM_OK;
}

gm_status gm_serving_policy(gm_ctx* ctx, int policy) {
  if (!ctx) return GM_ERR_INVALID;
  if (policy != GM_SERVE_ROUND_ROBIN && policy != GM_SERVE_FIFO && policy != GM_SERVE_SHORTEST_FIRST &&
      policy != GM_SERVE_RESPONSE_RATIO)
    return fail(ctx, GM_ERR_INVALID, "unknown serving policy");
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->serve_policy = policy;
  return GM_OK;
}

gm_status gm_submit(gm_ctx* ctx, const gm_request* req, gm_ticket* ticket) {
  if (!ctx || !req || !ticket) return GM_ERR_INVALID;
  if (!ctx->configured) return fail(ctx, GM_ERR_NOT_CONFIGURED, "gm_configure first");
  if (!req->iquv || !req->model || req->npix < 0 || req->nl != ctx->dev.nl)
    return fail(ctx, GM_ERR_INVALID, "bad request");
  if (ctx->dev.use_slight && ctx->dev.slight_per_pixel)
    return fail(ctx, GM_ERR_UNSUPPORTED, "serving takes one stray-light profile, not a per-pixel map");
  if (ctx->dev.lambda_per_pixel)
    return fail(ctx, GM_ERR_UNSUPPORTED, "serving takes one wavelength grid, not per-pixel grids");
  if (ctx->learned)
    return fail(ctx, GM_ERR_UNSUPPORTED, "serving starts from the classical estimates, not the learned guess");
  auto r = std::make_shared<Request>();
  r->req = *req;
  r->dev = ctx->dev;
  if (req->fix) {
    for (int i = 0; i < GM_NPAR; ++i) r->dev.fix[i] = req->fix[i] ? 1 : 0;
    r->dev.nterms = (r->dev.fix[9] && r->dev.fix[10]) ? 11 : 10;
  }
  r->bytes = request_bytes(*req);
  if (r->bytes > ctx->budget) return fail(ctx, GM_ERR_NOMEM, "request exceeds the context's HBM budget");
  r->t_submit = Clock::now();
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!ctx->worker.joinable()) ctx->worker = std::thread(serve_loop, ctx);
  const gm_ticket t = ctx->next_ticket++;
  ctx->reqs[t] = r;
  ctx->queue.push_back(t);
  *ticket = t;
  ctx->cv.notify_all();
  return GM_OK;
}

gm_status gm_poll(gm_ctx* ctx, gm_ticket ticket, int timeout_us) {
  if (!ctx) return GM_ERR_INVALID;
  std::unique_lock<std::mutex> lk(ctx->mu);
  auto it = ctx->reqs.find(ticket);
  if (it == ctx->reqs.end()) return fail(ctx, GM_ERR_INVALID, "unknown ticket");
  auto r = it->second;
  auto pred = [&] { return r->done; };
  if (timeout_us < 0) ctx->done_cv.wait(lk, pred);
  else if (!ctx->done_cv.wait_for(lk, std::chrono::microseconds(timeout_us), pred)) return GM_ERR_TIMEOUT;
  ctx->reqs.erase(ticket);
  return r->cancelled ? GM_ERR_CANCELLED : r->result;
}

gm_status gm_cancel(gm_ctx* ctx, gm_ticket ticket) {
  if (!ctx) return GM_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  auto it = ctx->reqs.find(ticket);
  if (it == ctx->reqs.end()) return fail(ctx, GM_ERR_INVALID, "unknown ticket");
  auto q = std::find(ctx->queue.begin(), ctx->queue.end(), ticket);
  if (q != ctx->queue.end()) {   // not admitted yet: nothing of it runs
    ctx->queue.erase(q);
    it->second->cancelled = true;
    it->second->done = true;
    ctx->done_cv.notify_all();
  }
  return GM_OK;
}

}  // extern "C"

namespace {

// Launch the next chunk of r on lane L (dispatcher thread only).
gm_status launch_chunk(gm_ctx* ctx, ServeLane& L, const std::shared_ptr<Request>& rp) {
  Request& r = *rp;
  const gm_request& q = r.req;
  const int nl = q.nl;
  const int64_t off = r.next;
  const int64_t n = std::min<int64_t>(ctx->serve_chunk, q.npix - off);
  const size_t row = 4 * (size_t)nl;
  cudaStream_t s = L.stream;
  cudaError_t e = cudaSuccess;
  if ((const void*)r.d_in != (const void*)q.iquv)
    e = cudaMemcpyAsync(r.d_in + off * row, q.iquv + off * row, sizeof(float) * row * n,
                        cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(L.work, 0, sizeof(gm::WorkCounters), s);
  if (e != cudaSuccess) return GM_ERR_CUDA;
  gm::InvertArgs ia{};
  ia.iquv = r.d_in + off * row;
  ia.npix = n;
  ia.model = r.d_model + off * 11;
  ia.chi2 = r.d_chi2 ? r.d_chi2 + off : nullptr;
  ia.iters = r.d_iters ? r.d_iters + off : nullptr;
  ia.status = r.d_status ? r.d_status + off : nullptr;
  ia.work = L.work;
  // the path of gm_invert: classical start models in a pre-pass, then the
  // wave-synchronous kernels where they cover the configuration
  gm::DevCfg d = r.dev;
  const bool lane_ok = L.scratch && L.nl == d.nl && L.miter == d.miter && n <= L.chunk;
  if (lane_ok && d.init_mode == 0) {
    double* cm = reinterpret_cast<double*>(static_cast<char*>(L.scratch) + L.wave_bytes);
    uint32_t* cs = reinterpret_cast<uint32_t*>(cm + 11 * L.chunk);
    e = gm::launch_classical(d, ia.iquv, n, cm, cs, true, s);
    if (e != cudaSuccess) return GM_ERR_CUDA;
    ia.init_models = cm;
    ia.init_status = cs;
    d.init_mode = 1;
  }
  if (lane_ok && want_waves(ctx, d, ia, q.npix)) {
    e = gm::launch_invert_waves(d, ia, gm::wave_buffers(L.scratch, d.nl, d.miter, L.chunk), s, nullptr);
  } else {
    const int64_t grid = invert_grid(d, ia.init_models != nullptr && !ia.init_status, ctx->sms, n, nullptr);
    e = gm::launch_invert(d, ia, (int)grid, s);
  }
  if (e != cudaSuccess) return GM_ERR_CUDA;
  auto back = [&](void* host, const void* dev, size_t bytes) {
    if (e == cudaSuccess && host && host != dev) e = cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, s);
  };
  back(q.model + off * 11, r.d_model + off * 11, sizeof(float) * 11 * n);
  if (q.chi2) back(q.chi2 + off, r.d_chi2 + off, sizeof(float) * n);
  if (q.iters) back(q.iters + off, r.d_iters + off, sizeof(int) * n);
  if (q.status) back(q.status + off, r.d_status + off, sizeof(uint32_t) * n);
  if (e == cudaSuccess) e = cudaEventRecord(L.done, s);
  if (e != cudaSuccess) return GM_ERR_CUDA;
  r.next = off + n;
  ++r.outstanding;
  if (!r.started) {
    r.started = true;
    r.t_start = Clock::now();
  }
  L.req = rp;
  L.busy = true;
  return GM_OK;
}

void finish(gm_ctx* ctx, const std::shared_ptr<Request>& r, gm_status st) {
  const auto now = Clock::now();
  if (r->req.latency_ms)
    *r->req.latency_ms = std::chrono::duration<double, std::milli>(now - r->t_submit).count();
  if (r->req.queue_ms)
    *r->req.queue_ms = std::chrono::duration<double, std::milli>((r->started ? r->t_start : now) - r->t_submit).count();
  release(*r);
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->serve_bytes -= r->bytes;
  ctx->active.erase(std::remove(ctx->active.begin(), ctx->active.end(), r), ctx->active.end());
  r->result = st;
  r->done = true;
  ctx->done_cv.notify_all();
}

void serve_loop(gm_ctx* ctx) {
  cudaSetDevice(ctx->device);
  {
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->lanes.resize(ctx->serve_streams);
    for (ServeLane& L : ctx->lanes) {
      cudaStreamCreateWithFlags(&L.stream, cudaStreamNonBlocking);
      cudaMalloc(&L.work, sizeof(gm::WorkCounters));
      cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming);
      L.nl = ctx->dev.nl;
      L.miter = ctx->dev.miter;
      L.chunk = ctx->serve_chunk;
      L.wave_bytes = (gm::wave_buffer_bytes(L.nl, L.miter, L.chunk) + 255) & ~(size_t)255;
      if (cudaMalloc(&L.scratch, L.wave_bytes + (sizeof(double) * 11 + sizeof(uint32_t)) * (size_t)L.chunk) !=
          cudaSuccess) {
        cudaGetLastError();
        L.scratch = nullptr;
      }
    }
  }
  for (;;) {
    bool progress = false;
    // admission in arrival order, within the request-count and memory limits
    std::vector<std::shared_ptr<Request>> admit;
    {
      std::lock_guard<std::mutex> lk(ctx->mu);
      while (!ctx->queue.empty() && (int)ctx->active.size() + (int)admit.size() < ctx->serve_max_active) {
        auto r = ctx->reqs[ctx->queue.front()];
        if (ctx->serve_bytes + r->bytes > ctx->budget && !(ctx->active.empty() && admit.empty())) break;
        ctx->queue.pop_front();
        ctx->serve_bytes += r->bytes;
        admit.push_back(r);
      }
    }
    for (auto& r : admit) {
      const gm_request& q = r->req;
      const size_t P = (size_t)q.npix;
      bool ok = device_view(*r, const_cast<float*>(q.iquv), sizeof(float) * 4 * (size_t)q.nl * P, &r->d_in) &&
                device_view(*r, q.model, sizeof(float) * 11 * P, &r->d_model) &&
                device_view(*r, q.chi2, sizeof(float) * P, &r->d_chi2) &&
                device_view(*r, q.iters, sizeof(int) * P, &r->d_iters) &&
                device_view(*r, q.status, sizeof(uint32_t) * P, &r->d_status);
      {
        std::lock_guard<std::mutex> lk(ctx->mu);
        ctx->active.push_back(r);
      }
      if (!ok) finish(ctx, r, GM_ERR_NOMEM);
      else if (q.npix == 0) finish(ctx, r, GM_OK);
      progress = true;
    }
    // completed chunks
    for (ServeLane& L : ctx->lanes) {
      if (!L.busy) continue;
      const cudaError_t e = cudaEventQuery(L.done);
      if (e == cudaErrorNotReady) continue;
      auto r = L.req;
      L.busy = false;
      L.req.reset();
      progress = true;
      if (e != cudaSuccess) {
        cudaGetLastError();
        r->result = GM_ERR_CUDA;
      }
      if (--r->outstanding == 0 && (r->next >= r->req.npix || r->result != GM_OK))
        finish(ctx, r, r->result);
    }
    // keep every lane busy with the next chunk of the request the policy
    // picks: round robin over the admitted requests, the earliest submitted,
    // the one with the fewest pixels left, or the one with the highest
    // response ratio (time since submission over its pixels; compared
    // cross-multiplied)
    for (ServeLane& L : ctx->lanes) {
      if (L.busy) continue;
      std::shared_ptr<Request> pick;
      {
        std::lock_guard<std::mutex> lk(ctx->mu);
        const Clock::time_point now = Clock::now();
        auto waited = [&](const Request& q) { return std::chrono::duration<double>(now - q.t_submit).count(); };
        const size_t n = ctx->active.size();
        for (size_t k = 0; k < n; ++k) {
          const size_t i = (ctx->rr + k) % n;
          auto& c = ctx->active[i];
          if (c->result != GM_OK || c->next >= c->req.npix || c->done) continue;
          bool better = !pick;
          if (pick && ctx->serve_policy == GM_SERVE_FIFO) better = c->t_submit < pick->t_submit;
          if (pick && ctx->serve_policy == GM_SERVE_SHORTEST_FIRST)
            better = c->req.npix - c->next < pick->req.npix - pick->next;
          if (pick && ctx->serve_policy == GM_SERVE_RESPONSE_RATIO)
            better = waited(*c) * (double)pick->req.npix > waited(*pick) * (double)c->req.npix;
          if (better) {
            pick = c;
            if (ctx->serve_policy == GM_SERVE_ROUND_ROBIN) {
              ctx->rr = (i + 1) % n;
              break;
            }
          }
        }
      }
      if (!pick) break;
      if (launch_chunk(ctx, L, pick) != GM_OK) {
        cudaGetLastError();
        pick->result = GM_ERR_CUDA;
        pick->next = pick->req.npix;
        if (pick->outstanding == 0) finish(ctx, pick, GM_ERR_CUDA);
      }
      progress = true;
    }
    std::unique_lock<std::mutex> lk(ctx->mu);
    bool idle = ctx->active.empty();
    for (const ServeLane& L : ctx->lanes) idle = idle && !L.busy;
    if (ctx->stopping && ctx->queue.empty() && idle) break;
    if (!progress) {
      if (idle && ctx->queue.empty()) ctx->cv.wait(lk, [&] { return ctx->stopping || !ctx->queue.empty(); });
      else ctx->cv.wait_for(lk, std::chrono::microseconds(50));
    }
  }
  for (ServeLane& L : ctx->lanes) {
    cudaStreamSynchronize(L.stream);
    cudaFree(L.work);
    if (L.scratch) cudaFree(L.scratch);
    cudaEventDestroy(L.done);
    cudaStreamDestroy(L.stream);
  }
  ctx->lanes.clear();
}

}  // namespace

// ---------------------------------------------------------------- ragged batches
namespace {

// One samples-per-lane class of a ragged batch: its grids' configurations,
// its ROIs in batch order, its pixels' grid indices and profile offsets, and
// the device buffers of its launch.
struct BatchClass {
  std::vector<gm::DevCfg> cfgs;
  std::vector<int> rois;              // indices into the batch
  std::vector<int64_t> first;         // first pixel of each of its ROIs
  std::vector<uint64_t> in_off;       // offset (floats) of each ROI's profiles
  int64_t pixels = 0;
  uint64_t floats = 0;                // profile floats of the class
  // device
  float* in = nullptr;
  float* model = nullptr;
  float* chi2 = nullptr;
  int* iters = nullptr;
  uint32_t* status = nullptr;
  double* cinit = nullptr;
  uint32_t* cstat = nullptr;
  gm::DevCfg* dcfgs = nullptr;
  uint16_t* grid = nullptr;
  uint64_t* off = nullptr;
  gm::WaveBuffers wb{};
  int bt = 0, ba = 0;                 // resident blocks per SM (full)
};

// The configuration of one grid: the context's, with the grid's samples and
// PSF taps (the host-side arithmetic of build_devcfg).
gm::DevCfg grid_devcfg(const gm::DevCfg& base, const gm_roi& r, double lambda0) {
  gm::DevCfg d = base;
  d.nl = r.nl;
  d.use_psf = r.psf ? 1 : 0;
  for (int l = 0; l < gm::kMaxNl; ++l) {
    const bool in = l < r.nl;
    const double off = in ? r.lambda[l] - lambda0 : 0.0;
    d.dl[l] = (float)off;
    d.dld[l] = off;
    d.lam[l] = in ? r.lambda[l] : 0.0;
    d.psfd[l] = (in && r.psf) ? r.psf[l] : 0.0;
  }
  d.init_mode = 1;   // start models from the classical pre-pass
  return d;
}

bool same_grid(const gm_roi& a, const gm_roi& b) {
  if (a.nl != b.nl || (a.psf == nullptr) != (b.psf == nullptr)) return false;
  if (std::memcmp(a.lambda, b.lambda, sizeof(double) * a.nl)) return false;
  return !a.psf || !std::memcmp(a.psf, b.psf, sizeof(double) * a.nl);
}

// The device work of a batch (both classes, class 1 on the auxiliary stream
// between a fork and a join), launched directly or captured.
cudaError_t batch_device_work(gm_ctx* ctx, BatchClass* cls, const int (*cap)[2], cudaStream_t s, int* launches) {
  cudaError_t e = cudaEventRecord(ctx->evx0, s);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->aux, ctx->evx0, 0);
  for (int c = 0; c < 2 && e == cudaSuccess; ++c) {
    BatchClass& k = cls[c];
    if (!k.pixels) continue;
    cudaStream_t q = c == 0 ? s : ctx->aux;
    gm::WorkCounters* w = c == 0 ? ctx->work : ctx->work2;
    gm::MultiGrid mg{k.dcfgs, k.grid, k.off};
    e = cudaMemsetAsync(w, 0, sizeof(gm::WorkCounters), q);
    if (e == cudaSuccess) e = gm::launch_classical_mg(k.cfgs[0], mg, k.in, k.pixels, k.cinit, k.cstat, q);
    if (e != cudaSuccess) break;
    gm::InvertArgs ia{};
    ia.iquv = k.in;
    ia.npix = k.pixels;
    ia.init_models = k.cinit;
    ia.init_status = k.cstat;
    ia.model = k.model;
    ia.chi2 = k.chi2;
    ia.iters = k.iters;
    ia.status = k.status;
    ia.work = w;
    int n = 0;
    e = gm::launch_invert_waves_mg(k.cfgs[0], mg, ia, k.wb, cap[c][0], cap[c][1], q, &n);
    *launches += n + 1;
  }
  if (e == cudaSuccess) e = cudaEventRecord(ctx->evx1, ctx->aux);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(s, ctx->evx1, 0);
  return e;
}

}  // namespace

extern "C" gm_status gm_invert_rois(gm_ctx* ctx, const gm_roi* rois, int nroi, const gm_batch_opts* opts,
                                    gm_batch_stats* stats, void* stream) {
  if (!ctx) return GM_ERR_INVALID;
  if (!rois || nroi < 0) return fail(ctx, GM_ERR_INVALID, "bad argument");
  if (!ctx->configured) return fail(ctx, GM_ERR_NOT_CONFIGURED, "gm_configure first");
  const gm::DevCfg& base = ctx->dev;
  if (base.use_slight || base.lambda_per_pixel || ctx->learned || ctx->cfg.init_mode != GM_INIT_CLASSICAL)
    return fail(ctx, GM_ERR_UNSUPPORTED,
                "ragged batches start from the classical estimates, without stray light or per-pixel grids");
  for (int i = 0; i < nroi; ++i) {
    const gm_roi& r = rois[i];
    if (!r.iquv || !r.model || !r.lambda || r.npix < 0 || r.nl < 2 || r.nl > GM_MAX_NL)
      return fail(ctx, GM_ERR_INVALID, "ROI " + std::to_string(i) + ": bad description");
  }
  gm_batch_opts def{};
  if (!opts) opts = &def;
  std::lock_guard<std::mutex> lk(ctx->call_mu);
  cudaSetDevice(ctx->device);
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  if (ctx->scratch_pending) cudaStreamWaitEvent(s, ctx->ev_scratch, 0);
  // grids, classes, the pixels' tables
  BatchClass cls[2];
  std::vector<const gm_roi*> gfirst[2];   // one ROI per grid of a class
  std::string key;
  for (int i = 0; i < nroi; ++i) {
    const gm_roi& r = rois[i];
    BatchClass& k = cls[r.nl <= 32 ? 0 : 1];
    auto& gl = gfirst[r.nl <= 32 ? 0 : 1];
    int g = 0;
    while (g < (int)gl.size() && !same_grid(*gl[g], r)) ++g;
    if (g == (int)gl.size()) {
      if (g >= 65535) return fail(ctx, GM_ERR_INVALID, "too many distinct grids in one batch");
      gl.push_back(&r);
      k.cfgs.push_back(grid_devcfg(base, r, ctx->cfg.lambda0));
    }
    k.rois.push_back(i);
    k.first.push_back(k.pixels);
    k.in_off.push_back(k.floats);
    k.pixels += r.npix;
    k.floats += 4 * (uint64_t)r.nl * r.npix;
    key += std::to_string(r.npix) + ":" + std::to_string(r.nl) + ":" + std::to_string(g) + ";";
  }
  for (int c = 0; c < 2; ++c) key += "|" + std::to_string(cls[c].cfgs.size());
  gm_batch_stats st{};
  int64_t total = cls[0].pixels + cls[1].pixels;
  st.pixels = total;
  st.grids = (int)(cls[0].cfgs.size() + cls[1].cfgs.size());
  if (total == 0) {
    if (stats) *stats = st;
    return GM_OK;
  }
  // device buffers within the budget: inputs, outputs, start models, tables
  size_t need = 0;
  for (int c = 0; c < 2; ++c)
    need += sizeof(float) * cls[c].floats +
            (size_t)cls[c].pixels * (11 * 4 + 4 + 4 + 4 + 11 * 8 + 4 + 2 + 8) + sizeof(gm::DevCfg) * cls[c].cfgs.size();
  gm_status stt;
  for (int c = 0; c < 2; ++c) {
    BatchClass& k = cls[c];
    if (!k.pixels) continue;
    const std::string p = c ? "rg1_" : "rg0_";
    void* q = nullptr;
    const int64_t P = k.pixels;
    if ((stt = ensure_buf(ctx, p + "in", sizeof(float) * k.floats, &q)) != GM_OK) return stt;
    k.in = (float*)q;
    if ((stt = ensure_buf(ctx, p + "model", sizeof(float) * 11 * P, &q)) != GM_OK) return stt;
    k.model = (float*)q;
    if ((stt = ensure_buf(ctx, p + "chi2", sizeof(float) * P, &q)) != GM_OK) return stt;
    k.chi2 = (float*)q;
    if ((stt = ensure_buf(ctx, p + "iters", sizeof(int) * P, &q)) != GM_OK) return stt;
    k.iters = (int*)q;
    if ((stt = ensure_buf(ctx, p + "status", sizeof(uint32_t) * P, &q)) != GM_OK) return stt;
    k.status = (uint32_t*)q;
    if ((stt = ensure_buf(ctx, p + "cinit", sizeof(double) * 11 * P, &q)) != GM_OK) return stt;
    k.cinit = (double*)q;
    if ((stt = ensure_buf(ctx, p + "cstat", sizeof(uint32_t) * P, &q)) != GM_OK) return stt;
    k.cstat = (uint32_t*)q;
    if ((stt = ensure_buf(ctx, p + "cfgs", sizeof(gm::DevCfg) * k.cfgs.size(), &q)) != GM_OK) return stt;
    k.dcfgs = (gm::DevCfg*)q;
    if ((stt = ensure_buf(ctx, p + "grid", sizeof(uint16_t) * P, &q)) != GM_OK) return stt;
    k.grid = (uint16_t*)q;
    if ((stt = ensure_buf(ctx, p + "off", sizeof(uint64_t) * P, &q)) != GM_OK) return stt;
    k.off = (uint64_t*)q;
    gm::waves_mg_occupancy(k.cfgs[0], &k.bt, &k.ba);
    if (k.bt < 1 || k.ba < 1) return fail(ctx, GM_ERR_CUDA, "ragged-batch kernels cannot be resident");
  }
  for (int c = 0; c < 2; ++c) {
    BatchClass& k = cls[c];
    if (!k.pixels) continue;
    const int64_t chunk = wave_chunk_for(ctx, k.cfgs[0], need, k.pixels, 2);
    if (!chunk) return fail(ctx, GM_ERR_NOMEM, "the batch's wave state does not fit the HBM budget");
    if ((stt = wave_buffers(ctx, c ? "rg1_waves" : "rg0_waves", k.cfgs[0], chunk, &k.wb)) != GM_OK) return stt;
    key += "|" + std::to_string(chunk) + "@" + std::to_string((uintptr_t)k.wb.w.state) + "/" +
           std::to_string((uintptr_t)k.in);
  }
  // uploads: the profiles, the grids' configurations, the per-pixel tables
  cudaError_t e = cudaSuccess;
  for (int c = 0; c < 2 && e == cudaSuccess; ++c) {
    BatchClass& k = cls[c];
    if (!k.pixels) continue;
    std::vector<uint16_t> grid((size_t)k.pixels);
    std::vector<uint64_t> off((size_t)k.pixels);
    for (size_t j = 0; j < k.rois.size(); ++j) {
      const gm_roi& r = rois[k.rois[j]];
      int g = 0;
      const auto& gl = gfirst[c];
      while (!same_grid(*gl[g], r)) ++g;
      const uint64_t row = 4 * (uint64_t)r.nl;
      for (int64_t p = 0; p < r.npix; ++p) {
        grid[(size_t)(k.first[j] + p)] = (uint16_t)g;
        off[(size_t)(k.first[j] + p)] = k.in_off[j] + (uint64_t)p * row;
      }
      if (e == cudaSuccess && r.npix)
        e = cudaMemcpyAsync(k.in + k.in_off[j], r.iquv, sizeof(float) * row * r.npix, cudaMemcpyDefault, s);
    }
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(k.dcfgs, k.cfgs.data(), sizeof(gm::DevCfg) * k.cfgs.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(k.grid, grid.data(), sizeof(uint16_t) * grid.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(k.off, off.data(), sizeof(uint64_t) * off.size(), cudaMemcpyHostToDevice, s);
  }
  if (e != cudaSuccess) return cuda_fail(ctx, e, "ragged-batch upload");
  // layout change: forget the captured work and the tuning
  if (key != ctx->batch_key) {
    if (ctx->batch_exec) cudaGraphExecDestroy(ctx->batch_exec);
    ctx->batch_exec = nullptr;
    ctx->batch_key = key;
    ctx->batch_tuned = false;
    for (int c = 0; c < 2; ++c) {
      ctx->batch_cap[c][0] = cls[c].bt;
      ctx->batch_cap[c][1] = cls[c].ba;
    }
  }
  int launches = 0;
  float ms = 0.f;
  if (opts->autotune && !ctx->batch_tuned) {
    // candidates: full, trial kernel at 3/4, accept kernel at 3/4, both at 1/2
    const int frac[4][2] = {{4, 4}, {3, 4}, {4, 3}, {2, 2}};
    float best = -1.f;
    int bestc = 0;
    for (int t = 0; t < 4; ++t) {
      int cap[2][2];
      for (int c = 0; c < 2; ++c) {
        cap[c][0] = std::max(1, cls[c].bt * frac[t][0] / 4);
        cap[c][1] = std::max(1, cls[c].ba * frac[t][1] / 4);
      }
      launches = 0;
      e = cudaEventRecord(ctx->ev0, s);
      if (e == cudaSuccess) e = batch_device_work(ctx, cls, cap, s, &launches);
      if (e == cudaSuccess) e = cudaEventRecord(ctx->ev1, s);
      if (e == cudaSuccess) e = cudaEventSynchronize(ctx->ev1);
      if (e != cudaSuccess) return cuda_fail(ctx, e, "ragged-batch tuning");
      cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
      if (best < 0 || ms < best) {
        best = ms;
        bestc = t;
      }
    }
    for (int c = 0; c < 2; ++c) {
      ctx->batch_cap[c][0] = std::max(1, cls[c].bt * frac[bestc][0] / 4);
      ctx->batch_cap[c][1] = std::max(1, cls[c].ba * frac[bestc][1] / 4);
    }
    ctx->batch_tuned = true;
    if (ctx->batch_exec) cudaGraphExecDestroy(ctx->batch_exec);
    ctx->batch_exec = nullptr;
  }
  launches = 0;
  if (opts->use_graph) {
    if (!ctx->batch_exec) {
      cudaGraph_t g = nullptr;
      e = cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed);
      if (e == cudaSuccess) {
        const cudaError_t we = batch_device_work(ctx, cls, ctx->batch_cap, s, &launches);
        e = cudaStreamEndCapture(s, &g);
        if (we != cudaSuccess) e = we;
      }
      if (e == cudaSuccess) e = cudaGraphInstantiate(&ctx->batch_exec, g, 0);
      if (g) cudaGraphDestroy(g);
      if (e != cudaSuccess) {
        ctx->batch_exec = nullptr;
        return cuda_fail(ctx, e, "ragged-batch graph capture");
      }
    } else {
      st.graph_replayed = 1;
      for (int c = 0; c < 2; ++c)
        if (cls[c].pixels) {
          const int waves = 1 + (cls[c].cfgs[0].miter > 1 ? cls[c].cfgs[0].miter : 1);
          const int64_t ch = cls[c].wb.chunk;
          launches += (int)((cls[c].pixels + ch - 1) / ch) * (2 * waves - 1) + 1;
        }
    }
    e = cudaEventRecord(ctx->ev0, s);
    if (e == cudaSuccess) e = cudaGraphLaunch(ctx->batch_exec, s);
  } else {
    e = cudaEventRecord(ctx->ev0, s);
    if (e == cudaSuccess) e = batch_device_work(ctx, cls, ctx->batch_cap, s, &launches);
  }
  if (e == cudaSuccess) e = cudaEventRecord(ctx->ev1, s);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "ragged-batch launch");
  // outputs back into the callers' buffers
  for (int c = 0; c < 2 && e == cudaSuccess; ++c) {
    BatchClass& k = cls[c];
    for (size_t j = 0; j < k.rois.size() && e == cudaSuccess; ++j) {
      const gm_roi& r = rois[k.rois[j]];
      if (!r.npix) continue;
      const int64_t f = k.first[j];
      e = cudaMemcpyAsync(r.model, k.model + f * 11, sizeof(float) * 11 * r.npix, cudaMemcpyDefault, s);
      if (e == cudaSuccess && r.chi2)
        e = cudaMemcpyAsync(r.chi2, k.chi2 + f, sizeof(float) * r.npix, cudaMemcpyDefault, s);
      if (e == cudaSuccess && r.iters)
        e = cudaMemcpyAsync(r.iters, k.iters + f, sizeof(int) * r.npix, cudaMemcpyDefault, s);
      if (e == cudaSuccess && r.status)
        e = cudaMemcpyAsync(r.status, k.status + f, sizeof(uint32_t) * r.npix, cudaMemcpyDefault, s);
    }
  }
  cudaEventRecord(ctx->ev_scratch, s);
  ctx->scratch_pending = true;
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "ragged batch");
  cudaEventElapsedTime(&st.device_ms, ctx->ev0, ctx->ev1);
  // lane occupancy: samples over lane slots, weighted by each pixel's trials
  double samples = 0, slots = 0;
  for (int c = 0; c < 2; ++c) {
    BatchClass& k = cls[c];
    if (!k.pixels) continue;
    std::vector<int> it((size_t)k.pixels);
    if (cudaMemcpy(it.data(), k.iters, sizeof(int) * it.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
      return fail(ctx, GM_ERR_CUDA, "ragged-batch statistics");
    for (size_t j = 0; j < k.rois.size(); ++j) {
      const gm_roi& r = rois[k.rois[j]];
      double trials = 0;
      for (int64_t p = 0; p < r.npix; ++p) trials += it[(size_t)(k.first[j] + p)] + 1;
      samples += trials * r.nl;
      slots += trials * 32.0 * (c + 1);
    }
  }
  st.lane_occupancy = slots > 0 ? samples / slots : 0.0;
  st.launches = launches;
  st.cap_trial = ctx->batch_cap[cls[0].pixels ? 0 : 1][0];
  st.cap_accept = ctx->batch_cap[cls[0].pixels ? 0 : 1][1];
  ctx->stats.pixels = total;
  ctx->stats.kernel_launches = launches;
  ctx->stats.kernel_ms = st.device_ms;
  if (stats) *stats = st;
  return GM_OK;
}

// ---------------------------------------------------------------- learned initial guess
extern "C" {

gm_status gm_mlp_init(gm_mlp* net, int nl, uint64_t seed) {
  if (!net || nl < 1 || 4 * nl > GM_MLP_IN) return GM_ERR_INVALID;
  gm::mlp::init_net(net, nl, seed);
  return GM_OK;
}

void gm_mlp_train_defaults(gm_mlp_train_opts* o) {
  if (!o) return;
  o->epochs = 8;
  o->batch = 16384;
  o->lr = 2e-3f;
  o->weight_decay = 0.f;
  o->seed = 1;
}

}  // extern "C"

// Training and gradients: the data staged onto the device when they are in
// host memory, then the training driver on the context's stream.
static gm_status mlp_train_impl(gm_ctx* ctx, gm_mlp* net, const float* iquv, const double* truth, int64_t n,
                                const gm_mlp_train_opts* o, float* loss, gm_mlp* grads, bool grads_only) {
  if (!ctx || !net || !iquv || !truth || n <= 0) return ctx ? fail(ctx, GM_ERR_INVALID, "bad argument") : GM_ERR_INVALID;
  if (net->abi_version != GM_ABI_VERSION) return fail(ctx, GM_ERR_INVALID, "gm_mlp.abi_version mismatch");
  if (net->nl < 1 || 4 * net->nl > GM_MLP_IN) return fail(ctx, GM_ERR_INVALID, "the network's nl must be 1..32");
  std::lock_guard<std::mutex> lk(ctx->call_mu);
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  const int nl = net->nl;
  Arg a_in, a_t;
  gm_status st;
  if ((st = stage_in(ctx, "mlp_iquv", iquv, sizeof(float) * 4 * (size_t)nl * n, &a_in, s)) != GM_OK) return st;
  if ((st = stage_in(ctx, "mlp_truth", truth, sizeof(double) * 11 * (size_t)n, &a_t, s)) != GM_OK) return st;
  gm_mlp_train_opts def;
  gm_mlp_train_defaults(&def);
  if (!o) o = &def;
  gm::mlp::TrainArgs ta{};
  ta.iquv = (const float*)a_in.dev;
  ta.truth = (const double*)a_t.dev;
  ta.n = n;
  ta.nl = nl;
  ta.epochs = o->epochs;
  ta.batch = o->batch;
  ta.lr = o->lr;
  ta.weight_decay = o->weight_decay;
  ta.seed = o->seed;
  ta.grads_only = grads_only;
  cudaMemsetAsync(ctx->mlp_err, 0, sizeof(int), s);
  const char* why = nullptr;
  cudaError_t e = gm::mlp::train(net, ta, loss, grads, ctx->mlp_err, s, &why);
  if (e == cudaErrorInvalidValue && why) return fail(ctx, GM_ERR_INVALID, why);
  if (e != cudaSuccess) return cuda_fail(ctx, e, why ? why : "training");
  return GM_OK;
}

extern "C" {

gm_status gm_mlp_train(gm_ctx* ctx, gm_mlp* net, const float* iquv, const double* truth, int64_t n,
                       const gm_mlp_train_opts* opts, float* loss_per_epoch) {
  return mlp_train_impl(ctx, net, iquv, truth, n, opts, loss_per_epoch, nullptr, false);
}

gm_status gm_mlp_gradients(gm_ctx* ctx, const gm_mlp* net, const float* iquv, const double* truth, int64_t n,
                           gm_mlp* grads, float* loss) {
  if (!grads) return ctx ? fail(ctx, GM_ERR_INVALID, "grads is NULL") : GM_ERR_INVALID;
  gm_mlp copy = net ? *net : gm_mlp{};
  if (n % gm::mlp::kTile) return ctx ? fail(ctx, GM_ERR_INVALID, "n must be a multiple of 128") : GM_ERR_INVALID;
  gm_mlp_train_opts o;
  gm_mlp_train_defaults(&o);
  o.batch = (int)n;
  o.epochs = 1;
  float l = 0.f;
  gm_status st = mlp_train_impl(ctx, net ? &copy : nullptr, iquv, truth, n, &o, &l, grads, true);
  if (st == GM_OK && loss) *loss = l;
  return st;
}

gm_status gm_mlp_predict(gm_ctx* ctx, const gm_mlp* net, const float* iquv, int64_t n, double* models,
                         void* stream) {
  if (!ctx) return GM_ERR_INVALID;
  if (!net || !iquv || !models || n < 0) return fail(ctx, GM_ERR_INVALID, "bad argument");
  if (!ctx->configured) return fail(ctx, GM_ERR_NOT_CONFIGURED, "gm_configure first");
  if (net->abi_version != GM_ABI_VERSION) return fail(ctx, GM_ERR_INVALID, "gm_mlp.abi_version mismatch");
  if (net->nl != ctx->dev.nl || 4 * net->nl > GM_MLP_IN)
    return fail(ctx, GM_ERR_INVALID, "the network was made for another grid");
  if (n == 0) return GM_OK;
  std::lock_guard<std::mutex> lk(ctx->call_mu);
  cudaSetDevice(ctx->device);
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  const int nl = net->nl;
  Arg a_in, a_out;
  gm_status st;
  if ((st = stage_in(ctx, "iquv", iquv, sizeof(float) * 4 * (size_t)nl * n, &a_in, s)) != GM_OK) return st;
  if (reinterpret_cast<uintptr_t>(a_in.dev) & 15u)
    return fail(ctx, GM_ERR_INVALID, "device profiles must start on a 16-byte boundary");
  if ((st = stage_out(ctx, "pmodels", models, sizeof(double) * 11 * (size_t)n, &a_out)) != GM_OK) return st;
  gm::mlp::DevNet d;
  cudaError_t e = gm::mlp::devnet_create(&d, net, s);
  int fix[GM_NPAR];
  for (int i = 0; i < GM_NPAR; ++i) fix[i] = ctx->dev.fix[i];
  if (e == cudaSuccess) e = cudaMemsetAsync(ctx->mlp_err, 0, sizeof(int), s);
  if (e == cudaSuccess)
    e = gm::mlp::predict(d, (const float*)a_in.dev, n, nl, ctx->cfg.init_model, fix, (double*)a_out.dev,
                         ctx->mlp_err, s);
  if (e == cudaSuccess && (st = copy_back(ctx, a_out, s)) != GM_OK) {
    gm::mlp::devnet_destroy(&d);
    return st;
  }
  // the network's device copy is released with the call
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  gm::mlp::devnet_destroy(&d);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "learned initial guess");
  return learned_check(ctx);
}

}  // extern "C"

// ---------------------------------------------------------------- no-alloc inversion
// Scratch of gm_invert_noalloc: the work-stealing counters at offset 0 and the
// global stray-light profile [4][nl] at offset 256.  A file-scope device array
// of fixed size, resident on every device that loads the library.
static __device__ __align__(256) unsigned char g_noalloc_scratch[GM_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kNoallocMaxDevices = 64;
constexpr size_t kNoallocSlightOffset = 256;
std::mutex g_noalloc_mu;
void* g_noalloc_addr[kNoallocMaxDevices] = {};

// Device address of the scratch array on the current device.  The first call
// per device (with that device current) looks it up and loads every variant
// of the inversion kernel (grids of <= 32 and <= 64 samples; 10 terms, 10
// terms with macroturbulence, 11 terms), so later calls do neither.
gm_status noalloc_scratch(int dev, void** out) {
  if (dev < 0 || dev >= kNoallocMaxDevices) return GM_ERR_INVALID;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return GM_ERR_CUDA;
    }
    for (int nl : {32, 64}) {
      for (int v = 0; v < 3; ++v) {
        gm::DevCfg probe{};
        probe.nl = nl;
        probe.nterms = v == 2 ? 11 : 10;
        probe.init[gm::MAC] = v == 1 ? 1.0 : 0.0;
        if (gm::invert_geometry(probe, false).blocks_per_sm < 1) {
          cudaGetLastError();
          return GM_ERR_CUDA;
        }
      }
    }
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return GM_OK;
}

}  // namespace

extern "C" gm_status gm_invert_noalloc(const gm_config* cfg, const float* iquv, int64_t npix, int nl,
                                       float* model, float* chi2, int* iters, float* fitted,
                                       uint32_t* status, void* stream) {
  if (!cfg || !iquv || !model || npix < 0) return GM_ERR_INVALID;
  gm::DevCfg d;
  gm_status st = build_devcfg(nullptr, *cfg, &d);
  if (st != GM_OK) return st;
  if (nl != d.nl) return GM_ERR_INVALID;
  if (d.lambda_per_pixel || cfg->init_mode == GM_INIT_LEARNED) return GM_ERR_UNSUPPORTED;
  const bool global_slight = d.use_slight && !d.slight_per_pixel;
  const size_t need = kNoallocSlightOffset + (global_slight ? sizeof(float) * 4 * (size_t)nl : 0);
  if (need > GM_NOALLOC_SCRATCH_BYTES) return GM_ERR_INVALID;
  if (d.use_slight && !cfg->slight) return GM_ERR_INVALID;
  // every array the kernel touches must already be device memory
  const void* dev_ptrs[] = {iquv, model, chi2, iters, fitted, status,
                            (d.use_slight && d.slight_per_pixel) ? (const void*)cfg->slight : nullptr};
  for (const void* p : dev_ptrs)
    if (p && !is_device_ptr(p)) return GM_ERR_INVALID;
  if (npix == 0) return GM_OK;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return GM_ERR_CUDA;
  void* scratch = nullptr;
  if ((st = noalloc_scratch(dev, &scratch)) != GM_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  // the counters must start at zero; the array keeps the previous call's values
  cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(gm::WorkCounters), s);
  if (e == cudaSuccess && global_slight) {
    float* dst = (float*)((unsigned char*)scratch + kNoallocSlightOffset);
    e = cudaMemcpyAsync(dst, cfg->slight, sizeof(float) * 4 * nl, cudaMemcpyDefault, s);
    d.slight = dst;
  } else if (d.use_slight) {
    d.slight = cfg->slight;
  }
  if (e != cudaSuccess) return GM_ERR_CUDA;
  gm::InvertArgs ia{};
  ia.iquv = iquv;
  ia.npix = npix;
  ia.model = model;
  ia.chi2 = chi2;
  ia.iters = iters;
  ia.fitted = fitted;
  ia.status = status;
  ia.work = (gm::WorkCounters*)scratch;
  const int64_t grid = invert_grid(d, false, sms, npix, nullptr);
  e = gm::launch_invert(d, ia, (int)grid, s);
  return e == cudaSuccess ? GM_OK : GM_ERR_CUDA;
}
