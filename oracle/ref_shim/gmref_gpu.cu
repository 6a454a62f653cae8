// gmref_gpu.cu -- host harness of the reference's lm_mils kernel built for
// sm_100a (benchmark and test infrastructure, never the product).
//
// It replays what the reference's main does around the image inversion
// (gmilos.cu:1008-1249): the __constant__ configuration symbols
// (gmilos.cu:46-68, filled as at gmilos.cu:213-239, 532-547, 636-641), the
// launch geometry -- blocks per stream = lm_mils's occupancy per SM with 32
// threads per block, NSTREAMS streams, each thread given a contiguous slice
// of its stream's pixels -- the device heap for the per-thread scratch, and
// cudaEvent timing of the launches on the legacy default stream.
//
// Two deliberate differences, both about safety on a shared GPU:
//   - the heap is 4x the reference's 37568 B per thread, so that the
//     per-launch leak of one ProfilesMemory per thread (lm_mils never frees
//     it) cannot exhaust it over repeated runs;
//   - device malloc goes through gm_shim_device_malloc, which counts failed
//     allocations and returns a sink buffer instead of NULL.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "definesCuda.cuh"
#include "milosUtils.cuh"
#include "gmref.h"

// ---- the reference's configuration symbols (gmilos.cu:46-68)
__constant__ int d_fix_const[11];
__constant__ PRECISION d_lambda_const[MAX_LAMBDA];
__constant__ PRECISION d_psfFunction_const[MAX_LAMBDA];
__constant__ REAL d_weight_const[4];
__constant__ REAL d_weight_sigma_const[4];
__constant__ PRECISION d_wlines_const[2];
__constant__ Cuantic d_cuantic_const;
__constant__ Init_Model d_initModel_const;
__constant__ int d_nlambda_const;
__constant__ PRECISION d_toplim_const;
__constant__ int d_miter_const;
__constant__ REAL d_sigma_const;
__constant__ REAL d_ilambda_const;
__constant__ int d_use_convolution_const;
__constant__ REAL d_ah_const;
__constant__ int d_logclambda_const;
__constant__ cuDoubleComplex d_zdenV[7];
__constant__ cuDoubleComplex d_zdivV[7];
__constant__ int cordicPosFila[TAMANIO_SVD * TAMANIO_SVD];
__constant__ int cordicPosCol[TAMANIO_SVD * TAMANIO_SVD];
__constant__ PRECISION LIMITE_INFERIOR_PRECISION_SVD;
__constant__ PRECISION LIMITE_INFERIOR_PRECISION_TRIG;
__constant__ PRECISION LIMITE_INFERIOR_PRECISION_SINCOS;

// ---- device-heap guard
constexpr size_t kSinkBytes = 64 * 1024;
__device__ __align__(16) unsigned char g_shim_sink[kSinkBytes];
__device__ unsigned int g_shim_malloc_failures;

__device__ void* gm_shim_device_malloc(size_t n) {
  void* p = malloc(n);
  if (p) return p;
  atomicAdd(&g_shim_malloc_failures, 1u);
  return n <= kSinkBytes ? (void*)g_shim_sink : nullptr;
}

__device__ void gm_shim_device_free(void* p) {
  if (p && p != (void*)g_shim_sink) free(p);
}

namespace {

std::mutex g_mu;
constexpr int kThreadsPerBlock = 32;          // gmilos.cu:1014
constexpr size_t kRefHeapPerThread = 37568;   // gmilos.cu:1027
constexpr size_t kHeapFactor = 4;
const int kPerm[TAMANIO_SVD] = {0, 2, 4, 1, 6, 3, 8, 5, 9, 7};

#define GMREF_CHECK(call)                                                      \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      rep->cuda_error = (int)e_;                                               \
      snprintf(rep->msg, sizeof(rep->msg), "%s: %s", #call, cudaGetErrorString(e_)); \
      goto fail;                                                               \
    }                                                                          \
  } while (0)

int make_cuantic(const gmref_setup* s, Cuantic* out) {
  PRECISION dat[8] = {1, s->quantum[0], s->quantum[1], s->quantum[2],
                      s->quantum[3], s->quantum[4], s->quantum[5], 1};
  Cuantic* c = create_cuantic(dat, 0);
  if (!c) return -1;
  *out = c[0];
  free(c);
  return 0;
}

cudaError_t upload(const gmref_setup* s) {
  const int nl = s->nl;
  Cuantic cu;
  if (make_cuantic(s, &cu)) return cudaErrorInvalidValue;
  PRECISION lam[MAX_LAMBDA] = {0}, psf[MAX_LAMBDA] = {0};
  for (int i = 0; i < nl; ++i) { lam[i] = s->lambda[i]; psf[i] = s->psf[i]; }
  PRECISION wl[2] = {1, s->lambda0};
  REAL ws[4];
  for (int k = 0; k < 4; ++k) ws[k] = s->weight[k] / s->noise;
  Init_Model im;
  im.eta0 = s->init[0]; im.B = s->init[1]; im.vlos = s->init[2]; im.dopp = s->init[3];
  im.aa = s->init[4]; im.gm = s->init[5]; im.az = s->init[6]; im.S0 = s->init[7];
  im.S1 = s->init[8]; im.mac = s->init[9]; im.alfa = s->init[10];
  cuDoubleComplex zden[7], zdiv[7];
  for (int k = 0; k < 7; ++k) {
    zden[k] = make_cuDoubleComplex(a_fvoigt[6 - k], 0);
    zdiv[k] = make_cuDoubleComplex(b_fvoigt[6 - k], 0);
  }
  int fila[TAMANIO_SVD * TAMANIO_SVD], col[TAMANIO_SVD * TAMANIO_SVD];
  for (int r = 0; r < TAMANIO_SVD; ++r)
    for (int c = 0; c < TAMANIO_SVD; ++c) {
      fila[r * TAMANIO_SVD + c] = kPerm[r];
      col[r * TAMANIO_SVD + c] = kPerm[c];
    }
  const PRECISION lim = pow(2.0, -39);
  REAL noise = s->noise, il = s->ilambda, mu = s->mu;
  cudaError_t e = cudaSuccess;
#define UP(sym, ptr, bytes) \
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(sym, ptr, bytes)
  UP(d_lambda_const, lam, sizeof(lam));
  UP(d_psfFunction_const, psf, sizeof(psf));
  UP(d_wlines_const, wl, sizeof(wl));
  UP(d_weight_const, s->weight, sizeof(REAL) * 4);
  UP(d_weight_sigma_const, ws, sizeof(ws));
  UP(d_initModel_const, &im, sizeof(im));
  UP(d_cuantic_const, &cu, sizeof(cu));
  UP(d_fix_const, s->fix, sizeof(int) * 11);
  UP(d_nlambda_const, &nl, sizeof(int));
  UP(d_toplim_const, &s->toplim, sizeof(PRECISION));
  UP(d_miter_const, &s->miter, sizeof(int));
  UP(d_sigma_const, &noise, sizeof(REAL));
  UP(d_ilambda_const, &il, sizeof(REAL));
  UP(d_use_convolution_const, &s->use_psf, sizeof(int));
  UP(d_ah_const, &mu, sizeof(REAL));
  UP(d_logclambda_const, &s->logclambda, sizeof(int));
  UP(d_zdenV, zden, sizeof(zden));
  UP(d_zdivV, zdiv, sizeof(zdiv));
  UP(cordicPosFila, fila, sizeof(fila));
  UP(cordicPosCol, col, sizeof(col));
  UP(LIMITE_INFERIOR_PRECISION_SVD, &lim, sizeof(lim));
  UP(LIMITE_INFERIOR_PRECISION_TRIG, &lim, sizeof(lim));
  UP(LIMITE_INFERIOR_PRECISION_SINCOS, &lim, sizeof(lim));
#undef UP
  return e;
}

}  // namespace

extern "C" int gmref_gpu_invert(const gmref_setup* s, const float* iquv, long long npix,
                                const float* slight, int slight_per_pixel, int nstreams,
                                double* model, float* chi2, int* iters, float* fitted,
                                gmref_gpu_report* rep) {
  std::lock_guard<std::mutex> lock(g_mu);
  gmref_gpu_report dummy;
  if (!rep) rep = &dummy;
  memset(rep, 0, sizeof(*rep));
  if (!s || s->nl < 2 || s->nl > MAX_LAMBDA || npix <= 0 || nstreams <= 0 || nstreams > 64 ||
      !iquv || !model || !chi2 || !iters) {
    snprintf(rep->msg, sizeof(rep->msg), "invalid argument");
    return -1;
  }
  const int nl = s->nl;
  const long long per_pix = 4LL * nl;
  if (per_pix * npix > 0x7fffffffLL) {  // the reference indexes with int
    snprintf(rep->msg, sizeof(rep->msg), "cube too large for int offsets");
    return -1;
  }
  const int P = (int)npix;

  float *d_spectro = nullptr, *d_fit = nullptr, *d_chi2 = nullptr, *d_slight = nullptr;
  Init_Model* d_models = nullptr;
  int *d_iter = nullptr, *d_displs_spectro = nullptr, *d_counts = nullptr, *d_displs_pix = nullptr;
  std::vector<cudaStream_t> streams;
  cudaEvent_t e0 = nullptr, e1 = nullptr, start = nullptr, stop = nullptr;
  std::vector<Init_Model> h_models;
  int num_blocks = 0, nrte = 0, map_slight = 0, rc = -1;
  bool use11 = false;
  const void* kern = nullptr;
  size_t heap_need = 0, heap_now = 0, stack_now = 0;
  unsigned zero = 0, failures = 0;
  cudaFuncAttributes attr;
  std::vector<int> counts, displs_pix, displs_spectro;
  const size_t cube_bytes = sizeof(float) * (size_t)per_pix * P;

  GMREF_CHECK(upload(s));
  use11 = s->fix[9] && s->fix[10];   // gmilos.cu:1016-1021
  kern = use11 ? (const void*)lm_mils_11 : (const void*)lm_mils;
  GMREF_CHECK(cudaFuncGetAttributes(&attr, kern));
  GMREF_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&num_blocks, kern, kThreadsPerBlock, 0));
  nrte = num_blocks * kThreadsPerBlock;
  rep->num_blocks = num_blocks;
  rep->threads_per_block = kThreadsPerBlock;
  rep->n_rte_parallel = nrte;
  rep->nstreams = nstreams;
  rep->local_bytes = attr.localSizeBytes;
  rep->regs = attr.numRegs;

  // device heap for the per-thread scratch (gmilos.cu:1024-1028)
  heap_need = kHeapFactor * kRefHeapPerThread * (size_t)nrte * (size_t)nstreams;
  GMREF_CHECK(cudaDeviceGetLimit(&heap_now, cudaLimitMallocHeapSize));
  if (heap_now < heap_need) {
    cudaError_t e = cudaDeviceSetLimit(cudaLimitMallocHeapSize, heap_need);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      snprintf(rep->msg, sizeof(rep->msg), "device heap is %zu B, need %zu B: %s", heap_now,
               heap_need, cudaGetErrorString(e));
      goto fail;
    }
    GMREF_CHECK(cudaDeviceGetLimit(&heap_now, cudaLimitMallocHeapSize));
  }
  rep->heap_bytes = heap_now;
  // per-thread stack: the kernel's own frame (static, no recursion) plus margin
  GMREF_CHECK(cudaDeviceGetLimit(&stack_now, cudaLimitStackSize));
  if (stack_now < attr.localSizeBytes + 4096) {
    GMREF_CHECK(cudaDeviceSetLimit(cudaLimitStackSize, attr.localSizeBytes + 4096));
    GMREF_CHECK(cudaDeviceGetLimit(&stack_now, cudaLimitStackSize));
  }
  rep->stack_bytes = stack_now;

  // pixel slices per stream and per thread (gmilos.cu:1036-1094)
  counts.assign((size_t)nstreams * nrte, 0);
  displs_pix.assign(counts.size(), 0);
  displs_spectro.assign(counts.size(), 0);
  {
    std::vector<int> per_stream(nstreams);
    int q = P / nstreams, r = P % nstreams;
    for (int i = 0; i < nstreams; ++i) per_stream[i] = q + (i < r ? 1 : 0);
    long long sum = 0, sum_sp = 0;
    for (int j = 0; j < nstreams; ++j) {
      int qq = per_stream[j] / nrte, rr = per_stream[j] % nrte;
      for (int i = 0; i < nrte; ++i) {
        const int k = j * nrte + i;
        counts[k] = qq + (i < rr ? 1 : 0);
        displs_pix[k] = (int)sum;
        displs_spectro[k] = (int)sum_sp;
        sum += counts[k];
        sum_sp += (long long)counts[k] * per_pix;
      }
    }
  }

  GMREF_CHECK(cudaMalloc(&d_spectro, cube_bytes));
  GMREF_CHECK(cudaMalloc(&d_fit, cube_bytes));
  GMREF_CHECK(cudaMalloc(&d_models, sizeof(Init_Model) * P));
  GMREF_CHECK(cudaMalloc(&d_chi2, sizeof(float) * P));
  GMREF_CHECK(cudaMalloc(&d_iter, sizeof(int) * P));
  GMREF_CHECK(cudaMalloc(&d_displs_spectro, sizeof(int) * counts.size()));
  GMREF_CHECK(cudaMalloc(&d_counts, sizeof(int) * counts.size()));
  GMREF_CHECK(cudaMalloc(&d_displs_pix, sizeof(int) * counts.size()));
  if (slight) {
    map_slight = slight_per_pixel ? 1 : 0;
    const size_t sb = sizeof(float) * (size_t)per_pix * (map_slight ? P : 1);
    GMREF_CHECK(cudaMalloc(&d_slight, sb));
    GMREF_CHECK(cudaMemcpy(d_slight, slight, sb, cudaMemcpyHostToDevice));
  }
  streams.assign(nstreams, nullptr);
  for (int i = 0; i < nstreams; ++i) GMREF_CHECK(cudaStreamCreate(&streams[i]));
  GMREF_CHECK(cudaEventCreate(&e0));
  GMREF_CHECK(cudaEventCreate(&e1));
  GMREF_CHECK(cudaEventCreate(&start));
  GMREF_CHECK(cudaEventCreate(&stop));
  GMREF_CHECK(cudaMemcpyToSymbol(g_shim_malloc_failures, &zero, sizeof(zero)));
  GMREF_CHECK(cudaDeviceSynchronize());

  GMREF_CHECK(cudaEventRecord(e0, 0));
  GMREF_CHECK(cudaMemcpy(d_spectro, iquv, cube_bytes, cudaMemcpyHostToDevice));
  GMREF_CHECK(cudaMemcpy(d_displs_spectro, displs_spectro.data(), sizeof(int) * counts.size(),
                         cudaMemcpyHostToDevice));
  GMREF_CHECK(cudaMemcpy(d_counts, counts.data(), sizeof(int) * counts.size(),
                         cudaMemcpyHostToDevice));
  GMREF_CHECK(cudaMemcpy(d_displs_pix, displs_pix.data(), sizeof(int) * counts.size(),
                         cudaMemcpyHostToDevice));
  GMREF_CHECK(cudaEventRecord(start, 0));
  for (int i = 0; i < nstreams; ++i) {
    if (use11)
      lm_mils_11<<<num_blocks, kThreadsPerBlock, 0, streams[i]>>>(
          d_spectro, d_models, d_chi2, d_slight, d_iter, d_fit, d_displs_spectro, d_counts,
          d_displs_pix, nrte, i, map_slight);
    else
      lm_mils<<<num_blocks, kThreadsPerBlock, 0, streams[i]>>>(
          d_spectro, d_models, d_chi2, d_slight, d_iter, d_fit, d_displs_spectro, d_counts,
          d_displs_pix, nrte, i, map_slight);
  }
  GMREF_CHECK(cudaGetLastError());
  GMREF_CHECK(cudaEventRecord(stop, 0));
  GMREF_CHECK(cudaEventSynchronize(stop));
  h_models.resize(P);
  if (fitted) GMREF_CHECK(cudaMemcpy(fitted, d_fit, cube_bytes, cudaMemcpyDeviceToHost));
  GMREF_CHECK(cudaMemcpy(h_models.data(), d_models, sizeof(Init_Model) * P,
                         cudaMemcpyDeviceToHost));
  GMREF_CHECK(cudaMemcpy(iters, d_iter, sizeof(int) * P, cudaMemcpyDeviceToHost));
  GMREF_CHECK(cudaMemcpy(chi2, d_chi2, sizeof(float) * P, cudaMemcpyDeviceToHost));
  GMREF_CHECK(cudaEventRecord(e1, 0));
  GMREF_CHECK(cudaEventSynchronize(e1));
  GMREF_CHECK(cudaEventElapsedTime(&rep->kernel_ms, start, stop));
  GMREF_CHECK(cudaEventElapsedTime(&rep->e2e_ms, e0, e1));
  GMREF_CHECK(cudaMemcpyFromSymbol(&failures, g_shim_malloc_failures, sizeof(failures)));
  rep->malloc_failures = failures;
  for (int p = 0; p < P; ++p) {
    const Init_Model& m = h_models[p];
    double* o = model + (size_t)p * 11;
    o[0] = m.eta0; o[1] = m.B; o[2] = m.vlos; o[3] = m.dopp; o[4] = m.aa; o[5] = m.gm;
    o[6] = m.az; o[7] = m.S0; o[8] = m.S1; o[9] = m.mac; o[10] = m.alfa;
  }
  rc = failures ? -2 : 0;
  if (failures) snprintf(rep->msg, sizeof(rep->msg), "%u device-heap allocations failed", failures);

fail:
  for (cudaStream_t st : streams)
    if (st) cudaStreamDestroy(st);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (start) cudaEventDestroy(start);
  if (stop) cudaEventDestroy(stop);
  cudaFree(d_spectro);
  cudaFree(d_fit);
  cudaFree(d_models);
  cudaFree(d_chi2);
  cudaFree(d_iter);
  cudaFree(d_displs_spectro);
  cudaFree(d_counts);
  cudaFree(d_displs_pix);
  cudaFree(d_slight);
  return rc;
}
