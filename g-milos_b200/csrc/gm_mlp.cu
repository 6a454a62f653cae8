// gm_mlp.cu -- the learned initial guess on the fifth-generation tensor
// cores: inference and training kernels and their host-side drivers.
//
// Every product is D[128 x N] = A[128 x K] B[N x K]^T with A and B in BF16,
// D in FP32 tensor memory: tcgen05.mma (kind::f16, one CTA, M = 128) issued
// by one thread, its operands in shared memory in the 128-byte-swizzled
// layout that TMA writes (rows of 64 BF16 elements; a K-major atom is 128
// rows x 128 bytes), completion signalled through an mbarrier by
// tcgen05.commit, the accumulator read back with tcgen05.ld (thread t of
// warp w reads row 32 w + t).  Weights come from BF16 copies in global
// memory (L2 resident) by 2-D TMA loads into a two-stage ring, so the load
// of the next weight block overlaps the current product and epilogue.
// Activations are written into the operand tile by the epilogue threads
// themselves (the swizzle computed in place), so a tile's three layers run
// back to back without leaving the SM.  Inference keeps two tiles in
// flight per CTA, a producer warp issuing one tile's products while eight
// epilogue warps work on the other's accumulator.
//
// Training runs per batch: (1) one fused kernel per 128-pixel tile for the
// forward pass, the loss, and the backward pass through the activations
// (dH2 = dOut W3, dZ2 = dH2 * GELU'(Z2), dH1 = dZ2 W2, dZ1 = dH1 * GELU'(Z1)),
// whose operands and gradients it stores row-major (TMA stores of the
// operand tiles) for (2) the weight-gradient kernel, dW = G^T A over the
// batch, with both operands MN-major; (3) the bias gradients; (4) Adam on the
// FP32 parameters, which also rewrites the BF16 copies.
//
// Waits are bounded: a wait that runs past 2 s sets an error flag that the
// host reads, and the kernel then stops issuing work, waits (bounded) for
// its copies in flight, frees its tensor memory and returns.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include "gm_mlp.cuh"

namespace gm {
namespace mlp {
namespace {

// Inference and training kernels: 8 epilogue warps, two per tensor-memory
// lane quarter -- warp w reads rows 32 (w % 4) .. + 31 of the accumulator,
// and the two warpgroups split each epilogue's columns (and the input
// features) in halves; inference adds a producer warp.  The weight-gradient
// kernel: 4 warps, one row each.
constexpr int kThreads = 256;
constexpr int kWThreads = 128;
constexpr uint64_t kWaitNs = 2000000000ull;   // a wait gives up after 2 s

// error codes written to the kernel's error word
enum : int { kErrNone = 0, kErrWaitLoad = 1, kErrWaitMma = 2, kErrWaitStage = 3 };

// ---------------------------------------------------------------- PTX wrappers
__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t now_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(saddr(b)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait for the phase of barrier b with the given parity.  Returns false when
// it gave up: after kWaitNs (it then records `code` in *err and raises the
// block's abort flag) or as soon as another thread has raised the flag.
__device__ __noinline__ bool mbar_wait_slow(uint64_t* b, uint32_t parity, volatile int* abort, int* err, int code,
                                            bool stop_on_abort) {
  const uint64_t t0 = now_ns();
  while (!mbar_test(b, parity)) {
    if (stop_on_abort && *abort) return false;
    if (now_ns() - t0 > kWaitNs) {
      *abort = 1;
      atomicCAS(err, kErrNone, code);
      return false;
    }
  }
  return true;
}
// The phase is usually complete by the time a thread asks (a weight block
// loaded during the previous products, the products during the epilogue):
// one test inline, the bounded loop out of line.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, volatile int* abort, int* err, int code,
                                          bool stop_on_abort = true) {
  if (mbar_test(b, parity)) return true;
  return mbar_wait_slow(b, parity, abort, err, code, stop_on_abort);
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 2-D TMA: box at (x = inner coordinate, y = row) into / out of shared memory
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          dst),
      "l"(map), "r"(x), "r"(y), "r"(saddr(bar))
      : "memory");
}
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, int x, int y, uint32_t src) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(map), "r"(x),
               "r"(y), "r"(src)
               : "memory");
}
__device__ __forceinline__ void tma_store_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void tma_store_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void tma_store_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// tensor memory: allocation by one warp, fences around thread syncs
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(dst)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor of a 128-byte-swizzled operand.  K-major:
// 8-row groups 1024 bytes apart (SBO); MN-major: 8-row (K) groups SBO apart
// and 64-element MN blocks LBO apart.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;   // descriptor version of this architecture
  d |= (uint64_t)2 << 61;   // 128-byte swizzle
  return d;
}
// Instruction descriptor: BF16 x BF16 -> FP32, M x N, K-major (0) or
// MN-major (1) operands.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
      "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
               : "memory");
}
// 32 columns of this warp's 32 lanes: the load is asynchronous; its
// registers are valid after tmem_wait32 on the same array, whose asm takes
// them as operands so that no read of them is placed before the wait.
__device__ __forceinline__ void tmem_issue32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait32(uint32_t (&r)[32]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                 "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                 "+r"(r[15]), "+r"(r[16]), "+r"(r[17]), "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]),
                 "+r"(r[22]), "+r"(r[23]), "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]),
                 "+r"(r[29]), "+r"(r[30]), "+r"(r[31])
               :
               : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  tmem_issue32(taddr, r);
  tmem_wait32(r);
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                 "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                 "+r"(r[15])
               :
               : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&h);
}

// 16-byte chunk j (elements 8j..8j+7 of its 64-element row) of row r of the
// K-major swizzled atom at `atom` (shared-memory address).
__device__ __forceinline__ void st_chunk(uint32_t atom, int r, int j, const uint32_t (&w)[4]) {
  const uint32_t a = atom + (uint32_t)((r >> 3) * 1024 + (r & 7) * 128 + ((j ^ (r & 7)) << 4));
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(a), "r"(w[0]), "r"(w[1]), "r"(w[2]), "r"(w[3])
               : "memory");
}

// GELU in its tanh form (Hendrycks & Gimpel, 2016): z (1 + tanh u) / 2 with
// u = sqrt(2 / pi) (z + 0.044715 z^3), written as z s, s = 1 / (1 + exp(-2 u))
// -- one exponential and one reciprocal on the special-function unit -- and
// its derivative s + z s (1 - s) d(2u)/dz.
__device__ __forceinline__ float gelu_s(float z, float* du2) {
  const float z2 = z * z;
  const float u2 = 1.5957691216057308f * z * (1.f + 0.044715f * z2);
  if (du2) *du2 = 1.5957691216057308f * (1.f + 0.134145f * z2);
  // exp(80) keeps the denominator inside the fast reciprocal's range
  return __fdividef(1.f, 1.f + __expf(fminf(-u2, 80.f)));
}
__device__ __forceinline__ float gelu(float z) { return z * gelu_s(z, nullptr); }
__device__ __forceinline__ float gelu_grad(float z) {
  float du2;
  const float s = gelu_s(z, &du2);
  return s + z * s * (1.f - s) * du2;
}


// ---------------------------------------------------------------- kernel layout
// Shared memory (offsets from a 1024-byte aligned base).
constexpr uint32_t kSA = 0;            // activation operand: 4 K-atoms x [128 rows x 128 B]
constexpr uint32_t kSW = 65536;        // weight ring: 2 stages x 64 KB
constexpr uint32_t kStage = 65536;
constexpr uint32_t kSD = 196608;       // output-gradient operand: 1 atom [128 x 64]
constexpr uint32_t kSBar = 212992;     // barriers, tensor-memory address, abort flag
constexpr uint32_t kSPar = kSBar + 128; // b1, b2, in_mean, in_scale (floats), read by every tile
constexpr int kParFloats = 256 + 256 + 128 + 128;
constexpr size_t kSmemBytes = kSPar + 4 * kParFloats + 1024;

struct NetMaps {
  CUtensorMap m[5];                    // w1b, w2b, w3b, w2tb, w3tb
};
enum { kMapW1 = 0, kMapW2, kMapW3, kMapW2t, kMapW3t };

// One weight block of a layer: `natoms` K-atoms (64 K each) of a weight copy
// with `rows` rows (N), multiplied with A-operand atoms a_first.. (of the
// activation tile, or of the output-gradient tile when a_sd), into tensor
// columns tcol.., accumulating onto what is there when acc, ending its layer
// (the epilogue waits for it) when end.  The weight block's K offset is
// that of its A atoms.
struct Job {
  uint8_t map, natoms, a_first, a_sd;
  uint16_t rows, tcol;
  uint8_t acc, end;
};
constexpr int kInferJobs = 4, kTrainJobs = 7;
__constant__ Job c_jobs[kTrainJobs] = {
    {kMapW1, 2, 0, 0, 256, 0, 0, 1},      // Z1 = X W1^T
    {kMapW2, 2, 0, 0, 256, 256, 0, 0},    // Z2 = H1 W2^T (K 0..127); column 0 in inference
    {kMapW2, 2, 2, 0, 256, 256, 1, 1},    //            (K 128..255)
    {kMapW3, 4, 0, 0, 16, 0, 0, 1},       // out = H2 W3^T
    {kMapW3t, 1, 0, 1, 256, 0, 0, 1},     // dH2 = dOut W3
    {kMapW2t, 2, 0, 0, 256, 256, 0, 0},   // dH1 = dZ2 W2 (K 0..127)
    {kMapW2t, 2, 2, 0, 256, 256, 1, 1},   //            (K 128..255)
};
// weight blocks of layer L: [first, last)
__device__ __forceinline__ int layer_first(int L, bool train) {
  return L == 0 ? 0 : (L == 1 ? 1 : (train ? L + 1 : 3));
}
__device__ __forceinline__ int layer_last(int L, bool train) {
  return L == 0 ? 1 : (L == 1 ? 3 : (L == 4 ? 7 : (train ? L + 2 : 4)));
}

struct Bars {
  uint64_t full[2], empty[2], mma;
  uint32_t tmem;
  int abort;
};

// Producer (thread 0): the TMA loads of one weight block into a stage.
__device__ __forceinline__ void load_job(const Job& j, const NetMaps& nm, uint32_t stage, uint64_t* full) {
  const uint32_t atom = (uint32_t)j.rows * 128u;
  mbar_expect_tx(full, atom * j.natoms);
  for (int a = 0; a < j.natoms; ++a) tma_load_2d(stage + a * atom, &nm.m[j.map], 64 * (j.a_first + a), 0, full);
}

// Issuer (thread 0): the products of one weight block, K in steps of 16
// (32 bytes along a swizzled 128-byte row).
__device__ __forceinline__ void mma_job(const Job& j, uint32_t tmem, uint32_t tcol, uint32_t sA, uint32_t sD,
                                        uint32_t stage) {
  const uint32_t idesc = idesc_bf16(128, j.rows, 0, 0);
  const uint32_t abase = j.a_sd ? sD : sA + j.a_first * 16384u;
  const uint32_t batom = (uint32_t)j.rows * 128u;
  for (int k = 0; k < j.natoms * 4; ++k) {
    const int a = k >> 2, kk = k & 3;
    const uint64_t ad = sw128_desc(abase + a * 16384u + kk * 32u, 16, 1024);
    const uint64_t bd = sw128_desc(stage + a * batom + kk * 32u, 16, 1024);
    mma_bf16(tmem + tcol, ad, bd, idesc, (k > 0 || j.acc) ? 1u : 0u);
  }
}

// Producer / issuer state (thread 0), and the epilogue barrier's parity
// (all threads).
struct Pipe {
  uint32_t fph[2] = {0, 0}, eph[2] = {0, 0};   // next parity to wait for
  bool pend[2] = {false, false};                // a commit on empty[s] not yet waited for
  bool inflight[2] = {false, false};            // a load into stage s not yet waited for
  uint32_t mph = 0;
  int g = 0;                                    // weight blocks issued so far
};

__device__ __forceinline__ void start_load(const Job& j, const NetMaps& nm, Bars* B, uint32_t base, int s,
                                           Pipe& p) {
  load_job(j, nm, base + kSW + s * kStage, &B->full[s]);
  p.inflight[s] = true;
}

// Thread 0: run weight block `j`: wait for its weights, issue its products,
// signal the stage free and (layer end) the epilogue, then start loading
// `next` into the other stage once the products that last read it are done.
// Returns false on abort.
__device__ bool run_job(const Job& j, const Job* next, bool train, const NetMaps& nm, Bars* B, uint32_t base,
                        Pipe& p, int* err) {
  const int s = p.g & 1;
  const uint32_t stage = base + kSW + s * kStage;
  if (!mbar_wait(&B->full[s], p.fph[s], &B->abort, err, kErrWaitLoad)) return false;
  p.fph[s] ^= 1u;
  p.inflight[s] = false;
  tc_fence_after();
  const uint32_t tcol = (train || j.tcol < 256) ? j.tcol : 0u;
  mma_job(j, B->tmem, tcol, base + kSA, base + kSD, stage);
  mma_commit(&B->empty[s]);
  p.pend[s] = true;
  if (j.end) mma_commit(&B->mma);
  ++p.g;
  if (next) {
    const int o = s ^ 1;
    if (p.pend[o]) {
      if (!mbar_wait(&B->empty[o], p.eph[o], &B->abort, err, kErrWaitStage)) return false;
      p.eph[o] ^= 1u;
      p.pend[o] = false;
    }
    start_load(*next, nm, B, base, o, p);
  }
  return true;
}

// Load a tile's inputs (batch rows row0.., pixel idx[row] or the row itself)
// standardised and rounded to BF16 into the activation atoms 0-1; this
// thread's row r, features [64 half, 64 half + 64) (atom `half`).  Rows of
// 4 nl floats start on 16-byte boundaries and the feature count is a
// multiple of 4, so every 4-feature group is read whole or not at all.
__device__ __forceinline__ void load_x(const float* spar, const float* __restrict__ iquv,
                                       const uint32_t* __restrict__ idx, int64_t row0, int64_t n, int nl,
                                       uint32_t sA, int r, int half) {
  const int64_t b = row0 + r;
  const int F = 4 * nl;
  const float4* src = nullptr;
  if (b < n) src = reinterpret_cast<const float4*>(iquv + (idx ? (int64_t)idx[b] : b) * F);
  const float4* mean = reinterpret_cast<const float4*>(spar + 512);
  const float4* scale = reinterpret_cast<const float4*>(spar + 640);
#pragma unroll 2
  for (int c = 8 * half; c < 8 * half + 8; ++c) {
    float v[8];
#pragma unroll
    for (int g = 0; g < 2; ++g) {
      const int f4 = 2 * c + g;   // 4-feature group
      float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
      if (src && 4 * f4 < F) {
        const float4 xi = __ldg(src + f4), mu = mean[f4], sc = scale[f4];
        x = make_float4((xi.x - mu.x) * sc.x, (xi.y - mu.y) * sc.y, (xi.z - mu.z) * sc.z, (xi.w - mu.w) * sc.w);
      }
      v[4 * g] = x.x;
      v[4 * g + 1] = x.y;
      v[4 * g + 2] = x.z;
      v[4 * g + 3] = x.w;
    }
    const uint32_t w[4] = {pack_bf16(v[0], v[1]), pack_bf16(v[2], v[3]), pack_bf16(v[4], v[5]),
                           pack_bf16(v[6], v[7])};
    st_chunk(sA + (c >> 3) * 16384u, r, c & 7, w);
  }
}

// Epilogue of a hidden layer over the accumulator at tensor column zcol:
// h = GELU(z + bias) into the activation atoms (K = feature); with zspill,
// z + bias also to zspill[0..256) (this row).  This thread: row r, columns
// [128 half, 128 half + 128) (atoms 2 half, 2 half + 1), 32 at a time, the
// next 32 columns' tensor-memory load in flight while these are processed.
// bias: 256 floats in shared memory.
__device__ __forceinline__ void hidden_chunk(const uint32_t (&zr)[32], int q, const float* bias, uint32_t sA,
                                             int r, float* zspill) {
  float z[32];
  const float4* b4 = reinterpret_cast<const float4*>(bias + 32 * q);
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const float4 bv = b4[u];
    z[4 * u] = __uint_as_float(zr[4 * u]) + bv.x;
    z[4 * u + 1] = __uint_as_float(zr[4 * u + 1]) + bv.y;
    z[4 * u + 2] = __uint_as_float(zr[4 * u + 2]) + bv.z;
    z[4 * u + 3] = __uint_as_float(zr[4 * u + 3]) + bv.w;
  }
  if (zspill) {
    float4* dst = reinterpret_cast<float4*>(zspill + 32 * q);
#pragma unroll
    for (int u = 0; u < 8; ++u) dst[u] = make_float4(z[4 * u], z[4 * u + 1], z[4 * u + 2], z[4 * u + 3]);
  }
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    uint32_t w[4];
#pragma unroll
    for (int h = 0; h < 4; ++h) w[h] = pack_bf16(gelu(z[8 * u + 2 * h]), gelu(z[8 * u + 2 * h + 1]));
    st_chunk(sA + (q >> 1) * 16384u, r, (q & 1) * 4 + u, w);
  }
}

__device__ __forceinline__ void hidden_epilogue(uint32_t tmem_row, uint32_t zcol, const float* bias, uint32_t sA,
                                                int r, int half, float* zspill) {
  const int q0 = 4 * half;
  const uint32_t t0 = tmem_row + zcol + 32 * q0;
  uint32_t za[32], zb[32];
  tmem_issue32(t0, za);
#pragma unroll
  for (int j = 0; j < 4; j += 2) {
    tmem_wait32(za);
    tmem_issue32(t0 + 32 * (j + 1), zb);
    hidden_chunk(za, q0 + j, bias, sA, r, zspill);
    tmem_wait32(zb);
    if (j + 2 < 4) tmem_issue32(t0 + 32 * (j + 2), za);
    hidden_chunk(zb, q0 + j + 1, bias, sA, r, zspill);
  }
}

// The parameters every tile reads (b1, b2, in_mean, in_scale) into the
// shared-memory block at spar, once per launch.
__device__ __forceinline__ void stage_params(const gm_mlp* __restrict__ P, float* spar) {
  for (int i = threadIdx.x; i < kParFloats; i += blockDim.x)
    spar[i] = i < 256 ? P->b1[i] : (i < 512 ? P->b2[i - 256] : (i < 640 ? P->in_mean[i - 512] : P->in_scale[i - 640]));
}

// Outputs (de-standardised) -> start model (Init_Model layout) within the
// reference's ranges (check, milosUtils.cu:160-238); fixed parameters and
// v_mac / filling factor from the guess model.
__device__ __forceinline__ void outputs_to_model(const float (&y)[kOut], const double* guess, const int* fix,
                                                 double* m) {
  const double bl = y[6], bq = y[7], bu = y[8];
  const double bt = sqrt(bq * bq + bu * bu);
  const double B = sqrt(bl * bl + bt * bt);
  const double gam = atan2(bt, bl) * (180.0 / 3.14159265358979323846);
  double phi = 0.5 * atan2(bu, bq) * (180.0 / 3.14159265358979323846);
  if (phi < 0) phi += 180.0;
  double v[11];
  v[0] = fmin(fmax((double)y[0], 1.0), 2500.0);
  v[1] = fmin(B, 5000.0);
  v[2] = fmin(fmax((double)y[1], -20.0), 20.0);
  v[3] = fmin(fmax((double)y[2], 1e-4), 0.6);
  v[4] = fmin(fmax((double)y[3], 1e-4), 10.0);
  v[5] = gam;
  v[6] = phi;
  v[7] = fmin(fmax((double)y[4], 1e-4), 2.0);
  v[8] = fmin(fmax((double)y[5], 1e-4), 2.0);
  v[9] = guess[9];
  v[10] = guess[10];
#pragma unroll
  for (int i = 0; i < 11; ++i) m[i] = (i < 9 && fix[i] && isfinite(v[i])) ? v[i] : guess[i];
}

struct InferArgs {
  const gm_mlp* p;
  const float* iquv;
  int64_t n;
  int nl;
  double guess[11];
  int fix[11];
  double* models;
  int* err;
};

struct TrainKArgs {
  const gm_mlp* p;
  const float* iquv;
  const float* y16;        // [pixels][16] standardised targets
  const uint32_t* idx;     // batch row -> pixel
  int64_t n;               // rows of this batch (a multiple of 128)
  int nl;
  float gscale;            // d loss / d output per unit of error: 2 / (rows x 9)
  float* zspill;           // [rows][256] pre-activations of layer 1
  float* loss;             // sum of squared errors (atomic)
  int* err;
};

struct ActMaps {
  // row-major BF16 [rows][128 | 256 | 256 | 64 | 256 | 256], boxes of 64 x 128
  CUtensorMap x, h1, h2, g3, g2, g1;
};

__device__ __forceinline__ void setup(Bars* B, uint32_t ncols) {
  const int tid = threadIdx.x;
  if (tid == 0) {
    mbar_init(&B->full[0], 1);
    mbar_init(&B->full[1], 1);
    mbar_init(&B->empty[0], 1);
    mbar_init(&B->empty[1], 1);
    mbar_init(&B->mma, 1);
    B->abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if ((tid >> 5) == 0) tmem_alloc(&B->tmem, ncols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
}

// End of a kernel (every thread): thread 0 waits, bounded, for the weight
// loads still in flight (there are none unless the kernel aborted), for its
// products (a last commit) and for its stores; then the tensor memory is
// freed.
__device__ __forceinline__ void teardown(Bars* B, Pipe& p, uint32_t ncols, int* err) {
  if (threadIdx.x == 0) {
    for (int s = 0; s < 2; ++s)
      if (p.inflight[s]) mbar_wait(&B->full[s], p.fph[s], &B->abort, err, kErrWaitLoad, false);
    mma_commit(&B->mma);
    mbar_wait(&B->mma, p.mph, &B->abort, err, kErrWaitMma, false);
    tma_store_wait_all();
  }
  tc_fence_before();
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) tmem_dealloc(B->tmem, ncols);
}

}  // namespace

// ---------------------------------------------------------------- inference
// Persistent and warp-specialised, two 128-pixel tiles in flight per CTA
// (slots 0 and 1: each its own activation tile in shared memory and 256
// tensor-memory columns).  Warps 0-7 are epilogue warps: they load a
// slot's inputs, and after each of its products turn the accumulator into
// the next operand (GELU) or the start models; warp 8's first thread
// streams the weights through two 32 KB stages by TMA and issues the
// products.  While the epilogue warps work on one slot, the tensor core
// works on the other: per pair of tiles (A in slot 0, B in slot 1) the
// products run L0(A) L0(B) L1(A) L1(B) L2(A) L2(B) and the epilogues
// E0(A) E0(B) E1(A) E1(B) OUT(A) X(A') OUT(B) X(B'), each product waiting
// for the epilogue that wrote its operand (hready, all 256 epilogue
// threads arrive) and each epilogue for its product (zready, a commit).
constexpr int kIThreads = 288;                 // 8 epilogue warps + the producer warp
constexpr uint32_t kIAct = 65536;              // one slot's activation tile (4 K-atoms)
constexpr uint32_t kIW = 2 * kIAct;            // weight stages
constexpr uint32_t kIStage = 32768;            // one K-atom of a 256-row weight
constexpr uint32_t kIBar = kIW + 2 * kIStage;
constexpr uint32_t kIPar = kIBar + 128;
constexpr size_t kISmemBytes = kIPar + 4 * kParFloats + 1024;

struct IBars {
  uint64_t full[2], empty[2];   // weight stages: loaded / free again
  uint64_t zready[2];           // slot's accumulator written (product committed)
  uint64_t hready[2];           // slot's operand tile written (256 epilogue threads)
  uint64_t fin;
  uint32_t tmem;
  int abort;
};

__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(saddr(b)) : "memory");
}

// Producer state (warp 8, lane 0)
struct Prod {
  uint32_t fph[2] = {0, 0}, eph[2] = {0, 0}, hph[2] = {0, 0};
  bool pend[2] = {false, false}, inflight[2] = {false, false};
};

// Load `natoms` K-atoms (from atom k0) of a weight into stage st, once the
// products that last read the stage are done.
__device__ __forceinline__ bool p_load(Prod& P, IBars* B, uint32_t wbase, int st, const CUtensorMap* map, int k0,
                                       int natoms, uint32_t atom_bytes, int* err) {
  if (P.pend[st]) {
    if (!mbar_wait(&B->empty[st], P.eph[st], &B->abort, err, kErrWaitStage)) return false;
    P.eph[st] ^= 1u;
    P.pend[st] = false;
  }
  mbar_expect_tx(&B->full[st], atom_bytes * natoms);
  for (int a = 0; a < natoms; ++a) tma_load_2d(wbase + st * kIStage + a * atom_bytes, map, 64 * (k0 + a), 0, &B->full[st]);
  P.inflight[st] = true;
  return true;
}
__device__ __forceinline__ bool p_wait(Prod& P, IBars* B, int st, int* err) {
  if (!mbar_wait(&B->full[st], P.fph[st], &B->abort, err, kErrWaitLoad)) return false;
  P.fph[st] ^= 1u;
  P.inflight[st] = false;
  tc_fence_after();
  return true;
}
__device__ __forceinline__ void p_release(Prod& P, IBars* B, int st) {
  mma_commit(&B->empty[st]);
  P.pend[st] = true;
}
__device__ __forceinline__ bool p_wait_operand(Prod& P, IBars* B, int slot, int* err) {
  if (!mbar_wait(&B->hready[slot], P.hph[slot], &B->abort, err, kErrWaitMma)) return false;
  P.hph[slot] ^= 1u;
  tc_fence_after();
  return true;
}
// The products of `natoms` K-atoms: A from the slot's tile (atoms a0..),
// B from a stage (atoms b_atom_bytes apart), N = rows, into tensor column
// tcol; the first accumulates onto what is there when acc.
__device__ __forceinline__ void mma_atoms(uint32_t tcol, uint32_t sa, int a0, uint32_t sb, uint32_t b_atom_bytes,
                                          int natoms, int rows, bool acc) {
  const uint32_t idesc = idesc_bf16(128, rows, 0, 0);
  for (int a = 0; a < natoms; ++a)
    for (int kk = 0; kk < 4; ++kk) {
      const uint64_t ad = sw128_desc(sa + (a0 + a) * 16384u + kk * 32u, 16, 1024);
      const uint64_t bd = sw128_desc(sb + a * b_atom_bytes + kk * 32u, 16, 1024);
      mma_bf16(tcol, ad, bd, idesc, (acc || a > 0 || kk > 0) ? 1u : 0u);
    }
}

// Epilogue thread: this thread's shared-memory writes and tensor-memory
// reads of the slot are done; the producer may go on with it.
__device__ __forceinline__ void epi_arrive(uint64_t* bar) {
  fence_proxy_async();
  tc_fence_before();
  mbar_arrive(bar);
}

__global__ void __launch_bounds__(kIThreads, 1)
mlp_infer_kernel(const __grid_constant__ NetMaps nm, const InferArgs a) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const uint32_t base = (saddr(smem_raw) + 1023u) & ~1023u;
  unsigned char* gbase = smem_raw + (base - saddr(smem_raw));
  IBars* B = reinterpret_cast<IBars*>(gbase + kIBar);
  float* spar = reinterpret_cast<float*>(gbase + kIPar);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int64_t tiles = (a.n + kTile - 1) / kTile;
  const int64_t G = gridDim.x;
  stage_params(a.p, spar);
  if (tid == 0) {
    for (int i = 0; i < 2; ++i) {
      mbar_init(&B->full[i], 1);
      mbar_init(&B->empty[i], 1);
      mbar_init(&B->zready[i], 1);
      mbar_init(&B->hready[i], 256);
    }
    mbar_init(&B->fin, 1);
    B->abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tmem_alloc(&B->tmem, 512);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t wbase = base + kIW;
  if (warp == 8) {
    // ---- producer: weights and products
    Prod P;
    bool ok = true;
    if ((tid & 31) == 0) {
      const CUtensorMap* w1 = &nm.m[kMapW1];
      const CUtensorMap* w2 = &nm.m[kMapW2];
      const CUtensorMap* w3 = &nm.m[kMapW3];
      for (int64_t tA = blockIdx.x; tA < tiles && ok; tA += 2 * G) {
        const bool hasB = tA + G < tiles;
        const int nslot = hasB ? 2 : 1;
        // L0: both K-atoms of W1 resident, the products of both slots
        ok = p_load(P, B, wbase, 0, w1, 0, 1, kIStage, a.err) && p_load(P, B, wbase, 1, w1, 1, 1, kIStage, a.err);
        ok = ok && p_wait(P, B, 0, a.err) && p_wait(P, B, 1, a.err);
        for (int sl = 0; sl < nslot && ok; ++sl) {
          ok = p_wait_operand(P, B, sl, a.err);
          if (!ok) break;
          const uint32_t tcol = B->tmem + 256u * sl, sa = base + sl * kIAct;
          mma_atoms(tcol, sa, 0, wbase, 0, 1, 256, false);
          mma_atoms(tcol, sa, 1, wbase + kIStage, 0, 1, 256, true);
          mma_commit(&B->zready[sl]);
        }
        if (!ok) break;
        p_release(P, B, 0);
        p_release(P, B, 1);
        // L1: the four K-atoms of W2 streamed through the stages, per slot
        for (int sl = 0; sl < nslot && ok; ++sl) {
          const uint32_t tcol = B->tmem + 256u * sl, sa = base + sl * kIAct;
          ok = p_load(P, B, wbase, 0, w2, 0, 1, kIStage, a.err) && p_load(P, B, wbase, 1, w2, 1, 1, kIStage, a.err);
          ok = ok && p_wait_operand(P, B, sl, a.err);
          for (int h = 0; h < 2 && ok; ++h) {
            if (h == 1)
              ok = p_load(P, B, wbase, 0, w2, 2, 1, kIStage, a.err) && p_load(P, B, wbase, 1, w2, 3, 1, kIStage, a.err);
            for (int st = 0; st < 2 && ok; ++st) {
              ok = p_wait(P, B, st, a.err);
              if (!ok) break;
              mma_atoms(tcol, sa, 2 * h + st, wbase + st * kIStage, 0, 1, 256, h + st > 0);
              p_release(P, B, st);
            }
          }
          if (ok) mma_commit(&B->zready[sl]);
        }
        if (!ok) break;
        // L2: W3 (16 rows, 4 K-atoms of 2 KB) in stage 0 for both slots
        ok = p_load(P, B, wbase, 0, w3, 0, 4, 16u * 128u, a.err) && p_wait(P, B, 0, a.err);
        for (int sl = 0; sl < nslot && ok; ++sl) {
          ok = p_wait_operand(P, B, sl, a.err);
          if (!ok) break;
          mma_atoms(B->tmem + 256u * sl, base + sl * kIAct, 0, wbase, 16u * 128u, 4, 16, false);
          mma_commit(&B->zready[sl]);
        }
        if (ok) p_release(P, B, 0);
      }
      if (!ok) atomicCAS(a.err, kErrNone, kErrWaitMma);
      // end: loads still in flight (only after an abort), then every product
      for (int st = 0; st < 2; ++st)
        if (P.inflight[st]) mbar_wait(&B->full[st], P.fph[st], &B->abort, a.err, kErrWaitLoad, false);
      mma_commit(&B->fin);
      mbar_wait(&B->fin, 0, &B->abort, a.err, kErrWaitMma, false);
    }
  } else {
    // ---- epilogue warps
    const int row = tid & (kTile - 1), half = tid >> 7;   // accumulator row, column half
    const uint32_t qoff = (uint32_t)((warp & 3) * 32) << 16;
    uint32_t zph[2] = {0, 0};
    bool ok = true;
    auto zwait = [&](int sl) {
      ok = ok && mbar_wait(&B->zready[sl], zph[sl], &B->abort, a.err, kErrWaitMma);
      zph[sl] ^= 1u;
      tc_fence_after();
      return ok;
    };
    for (int sl = 0; sl < 2; ++sl) {
      const int64_t t = blockIdx.x + sl * G;
      if (t < tiles) {
        load_x(spar, a.iquv, nullptr, t * kTile, a.n, a.nl, base + sl * kIAct, row, half);
        epi_arrive(&B->hready[sl]);
      }
    }
    for (int64_t tA = blockIdx.x; tA < tiles && ok; tA += 2 * G) {
      const int nslot = tA + G < tiles ? 2 : 1;
      for (int L = 0; L < 2 && ok; ++L)
        for (int sl = 0; sl < nslot; ++sl) {
          if (!zwait(sl)) break;
          hidden_epilogue(B->tmem + 256u * sl + qoff, 0, spar + 256 * L, base + sl * kIAct, row, half, nullptr);
          epi_arrive(&B->hready[sl]);
        }
      for (int sl = 0; sl < nslot && ok; ++sl) {
        if (!zwait(sl)) break;
        const int64_t t = tA + sl * G;
        if (half == 0) {
          const int64_t b = t * kTile + row;
          float o[16];
          tmem_ld16(B->tmem + 256u * sl + qoff, o);
          if (b < a.n) {
            float y[kOut];
#pragma unroll
            for (int j = 0; j < kOut; ++j) y[j] = (o[j] + a.p->b3[j]) * a.p->out_scale[j] + a.p->out_mean[j];
            double m[11];
            outputs_to_model(y, a.guess, a.fix, m);
#pragma unroll
            for (int i = 0; i < 11; ++i) a.models[b * 11 + i] = m[i];
          }
        }
        // this slot's next tile
        if (t + 2 * G < tiles) {
          load_x(spar, a.iquv, nullptr, (t + 2 * G) * kTile, a.n, a.nl, base + sl * kIAct, row, half);
          epi_arrive(&B->hready[sl]);
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(B->tmem, 512);
}

// ---------------------------------------------------------------- training: forward + activation backward
// Per tile of the batch: X -> Z1 -> H1 -> Z2 -> H2 -> out, the loss and
// dOut = 2 (out - y) / (rows x 9), then dH2 = dOut W3, dZ2 = dH2 GELU'(Z2),
// dH1 = dZ2 W2, dZ1 = dH1 GELU'(Z1).  Tensor columns: Z1 0..255 (kept in
// zspill), Z2 256..511 (kept until dZ2), out 0..15, dH2 0..255, dH1
// 256..511.  X, H1, H2, dOut, dZ2, dZ1 go row-major to global memory (TMA
// stores of the operand tiles) for the weight gradients.
__global__ void __launch_bounds__(kThreads, 1)
mlp_train_kernel(const __grid_constant__ NetMaps nm, const __grid_constant__ ActMaps am, const TrainKArgs a) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const uint32_t base = (saddr(smem_raw) + 1023u) & ~1023u;
  Bars* B = reinterpret_cast<Bars*>(smem_raw + (base - saddr(smem_raw)) + kSBar);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int row = tid & (kTile - 1), half = tid >> 7;   // accumulator row, column half
  float* spar = reinterpret_cast<float*>(smem_raw + (base - saddr(smem_raw)) + kSPar);
  stage_params(a.p, spar);
  setup(B, 512);
  const uint32_t trow = B->tmem + ((uint32_t)((warp & 3) * 32) << 16);
  const uint32_t sA = base + kSA, sD = base + kSD;
  const int64_t tiles = a.n / kTile;
  Pipe p;
  bool ok = true;
  if (tid == 0 && (int64_t)blockIdx.x < tiles) start_load(c_jobs[0], nm, B, base, 0, p);
  for (int64_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
    const bool last_tile = t + gridDim.x >= tiles;
    const int64_t b = t * kTile + row;   // this thread's batch row
    float* zrow = a.zspill + b * kHid;
    // the previous tile's stores must have read the operand tiles
    if (tid == 0) tma_store_wait_read();
    __syncthreads();
    load_x(spar, a.iquv, a.idx, t * kTile, a.n, a.nl, sA, row, half);
    fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      tma_store_2d(&am.x, 0, (int)(t * kTile), sA);
      tma_store_2d(&am.x, 64, (int)(t * kTile), sA + 16384u);
      tma_store_commit();
    }
    // five layers: 0 Z1, 1 Z2, 2 out, 3 dH2, 4 dH1
    for (int L = 0; L < 5 && ok; ++L) {
      if (tid == 0) {
        for (int j = layer_first(L, true); j < layer_last(L, true) && ok; ++j) {
          const Job* nx = (j + 1 < kTrainJobs) ? &c_jobs[j + 1] : (last_tile ? nullptr : &c_jobs[0]);
          ok = run_job(c_jobs[j], nx, true, nm, B, base, p, a.err);
        }
      }
      ok = mbar_wait(&B->mma, p.mph, &B->abort, a.err, kErrWaitMma) && ok;
      p.mph ^= 1u;
      // an epilogue that overwrites the activation tile waits for its stores
      if (tid == 0 && L != 2) tma_store_wait_read();
      __syncthreads();
      ok = ok && !B->abort;
      if (!ok) break;
      tc_fence_after();
      if (L == 0) {
        hidden_epilogue(trow, 0, spar, sA, row, half, zrow);
      } else if (L == 1) {
        hidden_epilogue(trow, 256, spar + 256, sA, row, half, nullptr);
      } else if (L == 2) {
        if (half == 0) {   // the 9 outputs: the first warpgroup
          float o[16];
          tmem_ld16(trow, o);
          const float* yt = a.y16 + (int64_t)a.idx[b] * 16;
          float sq = 0.f;
          float g[kOut];
#pragma unroll
          for (int j = 0; j < kOut; ++j) {
            const float d = o[j] + a.p->b3[j] - __ldg(yt + j);
            sq += d * d;
            g[j] = a.gscale * d;
          }
          uint32_t w[4] = {pack_bf16(g[0], g[1]), pack_bf16(g[2], g[3]), pack_bf16(g[4], g[5]),
                           pack_bf16(g[6], g[7])};
          st_chunk(sD, row, 0, w);
          w[0] = pack_bf16(g[8], 0.f);
          w[1] = w[2] = w[3] = 0u;
          st_chunk(sD, row, 1, w);
          w[0] = 0u;
#pragma unroll
          for (int j = 2; j < 8; ++j) st_chunk(sD, row, j, w);
#pragma unroll
          for (int o2 = 16; o2 > 0; o2 >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o2);
          if (lane == 0) atomicAdd(a.loss, sq);
        }
      } else {
        // dZ = dH GELU'(Z): L 3 -> dZ2 (dH2 at column 0, Z2 at 256);
        // L 4 -> dZ1 (dH1 at column 256, Z1 from the spill); this
        // warpgroup's half of the columns
#pragma unroll 1
        for (int q = 4 * half; q < 4 * half + 4; ++q) {
          float dh[32], z[32];
          if (L == 3) {
            tmem_ld32(trow + 32 * q, dh);
            tmem_ld32(trow + 256 + 32 * q, z);   // the product, without its bias
#pragma unroll
            for (int e = 0; e < 32; ++e) z[e] += spar[256 + 32 * q + e];
          } else {
            tmem_ld32(trow + 256 + 32 * q, dh);
            const float4* src = reinterpret_cast<const float4*>(zrow + 32 * q);
#pragma unroll
            for (int u = 0; u < 8; ++u) {
              const float4 v = src[u];
              z[4 * u] = v.x;
              z[4 * u + 1] = v.y;
              z[4 * u + 2] = v.z;
              z[4 * u + 3] = v.w;
            }
          }
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            uint32_t w[4];
#pragma unroll
            for (int h = 0; h < 4; ++h) {
              const int e = 8 * u + 2 * h;
              w[h] = pack_bf16(dh[e] * gelu_grad(z[e]), dh[e + 1] * gelu_grad(z[e + 1]));
            }
            st_chunk(sA + (q >> 1) * 16384u, row, (q & 1) * 4 + u, w);
          }
        }
      }
      fence_proxy_async();
      tc_fence_before();
      __syncthreads();
      tc_fence_after();
      // row-major copies for the weight gradients
      if (tid == 0) {
        const int y = (int)(t * kTile);
        const CUtensorMap* m = L == 0 ? &am.h1 : L == 1 ? &am.h2 : L == 2 ? &am.g3 : L == 3 ? &am.g2 : &am.g1;
        const uint32_t src = L == 2 ? sD : sA;
        const int natoms = L == 2 ? 1 : 4;
        for (int k = 0; k < natoms; ++k) tma_store_2d(m, 64 * k, y, src + 16384u * k);
        tma_store_commit();
      }
    }
  }
  teardown(B, p, 512, a.err);
}

// ---------------------------------------------------------------- training: weight gradients
// dW[m][n] += sum over a slice of the batch of A[b][m] Bm[b][n] for one
// 128 x 64 block; both operands row-major in global memory, MN-major in the
// product (8-row K groups 1024 bytes apart, 64-element M blocks 8 KB apart),
// 4-stage TMA ring.  Products: 0 dW1 = G1^T X (4 blocks), 1 dW2 = G2^T H1
// (8 blocks), 2 dW3^T = H2^T dOut (2 blocks, added transposed).  Blocks of
// one product add their slices into the FP32 gradient.
struct WgradArgs {
  float* dw1;   // [256][128]
  float* dw2;   // [256][256]
  float* dw3;   // [9][256]
  int64_t rows; // batch rows (a multiple of 64)
  int kslices;  // batch slices per block
  int* err;
};
struct WgradMaps {
  CUtensorMap a[3], b[3];   // boxes of 64 x 64 elements
};
constexpr int kWStages = 4;
constexpr uint32_t kWStageBytes = 16384 + 8192;   // A: 2 boxes (m 0..127), B: 1 box (n 0..63)
constexpr int kWBlocks = 14;
constexpr size_t kWgradSmem = kWStages * kWStageBytes + 256 + 1024;

__global__ void __launch_bounds__(kWThreads, 1)
mlp_wgrad_kernel(const __grid_constant__ WgradMaps wm, const WgradArgs a) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const uint32_t base = (saddr(smem_raw) + 1023u) & ~1023u;
  struct WB {
    uint64_t full[kWStages], empty[kWStages], done;
    uint32_t tmem;
    int abort;
  };
  WB* B = reinterpret_cast<WB*>(smem_raw + (base - saddr(smem_raw)) + kWStages * kWStageBytes);
  const int tid = threadIdx.x, warp = tid >> 5;
  int blk = blockIdx.x;
  const int slice = blk % a.kslices;
  blk /= a.kslices;
  int g, mb, nb;
  if (blk < 4) {
    g = 0; mb = blk >> 1; nb = blk & 1;
  } else if (blk < 12) {
    g = 1; mb = (blk - 4) >> 2; nb = (blk - 4) & 3;
  } else {
    g = 2; mb = blk - 12; nb = 0;
  }
  if (tid == 0) {
    for (int s = 0; s < kWStages; ++s) {
      mbar_init(&B->full[s], 1);
      mbar_init(&B->empty[s], 1);
    }
    mbar_init(&B->done, 1);
    B->abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tmem_alloc(&B->tmem, 64);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const int64_t ksteps = a.rows / 64;
  const int64_t k0 = ksteps * slice / a.kslices, k1 = ksteps * (slice + 1) / a.kslices;
  const CUtensorMap* ma = &wm.a[g];
  const CUtensorMap* mbm = &wm.b[g];
  bool inflight[kWStages] = {false, false, false, false};
  uint32_t fph[kWStages] = {0, 0, 0, 0};
  if (tid == 0) {
    const uint32_t idesc = idesc_bf16(128, 64, 1, 1);
    uint32_t eph[kWStages] = {0, 0, 0, 0};
    bool pend[kWStages] = {false, false, false, false};
    bool ok = true;
    auto issue = [&](int64_t k) -> bool {
      const int s = (int)((k - k0) % kWStages);
      const uint32_t st = base + s * kWStageBytes;
      if (pend[s]) {
        if (!mbar_wait(&B->empty[s], eph[s], &B->abort, a.err, kErrWaitStage)) return false;
        eph[s] ^= 1u;
        pend[s] = false;
      }
      mbar_expect_tx(&B->full[s], kWStageBytes);
      tma_load_2d(st, ma, mb * 128, (int)(k * 64), &B->full[s]);
      tma_load_2d(st + 8192u, ma, mb * 128 + 64, (int)(k * 64), &B->full[s]);
      tma_load_2d(st + 16384u, mbm, nb * 64, (int)(k * 64), &B->full[s]);
      inflight[s] = true;
      return true;
    };
    for (int64_t k = k0; k < k1 && k < k0 + kWStages - 1 && ok; ++k) ok = issue(k);
    for (int64_t k = k0; k < k1 && ok; ++k) {
      const int s = (int)((k - k0) % kWStages);
      const uint32_t st = base + s * kWStageBytes;
      if (!mbar_wait(&B->full[s], fph[s], &B->abort, a.err, kErrWaitLoad)) {
        ok = false;
        break;
      }
      fph[s] ^= 1u;
      inflight[s] = false;
      tc_fence_after();
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        // 16 batch rows = two 8-row groups of 1024 bytes
        const uint64_t ad = sw128_desc(st + kk * 2048u, 8192, 1024);
        const uint64_t bd = sw128_desc(st + 16384u + kk * 2048u, 8192, 1024);
        mma_bf16(B->tmem, ad, bd, idesc, (k > k0 || kk > 0) ? 1u : 0u);
      }
      mma_commit(&B->empty[s]);
      pend[s] = true;
      if (k + kWStages - 1 < k1) ok = issue(k + kWStages - 1);
    }
    // the last commit covers every product issued (also after an abort)
    mma_commit(&B->done);
  }
  __syncthreads();
  const bool ran = k1 > k0;
  bool ok = mbar_wait(&B->done, 0, &B->abort, a.err, kErrWaitMma, false) && ran;
  __syncthreads();
  ok = ok && !B->abort;
  if (ok) {
    tc_fence_after();
    const uint32_t trow = B->tmem + ((uint32_t)(warp * 32) << 16);
    const int m = mb * 128 + tid;
#pragma unroll 1
    for (int h = 0; h < 2; ++h) {
      float v[32];
      tmem_ld32(trow + 32 * h, v);
      if (g < 2) {
        // this thread's 32 columns are contiguous in its row of dW1 / dW2
        // (16-byte aligned): vector reductions, a quarter of the atomics
        float* dst = (g == 0 ? a.dw1 + m * kIn : a.dw2 + m * kHid) + nb * 64 + 32 * h;
#pragma unroll
        for (int e = 0; e < 32; e += 4)
          atomicAdd(reinterpret_cast<float4*>(dst + e), make_float4(v[e], v[e + 1], v[e + 2], v[e + 3]));
      } else {
#pragma unroll 4
        for (int e = 0; e < 32; ++e) {
          const int n = nb * 64 + 32 * h + e;
          if (n < kOut) atomicAdd(a.dw3 + n * kHid + m, v[e]);
        }
      }
    }
  }
  if (tid == 0)
    for (int s = 0; s < kWStages; ++s)
      if (inflight[s]) mbar_wait(&B->full[s], fph[s], &B->abort, a.err, kErrWaitLoad, false);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(B->tmem, 64);
}

// Bias gradients: column sums of the stored output gradients (BF16),
// gridDim.x slices of the batch, blockIdx.y the layer.
__global__ void mlp_bias_grad_kernel(const uint16_t* __restrict__ g1, const uint16_t* __restrict__ g2,
                                     const uint16_t* __restrict__ g3, int64_t rows, float* db1, float* db2,
                                     float* db3) {
  const int which = blockIdx.y;
  const int f = threadIdx.x;
  const int width = which == 2 ? kG : kHid;
  const int used = which == 2 ? kOut : kHid;
  if (f >= used) return;
  const uint16_t* g = which == 0 ? g1 : (which == 1 ? g2 : g3);
  float* db = which == 0 ? db1 : (which == 1 ? db2 : db3);
  const int64_t r0 = rows * blockIdx.x / gridDim.x, r1 = rows * (blockIdx.x + 1) / gridDim.x;
  float s = 0.f;
  for (int64_t r = r0; r < r1; ++r) s += __uint_as_float((uint32_t)g[r * width + f] << 16);
  atomicAdd(db + f, s);
}

// ---------------------------------------------------------------- parameters
// The FP32 parameters of a gm_mlp in one flat index: w1, b1, w2, b2, w3, b3.
constexpr int kNW1 = kHid * kIn, kNW2 = kHid * kHid, kNW3 = kOut * kHid;
constexpr int kParams = kNW1 + kHid + kNW2 + kHid + kNW3 + kOut;

__device__ __forceinline__ float* param_at(gm_mlp* p, int i, bool* bias) {
  *bias = false;
  if (i < kNW1) return &p->w1[0][0] + i;
  i -= kNW1;
  if (i < kHid) { *bias = true; return p->b1 + i; }
  i -= kHid;
  if (i < kNW2) return &p->w2[0][0] + i;
  i -= kNW2;
  if (i < kHid) { *bias = true; return p->b2 + i; }
  i -= kHid;
  if (i < kNW3) return &p->w3[0][0] + i;
  i -= kNW3;
  *bias = true;
  return p->b3 + i;
}

// The BF16 operand copies of parameter i (weights only); padding stays zero.
__device__ __forceinline__ void pack_one(const gm_mlp* p, uint16_t* pack, int i) {
  if (i < kNW1) {
    const int o = i / kIn, c = i % kIn;
    pack[kW1b + o * kIn + c] = __bfloat16_as_ushort(__float2bfloat16_rn(p->w1[o][c]));
    return;
  }
  i -= kNW1 + kHid;
  if (i >= 0 && i < kNW2) {
    const int o = i / kHid, c = i % kHid;
    const uint16_t v = __bfloat16_as_ushort(__float2bfloat16_rn(p->w2[o][c]));
    pack[kW2b + o * kHid + c] = v;
    pack[kW2tb + c * kHid + o] = v;
    return;
  }
  i -= kNW2 + kHid;
  if (i >= 0 && i < kNW3) {
    const int o = i / kHid, c = i % kHid;
    const uint16_t v = __bfloat16_as_ushort(__float2bfloat16_rn(p->w3[o][c]));
    pack[kW3b + o * kHid + c] = v;
    pack[kW3tb + c * kG + o] = v;
  }
}

__global__ void mlp_pack_kernel(const gm_mlp* p, uint16_t* pack) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kParams; i += gridDim.x * blockDim.x) pack_one(p, pack, i);
}

// Adam with decoupled weight decay (weights only) on every parameter, its
// BF16 copy rewritten, its gradient cleared for the next batch.  c1, c2: the
// bias corrections 1 / (1 - beta^t).
__global__ void mlp_adam_kernel(gm_mlp* p, gm_mlp* grad, gm_mlp* m1, gm_mlp* m2, uint16_t* pack, float lr,
                                float wd, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kParams; i += gridDim.x * blockDim.x) {
    bool bias;
    float* w = param_at(p, i, &bias);
    float* g = param_at(grad, i, &bias);
    float* ma = param_at(m1, i, &bias);
    float* mb = param_at(m2, i, &bias);
    const float gv = *g;
    const float av = 0.9f * *ma + 0.1f * gv;
    const float bv = 0.999f * *mb + 0.001f * gv * gv;
    *ma = av;
    *mb = bv;
    *w -= lr * ((av * c1) / (sqrtf(bv * c2) + 1e-8f) + (bias ? 0.f : wd * *w));
    *g = 0.f;
    pack_one(p, pack, i);
  }
}

// Standardised targets [n][16] of the models [n][11] (the 9 outputs, then
// zeros).
__global__ void mlp_targets_kernel(const double* __restrict__ truth, int64_t n, const gm_mlp* p, float* y16) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double* m = truth + i * 11;
    const double g = m[5] * (3.14159265358979323846 / 180.0);
    const double ph = 2.0 * m[6] * (3.14159265358979323846 / 180.0);
    const double v[kOut] = {m[0], m[2], m[3], m[4], m[7], m[8], m[1] * cos(g), m[1] * sin(g) * cos(ph),
                            m[1] * sin(g) * sin(ph)};
    for (int j = 0; j < 16; ++j)
      y16[i * 16 + j] = j < kOut ? (float)((v[j] - p->out_mean[j]) / p->out_scale[j]) : 0.f;
  }
}

// An epoch's visiting order: a pseudo-random permutation of [0, n) drawn on
// the device, so that no host shuffle or copy sits between epochs.  A
// 4-round Feistel network on 2 hb bits (2^(2 hb) >= n), its round function
// the MurmurHash3 finaliser of (half ^ round key), restricted to [0, n) by
// cycle walking (Black & Rogaway, "Ciphers with arbitrary finite domains",
// 2002): re-applying the bijection until the value falls inside keeps the
// map one to one and ends within the cycle of i, fewer than 4 n steps
// (expected under 4).  hb = 0 writes the identity.
__device__ __forceinline__ uint32_t fmix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x85ebca6bu;
  x ^= x >> 13;
  x *= 0xc2b2ae35u;
  x ^= x >> 16;
  return x;
}

__global__ void mlp_order_kernel(uint32_t* __restrict__ idx, uint32_t n, int hb, uint64_t key) {
  const uint32_t mask = hb ? (1u << hb) - 1u : 0u;
  const uint64_t cap = 4ull * n;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t x = i;
    if (hb) {
      uint64_t walk = 0;
      do {
        uint32_t l = x >> hb, r = x & mask;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const uint32_t f = fmix32(r ^ (uint32_t)(key >> (16 * k)) ^ (0x9e3779b9u * (uint32_t)(k + 1))) & mask;
          const uint32_t t = l ^ f;
          l = r;
          r = t;
        }
        x = (l << hb) | r;
      } while (x >= n && ++walk < cap);
    }
    idx[i] = x;
  }
}

// ---------------------------------------------------------------- host
namespace {

PFN_cuTensorMapEncodeTiled_v12000 encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }
  return fn;
}

// 2-D BF16 map of a row-major [rows][cols] matrix, boxes of 64 columns x
// box_rows rows, 128-byte swizzle.
bool make_map(CUtensorMap* m, const void* base, uint64_t cols, uint64_t rows, uint32_t box_rows) {
  auto enc = encoder();
  if (!enc) return false;
  cuuint64_t dims[2] = {cols, rows};
  cuuint64_t strides[1] = {cols * 2};
  cuuint32_t box[2] = {64, box_rows};
  cuuint32_t es[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool net_maps(const uint16_t* pack, NetMaps* nm) {
  return make_map(&nm->m[kMapW1], pack + kW1b, kIn, kHid, 256) &&
         make_map(&nm->m[kMapW2], pack + kW2b, kHid, kHid, 256) &&
         make_map(&nm->m[kMapW3], pack + kW3b, kHid, kOut16, 16) &&
         make_map(&nm->m[kMapW2t], pack + kW2tb, kHid, kHid, 256) &&
         make_map(&nm->m[kMapW3t], pack + kW3tb, kG, kHid, 256);
}

int sm_count() {
  int dev = 0, n = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n > 0 ? n : 1;
}

// A float array of a gm_mlp in device memory (no host dereference).
float* field(gm_mlp* dev, size_t offset) { return reinterpret_cast<float*>(reinterpret_cast<char*>(dev) + offset); }

// Device buffers of a training session, freed together.
struct Buffers {
  std::vector<void*> owned;
  template <typename T>
  cudaError_t get(T** p, size_t count) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, sizeof(T) * count);
    if (e == cudaSuccess) owned.push_back(q);
    *p = static_cast<T*>(q);
    return e;
  }
  ~Buffers() {
    for (void* q : owned) cudaFree(q);
  }
};

// Standardisation of inputs and targets from up to 65536 of the pixels.
cudaError_t standardise(gm_mlp* net, const float* iquv, const double* truth, int64_t n, int nl) {
  const int64_t m = std::min<int64_t>(n, 65536);
  const int F = 4 * nl;
  std::vector<float> x((size_t)m * F);
  std::vector<double> t((size_t)m * 11);
  cudaError_t e = cudaMemcpy(x.data(), iquv, sizeof(float) * x.size(), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(t.data(), truth, sizeof(double) * t.size(), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return e;
  for (int f = 0; f < kIn; ++f) {
    net->in_mean[f] = 0.f;
    net->in_scale[f] = 0.f;
    if (f >= F) continue;
    double s = 0, ss = 0;
    for (int64_t i = 0; i < m; ++i) {
      const double v = x[(size_t)i * F + f];
      s += v;
      ss += v * v;
    }
    const double mu = s / m, var = std::max(ss / m - mu * mu, 0.0);
    net->in_mean[f] = (float)mu;
    net->in_scale[f] = var > 1e-20 ? (float)(1.0 / std::sqrt(var)) : 0.f;
  }
  double s[kOut] = {}, ss[kOut] = {};
  for (int64_t i = 0; i < m; ++i) {
    float y[kOut];
    targets_of(&t[(size_t)i * 11], y);
    for (int j = 0; j < kOut; ++j) {
      s[j] += y[j];
      ss[j] += (double)y[j] * y[j];
    }
  }
  for (int j = 0; j < kOut16; ++j) {
    net->out_mean[j] = 0.f;
    net->out_scale[j] = 1.f;
  }
  for (int j = 0; j < kOut; ++j) {
    const double mu = s[j] / m, var = std::max(ss[j] / m - mu * mu, 0.0);
    net->out_mean[j] = (float)mu;
    net->out_scale[j] = var > 1e-20 ? (float)std::sqrt(var) : 1.f;
  }
  return cudaSuccess;
}

}  // namespace

void targets_of(const double* m, float* y) {
  const double g = m[5] * (M_PI / 180.0), ph = 2.0 * m[6] * (M_PI / 180.0);
  const double v[kOut] = {m[0], m[2], m[3], m[4], m[7], m[8], m[1] * std::cos(g), m[1] * std::sin(g) * std::cos(ph),
                          m[1] * std::sin(g) * std::sin(ph)};
  for (int j = 0; j < kOut; ++j) y[j] = (float)v[j];
}

void init_net(gm_mlp* net, int nl, uint64_t seed) {
  std::memset(net, 0, sizeof(*net));
  net->abi_version = GM_ABI_VERSION;
  net->nl = nl;
  for (int f = 0; f < kIn; ++f) net->in_scale[f] = f < 4 * nl ? 1.f : 0.f;
  for (int j = 0; j < kOut16; ++j) net->out_scale[j] = 1.f;
  std::mt19937_64 rng(seed);
  auto fill = [&](float* w, int fan_out, int fan_in, int used_in, float gain) {
    const float a = gain * std::sqrt(6.f / (float)used_in);   // variance 2 / fan-in
    std::uniform_real_distribution<float> u(-a, a);
    for (int o = 0; o < fan_out; ++o)
      for (int i = 0; i < fan_in; ++i) w[o * fan_in + i] = i < used_in ? u(rng) : 0.f;
  };
  fill(&net->w1[0][0], kHid, kIn, 4 * nl, 1.f);
  fill(&net->w2[0][0], kHid, kHid, kHid, 1.f);
  fill(&net->w3[0][0], kOut, kHid, kHid, 0.1f);   // outputs start near the mean
}

cudaError_t devnet_create(DevNet* d, const gm_mlp* host, cudaStream_t s) {
  devnet_destroy(d);
  cudaError_t e = cudaMalloc(&d->p, sizeof(gm_mlp));
  if (e == cudaSuccess) e = cudaMalloc(&d->pack, sizeof(uint16_t) * kPackElems);
  if (e == cudaSuccess) e = cudaMemsetAsync(d->pack, 0, sizeof(uint16_t) * kPackElems, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d->p, host, sizeof(gm_mlp), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return e;
  mlp_pack_kernel<<<256, 256, 0, s>>>(d->p, d->pack);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  NetMaps nm;
  if (!net_maps(d->pack, &nm)) return cudaErrorInvalidValue;
  d->mw1 = nm.m[kMapW1];
  d->mw2 = nm.m[kMapW2];
  d->mw3 = nm.m[kMapW3];
  d->mw2t = nm.m[kMapW2t];
  d->mw3t = nm.m[kMapW3t];
  d->nl = host->nl;
  return cudaSuccess;
}

void devnet_destroy(DevNet* d) {
  if (d->p) cudaFree(d->p);
  if (d->pack) cudaFree(d->pack);
  *d = DevNet{};
}

cudaError_t predict(const DevNet& d, const float* iquv, int64_t n, int nl, const double* guess, const int* fix,
                    double* models, int* err, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  if (nl != d.nl || 4 * nl > kIn || !err) return cudaErrorInvalidValue;
  // the input tiles are read in 16-byte vectors
  if (reinterpret_cast<uintptr_t>(iquv) & 15u) return cudaErrorInvalidValue;
  NetMaps nm;
  nm.m[kMapW1] = d.mw1;
  nm.m[kMapW2] = d.mw2;
  nm.m[kMapW3] = d.mw3;
  nm.m[kMapW2t] = d.mw2t;
  nm.m[kMapW3t] = d.mw3t;
  InferArgs a{};
  a.p = d.p;
  a.iquv = iquv;
  a.n = n;
  a.nl = nl;
  for (int i = 0; i < 11; ++i) {
    a.guess[i] = guess[i];
    a.fix[i] = fix ? fix[i] : 1;
  }
  a.models = models;
  a.err = err;
  cudaError_t e =
      cudaFuncSetAttribute(mlp_infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kISmemBytes);
  if (e != cudaSuccess) return e;
  const int64_t tiles = (n + kTile - 1) / kTile;
  const int grid = (int)std::min<int64_t>(tiles, sm_count());
  mlp_infer_kernel<<<grid, kIThreads, kISmemBytes, s>>>(nm, a);
  return cudaGetLastError();
}

cudaError_t train(gm_mlp* net, const TrainArgs& a, float* loss_out, gm_mlp* grads_out, int* err, cudaStream_t s,
                  const char** why) {
  auto fail = [&](const char* w, cudaError_t e) {
    if (why) *why = w;
    return e;
  };
  const int64_t B = a.grads_only ? a.n : (int64_t)a.batch;
  if (B <= 0 || B % kTile || a.n < B || B > (int64_t)1 << 30)
    return fail("the batch must be a positive multiple of 128 and at most the pixel count", cudaErrorInvalidValue);
  if (a.n > (int64_t)1 << 31) return fail("at most 2^31 training pixels", cudaErrorInvalidValue);
  if (a.nl < 1 || 4 * a.nl > kIn || net->nl != a.nl) return fail("the network's grid differs", cudaErrorInvalidValue);
  if (!err) return fail("no error word", cudaErrorInvalidValue);
  if (reinterpret_cast<uintptr_t>(a.iquv) & 15u)
    return fail("the profiles must start on a 16-byte boundary", cudaErrorInvalidValue);
  // the data may still be arriving on s
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail("data upload", e);
  if (net->steps == 0 && !a.grads_only) {
    e = standardise(net, a.iquv, a.truth, a.n, a.nl);
    if (e != cudaSuccess) return fail("standardisation", e);
  }
  Buffers buf;
  DevNet d;
  e = devnet_create(&d, net, s);
  if (e != cudaSuccess) {
    devnet_destroy(&d);
    return fail("network upload", e);
  }
  gm_mlp *grad = nullptr, *m1 = nullptr, *m2 = nullptr;
  uint16_t *x = nullptr, *h1 = nullptr, *h2 = nullptr, *g1 = nullptr, *g2 = nullptr, *g3 = nullptr;
  float *z = nullptr, *y16 = nullptr, *loss = nullptr;
  uint32_t* idx = nullptr;
  const int64_t n = a.n;
  if ((e = buf.get(&grad, 1)) != cudaSuccess || (e = buf.get(&m1, 1)) != cudaSuccess ||
      (e = buf.get(&m2, 1)) != cudaSuccess || (e = buf.get(&x, (size_t)B * kIn)) != cudaSuccess ||
      (e = buf.get(&h1, (size_t)B * kHid)) != cudaSuccess || (e = buf.get(&h2, (size_t)B * kHid)) != cudaSuccess ||
      (e = buf.get(&g1, (size_t)B * kHid)) != cudaSuccess || (e = buf.get(&g2, (size_t)B * kHid)) != cudaSuccess ||
      (e = buf.get(&g3, (size_t)B * kG)) != cudaSuccess || (e = buf.get(&z, (size_t)B * kHid)) != cudaSuccess ||
      (e = buf.get(&y16, (size_t)n * 16)) != cudaSuccess || (e = buf.get(&idx, (size_t)n)) != cudaSuccess ||
      (e = buf.get(&loss, 1)) != cudaSuccess) {
    devnet_destroy(&d);
    return fail("device allocation", e);
  }
  cudaMemsetAsync(grad, 0, sizeof(gm_mlp), s);
  cudaMemsetAsync(m1, 0, sizeof(gm_mlp), s);
  cudaMemsetAsync(m2, 0, sizeof(gm_mlp), s);
  NetMaps nm;
  ActMaps am;
  WgradMaps wm;
  bool maps = net_maps(d.pack, &nm) && make_map(&am.x, x, kIn, B, 128) && make_map(&am.h1, h1, kHid, B, 128) &&
              make_map(&am.h2, h2, kHid, B, 128) && make_map(&am.g3, g3, kG, B, 128) &&
              make_map(&am.g2, g2, kHid, B, 128) && make_map(&am.g1, g1, kHid, B, 128) &&
              make_map(&wm.a[0], g1, kHid, B, 64) && make_map(&wm.b[0], x, kIn, B, 64) &&
              make_map(&wm.a[1], g2, kHid, B, 64) && make_map(&wm.b[1], h1, kHid, B, 64) &&
              make_map(&wm.a[2], h2, kHid, B, 64) && make_map(&wm.b[2], g3, kG, B, 64);
  if (!maps) {
    devnet_destroy(&d);
    return fail("tensor-map encoding", cudaErrorInvalidValue);
  }
  mlp_targets_kernel<<<1024, 256, 0, s>>>(a.truth, n, d.p, y16);
  e = cudaFuncSetAttribute(mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(mlp_wgrad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kWgradSmem);
  if (e != cudaSuccess) {
    devnet_destroy(&d);
    return fail("kernel attributes", e);
  }
  const int sms = sm_count();
  const int64_t tiles = B / kTile;
  const int tgrid = (int)std::min<int64_t>(tiles, sms);
  const int kslices = (int)std::max<int64_t>(1, std::min<int64_t>(B / 64, sms / kWBlocks));
  const int bias_blocks = (int)std::max<int64_t>(1, std::min<int64_t>(B / 256, 64));
  const int epochs = a.grads_only ? 1 : std::max(1, a.epochs);
  const int64_t steps_per_epoch = n / B;
  const int64_t total = steps_per_epoch * epochs;
  // visiting order: the identity for a gradient check, else a fresh
  // permutation per epoch keyed by the seed
  int hb = 0;
  if (!a.grads_only)
    while ((uint64_t)1 << (2 * hb) < (uint64_t)n) ++hb;
  std::mt19937_64 rng(a.seed);
  const int order_blocks = (int)std::min<int64_t>((n + 255) / 256, 4 * (int64_t)sm_count());
  int64_t step = 0;
  int64_t t_adam = net->steps;
  for (int ep = 0; ep < epochs && e == cudaSuccess; ++ep) {
    mlp_order_kernel<<<order_blocks, 256, 0, s>>>(idx, (uint32_t)n, hb, rng());
    e = cudaMemsetAsync(loss, 0, sizeof(float), s);
    for (int64_t st = 0; st < steps_per_epoch && e == cudaSuccess; ++st, ++step) {
      TrainKArgs ka{};
      ka.p = d.p;
      ka.iquv = a.iquv;
      ka.y16 = y16;
      ka.idx = idx + st * B;
      ka.n = B;
      ka.nl = a.nl;
      ka.gscale = 2.f / (float)(B * kOut);
      ka.zspill = z;
      ka.loss = loss;
      ka.err = err;
      mlp_train_kernel<<<tgrid, kThreads, kSmemBytes, s>>>(nm, am, ka);
      mlp_bias_grad_kernel<<<dim3(bias_blocks, 3), 256, 0, s>>>(g1, g2, g3, B, field(grad, offsetof(gm_mlp, b1)),
                                                                field(grad, offsetof(gm_mlp, b2)),
                                                                field(grad, offsetof(gm_mlp, b3)));
      WgradArgs wa{};
      wa.dw1 = field(grad, offsetof(gm_mlp, w1));
      wa.dw2 = field(grad, offsetof(gm_mlp, w2));
      wa.dw3 = field(grad, offsetof(gm_mlp, w3));
      wa.rows = B;
      wa.kslices = kslices;
      wa.err = err;
      mlp_wgrad_kernel<<<kWBlocks * kslices, kWThreads, kWgradSmem, s>>>(wm, wa);
      if (!a.grads_only) {
        ++t_adam;
        const double lr = a.lr * 0.5 * (1.0 + std::cos(M_PI * (double)step / (double)std::max<int64_t>(1, total)));
        const float c1 = (float)(1.0 / (1.0 - std::pow(0.9, (double)t_adam)));
        const float c2 = (float)(1.0 / (1.0 - std::pow(0.999, (double)t_adam)));
        mlp_adam_kernel<<<(kParams + 255) / 256, 256, 0, s>>>(d.p, grad, m1, m2, d.pack, (float)lr,
                                                              a.weight_decay, c1, c2);
      }
      e = cudaGetLastError();
    }
    if (e == cudaSuccess && loss_out) {
      float sum = 0.f;
      e = cudaMemcpyAsync(&sum, loss, sizeof(float), cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      loss_out[ep] = sum / (float)((double)steps_per_epoch * B * kOut);
    }
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  int code = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&code, err, sizeof(int), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && code != 0) e = cudaErrorLaunchTimeout;
  if (e == cudaSuccess) {
    const int64_t steps0 = net->steps;
    if (a.grads_only) {
      if (grads_out) e = cudaMemcpy(grads_out, grad, sizeof(gm_mlp), cudaMemcpyDeviceToHost);
    } else {
      e = cudaMemcpy(net, d.p, sizeof(gm_mlp), cudaMemcpyDeviceToHost);
      net->steps = steps0 + total;
    }
  }
  devnet_destroy(&d);
  return e == cudaSuccess ? e : fail(code ? "a training kernel gave up waiting" : "training", e);
}

}  // namespace mlp
}  // namespace gm
