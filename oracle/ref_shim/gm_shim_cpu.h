/* Prelude force-included before every reference source in the host (CPU)
 * comparison build.  It maps the CUDA spellings used by the reference's
 * per-pixel routines onto plain host C++:
 *   - execution-space and memory-space qualifiers vanish;
 *   - __fdividef(a, b) becomes a / b and __sincosf becomes sincosf;
 *   - __ldg(p) becomes *p;
 *   - threadIdx / blockIdx / blockDim are per-thread variables that the
 *     driver leaves at 0 / 0 / 1, so every kernel body sees one thread;
 *   - __syncthreads() is a no-op (after the child launches are turned into
 *     loops, no kernel body runs with more than one thread).
 * Nothing here changes arithmetic beyond those substitutions. */
#ifndef GM_SHIM_CPU_H
#define GM_SHIM_CPU_H

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cuda_runtime.h>
#include <cuComplex.h>

#undef __global__
#undef __device__
#undef __host__
#undef __constant__
#undef __shared__
#undef __forceinline__
#define __global__
#define __device__
#define __host__
#define __constant__
#define __shared__
#define __forceinline__ inline

#define __fdividef(a, b) ((a) / (b))
#define __sincosf(x, s, c) sincosf((x), (s), (c))
#define __ldg(p) (*(p))
#define __syncthreads() ((void)0)

extern thread_local uint3 gm_shim_threadIdx;
extern thread_local uint3 gm_shim_blockIdx;
extern thread_local dim3 gm_shim_blockDim;
#define threadIdx gm_shim_threadIdx
#define blockIdx gm_shim_blockIdx
#define blockDim gm_shim_blockDim

#endif
