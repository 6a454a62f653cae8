/* Prelude force-included before every reference source in the sm_100a
 * comparison build.  It changes one thing: device-side malloc/free go
 * through a guard.  The reference takes each thread's scratch from the
 * device heap and does not check for NULL; the guard counts any failed
 * allocation and hands back a fixed sink buffer instead, so heap exhaustion
 * yields a reported failure (the harness rejects the run) rather than a
 * NULL dereference on the device.  Every allocation the reference makes for
 * up to 50 wavelength samples fits in the sink. */
#ifndef GM_SHIM_GPU_H
#define GM_SHIM_GPU_H

#include <cstdlib>
#include <cuda_runtime.h>

__device__ void* gm_shim_device_malloc(size_t n);
__device__ void gm_shim_device_free(void* p);

#ifdef __CUDA_ARCH__
#define malloc(n) gm_shim_device_malloc(n)
#define free(p) gm_shim_device_free(p)
#endif

#endif
