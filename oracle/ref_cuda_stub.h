/*
 * ref_cuda_stub.h -- host-only stand-ins for the handful of CUDA runtime
 * names that the reference's host sources (src/format.cu, src/decodeScanCPU.cu)
 * use, so those files compile with g++ into oracle/_ref/ as a coefficient
 * oracle.  TEST INFRASTRUCTURE ONLY.
 *
 * Device buffers are never read on the host path that the oracle runs, so
 * "device" allocations are tiny placeholders and host->device copies are
 * dropped (the reference sizes some of them at 8x-24x the file size).
 */
#ifndef REF_CUDA_STUB_H
#define REF_CUDA_STUB_H
#include <stdlib.h>
#include <string.h>

#define __host__
#define __device__
#define __global__

enum ref_stub_error { cudaSuccess = 0, cudaErrorMemoryAllocation = 2 };
enum ref_stub_kind { cudaMemcpyHostToDevice = 1, cudaMemcpyDeviceToHost = 2 };

template <class T>
static inline int cudaMalloc(T **p, size_t) {
  *p = (T *)malloc(16);
  return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
static inline int cudaFree(void *p) { free(p); return cudaSuccess; }
static inline int cudaMemcpy(void *, const void *, size_t, int) { return cudaSuccess; }
#endif
