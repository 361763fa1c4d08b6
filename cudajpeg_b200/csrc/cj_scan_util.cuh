// cj_scan_util.cuh -- warp / block prefix sums used by the destuffer and the
// segment and subsequence scans.
#pragma once
#include <stdint.h>

#define CJ_FULL 0xFFFFFFFFu

// Inclusive warp scan of an int2.
__device__ __forceinline__ int2 cj_warp_inclusive(int2 v) {
  int lane = threadIdx.x & 31;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    int ax = __shfl_up_sync(CJ_FULL, v.x, d);
    int ay = __shfl_up_sync(CJ_FULL, v.y, d);
    if (lane >= d) {
      v.x += ax;
      v.y += ay;
    }
  }
  return v;
}

// Exclusive block scan of an int2 over blockDim.x (a multiple of 32, <= 1024)
// threads.  `smem` holds 33 int2.  Returns the exclusive prefix; *total gets
// the block sum.  Contains __syncthreads: call from every thread.
__device__ __forceinline__ int2 cj_block_exclusive(int2 v, int2* smem, int2* total) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int2 inc = cj_warp_inclusive(v);
  if (lane == 31) smem[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    int2 w = lane < nw ? smem[lane] : make_int2(0, 0);
    int2 wi = cj_warp_inclusive(w);
    if (lane < nw) smem[lane] = make_int2(wi.x - w.x, wi.y - w.y);
    if (lane == nw - 1) smem[32] = wi;
  }
  __syncthreads();
  int2 base = smem[warp];
  int2 tot = smem[32];
  __syncthreads();
  *total = tot;
  return make_int2(base.x + inc.x - v.x, base.y + inc.y - v.y);
}
