// plane.cu -- per-component plane iDCT (cjIDCTPlane), the C launcher that
// replaces the reference's __global__ iDCT_GPU (include/pixelTransformGPU.h:6-10,
// src/pixelTransformGPU.cu:25-142), in two CUDA-core arithmetic forms:
//   CJ_IDCT_INT  the reference's fixed-point separable iDCT, bit-exact;
//   CJ_IDCT_F32  an FP32 separable iDCT (orthonormal DCT-II basis), rounded
//                to nearest at the end; the baseline for the tensor-core form
//                in idct_tc.cu.
// Input is the quantised int16 block buffer decodeScanGPU leaves on the
// device; the component's blocks are gathered from the MCU-interleaved order.
#include <math.h>
#include <stdio.h>

#include "../../include/pixelTransformGPU.h"
#include "cj_internal.h"
#include "cj_idct.cuh"

#define CJ_PLANE_BLOCKS 32   // 8x8 blocks per CTA
#define CJ_PLANE_THREADS 256  // one thread per (block, row)

__constant__ float c_idct_basis[64];  // [u][x] = C(u)/2 cos((2x+1)u pi/16)

struct CJPlaneArgs {
  const int16_t* coef;
  const int16_t* qnat;
  uint8_t* plane;
  int bpm, first, sx, sy, mcux, stride;
  int64_t nblocks;  // blocks of this component
};

// Global block index (MCU-interleaved) and plane origin of component block kb.
__device__ __forceinline__ int64_t cj_plane_src(const CJPlaneArgs& a, int64_t kb, int* bx, int* by) {
  int per = a.sx * a.sy;
  int64_t mcu = kb / per;
  int loc = (int)(kb - mcu * per);
  int64_t mrow = mcu / a.mcux;
  int mcol = (int)(mcu - mrow * a.mcux);
  *bx = mcol * a.sx + loc % a.sx;
  *by = (int)(mrow * a.sy + loc / a.sx);
  return mcu * a.bpm + a.first + loc;
}

template <int MODE>
__global__ void __launch_bounds__(CJ_PLANE_THREADS) k_idct_plane(CJPlaneArgs a) {
  __shared__ __align__(16) int tmp_i[CJ_PLANE_BLOCKS * 64];
  __shared__ __align__(16) uint8_t tile[CJ_PLANE_BLOCKS * 64];
  __shared__ int16_t q[64];
  float* tmp_f = reinterpret_cast<float*>(tmp_i);
  if (threadIdx.x < 64) q[threadIdx.x] = a.qnat[threadIdx.x];
  __syncthreads();
  const int kl = threadIdx.x >> 3, r = threadIdx.x & 7;
  const int64_t kb = (int64_t)blockIdx.x * CJ_PLANE_BLOCKS + kl;
  int bx = 0, by = 0;
  const bool live = kb < a.nblocks;
  int64_t gb = live ? cj_plane_src(a, kb, &bx, &by) : 0;
  if (live) {
    uint4 raw = __ldg(reinterpret_cast<const uint4*>(a.coef + gb * 64 + r * 8));
    int v[8];
    cj_unpack_dequant(raw, q + r * 8, v);
    if (MODE == CJ_IDCT_INT) {
      cj_idct_row(v);
      int4* o = reinterpret_cast<int4*>(tmp_i + kl * 64 + r * 8);
      o[0] = make_int4(v[0], v[1], v[2], v[3]);
      o[1] = make_int4(v[4], v[5], v[6], v[7]);
    } else {
      float o[8];
      cj_idct8_f32(v, c_idct_basis, o);
#pragma unroll
      for (int x = 0; x < 8; x++) tmp_f[kl * 64 + r * 8 + x] = o[x];
    }
  }
  __syncthreads();
  if (live) {
    const int col = r;
    uint32_t o[8];
    if (MODE == CJ_IDCT_INT) {
      int d[8];
#pragma unroll
      for (int j = 0; j < 8; j++) d[j] = tmp_i[kl * 64 + j * 8 + col];
      cj_idct_col(d, o);
    } else {
      float d[8], s[8];
#pragma unroll
      for (int j = 0; j < 8; j++) d[j] = tmp_f[kl * 64 + j * 8 + col];
      cj_idct8_f32f(d, c_idct_basis, s);
#pragma unroll
      for (int j = 0; j < 8; j++) o[j] = cj_clip8(__float2int_rn(s[j]) + 128);
    }
#pragma unroll
    for (int j = 0; j < 8; j++) tile[kl * 64 + j * 8 + col] = (uint8_t)o[j];
  }
  __syncthreads();
  if (live) {
    uint2 row = *reinterpret_cast<const uint2*>(tile + kl * 64 + r * 8);
    *reinterpret_cast<uint2*>(a.plane + (int64_t)(by * 8 + r) * a.stride + bx * 8) = row;
  }
}

// Raw FP32 iDCT values (before +128, rounding and clip) of a block list: the
// precision measurement against the FP64 oracle.
__global__ void __launch_bounds__(CJ_PLANE_THREADS)
k_idct_raw_f32(const int16_t* __restrict__ coef, const int16_t* __restrict__ qnat, float* out,
               int64_t nblocks) {
  __shared__ float tmp[CJ_PLANE_BLOCKS * 64];
  __shared__ int16_t q[64];
  if (threadIdx.x < 64) q[threadIdx.x] = qnat[threadIdx.x];
  __syncthreads();
  const int kl = threadIdx.x >> 3, r = threadIdx.x & 7;
  const int64_t kb = (int64_t)blockIdx.x * CJ_PLANE_BLOCKS + kl;
  const bool live = kb < nblocks;
  if (live) {
    uint4 raw = __ldg(reinterpret_cast<const uint4*>(coef + kb * 64 + r * 8));
    int v[8];
    cj_unpack_dequant(raw, q + r * 8, v);
    float o[8];
    cj_idct8_f32(v, c_idct_basis, o);
#pragma unroll
    for (int x = 0; x < 8; x++) tmp[kl * 64 + r * 8 + x] = o[x];
  }
  __syncthreads();
  if (live) {
    float d[8], s[8];
#pragma unroll
    for (int j = 0; j < 8; j++) d[j] = tmp[kl * 64 + j * 8 + r];
    cj_idct8_f32f(d, c_idct_basis, s);
#pragma unroll
    for (int j = 0; j < 8; j++) out[kb * 64 + j * 8 + r] = s[j];
  }
}

static int cj_basis_ready = -1;

int cj_upload_basis() {
  if (cj_basis_ready == 1) return 0;
  float b[64];
  for (int u = 0; u < 8; u++)
    for (int x = 0; x < 8; x++)
      b[u * 8 + x] = (float)((u ? 0.5 : 0.5 / sqrt(2.0)) * cos((2 * x + 1) * u * 3.14159265358979323846 / 16.0));
  CJ_CUDA_TRY(cudaMemcpyToSymbol(c_idct_basis, b, sizeof(b)), CUDA_MEM_ERROR);
  cj_basis_ready = 1;
  return 0;
}

int cj_idct_tc_plane(const CJPlaneArgs& a, cudaStream_t s);  // idct_tc.cu

extern "C" int cjIDCTPlane(const short* d_coef, int bpm, int first, int samples_x, int samples_y,
                           int mcux, int mcuy, const short* d_qnat, unsigned char* d_plane,
                           int stride, int mode, void* stream) {
  if (!d_coef || !d_qnat || !d_plane || bpm <= 0 || samples_x <= 0 || samples_y <= 0 ||
      mcux <= 0 || mcuy <= 0 || first < 0 || first + samples_x * samples_y > bpm ||
      stride < mcux * samples_x * 8 || (stride & 7))
    return PROGRAMMER_ERROR;
  CJPlaneArgs a;
  a.coef = (const int16_t*)d_coef;
  a.qnat = (const int16_t*)d_qnat;
  a.plane = d_plane;
  a.bpm = bpm;
  a.first = first;
  a.sx = samples_x;
  a.sy = samples_y;
  a.mcux = mcux;
  a.stride = stride;
  a.nblocks = (int64_t)mcux * mcuy * samples_x * samples_y;
  cudaStream_t s = (cudaStream_t)stream;
  unsigned grid = (unsigned)((a.nblocks + CJ_PLANE_BLOCKS - 1) / CJ_PLANE_BLOCKS);
  switch (mode) {
    case CJ_IDCT_INT: k_idct_plane<CJ_IDCT_INT><<<grid, CJ_PLANE_THREADS, 0, s>>>(a); break;
    case CJ_IDCT_F32:
      if (cj_upload_basis()) return CUDA_MEM_ERROR;
      k_idct_plane<CJ_IDCT_F32><<<grid, CJ_PLANE_THREADS, 0, s>>>(a);
      break;
    case CJ_IDCT_TC: return cj_idct_tc_plane(a, s);
    default: return PROGRAMMER_ERROR;
  }
  CJ_CUDA_TRY(cudaGetLastError(), CUDA_KERNEL_LAUNCH_ERROR);
  return 0;
}

int cj_idct_tc_raw(const int16_t* coef, const int16_t* qnat, float* out, int64_t nblocks,
                   cudaStream_t s);  // idct_tc.cu

extern "C" int cjIDCTBlocksRaw(const short* d_coef, long long nblocks, const short* d_qnat,
                               float* d_out, int mode, void* stream) {
  if (!d_coef || !d_qnat || !d_out || nblocks < 0) return PROGRAMMER_ERROR;
  if (!nblocks) return 0;
  cudaStream_t s = (cudaStream_t)stream;
  if (mode == CJ_IDCT_F32) {
    if (cj_upload_basis()) return CUDA_MEM_ERROR;
    unsigned grid = (unsigned)((nblocks + CJ_PLANE_BLOCKS - 1) / CJ_PLANE_BLOCKS);
    k_idct_raw_f32<<<grid, CJ_PLANE_THREADS, 0, s>>>((const int16_t*)d_coef, (const int16_t*)d_qnat,
                                                     d_out, nblocks);
    CJ_CUDA_TRY(cudaGetLastError(), CUDA_KERNEL_LAUNCH_ERROR);
    return 0;
  }
  if (mode == CJ_IDCT_TC)
    return cj_idct_tc_raw((const int16_t*)d_coef, (const int16_t*)d_qnat, d_out, nblocks, s);
  return PROGRAMMER_ERROR;
}
