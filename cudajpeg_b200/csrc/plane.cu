// plane.cu -- per-component plane iDCT (cjIDCTPlane), the C launcher that
// replaces the reference's __global__ iDCT_GPU (include/pixelTransformGPU.h:6-10,
// src/pixelTransformGPU.cu:25-142), in three arithmetic forms:
//   CJ_IDCT_INT  the reference's fixed-point separable iDCT, bit-exact;
//   CJ_IDCT_F32  an FP32 separable iDCT (orthonormal DCT-II basis), rounded
//                to nearest at the end; the baseline for the tensor-core form;
//   CJ_IDCT_TC   FP16 hi/lo Kronecker basis on tensor cores (k_idct_tc).
// Input is the quantised int16 block buffer decodeScanGPU leaves on the
// device; the component's blocks are gathered from the MCU-interleaved order.
#include <cuda_fp16.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>

#include "../../include/pixelTransformGPU.h"
#include "cj_internal.h"
#include "cj_idct.cuh"
#include "cj_pixel.cuh"
#include "cj_tc.cuh"

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

// constant memory is per device: one upload on each
static bool g_basis_ready[64];

int cj_upload_basis() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return CUDA_MEM_ERROR;
  if (g_basis_ready[dev]) return 0;
  float b[64];
  for (int u = 0; u < 8; u++)
    for (int x = 0; x < 8; x++)
      b[u * 8 + x] = (float)((u ? 0.5 : 0.5 / sqrt(2.0)) * cos((2 * x + 1) * u * 3.14159265358979323846 / 16.0));
  CJ_CUDA_TRY(cudaMemcpyToSymbol(c_idct_basis, b, sizeof(b)), CUDA_MEM_ERROR);
  g_basis_ready[dev] = true;
  return 0;
}


// ---------------------------------------------------------------- tensor cores
//
// The plane iDCT as one GEMM per 128-block tile (cj_tc.cuh): D = A * Khi +
// A * Klo with A the dequantised coefficients in FP16 (exact: |value| <= 2048
// for every block a real encoder produces; larger blocks are redone on CUDA
// cores in FP32), FP32 accumulation in tensor memory, a tcgen05.ld epilogue.

#define TC_M 128
#define TC_THREADS 128

// per device: Khi then Klo, core-matrix layout
#define CJ_MAX_DEVICES 64
static uint16_t* g_tc_basis_dev[CJ_MAX_DEVICES];
static std::mutex g_tc_basis_mu;

// One thread's block of a 128-block tile: its 8 coefficient rows as loaded
// (quantised int16), where it lives and where its pixels go.
struct TcRows {
  uint4 r[8];
  int64_t gb;  // block index in the coefficient buffer
  int bx, by;  // block position in the plane
  bool live;
};

template <bool RAW>
__device__ __forceinline__ void tc_fetch(const CJPlaneArgs& a, int64_t t, TcRows& x) {
  const int64_t kb = t * TC_M + threadIdx.x;
  x.live = kb < a.nblocks;
  x.bx = x.by = 0;
  x.gb = 0;
  if (x.live) x.gb = RAW ? kb : cj_plane_src(a, kb, &x.bx, &x.by);
#pragma unroll
  for (int k8 = 0; k8 < 8; k8++)
    x.r[k8] = x.live ? __ldg(reinterpret_cast<const uint4*>(a.coef + x.gb * 64 + k8 * 8)) : make_uint4(0, 0, 0, 0);
}

// RAW = true: write the FP32 values (before +128 / rounding / clip) of block
// list entries to raw_out; RAW = false: write pixels into the plane.
//
// Per 128-block tile: each of the 128 threads dequantises its block into the
// FP16 A tile (a block whose values FP16 cannot hold exactly is flagged),
// thread 0 issues the 8 MMAs, and -- while they run and during the epilogue
// -- every thread already has the loads of its block of the CTA's next tile
// in flight (register prefetch).  The epilogue reads the block's row of D
// from tensor memory in two halves of 32 values (pixel rows 0-3, 4-7).
// Flagged blocks are listed in shared memory and redone afterwards by the
// whole CTA on CUDA cores in FP32 (one thread per output pixel), a branch the
// CTA takes together, so the common path carries no call and no spills.
template <bool RAW>
__global__ void __launch_bounds__(TC_THREADS, 4) k_idct_tc(CJPlaneArgs a, const uint16_t* __restrict__ basis,
                                                          float* raw_out, int* status) {
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint64_t bar;
  __shared__ uint32_t tmem_base;
  __shared__ int16_t q[64];
  __shared__ int32_t q32[64];
  __shared__ float sbasis[64];
  __shared__ int s_nbig, s_big[TC_M];
  uint8_t* sA = smem;               // 128 x 64 fp16 = 16 KiB
  uint8_t* sB = smem + 16384;       // Khi, Klo: 2 x 64 x 64 fp16 = 16 KiB
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int k = tid; k < 16384 / 16; k += TC_THREADS)
    reinterpret_cast<uint4*>(sB)[k] = __ldg(reinterpret_cast<const uint4*>(basis) + k);
  if (tid < 64) {
    q[tid] = a.qnat[tid];
    q32[tid] = a.qnat[tid];
    sbasis[tid] = c_idct_basis[tid];
  }
  if (warp == 0) tc_alloc(&tmem_base, 64);
  if (tid == 0) cj_mbar_init(&bar, 1);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  const uint32_t aaddr = cj_smem_addr(sA), baddr = cj_smem_addr(sB);
  if (tid == 0) s_nbig = 0;
  const int64_t ntiles = (a.nblocks + TC_M - 1) / TC_M;
  uint32_t parity = 0;
  TcRows nx;
  if ((int64_t)blockIdx.x < ntiles) tc_fetch<RAW>(a, blockIdx.x, nx);
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    // ---- A tile: thread m owns block m; dequantise, check range, FP16
    const TcRows cur = nx;
    bool big = false;
#pragma unroll
    for (int k8 = 0; k8 < 8; k8++) {
      int v[8];
      cj_unpack_dequant(cur.r[k8], q + k8 * 8, v);
      uint32_t h[4];
#pragma unroll
      for (int j = 0; j < 4; j++) {
        big |= (v[2 * j] > 2048 || v[2 * j] < -2048 || v[2 * j + 1] > 2048 || v[2 * j + 1] < -2048);
        __half2 p2 = __floats2half2_rn((float)v[2 * j], (float)v[2 * j + 1]);
        h[j] = *reinterpret_cast<uint32_t*>(&p2);
      }
      *reinterpret_cast<uint4*>(sA + tc_core_off(tid, k8 * 8)) = make_uint4(h[0], h[1], h[2], h[3]);
    }
    if (big && cur.live) s_big[atomicAdd(&s_nbig, 1)] = tid;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) tc_idct_mmas(tmem, aaddr, baddr, cj_smem_addr(&bar));
    // ---- the next tile's loads fly while the MMAs run and the epilogue works
    if (t + gridDim.x < ntiles) tc_fetch<RAW>(a, t + gridDim.x, nx);
    const bool ok = cj_mbar_wait(&bar, parity);
    parity ^= 1;
    if (!__syncthreads_and(ok)) {
      if (tid == 0) atomicExch(status, 1);
      cj_mbar_wait(&bar, parity ^ 1);  // give an in-flight MMA a bounded chance to land
      break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // ---- D row m = block m: two halves of 32 FP32 values (pixel rows 0-3, 4-7)
#pragma unroll 1
    for (int h = 0; h < 2; h++) {
      float d[32];
      tc_ld32(tmem + ((uint32_t)(32 * warp) << 16) + 32u * h, d);
      if (!cur.live) continue;
      if (RAW) {
        float4* o = reinterpret_cast<float4*>(raw_out + (cur.gb * 64 + 32 * h));
#pragma unroll
        for (int k = 0; k < 8; k++) o[k] = make_float4(d[4 * k], d[4 * k + 1], d[4 * k + 2], d[4 * k + 3]);
      } else {
#pragma unroll
        for (int y = 0; y < 4; y++)
          *reinterpret_cast<uint2*>(a.plane + (int64_t)(cur.by * 8 + 4 * h + y) * a.stride + cur.bx * 8) =
              make_uint2(tc_level4(d[8 * y], d[8 * y + 1], d[8 * y + 2], d[8 * y + 3]),
                         tc_level4(d[8 * y + 4], d[8 * y + 5], d[8 * y + 6], d[8 * y + 7]));
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();  // TMEM and the A tile are free for the next tile
    const int nbig = s_nbig;
    if (nbig) {  // CTA-uniform, rare: FP32 redo of the flagged blocks
      for (int bi = 0; bi < nbig; bi++) {
        const int64_t kb = t * TC_M + s_big[bi];
        int bx = 0, by = 0;
        const int64_t gb = RAW ? kb : cj_plane_src(a, kb, &bx, &by);
        if (tid < 64) {
          const int y = tid >> 3, x = tid & 7;
          const int16_t* blk = a.coef + gb * 64;
          float acc = 0.f;
          for (int v = 0; v < 8; v++) {
            float row = 0.f;
            for (int u = 0; u < 8; u++) row = fmaf((float)(blk[8 * v + u] * q32[8 * v + u]), sbasis[u * 8 + x], row);
            acc = fmaf(row, sbasis[v * 8 + y], acc);
          }
          if (RAW) raw_out[gb * 64 + tid] = acc;
          else a.plane[(int64_t)(by * 8 + y) * a.stride + bx * 8 + x] = (uint8_t)cj_clip8(__float2int_rn(acc) + 128);
        }
      }
      __syncthreads();
      if (tid == 0) s_nbig = 0;
      __syncthreads();
    }
  }
  __syncthreads();
  if (warp == 0) tc_dealloc(tmem, 64);
}

// Khi / Klo of the Kronecker basis in the K-major core-matrix layout of B
// (row = pixel n = 8y+x, column = coefficient k = 8v+u).
static uint16_t* cj_tc_basis() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= CJ_MAX_DEVICES) return nullptr;
  std::lock_guard<std::mutex> lock(g_tc_basis_mu);
  if (g_tc_basis_dev[dev]) return g_tc_basis_dev[dev];
  static uint16_t h[2 * 64 * 64];
  double b[8][8];
  for (int u = 0; u < 8; u++)
    for (int x = 0; x < 8; x++)
      b[u][x] = (u ? 0.5 : 0.5 / sqrt(2.0)) * cos((2 * x + 1) * u * 3.14159265358979323846 / 16.0);
  for (int n = 0; n < 64; n++)
    for (int k = 0; k < 64; k++) {
      int y = n >> 3, x = n & 7, v = k >> 3, u = k & 7;
      double w = b[v][y] * b[u][x];
      __half hi = __double2half(w);
      __half lo = __double2half(w - (double)__half2float(hi));
      size_t off = (((n >> 3) * 8 + (k >> 3)) * 128 + (n & 7) * 16 + (k & 7) * 2) / 2;
      h[off] = *reinterpret_cast<uint16_t*>(&hi);
      h[4096 + off] = *reinterpret_cast<uint16_t*>(&lo);
    }
  uint16_t* d = nullptr;
  if (cudaMalloc(&d, sizeof(h)) != cudaSuccess) return nullptr;
  if (cudaMemcpy(d, h, sizeof(h), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(d);
    return nullptr;
  }
  g_tc_basis_dev[dev] = d;
  return d;
}

const uint16_t* cj_tc_basis_device() { return cj_tc_basis(); }

static int* g_tc_status_dev[CJ_MAX_DEVICES];  // per device: set when an MMA wait ran out

static int cj_idct_tc_launch(const CJPlaneArgs& a, float* raw, bool is_raw, cudaStream_t s) {
  const uint16_t* basis = cj_tc_basis();
  if (cj_upload_basis() || !basis) return CUDA_MEM_ERROR;
  int dev = 0;
  CJ_CUDA_TRY(cudaGetDevice(&dev), CUDA_MEM_ERROR);
  int*& status = g_tc_status_dev[dev];  // dev < CJ_MAX_DEVICES: cj_tc_basis checked it
  if (!status) {
    CJ_CUDA_TRY(cudaMalloc(&status, sizeof(int)), CUDA_MEM_ERROR);
    CJ_CUDA_TRY(cudaMemset(status, 0, sizeof(int)), CUDA_MEM_ERROR);
  }
  static bool attr[CJ_MAX_DEVICES];  // function attributes are set per device
  const int smem = 32768;
  if (!attr[dev]) {
    CJ_CUDA_TRY(cudaFuncSetAttribute(k_idct_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                CUDA_KERNEL_LAUNCH_ERROR);
    CJ_CUDA_TRY(cudaFuncSetAttribute(k_idct_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                CUDA_KERNEL_LAUNCH_ERROR);
    attr[dev] = true;
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int64_t ntiles = (a.nblocks + TC_M - 1) / TC_M;
  // CTAs per SM: as many as registers, shared memory and tensor memory (64
  // columns each) allow
  int per_sm = cj_tc_ctas_per_sm(is_raw ? (const void*)k_idct_tc<true> : (const void*)k_idct_tc<false>, TC_THREADS,
                                 smem, 64);
  if (per_sm < 1) return CUDA_KERNEL_LAUNCH_ERROR;
  unsigned grid = (unsigned)std::min<int64_t>(ntiles, (int64_t)sms * per_sm);
  if (grid < 1) grid = 1;
  if (is_raw)
    k_idct_tc<true><<<grid, TC_THREADS, smem, s>>>(a, basis, raw, status);
  else
    k_idct_tc<false><<<grid, TC_THREADS, smem, s>>>(a, basis, raw, status);
  CJ_CUDA_TRY(cudaGetLastError(), CUDA_KERNEL_LAUNCH_ERROR);
  return 0;
}

int cj_idct_tc_plane(const CJPlaneArgs& a, cudaStream_t s) { return cj_idct_tc_launch(a, nullptr, false, s); }

int cj_idct_tc_raw(const int16_t* coef, const int16_t* qnat, float* out, int64_t nblocks, cudaStream_t s) {
  CJPlaneArgs a;
  memset(&a, 0, sizeof(a));
  a.coef = coef;
  a.qnat = qnat;
  a.nblocks = nblocks;
  return cj_idct_tc_launch(a, out, true, s);
}

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
