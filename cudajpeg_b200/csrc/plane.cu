// plane.cu -- per-component plane iDCT (cjIDCTPlane), the C launcher that
// replaces the reference's __global__ iDCT_GPU (include/pixelTransformGPU.h:6-10,
// src/pixelTransformGPU.cu:25-142), in three arithmetic forms:
//   CJ_IDCT_INT  the reference's fixed-point separable iDCT, bit-exact;
//   CJ_IDCT_F32  an FP32 separable iDCT (orthonormal DCT-II basis), rounded
//                to nearest at the end; the baseline for the tensor-core form;
//   CJ_IDCT_TC   FP16 hi/lo Kronecker basis on tensor cores (k_idct_tc).
// Input is the quantised int16 block buffer decodeScanGPU leaves on the
// device; the component's blocks are gathered from the MCU-interleaved order.
#include <cuda.h>
#include <cudaTypedefs.h>
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
// A * Klo with A the dequantised coefficients in FP16 (exact: |value| < 2048
// for every block a real encoder produces; larger blocks are redone on CUDA
// cores in FP32), FP32 accumulation in tensor memory, a tcgen05.ld epilogue.

#define TC_M 128
#ifndef TC_THREADS
#define TC_THREADS 256
#endif
// The epilogue splits each block's 64 outputs over TC_THREADS / 128 threads
// (warps w, w + 4, ... share TMEM lanes 32 (w mod 4) .. +31): TC_COLS columns
// (TC_ROWS pixel rows) each.
#define TC_GROUPS (TC_THREADS / 128)
#define TC_COLS (64 / TC_GROUPS)
#define TC_ROWS (8 / TC_GROUPS)
static_assert(TC_THREADS == 256 || TC_THREADS == 512, "two or four threads per block in the epilogue");
#ifndef TC_STAGES
#define TC_STAGES 2                 // coefficient tiles in flight per CTA (TMA ring)
#endif
#ifndef TC_ABUF
#define TC_ABUF 1                   // A tiles (with one, a tile's A build waits for the previous MMAs)
#endif
#ifndef TC_MINB
#define TC_MINB 3                   // CTAs per SM the kernel is compiled for
#endif
#define TC_TILE_BYTES 16384         // 128 blocks x 64 int16
// dynamic shared memory: 1 KiB of alignment slack, the TMA ring, the
// swizzled A tile(s), the hi/lo basis, three slots of per-row range flags
#define TC_SMEM (1024 + TC_STAGES * TC_TILE_BYTES + TC_ABUF * 16384 + 16384 + 3 * 1024)

// per device: Khi then Klo, core-matrix layout
#define CJ_MAX_DEVICES 64
static uint16_t* g_tc_basis_dev[CJ_MAX_DEVICES];
static std::mutex g_tc_basis_mu;

// Thread 0: the TMA copy of a 128-block tile of the component (3-D tensor
// map: 64 coefficients x the component's blocks in an MCU x MCUs, box
// {64, per, 128 / per}) into `dst`, completing on `bar`.  Coordinates past
// the last MCU read zeros.
__device__ __forceinline__ void tc_tile_load(void* dst, const CUtensorMap* map, int mcu0, uint64_t* bar) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(cj_smem_addr(bar)),
               "r"((uint32_t)TC_TILE_BYTES)
               : "memory");
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(cj_smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(0), "r"(mcu0), "r"(cj_smem_addr(bar))
      : "memory");
}

// RAW = true: write the FP32 values (before +128 / rounding / clip) of block
// list entries to raw_out; RAW = false: write pixels into the plane.
//
// A persistent CTA runs its tiles k = 0, 1, ... (tile blockIdx.x + k *
// gridDim.x) through a software pipeline with one barrier per tile:
//   - TC_STAGES - 1 tiles ahead, thread 0 has TMA copies in flight into a
//     ring of shared-memory stages (mbarrier per stage);
//   - iteration k: every thread dequantises 4 coefficient rows of tile k
//     into the FP16 A tile (TC_ABUF of them, 128-byte swizzled; with one,
//     after tile k-1's MMAs have read it; for pixels the DC is biased by
//     TC_DC_BIAS; a row FP16 cannot hold exactly sets its range flag)
//     -- barrier -- thread 0 issues tile k's 8 MMAs into one of two
//     64-column accumulators and the next copy, while every thread runs tile
//     k-1's epilogue: wait for its MMAs, read its block's half row of D (32
//     values) with tcgen05.ld, floor (the bias did the rounding), level-
//     shift and clip, store.  A thread whose block has a range flag computes
//     its 32 outputs in FP32 from the coefficients in global memory instead.
// Range flags keep three slots, so a thread still in tile k-1's epilogue
// never sees tile k+1's flags.  A wait that runs out marks `status` and the
// tile's output is not written; the pipeline keeps its barriers.
template <bool RAW>
__global__ void __launch_bounds__(TC_THREADS, TC_MINB) k_idct_tc(const __grid_constant__ CUtensorMap tmap, CJPlaneArgs a,
                                                          const uint16_t* __restrict__ basis, float* raw_out,
                                                          int* status) {
  extern __shared__ uint8_t smem_raw[];
  __shared__ uint64_t full[TC_STAGES], mma_done[2];
  __shared__ uint32_t tmem_base;
  __shared__ int32_t q32[64];
  __shared__ float sbasis[64];
  uint8_t* smem = smem_raw + ((1024u - (cj_smem_addr(smem_raw) & 1023u)) & 1023u);
  uint8_t* stages = smem;
  uint8_t* sA = smem + TC_STAGES * TC_TILE_BYTES;  // A tile(s), 1024-byte aligned
  uint8_t* sB = sA + TC_ABUF * 16384;
  uint8_t* flags = sB + 16384;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int k = tid; k < 16384 / 16; k += TC_THREADS)
    reinterpret_cast<uint4*>(sB)[k] = __ldg(reinterpret_cast<const uint4*>(basis) + k);
  if (tid < 64) {
    q32[tid] = a.qnat[tid];
    sbasis[tid] = c_idct_basis[tid];
  }
  if (warp == 0) tc_alloc(&tmem_base, 128);
  if (tid == 0) {
    for (int s = 0; s < TC_STAGES; s++) cj_mbar_init(&full[s], 1);
    cj_mbar_init(&mma_done[0], 1);
    cj_mbar_init(&mma_done[1], 1);
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  const int64_t ntiles = (a.nblocks + TC_M - 1) / TC_M;
  const int64_t K = (int64_t)blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const int per = a.sx * a.sy, per_shift = __ffs(per) - 1;  // a power of two
  const int mcus_per_tile = TC_M / per;
  auto issue = [&](int64_t k) {
    const int64_t tile = blockIdx.x + k * gridDim.x;
    const int s = (int)(k % TC_STAGES);
    tc_tile_load(stages + s * TC_TILE_BYTES, &tmap, (int)(tile * mcus_per_tile), &full[s]);
  };
  if (tid == 0)
    for (int64_t k = 0; k < K && k < TC_STAGES - 1; k++) issue(k);
  // this thread always converts coefficient row v = tid & 7 of its blocks:
  // the row's 8 quantisation steps as FP16 pairs, once
  const int v = tid & 7;
  uint32_t qh[4];
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const __half2 q2 = __floats2half2_rn((float)q32[8 * v + 2 * j], (float)q32[8 * v + 2 * j + 1]);
    qh[j] = *reinterpret_cast<const uint32_t*>(&q2);
  }
  // row 0's DC carries the rounding bias (TC_DC_BIAS) for pixels; raw values
  // are left unbiased
  const __half2 bias = __floats2half2_rn(!RAW && v == 0 ? TC_DC_BIAS : 0.f, 0.f);
  bool bad = false;
  for (int64_t k = 0; k <= K; k++) {
    if (k < K) {  // ---- A tile of local tile k
      const int s = (int)(k % TC_STAGES);
      if (!cj_mbar_wait(&full[s], (uint32_t)((k / TC_STAGES) & 1))) bad = true;
      const uint8_t* st = stages + s * TC_TILE_BYTES;
      uint8_t* a_k = sA + (k % TC_ABUF) * 16384;
      // with one A tile, tile k - 1's MMAs must have read it (bounded wait;
      // the epilogue below waits for the same phase)
      if (TC_ABUF == 1 && k >= 1 && !cj_mbar_wait(&mma_done[(k - 1) & 1], (uint32_t)(((k - 1) >> 1) & 1)))
        bad = true;
      uint8_t* fl = flags + (k % 3) * 1024;
#pragma unroll
      for (int j = 0; j < 1024 / TC_THREADS; j++) {
        const int t = tid + TC_THREADS * j, kb = t >> 3;  // row (kb, v) sits at t * 16
        const uint4 raw = *reinterpret_cast<const uint4*>(st + t * 16);
        const uint32_t rw[4] = {raw.x, raw.y, raw.z, raw.w};
        uint32_t p[4], acc = 0;
#pragma unroll
        for (int i = 0; i < 4; i++) {
          const __half2 c2 = __halves2half2(__short2half_rn((short)(rw[i] & 0xFFFFu)),
                                            __short2half_rn((short)(rw[i] >> 16)));
          __half2 pr = __hmul2(c2, *reinterpret_cast<const __half2*>(&qh[i]));
          if (i == 0) pr = __hadd2(pr, bias);
          p[i] = *reinterpret_cast<const uint32_t*>(&pr);
          // per half: |x| >= 2048 (0x6800, NaN and Inf above) sets bit 15 of
          // (bits & 0x7FFF) + 0x1800; no carry crosses into the upper half
          acc |= (p[i] & 0x7FFF7FFFu) + 0x18001800u;
        }
        fl[t] = (acc & 0x80008000u) != 0;
        *reinterpret_cast<uint4*>(a_k + tc_sw128_off(kb, v)) = make_uint4(p[0], p[1], p[2], p[3]);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (k < K && tid == 0) {  // ---- tile k's MMAs, then the copy TC_STAGES - 1 tiles ahead
      tc_idct_mmas_asw(tmem + (uint32_t)(k & 1) * 64u, cj_smem_addr(sA + (k % TC_ABUF) * 16384), cj_smem_addr(sB),
                       cj_smem_addr(&mma_done[k & 1]));
      if (k + TC_STAGES - 1 < K) issue(k + TC_STAGES - 1);
    }
    if (k >= 1) {  // ---- epilogue of local tile k - 1
      const int64_t kk = k - 1;
      const bool ok = cj_mbar_wait(&mma_done[kk & 1], (uint32_t)((kk >> 1) & 1));
      if (!ok) bad = true;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int quad = warp & 3, h = warp >> 2, m = 32 * quad + lane;
      const int64_t kb = (blockIdx.x + kk * gridDim.x) * TC_M + m;
      const bool live = ok && kb < a.nblocks;
      const bool flagged = live && *reinterpret_cast<const uint64_t*>(flags + (kk % 3) * 1024 + m * 8) != 0;
      int bx = 0, by = 0;
      int64_t gb = 0;
      if (live && RAW) {
        gb = kb;
      } else if (live) {  // cj_plane_src in 32-bit arithmetic (the launcher bounds the MCU count below 2^31)
        const uint32_t mcu = (uint32_t)kb >> per_shift, loc = (uint32_t)kb & (uint32_t)(per - 1);
        const uint32_t mrow = mcu / (uint32_t)a.mcux, mcol = mcu - mrow * (uint32_t)a.mcux;
        bx = (int)(mcol * a.sx + loc % (uint32_t)a.sx);
        by = (int)(mrow * a.sy + loc / (uint32_t)a.sx);
        gb = (int64_t)mcu * a.bpm + a.first + loc;
      }
      const uint32_t ta = tmem + (uint32_t)(kk & 1) * 64u + ((uint32_t)(32 * quad) << 16) + (uint32_t)(TC_COLS * h);
#pragma unroll
      for (int j = 0; j < TC_COLS / 16; j++) {
        float d[16];
        tc_ld16(ta + 16u * j, d);
        if (!live || flagged) continue;
        if (RAW) {
          float4* o = reinterpret_cast<float4*>(raw_out + (gb * 64 + TC_COLS * h + 16 * j));
#pragma unroll
          for (int i = 0; i < 4; i++) o[i] = make_float4(d[4 * i], d[4 * i + 1], d[4 * i + 2], d[4 * i + 3]);
        } else {
#pragma unroll
          for (int y = 0; y < 2; y++)
            *reinterpret_cast<uint2*>(a.plane + (int64_t)(by * 8 + TC_ROWS * h + 2 * j + y) * a.stride + bx * 8) =
                make_uint2(tc_level4(d[8 * y], d[8 * y + 1], d[8 * y + 2], d[8 * y + 3]),
                           tc_level4(d[8 * y + 4], d[8 * y + 5], d[8 * y + 6], d[8 * y + 7]));
        }
      }
      if (flagged) {  // rare: this thread's TC_COLS outputs (its TC_ROWS pixel rows) in FP32
        const int16_t* blk = a.coef + gb * 64;
#pragma unroll 1
        for (int x = 0; x < 8; x++) {
          float col[8];
#pragma unroll 1
          for (int vv = 0; vv < 8; vv++) {
            float r = 0.f;
            for (int u = 0; u < 8; u++) r = fmaf((float)(blk[8 * vv + u] * q32[8 * vv + u]), sbasis[u * 8 + x], r);
            col[vv] = r;
          }
#pragma unroll 1
          for (int y = TC_ROWS * h; y < TC_ROWS * (h + 1); y++) {
            float s = 0.f;
            for (int vv = 0; vv < 8; vv++) s = fmaf(col[vv], sbasis[vv * 8 + y], s);
            if (RAW) raw_out[gb * 64 + y * 8 + x] = s;
            else a.plane[(int64_t)(by * 8 + y) * a.stride + bx * 8 + x] = (uint8_t)cj_clip8(tc_round(s) + 128);
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (bad) atomicExch(status, 1);
  if (warp == 0) tc_dealloc(tmem, 128);
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

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime
// (no link-time dependency on libcuda)
static PFN_cuTensorMapEncodeTiled_v12000 cj_encode_tiled() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

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
  const int per = a.sx * a.sy;
  if (per < 1 || per > 16 || (per & (per - 1)) || a.bpm <= 0) return PROGRAMMER_ERROR;
  const int64_t nmcu = a.nblocks / per;
  // block indices stay in 32 bits (the epilogue's arithmetic)
  if (nmcu < 1 || a.nblocks > ((int64_t)1 << 31) - TC_M) return PROGRAMMER_ERROR;
  // the component's blocks as a 3-D tensor: 64 coefficients x `per` blocks
  // in an MCU x MCUs, starting at its first block (16-byte aligned: 128 bytes
  // per block); tiles are 128 / per MCUs
  PFN_cuTensorMapEncodeTiled_v12000 encode = cj_encode_tiled();
  if (!encode) return CUDA_KERNEL_LAUNCH_ERROR;
  CUtensorMap map;
  const cuuint64_t dims[3] = {64, (cuuint64_t)per, (cuuint64_t)nmcu};
  const cuuint64_t strides[2] = {128, (cuuint64_t)a.bpm * 128};
  const cuuint32_t box[3] = {64, (cuuint32_t)per, (cuuint32_t)(TC_M / per)};
  const cuuint32_t estr[3] = {1, 1, 1};
  if (encode(&map, CU_TENSOR_MAP_DATA_TYPE_UINT16, 3, (void*)(a.coef + (int64_t)a.first * 64), dims, strides, box,
             estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return PROGRAMMER_ERROR;
  static bool attr[CJ_MAX_DEVICES];  // function attributes are set per device
  if (!attr[dev]) {
    CJ_CUDA_TRY(cudaFuncSetAttribute(k_idct_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM),
                CUDA_KERNEL_LAUNCH_ERROR);
    CJ_CUDA_TRY(cudaFuncSetAttribute(k_idct_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM),
                CUDA_KERNEL_LAUNCH_ERROR);
    attr[dev] = true;
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t ntiles = (a.nblocks + TC_M - 1) / TC_M;
  // persistent CTAs: as many per SM as registers, shared memory and tensor
  // memory (128 columns each) allow.  L2 fills are promoted to 128 bytes
  // (one block): a component's blocks are 128-byte runs at a stride of the
  // MCU's blocks, and 256-byte promotion read 1.5x the bytes on 4:4:4.
  const int per_sm = cj_tc_ctas_per_sm(is_raw ? (const void*)k_idct_tc<true> : (const void*)k_idct_tc<false>,
                                       TC_THREADS, TC_SMEM, 128);
  if (per_sm < 1) return CUDA_KERNEL_LAUNCH_ERROR;
  unsigned grid = (unsigned)std::min<int64_t>(ntiles, (int64_t)sms * per_sm);
  if (grid < 1) grid = 1;
  if (is_raw)
    k_idct_tc<true><<<grid, TC_THREADS, TC_SMEM, s>>>(map, a, basis, raw, status);
  else
    k_idct_tc<false><<<grid, TC_THREADS, TC_SMEM, s>>>(map, a, basis, raw, status);
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
  a.bpm = a.sx = a.sy = a.mcux = 1;
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
