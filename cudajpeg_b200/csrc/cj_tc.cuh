// cj_tc.cuh -- tensor-core (tcgen05) building blocks of the FP16 hi/lo
// iDCT, shared by the plane kernel (plane.cu) and the batch pixel kernel.
//
// The 2-D iDCT of a block is one linear map on its 64 coefficients:
//   s[8y+x] = sum_{v,u} F[8v+u] * B[v][y] * B[u][x],
//   B[u][x] = c(u)/2 cos((2x+1) u pi / 16), c(0) = 1/sqrt(2)  (T.81 A.3.3)
// so M blocks are one GEMM  D[M x 64] = A[M x 64] * K[64 x 64] with
// K[8v+u][8y+x] = B[v][y] B[u][x].  A holds dequantised coefficients in FP16
// (exact while |value| < 2048); K is split into FP16 halves Khi = fp16(K),
// Klo = fp16(K - Khi) and D = A*Khi + A*Klo accumulates in FP32 in tensor
// memory (tcgen05.mma kind::f16, M = 128, N = 64, K = 16 per instruction).
//
// Shared-memory operands use the K-major no-swizzle canonical layout: 8x8
// "core matrices" of 8 rows x 16 bytes; core (r8, k8) of a 64-wide K operand
// sits at ((r8 * 8 + k8) * 128) bytes.  LBO (next core along K) = 128 B,
// SBO (next 8-row group) = 1024 B.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

// CTAs per SM of a kernel that allocates `tmem_cols` tensor-memory columns
// per CTA, launched with `threads` threads and `dyn_smem` bytes of dynamic
// shared memory.  The runtime's occupancy query answers 1 for every kernel
// that contains tcgen05 instructions (it cannot know how many columns a CTA
// takes), so the residency is worked out here from the kernel's registers
// and static shared memory and the SM's limits: registers (allocated per
// warp in units of 256), shared memory (plus the per-CTA reservation),
// threads, CTA slots, and the 512 columns of tensor memory.  Returns 0 if
// an attribute cannot be read.
static inline int cj_tc_ctas_per_sm(const void* kernel, int threads, size_t dyn_smem, int tmem_cols) {
  cudaFuncAttributes at;
  int dev = 0, regs_sm = 0, smem_sm = 0, smem_rsv = 0, thr_sm = 0, blk_sm = 0;
  if (cudaFuncGetAttributes(&at, kernel) != cudaSuccess || cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&smem_rsv, cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&thr_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&blk_sm, cudaDevAttrMaxBlocksPerMultiprocessor, dev) != cudaSuccess)
    return 0;
  const int warps = (threads + 31) / 32;
  const int regs_warp = ((at.numRegs * 32 + 255) / 256) * 256;
  int n = std::min(thr_sm / (warps * 32), blk_sm);
  if (regs_warp > 0) n = std::min(n, regs_sm / (regs_warp * warps));
  n = std::min(n, (int)((size_t)smem_sm / (at.sharedSizeBytes + dyn_smem + (size_t)smem_rsv)));
  if (tmem_cols > 0) n = std::min(n, 512 / tmem_cols);
  return std::max(n, 0);
}

__device__ __forceinline__ uint32_t tc_core_off(int r, int k) {
  return (uint32_t)((((r >> 3) * 8 + (k >> 3)) * 128) + (r & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint64_t tc_smem_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) |
         ((uint64_t)(1024 >> 4) << 32) | (1ull << 46);
}

// The same K-major operand with the 128-byte swizzle: rows of 128 bytes (the
// whole K = 64 FP16 row) in 8-row atoms of 1024 bytes (SBO), the 16-byte
// chunk c of row r stored at chunk c ^ (r & 7).  The atom must start on a
// 1024-byte boundary; a K step of 16 inside the atom advances the start
// address by 32 bytes (the swizzle is applied to the absolute address).
__device__ __forceinline__ uint32_t tc_sw128_off(int r, int chunk) {
  return (uint32_t)(r * 128 + ((chunk ^ (r & 7)) << 4));
}

__device__ __forceinline__ uint64_t tc_smem_desc_sw128(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | (1ull << 16) | ((uint64_t)(1024 >> 4) << 32) | (1ull << 46) |
         (2ull << 61);
}

// kind::f16, D = F32, A = B = F16, both K-major, N = 64, M = 128
#define TC_IDESC ((1u << 4) | (0u << 7) | (0u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24))

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"((uint32_t)TC_IDESC), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// The 8 MMAs of one 128-block tile (A at a_addr, Khi at b_addr, Klo at
// b_addr + 8 KiB) into the accumulator at tmem, then a commit that arrives
// on `bar` when they are done.  One thread.
__device__ __forceinline__ void tc_idct_mmas(uint32_t tmem, uint32_t a_addr, uint32_t b_addr, uint32_t bar_addr) {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
  for (int kk = 0; kk < 4; kk++) tc_mma(tmem, tc_smem_desc(a_addr + kk * 256), tc_smem_desc(b_addr + kk * 256), kk > 0);
#pragma unroll
  for (int kk = 0; kk < 4; kk++)
    tc_mma(tmem, tc_smem_desc(a_addr + kk * 256), tc_smem_desc(b_addr + 8192 + kk * 256), 1u);
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar_addr)
               : "memory");
}

// tc_idct_mmas with A in the 128-byte swizzled layout (tc_sw128_off).
__device__ __forceinline__ void tc_idct_mmas_asw(uint32_t tmem, uint32_t a_addr, uint32_t b_addr, uint32_t bar_addr) {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
  for (int kk = 0; kk < 4; kk++)
    tc_mma(tmem, tc_smem_desc_sw128(a_addr + kk * 32), tc_smem_desc(b_addr + kk * 256), kk > 0);
#pragma unroll
  for (int kk = 0; kk < 4; kk++)
    tc_mma(tmem, tc_smem_desc_sw128(a_addr + kk * 32), tc_smem_desc(b_addr + 8192 + kk * 256), 1u);
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar_addr)
               : "memory");
}

__device__ __forceinline__ void tc_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
        "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
        "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 32; k++) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ void tc_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 16; k++) v[k] = __uint_as_float(r[k]);
}

// Tensor-memory columns of one CTA (warp 0 allocates and frees; the address
// lands in *slot).  A power of two >= 32.
__device__ __forceinline__ void tc_alloc(uint32_t* slot, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   (uint32_t)__cvta_generic_to_shared(slot)),
               "r"(cols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tc_dealloc(uint32_t tmem, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(cols) : "memory");
}

// Rounding folded into the GEMM: every output of a block gets DC * K[0][n]
// with K[0][n] = 1/8 exactly (B[0][y] B[0][x] = 1/8; its FP16 hi half is
// exact and the lo half zero), so adding TC_DC_BIAS = 4 = 8 * 0.5 to the
// dequantised DC coefficient adds exactly 0.5 to all 64 outputs, and the
// epilogue rounds ties up -- floor(s + 0.5), as the oracle's
// clip(floor(s + 0.5) + 128) and the reference's fixed-point rounding do --
// with a single floor().  Ties are common: a DC-only block's samples are
// DC / 8 exactly, and the hi/lo basis reproduces them exactly.  The biased
// DC stays an integer far inside FP16's exact range (|DC| <= 1024 for 8-bit
// samples).
#define TC_DC_BIAS 4.0f

// Four biased iDCT outputs -> the bytes clip(floor(v) + 128), v0 in the low
// byte: signed saturating packs to [-128, 127], then a flip of each top bit
// (s + 128 == s ^ 0x80 for a signed byte).
__device__ __forceinline__ uint32_t tc_level4(float a, float b, float c, float d) {
  uint32_t hi, r;
  asm("cvt.pack.sat.s8.s32.b32 %0, %1, %2, 0;" : "=r"(hi) : "r"(__float2int_rd(d)), "r"(__float2int_rd(c)));
  asm("cvt.pack.sat.s8.s32.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(__float2int_rd(b)), "r"(__float2int_rd(a)), "r"(hi));
  return r ^ 0x80808080u;
}

// The FP32 range fallback's rounding: floor(v + 0.5), ties up as above
// (v + 0.5 is exact for |v| < 2^22).
__device__ __forceinline__ int tc_round(float v) { return __float2int_rd(v + 0.5f); }
