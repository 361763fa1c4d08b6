// cj_pixel.cuh -- one MCU tile of the fused pixel stage: TMA bulk copy of
// the tile's coefficient blocks into shared memory, dequantise + integer iDCT
// (rows, then columns) into per-component plane tiles, then nearest chroma
// upsampling + YCbCr->RGB (or a grey copy) straight into the output image.
// Used by the per-image kernel (pixel.cu) and the batch kernel (batch.cu).
#pragma once
#include <stdint.h>

#include "cj_core.h"
#include "cj_idct.cuh"
#include "cj_tc.cuh"

#define CJ_PIX_THREADS 256

// iDCT arithmetic of the pixel stage (include/pixelTransformGPU.h CJ_IDCT_*)
#define CJ_PIX_IDCT_INT 0  // the reference's fixed point: bit-exact
#define CJ_PIX_IDCT_TC 2   // FP16 hi/lo tensor cores, FP32 accumulation
// Output formats (include/cudajpeg.h CJ_OUTPUT_*)
#define CJ_OUT_RGB 0     // interleaved RGB (grey: one plane), the reference's output
#define CJ_OUT_PLANAR 1  // Y plane, then Cb and Cr planes at chroma resolution
#define CJ_OUT_NV12 2    // Y plane, then Cb/Cr interleaved at chroma resolution
#define CJ_OUT_RGB_FANCY 3  // interleaved RGB with fancy (triangle) chroma upsampling

// ---------------------------------------------------------------- TMA helpers
__device__ __forceinline__ uint32_t cj_smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void cj_mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(cj_smem_addr(bar)), "r"(count)
               : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void cj_bulk_load(void* dst, const void* src, uint32_t bytes,
                                             uint64_t* bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(cj_smem_addr(bar)),
               "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          cj_smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(cj_smem_addr(bar))
      : "memory");
}

// Wait for phase `parity` of the barrier; gives up after a bounded number of
// polls and returns false.
__device__ __forceinline__ bool cj_mbar_wait(uint64_t* bar, uint32_t parity) {
  for (uint32_t it = 0; it < (1u << 22); it++) {
    uint32_t ok;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(ok)
        : "r"(cj_smem_addr(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
    if (it > 64) __nanosleep(32);
  }
  return false;
}

struct CJPixGeom {
  int nch, bpm, mcux, mcuy, width, height;
  int hmax, vmax, xs, ys;
  int T;                  // MCUs per tile (one MCU row)
  int y_stride, c_stride; // tile plane strides (bytes)
  int ipr_shift;          // log2 of 8-pixel items per tile row (T * hmax)
  int sc1_off, tmp_off, y_off, cb_off, cr_off;
  int a_off, b_off, big_off;  // tensor-core form: A tile, Kronecker basis, range flags
  int cw, ch;             // chroma plane size (planar outputs)
};

// Row-pass results of one block: 8 rows of 8 int32, padded to 72 words so
// that the column pass (lanes = 4 blocks x 8 columns) reads 32 distinct banks.
#define CJ_TMP_STRIDE 72

// Blocks of one tensor-core tile: the rows of its 128-row A operand.  The
// CUDA-core forms keep at most 64 blocks per tile (cj_pix_tile_mcus).
#ifndef CJ_TC_MAXB
#define CJ_TC_MAXB 128
#endif
// Coefficient buffers of a tensor-core tile (TMA bulk copies in flight) and
// the CTAs per SM its kernel is compiled for (its register cap).  Measured on
// the 1024-image mix: one buffer at 3 CTAs/SM (60 KB of shared memory each)
// runs the pixel stage in 1.04 ms, two buffers at 2 CTAs/SM in 1.24 ms, and
// 64-block tiles at 4 CTAs/SM in 1.42-1.48 ms.
#ifndef CJ_TC_NBUF
#define CJ_TC_NBUF 1
#endif
#ifndef CJ_TC_MINB
#define CJ_TC_MINB 3
#endif
// Threads of a tensor-core pixel CTA: the epilogue splits each block's 64
// outputs over CJ_TC_THREADS / 128 threads (warps w, w + 4, ... share TMEM
// lanes 32 (w mod 4) .. +31), CJ_TC_COLS columns = CJ_TC_ROWS pixel rows each.
#ifndef CJ_TC_THREADS
#define CJ_TC_THREADS 256
#endif
#define CJ_TC_COLS (64 / (CJ_TC_THREADS / 128))
#define CJ_TC_ROWS (8 / (CJ_TC_THREADS / 128))
static_assert(CJ_TC_THREADS == 256 || CJ_TC_THREADS == 512, "two or four epilogue threads per block");

struct alignas(16) CJPixSmemParams {
  int32_t q[4][64];       // dequantisation tables, natural order (int32: no unpacking per row)
  uint16_t qh[4][64];     // the same as FP16 bit patterns (tensor-core form)
  uint16_t boff[CJ_TC_MAXB];  // per block of the tile: smem offset of its 8x8 destination
  uint8_t bc[CJ_TC_MAXB];     // per block of the tile: component
  uint8_t bq[CJ_TC_MAXB];     // per block of the tile: quantisation table
};

// MCUs per tile: 128 output pixels across, at most 64 blocks of coefficients.
CJ_HD int cj_pix_tile_mcus(int hmax, int bpm) {
  int T = 16 / hmax;
  if (T < 1) T = 1;
  while (T > 1 && T * bpm > 64) T >>= 1;
  return T;
}

// MCUs per tensor-core tile: as many as fill the A operand (at most
// CJ_TC_MAXB blocks), at most 1024 output pixels across.  The tile's plane
// samples (64 per block) then fit in 64 * CJ_TC_MAXB bytes.
CJ_HD int cj_pix_tile_mcus_tc(int hmax, int bpm) {
  int T = 128 / hmax;
  if (T < 1) T = 1;
  while (T > 1 && T * bpm > CJ_TC_MAXB) T >>= 1;
  return T;
}

// The tile layout needs full-resolution luma and chroma at an exact power-of-
// two fraction of it (true for every SOF0 geometry the parser accepts except
// 1-pixel-wide or -high oddities).
CJ_HD int cj_pix_check(const CJScanParams* hp) {
  if (hp->comp_sx[0] != hp->hmax || hp->comp_sy[0] != hp->vmax) return 2;  // UNSUPPORTED_ERROR
  if (hp->nch == 3 && ((hp->comp_sx[1] << hp->xshift) != hp->hmax ||
                       (hp->comp_sy[1] << hp->yshift) != hp->vmax))
    return 2;
  return 0;
}

// Shared-memory layout of a tile; returns its size in bytes.  With nbuf = 2
// the two coefficient buffers sit at fixed offsets 0 and 8 KiB (a tile holds
// at most 64 blocks), so tiles of different geometry -- consecutive tiles of
// a batch CTA may come from different images -- never overlap the current
// tile's working space.  The tensor-core form (tc) has a layout of its own
// whose regions do not depend on the geometry either: the plane tiles first
// (64 bytes per block: at most CJ_TC_SC_OFF), then CJ_TC_NBUF coefficient
// buffers of CJ_TC_MAXB blocks, the 128-row FP16 A tile (16 KiB, in the
// 128-byte swizzled layout, which must start on a 1024-byte boundary: the
// region holds 1 KiB of slack and the kernel aligns the tile inside it), the
// hi/lo Kronecker basis (16 KiB) and one range flag per block row.
#define CJ_TC_COEF_BYTES (CJ_TC_MAXB * 128)
#define CJ_TC_SC_OFF (CJ_TC_MAXB * 64)
#define CJ_TC_A_OFF (CJ_TC_SC_OFF + CJ_TC_NBUF * CJ_TC_COEF_BYTES)
#define CJ_TC_A_BYTES (16384 + 1024)
#define CJ_TC_B_OFF (CJ_TC_A_OFF + CJ_TC_A_BYTES)
#define CJ_TC_BIG_OFF (CJ_TC_B_OFF + 16384)
#define CJ_TC_SMEM_BYTES (CJ_TC_BIG_OFF + CJ_TC_MAXB * 8)
CJ_HD size_t cj_pix_layout(CJPixGeom* g, int csx, int csy, int nbuf = 1, bool tc = false) {
  g->y_stride = g->T * 8 * g->hmax;
  g->c_stride = g->nch == 3 ? g->T * 8 * csx : 0;
  g->ipr_shift = 0;
  while ((1 << g->ipr_shift) < g->T * g->hmax) g->ipr_shift++;
  const int csz_tc = g->nch == 3 ? g->c_stride * 8 * csy : 0;
  if (tc) {  // plane tiles at 0 (64 bytes per block, multiples of 64 each)
    g->y_off = 0;
    g->cb_off = g->y_stride * 8 * g->vmax;
    g->cr_off = g->cb_off + csz_tc;
    g->sc1_off = CJ_TC_COEF_BYTES;  // from one coefficient buffer to the next
    g->tmp_off = 0;                 // unused
    g->a_off = CJ_TC_A_OFF;
    g->b_off = CJ_TC_B_OFF;
    g->big_off = CJ_TC_BIG_OFF;
    return CJ_TC_SMEM_BYTES;
  }
  const size_t coef_bytes = (size_t)g->T * g->bpm * 128;
  size_t off = coef_bytes;
  g->sc1_off = 0;
  if (nbuf == 2) {
    g->sc1_off = 8192;
    off = 16384;
  }
  g->a_off = g->b_off = g->big_off = 0;
  g->tmp_off = (int)off;
  off += (size_t)g->T * g->bpm * CJ_TMP_STRIDE * 4;
  g->y_off = (int)off;
  off += (size_t)g->y_stride * 8 * g->vmax;
  off = (off + 15) & ~(size_t)15;
  g->cb_off = (int)off;
  size_t csz = g->nch == 3 ? (size_t)g->c_stride * 8 * csy : 0;
  off += csz;
  g->cr_off = (int)off;
  off += csz;
  return (off + 15) & ~(size_t)15;
}

// Thread 0: start the TMA bulk copy of tile (mrow, mc0)'s coefficient blocks
// (contiguous in MCU scan order) into `dst`, completing on `bar`.
__device__ __forceinline__ void cj_pixel_issue(const int16_t* __restrict__ coef, const CJPixGeom& g,
                                               int mrow, int mc0, int16_t* dst, uint64_t* bar) {
  const int nm = min(g.T, g.mcux - mc0);
  const int16_t* src = coef + ((int64_t)mrow * g.mcux + mc0) * g.bpm * 64;
  // earlier generic reads of `dst` are ordered before the async-proxy write
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  cj_bulk_load(dst, src, (uint32_t)(nm * g.bpm) * 128u, bar);
}

__device__ __forceinline__ uint32_t cj_rgb_pack(int yy, int cb, int cr, int k) {
  // byte k of the pixel's R, G, B (JFIF integer transform, CPUonly/src/pixelTransformCPU.c:152-154)
  return k == 0 ? cj_clip8((yy + 359 * cr + 128) >> 8)
                : (k == 1 ? cj_clip8((yy - 88 * cb - 183 * cr + 128) >> 8) : cj_clip8((yy + 454 * cb + 128) >> 8));
}

// The same transform split per chroma sample: with yy = Y << 8 a multiple of
// 256, (yy + t) >> 8 == Y + (t >> 8) for every t (arithmetic shift = floor),
// so R = clip(Y + dR) etc. with the d terms computed once per chroma sample
// and shared by the 1, 2 or 4 pixels it covers.
struct CJChromaTerms {
  int r, g, b;
};
__device__ __forceinline__ CJChromaTerms cj_chroma_terms(int cb_byte, int cr_byte) {
  const int cb = cb_byte - 128, cr = cr_byte - 128;
  return {(359 * cr + 128) >> 8, (-88 * cb - 183 * cr + 128) >> 8, (454 * cb + 128) >> 8};
}

// Four int32 values saturated to [0, 255] and packed little-endian
// (v0 in the low byte): cvt.pack.sat packs two saturated bytes under the
// low half of its third operand.
__device__ __forceinline__ uint32_t cj_pack_sat4(int v0, int v1, int v2, int v3) {
  uint32_t hi, d;
  asm("cvt.pack.sat.u8.s32.b32 %0, %1, %2, 0;" : "=r"(hi) : "r"(v3), "r"(v2));
  asm("cvt.pack.sat.u8.s32.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(v1), "r"(v0), "r"(hi));
  return d;
}

// 8 pixels of one row (Y bytes in yv) -> 24 RGB bytes in six words; pixel k
// takes chroma terms d[k >> dshift].  R = clip(Y + dR) etc. (cj_chroma_terms).
__device__ __forceinline__ void cj_rgb8(uint2 yv, const CJChromaTerms* d, int dshift, uint32_t* wds) {
  int c[24];
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const int Y = (int)(((k < 4 ? yv.x : yv.y) >> (8 * (k & 3))) & 0xFF);
    const CJChromaTerms t = d[k >> dshift];
    c[3 * k] = Y + t.r;
    c[3 * k + 1] = Y + t.g;
    c[3 * k + 2] = Y + t.b;
  }
#pragma unroll
  for (int w = 0; w < 6; w++) wds[w] = cj_pack_sat4(c[4 * w], c[4 * w + 1], c[4 * w + 2], c[4 * w + 3]);
}

// Per-image part of the tile setup (all threads; the caller's barrier after
// it orders it before use): dequantisation tables and,
// for every block of a full tile, its destination in the plane tiles, its
// component and its quantisation table.  A shorter last tile of an MCU row
// uses a prefix of the same entries.
__device__ __forceinline__ void cj_pixel_setup(const CJScanParams& prmr, const CJPixGeom& g, CJPixSmemParams* Pp) {
  const CJScanParams* prm = &prmr;
  CJPixSmemParams& P = *Pp;
  const int nblk = g.T * g.bpm;
  for (int k = threadIdx.x; k < 4 * 64; k += blockDim.x) {
    const int q = prm->qnat[k >> 6][k & 63];
    P.q[k >> 6][k & 63] = q;
    P.qh[k >> 6][k & 63] = __half_as_ushort(__int2half_rn(q));  // exact: 8-bit tables
  }
  for (int k = threadIdx.x; k < nblk; k += blockDim.x) {
    const int mi = k / g.bpm, ph = k - mi * g.bpm;
    const int c = prm->phase_comp[ph], bl = prm->phase_blk[ph], sxc = prm->comp_sx[c];
    const int bx = mi * sxc + bl % sxc, by = bl / sxc;
    const int base = c == 0 ? g.y_off : (c == 1 ? g.cb_off : g.cr_off);
    const int ps = c == 0 ? g.y_stride : g.c_stride;
    P.boff[k] = (uint16_t)(base + by * 8 * ps + bx * 8);
    P.bc[k] = (uint8_t)c;
    P.bq[k] = prm->comp_q[c];
  }
}

// A thread whose wait for the tile's coefficient copy (or, in the
// tensor-core form, for its MMAs) ran out sets cj_tile_fail; the CTA reads it
// after its next barrier and leaves together, with the image's error
// recorded.  Every kernel that runs tiles clears it before its first barrier.
static __shared__ int cj_tile_fail;

__device__ __forceinline__ bool cj_pixel_failed(CJStatus* st) {
  if (!cj_tile_fail) return false;
  if (threadIdx.x == 0) atomicMax(&st->dec_err_key, ~((unsigned long long)CJ_DEV_CAPACITY));
  return true;
}

// Integer iDCT of a tile's blocks (coefficients in `sc`) into the plane
// tiles: row pass with dequantisation on load, then column pass with level
// shift and clip.  Ends with a barrier; false if a wait of the tile failed.
__device__ __forceinline__ bool cj_pixel_idct_int(const CJPixGeom& g, int nblk, const int16_t* sc, uint8_t* smem,
                                                  const CJPixSmemParams& P, CJStatus* st) {
  int* tmp = reinterpret_cast<int*>(smem + g.tmp_off);
  // Row pass: one thread per (block, row); dequantise on load.
  for (int t = threadIdx.x; t < nblk * 8; t += blockDim.x) {
    const int k = t >> 3, r = t & 7;
    const int4* qp = reinterpret_cast<const int4*>(&P.q[P.bq[k]][r * 8]);
    const int4 qa = qp[0], qb = qp[1];
    const int q[8] = {qa.x, qa.y, qa.z, qa.w, qb.x, qb.y, qb.z, qb.w};
    uint4 raw = *reinterpret_cast<const uint4*>(sc + k * 64 + r * 8);
    int v[8];
    cj_unpack_dequant32(raw, q, v);
    cj_idct_row(v);
    int4* o = reinterpret_cast<int4*>(tmp + k * CJ_TMP_STRIDE + r * 8);
    o[0] = make_int4(v[0], v[1], v[2], v[3]);
    o[1] = make_int4(v[4], v[5], v[6], v[7]);
  }
  __syncthreads();
  if (cj_pixel_failed(st)) return false;

  // Column pass: one thread per (block, column pair); the two columns' 8
  // samples go into the plane tile as one 16-bit store per row.
  for (int t = threadIdx.x; t < nblk * 4; t += blockDim.x) {
    const int k = t >> 2, c0 = (t & 3) * 2;
    int d0[8], d1[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int2 v = *reinterpret_cast<const int2*>(tmp + k * CJ_TMP_STRIDE + j * 8 + c0);
      d0[j] = v.x;
      d1[j] = v.y;
    }
    int o0[8], o1[8];
    cj_idct_col_s(d0, o0);
    cj_idct_col_s(d1, o1);
    const int ps = P.bc[k] == 0 ? g.y_stride : g.c_stride;
    uint8_t* dst = smem + P.boff[k] + c0;
#pragma unroll
    for (int j = 0; j < 8; j++) *reinterpret_cast<uint16_t*>(dst + j * ps) = (uint16_t)cj_level2(o0[j], o1[j]);
  }
  __syncthreads();
  return true;
}

// Tensor-memory state of a CTA running the tensor-core form: its 64-column
// accumulator, the MMA-completion barrier and the phase it waits for next,
// the float basis [u][x] (range fallback).
struct CJTcState {
  uint32_t tmem;
  uint64_t* bar;
  uint32_t parity;
  const float* basis;
  uint8_t* a_tile;  // the swizzled A tile: inside the A region, on a 1024-byte boundary
};

// Tensor-core iDCT of a tile's blocks (at most CJ_TC_MAXB, rows of the
// 128-row A tile), in three steps the tile loop (batch.cu) interleaves with
// the neighbouring tiles' work:
//
// cj_tc_build_a: A row kb = block kb's 64 coefficients dequantised in FP16,
// the DC biased by TC_DC_BIAS (exact below 2048; a block row at or above it
// sets the row's range flag),
// in the 128-byte swizzled layout (conflict-free stores of a block's 8 rows),
// then the proxy fence that makes the rows visible to the MMAs.
__device__ __forceinline__ void cj_tc_build_a(int nblk, const int16_t* sc, uint8_t* sA, uint8_t* big,
                                              const CJPixSmemParams& P) {
  // a thread always builds row v = threadIdx.x & 7 (blockDim.x is a multiple
  // of 8); row 0's DC gets the rounding bias (TC_DC_BIAS)
  const __half2 bias = __halves2half2(__float2half_rn((threadIdx.x & 7) ? 0.f : TC_DC_BIAS), __float2half_rn(0.f));
  for (int t = threadIdx.x; t < nblk * 8; t += blockDim.x) {
    const int kb = t >> 3, v = t & 7;
    const uint4 raw = *reinterpret_cast<const uint4*>(sc + kb * 64 + v * 8);
    const uint4 qv = *reinterpret_cast<const uint4*>(&P.qh[P.bq[kb]][v * 8]);
    const uint32_t rw[4] = {raw.x, raw.y, raw.z, raw.w}, qw[4] = {qv.x, qv.y, qv.z, qv.w};
    uint32_t p[4], acc = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const __half2 c2 = __halves2half2(__short2half_rn((short)(rw[j] & 0xFFFFu)), __short2half_rn((short)(rw[j] >> 16)));
      __half2 pr = __hmul2(c2, *reinterpret_cast<const __half2*>(&qw[j]));
      if (j == 0) pr = __hadd2(pr, bias);
      p[j] = *reinterpret_cast<const uint32_t*>(&pr);
      // per half: |x| >= 2048 (0x6800, NaN and Inf above) sets bit 15 of
      // (bits & 0x7FFF) + 0x1800; no carry crosses into the upper half
      acc |= (p[j] & 0x7FFF7FFFu) + 0x18001800u;
    }
    big[t] = (acc & 0x80008000u) != 0;
    *reinterpret_cast<uint4*>(sA + tc_sw128_off(kb, v)) = make_uint4(p[0], p[1], p[2], p[3]);
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// cj_tc_epilogue (after the MMAs' barrier phase completed): D row kb = block
// kb's 64 outputs, read from tensor memory 16 columns (two pixel rows) at a
// time -- warps w and w + 4 share lanes 32 (w & 3) .. +31 and take pixel rows
// 0-3 and 4-7; a warp whose lanes hold no block of the tile skips the reads
// -- floored (the bias did the rounding), level-shifted, clipped and stored
// into the plane tiles.
// `ok` false (the MMAs did not complete): nothing is stored.  Returns true
// for the thread of a block with a range flag set (FP32 redo needed).
__device__ __forceinline__ bool cj_tc_epilogue(const CJPixGeom& g, int nblk, uint8_t* smem, const uint8_t* big,
                                               const CJPixSmemParams& P, const CJTcState& tc, bool ok) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int quad = w & 3, h = w >> 2, kb = 32 * quad + lane;
  if (32 * quad >= nblk) return false;  // warp-uniform
  const uint32_t ta = tc.tmem + ((uint32_t)(32 * quad) << 16) + (uint32_t)(CJ_TC_COLS * h);
  const bool live = ok && kb < nblk;
  const int ps = live && P.bc[kb] != 0 ? g.c_stride : g.y_stride;
  uint8_t* dst = smem + (live ? P.boff[kb] : 0) + CJ_TC_ROWS * h * ps;
#pragma unroll
  for (int j = 0; j < CJ_TC_COLS / 16; j++) {
    float d[16];
    tc_ld16(ta + 16u * j, d);
    if (live) {
#pragma unroll
      for (int y = 0; y < 2; y++)
        *reinterpret_cast<uint2*>(dst + (2 * j + y) * ps) =
            make_uint2(tc_level4(d[8 * y], d[8 * y + 1], d[8 * y + 2], d[8 * y + 3]),
                       tc_level4(d[8 * y + 4], d[8 * y + 5], d[8 * y + 6], d[8 * y + 7]));
    }
  }
  return kb < nblk && h == 0 && *reinterpret_cast<const uint64_t*>(big + kb * 8) != 0;
}

// cj_tc_fallback (rare; the whole CTA): blocks with a range flag redone on
// CUDA cores in FP32, one thread per output sample, from their coefficients
// in global memory (`blocks` = the tile's first block).  Ends with a barrier.
__device__ __forceinline__ void cj_tc_fallback(const CJPixGeom& g, int nblk, const int16_t* __restrict__ blocks,
                                               uint8_t* smem, const uint8_t* big, const CJPixSmemParams& P,
                                               const CJTcState& tc) {
  for (int k = 0; k < nblk; k++) {
    if (!*reinterpret_cast<const uint64_t*>(big + k * 8)) continue;  // the same for every thread
    if (threadIdx.x < 64) {
      const int y = threadIdx.x >> 3, x = threadIdx.x & 7;
      const int16_t* blk = blocks + (int64_t)k * 64;
      const int32_t* q = P.q[P.bq[k]];
      float acc = 0.f;
      for (int v = 0; v < 8; v++) {
        float row = 0.f;
        for (int u = 0; u < 8; u++) row = fmaf((float)(blk[8 * v + u] * q[8 * v + u]), tc.basis[u * 8 + x], row);
        acc = fmaf(row, tc.basis[v * 8 + y], acc);
      }
      const int ps = P.bc[k] == 0 ? g.y_stride : g.c_stride;
      smem[P.boff[k] + y * ps + x] = (uint8_t)cj_clip8(tc_round(acc) + 128);
    }
  }
  __syncthreads();
}

// Nearest upsampling + YCbCr->RGB (or a grey copy) of a tile's plane tiles
// into the output image (CPUonly/src/pixelTransformCPU.c:110-172).
__device__ __forceinline__ void cj_pixel_emit_rgb(uint8_t* __restrict__ out, const CJPixGeom& g, int mrow, int mc0,
                                                  int nm, const uint8_t* smem) {
  const uint8_t* py = smem + g.y_off;
  const uint8_t* pcb = smem + g.cb_off;
  const uint8_t* pcr = smem + g.cr_off;
  const int X0 = mc0 * 8 * g.hmax, Y0 = mrow * 8 * g.vmax;
  const int w = min(nm * 8 * g.hmax, g.width - X0);
  const int h = min(8 * g.vmax, g.height - Y0);
  if (w <= 0 || h <= 0) return;
  if ((g.width & 7) == 0 && (((uintptr_t)out) & 7) == 0) {
    // 8 pixels per item, items laid out (row, 8-pixel column) with a
    // power-of-two number of items per tile row; 8-byte aligned stores
    const int ipr = 1 << g.ipr_shift, per_row = w >> 3;
    for (int t = threadIdx.x; t < (h << g.ipr_shift); t += blockDim.x) {
      const int y = t >> g.ipr_shift, xi = t & (ipr - 1);
      if (xi >= per_row) continue;
      const int x0 = xi * 8;
      const uint2 yv = *reinterpret_cast<const uint2*>(py + y * g.y_stride + x0);
      if (g.nch == 3) {
        const uint8_t* crow_b = pcb + (y >> g.ys) * g.c_stride;
        const uint8_t* crow_r = pcr + (y >> g.ys) * g.c_stride;
        CJChromaTerms d[8];
        int dshift;
        if (g.xs == 1) {  // 4 chroma samples, 4-byte aligned (x0 / 2 is a multiple of 4)
          const uint32_t b4 = *reinterpret_cast<const uint32_t*>(crow_b + (x0 >> 1));
          const uint32_t r4 = *reinterpret_cast<const uint32_t*>(crow_r + (x0 >> 1));
#pragma unroll
          for (int j = 0; j < 4; j++) d[j] = cj_chroma_terms((b4 >> (8 * j)) & 0xFF, (r4 >> (8 * j)) & 0xFF);
          dshift = 1;
        } else if (g.xs == 0) {  // 8 chroma samples, 8-byte aligned
          const uint2 b8 = *reinterpret_cast<const uint2*>(crow_b + x0);
          const uint2 r8 = *reinterpret_cast<const uint2*>(crow_r + x0);
#pragma unroll
          for (int j = 0; j < 8; j++)
            d[j] = cj_chroma_terms(((j < 4 ? b8.x : b8.y) >> (8 * (j & 3))) & 0xFF,
                                   ((j < 4 ? r8.x : r8.y) >> (8 * (j & 3))) & 0xFF);
          dshift = 0;
        } else {  // wider chroma subsampling: per pixel
#pragma unroll
          for (int j = 0; j < 8; j++) d[j] = cj_chroma_terms(crow_b[(x0 + j) >> g.xs], crow_r[(x0 + j) >> g.xs]);
          dshift = 0;
        }
        uint32_t wds[6];
        if (dshift) cj_rgb8(yv, d, 1, wds);
        else cj_rgb8(yv, d, 0, wds);
        uint2* o = reinterpret_cast<uint2*>(out + ((int64_t)(Y0 + y) * g.width + X0 + x0) * 3);
        o[0] = make_uint2(wds[0], wds[1]);
        o[1] = make_uint2(wds[2], wds[3]);
        o[2] = make_uint2(wds[4], wds[5]);
      } else {
        *reinterpret_cast<uint2*>(out + (int64_t)(Y0 + y) * g.width + X0 + x0) = yv;
      }
    }
  } else if (g.nch == 3) {
    for (int t = threadIdx.x; t < w * h; t += blockDim.x) {
      int y = t / w, x = t - y * w;
      int yy = py[y * g.y_stride + x] << 8;
      int ci = (y >> g.ys) * g.c_stride + (x >> g.xs);
      int cb = (int)pcb[ci] - 128, cr = (int)pcr[ci] - 128;
      uint8_t* o = out + ((int64_t)(Y0 + y) * g.width + X0 + x) * 3;
      o[0] = (uint8_t)cj_rgb_pack(yy, cb, cr, 0);
      o[1] = (uint8_t)cj_rgb_pack(yy, cb, cr, 1);
      o[2] = (uint8_t)cj_rgb_pack(yy, cb, cr, 2);
    }
  } else {
    for (int t = threadIdx.x; t < w * h; t += blockDim.x) {
      int y = t / w, x = t - y * w;
      out[(int64_t)(Y0 + y) * g.width + X0 + x] = py[y * g.y_stride + x];
    }
  }
}

// Planar (Y, Cb, Cr planes) or NV12 (Y plane, then Cb/Cr interleaved) copy
// of a tile's plane tiles, chroma at its own resolution (no upsampling, no
// colour transform): the decoded samples themselves.  Chroma planes are
// g.cw x g.ch (the reference's channel width and height, src/format.cu
// decodeSOF); grey images have the Y plane only.
template <int OUT>
__device__ __forceinline__ void cj_pixel_emit_planes(uint8_t* __restrict__ out, const CJPixGeom& g, int mrow,
                                                     int mc0, int nm, const uint8_t* smem) {
  const int X0 = mc0 * 8 * g.hmax, Y0 = mrow * 8 * g.vmax;
  const int w = min(nm * 8 * g.hmax, g.width - X0);
  const int h = min(8 * g.vmax, g.height - Y0);
  const uint8_t* py = smem + g.y_off;
  for (int t = threadIdx.x; t < w * h; t += blockDim.x) {
    const int y = t / w, x = t - y * w;
    out[(int64_t)(Y0 + y) * g.width + X0 + x] = py[y * g.y_stride + x];
  }
  if (g.nch != 3) return;
  const int cs = g.hmax >> g.xs, csy = g.vmax >> g.ys;  // chroma blocks per MCU across / down
  const int cX0 = mc0 * 8 * cs, cY0 = mrow * 8 * csy;
  const int cw = min(nm * 8 * cs, g.cw - cX0), ch = min(8 * csy, g.ch - cY0);
  if (cw <= 0 || ch <= 0) return;
  uint8_t* cbase = out + (int64_t)g.width * g.height;
  const uint8_t* pcb = smem + g.cb_off;
  const uint8_t* pcr = smem + g.cr_off;
  for (int t = threadIdx.x; t < cw * ch; t += blockDim.x) {
    const int y = t / cw, x = t - y * cw;
    const uint8_t b = pcb[y * g.c_stride + x], r = pcr[y * g.c_stride + x];
    const int64_t o = (int64_t)(cY0 + y) * g.cw + cX0 + x;
    if (OUT == CJ_OUT_NV12) {
      cbase[2 * o] = b;
      cbase[2 * o + 1] = r;
    } else {
      cbase[o] = b;
      cbase[(int64_t)g.cw * g.ch + o] = r;
    }
  }
}

// One tile (after cj_pixel_setup for its image), MCU row `mrow`, MCUs
// [mc0, mc0 + T), whose coefficients arrive in `sc` on phase `parity` of
// `bar`: the integer iDCT (MODE) into plane tiles, then the output (OUT) into
// `out`.  Returns false if the copy did not land within the wait bound
// (recorded).  Ends with a barrier, so `sc` and the plane tiles are free
// afterwards.
template <int MODE, int OUT>
__device__ __forceinline__ bool cj_pixel_tile(uint8_t* __restrict__ out, CJStatus* st, const CJPixGeom& g, int mrow,
                                              int mc0, const int16_t* sc, uint8_t* smem, uint64_t* barp,
                                              uint32_t parity, CJPixSmemParams* Pp) {
  const int nm = min(g.T, g.mcux - mc0);
  const int nblk = nm * g.bpm;
  // each thread reads the copied blocks only after its own wait; a wait that
  // ran out is agreed on at the iDCT's first barrier (no barrier here)
  if (!cj_mbar_wait(barp, parity)) cj_tile_fail = 1;
  static_assert(MODE == CJ_PIX_IDCT_INT, "tensor-core tiles run in their own loop (bt_pixel_tiles_tc)");
  if (!cj_pixel_idct_int(g, nblk, sc, smem, *Pp, st)) return false;
  if (OUT == CJ_OUT_RGB) cj_pixel_emit_rgb(out, g, mrow, mc0, nm, smem);
  else cj_pixel_emit_planes<OUT>(out, g, mrow, mc0, nm, smem);
  __syncthreads();
  return true;
}

// The reference output with the reference arithmetic: integer iDCT, RGB.
__device__ __forceinline__ bool cj_pixel_compute(uint8_t* __restrict__ out, CJStatus* st, const CJPixGeom& g,
                                                 int mrow, int mc0, const int16_t* sc, uint8_t* smem,
                                                 uint64_t* barp, uint32_t parity, CJPixSmemParams* Pp) {
  return cj_pixel_tile<CJ_PIX_IDCT_INT, CJ_OUT_RGB>(out, st, g, mrow, mc0, sc, smem, barp, parity, Pp);
}

// Fancy (triangle) upsampling of a cw x ch chroma plane by 2^xs x 2^ys: the
// sample at output (x, y), as the IJG decoder's h2v1 / h1v2 / h2v2 fancy
// upsamplers give it (weights 3/4 and 1/4 toward the nearer and the farther
// sample, alternating rounding biases, edge samples alone at the first and
// last column, the first and last rows repeated above and below); other
// factors replicate.  An optional output mode: the reference upsamples by
// nearest replication (CPUonly/src/pixelTransformCPU.c:110-127).
__device__ __forceinline__ int cj_fancy_at(const uint8_t* __restrict__ pl, int cw, int ch, int xs, int ys, int x,
                                           int y) {
  const int r = min(y >> ys, ch - 1), i = min(x >> xs, cw - 1);
  const bool fancy = (xs == 1 && ys <= 1) || (xs == 0 && ys == 1);
  const uint8_t* row = pl + (int64_t)r * cw;
  if (!fancy) return row[i];
  int nb = r;
  if (ys == 1) nb = (y & 1) ? min(r + 1, ch - 1) : max(r - 1, 0);
  const uint8_t* nrow = pl + (int64_t)nb * cw;
  if (xs == 0) return (3 * row[i] + nrow[i] + ((y & 1) ? 2 : 1)) >> 2;
  if (ys == 0) {
    if (x & 1) return i == cw - 1 ? row[i] : (3 * row[i] + row[i + 1] + 2) >> 2;
    return i == 0 ? row[i] : (3 * row[i] + row[i - 1] + 1) >> 2;
  }
  const int cs = 3 * row[i] + nrow[i];
  if (x & 1) return i == cw - 1 ? (4 * cs + 7) >> 4 : (3 * cs + 3 * row[i + 1] + nrow[i + 1] + 7) >> 4;
  return i == 0 ? (4 * cs + 8) >> 4 : (3 * cs + 3 * row[i - 1] + nrow[i - 1] + 8) >> 4;
}
