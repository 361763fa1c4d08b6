// cj_pixel.cuh -- one MCU tile of the fused pixel stage: TMA bulk copy of
// the tile's coefficient blocks into shared memory, dequantise + integer iDCT
// (rows, then columns) into per-component plane tiles, then nearest chroma
// upsampling + YCbCr->RGB (or a grey copy) straight into the output image.
// Used by the per-image kernel (pixel.cu) and the batch kernel (batch.cu).
#pragma once
#include <stdint.h>

#include "cj_core.h"
#include "cj_idct.cuh"

#define CJ_PIX_THREADS 256

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
  int sc1_off, tmp_off, y_off, cb_off, cr_off;
};

struct CJPixSmemParams {
  int16_t q[4][64];
  uint8_t pc[CJ_MAX_BPM], pb[CJ_MAX_BPM];
  uint8_t cq[4], csx[4], csy[4];
};

// MCUs per tile: 128 output pixels across, at most 64 blocks of coefficients.
CJ_HD int cj_pix_tile_mcus(int hmax, int bpm) {
  int T = 16 / hmax;
  if (T < 1) T = 1;
  while (T > 1 && T * bpm > 64) T >>= 1;
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
// tile's working space.
CJ_HD size_t cj_pix_layout(CJPixGeom* g, int csx, int csy, int nbuf = 1) {
  g->y_stride = g->T * 8 * g->hmax;
  g->c_stride = g->nch == 3 ? g->T * 8 * csx : 0;
  const size_t coef_bytes = (size_t)g->T * g->bpm * 128;
  size_t off = coef_bytes;
  g->sc1_off = 0;
  if (nbuf == 2) {
    g->sc1_off = 8192;
    off = 16384;
  }
  g->tmp_off = (int)off;
  off += (size_t)g->T * g->bpm * 256;
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

// One tile, MCU row `mrow`, MCUs [mc0, mc0 + T), whose coefficients arrive
// in `sc` on phase `parity` of `bar`: dequantise + integer iDCT into plane
// tiles, then nearest upsampling + YCbCr->RGB (or a grey copy) into `out`.
// Returns false if the copy did not land within the wait bound (recorded).
// Ends with a barrier, so `sc` and the plane tiles are free afterwards.
__device__ __forceinline__ bool cj_pixel_compute(const CJScanParams& prmr, uint8_t* __restrict__ out,
                                                 CJStatus* st, const CJPixGeom& g, int mrow, int mc0,
                                                 const int16_t* sc, uint8_t* smem, uint64_t* barp,
                                                 uint32_t parity, CJPixSmemParams* Pp) {
  const CJScanParams* prm = &prmr;
  CJPixSmemParams& P = *Pp;
  const int nm = min(g.T, g.mcux - mc0);
  const int nblk = nm * g.bpm;
  int* tmp = reinterpret_cast<int*>(smem + g.tmp_off);
  uint8_t* py = smem + g.y_off;
  uint8_t* pcb = smem + g.cb_off;
  uint8_t* pcr = smem + g.cr_off;
  for (int k = threadIdx.x; k < 4 * 64; k += blockDim.x) P.q[k >> 6][k & 63] = prm->qnat[k >> 6][k & 63];
  if (threadIdx.x < CJ_MAX_BPM) {
    P.pc[threadIdx.x] = prm->phase_comp[threadIdx.x];
    P.pb[threadIdx.x] = prm->phase_blk[threadIdx.x];
  }
  if (threadIdx.x < 3) {
    P.cq[threadIdx.x] = prm->comp_q[threadIdx.x];
    P.csx[threadIdx.x] = prm->comp_sx[threadIdx.x];
    P.csy[threadIdx.x] = prm->comp_sy[threadIdx.x];
  }
  bool ok = cj_mbar_wait(barp, parity);
  if (!__syncthreads_and(ok)) {
    if (threadIdx.x == 0) atomicMax(&st->dec_err_key, ~((unsigned long long)CJ_DEV_CAPACITY));
    return false;
  }

  // Row pass: one thread per (block, row); dequantise on load.
  for (int t = threadIdx.x; t < nblk * 8; t += blockDim.x) {
    int k = t >> 3, r = t & 7;
    int c = P.pc[k % g.bpm];
    const int16_t* q = &P.q[P.cq[c]][r * 8];
    uint4 raw = *reinterpret_cast<const uint4*>(sc + k * 64 + r * 8);
    int v[8];
    cj_unpack_dequant(raw, q, v);
    cj_idct_row(v);
    int4* o = reinterpret_cast<int4*>(tmp + k * 64 + r * 8);
    o[0] = make_int4(v[0], v[1], v[2], v[3]);
    o[1] = make_int4(v[4], v[5], v[6], v[7]);
  }
  __syncthreads();

  // Column pass: one thread per (block, column); 8 samples into the plane tile.
  for (int t = threadIdx.x; t < nblk * 8; t += blockDim.x) {
    int k = t >> 3, col = t & 7;
    int d[8];
#pragma unroll
    for (int j = 0; j < 8; j++) d[j] = tmp[k * 64 + j * 8 + col];
    uint32_t o[8];
    cj_idct_col(d, o);
    int mi = k / g.bpm, ph = k - mi * g.bpm;
    int c = P.pc[ph], bl = P.pb[ph], sxc = P.csx[c];
    int bx = mi * sxc + bl % sxc, by = bl / sxc;
    uint8_t* plane = c == 0 ? py : (c == 1 ? pcb : pcr);
    int ps = c == 0 ? g.y_stride : g.c_stride;
    uint8_t* dst = plane + (by * 8) * ps + bx * 8 + col;
#pragma unroll
    for (int j = 0; j < 8; j++) dst[j * ps] = (uint8_t)o[j];
  }
  __syncthreads();

  // Upsample + colour (or copy for grey) into the output image.
  const int X0 = mc0 * 8 * g.hmax, Y0 = mrow * 8 * g.vmax;
  const int w = min(nm * 8 * g.hmax, g.width - X0);
  const int h = min(8 * g.vmax, g.height - Y0);
  if (w > 0 && h > 0) {
    if ((g.width & 7) == 0 && (((uintptr_t)out) & 7) == 0) {
      // 8 pixels per item: 24 (or 8) bytes, 8-byte aligned stores
      const int per_row = w >> 3;
      for (int t = threadIdx.x; t < h * per_row; t += blockDim.x) {
        int y = t / per_row, x0 = (t - y * per_row) * 8;
        uint2 yv = *reinterpret_cast<const uint2*>(py + y * g.y_stride + x0);
        if (g.nch == 3) {
          uint32_t wds[6] = {0, 0, 0, 0, 0, 0};
          const uint8_t* crow_b = pcb + (y >> g.ys) * g.c_stride;
          const uint8_t* crow_r = pcr + (y >> g.ys) * g.c_stride;
#pragma unroll
          for (int k = 0; k < 8; k++) {
            int yy = (int)(((k < 4 ? yv.x : yv.y) >> (8 * (k & 3))) & 0xFF) << 8;
            int cb = (int)crow_b[(x0 + k) >> g.xs] - 128, cr = (int)crow_r[(x0 + k) >> g.xs] - 128;
#pragma unroll
            for (int cc = 0; cc < 3; cc++) {
              int byte = 3 * k + cc;
              wds[byte >> 2] |= cj_rgb_pack(yy, cb, cr, cc) << (8 * (byte & 3));
            }
          }
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
  __syncthreads();
  return true;
}
