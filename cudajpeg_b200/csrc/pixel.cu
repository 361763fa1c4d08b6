// pixel.cu -- the pixel stage of libcudajpeg: dequantise + integer iDCT +
// nearest chroma upsampling + YCbCr->RGB, fused in one kernel that reads the
// coefficient blocks decodeScanGPU left on the device and writes the final
// interleaved RGB (or grey) image.
//
// Arithmetic follows the reference bit for bit:
//   fixed-point iDCT ........ src/pixelTransformGPU.cu:25-142 (row pass :43-80,
//                             column pass :87-141; same as CPUonly/src/
//                             pixelTransformCPU.c:14-107)
//   upsample + colour ....... CPUonly/src/pixelTransformCPU.c:110-172 (nearest
//                             replication, JFIF integer RGB with clipping)
// The reference GPU kernel's rounding of its grid to 64 threads without a
// bounds check (pixelTransformGPU.cu:485-510, 652-653) is not reproduced:
// every output pixel is written once, inside the image.
#include <stdio.h>
#include <string.h>
#include <time.h>

#include "../../include/pixelTransformGPU.h"
#include "cj_internal.h"
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

// ---------------------------------------------------------------- fused kernel

struct CJPixGeom {
  int nch, bpm, mcux, mcuy, width, height;
  int hmax, vmax, xs, ys;
  int T;                 // MCUs per CTA (one MCU row)
  int y_stride, c_stride; // tile plane strides (bytes)
  int tmp_off, y_off, cb_off, cr_off;
};

struct CJPixSmemParams {
  int16_t q[4][64];
  uint8_t pc[CJ_MAX_BPM], pb[CJ_MAX_BPM];
  uint8_t cq[4], csx[4], csy[4];
};

__global__ void __launch_bounds__(CJ_PIX_THREADS)
k_pixel(const CJScanParams* __restrict__ prm, const int16_t* __restrict__ coef,
        uint8_t* __restrict__ out, CJStatus* st, CJPixGeom g) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ uint64_t bar;
  __shared__ CJPixSmemParams P;
  const int mrow = blockIdx.y;
  const int mc0 = blockIdx.x * g.T;
  const int nm = min(g.T, g.mcux - mc0);
  const int nblk = nm * g.bpm;
  int16_t* sc = reinterpret_cast<int16_t*>(smem);
  int* tmp = reinterpret_cast<int*>(smem + g.tmp_off);
  uint8_t* py = smem + g.y_off;
  uint8_t* pcb = smem + g.cb_off;
  uint8_t* pcr = smem + g.cr_off;

  if (threadIdx.x == 0) cj_mbar_init(&bar, 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    const int16_t* src = coef + ((int64_t)mrow * g.mcux + mc0) * g.bpm * 64;
    cj_bulk_load(sc, src, (uint32_t)nblk * 128u, &bar);
  }
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
  bool ok = cj_mbar_wait(&bar, 0);
  if (!__syncthreads_and(ok)) {
    if (threadIdx.x == 0) atomicMax(&st->err_key, ~((unsigned long long)CJ_DEV_CAPACITY));
    return;
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
  if (w <= 0 || h <= 0) return;
  if (g.nch == 3) {
    for (int t = threadIdx.x; t < w * h; t += blockDim.x) {
      int y = t / w, x = t - y * w;
      int yy = py[y * g.y_stride + x] << 8;
      int ci = (y >> g.ys) * g.c_stride + (x >> g.xs);
      int cb = (int)pcb[ci] - 128, cr = (int)pcr[ci] - 128;
      uint8_t* o = out + ((int64_t)(Y0 + y) * g.width + X0 + x) * 3;
      o[0] = (uint8_t)cj_clip8((yy + 359 * cr + 128) >> 8);
      o[1] = (uint8_t)cj_clip8((yy - 88 * cb - 183 * cr + 128) >> 8);
      o[2] = (uint8_t)cj_clip8((yy + 454 * cb + 128) >> 8);
    }
  } else {
    for (int t = threadIdx.x; t < w * h; t += blockDim.x) {
      int y = t / w, x = t - y * w;
      out[(int64_t)(Y0 + y) * g.width + X0 + x] = py[y * g.y_stride + x];
    }
  }
}

// Dequantised int32 coefficients in the reference's per-channel layout
// (channels[c].working_space, src/decodeScanGPU.cu:78-100).
__global__ void k_export_coef(const CJScanParams* __restrict__ prm, const int16_t* __restrict__ coef,
                              int32_t* out0, int32_t* out1, int32_t* out2, int64_t total_blocks) {
  int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total_blocks * 64) return;
  int64_t b = idx >> 6;
  int j = (int)(idx & 63);
  int bpm = prm->bpm;
  int64_t mcu = b / bpm;
  int ph = (int)(b - mcu * bpm);
  int c = prm->phase_comp[ph];
  int per = prm->comp_sx[c] * prm->comp_sy[c];
  int64_t local = mcu * per + prm->phase_blk[ph];
  int32_t* o = c == 0 ? out0 : (c == 1 ? out1 : out2);
  o[local * 64 + j] = (int32_t)coef[idx] * (int32_t)prm->qnat[prm->comp_q[c]][j];
}

// ---------------------------------------------------------------- host side

static int cj_pixel_geom(JPGReader* jpg, CJPixGeom* g, size_t* smem) {
  const CJScanParams* hp = (const CJScanParams*)jpg->dev->h_params.p;
  g->nch = hp->nch;
  g->bpm = hp->bpm;
  g->mcux = hp->mcux;
  g->mcuy = hp->mcuy;
  g->width = hp->width;
  g->height = hp->height;
  g->hmax = hp->hmax;
  g->vmax = hp->vmax;
  g->xs = hp->xshift;
  g->ys = hp->yshift;
  // the tile layout needs full-resolution luma and chroma at an exact power-
  // of-two fraction of it (always true for the SOF0 geometries the parser
  // accepts, except 1-pixel-wide or -high oddities)
  if (hp->comp_sx[0] != hp->hmax || hp->comp_sy[0] != hp->vmax) return UNSUPPORTED_ERROR;
  if (hp->nch == 3 && ((hp->comp_sx[1] << hp->xshift) != hp->hmax ||
                       (hp->comp_sy[1] << hp->yshift) != hp->vmax))
    return UNSUPPORTED_ERROR;
  int T = 16 / g->hmax;
  if (T < 1) T = 1;
  while (T > 1 && T * g->bpm > 64) T >>= 1;
  g->T = T;
  g->y_stride = T * 8 * g->hmax;
  g->c_stride = g->nch == 3 ? T * 8 * hp->comp_sx[1] : 0;
  size_t coef_bytes = (size_t)T * g->bpm * 128;
  size_t off = coef_bytes;
  g->tmp_off = (int)off;
  off += (size_t)T * g->bpm * 256;
  g->y_off = (int)off;
  off += (size_t)g->y_stride * 8 * g->vmax;
  off = (off + 15) & ~(size_t)15;
  g->cb_off = (int)off;
  size_t csz = g->nch == 3 ? (size_t)g->c_stride * 8 * hp->comp_sy[1] : 0;
  off += csz;
  g->cr_off = (int)off;
  off += csz;
  *smem = (off + 15) & ~(size_t)15;
  return 0;
}

int cj_pixel_launch(JPGReader* jpg, bool copy_out) {
  CJReaderDevice* d = jpg->dev;
  CJPixGeom g;
  size_t smem;
  int err = cj_pixel_geom(jpg, &g, &smem);
  if (err) return err;
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(k_pixel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr_set = true;
  }
  const size_t npix = (size_t)g.width * g.height * (g.nch == 3 ? 3 : 1);
  if (cj_dev_ensure(d->pix, npix + 16)) return CUDA_MEM_ERROR;
  if (cj_host_ensure(d->h_pixels, npix + 16)) return OOM_ERROR;
  dim3 grid((g.mcux + g.T - 1) / g.T, g.mcuy);
  k_pixel<<<grid, CJ_PIX_THREADS, smem, d->stream>>>((const CJScanParams*)d->params.p,
                                                      (const int16_t*)d->coef.p, (uint8_t*)d->pix.p,
                                                      (CJStatus*)d->status.p, g);
  cj_after_launch(d, CJ_K_PIXEL);
  CJ_CUDA_TRY(cudaGetLastError(), CUDA_KERNEL_LAUNCH_ERROR);
  CJ_CUDA_TRY(cudaEventRecord(d->ev_end, d->stream), CUDA_KERNEL_LAUNCH_ERROR);
  if (!copy_out) return 0;
  CJ_CUDA_TRY(cudaMemcpyAsync(d->h_pixels.p, d->pix.p, npix, cudaMemcpyDeviceToHost, d->stream),
              CUDA_MEM_ERROR);
  CJ_CUDA_TRY(cudaMemcpyAsync(d->h_status.p, d->status.p, sizeof(CJStatus), cudaMemcpyDeviceToHost,
                              d->stream),
              CUDA_MEM_ERROR);
  return 0;
}

int cj_export_coefficients(JPGReader* jpg) {
  CJReaderDevice* d = jpg->dev;
  const CJScanParams* hp = (const CJScanParams*)d->h_params.p;
  size_t total = 0, off[3] = {0, 0, 0};
  for (int c = 0; c < hp->nch; c++) {
    off[c] = total;
    total += (size_t)jpg->channels[c].num_blocks * 64;
  }
  if (cj_dev_ensure(d->wcoef, total * 4 + 16)) return CUDA_MEM_ERROR;
  int32_t* base = (int32_t*)d->wcoef.p;
  int64_t n = d->total_blocks * 64;
  k_export_coef<<<(unsigned)((n + 255) / 256), 256, 0, d->stream>>>(
      (const CJScanParams*)d->params.p, (const int16_t*)d->coef.p, base + off[0], base + off[1],
      base + off[2], d->total_blocks);
  CJ_CUDA_TRY(cudaGetLastError(), CUDA_KERNEL_LAUNCH_ERROR);
  for (int c = 0; c < hp->nch; c++) {
    ManagedIntMem* w = &jpg->channels[c].working_space;
    unsigned int need = (unsigned int)(jpg->channels[c].num_blocks * 64);
    if (!w->mem || w->max_size < need) {
      free(w->mem);
      w->mem = (int*)malloc((size_t)need * 4);
      if (!w->mem) return OOM_ERROR;
      w->max_size = need;
    }
    w->size = need;
    CJ_CUDA_TRY(cudaMemcpyAsync(w->mem, base + off[c], (size_t)need * 4, cudaMemcpyDeviceToHost,
                                d->stream),
                CUDA_MEM_ERROR);
  }
  return 0;
}

extern "C" void iDCT_resample_colourTransform(JPGReader* jpg) {
  CJReaderDevice* d = jpg->dev;
  if (!d || !d->scan_pending) THROW(PROGRAMMER_ERROR);
  d->scan_pending = 0;
  int err = cj_pixel_launch(jpg, true);
  if (err) THROW(err);
  CJStatus* hs = (CJStatus*)d->h_status.p;
  cudaError_t e = cudaStreamSynchronize(d->stream);
  if (e != cudaSuccess) {
    cj_note_cuda_error(e, "cudaStreamSynchronize", __FILE__, __LINE__);
    THROW(CUDA_KERNEL_LAUNCH_ERROR);
  }
  if (hs->unstable) {
    // rare: re-run the fix-up passes to a fixed point, then redo the output
    if ((err = cj_scan_resync(jpg)) || (err = cj_pixel_launch(jpg, true))) THROW(err);
    if (cudaStreamSynchronize(d->stream) != cudaSuccess) THROW(CUDA_KERNEL_LAUNCH_ERROR);
  }
  err = cj_status_error(hs);
  if (err) {
    jpg->error = err;
    jpg->error_line = 0;
    jpg->error_file = (char*)"device";
    jpg->error_func = (char*)"decodeScanGPU";
    return;
  }
  if (jpg->flags & CJ_READER_HOST_COEFFICIENTS) {
    if ((err = cj_export_coefficients(jpg))) THROW(err);
    if (cudaStreamSynchronize(d->stream) != cudaSuccess) THROW(CUDA_KERNEL_LAUNCH_ERROR);
  }
  float ms = 0;
  cudaEventElapsedTime(&ms, d->ev_begin, d->ev_end);
  jpg->time = (clock_t)(ms * (CLOCKS_PER_SEC / 1000.0));
  unsigned char* px = (unsigned char*)d->h_pixels.p;
  jpg->pixels = px;
  jpg->max_pixels_size = (int)d->h_pixels.cap;
  jpg->channels[0].pixels.mem = px;
  jpg->channels[0].pixels.size = (unsigned int)((size_t)jpg->width * jpg->height);
  jpg->channels[0].pixels.max_size = (unsigned int)d->h_pixels.cap;
}
