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
#include "cj_pixel.cuh"


__global__ void __launch_bounds__(CJ_PIX_THREADS)
k_pixel(const CJScanParams* __restrict__ prm, const int16_t* __restrict__ coef,
        uint8_t* __restrict__ out, CJStatus* st, CJPixGeom g) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ uint64_t bar;
  __shared__ CJPixSmemParams P;
  if (threadIdx.x == 0) {
    cj_tile_fail = 0;
    cj_mbar_init(&bar, 1);
    cj_pixel_issue(coef, g, blockIdx.y, blockIdx.x * g.T, reinterpret_cast<int16_t*>(smem), &bar);
  }
  __syncthreads();
  cj_pixel_setup(*prm, g, &P);
  __syncthreads();
  cj_pixel_compute(out, st, g, blockIdx.y, blockIdx.x * g.T, reinterpret_cast<int16_t*>(smem), smem, &bar, 0, &P);
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
  int err = cj_pix_check(hp);
  if (err) return err;
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
  g->T = cj_pix_tile_mcus(hp->hmax, hp->bpm);
  *smem = cj_pix_layout(g, hp->comp_sx[1], hp->comp_sy[1]);
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
  int err = d->progressive ? cj_prog_finish(jpg) : 0;
  if (!err) err = cj_pixel_launch(jpg, true);
  if (err) THROW(err);
  CJStatus* hs = (CJStatus*)d->h_status.p;
  cudaError_t e = cudaStreamSynchronize(d->stream);
  if (e != cudaSuccess) {
    cj_note_cuda_error(e, "cudaStreamSynchronize", __FILE__, __LINE__);
    THROW(CUDA_KERNEL_LAUNCH_ERROR);
  }
  err = cj_reader_decode_status(jpg);
  if (!err) err = cj_status_error(hs);
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

// The reference's alternative final stages (include/pixelTransformGPU.h:18-20)
// map onto the fused pixel stage: run it if the scan's pixels are pending.
static void cj_pixel_stage_alias(JPGReader* jpg) {
  if (jpg && jpg->dev && jpg->dev->scan_pending) iDCT_resample_colourTransform(jpg);
}

extern "C" void upsampleAndColourTransformHybrid(JPGReader* jpg) { cj_pixel_stage_alias(jpg); }
extern "C" void upsampleAndColourTransformGPU(JPGReader* jpg) { cj_pixel_stage_alias(jpg); }
extern "C" void upsampleAndColourTransformCPU(JPGReader* jpg) { cj_pixel_stage_alias(jpg); }
