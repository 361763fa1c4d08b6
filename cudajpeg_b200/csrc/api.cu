// api.cu -- plain-C accessors and tuning knobs of libcudajpeg (cudajpeg.h).
#include <stddef.h>

#include "../../include/cj_dlpack.h"
#include "../../include/cudajpeg.h"
#include "cj_internal.h"
#include <new>
#include "cj_tables.h"

extern "C" {

void cjReaderInfo(const JPGReader* r, int64_t* info) {
  const CJReaderDevice* d = r->dev;
  const CJStatus* st = (d && d->h_status.p) ? (const CJStatus*)d->h_status.p : nullptr;
  const CJScanParams* hp = (d && d->h_params.p) ? (const CJScanParams*)d->h_params.p : nullptr;
  info[0] = r->width;
  info[1] = r->height;
  info[2] = r->num_channels;
  info[3] = r->num_blocks_x;
  info[4] = r->num_blocks_y;
  info[5] = r->restart_interval;
  info[6] = hp ? hp->bpm : 0;
  info[7] = st ? st->nsub : 0;
  info[8] = st ? st->destuffed : 0;
  info[9] = st ? st->nmarkers : 0;
  info[10] = d ? (int64_t)d->raw_len : 0;
  info[11] = d ? (int64_t)d->param_bytes : 0;
}

const unsigned char* cjReaderPixels(const JPGReader* r) { return r->pixels; }

void cjReaderSetFlags(JPGReader* r, int flags) { r->flags = flags; }

int cjReaderSetSubsequenceBits(JPGReader* r, int bits) {
  const bool autosel = bits == 0;
  if (bits == 0) bits = CJ_SUB_BITS_DEFAULT;
  if (bits < 128 || bits > 65536 || (bits & 31)) return PROGRAMMER_ERROR;
  r->dev->sub_bits = bits;
  r->dev->sub_bits_auto = autosel;
  return 0;
}

void cjReaderStageTimes(const JPGReader* r, float* ms) {
  const CJReaderDevice* d = r->dev;
  ms[0] = ms[1] = 0.f;
  if (!d->gpu_ready) return;
  cudaEventElapsedTime(&ms[0], d->ev_begin, d->ev_scan);
  cudaEventElapsedTime(&ms[1], d->ev_scan, d->ev_end);
}

const short* cjReaderDeviceCoefficients(const JPGReader* r, int64_t* nblocks) {
  *nblocks = r->dev->total_blocks;
  return (const short*)r->dev->coef.p;
}

const short* cjReaderDeviceQuantTable(const JPGReader* r, int t) {
  if (!r->dev->params.p || t < 0 || t > 3) return nullptr;
  return ((const CJScanParams*)r->dev->params.p)->qnat[t];
}

void* cjReaderStream(const JPGReader* r) { return (void*)r->dev->stream; }

int cjReaderRedecodeDevice(JPGReader* r) {
  CJReaderDevice* d = r->dev;
  // (baseline frames: a progressive frame's scans are not kept for a re-run)
  if (!d->gpu_ready || !d->raw.p || !d->total_blocks || !d->b_grid || d->progressive) return PROGRAMMER_ERROR;
  int err = cj_reader_decode(r, false);
  if (!err) err = cj_pixel_launch(r, false);
  return err;
}

int cjReaderSync(JPGReader* r) {
  CJReaderDevice* d = r->dev;
  if (!d->gpu_ready) return PROGRAMMER_ERROR;
  CJ_CUDA_TRY(cudaMemcpyAsync(d->h_status.p, d->status.p, sizeof(CJStatus), cudaMemcpyDeviceToHost,
                              d->stream),
              CUDA_MEM_ERROR);
  CJ_CUDA_TRY(cudaStreamSynchronize(d->stream), CUDA_KERNEL_LAUNCH_ERROR);
  int err = cj_reader_decode_status(r);
  return err ? err : cj_status_error((const CJStatus*)d->h_status.p);
}

const unsigned char* cjReaderDevicePixels(const JPGReader* r) {
  return (const unsigned char*)r->dev->pix.p;
}

void cjReaderSetProfile(JPGReader* r, int on) { r->dev->profile = on != 0; }

int cjReaderKernelTimes(const JPGReader* r, int* ids, float* ms, int max) {
  const CJReaderDevice* d = r->dev;
  int n = d->nkev < max ? d->nkev : max;
  for (int k = 0; k < n; k++) {
    ids[k] = d->kslot[k];
    ms[k] = 0.f;
    cudaEventElapsedTime(&ms[k], d->kev[k], d->kev[k + 1]);
  }
  return n;
}

long long cjReaderLaunchCount(const JPGReader* r) { return r->dev->launches; }

int cjDebugHuffDecode(const unsigned char counts[16], const unsigned char* symbols,
                      unsigned int win16) {
  CJHuff t;
  cj_build_huff(counts, symbols, &t);
  return (int)cj_huff_decode(t, win16 & 0xFFFF);
}

int cjDebugStepTable(const unsigned char counts[16], const unsigned char* symbols, int ac,
                     unsigned short* out) {
  CJScanParams* sp = new (std::nothrow) CJScanParams;
  if (!sp || !out) {
    delete sp;
    return PROGRAMMER_ERROR;
  }
  memset(sp, 0, sizeof(*sp));
  const int slot = ac ? 2 : 0;
  cj_build_huff(counts, symbols, &sp->huff[slot]);
  cj_build_steps(sp->huff[slot], counts, true, slot, &sp->steps);
  for (uint32_t w = 0; w < 65536; w++) out[w] = (unsigned short)cj_step(*sp, slot, w << 16);
  delete sp;
  return 0;
}

}  // extern "C"

// Never launched: its attributes tell which device code the library holds.
__global__ void k_build_probe() {}

extern "C" int cjBuildInfo(int* archs, int max_archs, int* binary_version) {
#ifdef __CUDA_ARCH_LIST__
  static const int list[] = {__CUDA_ARCH_LIST__};
#else
  static const int list[] = {0};
#endif
  const int n = (int)(sizeof(list) / sizeof(list[0]));
  for (int k = 0; k < n && k < max_archs; k++) archs[k] = list[k];
  if (binary_version) {
    *binary_version = 0;
    int devices = 0;
    if (cudaGetDeviceCount(&devices) == cudaSuccess && devices > 0) {
      cudaFuncAttributes fa;
      if (cudaFuncGetAttributes(&fa, k_build_probe) == cudaSuccess) *binary_version = fa.binaryVersion;
    }
    cudaGetLastError();
  }
  return n;
}

// ---------------------------------------------------------------- DLPack views

// The descriptor and its shape / strides in one allocation.
struct CJDLTensor {
  DLManagedTensor t;
  int64_t shape[3];
  int64_t strides[3];
};

static void cj_dl_delete(DLManagedTensor* self) { delete static_cast<CJDLTensor*>(self->manager_ctx); }

// A compact row-major uint8 tensor view of device memory.
DLManagedTensor* cj_dl_view(void* data, int device, int ndim, const int64_t* shape) {
  if (!data || ndim < 1 || ndim > 3) return nullptr;
  CJDLTensor* d = new (std::nothrow) CJDLTensor;
  if (!d) return nullptr;
  int64_t stride = 1;
  for (int k = ndim - 1; k >= 0; k--) {
    d->shape[k] = shape[k];
    d->strides[k] = stride;
    stride *= shape[k];
  }
  DLTensor& x = d->t.dl_tensor;
  x.data = data;
  x.device.device_type = kDLCUDA;
  x.device.device_id = device;
  x.ndim = ndim;
  x.dtype.code = kDLUInt;
  x.dtype.bits = 8;
  x.dtype.lanes = 1;
  x.shape = d->shape;
  x.strides = d->strides;
  x.byte_offset = 0;
  d->t.manager_ctx = d;
  d->t.deleter = cj_dl_delete;
  return &d->t;
}

extern "C" void cjDLPackFree(DLManagedTensor* t) {
  if (t && t->deleter) t->deleter(t);
}
