// scan.cu -- the drop-in scan decode (decodeScanGPU) and the reader's
// device state.
//
// Replaces the reference's host-side serial decode (src/decodeScanGPU.cu:
// 123-491) and its speculative per-bit-position kernels
// (src/entropyRLEdecodeGPU.cu:7-238).  A scan is decoded as one image of the
// batch decoder's cooperative kernel (cj_reader_decode, batch.cu): Huffman
// tables built on the device, destuffing and restart-marker search,
// speculative self-synchronising Huffman decode with the fix-up passes
// looped on the device, block/DC prefix scan and the run-length / zig-zag
// coefficient write-out -- one launch; the pixel stage (pixel.cu) is the
// second.  This file keeps the reader's buffers, the SOS header checks and
// the host-side scan geometry the pixel stage and the accessors read.
#include <stdio.h>
#include <string.h>

#include "../../include/decodeScanCPU.h"
#include "../../include/decodeScanGPU.h"
#include "cj_internal.h"
#include "cj_tables.h"

// ---------------------------------------------------------------- host helpers

void cj_note_cuda_error(cudaError_t e, const char* what, const char* file, int line) {
  fprintf(stderr, "libcudajpeg: %s failed: %s (%s:%d)\n", what, cudaGetErrorString(e), file, line);
}

int cj_dev_ensure(CJDevBuf& b, size_t bytes) {
  if (b.p && bytes <= b.cap) return 0;
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.cap = 0;
  size_t cap = bytes + bytes / 4 + 256;
  cudaError_t e = cudaMalloc(&b.p, cap);
  if (e != cudaSuccess) {
    cj_note_cuda_error(e, "cudaMalloc", __FILE__, __LINE__);
    b.p = nullptr;
    return CUDA_MEM_ERROR;
  }
  b.cap = cap;
  return 0;
}

int cj_host_ensure(CJHostBuf& b, size_t bytes) {
  if (b.p && bytes <= b.cap) return 0;
  if (b.p) cudaFreeHost(b.p);
  b.p = nullptr;
  b.cap = 0;
  size_t cap = bytes + bytes / 4 + 256;
  cudaError_t e = cudaMallocHost(&b.p, cap);
  if (e != cudaSuccess) {
    cj_note_cuda_error(e, "cudaMallocHost", __FILE__, __LINE__);
    b.p = nullptr;
    return OOM_ERROR;
  }
  b.cap = cap;
  return 0;
}

int cj_gpu_init(JPGReader* jpg) {
  CJReaderDevice* d = jpg->dev;
  if (d->gpu_ready) return 0;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    fprintf(stderr, "libcudajpeg: no CUDA device available (%s); the decoder has no CPU path\n",
            e == cudaSuccess ? "0 devices" : cudaGetErrorString(e));
    cudaGetLastError();
    return CUDA_MEM_ERROR;
  }
  CJ_CUDA_TRY(cudaGetDevice(&d->device), CUDA_MEM_ERROR);
  CJ_CUDA_TRY(cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking), CUDA_MEM_ERROR);
  CJ_CUDA_TRY(cudaEventCreate(&d->ev_begin), CUDA_MEM_ERROR);
  CJ_CUDA_TRY(cudaEventCreate(&d->ev_scan), CUDA_MEM_ERROR);
  CJ_CUDA_TRY(cudaEventCreate(&d->ev_end), CUDA_MEM_ERROR);
  for (int k = 0; k <= CJ_KERNEL_SLOTS; k++)
    CJ_CUDA_TRY(cudaEventCreate(&d->kev[k]), CUDA_MEM_ERROR);
  if (cj_host_ensure(d->h_params, sizeof(CJScanParams))) return OOM_ERROR;
  if (cj_host_ensure(d->h_status, sizeof(CJStatus))) return OOM_ERROR;
  d->gpu_ready = true;
  return 0;
}

void cj_dev_release(CJReaderDevice* d) {
  if (!d->gpu_ready) return;
  cudaStreamSynchronize(d->stream);
  CJDevBuf* bufs[] = {&d->raw,  &d->data, &d->tile_keep, &d->tile_mark, &d->mpos,
                      &d->mcode, &d->segs, &d->recs, &d->ckpt,     &d->snap,      &d->wagg,
                      &d->carry, &d->coef, &d->pix,      &d->params,    &d->status,
                      &d->wcoef, &d->bhdr, &d->bdesc, &d->bctl, &d->pscan, &d->hrecs, &d->hckpt, &d->hmap};
  for (CJDevBuf* b : bufs)
    if (b->p) cudaFree(b->p);
  CJHostBuf* hb[] = {&d->h_params, &d->h_status, &d->h_pixels, &d->h_file, &d->h_bctl};
  for (CJHostBuf* b : hb)
    if (b->p) cudaFreeHost(b->p);
  cudaEventDestroy(d->ev_begin);
  cudaEventDestroy(d->ev_scan);
  cudaEventDestroy(d->ev_end);
  for (int k = 0; k <= CJ_KERNEL_SLOTS; k++)
    if (d->kev[k]) cudaEventDestroy(d->kev[k]);
  cudaStreamDestroy(d->stream);
  d->gpu_ready = false;
}

void cj_profile_begin(CJReaderDevice* d) {
  d->nkev = 0;
  if (d->profile) cudaEventRecord(d->kev[0], d->stream);
}

void cj_after_launch(CJReaderDevice* d, int kernel_id) {
  d->launches++;
  if (d->profile && d->nkev < CJ_KERNEL_SLOTS) {
    d->kslot[d->nkev] = kernel_id;
    cudaEventRecord(d->kev[d->nkev + 1], d->stream);
    d->nkev++;
  }
}

int cj_status_error(const CJStatus* st) {
  unsigned long long k = st->err_key > st->dec_err_key ? st->err_key : st->dec_err_key;
  if (!k) return 0;
  unsigned long long key = ~k;
  int code = (int)(key & 0xFF);
  if (code == CJ_DEV_DC_RANGE) return UNSUPPORTED_ERROR;
  if (code == CJ_DEV_CAPACITY) return PROGRAMMER_ERROR;
  return SYNTAX_ERROR;
}

// ---------------------------------------------------------------- host side

// The scan's geometry and quantisation tables on the host (the pixel
// stage's launch shape, the accessors, a progressive frame's pixel stage);
// a baseline scan's tables are built on the device by the decode kernel.
void cj_fill_params(JPGReader* jpg, CJScanParams* hp) {
  CJReaderDevice* d = jpg->dev;
  memset(hp, 0, sizeof(*hp));
  static const uint8_t zz[64] = CJ_ZIGZAG_INIT;
  memcpy(hp->zz, zz, 64);
  for (int t = 0; t < 4; t++)
    for (int k = 0; k < 64; k++) hp->qnat[t][zz[k]] = (int16_t)d->dq16[t][k];
  int k = 0;
  for (int c = 0; c < jpg->num_channels; c++) {
    const ColourChannel* ch = &jpg->channels[c];
    d->comp_first[c] = k;
    for (int j = 0; j < ch->samples_x * ch->samples_y; j++, k++) {
      hp->phase_comp[k] = (uint8_t)c;
      hp->phase_blk[k] = (uint8_t)j;
    }
    hp->comp_dc[c] = (uint8_t)ch->dc_id;
    hp->comp_ac[c] = (uint8_t)ch->ac_id;
    hp->comp_q[c] = (uint8_t)ch->dq_id;
    hp->comp_sx[c] = (uint8_t)ch->samples_x;
    hp->comp_sy[c] = (uint8_t)ch->samples_y;
    hp->comp_stride[c] = ch->stride;
    hp->comp_rows[c] = ch->block_stride;
  }
  hp->nch = jpg->num_channels;
  hp->bpm = k;
  hp->mcux = jpg->num_blocks_x;
  hp->mcuy = jpg->num_blocks_y;
  hp->width = jpg->width;
  hp->height = jpg->height;
  hp->hmax = jpg->block_size_x >> 3;
  hp->vmax = jpg->block_size_y >> 3;
  int xs = 0, ys = 0;
  if (jpg->num_channels == 3) {
    // chroma upsampling factor as CPUonly/src/pixelTransformCPU.c:113-114
    while ((jpg->channels[1].width << xs) < jpg->width) xs++;
    while ((jpg->channels[1].height << ys) < jpg->height) ys++;
  }
  hp->xshift = xs;
  hp->yshift = ys;
  hp->restart_interval = jpg->restart_interval;
  int64_t mcus = (int64_t)hp->mcux * hp->mcuy;
  hp->nseg_expected = jpg->restart_interval ? (int)((mcus + jpg->restart_interval - 1) / jpg->restart_interval) : 1;
  hp->total_blocks = mcus * hp->bpm;
}

int cj_scan_launch(JPGReader* jpg) {
  int err = cj_gpu_init(jpg);
  if (err) return err;
  cj_fill_params(jpg, (CJScanParams*)jpg->dev->h_params.p);
  return cj_reader_decode(jpg, true);
}

// SOS header: the checks of src/decodeScanGPU.cu:124-141.  Returns 0 or a
// format.h error code; on success jpg->pos is on the first entropy byte.
int cj_parse_sos(JPGReader* jpg) {
  unsigned char* pos = jpg->pos;
  if (pos + 2 > jpg->end + 2) return SYNTAX_ERROR;
  unsigned int header_len = read16(pos);
  if (pos + header_len > jpg->end) return SYNTAX_ERROR;
  pos += 2;
  if (!jpg->num_channels) return SYNTAX_ERROR;  // SOS before SOF
  if (header_len < 4u + 2u * jpg->num_channels) return SYNTAX_ERROR;
  if (*(pos++) != jpg->num_channels) return UNSUPPORTED_ERROR;
  for (int i = 0; i < jpg->num_channels; i++, pos += 2) {
    ColourChannel* ch = &jpg->channels[i];
    if (pos[0] != ch->id) return SYNTAX_ERROR;
    if (pos[1] & 0xEE) return SYNTAX_ERROR;
    ch->dc_id = pos[1] >> 4;
    ch->ac_id = (pos[1] & 1) | 2;
    // the reference would decode with an uninitialised table here
    if (!(jpg->huff_defined & (1 << ch->dc_id)) || !(jpg->huff_defined & (1 << ch->ac_id)))
      return SYNTAX_ERROR;
  }
  if (pos[0] || pos[1] != 63 || pos[2]) return UNSUPPORTED_ERROR;
  jpg->pos += header_len;
  if ((size_t)(jpg->end - jpg->pos) > CJ_MAX_SCAN_BYTES) return UNSUPPORTED_ERROR;
  return 0;
}

extern "C" void decodeScanGPU(JPGReader* jpg) {
  if (jpg->dev->progressive) {
    // one scan of a progressive frame; the marker loop continues after it
    int err = cj_prog_scan(jpg);
    if (err) THROW(err);
    jpg->scan_seen = 1;
    jpg->dev->scan_pending = 1;
    return;
  }
  int err = cj_parse_sos(jpg);
  if (err) THROW(err);
  err = cj_scan_launch(jpg);
  if (err) THROW(err);
  // The entropy-coded data runs to the end of the file (as in the reference,
  // which unstuffs and decodes up to jpg->end); device errors are folded in
  // when the pixel stage synchronises.
  jpg->pos = jpg->end;
  jpg->scan_seen = 1;
  jpg->dev->scan_pending = 1;
}

// include/decodeScanCPU.h: the reference's host scan decoder's name
// (src/decodeScanCPU.cu:98-152), decoding on the device like decodeScanGPU.
extern "C" void decodeScanCPU(JPGReader* jpg) { decodeScanGPU(jpg); }
