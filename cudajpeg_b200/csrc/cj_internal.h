// cj_internal.h -- host-side state shared by the libcudajpeg translation units.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../../include/format.h"
#include "cj_core.h"

// Grow-only device allocation (the reference's ensureMemSize with
// USE_CUDA_MALLOC, src/format.cu:81-110, without the per-image shrink).
struct CJDevBuf {
  void* p = nullptr;
  size_t cap = 0;
};

// Grow-only pinned host allocation.
struct CJHostBuf {
  void* p = nullptr;
  size_t cap = 0;
};

// Huffman table as parsed from a DHT segment, before device packing.
struct CJHostHuff {
  uint8_t counts[16];
  uint8_t symbols[256];
  int nsym;
};

#define CJ_KERNEL_SLOTS 24

struct CJReaderDevice {
  // host-side tables (valid without a GPU)
  CJHostHuff huff[4];
  // GPU resources, created on the first scan
  bool gpu_ready = false;
  int device = -1;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_begin = nullptr, ev_scan = nullptr, ev_end = nullptr;
  CJDevBuf raw, data, tile_keep, tile_mark, mpos, mcode, segs, recs, ckpt, snap, wagg, carry, coef,
      pix, params, status, wcoef;
  CJHostBuf h_params, h_status, h_pixels, h_file;
  // per-scan bookkeeping
  int sub_bits = CJ_SUB_BITS_DEFAULT;
  size_t raw_len = 0;
  int64_t total_blocks = 0;
  int nsub_cap = 0, nwarp_cap = 0, nseg_exp = 0, mark_cap = 0;
  int scan_pending = 0;   // a scan was launched and its status is not yet checked
  int snap_parity = 0;    // which last-exit snapshot the next fix-up pass reads
  int comp_first[3];      // first block of each component inside an MCU
  // kernel accounting: launches since reader creation, and (when profiling)
  // one event after each kernel of the last decode
  long long launches = 0;
  bool profile = false;
  cudaEvent_t kev[CJ_KERNEL_SLOTS + 1] = {};
  int kslot[CJ_KERNEL_SLOTS] = {};
  int nkev = 0;
};

// Kernel ids for per-kernel timing (cjReaderKernelTimes)
enum {
  CJ_K_DESTUFF_COUNT = 0, CJ_K_SCAN_TILES, CJ_K_DESTUFF_SCATTER, CJ_K_SEGMENTS, CJ_K_SYNC_INTRA,
  CJ_K_SYNC_INTER, CJ_K_SCAN_WARPS, CJ_K_DECODE_WRITE, CJ_K_PIXEL, CJ_K_COUNT
};

// Count a kernel launch and, when profiling, timestamp its end.
void cj_after_launch(CJReaderDevice* d, int kernel_id);
void cj_profile_begin(CJReaderDevice* d);

// Device memory helpers (scan.cu)
int cj_dev_ensure(CJDevBuf& b, size_t bytes);
int cj_host_ensure(CJHostBuf& b, size_t bytes);
int cj_gpu_init(JPGReader* jpg);
void cj_dev_release(CJReaderDevice* d);

// Scan stages (scan.cu).  cj_scan_launch stages the scan parameters and the
// entropy-coded data [jpg->pos, jpg->end) on the device and enqueues the
// device decode (cj_scan_device) on the reader's stream.
int cj_scan_launch(JPGReader* jpg);
int cj_scan_device(JPGReader* jpg);
// Re-runs fix-up passes until stable and re-decodes (rare path).
int cj_scan_resync(JPGReader* jpg);
// Launch the coefficient write-out pass only (used by the rare path).
int cj_scan_write(JPGReader* jpg);

// Pixel stage (pixel.cu): enqueue the fused kernel + D2H of the output.
int cj_pixel_launch(JPGReader* jpg, bool copy_out);
// Export int32 dequantised coefficients to channels[c].working_space.
int cj_export_coefficients(JPGReader* jpg);

// Host parse helpers (format.cu / scan.cu)
int cj_parse_sos(JPGReader* jpg);
extern "C" int cj_parse_to_scan(JPGReader* r, const unsigned char* buf, size_t size);

// Map a device status word to a format.h error code (0 = fine).
int cj_status_error(const CJStatus* st);

#define CJ_CUDA_TRY(expr, code)                  \
  do {                                           \
    cudaError_t e_ = (expr);                     \
    if (e_ != cudaSuccess) {                     \
      cj_note_cuda_error(e_, #expr, __FILE__, __LINE__); \
      return (code);                             \
    }                                            \
  } while (0)

void cj_note_cuda_error(cudaError_t e, const char* what, const char* file, int line);

// A compact row-major uint8 DLPack view of device memory (api.cu); the
// descriptor is freed by its deleter.
struct DLManagedTensor;
DLManagedTensor* cj_dl_view(void* data, int device, int ndim, const int64_t* shape);
