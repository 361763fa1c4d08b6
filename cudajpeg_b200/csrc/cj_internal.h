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
  uint16_t dq16[4][64];   // quantisation tables as parsed (8- or 16-bit), zig-zag order
  bool progressive = false;  // the frame is SOF2
  int prog_scans = 0;        // progressive scans queued for this frame
  // GPU resources, created on the first scan
  bool gpu_ready = false;
  int device = -1;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_begin = nullptr, ev_scan = nullptr, ev_end = nullptr;
  CJDevBuf raw, data, tile_keep, tile_mark, mpos, mcode, segs, recs, ckpt, snap, wagg, carry, coef,
      pix, params, status, wcoef, bhdr, bdesc, bctl, pscan, hrecs, hckpt, hmap;
  CJHostBuf h_params, h_status, h_pixels, h_file, h_bctl;
  // per-scan bookkeeping
  int sub_bits = CJ_SUB_BITS_DEFAULT;
  bool sub_bits_auto = true;  // no size set: the decode picks 512 or 1024 bits per image
  size_t raw_len = 0;
  int64_t total_blocks = 0;
  int nsub_cap = 0, nwarp_cap = 0, nseg_exp = 0, mark_cap = 0;
  int scan_pending = 0;   // a scan was launched and its status is not yet checked
  int comp_first[3];      // first block of each component inside an MCU
  // the scan as one image of the batch decode kernel (cj_reader_decode)
  int b_grid = 0, b_ntiles = 0, b_nwarps = 0, b_nptiles = 0, b_nhyp = 1, b_ctas = 4;
  size_t param_bytes = 0;  // header + plan bytes copied to the device per scan
  // kernel accounting: launches since reader creation, and (when profiling)
  // one event after each kernel of the last decode
  long long launches = 0;
  bool profile = false;
  cudaEvent_t kev[CJ_KERNEL_SLOTS + 1] = {};
  int kslot[CJ_KERNEL_SLOTS] = {};
  int nkev = 0;
};

// Kernel ids for per-kernel timing (cjReaderKernelTimes)
enum { CJ_K_DECODE_BATCH = 0, CJ_K_PIXEL, CJ_K_PROG_SCAN, CJ_K_COUNT };

// Count a kernel launch and, when profiling, timestamp its end.
void cj_after_launch(CJReaderDevice* d, int kernel_id);
void cj_profile_begin(CJReaderDevice* d);

// Device memory helpers (scan.cu)
int cj_dev_ensure(CJDevBuf& b, size_t bytes);
int cj_host_ensure(CJHostBuf& b, size_t bytes);
int cj_gpu_init(JPGReader* jpg);
void cj_dev_release(CJReaderDevice* d);

// Scan stage (scan.cu).  cj_scan_launch fills the reader's host-side scan
// geometry and enqueues cj_reader_decode(stage = true) on its stream.
int cj_scan_launch(JPGReader* jpg);
// The scan's geometry and quantisation tables on the host (scan.cu).
void cj_fill_params(JPGReader* jpg, CJScanParams* hp);
// One scan of a progressive frame, as its kernel sees it.
struct CJProgScan {
  int32_t ns, ss, se, ah, al;
  int32_t dc_slot[3], ac_slot[3];
  int32_t first[3];  // first block of the scan component inside an MCU
  int32_t sx[3], sy[3];
  int32_t bpm, mcux;
  int32_t bw, bh;    // one-component scans: the component's block grid
  int32_t ri;        // units (MCUs, or blocks of a one-component scan) per interval; 0 = none
  int32_t nunits, nint;
};
// Check a progressive frame's SOS header at jpg->pos (0 or a format.h code).
int cj_parse_prog_sos(JPGReader* jpg, CJProgScan* s);
// Progressive frames (progressive.cu): queue one SOS's scan; at EOI, the
// pixel stage's parameters.
int cj_prog_scan(JPGReader* jpg);
int cj_prog_finish(JPGReader* jpg);
// The scan's entropy decode as one image of the batch decode kernel
// (batch.cu): with stage = true, plan the image and copy its header and
// entropy-coded bytes [jpg->pos, jpg->end) to the device first; otherwise
// re-run the decode over what is already there.  Asynchronous on the
// reader's stream.
int cj_reader_decode(JPGReader* jpg, bool stage);
// After the reader's stream has been synchronised: CUDA_KERNEL_LAUNCH_ERROR
// when a grid-barrier wait of the last decode timed out, else 0.
int cj_reader_decode_status(const JPGReader* jpg);

// Pixel stage (pixel.cu): enqueue the fused kernel + D2H of the output.
int cj_pixel_launch(JPGReader* jpg, bool copy_out);
// Export int32 dequantised coefficients to channels[c].working_space.
int cj_export_coefficients(JPGReader* jpg);

// Host parse helpers (format.cu / scan.cu)
int cj_parse_sos(JPGReader* jpg);
extern "C" int cj_parse_to_scan(JPGReader* r, const unsigned char* buf, size_t size);

// Map a device status word to a format.h error code (0 = fine).
int cj_status_error(const CJStatus* st);

// Khi then Klo of the tensor-core iDCT's Kronecker basis (8192 FP16 values in
// the B operand's core-matrix layout) on the current device, built on first
// use; nullptr if it could not be allocated.
const uint16_t* cj_tc_basis_device();

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
