/*
 * cudajpeg.h -- libcudajpeg additions that have no counterpart in the
 * reference: plain-C accessors for FFI callers that cannot read the
 * JPGReader struct directly, and decoder tuning knobs.
 */
#ifndef CUDAJPEG_H
#define CUDAJPEG_H

#include <stddef.h>
#include <stdint.h>

#include "format.h"

#ifdef __cplusplus
extern "C" {
#endif

/* info[0..11]: width, height, channels, MCUs across, MCUs down, restart
 * interval, blocks per MCU, subsequences of the last scan, destuffed scan
 * bytes, markers found, entropy-coded bytes copied to the device, parameter
 * bytes copied to the device (the raw Huffman / quantisation tables and
 * geometry, and the work plan; the decode tables are built on the GPU). */
void cjReaderInfo(const JPGReader *r, int64_t *info);

/* The decoded image of the last successful openJPG / openJPGMem: RGB
 * (width*height*3) or grey (width*height), in the reader's pinned buffer. */
const unsigned char *cjReaderPixels(const JPGReader *r);

/* Reader flags (CJ_READER_* in format.h). */
void cjReaderSetFlags(JPGReader *r, int flags);

/* Bits per speculative subsequence of the parallel Huffman decode
 * (multiple of 32, 128..65536); 0 restores the default, which picks per
 * image: 512 bits where the MCU-phase hypothesis decodes of so many
 * subsequences still fit in one round of the GPU (small images, the lowest
 * latency), else 1024. */
int cjReaderSetSubsequenceBits(JPGReader *r, int bits);

/* Device time of the last decode split by stage, in milliseconds:
 * [0] entropy stages (destuff .. coefficient write), [1] pixel kernel. */
void cjReaderStageTimes(const JPGReader *r, float *ms);

/* Device pointer to the quantised int16 coefficient blocks of the last scan
 * (natural order, MCU scan order, 64 per block) and their count. */
const short *cjReaderDeviceCoefficients(const JPGReader *r, int64_t *nblocks);

/* Device pointer to the natural-order int16 quantisation table `t` (0..3)
 * of the last scan. */
const short *cjReaderDeviceQuantTable(const JPGReader *r, int t);

/* The reader's CUDA stream (cudaStream_t). */
void *cjReaderStream(const JPGReader *r);

/* Re-run the whole device decode of the last successfully decoded baseline
 * file (PROGRAMMER_ERROR after a progressive one) from
 * its compressed bytes already resident on the GPU (destuff .. pixel
 * kernel), leaving the image in device memory and skipping every host<->
 * device copy.  Asynchronous on the reader's stream; check the result with
 * cjReaderSync.  Returns 0 or a format.h error code. */
int cjReaderRedecodeDevice(JPGReader *r);

/* Wait for the reader's stream and return the device decode status of the
 * last decode (0 or a format.h error code). */
int cjReaderSync(JPGReader *r);

/* Device pointer to the decoded image of the last decode. */
const unsigned char *cjReaderDevicePixels(const JPGReader *r);

/* Per-kernel timing: when on, every kernel launch is followed by a CUDA event
 * on the reader's stream; cjReaderKernelTimes then returns, for the last
 * decode, up to `max` (kernel id, milliseconds) pairs in launch order and
 * their count.  Kernel ids: 0 the entropy decode (the batch decoder's
 * cooperative kernel on this one image), 1 the pixel kernel, 2 one scan of a
 * progressive frame. */
void cjReaderSetProfile(JPGReader *r, int on);
int cjReaderKernelTimes(const JPGReader *r, int *ids, float *ms, int max);

/* Kernels launched by this reader since it was created. */
long long cjReaderLaunchCount(const JPGReader *r);

/* Host check of the Huffman table builder: decode the left-aligned 16-bit
 * window `win16` with the table built from a DHT segment's 16 code-length
 * counts and symbols.  Returns (code length << 8) | symbol, or 0 when no
 * code matches -- the {num_bits, tuple} entry of the reference's 64K table
 * (src/format.cu:357-391) for the same window. */
int cjDebugHuffDecode(const unsigned char counts[16], const unsigned char *symbols,
                      unsigned int win16);

/* Host check of the decode-step tables the entropy kernels use: for every
 * 16-bit window w, out[w] = the step entry for a DC (ac = 0) or AC table built
 * from the DHT counts and symbols -- bits consumed (code + magnitude) in bits
 * 0-4, zig-zag advance in bits 5-11 (DC 1, AC run + 1, ZRL 16, EOB 64,
 * invalid symbol 96, no code 97), magnitude size in bits 12-15. */
int cjDebugStepTable(const unsigned char counts[16], const unsigned char *symbols, int ac,
                     unsigned short *out);

/* Host check of the batch decoder's marker parse: the parse function the
 * GPU runs per file (cjBatchSetParse), run here on the host, against the
 * host marker loop of openJPGMem up to the scan (a fresh reader).  Stores
 * both error codes; returns 0 when they agree and, on success, the scan
 * range and every byte of the device header agree too (else a bit mask:
 * 1 error code, 2 scan range, 4 header). */
int cjDebugParseCompare(const unsigned char *data, size_t size, int *err_host, int *err_parse);

/* Which device code the library was built with: archs[0..] receives the
 * compute capabilities compiled in (1000 = sm_100a), up to max_archs of
 * them, and the count is returned; *binary_version (may be NULL) receives
 * the binary version of the device code the current GPU would run (100 on
 * a B200), or 0 without a GPU. */
int cjBuildInfo(int *archs, int max_archs, int *binary_version);

/* ---- Batched decoder: many JPEGs in one persistent, cooperative kernel ----
 *
 * The files of a batch lie back to back in one host buffer `blob` (pinned
 * memory gives the fastest copy) at offsets[i], sizes[i].  Each image is
 * parsed on the host up to its scan; everything after -- Huffman table
 * build, destuffing, restart intervals, the parallel Huffman decode,
 * coefficient write-out and the fused iDCT / upsample / colour stage -- runs
 * in ONE kernel launch for the whole batch.  Images are independent: a
 * corrupt image reports its own error and the others still decode.  Output
 * i is RGB (width*height*3) or grey (width*height), identical to openJPG's
 * for the same file. */
typedef struct CJBatch CJBatch;

CJBatch *cjBatchCreate(void);
void cjBatchDestroy(CJBatch *b);
int cjBatchSetSubsequenceBits(CJBatch *b, int bits);

/* Tuning of later stages/runs: bits per speculative subsequence (0 =
 * default, 4096 for a batch; multiple of 32, 128..65536), decode-kernel CTAs per SM (3, 4 or 5,
 * 0 = 4: the register budget per thread of the entropy kernel, 80/64/48), and
 * the largest pixel tile in MCUs (power of two, 0 = the layout maximum:
 * 128 pixels across). */
int cjBatchSetTuning(CJBatch *b, int sub_bits, int decode_ctas_per_sm, int pixel_tile_cap);
void cjBatchGetTuning(const CJBatch *b, int *sub_bits, int *decode_ctas_per_sm, int *pixel_tile_cap);
/* Chroma sampling classes of a batch's images (by the sampling factors of
 * SOF: Y 2x2 / 2x1 / 1x1 with 1x1 chroma, one component, anything else). */
#define CJ_SAMPLING_420 0
#define CJ_SAMPLING_422 1
#define CJ_SAMPLING_444 2
#define CJ_SAMPLING_GRAY 3
#define CJ_SAMPLING_OTHER 4
#define CJ_SAMPLING_CLASSES 5
/* Bits per speculative subsequence for the images of one sampling class
 * (staged from now on), overriding cjBatchSetSubsequenceBits for them: the
 * distance a speculative decode runs before it falls into step differs by
 * class (4:2:0 scans the longest), and so does the best size.  bits: as
 * cjBatchSetSubsequenceBits, 0 = follow the batch-wide size.  The getter
 * returns the size in force for the class. */
int cjBatchSetSubsequenceBitsFor(CJBatch *b, int sampling_class, int bits);
int cjBatchGetSubsequenceBitsFor(const CJBatch *b, int sampling_class);
/* Output of a batch staged from now on.  format: CJ_OUTPUT_RGB (default:
 * interleaved RGB, grey as one plane -- the reference's output),
 * CJ_OUTPUT_PLANAR (the Y plane width*height, then the Cb and Cr planes at
 * chroma resolution cw*ch, cw = ceil(width * Hc / Hmax), ch = ceil(height *
 * Vc / Vmax), the reference's channel sizes, src/format.cu:242-354; no
 * upsampling, no colour transform) or CJ_OUTPUT_NV12 (the Y plane, then Cb
 * and Cr interleaved at chroma resolution) or CJ_OUTPUT_RGB_FANCY (interleaved
 * RGB like CJ_OUTPUT_RGB, but chroma upsampled by the IJG decoder's "fancy"
 * triangle filter -- weights 3/4 and 1/4 toward the nearer and the farther
 * chroma sample, for factor-2 directions -- instead of the reference's
 * nearest replication; the colour transform is the reference's).  Grey
 * images have the Y plane only in every format.  idct: CJ_IDCT_INT (default: the reference's fixed
 * point, src/pixelTransformGPU.cu:25-142, bit-exact) or CJ_IDCT_TC (FP16
 * hi/lo basis on tensor cores, FP32 accumulation: within 0.5 of an exact
 * iDCT before rounding, samples within +-1 of CJ_IDCT_INT).  Returns
 * PROGRAMMER_ERROR for anything else. */
#define CJ_OUTPUT_RGB 0
#define CJ_OUTPUT_PLANAR 1
#define CJ_OUTPUT_NV12 2
#define CJ_OUTPUT_RGB_FANCY 3
int cjBatchSetOutput(CJBatch *b, int format, int idct);
/* Where a batch staged from now on has its files' marker segments parsed:
 * on the GPU (on_device != 0, the default: the files are copied to the
 * device first and one thread per file walks its segments there, the reference's
 * marker loop src/format.cu:159-215 with the segment checks of
 * src/format.cu:242-442 and the scan-header check of
 * src/decodeScanGPU.cu:124-144) or on the host (on_device == 0: the marker
 * loop of openJPG, one file after another).  Both give the same headers and
 * error codes.  With the GPU parse, cjBatchStage waits for the files' copy
 * and the parse before it plans the batch. */
int cjBatchSetParse(CJBatch *b, int on_device);
/* MCU-phase hypotheses of the entropy decode (on != 0, the default): when a
 * staged batch's speculative decodes leave most of the GPU idle (a few
 * images), each subsequence of a multi-component scan is also decoded from
 * its first bit under every other MCU phase and then from each of its
 * predecessor's hypothesis exits; the settle takes those decodes instead of
 * re-decoding lane after lane.  Results are identical either way; only the
 * time to settle changes (device memory: two records and checkpoint sets
 * per subsequence and hypothesis). */
int cjBatchSetHypotheses(CJBatch *b, int on);
void cjBatchGetOutput(const CJBatch *b, int *format, int *idct);
/* Bound on each grid-barrier wait of the decode kernel, in polls of about
 * 128 ns (0 = the default, 2^24 polls: about 2 s).  A wait that runs out
 * ends the run early -- every CTA leaves the kernel at its next barrier and
 * the pixel kernel does nothing -- and cjBatchWait then reports
 * CUDA_KERNEL_LAUNCH_ERROR for the batch and for every image of it.  The
 * batch stays usable: the next run (e.g. after restoring the default)
 * decodes normally.  A tiny limit is a way to test that path. */
int cjBatchSetWaitLimit(CJBatch *b, unsigned polls);
/* Autotuner: times the given batch (device time, median of `reps` runs)
 * under every subsequence size in {512, 1024, 2048, 4096} x decode CTAs per
 * SM in {3, 4, 5}; then, one sampling class of the batch at a time (classes
 * holding at least 1/16 of its scan bytes), the sizes {1024 .. 16384} other
 * than the batch-wide best for that class alone; then pixel tile caps
 * {8, 4, 2}; and keeps the fastest tuning in `b` (per-class sizes equal to
 * the batch-wide one are stored as 0).  The batch is left staged under it.
 * trials_ms (may be NULL) receives up to max_trials timings in that order;
 * *best_ms (may be NULL) the best. */
int cjBatchAutotune(CJBatch *b, int n, const unsigned char *blob, const int64_t *offsets,
                    const int64_t *sizes, int reps, float *best_ms, float *trials_ms, int max_trials);

/* Parse, plan and queue the host->device copy of a batch (asynchronous). */
int cjBatchStage(CJBatch *b, int n, const unsigned char *blob, const int64_t *offsets,
                 const int64_t *sizes);
/* Queue the decode over the staged batch (inputs already on the device; may
 * be re-run to re-decode them): one CUDA graph launch -- clear the control
 * block, the cooperative decode kernel, the pixel kernel -- built once per
 * stage. */
int cjBatchRun(CJBatch *b);
/* Queue the device->host copy of all outputs into the batch's pinned buffer. */
int cjBatchFetch(CJBatch *b);
/* Wait for the queued work; errors[i] (may be NULL) gets image i's format.h
 * code.  Returns 0 or a batch-level error (CUDA_KERNEL_LAUNCH_ERROR when a
 * grid-barrier wait of the decode kernel timed out; see
 * cjBatchSetWaitLimit). */
int cjBatchWait(CJBatch *b, int *errors);
/* Stage + run + fetch + wait. */
int cjBatchDecode(CJBatch *b, int n, const unsigned char *blob, const int64_t *offsets,
                  const int64_t *sizes, int *errors);
/* Output of image i after a fetch (host) or a run (device); NULL if image i
 * was rejected by the host parse. */
const unsigned char *cjBatchImage(const CJBatch *b, int i, int *width, int *height, int *channels);
const unsigned char *cjBatchDeviceImage(const CJBatch *b, int i);
/* Width, height and channels of image i of the staged batch (known after
 * cjBatchStage); PROGRAMMER_ERROR if image i was rejected by the host parse. */
int cjBatchImageGeometry(const CJBatch *b, int i, int *width, int *height, int *channels);
/* Chroma plane width and height of image i (0 for grey): the Cb / Cr plane
 * size of the planar and NV12 output formats. */
int cjBatchChromaGeometry(const CJBatch *b, int i, int *cw, int *ch);
void *cjBatchStream(const CJBatch *b);
/* Copy image i's quantised int16 coefficient blocks of the last run to host
 * memory `dst` (natural order, 64 per block, blocks in MCU scan order with
 * all components interleaved, DC already predicted -- the reference's
 * working_space content divided by the quantisation table, before the
 * split into components, src/decodeScanGPU.cu:435-452).  Waits for the
 * batch's stream.  Returns the number of blocks, or PROGRAMMER_ERROR when
 * image i was rejected or max_blocks is too small. */
long long cjBatchCopyCoefficients(CJBatch *b, int i, short *dst, long long max_blocks);
/* stats[0..15]: images submitted, images on the device, decode-kernel CTAs,
 * warp items, destuff tiles, pixel tiles, fix-up passes of the last run,
 * input bytes, output bytes, pixel-kernel dynamic shared memory, kernel
 * launches so far, pixel-kernel CTAs, runs launched as a CUDA graph, graph
 * builds that failed (those runs used plain launches), coefficient blocks,
 * entropy-coded bytes on the device (16-byte padded per image). */
void cjBatchStats(const CJBatch *b, int64_t *stats);
/* Device time of the last cjBatchRun, in milliseconds. */
float cjBatchKernelMs(const CJBatch *b);
/* Split of the last run (after cjBatchWait), in ms: its 10 phases --
 * tables, destuff-count, tile-scan, destuff-scatter, segments, sync, fix-up,
 * warp-scan, write (the decode kernel), pixel (the pixel kernel) -- and the
 * remainder of the run (graph launch, control-block clear, the boundary
 * between the kernels).  Returns the number of entries (11). */
int cjBatchPhaseTimes(const CJBatch *b, float *ms);

/* ---- Decoding without allocating: cjDecodeNoAlloc ----
 *
 * No counterpart in the reference.  Decodes one baseline JPEG held in host
 * memory into a device buffer the caller owns, and allocates no device (or
 * host) memory on the way: for callers that cannot call cudaMalloc while
 * decoding -- a host application whose own caching allocator owns all of the
 * GPU's memory, or a latency-critical loop where an allocation (and the
 * device synchronisation a cudaFree implies) is not acceptable.
 *
 * All working memory (compressed and destuffed bytes, tables, decoder state,
 * coefficient blocks) comes from one static device array of 24 MiB that every
 * GPU which loads the library keeps until the process exits.  The working set
 * is roughly 4-12 bytes per pixel depending on subsampling and compression, so
 * images up to about 2-5 megapixels fit; a larger image is rejected with
 * UNSUPPORTED_ERROR and a message on stderr naming the bytes it needs.
 *
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current and remembers it for the
 * life of the process; make that first call before any stream capture.  The
 * remembered address belongs to the device's context: after a
 * cudaDeviceReset the function must not be called again in this process.
 * Every call shares the array, so calls that overlap on the GPU (from
 * different host threads or streams) race: run them one after another.
 * Before queueing any GPU work the call checks everything it can (header,
 * output capacity, working-memory size, launch shapes); once work is queued,
 * every return -- success or error -- comes after the stream has finished
 * it.  d_out receives RGB (width*height*3) or grey
 * (width*height) bytes and out_capacity is its size in bytes (too small:
 * PROGRAMMER_ERROR).  width/height/channels are filled once the header has
 * been parsed.  The call waits for its own work on `stream` (NULL = the
 * default stream) before returning 0 or a format.h error code. */
int cjDecodeNoAlloc(const unsigned char *jpeg, size_t size, unsigned char *d_out,
                    size_t out_capacity, int *width, int *height, int *channels, void *stream);

/* ---- Decode server: continuous batching of single-image requests ----
 *
 * No counterpart in the reference (its driver decodes one file per process,
 * src/main.cu).  Any host thread submits one JPEG per request; a worker
 * thread groups waiting requests into batches for `engines` batch decoders
 * (each with its own stream, so one batch's copies and host parse overlap
 * another's kernel), admitting a request only while the projected device
 * bytes of all batches in flight stay within `hbm_budget_bytes` (a lone
 * request is always admitted).  Results stay in the engine's device buffer
 * until released; an engine is reused once all of its results are released.
 * Each result is byte-identical to decoding the same file alone. */
typedef struct CJServer CJServer;
typedef struct CJServerResult {
  int error;                           /* format.h code of this request */
  int width, height, channels;
  const unsigned char *device_pixels;  /* valid until cjServerRelease */
  double latency_ms;                   /* submit -> batch finished on the GPU */
} CJServerResult;

/* engines <= 0: 2; hbm_budget_bytes <= 0: 8 GiB; max_batch_images <= 0: 256.
 * NULL if no CUDA device is available.  Uses the current device. */
CJServer *cjServerCreate(int engines, long long hbm_budget_bytes, int max_batch_images);
void cjServerDestroy(CJServer *s);
/* Copies the file; returns a ticket >= 0 or a negative value on a fatal
 * server error. */
long long cjServerSubmit(CJServer *s, const unsigned char *jpeg, size_t size);
/* Waits up to timeout_s seconds: 0 = done (result in *out), 1 = still
 * waiting, else PROGRAMMER_ERROR (unknown ticket). */
int cjServerWait(CJServer *s, long long ticket, double timeout_s, CJServerResult *out);
/* Copies a finished request's pixels to host memory. */
int cjServerCopyOut(CJServer *s, long long ticket, unsigned char *host_dst, size_t capacity);
/* Ends a finished request; its device pixels may be reused afterwards. */
void cjServerRelease(CJServer *s, long long ticket);
/* Batch tuning (as cjBatchSetTuning) for the batches staged from now on.
 * The server's default is 512-bit subsequences (the lowest latency for the
 * small batches of light load), 4 decode CTAs per SM, full pixel tiles. */
int cjServerSetTuning(CJServer *s, int sub_bits, int decode_ctas_per_sm, int pixel_tile_cap);
/* stats[0..5]: batches launched, images admitted, most batches in flight at
 * once, largest batch, requests waiting, projected bytes in flight. */
void cjServerStats(CJServer *s, long long *stats);
/* Open-loop load replay (for measuring the server): request k is file
 * k % nfiles of `blob` (offsets/sizes as for cjBatchStage; the blob must stay
 * valid, it is not copied), submitted at arrival_s[k] seconds after the
 * start.  A collector thread waits for each request in order, writes
 * latency_ms[k] (scheduled arrival -> its batch finished on the GPU) and
 * errors[k] (may be NULL), and releases it.  *wall_s (may be NULL) gets start
 * -> last completion.  Returns 0 or the server's fatal error. */
int cjServerReplay(CJServer *s, const unsigned char *blob, const int64_t *offsets,
                   const int64_t *sizes, int nfiles, const double *arrival_s, int nreq,
                   double *latency_ms, int *errors, double *wall_s);

#ifdef __cplusplus
}
#endif
#endif /* CUDAJPEG_H */
