// scan.cu -- device entropy decode of one baseline scan (decodeScanGPU).
//
// Replaces the reference's host-side serial decode (src/decodeScanGPU.cu:
// 123-491) and its speculative per-bit-position kernels
// (src/entropyRLEdecodeGPU.cu:7-238) with five stages, all on one stream:
//
//   1. destuff    k_destuff_count / k_scan_tiles / k_destuff_scatter: remove
//                 the 00 after every FF, cut the data at RSTn markers
//                 (src/decodeScanGPU.cu:11-24 keeps them in the buffer);
//   2. segments   k_build_segments: one segment per restart interval, checked
//                 against DRI, and its share of the speculative subsequences;
//   3. sync       k_sync_intra + k_sync_inter: every lane decodes a fixed
//                 S-bit subsequence speculatively from a guessed block start,
//                 then lanes take their predecessor's exit state (warp shuffle
//                 inside a warp, a snapshot between warps) and re-decode until
//                 nothing changes.  The fixed point is unique, so the result
//                 equals a serial decode; self-synchronisation of the code only
//                 decides how many re-decodes it takes;
//   4. scan       k_scan_warps + a segmented warp scan: the global index of each
//                 subsequence's first block and its DC predictors;
//   5. write      k_decode_write: the final decode writes quantised int16
//                 coefficients, natural order, MCU scan order; DC is predicted
//                 per component and reset at every restart interval.
#include <stdio.h>
#include <string.h>

#include "../../include/decodeScanCPU.h"
#include "../../include/decodeScanGPU.h"
#include "cj_internal.h"
#include "cj_entropy.cuh"
#include "cj_scan_util.cuh"
#include "cj_tables.h"

#define CJ_TILE_THREADS 256
#define CJ_TILE_BYTES (CJ_TILE_THREADS * 16)
#define CJ_SYNC_THREADS 128

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
                      &d->wcoef};
  for (CJDevBuf* b : bufs)
    if (b->p) cudaFree(b->p);
  CJHostBuf* hb[] = {&d->h_params, &d->h_status, &d->h_pixels, &d->h_file};
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

// ---------------------------------------------------------------- device helpers

// Stage 1a: kept bytes and markers per 4 KiB tile.
__global__ void __launch_bounds__(CJ_TILE_THREADS)
k_destuff_count(const uint8_t* __restrict__ raw, int64_t n, int32_t* tile_keep, int32_t* tile_mark,
                CJStatus* st) {
  __shared__ int2 sm[33];
  int64_t base = (int64_t)blockIdx.x * CJ_TILE_BYTES + threadIdx.x * 16;
  CJChunk c = cj_classify(raw, n, base);
  int2 tot;
  cj_block_exclusive(make_int2(__popc(c.keep), __popc(c.mark)), sm, &tot);
  if (threadIdx.x == 0) {
    tile_keep[blockIdx.x] = tot.x;
    tile_mark[blockIdx.x] = tot.y;
  }
  if (c.bad) cj_raise(st, 0, CJ_DEV_MARKER);
}

// Stage 1b: exclusive offsets of the tiles (one CTA).
__global__ void __launch_bounds__(1024)
k_scan_tiles(int32_t* tile_keep, int32_t* tile_mark, int ntiles, CJStatus* st) {
  __shared__ int2 sm[33];
  int per = (ntiles + blockDim.x - 1) / blockDim.x;
  int lo = threadIdx.x * per, hi = min(ntiles, lo + per);
  int2 s = make_int2(0, 0);
  for (int t = lo; t < hi; t++) {
    s.x += tile_keep[t];
    s.y += tile_mark[t];
  }
  int2 tot;
  int2 ex = cj_block_exclusive(s, sm, &tot);
  for (int t = lo; t < hi; t++) {
    int k = tile_keep[t], m = tile_mark[t];
    tile_keep[t] = ex.x;
    tile_mark[t] = ex.y;
    ex.x += k;
    ex.y += m;
  }
  if (threadIdx.x == 0) {
    st->destuffed = tot.x;
    st->nmarkers = tot.y;
  }
}

// Stage 1c: write the destuffed bytes and record each marker's position.
__global__ void __launch_bounds__(CJ_TILE_THREADS)
k_destuff_scatter(const uint8_t* __restrict__ raw, int64_t n, const int32_t* tile_keep,
                  const int32_t* tile_mark, uint8_t* __restrict__ out, uint32_t* mpos,
                  uint8_t* mcode, int mcap) {
  __shared__ int2 sm[33];
  int64_t base = (int64_t)blockIdx.x * CJ_TILE_BYTES + threadIdx.x * 16;
  CJChunk c = cj_classify(raw, n, base);
  int2 tot;
  int2 ex = cj_block_exclusive(make_int2(__popc(c.keep), __popc(c.mark)), sm, &tot);
  int64_t o = (int64_t)tile_keep[blockIdx.x] + ex.x;
  int r = tile_mark[blockIdx.x] + ex.y;
#pragma unroll
  for (int j = 0; j < 16; j++) {
    if (c.keep & (1u << j)) out[o++] = (uint8_t)cj_byte(c, j);
    if (c.mark & (1u << j)) {
      if (r < mcap) {
        mpos[r] = (uint32_t)o;
        mcode[r] = (uint8_t)(j < 15 ? cj_byte(c, j + 1) : c.next);
      }
      r++;
    }
  }
}

// Stage 2: restart intervals -> segments, and each segment's subsequences.
__global__ void __launch_bounds__(1024)
k_build_segments(const CJScanParams* __restrict__ prm, CJStatus* st, const uint32_t* mpos,
                 const uint8_t* mcode, int mcap, CJSegment* segs, int seg_cap, int sub_bits,
                 int rec_cap) {
  __shared__ int2 sm[33];
  const int M = st->nmarkers;
  const int64_t L = st->destuffed;
  const int RI = prm->restart_interval;
  const int E = RI ? prm->nseg_expected : 1;
  const int64_t per_seg = RI ? (int64_t)RI * prm->bpm : prm->total_blocks;
  bool ok = true;
  int nseg = E;
  if (RI == 0) ok = (M == 0);
  else if (M == E - 1) ok = true;
  else if (M == E && M <= mcap && mpos[M - 1] == (uint32_t)L) ok = true;  // trailing RSTn
  else ok = false;
  if (M > mcap || nseg > seg_cap) ok = false;
  if (!ok) {
    if (threadIdx.x == 0) {
      cj_raise(st, 0, CJ_DEV_MARKER);
      st->nsub = 0;
      st->nseg = 0;
    }
    return;
  }
  int running = 0;
  for (int k0 = 0; k0 < nseg; k0 += blockDim.x) {
    int k = k0 + threadIdx.x;
    int64_t begin = 0, end = 0;
    int nsub = 0;
    if (k < nseg) {
      begin = k ? mpos[k - 1] : 0;
      end = k < M ? (int64_t)mpos[k] : L;
      if (k < M && mcode[k] != 0xD0 + (k & 7)) cj_raise(st, (int64_t)k * per_seg, CJ_DEV_MARKER);
      int64_t bits = (end - begin) * 8;
      nsub = (int)((bits + sub_bits - 1) / sub_bits);
      if (nsub < 1) nsub = 1;
    }
    int2 tot;
    int2 ex = cj_block_exclusive(make_int2(nsub, 0), sm, &tot);
    if (k < nseg) {
      CJSegment s;
      s.bit_begin = (uint64_t)begin * 8;
      s.bit_end = (uint64_t)end * 8;
      s.first_block = (int64_t)k * per_seg;
      s.nblocks = min(per_seg, prm->total_blocks - s.first_block);
      s.first_sub = running + ex.x;
      s.nsub = nsub;
      s.marker_follows = k < M;
      s.pad = 0;
      segs[k] = s;
    }
    running += tot.x;
  }
  if (threadIdx.x == 0) {
    st->nseg = nseg;
    if (running > rec_cap) {
      cj_raise(st, 0, CJ_DEV_CAPACITY);
      running = 0;
    }
    st->nsub = running;
  }
}

// Shared-memory copy of the scan parameters for the decode kernels.
__device__ __forceinline__ void cj_load_params(CJScanParams& sp, const CJScanParams* prm) {
  const int4* src = reinterpret_cast<const int4*>(prm);
  int4* dst = reinterpret_cast<int4*>(&sp);
  for (int k = threadIdx.x; k < (int)(sizeof(CJScanParams) / 16); k += blockDim.x) dst[k] = src[k];
  __syncthreads();
}

// Stage 3a: speculative decode + settle inside each warp.
__global__ void __launch_bounds__(CJ_SYNC_THREADS)
k_sync_intra(const CJScanParams* __restrict__ prm, const CJSegment* __restrict__ segs,
             const uint32_t* __restrict__ words, CJSubRec* recs, CJCkpt* ckpt, uint64_t* snap_out,
             const CJStatus* st, int sub_bits) {
  __shared__ CJScanParams sp;
  cj_load_params(sp, prm);
  const int nsub = st->nsub, nseg = st->nseg;
  int warp = blockIdx.x * (CJ_SYNC_THREADS / 32) + (threadIdx.x >> 5);
  int lane = threadIdx.x & 31;
  if (warp * 32 >= nsub) return;
  int i = warp * 32 + lane;
  CJLane ln = cj_lane(segs, nseg, nsub, i, sub_bits);
  CJSubRec r;
  r.start = cj_state(ln.begin, 0);
  r.exit = r.start;
  r.nblocks = r.dc[0] = r.dc[1] = r.dc[2] = 0;
  CJCkpt* ck = cj_lane_ckpts(ckpt, i);
  const uint32_t cs = cj_ckpt_step(sub_bits);
  if (ln.active) r = cj_spec_decode<false>(sp, sp.steps, words, ln, r.start, ck, r, cs);
  cj_warp_settle(sp, sp.steps, words, ln, r, r.start, ck, cs);
  if (ln.active) recs[i] = r;
  unsigned act = __ballot_sync(CJ_FULL, ln.active);
  if (lane == 31 - __clz(act)) snap_out[warp] = r.exit;
}

// Stage 3b: fix-up pass between warps.  Lane 0 of each warp takes the last
// exit state of the previous warp from `snap_in`; counts warps whose own
// last exit differs from what the next warp read.
__global__ void __launch_bounds__(CJ_SYNC_THREADS)
k_sync_inter(const CJScanParams* __restrict__ prm, const CJSegment* __restrict__ segs,
             const uint32_t* __restrict__ words, CJSubRec* recs, CJCkpt* ckpt, const uint64_t* snap_in,
             uint64_t* snap_out, CJWarpAgg* wagg, CJStatus* st, int sub_bits) {
  __shared__ CJScanParams sp;
  cj_load_params(sp, prm);
  const int nsub = st->nsub, nseg = st->nseg;
  int warp = blockIdx.x * (CJ_SYNC_THREADS / 32) + (threadIdx.x >> 5);
  int lane = threadIdx.x & 31;
  if (warp * 32 >= nsub) return;
  int i = warp * 32 + lane;
  CJLane ln = cj_lane(segs, nseg, nsub, i, sub_bits);
  CJSubRec r;
  if (ln.active) r = recs[i];
  else {
    r.start = r.exit = 0;
    r.nblocks = r.dc[0] = r.dc[1] = r.dc[2] = 0;
  }
  uint64_t in0 = (warp > 0) ? snap_in[warp - 1] : r.start;
  if (lane != 0) in0 = 0;
  if (cj_warp_settle(sp, sp.steps, words, ln, r, in0, cj_lane_ckpts(ckpt, i), cj_ckpt_step(sub_bits)) && ln.active)
    recs[i] = r;
  unsigned act = __ballot_sync(CJ_FULL, ln.active);
  if (lane == 31 - __clz(act)) {
    if (r.exit != snap_in[warp]) atomicAdd(&st->unstable, 1);
    snap_out[warp] = r.exit;
  }
  // segmented warp aggregate: lanes from the last segment head on
  unsigned heads = __ballot_sync(CJ_FULL, ln.active && ln.head);
  int h = heads ? 31 - __clz(heads) : 0;
  bool use = ln.active && lane >= h;
  int v0 = use ? r.nblocks : 0, v1 = use ? r.dc[0] : 0, v2 = use ? r.dc[1] : 0,
      v3 = use ? r.dc[2] : 0;
#pragma unroll
  for (int d = 16; d; d >>= 1) {
    v0 += __shfl_xor_sync(CJ_FULL, v0, d);
    v1 += __shfl_xor_sync(CJ_FULL, v1, d);
    v2 += __shfl_xor_sync(CJ_FULL, v2, d);
    v3 += __shfl_xor_sync(CJ_FULL, v3, d);
  }
  if (lane == 0) {
    CJWarpAgg a;
    a.has_head = heads != 0;
    a.nblocks = v0;
    a.dc[0] = v1;
    a.dc[1] = v2;
    a.dc[2] = v3;
    a.pad[0] = a.pad[1] = a.pad[2] = 0;
    wagg[warp] = a;
  }
}

// Stage 4a: exclusive segmented scan of the warp aggregates (one CTA).
__global__ void __launch_bounds__(1024)
k_scan_warps(const CJWarpAgg* __restrict__ wagg, CJWarpAgg* carry, const CJStatus* st) {
  __shared__ CJAgg5 sm[1024];
  const int nw = (st->nsub + 31) / 32;
  int per = (nw + blockDim.x - 1) / blockDim.x;
  int lo = threadIdx.x * per, hi = min(nw, lo + per);
  CJAgg5 acc = {0, 0, 0, 0, 0};
  for (int w = lo; w < hi; w++) {
    CJWarpAgg g = wagg[w];
    CJAgg5 y = {g.has_head, g.nblocks, g.dc[0], g.dc[1], g.dc[2]};
    acc = cj_op(acc, y);
  }
  sm[threadIdx.x] = acc;
  __syncthreads();
  for (int d = 1; d < (int)blockDim.x; d <<= 1) {
    CJAgg5 x = sm[threadIdx.x];
    CJAgg5 y = threadIdx.x >= (unsigned)d ? sm[threadIdx.x - d] : CJAgg5{0, 0, 0, 0, 0};
    __syncthreads();
    if (threadIdx.x >= (unsigned)d) sm[threadIdx.x] = cj_op(y, x);
    __syncthreads();
  }
  CJAgg5 run = threadIdx.x ? sm[threadIdx.x - 1] : CJAgg5{0, 0, 0, 0, 0};
  for (int w = lo; w < hi; w++) {
    CJWarpAgg o;
    o.has_head = run.f;
    o.nblocks = run.n;
    o.dc[0] = run.a;
    o.dc[1] = run.b;
    o.dc[2] = run.c;
    o.pad[0] = o.pad[1] = o.pad[2] = 0;
    carry[w] = o;
    CJWarpAgg g = wagg[w];
    CJAgg5 y = {g.has_head, g.nblocks, g.dc[0], g.dc[1], g.dc[2]};
    run = cj_op(run, y);
  }
}

// Stage 5: final decode from the settled start states, writing coefficients.
__global__ void __launch_bounds__(CJ_SYNC_THREADS)
k_decode_write(const CJScanParams* __restrict__ prm, const CJSegment* __restrict__ segs,
               const uint32_t* __restrict__ words, const CJSubRec* __restrict__ recs,
               const CJWarpAgg* __restrict__ carry, int16_t* __restrict__ coef, CJStatus* st,
               int sub_bits) {
  __shared__ CJScanParams sp;
  cj_load_params(sp, prm);
  const int nsub = st->nsub, nseg = st->nseg;
  int warp = blockIdx.x * (CJ_SYNC_THREADS / 32) + (threadIdx.x >> 5);
  int lane = threadIdx.x & 31;
  if (warp * 32 >= nsub) return;
  int i = warp * 32 + lane;
  CJLane ln = cj_lane(segs, nseg, nsub, i, sub_bits);
  CJSubRec r;
  if (ln.active) r = recs[i];
  else {
    r.start = r.exit = 0;
    r.nblocks = r.dc[0] = r.dc[1] = r.dc[2] = 0;
  }
  int64_t e0;
  int e1, e2, e3;
  const CJWarpAgg cw = carry[warp];
  cj_warp_prefix(r, ln, cw.nblocks, cw.dc[0], cw.dc[1], cw.dc[2], &e0, &e1, &e2, &e3);
  const CJSegment seg = segs[ln.seg];
  const int64_t first = seg.first_block + e0;
  cj_warp_zero_range(coef, ln.active, first, cj_lane_write_end(ln, seg, r, first));
  if (!ln.active) return;
  cj_write_lane(sp, sp.steps, words, ln, seg, r.start, first, e1, e2, e3, coef, st, sp.zz, ~0ull);
}

// ---------------------------------------------------------------- host side

static void cj_fill_params(JPGReader* jpg, CJScanParams* hp) {
  CJReaderDevice* d = jpg->dev;
  memset(hp, 0, sizeof(*hp));
  for (int s = 0; s < 4; s++) {
    const bool defined = (jpg->huff_defined & (1 << s)) != 0;
    if (defined) cj_build_huff(d->huff[s].counts, d->huff[s].symbols, &hp->huff[s]);
    cj_build_steps(hp->huff[s], d->huff[s].counts, defined, s, &hp->steps);
  }
  static const uint8_t zz[64] = CJ_ZIGZAG_INIT;
  memcpy(hp->zz, zz, 64);
  for (int t = 0; t < 4; t++)
    for (int k = 0; k < 64; k++) hp->qnat[t][zz[k]] = jpg->dq_tables[t][k];
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
  hp->phase_pack = cj_phase_pack(*hp);
}

int cj_scan_launch(JPGReader* jpg) {
  CJReaderDevice* d = jpg->dev;
  int err = cj_gpu_init(jpg);
  if (err) return err;
  CJScanParams* hp = (CJScanParams*)d->h_params.p;
  cj_fill_params(jpg, hp);
  const size_t n = (size_t)(jpg->end - jpg->pos);
  const int S = d->sub_bits;
  d->raw_len = n;
  d->total_blocks = hp->total_blocks;
  d->nseg_exp = hp->nseg_expected;
  d->mark_cap = d->nseg_exp + 1;
  d->nsub_cap = (int)((n * 8 + S - 1) / S) + d->nseg_exp + 1;
  d->nwarp_cap = (d->nsub_cap + 31) / 32;
  const int ntiles = (int)((n + CJ_TILE_BYTES - 1) / CJ_TILE_BYTES) + 1;
  if (cj_dev_ensure(d->params, sizeof(CJScanParams)) || cj_dev_ensure(d->status, sizeof(CJStatus)) ||
      cj_dev_ensure(d->raw, n + 64) || cj_dev_ensure(d->data, n + 64) ||
      cj_dev_ensure(d->tile_keep, (size_t)ntiles * 4) || cj_dev_ensure(d->tile_mark, (size_t)ntiles * 4) ||
      cj_dev_ensure(d->mpos, (size_t)d->mark_cap * 4) || cj_dev_ensure(d->mcode, (size_t)d->mark_cap) ||
      cj_dev_ensure(d->segs, (size_t)d->nseg_exp * sizeof(CJSegment)) ||
      cj_dev_ensure(d->recs, (size_t)d->nsub_cap * sizeof(CJSubRec)) ||
      cj_dev_ensure(d->ckpt, (size_t)d->nsub_cap * CJ_CKPTS * sizeof(CJCkpt)) ||
      cj_dev_ensure(d->snap, (size_t)2 * d->nwarp_cap * sizeof(uint64_t)) ||
      cj_dev_ensure(d->wagg, (size_t)d->nwarp_cap * sizeof(CJWarpAgg)) ||
      cj_dev_ensure(d->carry, (size_t)d->nwarp_cap * sizeof(CJWarpAgg)) ||
      cj_dev_ensure(d->coef, (size_t)d->total_blocks * 128 + 128))
    return CUDA_MEM_ERROR;
  cudaStream_t s = d->stream;
  CJ_CUDA_TRY(cudaEventRecord(d->ev_begin, s), CUDA_KERNEL_LAUNCH_ERROR);
  CJ_CUDA_TRY(cudaMemcpyAsync(d->params.p, hp, sizeof(CJScanParams), cudaMemcpyHostToDevice, s),
              CUDA_MEM_ERROR);
  if (n) CJ_CUDA_TRY(cudaMemcpyAsync(d->raw.p, jpg->pos, n, cudaMemcpyHostToDevice, s), CUDA_MEM_ERROR);
  return cj_scan_device(jpg);
}

// The device decode of the scan staged in d->raw / d->params.
int cj_scan_device(JPGReader* jpg) {
  CJReaderDevice* d = jpg->dev;
  cudaStream_t s = d->stream;
  const size_t n = d->raw_len;
  const int S = d->sub_bits;
  const int ntiles = (int)((n + CJ_TILE_BYTES - 1) / CJ_TILE_BYTES) + 1;
  cj_profile_begin(d);
  CJ_CUDA_TRY(cudaMemsetAsync(d->status.p, 0, sizeof(CJStatus), s), CUDA_MEM_ERROR);
  CJStatus* st = (CJStatus*)d->status.p;
  const uint8_t* raw = (const uint8_t*)d->raw.p;
  k_destuff_count<<<ntiles, CJ_TILE_THREADS, 0, s>>>(raw, (int64_t)n, (int32_t*)d->tile_keep.p,
                                                      (int32_t*)d->tile_mark.p, st);
  cj_after_launch(d, CJ_K_DESTUFF_COUNT);
  k_scan_tiles<<<1, 1024, 0, s>>>((int32_t*)d->tile_keep.p, (int32_t*)d->tile_mark.p, ntiles, st);
  cj_after_launch(d, CJ_K_SCAN_TILES);
  k_destuff_scatter<<<ntiles, CJ_TILE_THREADS, 0, s>>>(
      raw, (int64_t)n, (const int32_t*)d->tile_keep.p, (const int32_t*)d->tile_mark.p,
      (uint8_t*)d->data.p, (uint32_t*)d->mpos.p, (uint8_t*)d->mcode.p, d->mark_cap);
  cj_after_launch(d, CJ_K_DESTUFF_SCATTER);
  k_build_segments<<<1, 1024, 0, s>>>((const CJScanParams*)d->params.p, st,
                                      (const uint32_t*)d->mpos.p, (const uint8_t*)d->mcode.p,
                                      d->mark_cap, (CJSegment*)d->segs.p, d->nseg_exp, S, d->nsub_cap);
  cj_after_launch(d, CJ_K_SEGMENTS);
  const int sync_blocks = (d->nwarp_cap + (CJ_SYNC_THREADS / 32) - 1) / (CJ_SYNC_THREADS / 32);
  uint64_t* snap0 = (uint64_t*)d->snap.p;
  uint64_t* snap1 = snap0 + d->nwarp_cap;
  k_sync_intra<<<sync_blocks, CJ_SYNC_THREADS, 0, s>>>(
      (const CJScanParams*)d->params.p, (const CJSegment*)d->segs.p, (const uint32_t*)d->data.p,
      (CJSubRec*)d->recs.p, (CJCkpt*)d->ckpt.p, snap0, st, S);
  cj_after_launch(d, CJ_K_SYNC_INTRA);
  k_sync_inter<<<sync_blocks, CJ_SYNC_THREADS, 0, s>>>(
      (const CJScanParams*)d->params.p, (const CJSegment*)d->segs.p, (const uint32_t*)d->data.p,
      (CJSubRec*)d->recs.p, (CJCkpt*)d->ckpt.p, snap0, snap1, (CJWarpAgg*)d->wagg.p, st, S);
  cj_after_launch(d, CJ_K_SYNC_INTER);
  d->snap_parity = 1;
  CJ_CUDA_TRY(cudaGetLastError(), CUDA_KERNEL_LAUNCH_ERROR);
  return cj_scan_write(jpg);
}

int cj_scan_write(JPGReader* jpg) {
  CJReaderDevice* d = jpg->dev;
  cudaStream_t s = d->stream;
  CJStatus* st = (CJStatus*)d->status.p;
  const int sync_blocks = (d->nwarp_cap + (CJ_SYNC_THREADS / 32) - 1) / (CJ_SYNC_THREADS / 32);
  CJ_CUDA_TRY(cudaMemsetAsync(&st->dec_err_key, 0, sizeof(unsigned long long), s), CUDA_MEM_ERROR);
  k_scan_warps<<<1, 1024, 0, s>>>((const CJWarpAgg*)d->wagg.p, (CJWarpAgg*)d->carry.p, st);
  cj_after_launch(d, CJ_K_SCAN_WARPS);
  k_decode_write<<<sync_blocks, CJ_SYNC_THREADS, 0, s>>>(
      (const CJScanParams*)d->params.p, (const CJSegment*)d->segs.p, (const uint32_t*)d->data.p,
      (const CJSubRec*)d->recs.p, (const CJWarpAgg*)d->carry.p, (int16_t*)d->coef.p, st,
      d->sub_bits);
  cj_after_launch(d, CJ_K_DECODE_WRITE);
  CJ_CUDA_TRY(cudaEventRecord(d->ev_scan, s), CUDA_KERNEL_LAUNCH_ERROR);
  CJ_CUDA_TRY(cudaGetLastError(), CUDA_KERNEL_LAUNCH_ERROR);
  return 0;
}

// Rare path: a warp's last exit moved during the first fix-up pass, so the
// next warp started from a stale state.  Repeat passes (each one settles at
// least one more warp) until none moves, then redo the write-out.
int cj_scan_resync(JPGReader* jpg) {
  CJReaderDevice* d = jpg->dev;
  cudaStream_t s = d->stream;
  CJStatus* st = (CJStatus*)d->status.p;
  CJStatus* hs = (CJStatus*)d->h_status.p;
  const int sync_blocks = (d->nwarp_cap + (CJ_SYNC_THREADS / 32) - 1) / (CJ_SYNC_THREADS / 32);
  uint64_t* snap[2] = {(uint64_t*)d->snap.p, (uint64_t*)d->snap.p + d->nwarp_cap};
  for (int pass = 0; pass <= d->nwarp_cap + 1; pass++) {
    CJ_CUDA_TRY(cudaMemsetAsync(&st->unstable, 0, sizeof(int32_t), s), CUDA_MEM_ERROR);
    int in = d->snap_parity;
    k_sync_inter<<<sync_blocks, CJ_SYNC_THREADS, 0, s>>>(
        (const CJScanParams*)d->params.p, (const CJSegment*)d->segs.p, (const uint32_t*)d->data.p,
        (CJSubRec*)d->recs.p, (CJCkpt*)d->ckpt.p, snap[in], snap[in ^ 1], (CJWarpAgg*)d->wagg.p, st,
        d->sub_bits);
    cj_after_launch(d, CJ_K_SYNC_INTER);
    d->snap_parity = in ^ 1;
    CJ_CUDA_TRY(cudaMemcpyAsync(hs, st, sizeof(CJStatus), cudaMemcpyDeviceToHost, s), CUDA_MEM_ERROR);
    CJ_CUDA_TRY(cudaStreamSynchronize(s), CUDA_KERNEL_LAUNCH_ERROR);
    if (!hs->unstable) break;
  }
  return cj_scan_write(jpg);
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
