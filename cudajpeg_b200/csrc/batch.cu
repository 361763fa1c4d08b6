// batch.cu -- persistent, cooperative batch decoder: many JPEGs of uneven
// size, subsampling and restart structure decoded by ONE kernel launch.
//
// The whole decode path of scan.cu + pixel.cu runs as phases 0-8 of a single
// cooperative kernel (every CTA co-resident), separated by a grid barrier,
// followed on the same stream by the pixel kernel (phase 9):
//
//   0 tables     build each image's canonical Huffman tables and geometry on
//                the device from its raw DHT/DQT bytes
//   1-3 destuff  count / per-image scan / scatter of every 4 KiB tile
//   4 segments   restart intervals -> segments -> speculative subsequences
//   5 sync       speculative decode + warp settle (every warp item)
//   6 fix-up     passes between warps until no warp's exit moves; the loop is
//                driven on the device, no host round trip
//   7 scan       segmented block / DC prefix over warps
//   8 write      coefficient write-out
//   9 pixel      TMA-staged integer iDCT + upsample + colour per MCU tile
//                (k_pixel_batch, its own launch)
//
// Warp items of phases 5, 6 and 8 are handed out through global work
// counters, so slow items (long synchronisation tails) do not hold up the
// warps behind them.  Data one CTA writes and another
// reads inside the kernel is read with L2-coherent loads (__ldcg).  Errors
// are kept per image: a corrupt image fails alone.
#include <stddef.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include "../../include/cj_dlpack.h"
#include "../../include/cudajpeg.h"
#include "cj_entropy.cuh"
#include "cj_idct.cuh"
#include "cj_internal.h"
#include "cj_parse.cuh"
#include "cj_pixel.cuh"
#include "cj_scan_util.cuh"
#include "cj_tables.h"

#define BT_THREADS 256
// Default bits per speculative subsequence of a batch: with many images
// decoding side by side, long subsequences (fewer lanes and settle chains)
// win; the autotuner chooses 4096 on the mixed 1024-image workload.  The
// single-image paths keep CJ_SUB_BITS_DEFAULT (more lanes per image).
#define BT_SUB_BITS_DEFAULT 4096
#define BT_WARPS (BT_THREADS / 32)
// MCU-phase hypotheses per subsequence at most (the standard's largest MCU
// has 10 blocks)
#define BT_MAX_HYP 10
#define BT_TILE_BYTES 4096  // destuff tile: 256 threads x 16 bytes
#define BT_TILE_BAD (1 << 30)  // flag in a tile's marker count: malformed FF sequence
// fixed shared-memory offsets of the tensor-core form's A tile and basis
// (cj_pix_layout with two coefficient buffers)

// ---------------------------------------------------------------- layouts

// Where one image's data lives in the batch buffers (host-planned).
struct CJImageDesc {
  int64_t src_off, raw_len;  // entropy-coded bytes in the input blob
  int64_t data_off;          // destuffed bytes (16-byte aligned)
  int32_t tile0, ntiles;     // destuff tiles
  int32_t mark0, mark_cap;   // RSTn positions
  int32_t seg0, seg_cap;     // segments
  int32_t sub0, sub_cap;     // subsequences (multiples of 32)
  int32_t ptile0, nptiles;   // pixel tiles
  int32_t T, sub_bits;       // MCUs per pixel tile; bits per subsequence
  int64_t coef0;             // first block in the coefficient buffer
  int64_t out_off;           // output byte offset (fancy mode: of the planar samples)
  int64_t rgb_off;           // fancy mode: byte offset of the RGB output
  int64_t pix0;              // fancy mode: first pixel of the image in the batch's pixel order
};

#define BT_NPHASE 10
struct CJBatchCtl {
  unsigned bar_count, bar_gen;
  int unstable[3];
  int timeout;
  int passes;
  int pad;
  int next_sync, next_write, next_fix[3];  // dynamic work counters
  unsigned pix_done;                      // pixel-kernel CTAs finished
  int next_hyp, next_probe;               // work counters of the phase-hypothesis decodes and probes
  // %globaltimer (ns) at each phase start (CTA 0); t[BT_NPHASE] = end of the
  // pixel kernel (its last CTA)
  unsigned long long t[BT_NPHASE + 1];
};

__device__ __forceinline__ void bt_stamp_any(CJBatchCtl* ctl, int k) {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  ctl->t[k] = t;
}

__device__ __forceinline__ void bt_stamp(CJBatchCtl* ctl, int k) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    ctl->t[k] = t;
  }
}

struct CJBatchArgs {
  const CJImageHeader* hdr;
  const CJImageDesc* desc;
  CJScanParams* prm;
  CJStatus* st;
  const uint8_t* blob;
  uint8_t* data;
  int32_t* tile_keep;
  int32_t* tile_mark;
  uint32_t* mpos;
  uint8_t* mcode;
  CJSegment* segs;
  CJSubRec* recs;
  CJCkpt* ckpt;
  uint64_t* snap0;
  uint64_t* snap1;
  CJWarpAgg* wagg;
  CJWarpAgg* carry;
  int16_t* coef;
  const uint16_t* tc_basis;  // tensor-core form: the Kronecker basis (Khi, Klo) to stage per CTA
  uint8_t* out;
  uint8_t* rgb;   // fancy mode: the RGB output (out then holds planar samples)
  int64_t npix;   // fancy mode: pixels of the batch
  CJBatchCtl* ctl;
  int n, ntiles, nwarps, nptiles, max_passes;
  unsigned wait_limit;  // grid-barrier polls before a timeout (0 = default)
  // MCU-phase hypotheses (0 or 1: none): subsequences not at a segment start
  // are also decoded from their first bit under MCU phases 0 .. nhyp - 1
  // (below each image's blocks per MCU) before the settle, and then from
  // each of their predecessor's hypothesis exits (probes).  Per global
  // subsequence gs: records and checkpoint sets gs * 2 * nhyp + k for
  // hypothesis k and gs * 2 * nhyp + nhyp + p for the probe from the
  // predecessor's hypothesis p; hmap[gs * 16 + p] = the hypothesis whose exit
  // that probe ends on (15: none)
  int nhyp;
  CJSubRec* hrecs;
  CJCkpt* hckpt;
  uint8_t* hmap;
};

// ---------------------------------------------------------------- device helpers

__device__ __forceinline__ void bt_raise(CJStatus* st, int64_t block, int code) {
  atomicMax(&st->err_key, ~(((unsigned long long)block << 8) | (unsigned)code));
}
__device__ __forceinline__ void bt_raise_dec(CJStatus* st, int64_t block, int code) {
  atomicMax(&st->dec_err_key, ~(((unsigned long long)block << 8) | (unsigned)code));
}

// Grid barrier for a cooperative launch (all CTAs co-resident).  The wait is
// bounded by `limit` polls (0: 2^24, about 2 s): a CTA whose wait runs out
// flags the batch (ctl->timeout, read by the host) and returns false, and the
// caller leaves the kernel at once, so no CTA ever runs a phase whose inputs
// the barrier did not complete.  The CTAs still waiting time out in turn.
__device__ __forceinline__ bool bt_grid_sync(CJBatchCtl* ctl, unsigned& gen, unsigned limit, int* s_ok) {
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned g = gen;
    int ok = 1;
    if (atomicAdd(&ctl->bar_count, 1) == gridDim.x - 1) {
      atomicExch(&ctl->bar_count, 0);
      __threadfence();
      atomicAdd(&ctl->bar_gen, 1);
    } else {
      // poll with a relaxed load, not an atomic: hundreds of CTAs polling
      // one word by atomics serialise at its L2 slice, and the releasing
      // CTA's atomics then queue behind them (tens of microseconds when most
      // CTAs wait long, as in the fix-up passes).  Not an acquire load
      // either: each would invalidate the SM's L1 under the warps of other
      // CTAs still working there.  The fence after the loop orders what
      // follows (the releasing CTA fenced before its increment).
      const unsigned lim = limit ? limit : (1u << 24);
      unsigned it = 0, v;
      for (;;) {
        asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(&ctl->bar_gen) : "memory");
        if (v != g) break;
        if (++it >= lim) {
          atomicExch(&ctl->timeout, 1);
          ok = 0;
          break;
        }
        __nanosleep(128);
      }
    }
    __threadfence();
    gen = g + 1;
    *s_ok = ok;
  }
  __syncthreads();
  return *s_ok != 0;
}

// L2-coherent loads of records another SM may have rewritten in this kernel.
__device__ __forceinline__ CJSubRec bt_load_rec(const CJSubRec* p) {
  CJSubRec r;
  const int4* q = reinterpret_cast<const int4*>(p);
  *reinterpret_cast<int4*>(&r) = __ldcg(q);
  *(reinterpret_cast<int4*>(&r) + 1) = __ldcg(q + 1);
  return r;
}
__device__ __forceinline__ CJWarpAgg bt_load_agg(const CJWarpAgg* p) {
  CJWarpAgg r;
  const int4* q = reinterpret_cast<const int4*>(p);
  *reinterpret_cast<int4*>(&r) = __ldcg(q);
  *(reinterpret_cast<int4*>(&r) + 1) = __ldcg(q + 1);
  return r;
}

// ---- hypothesis maps.  A lane's map sends the index p of a predecessor
// hypothesis to the index of its own hypothesis whose exit the decode from
// the predecessor's hypothesis-p exit ends on (15: none of them), packed as
// 16 nibbles; a map of constant value c is c in every nibble.
#define BT_MAP_NONE 0xFFFFFFFFFFFFFFFFull
#define BT_MAP_ID 0xFEDCBA9876543210ull
__device__ __forceinline__ uint32_t bt_map_at(uint64_t f, uint32_t i) {
  return i >= 15 ? 15u : (uint32_t)(f >> (4 * i)) & 15u;
}
__device__ __forceinline__ uint64_t bt_map_const(uint32_t c) { return c >= 15 ? BT_MAP_NONE : 0x1111111111111111ull * c; }
// f after g, on the first n entries (the rest: none)
__device__ __forceinline__ uint64_t bt_map_compose(uint64_t f, uint64_t g, int n) {
  uint64_t o = BT_MAP_NONE;
  for (int i = 0; i < n; i++) o &= ~((uint64_t)(15u ^ bt_map_at(f, bt_map_at(g, (uint32_t)i))) << (4 * i));
  return o;
}

// The settle of the hypothesis variant: cj_warp_settle's loop and fixed
// point, with the probe decodes as shortcuts.  Each round the first lane u
// whose input moved has a final input (every lane before it is consistent).
// If that input is one of its predecessor's hypothesis exits, the lanes from
// u on follow the maps (a warp-wide prefix composition) to the hypothesis
// each predecessor ends on, and every lane with a known predecessor
// hypothesis takes the probe decode from that hypothesis's exit (record and
// checkpoints) without decoding; the other moved lanes re-decode as in
// cj_warp_settle.  Lane u is final after the round, so the loop ends within
// 33 rounds; with the maps defined it ends after one.
__device__ __forceinline__ bool bt_settle_map(const CJBatchArgs& a, const CJScanParams& sp, const CJSteps& T,
                                           const uint32_t* words, const CJLane& ln, bool pred_head, CJSubRec& r,
                                           uint64_t lane0_in, CJCkpt* ck, uint32_t cs, int64_t gs, int nhi) {
  const int lane = threadIdx.x & 31;
  const int NH = a.nhyp;
  const int64_t hb = gs * 2 * NH;
  const CJCkpt* hck = cj_lane_ckpts(a.hckpt, hb);
  const CJSubRec* hrec = a.hrecs + hb;
  uint64_t M = BT_MAP_NONE;
  if (ln.active && ln.head) {
    M = 0;  // a segment's first subsequence starts exactly: its hypothesis 0
  } else if (ln.active) {
    const uint4 mb = __ldcg(reinterpret_cast<const uint4*>(a.hmap + gs * 16));
    const uint32_t wv[4] = {mb.x, mb.y, mb.z, mb.w};
#pragma unroll
    for (int p = 0; p < 16; p++)
      if (p < NH) M &= ~((uint64_t)(15u ^ ((wv[p >> 2] >> (8 * (p & 3))) & 15u)) << (4 * p));
  }
  bool dirty = false;
  for (int it = 0; it < 34; it++) {
    const uint64_t pred = __shfl_up_sync(CJ_FULL, r.exit, 1);
    const uint64_t want = ln.head ? r.start : (lane == 0 ? lane0_in : pred);
    const bool change = ln.active && want != r.start;
    const unsigned cb = __ballot_sync(CJ_FULL, change);
    if (!cb) break;
    const int u = __ffs(cb) - 1;
    uint32_t q = 15;  // lane u: its input as a predecessor hypothesis
    if (lane == u) {
      const CJSubRec* ph = a.hrecs + (gs - 1) * 2 * NH;
      const int pmax = pred_head ? 0 : nhi;
      for (int p = 0; p <= pmax; p++)
        if (__ldcg(&ph[p].exit) == want) {
          q = (uint32_t)p;
          break;
        }
    }
    uint64_t v = lane < u ? BT_MAP_ID : (lane == u ? bt_map_const(bt_map_at(M, q)) : M);
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint64_t g = __shfl_up_sync(CJ_FULL, v, d);
      if (lane >= d) v = bt_map_compose(v, g, NH);
    }
    uint32_t pidx = __shfl_up_sync(CJ_FULL, (uint32_t)v & 15u, 1);
    if (lane == u) pidx = q;
    if (ln.active && !ln.head && lane >= u && pidx < 15) {
      const CJSubRec* pr = hrec + NH + pidx;
      if (__ldcg(&pr->start) != r.start) {
        r = bt_load_rec(pr);
        const CJCkpt* pc = cj_lane_ckpts(a.hckpt, hb + NH + pidx);
        for (int k = 0; k < CJ_CKPTS; k++)
          ck[k] = CJCkpt{__ldcg(&pc[k].pp), __ldcg(&pc[k].nb), __ldcg(&pc[k].d0), __ldcg(&pc[k].d1),
                         __ldcg(&pc[k].d2)};
        dirty = true;
      }
    } else if (change) {
      r = cj_spec_decode<true, true>(sp, T, words, ln, want, ck, r, cs, hck, hrec, nhi + 1);
      dirty = true;
    }
  }
  return dirty;
}

// Next warp item from a work counter (lane 0 takes it, the warp shares it).
__device__ __forceinline__ int bt_next_item(int* counter) {
  int w = 0;
  if ((threadIdx.x & 31) == 0) w = atomicAdd(counter, 1);
  return __shfl_sync(0xFFFFFFFFu, w, 0);
}

// Next group of BT_WARPS consecutive items for the whole CTA (thread 0 takes
// it, the CTA shares it).  The leading barrier also ends the previous group:
// every warp is done with it and with the tables staged for it.
__device__ __forceinline__ int bt_next_group(int* counter, int* s_slot) {
  __syncthreads();
  if (threadIdx.x == 0) *s_slot = atomicAdd(counter, BT_WARPS);
  __syncthreads();
  return *s_slot;
}

// Copy one image's decode-step tables (16 KB) into shared memory.  The
// tables were built by another CTA in this kernel: read them from L2.
__device__ __forceinline__ void bt_copy_steps(CJSteps* dst, const CJSteps* src) {
  const int4* s = reinterpret_cast<const int4*>(src);
  int4* d = reinterpret_cast<int4*>(dst);
  for (int k = threadIdx.x; k < (int)(sizeof(CJSteps) / 16); k += blockDim.x) d[k] = __ldcg(s + k);
}

// Largest i with key(i) <= v over a sorted int32 field of the descriptors.
template <class F>
__device__ __forceinline__ int bt_find(int n, int v, F key) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (key(mid) <= v) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Step tables of the sync and fix-up phases, staged per item group: a group's warps
// [wa, wb] span few images, and the step tables of the first and the last
// of them are copied into shared memory (slots 0 and 1), so every symbol
// lookup is a shared-memory load instead of an L2 round trip (the tables of
// all images of a batch do not fit in L1).  Images strictly between the two
// (a run of tiny images) read their tables from global memory.
struct BTStaged {
  int ia, ib;
};
// Dynamic shared memory of the decode kernel: two staged table slots in the
// sync and fix-up phases, the write-out's block buffers (one 64-entry int16
// block per thread) in phase 8.  More would shrink the L1 share the
// bitstream reads of the sync phase depend on.
#define BT_WBUF_BYTES (BT_THREADS * 64 * 2)
#define BT_DECODE_SMEM (2 * sizeof(CJSteps))
static_assert(BT_DECODE_SMEM >= BT_WBUF_BYTES, "write-out block buffers");
static_assert(sizeof(CJSteps) % 16 == 0 && offsetof(CJScanParams, steps) % 16 == 0, "int4 table copy");
static_assert(BT_DECODE_SMEM >= BT_THREADS * sizeof(CJAgg5), "phase 7 scan space");

__device__ __forceinline__ int bt_image_of_warp(const CJBatchArgs& a, int w) {
  return bt_find(a.n, w, [&](int k) { return a.desc[k].sub0 >> 5; });
}

// All threads of the CTA: stage the tables of warps [wa, wb]'s first and last image.
__device__ __forceinline__ BTStaged bt_stage(const CJBatchArgs& a, int wa, int wb, CJSteps* tab) {
  BTStaged g;
  g.ia = bt_image_of_warp(a, wa);
  g.ib = bt_image_of_warp(a, wb);
  bt_copy_steps(&tab[0], &a.prm[g.ia].steps);
  if (g.ib != g.ia) bt_copy_steps(&tab[1], &a.prm[g.ib].steps);
  __syncthreads();
  return g;
}

__device__ __forceinline__ const CJSteps& bt_steps_of(const CJBatchArgs& a, const BTStaged& g, const CJSteps* tab,
                                                      int i) {
  return i == g.ia ? tab[0] : (i == g.ib ? tab[1] : a.prm[i].steps);
}

__constant__ uint8_t c_bt_zz[64] = CJ_ZIGZAG_INIT;  // zig-zag -> natural index

// Phase 0: one CTA builds one image's CJScanParams (the device twin of
// cj_build_huff + cj_fill_params).
__device__ void bt_build_params(const CJImageHeader& h, CJScanParams& p) {
  for (int e = threadIdx.x; e < 4 * (1 << CJ_FAST_BITS); e += blockDim.x) {
    int slot = e >> CJ_FAST_BITS, f = e & ((1 << CJ_FAST_BITS) - 1);
    uint16_t out = 0;
    if (h.huff_mask & (1 << slot)) {
      int code = 0, k = 0;
      for (int l = 1; l <= CJ_FAST_BITS; l++) {
        int n = h.counts[slot][l - 1];
        int c = f >> (CJ_FAST_BITS - l);
        if (c >= code && c < code + n) {
          out = (uint16_t)((l << 8) | h.symbols[slot][k + c - code]);
          break;
        }
        k += n;
        code = (code + n) << 1;
      }
    }
    p.huff[slot].fast[f] = out;
  }
  for (int e = threadIdx.x; e < 4 * 256; e += blockDim.x) p.huff[e >> 8].vals[e & 255] = h.symbols[e >> 8][e & 255];
  if (threadIdx.x < 4) {
    int slot = threadIdx.x;
    int code = 0, k = 0;
    p.huff[slot].maxcode[0] = -1;
    p.huff[slot].valoff[0] = 0;
    for (int l = 1; l <= 16; l++) {
      int n = h.counts[slot][l - 1];
      p.huff[slot].valoff[l] = k - code;
      code += n;
      k += n;
      p.huff[slot].maxcode[l] = n ? code - 1 : -1;
      code <<= 1;
    }
    p.huff[slot].maxcode[17] = -1;
    p.huff[slot].valoff[17] = 0;
  }
  // decode steps from the finished canonical tables (cj_build_steps); the
  // long-code prefix range of each slot is computed once
  __shared__ int s_pre[4][2];
  if (threadIdx.x < 4) {
    int pmin = 1 << CJ_FAST_BITS, pmax = -1;
    if (h.huff_mask & (1 << threadIdx.x)) cj_long_prefixes(h.counts[threadIdx.x], &pmin, &pmax);
    s_pre[threadIdx.x][0] = pmin;
    s_pre[threadIdx.x][1] = pmax;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < 4 * (1 << CJ_FAST_BITS); e += blockDim.x) {
    const int slot = e >> CJ_FAST_BITS, f = e & ((1 << CJ_FAST_BITS) - 1);
    const bool defined = (h.huff_mask & (1 << slot)) != 0;
    p.steps.pri[slot][f] = defined ? cj_step_primary(p.huff[slot], s_pre[slot][0], s_pre[slot][1], f, slot >= 2)
                                   : (uint16_t)CJ_STEP_BAD;
  }
  for (int e = threadIdx.x; e < 4 * CJ_STEP_SUBS * 64; e += blockDim.x) {
    const int slot = e / (CJ_STEP_SUBS * 64), i = (e >> 6) % CJ_STEP_SUBS, j = e & 63;
    const int pmin = s_pre[slot][0], pmax = s_pre[slot][1];
    const bool used = (h.huff_mask & (1 << slot)) && pmin + i <= pmax;
    p.steps.sub[slot][i][j] = used ? cj_step_sub(p.huff[slot], pmin, i, j, slot >= 2) : (uint16_t)CJ_STEP_BAD;
  }
  __syncthreads();  // s_pre is reused by the next image of this CTA
  for (int e = threadIdx.x; e < 4 * 64; e += blockDim.x) p.qnat[e >> 6][c_bt_zz[e & 63]] = h.dq[e >> 6][e & 63];
  if (threadIdx.x < 64) p.zz[threadIdx.x] = c_bt_zz[threadIdx.x];
  if (threadIdx.x == 0) {
    int k = 0;
    for (int c = 0; c < h.nch; c++)
      for (int j = 0; j < h.comp_sx[c] * h.comp_sy[c]; j++, k++) {
        p.phase_comp[k] = (uint8_t)c;
        p.phase_blk[k] = (uint8_t)j;
      }
    for (int c = 0; c < 3; c++) {
      p.comp_dc[c] = h.comp_dc[c];
      p.comp_ac[c] = h.comp_ac[c];
      p.comp_q[c] = h.comp_q[c];
      p.comp_sx[c] = h.comp_sx[c];
      p.comp_sy[c] = h.comp_sy[c];
      p.comp_stride[c] = h.mcux * h.comp_sx[c] * 8;
      p.comp_rows[c] = h.mcuy * h.comp_sy[c] * 8;
    }
    p.nch = h.nch;
    p.bpm = k;
    p.mcux = h.mcux;
    p.mcuy = h.mcuy;
    p.width = h.width;
    p.height = h.height;
    p.hmax = h.hmax;
    p.vmax = h.vmax;
    p.xshift = h.xshift;
    p.yshift = h.yshift;
    p.restart_interval = h.restart_interval;
    p.nseg_expected = h.nseg_expected;
    p.total_blocks = h.total_blocks;
    p.phase_pack = cj_phase_pack(p);
  }
}

// ---------------------------------------------------------------- the kernel

__device__ __forceinline__ uint32_t bt_smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// MINB = CTAs per SM the register allocation is sized for (64 registers at
// 4); the autotuner picks among the compiled variants.  HYP: the variant
// with MCU-phase hypotheses (phase 5a), launched only for latency-bound
// decodes (a.nhyp > 1), so the throughput variants carry none of its code.
template <int MINB, bool HYP = false>
__global__ void __launch_bounds__(BT_THREADS, MINB) k_decode_batch(CJBatchArgs a) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ int2 sm2[33];
  __shared__ uint8_t s_zz[64];
  __shared__ int s_grp, s_ok;
  unsigned gen = 0;
  if (threadIdx.x == 0) gen = atomicAdd(&a.ctl->bar_gen, 0);
  if (threadIdx.x < 64) s_zz[threadIdx.x] = c_bt_zz[threadIdx.x];
  const int lane = threadIdx.x & 31;

  bt_stamp(a.ctl, 0);
  // ---- phase 0: tables + status
  for (int i = blockIdx.x; i < a.n; i += gridDim.x) {
    bt_build_params(a.hdr[i], a.prm[i]);
    if (threadIdx.x == 0) {
      CJStatus z;
      memset(&z, 0, sizeof(z));
      a.st[i] = z;
    }
  }
  // no grid barrier: phase 1 reads nothing phase 0 writes (a tile's marker
  // error goes to its count and reaches the image's status in phase 2)

  bt_stamp(a.ctl, 1);
  // ---- phase 1: destuff count.  Each CTA takes a contiguous run of tiles
  // (equal 4 KB pieces), so the image index only walks forward.
  const int tper = (a.ntiles + gridDim.x - 1) / gridDim.x;
  const int tt0 = blockIdx.x * tper, tt1 = min(tt0 + tper, a.ntiles);
  const int timg0 = tt0 < tt1 ? bt_find(a.n, tt0, [&](int k) { return a.desc[k].tile0; }) : 0;
  // a tile's chunk (tile t of the run, image index i walking forward)
  auto tile_in = [&](int t, int& i) -> CJChunkIn {
    while (t >= a.desc[i].tile0 + a.desc[i].ntiles) i++;
    const CJImageDesc& d = a.desc[i];
    return cj_chunk_load(a.blob + d.src_off, d.raw_len, (int64_t)(t - d.tile0) * BT_TILE_BYTES + threadIdx.x * 16);
  };
  int pi = timg0;  // image of the prefetched tile
  CJChunkIn nx;
  if (tt0 < tt1) nx = tile_in(tt0, pi);
  for (int t = tt0, i = timg0; t < tt1; t++) {
    while (t >= a.desc[i].tile0 + a.desc[i].ntiles) i++;
    const CJImageDesc& d = a.desc[i];
    int64_t base = (int64_t)(t - d.tile0) * BT_TILE_BYTES + threadIdx.x * 16;
    const CJChunkIn in = nx;
    if (t + 1 < tt1) nx = tile_in(t + 1, pi);  // the next tile's load overlaps this one's scan
    CJChunk c = cj_classify_in(in, d.raw_len, base);
    int2 tot;
    cj_block_exclusive(make_int2(__popc(c.keep), __popc(c.mark)), sm2, &tot);
    const int bad = __syncthreads_or(c.bad);
    if (threadIdx.x == 0) {
      a.tile_keep[t] = tot.x;
      a.tile_mark[t] = tot.y | (bad ? BT_TILE_BAD : 0);  // counts stay below 2^13
    }
  }
  if (!bt_grid_sync(a.ctl, gen, a.wait_limit, &s_ok)) return;

  bt_stamp(a.ctl, 2);
  // ---- phase 2: per-image tile offsets
  for (int i = blockIdx.x; i < a.n; i += gridDim.x) {
    const CJImageDesc& d = a.desc[i];
    int2 run = make_int2(0, 0);
    int bad = 0;
    for (int t0 = 0; t0 < d.ntiles; t0 += blockDim.x) {
      int t = t0 + threadIdx.x;
      int2 v = make_int2(0, 0);
      if (t < d.ntiles) v = make_int2(__ldcg(&a.tile_keep[d.tile0 + t]), __ldcg(&a.tile_mark[d.tile0 + t]));
      bad |= v.y & BT_TILE_BAD;
      v.y &= ~BT_TILE_BAD;
      int2 tot;
      int2 ex = cj_block_exclusive(v, sm2, &tot);
      if (t < d.ntiles) {
        a.tile_keep[d.tile0 + t] = run.x + ex.x;
        a.tile_mark[d.tile0 + t] = run.y + ex.y;
      }
      run.x += tot.x;
      run.y += tot.y;
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) bt_raise(&a.st[i], 0, CJ_DEV_MARKER);
    if (threadIdx.x == 0) {
      a.st[i].destuffed = run.x;
      a.st[i].nmarkers = run.y;
    }
  }
  if (!bt_grid_sync(a.ctl, gen, a.wait_limit, &s_ok)) return;

  bt_stamp(a.ctl, 3);
  // ---- phase 3: destuff scatter, over the same tile runs.  A tile's kept
  // bytes are compacted in shared memory and then written to their
  // contiguous destination [o0, o0 + n) as aligned 4-byte words; only the
  // partial words at the two ends, which may border another tile's bytes,
  // are written byte by byte.
  pi = timg0;
  if (tt0 < tt1) nx = tile_in(tt0, pi);
  for (int t = tt0, i = timg0; t < tt1; t++) {
    while (t >= a.desc[i].tile0 + a.desc[i].ntiles) i++;
    const CJImageDesc& d = a.desc[i];
    int64_t base = (int64_t)(t - d.tile0) * BT_TILE_BYTES + threadIdx.x * 16;
    const CJChunkIn in = nx;
    if (t + 1 < tt1) nx = tile_in(t + 1, pi);
    CJChunk c = cj_classify_in(in, d.raw_len, base);
    int2 tot;
    int2 ex = cj_block_exclusive(make_int2(__popc(c.keep), __popc(c.mark)), sm2, &tot);
    const int64_t o0 = (int64_t)__ldcg(&a.tile_keep[t]);
    int q = ex.x;
    int r = __ldcg(&a.tile_mark[t]) + ex.y;
#pragma unroll
    for (int j = 0; j < 16; j++) {
      if (c.keep & (1u << j)) smem[q++] = (uint8_t)cj_byte(c, j);
      if (c.mark & (1u << j)) {
        if (r < d.mark_cap) {
          a.mpos[d.mark0 + r] = (uint32_t)(o0 + q);
          a.mcode[d.mark0 + r] = (uint8_t)(j < 15 ? cj_byte(c, j + 1) : c.next);
        }
        r++;
      }
    }
    __syncthreads();
    uint8_t* out = a.data + d.data_off;
    const int n = tot.x;
    const int64_t wb = (o0 + 3) >> 2, we = (o0 + n) >> 2;  // words wholly inside the range
    if (wb < we) {
      for (int64_t w = wb + threadIdx.x; w < we; w += BT_THREADS) {
        const int sofs = (int)(4 * w - o0);
        reinterpret_cast<uint32_t*>(out)[w] = (uint32_t)smem[sofs] | ((uint32_t)smem[sofs + 1] << 8) |
                                              ((uint32_t)smem[sofs + 2] << 16) | ((uint32_t)smem[sofs + 3] << 24);
      }
      const int head = (int)(4 * wb - o0), tail = (int)(o0 + n - 4 * we);
      if ((int)threadIdx.x < head) out[o0 + threadIdx.x] = smem[threadIdx.x];
      if ((int)threadIdx.x < tail) out[4 * we + threadIdx.x] = smem[4 * we - o0 + threadIdx.x];
    } else {
      for (int k = threadIdx.x; k < n; k += BT_THREADS) out[o0 + k] = smem[k];
    }
    __syncthreads();
  }
  if (!bt_grid_sync(a.ctl, gen, a.wait_limit, &s_ok)) return;

  bt_stamp(a.ctl, 4);
  // ---- phase 4: segments and subsequences, one CTA per image
  for (int i = blockIdx.x; i < a.n; i += gridDim.x) {
    const CJImageDesc& d = a.desc[i];
    const CJScanParams& p = a.prm[i];
    CJStatus* st = &a.st[i];
    const int M = __ldcg(&st->nmarkers);
    const int64_t L = __ldcg(&st->destuffed);
    const int RI = __ldcg(&p.restart_interval);
    const int E = RI ? __ldcg(&p.nseg_expected) : 1;
    const int64_t total = __ldcg(&p.total_blocks);
    const int64_t per_seg = RI ? (int64_t)RI * __ldcg(&p.bpm) : total;
    const uint32_t* mpos = a.mpos + d.mark0;
    const uint8_t* mcode = a.mcode + d.mark0;
    bool ok;
    if (RI == 0) ok = (M == 0);
    else if (M == E - 1) ok = true;
    else if (M == E && M <= d.mark_cap && __ldcg(&mpos[M - 1]) == (uint32_t)L) ok = true;
    else ok = false;
    if (M > d.mark_cap || E > d.seg_cap) ok = false;
    if (!ok) {
      if (threadIdx.x == 0) {
        bt_raise(st, 0, CJ_DEV_MARKER);
        st->nsub = 0;
        st->nseg = 0;
      }
      continue;
    }
    int running = 0;
    for (int k0 = 0; k0 < E; k0 += blockDim.x) {
      int k = k0 + threadIdx.x;
      int64_t begin = 0, end = 0;
      int nsub = 0;
      if (k < E) {
        begin = k ? __ldcg(&mpos[k - 1]) : 0;
        end = k < M ? (int64_t)__ldcg(&mpos[k]) : L;
        if (k < M && __ldcg(&mcode[k]) != 0xD0 + (k & 7)) bt_raise(st, (int64_t)k * per_seg, CJ_DEV_MARKER);
        nsub = (int)(((end - begin) * 8 + d.sub_bits - 1) / d.sub_bits);
        if (nsub < 1) nsub = 1;
      }
      int2 tot;
      int2 ex = cj_block_exclusive(make_int2(nsub, 0), sm2, &tot);
      if (k < E) {
        CJSegment s;
        s.bit_begin = (uint64_t)begin * 8;
        s.bit_end = (uint64_t)end * 8;
        s.first_block = (int64_t)k * per_seg;
        s.nblocks = min(per_seg, total - s.first_block);
        s.first_sub = running + ex.x;
        s.nsub = nsub;
        s.marker_follows = k < M;
        s.pad = 0;
        a.segs[d.seg0 + k] = s;
      }
      running += tot.x;
    }
    if (threadIdx.x == 0) {
      st->nseg = E;
      if (running > d.sub_cap) {
        bt_raise(st, 0, CJ_DEV_CAPACITY);
        running = 0;
      }
      st->nsub = running;
    }
  }
  if (!bt_grid_sync(a.ctl, gen, a.wait_limit, &s_ok)) return;

  bt_stamp(a.ctl, 5);
  CJSteps* tab = reinterpret_cast<CJSteps*>(smem);
  // ---- phase 5a (latency-bound decodes only): MCU-phase hypotheses.  A
  // subsequence's guessed start (its first bit, MCU phase 0) lines up with
  // the true decode only after hundreds to thousands of bits for
  // multi-component scans, while one of the decodes from its first bit
  // under the other phases usually does within a few blocks; the settle
  // below may join any of them at a checkpoint.  Items: (hypothesis, group
  // of BT_WARPS warps), each hypothesis's warps padded to whole groups.
  const int nh = HYP && a.nhyp > 1 ? a.nhyp - 1 : 0;
  if (HYP && nh) {
    const int nw8 = (a.nwarps + BT_WARPS - 1) / BT_WARPS * BT_WARPS;
    for (;;) {
      const int g0 = bt_next_group(&a.ctl->next_hyp, &s_grp);
      if (g0 >= (nh + 1) * nw8) break;
      const int h = g0 / nw8, wg = g0 - h * nw8;  // hypothesis h = 0 .. nh (0: the usual guess)
      if (wg >= a.nwarps) continue;  // CTA-uniform
      const BTStaged sg = bt_stage(a, wg, min(wg + BT_WARPS, a.nwarps) - 1, tab);
      const int w = wg + (int)(threadIdx.x >> 5);
      if (w >= a.nwarps) continue;  // warp-uniform
      const int i = bt_image_of_warp(a, w);
      const CJImageDesc& d = a.desc[i];
      const int nsub = __ldcg(&a.st[i].nsub), nseg = __ldcg(&a.st[i].nseg);
      const int j0 = w * 32 - d.sub0;
      if (j0 >= nsub) continue;  // warp-uniform
      const CJScanParams& sp = a.prm[i];
      if (h && h >= sp.bpm) continue;  // warp-uniform: no such phase in this image
      CJLane ln = cj_lane(a.segs + d.seg0, nseg, nsub, j0 + lane, d.sub_bits);
      // a segment's first subsequence starts exactly: phase 0 only.
      // Hypothesis 0 is also the settle's starting record.
      if (ln.active && (h == 0 || !ln.head)) {
        const int64_t gs = d.sub0 + j0 + lane, hs = gs * 2 * (nh + 1) + h;
        CJSubRec r;
        r.start = cj_state(ln.begin, (uint32_t)h);
        r.exit = r.start;
        r.nblocks = r.dc[0] = r.dc[1] = r.dc[2] = 0;
        CJCkpt* hc = cj_lane_ckpts(a.hckpt, hs);
        r = cj_spec_decode<false>(sp, bt_steps_of(a, sg, tab, i),
                                  reinterpret_cast<const uint32_t*>(a.data + d.data_off), ln, r.start, hc, r,
                                  cj_ckpt_step(d.sub_bits));
        a.hrecs[hs] = r;
        if (h == 0) {
          a.recs[gs] = r;
          CJCkpt* ck = cj_lane_ckpts(a.ckpt, gs);
          for (int k = 0; k < CJ_CKPTS; k++) ck[k] = hc[k];
        }
      }
    }
    if (!bt_grid_sync(a.ctl, gen, a.wait_limit, &s_ok)) return;
    // ---- phase 5b: probes.  Each subsequence decoded from each of its
    // predecessor's hypothesis exits (joining its own hypotheses at a
    // checkpoint, usually the first): the decode it takes once its
    // predecessor is known to end on that hypothesis, and the map entry
    // naming the hypothesis it ends on.  Items: (predecessor hypothesis,
    // group of BT_WARPS warps), as in phase 5a.
    for (;;) {
      const int g0 = bt_next_group(&a.ctl->next_probe, &s_grp);
      if (g0 >= (nh + 1) * nw8) break;
      const int p = g0 / nw8, wg = g0 - p * nw8;
      if (wg >= a.nwarps) continue;  // CTA-uniform
      const BTStaged sg = bt_stage(a, wg, min(wg + BT_WARPS, a.nwarps) - 1, tab);
      const int w = wg + (int)(threadIdx.x >> 5);
      if (w >= a.nwarps) continue;  // warp-uniform
      const int i = bt_image_of_warp(a, w);
      const CJImageDesc& d = a.desc[i];
      const int nsub = __ldcg(&a.st[i].nsub), nseg = __ldcg(&a.st[i].nseg);
      const int j0 = w * 32 - d.sub0;
      if (j0 >= nsub) continue;  // warp-uniform
      const CJScanParams& sp = a.prm[i];
      const int nhi = min(nh, sp.bpm - 1);
      CJLane ln = cj_lane(a.segs + d.seg0, nseg, nsub, j0 + lane, d.sub_bits);
      const int64_t gs = d.sub0 + j0 + lane, hb = gs * 2 * (nh + 1);
      uint8_t mk = 15;
      const bool pred_head = ln.active && !ln.head && j0 + lane - 1 == a.segs[d.seg0 + ln.seg].first_sub;
      if (ln.active && !ln.head && p <= (pred_head ? 0 : nhi)) {
        CJCkpt* pc = cj_lane_ckpts(a.hckpt, hb + (nh + 1) + p);
        for (int k = 0; k < CJ_CKPTS; k++) pc[k].pp = 0xFFFFFFFFu;  // matches no decode state
        CJSubRec r;
        r.start = r.exit = __ldcg(&a.hrecs[(gs - 1) * 2 * (nh + 1) + p].exit);
        r.nblocks = r.dc[0] = r.dc[1] = r.dc[2] = 0;
        r = cj_spec_decode<true, true>(sp, bt_steps_of(a, sg, tab, i),
                                       reinterpret_cast<const uint32_t*>(a.data + d.data_off), ln, r.start, pc, r,
                                       cj_ckpt_step(d.sub_bits), cj_lane_ckpts(a.hckpt, hb), a.hrecs + hb, nhi + 1);
        a.hrecs[hb + (nh + 1) + p] = r;
        for (int k = 0; k <= nhi; k++)
          if (__ldcg(&a.hrecs[hb + k].exit) == r.exit) {
            mk = (uint8_t)k;
            break;
          }
      }
      if (ln.active) a.hmap[gs * 16 + p] = mk;
    }
    if (!bt_grid_sync(a.ctl, gen, a.wait_limit, &s_ok)) return;
  }
  // ---- phase 5: speculative decode + warp settle, in groups of BT_WARPS
  // consecutive warps per CTA (handed out dynamically) with staged tables
  for (;;) {
    const int g0 = bt_next_group(&a.ctl->next_sync, &s_grp);
    if (g0 >= a.nwarps) break;
    const BTStaged sg = bt_stage(a, g0, min(g0 + BT_WARPS, a.nwarps) - 1, tab);
    const int w = g0 + (int)(threadIdx.x >> 5);
    if (w >= a.nwarps) continue;  // warp-uniform
    const int i = bt_image_of_warp(a, w);
    const CJImageDesc& d = a.desc[i];
    const int nsub = __ldcg(&a.st[i].nsub), nseg = __ldcg(&a.st[i].nseg);
    const int j0 = w * 32 - d.sub0;
    if (j0 >= nsub) continue;  // warp-uniform
    const CJScanParams& sp = a.prm[i];
    const CJSteps& T = bt_steps_of(a, sg, tab, i);
    const uint32_t* words = reinterpret_cast<const uint32_t*>(a.data + d.data_off);
    CJLane ln = cj_lane(a.segs + d.seg0, nseg, nsub, j0 + lane, d.sub_bits);
    CJSubRec r;
    r.start = cj_state(ln.begin, 0);
    r.exit = r.start;
    r.nblocks = r.dc[0] = r.dc[1] = r.dc[2] = 0;
    CJCkpt* ck = cj_lane_ckpts(a.ckpt, d.sub0 + j0 + lane);
    const uint32_t cs = cj_ckpt_step(d.sub_bits);
    if constexpr (HYP) {
      // The phase-0 decodes of phase 5a, settled with the probes of phase 5b
      // (lane 0 keeps its guess until the fix-up passes)
      if (nh) {
        const int64_t gs = d.sub0 + j0 + lane;
        const bool pred_head = ln.active && !ln.head && j0 + lane - 1 == a.segs[d.seg0 + ln.seg].first_sub;
        if (ln.active) r = bt_load_rec(&a.recs[gs]);
        bt_settle_map(a, sp, T, words, ln, pred_head, r, r.start, ck, cs, gs, min(nh, sp.bpm - 1));
      } else {
        if (ln.active) r = cj_spec_decode<false>(sp, T, words, ln, r.start, ck, r, cs);
        cj_warp_settle(sp, T, words, ln, r, r.start, ck, cs);
      }
    } else {
      if (ln.active) r = cj_spec_decode<false>(sp, T, words, ln, r.start, ck, r, cs);
      cj_warp_settle(sp, T, words, ln, r, r.start, ck, cs);
    }
    if (ln.active) a.recs[d.sub0 + j0 + lane] = r;
    unsigned act = __ballot_sync(CJ_FULL, ln.active);
    if (lane == 31 - __clz(act)) a.snap0[w] = r.exit;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.ctl->unstable[0] = 0;
    a.ctl->unstable[1] = 0;
  }
  if (!bt_grid_sync(a.ctl, gen, a.wait_limit, &s_ok)) return;

  bt_stamp(a.ctl, 6);
  // ---- phase 6: fix-up passes until no warp's last exit moves
  int pass = 0;
  for (; pass < a.max_passes; pass++) {
    const uint64_t* snap_in = (pass & 1) ? a.snap1 : a.snap0;
    uint64_t* snap_out = (pass & 1) ? a.snap0 : a.snap1;
    int* unstable = &a.ctl->unstable[pass % 3];
    int* next = &a.ctl->next_fix[pass % 3];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      a.ctl->unstable[(pass + 1) % 3] = 0;
      a.ctl->next_fix[(pass + 1) % 3] = 0;
    }
    for (;;) {
      const int g0 = bt_next_group(next, &s_grp);
      if (g0 >= a.nwarps) break;
      const int w = g0 + (int)(threadIdx.x >> 5);
      bool work = w < a.nwarps;  // warp-uniform, like everything below
      int i = 0, nsub = 0, nseg = 0, j0 = 0;
      if (work) {
        i = bt_image_of_warp(a, w);
        nsub = __ldcg(&a.st[i].nsub);
        nseg = __ldcg(&a.st[i].nseg);
        j0 = w * 32 - a.desc[i].sub0;
        if (j0 >= nsub) {
          if (lane == 0) {
            CJWarpAgg z;
            memset(&z, 0, sizeof(z));
            a.wagg[w] = z;
          }
          work = false;
        }
      }
      const CJImageDesc& d = a.desc[i];
      CJLane ln = cj_lane(a.segs + d.seg0, nseg, work ? nsub : 0, j0 + lane, d.sub_bits);
      CJSubRec r;
      if (ln.active) r = bt_load_rec(&a.recs[d.sub0 + j0 + lane]);
      else {
        r.start = r.exit = 0;
        r.nblocks = r.dc[0] = r.dc[1] = r.dc[2] = 0;
      }
      const uint64_t in0 = (work && j0 > 0 && lane == 0) ? __ldcg(&snap_in[w - 1]) : r.start;
      // the settle's first test; only a group with a lane to re-decode stages tables
      const uint64_t pred = __shfl_up_sync(CJ_FULL, r.exit, 1);
      const uint64_t want = ln.head ? r.start : (lane == 0 ? in0 : pred);
      BTStaged sg = {-1, -1};
      if (__syncthreads_or(ln.active && want != r.start)) sg = bt_stage(a, g0, min(g0 + BT_WARPS, a.nwarps) - 1, tab);
      if (!work) continue;
      const CJScanParams& sp = a.prm[i];
      const uint32_t* words = reinterpret_cast<const uint32_t*>(a.data + d.data_off);
      const CJSteps& T = bt_steps_of(a, sg, tab, i);
      CJCkpt* ck = cj_lane_ckpts(a.ckpt, d.sub0 + j0 + lane);
      const uint32_t cs = cj_ckpt_step(d.sub_bits);
      bool moved;
      if constexpr (HYP) {
        if (nh) {
          const bool pred_head = ln.active && !ln.head && j0 + lane - 1 == a.segs[d.seg0 + ln.seg].first_sub;
          moved = bt_settle_map(a, sp, T, words, ln, pred_head, r, in0, ck, cs, (int64_t)(d.sub0 + j0 + lane),
                                min(nh, sp.bpm - 1));
        } else {
          moved = cj_warp_settle(sp, T, words, ln, r, in0, ck, cs);
        }
      } else {
        moved = cj_warp_settle(sp, T, words, ln, r, in0, ck, cs);
      }
      if (moved && ln.active)
        a.recs[d.sub0 + j0 + lane] = r;
      unsigned act = __ballot_sync(CJ_FULL, ln.active);
      if (lane == 31 - __clz(act)) {
        if (r.exit != __ldcg(&snap_in[w])) atomicAdd(unstable, 1);
        snap_out[w] = r.exit;
      }
      unsigned heads = __ballot_sync(CJ_FULL, ln.active && ln.head);
      int h = heads ? 31 - __clz(heads) : 0;
      bool use = ln.active && lane >= h;
      int v0 = use ? r.nblocks : 0, v1 = use ? r.dc[0] : 0, v2 = use ? r.dc[1] : 0,
          v3 = use ? r.dc[2] : 0;
#pragma unroll
      for (int dd = 16; dd; dd >>= 1) {
        v0 += __shfl_xor_sync(CJ_FULL, v0, dd);
        v1 += __shfl_xor_sync(CJ_FULL, v1, dd);
        v2 += __shfl_xor_sync(CJ_FULL, v2, dd);
        v3 += __shfl_xor_sync(CJ_FULL, v3, dd);
      }
      if (lane == 0) {
        CJWarpAgg g;
        g.has_head = heads != 0;
        g.nblocks = v0;
        g.dc[0] = v1;
        g.dc[1] = v2;
        g.dc[2] = v3;
        g.pad[0] = g.pad[1] = g.pad[2] = 0;
        a.wagg[w] = g;
      }
    }
    if (!bt_grid_sync(a.ctl, gen, a.wait_limit, &s_ok)) return;
    // the barrier orders every increment before this read; a load, not an
    // atomic (one per thread of the grid would serialise at the word's slice)
    if (__ldcg(unstable) == 0) break;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) a.ctl->passes = pass + 1;
  // the last pass wrote its exits into the other snapshot; nothing reads them

  bt_stamp(a.ctl, 7);
  // ---- phase 7: segmented scan of the warp aggregates (CTA 0)
  if (blockIdx.x == 0) {
    CJAgg5* sm = reinterpret_cast<CJAgg5*>(smem);  // BT_THREADS entries (within BT_DECODE_SMEM)
    const int nw = a.nwarps;
    int per = (nw + blockDim.x - 1) / blockDim.x;
    int lo = threadIdx.x * per, hi = min(nw, lo + per);
    CJAgg5 acc = {0, 0, 0, 0, 0};
    for (int w = lo; w < hi; w++) {
      CJWarpAgg g = bt_load_agg(&a.wagg[w]);
      acc = cj_op(acc, CJAgg5{g.has_head, g.nblocks, g.dc[0], g.dc[1], g.dc[2]});
    }
    sm[threadIdx.x] = acc;
    __syncthreads();
    for (int dd = 1; dd < (int)blockDim.x; dd <<= 1) {
      CJAgg5 x = sm[threadIdx.x];
      CJAgg5 y = threadIdx.x >= (unsigned)dd ? sm[threadIdx.x - dd] : CJAgg5{0, 0, 0, 0, 0};
      __syncthreads();
      if (threadIdx.x >= (unsigned)dd) sm[threadIdx.x] = cj_op(y, x);
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
      a.carry[w] = o;
      CJWarpAgg g = bt_load_agg(&a.wagg[w]);
      run = cj_op(run, CJAgg5{g.has_head, g.nblocks, g.dc[0], g.dc[1], g.dc[2]});
    }
  }
  if (!bt_grid_sync(a.ctl, gen, a.wait_limit, &s_ok)) return;

  bt_stamp(a.ctl, 8);
  // ---- phase 8: coefficient write-out in units of a quarter subsequence.
  // Unit (lane, q) starts at checkpoint q - 1 of the lane's settled decode --
  // its exact state: position, MCU phase, blocks and DC sums so far -- and
  // stops at checkpoint q's block boundary (the last unit at the lane's end),
  // so write items are a quarter as long as sync items whatever the
  // subsequence size.  An item is 8 lanes x 4 units of one 32-lane warp w,
  // whose block / DC prefix it recomputes; the warp writes its 32 units'
  // blocks cooperatively (cj_write_units_warp).  (In a corrupt stream a unit may
  // write past an error an earlier unit stopped at; only blocks after that
  // error, so the first error of the image is the same.)
  {
    constexpr int UNITS = CJ_CKPTS + 1, LANES = 32 / UNITS;
    const int nitems = a.nwarps * UNITS;
    // the warp's block buffers, zero between blocks (the step tables are read
    // from global memory here: the buffers take the staging space)
    int16_t* wbuf = reinterpret_cast<int16_t*>(smem) + (threadIdx.x >> 5) * 32 * 64;
    for (int k = lane; k < 32 * 64 * 2 / 16; k += 32) reinterpret_cast<uint4*>(wbuf)[k] = make_uint4(0, 0, 0, 0);
    __syncwarp();
    for (int t = bt_next_item(&a.ctl->next_write); t < nitems; t = bt_next_item(&a.ctl->next_write)) {
      const int w = t / UNITS, part = t % UNITS;
      const int i = bt_image_of_warp(a, w);
      const CJImageDesc& d = a.desc[i];
      CJStatus* st = &a.st[i];
      const int nsub = __ldcg(&st->nsub), nseg = __ldcg(&st->nseg);
      const int j0 = w * 32 - d.sub0;
      if (j0 >= nsub) continue;
      const CJScanParams& sp = a.prm[i];
      const CJSteps& T = sp.steps;
      const uint32_t* words = reinterpret_cast<const uint32_t*>(a.data + d.data_off);
      // block / DC prefix of the 32 lanes of warp w (thread = lane `lane`)
      const CJLane lw = cj_lane(a.segs + d.seg0, nseg, nsub, j0 + lane, d.sub_bits);
      CJSubRec rw;
      if (lw.active) rw = bt_load_rec(&a.recs[d.sub0 + j0 + lane]);
      else {
        rw.start = rw.exit = 0;
        rw.nblocks = rw.dc[0] = rw.dc[1] = rw.dc[2] = 0;
      }
      int64_t bw;
      int e0, e1, e2;
      cj_warp_prefix(rw, lw, __ldcg(&a.carry[w].nblocks), __ldcg(&a.carry[w].dc[0]),
                     __ldcg(&a.carry[w].dc[1]), __ldcg(&a.carry[w].dc[2]), &bw, &e0, &e1, &e2);
      const int64_t firstw = bw + (lw.active ? a.segs[d.seg0 + lw.seg].first_block : 0);
      // this thread's unit: lane ul of warp w, quarter q
      const int ul = part * LANES + lane / UNITS, q = lane % UNITS;
      const int64_t lane_first = __shfl_sync(CJ_FULL, firstw, ul);
      int dc0 = __shfl_sync(CJ_FULL, e0, ul), dc1 = __shfl_sync(CJ_FULL, e1, ul), dc2 = __shfl_sync(CJ_FULL, e2, ul);
      CJSubRec r;
      r.start = __shfl_sync(CJ_FULL, rw.start, ul);
      r.nblocks = __shfl_sync(CJ_FULL, rw.nblocks, ul);
      const CJLane ln = cj_lane(a.segs + d.seg0, nseg, nsub, j0 + ul, d.sub_bits);
      const CJSegment seg = a.segs[d.seg0 + (ln.active ? ln.seg : 0)];
      const CJCkpt* ck = cj_lane_ckpts(a.ckpt, d.sub0 + j0 + ul);
      uint64_t start = r.start, stop = ~0ull;
      int64_t first = lane_first, end = 0;
      if (ln.active) {
        if (q > 0) {
          const uint32_t pp = __ldcg(&ck[q - 1].pp);
          start = cj_state(ln.begin + (pp & 0xFFFFFFu), pp >> 24);
          first += __ldcg(&ck[q - 1].nb);
          dc0 += __ldcg(&ck[q - 1].d0);
          dc1 += __ldcg(&ck[q - 1].d1);
          dc2 += __ldcg(&ck[q - 1].d2);
        }
        if (q < UNITS - 1) {
          stop = ln.begin + (__ldcg(&ck[q].pp) & 0xFFFFFFu);
          const int64_t bend = seg.first_block + seg.nblocks;
          end = lane_first + __ldcg(&ck[q].nb);
          if (end > bend) end = bend;
        } else {
          end = cj_lane_write_end(ln, seg, r, lane_first);
        }
      }
      cj_write_units_warp(sp, T, words, ln, seg, start, first, dc0, dc1, dc2, a.coef + d.coef0 * 64, st, s_zz, stop,
                          end, ln.active, wbuf);
    }
  }
}

typedef void (*bt_decode_fn)(CJBatchArgs);
#define BT_DECODE_CTAS_DEFAULT 4
static bt_decode_fn bt_decode_kernel(int ctas_per_sm, bool hyp = false) {
  switch (ctas_per_sm) {
    case 3: return hyp ? k_decode_batch<3, true> : k_decode_batch<3>;
    case 5: return hyp ? k_decode_batch<5, true> : k_decode_batch<5>;
    default: return hyp ? k_decode_batch<4, true> : k_decode_batch<4>;
  }
}

// The decode kernels' dynamic shared memory is above the 48 KB a launch gets
// without opting in.
static cudaError_t bt_decode_attrs() {
  const int bytes = (int)BT_DECODE_SMEM;
  cudaError_t e = cudaSuccess;
  for (int c = 3; c <= 5 && e == cudaSuccess; c++)
    for (int h = 0; h < 2 && e == cudaSuccess; h++)
      e = cudaFuncSetAttribute((const void*)bt_decode_kernel(c, h != 0), cudaFuncAttributeMaxDynamicSharedMemorySize,
                               bytes);
  return e;
}

template <int MODE, int OUT>
__device__ __forceinline__ void bt_pixel_tiles(const CJBatchArgs& a, int t0, int t1, uint8_t* smem,
                                               uint64_t* bar2, CJPixSmemParams* Pp);
template <int OUT>
__device__ __forceinline__ void bt_pixel_tiles_tc(const CJBatchArgs& a, int t0, int t1, uint8_t* smem,
                                                  uint64_t* bar2, CJPixSmemParams* Pp, CJTcState* tc);

// Phase 9 runs as its own kernel, launched right after k_decode_batch on the
// same stream: the pixel work needs no grid barrier, and on its own it runs
// at the occupancy of its 32-40 registers per thread instead of the entropy
// phases' 64.  Pixel tiles, double-buffered: the TMA copy of a CTA's next
// tile is in flight while it computes the current one.  MODE is the iDCT
// arithmetic (integer: the reference's, bit-exact; tensor cores: FP16 hi/lo
// with FP32 accumulation), OUT the output format.  The tensor-core form
// keeps a 64-column accumulator in tensor memory per CTA and the hi/lo
// Kronecker basis, built by the CTA, in shared memory.
template <int MODE, int OUT>
__global__ void __launch_bounds__(MODE == CJ_PIX_IDCT_TC ? CJ_TC_THREADS : CJ_PIX_THREADS,
                                  MODE == CJ_PIX_IDCT_TC ? CJ_TC_MINB : 6) k_pixel_batch(CJBatchArgs a) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ uint64_t bar2[2];
  __shared__ CJPixSmemParams P;
  // a decode kernel whose grid barrier timed out left no settled
  // coefficients: nothing to transform
  if (__ldcg(&a.ctl->timeout)) return;
  __shared__ uint64_t s_mma_bar;
  __shared__ uint32_t s_tmem;
  __shared__ float s_b32[64];
  if (threadIdx.x == 0) {
    cj_tile_fail = 0;
    cj_mbar_init(&bar2[0], 1);
    cj_mbar_init(&bar2[1], 1);
    if (MODE == CJ_PIX_IDCT_TC) cj_mbar_init(&s_mma_bar, 1);
  }
  CJTcState tc;
  if (MODE == CJ_PIX_IDCT_TC) {
    // the swizzled A tile starts on the first 1024-byte boundary of its
    // region (the dynamic shared memory itself need not be so aligned)
    uint8_t* a_region = smem + CJ_TC_A_OFF;
    tc.a_tile = a_region + ((1024u - (cj_smem_addr(a_region) & 1023u)) & 1023u);
    // the A tile starts zeroed (rows past a tile's blocks are never written)
    for (int k = threadIdx.x; k < 16384 / 16; k += blockDim.x)
      reinterpret_cast<uint4*>(tc.a_tile)[k] = make_uint4(0, 0, 0, 0);
    // the hi/lo Kronecker basis, built once per device, into the B operand
    const uint4* gb = reinterpret_cast<const uint4*>(a.tc_basis);
    for (int k = threadIdx.x; k < 16384 / 16; k += blockDim.x)
      reinterpret_cast<uint4*>(smem + CJ_TC_B_OFF)[k] = __ldg(gb + k);
    // the 8x8 basis B[u][x] in FP32 for the range fallback
    if (threadIdx.x < 64) {
      const int u = threadIdx.x >> 3, x = threadIdx.x & 7;
      s_b32[threadIdx.x] = (float)((u ? 0.5 : 0.5 * sqrt(0.5)) * cospi((double)((2 * x + 1) * u) / 16.0));
    }
    if ((threadIdx.x >> 5) == 0) tc_alloc(&s_tmem, 64);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  }
  bt_stamp(a.ctl, 9);
  __syncthreads();
  if (MODE == CJ_PIX_IDCT_TC) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    tc.tmem = s_tmem;
    tc.bar = &s_mma_bar;
    tc.parity = 0;
    tc.basis = s_b32;
  }
  // Each CTA takes a contiguous run of tiles, so consecutive tiles mostly
  // belong to one image: the image index only ever moves forward and the
  // tile geometry is rebuilt only when it changes.
  const int per = (a.nptiles + gridDim.x - 1) / gridDim.x;
  const int t0 = blockIdx.x * per, t1 = min(t0 + per, a.nptiles);
  if (t0 < t1) {
    if constexpr (MODE == CJ_PIX_IDCT_TC) bt_pixel_tiles_tc<OUT>(a, t0, t1, smem, bar2, &P, &tc);
    else bt_pixel_tiles<MODE, OUT>(a, t0, t1, smem, bar2, &P);
  }
  __syncthreads();
  if (MODE == CJ_PIX_IDCT_TC && (threadIdx.x >> 5) == 0) tc_dealloc(s_tmem, 64);
  if (threadIdx.x == 0 && atomicAdd(&a.ctl->pix_done, 1) == gridDim.x - 1) bt_stamp_any(a.ctl, BT_NPHASE);
}

// Geometry of image i's pixel tiles.
__device__ __forceinline__ CJPixGeom bt_pix_geom(const CJBatchArgs& a, int i, bool tc) {
  const CJScanParams& prm = a.prm[i];
  CJPixGeom gg;
  gg.nch = prm.nch;
  gg.bpm = prm.bpm;
  gg.mcux = prm.mcux;
  gg.mcuy = prm.mcuy;
  gg.width = prm.width;
  gg.height = prm.height;
  gg.hmax = prm.hmax;
  gg.vmax = prm.vmax;
  gg.xs = prm.xshift;
  gg.ys = prm.yshift;
  gg.T = a.desc[i].T;
  gg.cw = prm.nch == 3 ? (prm.width * prm.comp_sx[1] + prm.hmax - 1) / prm.hmax : 0;
  gg.ch = prm.nch == 3 ? (prm.height * prm.comp_sy[1] + prm.vmax - 1) / prm.vmax : 0;
  cj_pix_layout(&gg, prm.comp_sx[1], prm.comp_sy[1], 2, tc);
  return gg;
}

// Tiles [t0, t1) of one pixel-kernel CTA.
template <int MODE, int OUT>
__device__ __forceinline__ void bt_pixel_tiles(const CJBatchArgs& a, int t0, int t1, uint8_t* smem,
                                               uint64_t* bar2, CJPixSmemParams* Pp) {
  constexpr bool TC = false;
  CJPixSmemParams& P = *Pp;
  auto advance = [&](int tt, int i) {
    while (tt >= a.desc[i].ptile0 + a.desc[i].nptiles) i++;
    return i;
  };
  // thread 0 issues each tile's copy one tile ahead of the compute; it keeps
  // the geometry of the image it prefetches from
  __shared__ CJPixGeom s_pg;  // thread 0's prefetch geometry (kept out of registers)
  __shared__ int s_pimg;
  if (threadIdx.x == 0) s_pimg = -1;
  CJPixGeom& pg = s_pg;
  auto issue = [&](int tt, int i, int which) {
    if (i != s_pimg) {
      pg = bt_pix_geom(a, i, TC);
      s_pimg = i;
    }
    const int local = tt - a.desc[i].ptile0, gx = (pg.mcux + pg.T - 1) / pg.T;
    cj_pixel_issue(a.coef + a.desc[i].coef0 * 64, pg, local / gx, (local % gx) * pg.T,
                   reinterpret_cast<int16_t*>(smem + which * pg.sc1_off), &bar2[which]);
  };
  int img = bt_find(a.n, t0, [&](int k) { return a.desc[k].ptile0; });
  if (threadIdx.x == 0) issue(t0, img, 0);
  int nimg = img;  // image of the next tile to prefetch (thread 0)
  CJPixGeom g = bt_pix_geom(a, img, TC);
  int gimg = img;
  cj_pixel_setup(a.prm[img], g, &P);
  __syncthreads();  // the setup before any use (a tile has no barrier before its iDCT)
  // tile position in its image's grid, advanced tile by tile
  int gx = (g.mcux + g.T - 1) / g.T;
  int trow = (t0 - a.desc[img].ptile0) / gx, tcol = (t0 - a.desc[img].ptile0) % gx;
  int buf = 0;
  uint32_t par = 0;  // bit b: the phase parity buffer b's barrier waits for next
  for (int t = t0; t < t1; t++) {
    if (t + 1 < t1 && threadIdx.x == 0) {
      nimg = advance(t + 1, nimg);
      issue(t + 1, nimg, buf ^ 1);
    }
    img = advance(t, img);
    if (img != gimg) {  // CTA-uniform; the previous tile ended with a barrier
      g = bt_pix_geom(a, img, TC);
      gimg = img;
      cj_pixel_setup(a.prm[img], g, &P);
      __syncthreads();
      gx = (g.mcux + g.T - 1) / g.T;
      trow = tcol = 0;  // a new image starts at its first tile
    }
    const CJImageDesc& d = a.desc[img];
    const int16_t* sc = reinterpret_cast<const int16_t*>(smem + buf * g.sc1_off);
    if (!cj_pixel_tile<MODE, OUT>(a.out + d.out_off, &a.st[img], g, trow, tcol * g.T, sc, smem, &bar2[buf],
                                  (par >> buf) & 1u, &P)) {
      if (t + 1 < t1) cj_mbar_wait(&bar2[buf ^ 1], (par >> (buf ^ 1)) & 1u);  // the prefetch in flight
      break;
    }
    if (++tcol == gx) {
      tcol = 0;
      trow++;
    }
    par ^= 1u << buf;
    buf ^= 1;
  }
}

// Tiles [t0, t1) of one pixel-kernel CTA in the tensor-core form.  A tile
// holds up to CJ_TC_MAXB blocks (cj_pix_tile_mcus_tc) and costs two
// barrier-separated phases:
//   1. thread 0 issues the tile's 8 MMAs (its A tile was built in the
//      previous phase) and the bulk copy of the coefficients of the tile
//      CJ_TC_NBUF ahead (into the buffer this tile's A was built from);
//      every thread waits for the MMAs and runs the epilogue into the plane
//      tiles -- barrier -- (rare: the FP32 redo of range-flagged blocks);
//   2. the output of the tile from the plane tiles, then the A tile of the
//      next tile from its copied coefficients -- barrier.
// The output and the next A build share a phase, so no warp idles through
// a phase of its own, and the MMAs' latency is covered by the other CTAs of
// the SM.  An image change between two tiles adds two barriers (the new
// image's tables and block destinations replace the old ones after the
// output).
template <int OUT>
__device__ __forceinline__ void bt_pixel_tiles_tc(const CJBatchArgs& a, int t0, int t1, uint8_t* smem,
                                                  uint64_t* bar2, CJPixSmemParams* Pp, CJTcState* tc) {
  CJPixSmemParams& P = *Pp;
  uint8_t* big = smem + CJ_TC_BIG_OFF;
  auto advance = [&](int tt, int i) {
    while (tt >= a.desc[i].ptile0 + a.desc[i].nptiles) i++;
    return i;
  };
  // tile u's coefficient buffer, and the wait for its copy (each buffer's
  // barrier completes one phase per tile it receives)
  auto sc_of = [&](int u) {
    return reinterpret_cast<int16_t*>(smem + CJ_TC_SC_OFF + ((u - t0) % CJ_TC_NBUF) * CJ_TC_COEF_BYTES);
  };
  auto wait_copy = [&](int u) {
    return cj_mbar_wait(&bar2[(u - t0) % CJ_TC_NBUF], (uint32_t)(((u - t0) / CJ_TC_NBUF) & 1));
  };
  // thread 0 issues the copies in tile order and keeps the geometry of the
  // image it issues from
  __shared__ CJPixGeom s_pg;
  __shared__ int s_pimg;
  int nimg = 0;
  auto issue = [&](int u) {
    nimg = advance(u, nimg);
    if (nimg != s_pimg) {
      s_pg = bt_pix_geom(a, nimg, true);
      s_pimg = nimg;
    }
    const int local = u - a.desc[nimg].ptile0, gx = (s_pg.mcux + s_pg.T - 1) / s_pg.T;
    cj_pixel_issue(a.coef + a.desc[nimg].coef0 * 64, s_pg, local / gx, (local % gx) * s_pg.T, sc_of(u),
                   &bar2[(u - t0) % CJ_TC_NBUF]);
  };
  int img = bt_find(a.n, t0, [&](int k) { return a.desc[k].ptile0; });
  int issued_to = min(t0 + CJ_TC_NBUF, t1);  // copies of tiles [.., issued_to) are issued
  int waited_to = t0;                         // and those of [.., waited_to) waited for
  if (threadIdx.x == 0) {
    s_pimg = -1;
    nimg = img;
    for (int u = t0; u < issued_to; u++) issue(u);
  }
  // on leaving early: a bounded wait for every copy still in flight
  auto leave = [&]() {
    for (int u = waited_to; u < issued_to; u++) wait_copy(u);
  };
  // the geometry of the current image lives in shared memory (written by
  // thread 0), not in every thread's registers
  __shared__ CJPixGeom s_g;
  const CJPixGeom& g = s_g;
  if (threadIdx.x == 0) s_g = bt_pix_geom(a, img, true);
  __syncthreads();
  cj_pixel_setup(a.prm[img], g, &P);
  int gx = (g.mcux + g.T - 1) / g.T;
  int trow = (t0 - a.desc[img].ptile0) / gx, tcol = (t0 - a.desc[img].ptile0) % gx;
  int nblk = min(g.T, g.mcux - tcol * g.T) * g.bpm;
  __syncthreads();  // the setup before the first A build
  if (!wait_copy(t0)) cj_tile_fail = 1;
  waited_to = t0 + 1;
  cj_tc_build_a(nblk, sc_of(t0), tc->a_tile, big, P);
  __syncthreads();
  if (cj_pixel_failed(&a.st[img])) {
    leave();
    return;
  }
  for (int t = t0; t < t1; t++) {
    // ---- phase 1: the tile's MMAs, the copy CJ_TC_NBUF tiles ahead, the epilogue
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (threadIdx.x == 0) {
      tc_idct_mmas_asw(tc->tmem, cj_smem_addr(tc->a_tile), cj_smem_addr(smem + CJ_TC_B_OFF), cj_smem_addr(tc->bar));
      if (t + CJ_TC_NBUF < t1) issue(t + CJ_TC_NBUF);
    }
    if (t + CJ_TC_NBUF < t1) issued_to = t + CJ_TC_NBUF + 1;
    const bool ok = cj_mbar_wait(tc->bar, tc->parity);
    tc->parity ^= 1u;
    if (!ok) cj_tile_fail = 1;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const bool flagged = cj_tc_epilogue(g, nblk, smem, big, P, *tc, ok);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    const CJImageDesc& d = a.desc[img];
    if (__syncthreads_or(flagged || !ok)) {  // rare: a failed wait, or an FP32 redo
      if (cj_pixel_failed(&a.st[img])) {
        cj_mbar_wait(tc->bar, tc->parity ^ 1u);  // a bounded second chance for MMAs still in flight
        leave();
        return;
      }
      cj_tc_fallback(g, nblk, a.coef + (d.coef0 + ((int64_t)trow * g.mcux + (int64_t)tcol * g.T) * g.bpm) * 64,
                     smem, big, P, *tc);
    }
    // ---- phase 2: the tile's output, then the next tile's A
    const int nm = min(g.T, g.mcux - tcol * g.T);
    if (OUT == CJ_OUT_RGB) cj_pixel_emit_rgb(a.out + d.out_off, g, trow, tcol * g.T, nm, smem);
    else cj_pixel_emit_planes<OUT>(a.out + d.out_off, g, trow, tcol * g.T, nm, smem);
    if (t + 1 < t1) {
      const int img1 = advance(t + 1, img);
      if (img1 != img) {  // CTA-uniform
        __syncthreads();  // the plane tiles, P and the geometry of the old image are read no more
        img = img1;
        if (threadIdx.x == 0) s_g = bt_pix_geom(a, img, true);
        __syncthreads();
        cj_pixel_setup(a.prm[img], g, &P);
        gx = (g.mcux + g.T - 1) / g.T;
        trow = tcol = 0;  // a new image starts at its first tile
        __syncthreads();
      } else if (++tcol == gx) {
        tcol = 0;
        trow++;
      }
      nblk = min(g.T, g.mcux - tcol * g.T) * g.bpm;
      if (!wait_copy(t + 1)) cj_tile_fail = 1;
      waited_to = t + 2;
      cj_tc_build_a(nblk, sc_of(t + 1), tc->a_tile, big, P);
    }
    __syncthreads();  // the output is written, the next A tile is complete
    if (cj_pixel_failed(&a.st[img])) {
      leave();
      return;
    }
  }
}

typedef void (*bt_pixel_fn)(CJBatchArgs);
static bt_pixel_fn bt_pixel_kernel(int mode, int out) {
  if (mode == CJ_PIX_IDCT_TC) {
    if (out == CJ_OUT_PLANAR) return k_pixel_batch<CJ_PIX_IDCT_TC, CJ_OUT_PLANAR>;
    if (out == CJ_OUT_NV12) return k_pixel_batch<CJ_PIX_IDCT_TC, CJ_OUT_NV12>;
    return k_pixel_batch<CJ_PIX_IDCT_TC, CJ_OUT_RGB>;
  }
  if (out == CJ_OUT_PLANAR) return k_pixel_batch<CJ_PIX_IDCT_INT, CJ_OUT_PLANAR>;
  if (out == CJ_OUT_NV12) return k_pixel_batch<CJ_PIX_IDCT_INT, CJ_OUT_NV12>;
  return k_pixel_batch<CJ_PIX_IDCT_INT, CJ_OUT_RGB>;
}

// Every pixel-kernel variant may use up to 96 KiB of dynamic shared memory.
static cudaError_t bt_pixel_attrs() {
  const int modes[] = {CJ_PIX_IDCT_INT, CJ_PIX_IDCT_TC};
  const int outs[] = {CJ_OUT_RGB, CJ_OUT_PLANAR, CJ_OUT_NV12};
  for (int m : modes)
    for (int o : outs) {
      cudaError_t e = cudaFuncSetAttribute((const void*)bt_pixel_kernel(m, o),
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
      if (e != cudaSuccess) return e;
    }
  return cudaSuccess;
}

// Fancy mode, after the pixel kernel left each image's planar samples at
// out + out_off: one thread per output pixel upsamples Cb and Cr with the
// triangle filter (cj_fancy_at) and applies the reference's colour
// transform (CPUonly/src/pixelTransformCPU.c:147-158) into rgb + rgb_off;
// grey images are copied.
__global__ void __launch_bounds__(256) k_fancy_rgb(CJBatchArgs a) {
  if (__ldcg(&a.ctl->timeout)) return;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < a.npix;
       p += (int64_t)gridDim.x * blockDim.x) {
    int lo = 0, hi = a.n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (a.desc[mid].pix0 <= p) lo = mid;
      else hi = mid - 1;
    }
    const CJImageDesc& d = a.desc[lo];
    const CJScanParams& prm = a.prm[lo];
    const int W = prm.width, H = prm.height;
    const int64_t k = p - d.pix0;
    const uint8_t* pl = a.out + d.out_off;
    if (prm.nch != 3) {
      a.rgb[d.rgb_off + k] = pl[k];
      continue;
    }
    const int y = (int)(k / W), x = (int)(k - (int64_t)y * W);
    const int cw = (W * prm.comp_sx[1] + prm.hmax - 1) / prm.hmax;
    const int ch = (H * prm.comp_sy[1] + prm.vmax - 1) / prm.vmax;
    const uint8_t* cbp = pl + (int64_t)W * H;
    const int cb = cj_fancy_at(cbp, cw, ch, prm.xshift, prm.yshift, x, y);
    const int cr = cj_fancy_at(cbp + (int64_t)cw * ch, cw, ch, prm.xshift, prm.yshift, x, y);
    const int yy = pl[k] << 8;
    uint8_t* o = a.rgb + d.rgb_off + 3 * k;
    o[0] = (uint8_t)cj_rgb_pack(yy, cb - 128, cr - 128, 0);
    o[1] = (uint8_t)cj_rgb_pack(yy, cb - 128, cr - 128, 1);
    o[2] = (uint8_t)cj_rgb_pack(yy, cb - 128, cr - 128, 2);
  }
}

// Output bytes of one image in a format (fancy mode: its planar samples;
// the RGB output is counted apart).
static int64_t bt_out_bytes(const CJImageHeader& h, int out) {
  const int64_t y = (int64_t)h.width * h.height;
  if (h.nch != 3) return y;
  if (out == CJ_OUT_RGB) return 3 * y;
  const int64_t cw = ((int64_t)h.width * h.comp_sx[1] + h.hmax - 1) / h.hmax;
  const int64_t ch = ((int64_t)h.height * h.comp_sy[1] + h.vmax - 1) / h.vmax;
  return y + 2 * cw * ch;
}

// ---------------------------------------------------------------- device header parse

// What the host plan needs of a parsed file: everything of its header but
// the tables (which stay on the device), its scan range and its error code.
struct alignas(16) CJParseSummary {
  int64_t scan_off, scan_len, total_blocks;
  int32_t err, mcux, mcuy, width, height, hmax, vmax, restart_interval, nseg_expected;
  uint8_t nch, huff_mask, xshift, yshift;
  uint8_t comp_dc[3], comp_ac[3], comp_q[3], comp_sx[3], comp_sy[3], pad[1];
};
static_assert(sizeof(CJParseSummary) == 80, "summary size");
static_assert(sizeof(CJImageHeader) % 16 == 0, "headers are copied in 16-byte words");

#define BT_PARSE_THREADS 128

// The batch's marker parse on the GPU: thread i walks file i's marker
// segments (cj_parse_header) in the blob already copied to the device and
// leaves its header in `hdr` (device memory).  The CTA's summaries are
// written to `sum`, pinned host memory mapped into the device's address
// space, as one contiguous run of 16-byte stores: they reach the host
// without a device-to-host copy (which would queue behind any other copy in
// that direction).
__global__ void __launch_bounds__(BT_PARSE_THREADS) k_parse_headers(const uint8_t* __restrict__ blob,
                                                                   const int64_t* __restrict__ offsets,
                                                                   const int64_t* __restrict__ sizes, int n,
                                                                   CJImageHeader* hdr, CJParseSummary* sum) {
  __shared__ CJParseSummary s_sum[BT_PARSE_THREADS];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    int64_t so = 0, sl = 0;
    CJImageHeader* h = &hdr[i];
    const int e = cj_parse_header(blob + offsets[i], sizes[i], h, &so, &sl);
    CJParseSummary& q = s_sum[threadIdx.x];
    q.scan_off = so;
    q.scan_len = sl;
    q.total_blocks = h->total_blocks;
    q.err = e;
    q.mcux = h->mcux;
    q.mcuy = h->mcuy;
    q.width = h->width;
    q.height = h->height;
    q.hmax = h->hmax;
    q.vmax = h->vmax;
    q.restart_interval = h->restart_interval;
    q.nseg_expected = h->nseg_expected;
    q.nch = h->nch;
    q.huff_mask = h->huff_mask;
    q.xshift = h->xshift;
    q.yshift = h->yshift;
    for (int c = 0; c < 3; c++) {
      q.comp_dc[c] = h->comp_dc[c];
      q.comp_ac[c] = h->comp_ac[c];
      q.comp_q[c] = h->comp_q[c];
      q.comp_sx[c] = h->comp_sx[c];
      q.comp_sy[c] = h->comp_sy[c];
    }
    q.pad[0] = 0;
  }
  __syncthreads();
  const int first = blockIdx.x * blockDim.x, cnt = min((int)blockDim.x, n - first);
  const uint4* src = reinterpret_cast<const uint4*>(s_sum);
  uint4* dst = reinterpret_cast<uint4*>(sum + first);
  const int words = cnt * (int)(sizeof(CJParseSummary) / 16);
  for (int k = threadIdx.x; k < words; k += blockDim.x) dst[k] = src[k];
}

// The headers of the planned images, compacted: hdr[d] = parsed[file_of[d]]
// (one CTA per image, 16-byte copies).
__global__ void __launch_bounds__(128) k_gather_headers(const CJImageHeader* __restrict__ parsed,
                                                        const int32_t* __restrict__ file_of,
                                                        CJImageHeader* hdr) {
  const uint4* src = reinterpret_cast<const uint4*>(parsed + file_of[blockIdx.x]);
  uint4* dst = reinterpret_cast<uint4*>(hdr + blockIdx.x);
  for (int k = threadIdx.x; k < (int)(sizeof(CJImageHeader) / 16); k += blockDim.x) dst[k] = src[k];
}

// ---------------------------------------------------------------- host side

struct CJBatch {
  bool ready = false;
  int device = 0, sm_count = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // tuning (cjBatchSetTuning / cjBatchAutotune)
  int sub_bits = BT_SUB_BITS_DEFAULT;
  int sub_bits_class[CJ_SAMPLING_CLASSES] = {0, 0, 0, 0, 0};  // 0: sub_bits
  int decode_ctas = BT_DECODE_CTAS_DEFAULT;  // decode-kernel CTAs per SM (3, 4 or 5)
  int tile_cap = 0;                          // max MCUs per pixel tile (0 = layout maximum)
  unsigned wait_limit = 0;                   // grid-barrier polls before a timeout (0 = default)
  int idct = CJ_PIX_IDCT_INT;                // pixel-stage iDCT arithmetic
  int out_format = CJ_OUT_RGB;               // output format
  JPGReader* parser = nullptr;  // host marker parse, one image at a time
  bool parse_on_device = true;   // marker parse on the GPU (k_parse_headers) or on the host
  // device buffers (grow-only)
  CJDevBuf hrecs, hckpt, hmap;  // MCU-phase hypotheses and probes of a latency-bound batch
  int nhyp = 1;
  bool hyp_enabled = true;  // cjBatchSetHypotheses
  CJDevBuf hdr, desc, prm, st, blob, data, tile_keep, tile_mark, mpos, mcode, segs, recs, ckpt, snap,
      wagg, carry, coef, out, ctl, fancy;  // fancy: planar samples of the fancy mode
  CJDevBuf p_size, p_hdr, p_map;           // device parse: file offsets + sizes, headers, image -> file
  // pinned host staging
  CJHostBuf h_hdr, h_desc, h_out, h_st, h_ctl, h_psize, h_pmap;
  // device parse summaries: pinned host memory mapped into the device
  CJParseSummary* h_psum = nullptr;
  CJParseSummary* d_psum = nullptr;
  size_t psum_cap = 0;
  // plan of the staged batch
  int n_in = 0, n_dev = 0;
  std::vector<int> dev_of;     // device slot of each submitted image, -1 if rejected
  std::vector<int32_t> file_of;  // device parse: submitted image of each device slot
  std::vector<int> host_err;   // host-side (parse) error of each submitted image
  std::vector<int> dims;       // width, height, channels, chroma width, chroma height per device slot
  std::vector<int64_t> outoff; // output offset per device slot
  int ntiles = 0, nwarps = 0, nptiles = 0;
  int64_t blob_bytes = 0, out_total = 0, blocks = 0, scan_bytes = 0, planar_total = 0, npix = 0;
  size_t smem = 0, smem_pix = 0;
  int grid = 0, grid_pix = 0;
  long long launches = 0;
  // the run as a CUDA graph (rebuilt after each stage)
  bool use_graph = true, graph_stale = true;
  cudaGraphExec_t gexec = nullptr;
  long long graph_launches = 0, graph_failures = 0;
};

// Grow-only device buffer in the batch's stream order: the old buffer is
// freed and the new one allocated on b->stream (stream-ordered allocator),
// so growing one batch's buffers never waits for work on other streams, as
// cudaFree would.  50% headroom keeps regrowth rare.
static int bt_ensure(CJBatch* b, CJDevBuf& d, size_t bytes) {
  if (d.p && bytes <= d.cap) return 0;
  if (d.p) cudaFreeAsync(d.p, b->stream);
  d.p = nullptr;
  d.cap = 0;
  size_t cap = bytes + bytes / 2 + 256;
  cudaError_t e = cudaMallocAsync(&d.p, cap, b->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    fprintf(stderr, "libcudajpeg: cudaMallocAsync(%zu) failed: %s\n", cap, cudaGetErrorString(e));
    d.p = nullptr;
    return CUDA_MEM_ERROR;
  }
  d.cap = cap;
  return 0;
}

// The pixel kernel's output format (fancy mode: planar samples for k_fancy_rgb).
static int bt_pix_format(const CJBatch* b) {
  return b->out_format == CJ_OUT_RGB_FANCY ? CJ_OUT_PLANAR : b->out_format;
}

static int bt_init(CJBatch* b) {
  if (b->ready) return 0;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    fprintf(stderr, "libcudajpeg: no CUDA device available; the decoder has no CPU path\n");
    return CUDA_MEM_ERROR;
  }
  CJ_CUDA_TRY(cudaGetDevice(&b->device), CUDA_MEM_ERROR);
  CJ_CUDA_TRY(cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, b->device),
              CUDA_MEM_ERROR);
  int coop = 0;
  CJ_CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, b->device), CUDA_MEM_ERROR);
  if (!coop) return UNSUPPORTED_ERROR;
  CJ_CUDA_TRY(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), CUDA_MEM_ERROR);
  CJ_CUDA_TRY(cudaEventCreate(&b->ev0), CUDA_MEM_ERROR);
  CJ_CUDA_TRY(cudaEventCreate(&b->ev1), CUDA_MEM_ERROR);
  CJ_CUDA_TRY(bt_pixel_attrs(), CUDA_MEM_ERROR);
  CJ_CUDA_TRY(bt_decode_attrs(), CUDA_MEM_ERROR);
  b->parser = newJPGReader();
  if (!b->parser) return OOM_ERROR;
  b->ready = true;
  return 0;
}

// The device header of a reader parsed up to its scan (tables as parsed,
// geometry); UNSUPPORTED_ERROR for a geometry the pixel tiles do not cover
// (cj_pix_check).
static int bt_fill_header(const JPGReader* r, CJImageHeader* h) {
  memset(h, 0, sizeof(*h));
  for (int s = 0; s < 4; s++) {
    memcpy(h->counts[s], r->dev->huff[s].counts, 16);
    memcpy(h->symbols[s], r->dev->huff[s].symbols, 256);
  }
  h->huff_mask = (uint8_t)r->huff_defined;
  memcpy(h->dq, r->dev->dq16, sizeof(h->dq));
  h->nch = r->num_channels;
  for (int c = 0; c < r->num_channels; c++) {
    h->comp_dc[c] = (uint8_t)r->channels[c].dc_id;
    h->comp_ac[c] = (uint8_t)r->channels[c].ac_id;
    h->comp_q[c] = (uint8_t)r->channels[c].dq_id;
    h->comp_sx[c] = (uint8_t)r->channels[c].samples_x;
    h->comp_sy[c] = (uint8_t)r->channels[c].samples_y;
  }
  h->mcux = r->num_blocks_x;
  h->mcuy = r->num_blocks_y;
  h->width = r->width;
  h->height = r->height;
  h->hmax = r->block_size_x >> 3;
  h->vmax = r->block_size_y >> 3;
  int xs = 0, ys = 0;
  if (r->num_channels == 3) {
    while ((r->channels[1].width << xs) < r->width) xs++;
    while ((r->channels[1].height << ys) < r->height) ys++;
  }
  h->xshift = (uint8_t)xs;
  h->yshift = (uint8_t)ys;
  h->restart_interval = r->restart_interval;
  int64_t mcus = (int64_t)h->mcux * h->mcuy;
  h->nseg_expected = r->restart_interval ? (int)((mcus + r->restart_interval - 1) / r->restart_interval) : 1;
  int bpm = 0;
  for (int c = 0; c < h->nch; c++) bpm += h->comp_sx[c] * h->comp_sy[c];
  h->total_blocks = mcus * bpm;
  // the pixel tile layout's geometry condition (cj_pix_check)
  if (h->comp_sx[0] != h->hmax || h->comp_sy[0] != h->vmax) return UNSUPPORTED_ERROR;
  if (h->nch == 3 && ((h->comp_sx[1] << xs) != h->hmax || (h->comp_sy[1] << ys) != h->vmax))
    return UNSUPPORTED_ERROR;
  return 0;
}

// Host parse of one file up to its scan; fills the device header.
static int bt_parse(CJBatch* b, const unsigned char* data, size_t size, CJImageHeader* h,
                    int64_t* scan_off, int64_t* scan_len) {
  JPGReader* r = b->parser;
  r->huff_defined = 0;  // images of a batch are independent
  int e = cj_parse_to_scan(r, data, size);
  if (e) return e;
  e = bt_fill_header(r, h);
  if (e) return e;
  *scan_off = (int64_t)(r->pos - data);
  *scan_len = (int64_t)(r->end - r->pos);
  return 0;
}

// The plan of one image alone at the start of every buffer: destuff tiles,
// markers, segments, subsequences of `sub_bits`, pixel tiles.
static void bt_plan_one(const CJImageHeader& h, int64_t scan_len, int sub_bits, CJImageDesc* d) {
  memset(d, 0, sizeof(*d));
  int bpm = 0;
  for (int c = 0; c < h.nch; c++) bpm += h.comp_sx[c] * h.comp_sy[c];
  d->raw_len = scan_len;
  d->ntiles = (int)std::max<int64_t>(1, (scan_len + BT_TILE_BYTES - 1) / BT_TILE_BYTES);
  d->mark_cap = h.nseg_expected + 1;
  d->seg_cap = h.nseg_expected;
  d->sub_bits = sub_bits;
  d->sub_cap = ((int)((scan_len * 8 + sub_bits - 1) / sub_bits) + h.nseg_expected + 1 + 31) & ~31;
  d->T = cj_pix_tile_mcus(h.hmax, bpm);
  d->nptiles = h.mcuy * ((h.mcux + d->T - 1) / d->T);
}

extern "C" {

CJBatch* cjBatchCreate(void) { return new (std::nothrow) CJBatch(); }

void cjBatchDestroy(CJBatch* b) {
  if (!b) return;
  if (b->ready) {
    cudaStreamSynchronize(b->stream);
    CJDevBuf* bufs[] = {&b->hdr,  &b->desc, &b->prm,   &b->st,   &b->blob,  &b->data,
                        &b->tile_keep, &b->tile_mark, &b->mpos, &b->mcode, &b->segs,
                        &b->recs, &b->ckpt, &b->snap, &b->wagg, &b->carry, &b->coef, &b->out, &b->ctl,
                        &b->fancy, &b->p_size, &b->p_hdr, &b->p_map, &b->hrecs, &b->hckpt, &b->hmap};
    for (CJDevBuf* d : bufs)
      if (d->p) cudaFree(d->p);
    CJHostBuf* hb[] = {&b->h_hdr, &b->h_desc, &b->h_out, &b->h_st, &b->h_ctl, &b->h_psize, &b->h_pmap};
    for (CJHostBuf* h : hb)
      if (h->p) cudaFreeHost(h->p);
    if (b->h_psum) cudaFreeHost(b->h_psum);
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    cudaEventDestroy(b->ev0);
    cudaEventDestroy(b->ev1);
    cudaStreamDestroy(b->stream);
    delJPGReader(b->parser);
  }
  delete b;
}

}  // extern "C"

// Sampling class of an image (CJ_SAMPLING_*).
static int bt_sampling_class(const CJImageHeader& h) {
  if (h.nch == 1) return CJ_SAMPLING_GRAY;
  if (h.comp_sx[1] != 1 || h.comp_sy[1] != 1 || h.comp_sx[2] != 1 || h.comp_sy[2] != 1) return CJ_SAMPLING_OTHER;
  if (h.comp_sx[0] == 2 && h.comp_sy[0] == 2) return CJ_SAMPLING_420;
  if (h.comp_sx[0] == 2 && h.comp_sy[0] == 1) return CJ_SAMPLING_422;
  if (h.comp_sx[0] == 1 && h.comp_sy[0] == 1) return CJ_SAMPLING_444;
  return CJ_SAMPLING_OTHER;
}

static int bt_sub_bits_for(const CJBatch* b, const CJImageHeader& h) {
  const int c = b->sub_bits_class[bt_sampling_class(h)];
  return c ? c : b->sub_bits;
}

static bool bt_sub_bits_ok(int bits) { return bits >= 128 && bits <= 65536 && !(bits & 31); }

extern "C" {

int cjBatchSetSubsequenceBitsFor(CJBatch* b, int sampling_class, int bits) {
  if (!b || sampling_class < 0 || sampling_class >= CJ_SAMPLING_CLASSES) return PROGRAMMER_ERROR;
  if (bits && !bt_sub_bits_ok(bits)) return PROGRAMMER_ERROR;
  b->sub_bits_class[sampling_class] = bits;
  return 0;
}

int cjBatchGetSubsequenceBitsFor(const CJBatch* b, int sampling_class) {
  if (!b || sampling_class < 0 || sampling_class >= CJ_SAMPLING_CLASSES) return PROGRAMMER_ERROR;
  return b->sub_bits_class[sampling_class] ? b->sub_bits_class[sampling_class] : b->sub_bits;
}

int cjBatchSetSubsequenceBits(CJBatch* b, int bits) {
  if (bits == 0) bits = BT_SUB_BITS_DEFAULT;
  if (!b || !bt_sub_bits_ok(bits)) return PROGRAMMER_ERROR;
  b->sub_bits = bits;
  return 0;
}

int cjBatchSetTuning(CJBatch* b, int sub_bits, int decode_ctas_per_sm, int pixel_tile_cap) {
  if (!b) return PROGRAMMER_ERROR;
  if (decode_ctas_per_sm == 0) decode_ctas_per_sm = BT_DECODE_CTAS_DEFAULT;
  if (decode_ctas_per_sm < 3 || decode_ctas_per_sm > 5) return PROGRAMMER_ERROR;
  if (pixel_tile_cap < 0 || (pixel_tile_cap & (pixel_tile_cap - 1))) return PROGRAMMER_ERROR;
  int e = cjBatchSetSubsequenceBits(b, sub_bits);
  if (e) return e;
  b->decode_ctas = decode_ctas_per_sm;
  b->tile_cap = pixel_tile_cap;
  return 0;
}

int cjBatchSetOutput(CJBatch* b, int format, int idct) {
  if (!b) return PROGRAMMER_ERROR;
  if (format != CJ_OUT_RGB && format != CJ_OUT_PLANAR && format != CJ_OUT_NV12 && format != CJ_OUT_RGB_FANCY)
    return PROGRAMMER_ERROR;
  if (idct != CJ_PIX_IDCT_INT && idct != CJ_PIX_IDCT_TC) return PROGRAMMER_ERROR;
  b->out_format = format;
  b->idct = idct;
  return 0;
}

int cjBatchSetHypotheses(CJBatch* b, int on) {
  if (!b) return PROGRAMMER_ERROR;
  b->hyp_enabled = on != 0;
  return 0;
}

int cjBatchSetParse(CJBatch* b, int on_device) {
  if (!b) return PROGRAMMER_ERROR;
  b->parse_on_device = on_device != 0;
  return 0;
}

// Host check of the device header parse: cj_parse_header (the function
// k_parse_headers runs, here on the host) against the host marker loop of
// the drop-in path with a fresh reader (cj_parse_to_scan + bt_fill_header).
int cjDebugParseCompare(const unsigned char* data, size_t size, int* err_host, int* err_parse) {
  if (!data || !err_host || !err_parse) return PROGRAMMER_ERROR;
  JPGReader* r = newJPGReader();
  if (!r) return OOM_ERROR;
  CJImageHeader* h1 = new (std::nothrow) CJImageHeader;
  CJImageHeader* h2 = new (std::nothrow) CJImageHeader;
  if (!h1 || !h2) {
    delete h1;
    delete h2;
    delJPGReader(r);
    return OOM_ERROR;
  }
  memset(h1, 0, sizeof(*h1));
  int64_t so1 = 0, sl1 = 0, so2 = 0, sl2 = 0;
  int e1 = cj_parse_to_scan(r, data, size);
  if (!e1) {
    e1 = bt_fill_header(r, h1);
    so1 = (int64_t)(r->pos - data);
    sl1 = (int64_t)(r->end - r->pos);
  }
  if (!e1 && (uint64_t)sl1 > CJ_MAX_SCAN_BYTES) e1 = UNSUPPORTED_ERROR;
  const int e2 = cj_parse_header(data, (int64_t)size, h2, &so2, &sl2);
  *err_host = e1;
  *err_parse = e2;
  int diff = 0;
  if (e1 != e2) diff |= 1;
  if (!e1 && !e2) {
    if (so1 != so2 || sl1 != sl2) diff |= 2;
    if (memcmp(h1, h2, sizeof(CJImageHeader))) diff |= 4;
  }
  delete h1;
  delete h2;
  delJPGReader(r);
  return diff;
}

void cjBatchGetOutput(const CJBatch* b, int* format, int* idct) {
  if (format) *format = b->out_format;
  if (idct) *idct = b->idct;
}

int cjBatchSetWaitLimit(CJBatch* b, unsigned polls) {
  if (!b) return PROGRAMMER_ERROR;
  b->wait_limit = polls;
  b->graph_stale = true;  // the limit is a kernel argument baked into the graph
  return 0;
}

void cjBatchGetTuning(const CJBatch* b, int* sub_bits, int* decode_ctas_per_sm, int* pixel_tile_cap) {
  if (sub_bits) *sub_bits = b->sub_bits;
  if (decode_ctas_per_sm) *decode_ctas_per_sm = b->decode_ctas;
  if (pixel_tile_cap) *pixel_tile_cap = b->tile_cap;
}

int cjBatchStage(CJBatch* b, int n, const unsigned char* blob, const int64_t* offsets,
                 const int64_t* sizes) {
  int err = bt_init(b);
  if (err) return err;
  if (n < 0) return PROGRAMMER_ERROR;
  b->n_in = n;
  b->graph_stale = true;
  b->dev_of.assign(n, -1);
  b->host_err.assign(n, 0);
  b->dims.clear();
  b->outoff.clear();
  int64_t blob_bytes = 0;
  for (int i = 0; i < n; i++) blob_bytes = std::max(blob_bytes, offsets[i] + sizes[i]);
  if (cj_host_ensure(b->h_hdr, (size_t)std::max(n, 1) * sizeof(CJImageHeader)) ||
      cj_host_ensure(b->h_desc, (size_t)std::max(n, 1) * sizeof(CJImageDesc)))
    return OOM_ERROR;
  CJImageHeader* hh = (CJImageHeader*)b->h_hdr.p;
  CJImageDesc* dd = (CJImageDesc*)b->h_desc.p;
  // Marker parse on the GPU: the files go to the device first, one thread per
  // file parses its segments there (k_parse_headers); the headers stay on
  // the device and only the summaries the plan needs come back, through
  // mapped pinned memory.  The same parse runs on the host with
  // cjBatchSetParse(b, 0).
  const bool dev_parse = b->parse_on_device && n > 0;
  const CJParseSummary* psum = nullptr;
  if (dev_parse) {
    const size_t nn = (size_t)n;
    if (cj_host_ensure(b->h_psize, nn * 16)) return OOM_ERROR;
    if (nn > b->psum_cap) {
      if (b->h_psum) cudaFreeHost(b->h_psum);
      b->h_psum = b->d_psum = nullptr;
      b->psum_cap = 0;
      const size_t cap = nn + nn / 2 + 64;
      void* hp = nullptr;
      if (cudaHostAlloc(&hp, cap * sizeof(CJParseSummary), cudaHostAllocMapped) != cudaSuccess) {
        cudaGetLastError();
        return OOM_ERROR;
      }
      void* dp = nullptr;
      if (cudaHostGetDevicePointer(&dp, hp, 0) != cudaSuccess) {
        cudaGetLastError();
        cudaFreeHost(hp);
        return CUDA_MEM_ERROR;
      }
      b->h_psum = (CJParseSummary*)hp;
      b->d_psum = (CJParseSummary*)dp;
      b->psum_cap = cap;
    }
    if (bt_ensure(b, b->blob, (size_t)blob_bytes + 64) || bt_ensure(b, b->p_size, nn * 16) ||
        bt_ensure(b, b->p_hdr, nn * sizeof(CJImageHeader)))
      return CUDA_MEM_ERROR;
    int64_t* hs = (int64_t*)b->h_psize.p;
    memcpy(hs, offsets, nn * 8);
    memcpy(hs + n, sizes, nn * 8);
    cudaStream_t s = b->stream;
    CJ_CUDA_TRY(cudaMemcpyAsync(b->blob.p, blob, (size_t)blob_bytes, cudaMemcpyHostToDevice, s), CUDA_MEM_ERROR);
    CJ_CUDA_TRY(cudaMemcpyAsync(b->p_size.p, hs, nn * 16, cudaMemcpyHostToDevice, s), CUDA_MEM_ERROR);
    const int64_t* d_off = (const int64_t*)b->p_size.p;
    k_parse_headers<<<(n + BT_PARSE_THREADS - 1) / BT_PARSE_THREADS, BT_PARSE_THREADS, 0, s>>>(
        (const uint8_t*)b->blob.p, d_off, d_off + n, n, (CJImageHeader*)b->p_hdr.p, b->d_psum);
    CJ_CUDA_TRY(cudaGetLastError(), CUDA_KERNEL_LAUNCH_ERROR);
    b->launches++;
    CJ_CUDA_TRY(cudaStreamSynchronize(s), CUDA_KERNEL_LAUNCH_ERROR);
    psum = b->h_psum;
  }
  std::vector<int32_t>& file_of = b->file_of;
  file_of.clear();
  int nd = 0, ntiles = 0, nsubw = 0, nptiles = 0, nmark = 0, nseg = 0;
  int64_t data_bytes = 0, blocks = 0, out_total = 0, planar_total = 0, npix = 0;
  const bool fancy = b->out_format == CJ_OUT_RGB_FANCY;
  // the pixel kernel's format: fancy mode writes planar samples for k_fancy_rgb
  const int pix_format = fancy ? CJ_OUT_PLANAR : b->out_format;
  size_t smem = 0;
  for (int i = 0; i < n; i++) {
    int64_t so = 0, sl = 0;
    int e;
    if (dev_parse) {  // the header without its tables (they stay on the device)
      const CJParseSummary& q = psum[i];
      e = q.err;
      so = q.scan_off;
      sl = q.scan_len;
      if (!e) {
        CJImageHeader& h = hh[nd];
        memset(&h, 0, sizeof(h));
        h.total_blocks = q.total_blocks;
        h.mcux = q.mcux;
        h.mcuy = q.mcuy;
        h.width = q.width;
        h.height = q.height;
        h.hmax = q.hmax;
        h.vmax = q.vmax;
        h.restart_interval = q.restart_interval;
        h.nseg_expected = q.nseg_expected;
        h.nch = q.nch;
        h.huff_mask = q.huff_mask;
        h.xshift = q.xshift;
        h.yshift = q.yshift;
        for (int c = 0; c < 3; c++) {
          h.comp_dc[c] = q.comp_dc[c];
          h.comp_ac[c] = q.comp_ac[c];
          h.comp_q[c] = q.comp_q[c];
          h.comp_sx[c] = q.comp_sx[c];
          h.comp_sy[c] = q.comp_sy[c];
        }
      }
    } else {
      e = bt_parse(b, blob + offsets[i], (size_t)sizes[i], &hh[nd], &so, &sl);
    }
    if (!e && (uint64_t)sl > CJ_MAX_SCAN_BYTES) e = UNSUPPORTED_ERROR;
    if (e) {
      b->host_err[i] = e;
      continue;
    }
    const CJImageHeader& h = hh[nd];
    CJImageDesc& d = dd[nd];
    memset(&d, 0, sizeof(d));
    d.src_off = offsets[i] + so;
    d.raw_len = sl;
    d.data_off = data_bytes;
    data_bytes += (sl + 16 + 15) & ~(int64_t)15;
    d.tile0 = ntiles;
    d.ntiles = (int)((sl + BT_TILE_BYTES - 1) / BT_TILE_BYTES);
    if (d.ntiles < 1) d.ntiles = 1;
    ntiles += d.ntiles;
    d.mark0 = nmark;
    d.mark_cap = h.nseg_expected + 1;
    nmark += d.mark_cap;
    d.seg0 = nseg;
    d.seg_cap = h.nseg_expected;
    nseg += d.seg_cap;
    d.sub_bits = bt_sub_bits_for(b, h);
    int sub_cap = (int)((sl * 8 + d.sub_bits - 1) / d.sub_bits) + h.nseg_expected + 1;
    sub_cap = (sub_cap + 31) & ~31;
    d.sub0 = nsubw * 32;
    d.sub_cap = sub_cap;
    nsubw += sub_cap / 32;
    int bpm = (int)(h.total_blocks / ((int64_t)h.mcux * h.mcuy));
    d.T = b->idct == CJ_PIX_IDCT_TC ? cj_pix_tile_mcus_tc(h.hmax, bpm) : cj_pix_tile_mcus(h.hmax, bpm);
    while (b->tile_cap > 0 && d.T > b->tile_cap && d.T > 1) d.T >>= 1;
    d.ptile0 = nptiles;
    d.nptiles = h.mcuy * ((h.mcux + d.T - 1) / d.T);
    nptiles += d.nptiles;
    d.coef0 = blocks;
    blocks += h.total_blocks;
    int ch = h.nch == 3 ? 3 : 1;
    if (fancy) {
      d.out_off = planar_total;
      planar_total += (bt_out_bytes(h, CJ_OUT_PLANAR) + 15) & ~(int64_t)15;
      d.rgb_off = out_total;
      out_total += ((int64_t)h.width * h.height * ch + 15) & ~(int64_t)15;
      d.pix0 = npix;
      npix += (int64_t)h.width * h.height;
    } else {
      d.out_off = out_total;
      out_total += (bt_out_bytes(h, pix_format) + 15) & ~(int64_t)15;  // 16-byte aligned starts
    }
    CJPixGeom g;
    g.nch = h.nch;
    g.bpm = bpm;
    g.hmax = h.hmax;
    g.vmax = h.vmax;
    g.T = d.T;
    smem = std::max(smem, cj_pix_layout(&g, h.comp_sx[1], h.comp_sy[1], 2, b->idct == CJ_PIX_IDCT_TC));
    b->dev_of[i] = nd;
    if (dev_parse) file_of.push_back(i);
    b->dims.push_back(h.width);
    b->dims.push_back(h.height);
    b->dims.push_back(ch);
    b->dims.push_back(h.nch == 3 ? (h.width * h.comp_sx[1] + h.hmax - 1) / h.hmax : 0);
    b->dims.push_back(h.nch == 3 ? (h.height * h.comp_sy[1] + h.vmax - 1) / h.vmax : 0);
    b->outoff.push_back(fancy ? d.rgb_off : d.out_off);
    nd++;
  }
  b->n_dev = nd;
  b->ntiles = ntiles;
  b->nwarps = nsubw;
  b->nptiles = nptiles;
  b->blob_bytes = blob_bytes;
  b->out_total = out_total;
  b->planar_total = planar_total;
  b->npix = npix;
  b->blocks = blocks;
  b->scan_bytes = data_bytes;
  b->smem = BT_DECODE_SMEM;
  b->smem_pix = smem;
  if (!nd) return 0;
  size_t nd_ = (size_t)nd;
  if (bt_ensure(b, b->hdr, nd_ * sizeof(CJImageHeader)) || bt_ensure(b, b->desc, nd_ * sizeof(CJImageDesc)) ||
      bt_ensure(b, b->prm, nd_ * sizeof(CJScanParams)) || bt_ensure(b, b->st, nd_ * sizeof(CJStatus)) ||
      bt_ensure(b, b->blob, (size_t)blob_bytes + 64) || bt_ensure(b, b->data, (size_t)data_bytes + 64) ||
      bt_ensure(b, b->tile_keep, (size_t)ntiles * 4) || bt_ensure(b, b->tile_mark, (size_t)ntiles * 4) ||
      bt_ensure(b, b->mpos, (size_t)nmark * 4) || bt_ensure(b, b->mcode, (size_t)nmark) ||
      bt_ensure(b, b->segs, (size_t)nseg * sizeof(CJSegment)) ||
      bt_ensure(b, b->recs, (size_t)nsubw * 32 * sizeof(CJSubRec)) ||
      bt_ensure(b, b->ckpt, (size_t)nsubw * 32 * CJ_CKPTS * sizeof(CJCkpt)) ||
      bt_ensure(b, b->snap, (size_t)2 * nsubw * sizeof(uint64_t)) ||
      bt_ensure(b, b->wagg, (size_t)nsubw * sizeof(CJWarpAgg)) ||
      bt_ensure(b, b->carry, (size_t)nsubw * sizeof(CJWarpAgg)) ||
      bt_ensure(b, b->coef, (size_t)blocks * 128 + 128) || bt_ensure(b, b->out, (size_t)out_total + 64) ||
      (fancy && bt_ensure(b, b->fancy, (size_t)planar_total + 64)) ||
      bt_ensure(b, b->ctl, sizeof(CJBatchCtl)))
    return CUDA_MEM_ERROR;
  if (cj_host_ensure(b->h_st, nd_ * sizeof(CJStatus)) || cj_host_ensure(b->h_ctl, sizeof(CJBatchCtl)))
    return OOM_ERROR;
  cudaStream_t s = b->stream;
  if (dev_parse) {  // the parsed headers, compacted to the planned images on the device
    if (cj_host_ensure(b->h_pmap, nd_ * 4) || bt_ensure(b, b->p_map, nd_ * 4)) return CUDA_MEM_ERROR;
    memcpy(b->h_pmap.p, file_of.data(), nd_ * 4);
    CJ_CUDA_TRY(cudaMemcpyAsync(b->p_map.p, b->h_pmap.p, nd_ * 4, cudaMemcpyHostToDevice, s), CUDA_MEM_ERROR);
    k_gather_headers<<<nd, 128, 0, s>>>((const CJImageHeader*)b->p_hdr.p, (const int32_t*)b->p_map.p,
                                        (CJImageHeader*)b->hdr.p);
    CJ_CUDA_TRY(cudaGetLastError(), CUDA_KERNEL_LAUNCH_ERROR);
    b->launches++;
  } else {
    CJ_CUDA_TRY(cudaMemcpyAsync(b->hdr.p, hh, nd_ * sizeof(CJImageHeader), cudaMemcpyHostToDevice, s),
                CUDA_MEM_ERROR);
  }
  CJ_CUDA_TRY(cudaMemcpyAsync(b->desc.p, dd, nd_ * sizeof(CJImageDesc), cudaMemcpyHostToDevice, s),
              CUDA_MEM_ERROR);
  if (!dev_parse)  // (the device parse copied the files already)
    CJ_CUDA_TRY(cudaMemcpyAsync(b->blob.p, blob, (size_t)blob_bytes, cudaMemcpyHostToDevice, s),
                CUDA_MEM_ERROR);
  int per_sm = 0;
  CJ_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)bt_decode_kernel(b->decode_ctas),
                                                            BT_THREADS, b->smem),
              CUDA_KERNEL_LAUNCH_ERROR);
  if (per_sm < 1) return UNSUPPORTED_ERROR;
  b->grid = std::min(per_sm, b->decode_ctas) * b->sm_count;
  // MCU-phase hypotheses only where their decodes fit beside the batch's own
  // warps in one round of the grid: a batch of a few images leaves most of
  // the GPU idle while its settle chains run, a full batch has no room
  b->nhyp = 1;
  if (b->hyp_enabled) {
    int maxbpm = 1;
    for (int k = 0; k < nd; k++) {
      int bpm = 0;
      for (int c = 0; c < hh[k].nch; c++) bpm += hh[k].comp_sx[c] * hh[k].comp_sy[c];
      maxbpm = std::max(maxbpm, bpm);
    }
    const int nh = std::min(maxbpm, BT_MAX_HYP);
    int per_sm_hyp = 0;  // the hypothesis variant must fit the same cooperative grid
    CJ_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                    &per_sm_hyp, (const void*)bt_decode_kernel(b->decode_ctas, true), BT_THREADS, b->smem),
                CUDA_KERNEL_LAUNCH_ERROR);
    if (nh > 1 && per_sm_hyp * b->sm_count >= b->grid && (int64_t)nsubw * nh <= (int64_t)b->grid * BT_WARPS) {
      const size_t nsub = (size_t)nsubw * 32, nrec = nsub * 2 * nh;  // hypotheses and probes
      if (bt_ensure(b, b->hrecs, nrec * sizeof(CJSubRec)) || bt_ensure(b, b->hckpt, nrec * CJ_CKPTS * sizeof(CJCkpt)) ||
          bt_ensure(b, b->hmap, nsub * 16))
        return CUDA_MEM_ERROR;
      b->nhyp = nh;
    }
  }
  const void* pk = (const void*)bt_pixel_kernel(b->idct, bt_pix_format(b));
  if (b->idct == CJ_PIX_IDCT_TC && !cj_tc_basis_device()) return CUDA_MEM_ERROR;
  if (b->idct == CJ_PIX_IDCT_TC)  // 64 tensor-memory columns per CTA
    per_sm = cj_tc_ctas_per_sm(pk, CJ_TC_THREADS, b->smem_pix, 64);
  else
    CJ_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pk, CJ_PIX_THREADS, b->smem_pix),
                CUDA_KERNEL_LAUNCH_ERROR);
  if (per_sm < 1) return UNSUPPORTED_ERROR;
  b->grid_pix = std::min(nptiles, per_sm * b->sm_count);
  return 0;
}

static CJBatchArgs bt_args(const CJBatch* b) {
  CJBatchArgs a{};
  a.hdr = (const CJImageHeader*)b->hdr.p;
  a.desc = (const CJImageDesc*)b->desc.p;
  a.prm = (CJScanParams*)b->prm.p;
  a.st = (CJStatus*)b->st.p;
  a.blob = (const uint8_t*)b->blob.p;
  a.data = (uint8_t*)b->data.p;
  a.tile_keep = (int32_t*)b->tile_keep.p;
  a.tile_mark = (int32_t*)b->tile_mark.p;
  a.mpos = (uint32_t*)b->mpos.p;
  a.mcode = (uint8_t*)b->mcode.p;
  a.segs = (CJSegment*)b->segs.p;
  a.recs = (CJSubRec*)b->recs.p;
  a.ckpt = (CJCkpt*)b->ckpt.p;
  a.snap0 = (uint64_t*)b->snap.p;
  a.snap1 = a.snap0 + b->nwarps;
  a.wagg = (CJWarpAgg*)b->wagg.p;
  a.carry = (CJWarpAgg*)b->carry.p;
  a.coef = (int16_t*)b->coef.p;
  a.tc_basis = b->idct == CJ_PIX_IDCT_TC ? cj_tc_basis_device() : nullptr;
  const bool fancy = b->out_format == CJ_OUT_RGB_FANCY;
  a.out = (uint8_t*)(fancy ? b->fancy.p : b->out.p);
  a.rgb = fancy ? (uint8_t*)b->out.p : nullptr;
  a.npix = fancy ? b->npix : 0;
  a.ctl = (CJBatchCtl*)b->ctl.p;
  a.n = b->n_dev;
  a.ntiles = b->ntiles;
  a.nwarps = b->nwarps;
  a.nptiles = b->nptiles;
  a.max_passes = b->nwarps + 2;
  a.wait_limit = b->wait_limit;
  a.nhyp = b->nhyp;
  a.hrecs = (CJSubRec*)b->hrecs.p;
  a.hckpt = (CJCkpt*)b->hckpt.p;
  a.hmap = (uint8_t*)b->hmap.p;
  return a;
}

// The run of a staged batch as one CUDA graph: clear the control block, the
// cooperative decode kernel (graph kernel node with the cooperative launch
// attribute), the pixel kernel.  Buffers, counts and the decode-kernel
// variant are baked into the nodes, so after every stage the graph is
// rebuilt and the executable graph updated in place (instantiated again only
// when that update is refused).
static void bt_drop_graph(CJBatch* b) {
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  b->gexec = nullptr;
}

static bool bt_build_graph(CJBatch* b) {
  const CJBatchArgs a = bt_args(b);
  cudaGraph_t g = nullptr;
  if (cudaGraphCreate(&g, 0) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  bool ok = true;
  cudaGraphNode_t n_mem = nullptr, n_dec = nullptr, n_pix = nullptr;
  cudaMemsetParams mp;
  memset(&mp, 0, sizeof(mp));
  mp.dst = b->ctl.p;
  mp.value = 0;
  mp.elementSize = 1;
  mp.width = sizeof(CJBatchCtl);
  mp.height = 1;
  mp.pitch = 0;
  ok = ok && cudaGraphAddMemsetNode(&n_mem, g, nullptr, 0, &mp) == cudaSuccess;
  CJBatchArgs a1 = a;
  void* args[] = {&a1};
  cudaKernelNodeParams kp;
  memset(&kp, 0, sizeof(kp));
  kp.func = (void*)bt_decode_kernel(b->decode_ctas, b->nhyp > 1);
  kp.gridDim = dim3(b->grid);
  kp.blockDim = dim3(BT_THREADS);
  kp.sharedMemBytes = (unsigned)b->smem;
  kp.kernelParams = args;
  ok = ok && cudaGraphAddKernelNode(&n_dec, g, &n_mem, 1, &kp) == cudaSuccess;
  if (ok) {
    cudaLaunchAttributeValue v;
    memset(&v, 0, sizeof(v));
    v.cooperative = 1;
    ok = cudaGraphKernelNodeSetAttribute(n_dec, cudaLaunchAttributeCooperative, &v) == cudaSuccess;
  }
  if (ok && b->grid_pix > 0) {
    cudaKernelNodeParams pp = kp;
    pp.func = (void*)bt_pixel_kernel(b->idct, bt_pix_format(b));
    pp.gridDim = dim3(b->grid_pix);
    pp.blockDim = dim3(b->idct == CJ_PIX_IDCT_TC ? CJ_TC_THREADS : CJ_PIX_THREADS);
    pp.sharedMemBytes = (unsigned)b->smem_pix;
    ok = cudaGraphAddKernelNode(&n_pix, g, &n_dec, 1, &pp) == cudaSuccess;
  }
  if (ok && n_pix && b->out_format == CJ_OUT_RGB_FANCY && b->npix > 0) {
    cudaGraphNode_t n_fancy = nullptr;
    cudaKernelNodeParams fp = kp;
    fp.func = (void*)k_fancy_rgb;
    fp.gridDim = dim3(b->sm_count * 8);
    fp.blockDim = dim3(256);
    fp.sharedMemBytes = 0;
    ok = cudaGraphAddKernelNode(&n_fancy, g, &n_pix, 1, &fp) == cudaSuccess;
  }
  if (ok && b->gexec) {
    // same topology as the instantiated graph: update its nodes in place
    // (much cheaper than instantiating; batches are staged back to back)
    cudaGraphExecUpdateResultInfo info;
    if (cudaGraphExecUpdate(b->gexec, g, &info) != cudaSuccess) {
      cudaGetLastError();
      bt_drop_graph(b);
    }
  }
  if (ok && !b->gexec) ok = cudaGraphInstantiate(&b->gexec, g, 0) == cudaSuccess;
  cudaGraphDestroy(g);
  if (!ok) {
    cudaGetLastError();
    bt_drop_graph(b);
  }
  return ok;
}

int cjBatchRun(CJBatch* b) {
  if (!b->ready) return PROGRAMMER_ERROR;
  if (!b->n_dev) return 0;
  cudaStream_t s = b->stream;
  if (b->use_graph && b->graph_stale) {
    b->graph_stale = false;
    if (!bt_build_graph(b)) b->graph_failures++;
  }
  if (b->use_graph && b->gexec) {
    CJ_CUDA_TRY(cudaEventRecord(b->ev0, s), CUDA_KERNEL_LAUNCH_ERROR);
    CJ_CUDA_TRY(cudaGraphLaunch(b->gexec, s), CUDA_KERNEL_LAUNCH_ERROR);
    CJ_CUDA_TRY(cudaEventRecord(b->ev1, s), CUDA_KERNEL_LAUNCH_ERROR);
    b->launches += (b->grid_pix > 0 ? 2 : 1) + (b->out_format == CJ_OUT_RGB_FANCY && b->grid_pix > 0 && b->npix > 0);
    b->graph_launches++;
    return 0;
  }
  CJBatchArgs a = bt_args(b);
  CJ_CUDA_TRY(cudaMemsetAsync(b->ctl.p, 0, sizeof(CJBatchCtl), s), CUDA_MEM_ERROR);
  CJ_CUDA_TRY(cudaEventRecord(b->ev0, s), CUDA_KERNEL_LAUNCH_ERROR);
  void* args[] = {&a};
  CJ_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)bt_decode_kernel(b->decode_ctas, b->nhyp > 1), dim3(b->grid),
                                          dim3(BT_THREADS), args, b->smem, s),
              CUDA_KERNEL_LAUNCH_ERROR);
  b->launches++;
  if (b->grid_pix > 0) {
    bt_pixel_kernel(b->idct, bt_pix_format(b))<<<b->grid_pix, b->idct == CJ_PIX_IDCT_TC ? CJ_TC_THREADS : CJ_PIX_THREADS,
                                                 b->smem_pix, s>>>(a);
    CJ_CUDA_TRY(cudaGetLastError(), CUDA_KERNEL_LAUNCH_ERROR);
    b->launches++;
    if (b->out_format == CJ_OUT_RGB_FANCY && b->npix > 0) {
      k_fancy_rgb<<<b->sm_count * 8, 256, 0, s>>>(a);
      CJ_CUDA_TRY(cudaGetLastError(), CUDA_KERNEL_LAUNCH_ERROR);
      b->launches++;
    }
  }
  CJ_CUDA_TRY(cudaEventRecord(b->ev1, s), CUDA_KERNEL_LAUNCH_ERROR);
  return 0;
}

int cjBatchFetch(CJBatch* b) {
  if (!b->ready) return PROGRAMMER_ERROR;
  if (!b->n_dev) return 0;
  if (cj_host_ensure(b->h_out, (size_t)b->out_total + 64)) return OOM_ERROR;
  cudaStream_t s = b->stream;
  CJ_CUDA_TRY(cudaMemcpyAsync(b->h_out.p, b->out.p, (size_t)b->out_total, cudaMemcpyDeviceToHost, s),
              CUDA_MEM_ERROR);
  return 0;
}

int cjBatchWait(CJBatch* b, int* errors) {
  if (!b->ready) return PROGRAMMER_ERROR;
  cudaStream_t s = b->stream;
  if (b->n_dev) {
    CJ_CUDA_TRY(cudaMemcpyAsync(b->h_st.p, b->st.p, (size_t)b->n_dev * sizeof(CJStatus),
                                cudaMemcpyDeviceToHost, s),
                CUDA_MEM_ERROR);
    CJ_CUDA_TRY(cudaMemcpyAsync(b->h_ctl.p, b->ctl.p, sizeof(CJBatchCtl), cudaMemcpyDeviceToHost, s),
                CUDA_MEM_ERROR);
  }
  CJ_CUDA_TRY(cudaStreamSynchronize(s), CUDA_KERNEL_LAUNCH_ERROR);
  const CJBatchCtl* ctl = (const CJBatchCtl*)b->h_ctl.p;
  int batch_err = 0;
  if (b->n_dev && ctl->timeout) batch_err = CUDA_KERNEL_LAUNCH_ERROR;  // a grid barrier's wait ran out
  else if (b->n_dev && ctl->passes > b->nwarps + 2) batch_err = PROGRAMMER_ERROR;
  const CJStatus* st = (const CJStatus*)b->h_st.p;
  if (errors)
    for (int i = 0; i < b->n_in; i++) {
      int k = b->dev_of[i];
      errors[i] = k < 0 ? b->host_err[i] : (batch_err ? batch_err : cj_status_error(&st[k]));
    }
  return batch_err;
}

int cjBatchDecode(CJBatch* b, int n, const unsigned char* blob, const int64_t* offsets,
                  const int64_t* sizes, int* errors) {
  int e = cjBatchStage(b, n, blob, offsets, sizes);
  if (!e) e = cjBatchRun(b);
  if (!e) e = cjBatchFetch(b);
  int w = cjBatchWait(b, errors);
  return e ? e : w;
}

const unsigned char* cjBatchImage(const CJBatch* b, int i, int* w, int* h, int* c) {
  if (i < 0 || i >= b->n_in || b->dev_of[i] < 0 || !b->h_out.p) return NULL;
  int k = b->dev_of[i];
  if (w) *w = b->dims[5 * k];
  if (h) *h = b->dims[5 * k + 1];
  if (c) *c = b->dims[5 * k + 2];
  return (const unsigned char*)b->h_out.p + b->outoff[k];
}

int cjBatchImageGeometry(const CJBatch* b, int i, int* w, int* h, int* c) {
  if (i < 0 || i >= b->n_in || b->dev_of[i] < 0) return PROGRAMMER_ERROR;
  int k = b->dev_of[i];
  if (w) *w = b->dims[5 * k];
  if (h) *h = b->dims[5 * k + 1];
  if (c) *c = b->dims[5 * k + 2];
  return 0;
}

int cjBatchChromaGeometry(const CJBatch* b, int i, int* cw, int* ch) {
  if (i < 0 || i >= b->n_in || b->dev_of[i] < 0) return PROGRAMMER_ERROR;
  int k = b->dev_of[i];
  if (cw) *cw = b->dims[5 * k + 3];
  if (ch) *ch = b->dims[5 * k + 4];
  return 0;
}

const unsigned char* cjBatchDeviceImage(const CJBatch* b, int i) {
  if (i < 0 || i >= b->n_in || b->dev_of[i] < 0) return NULL;
  return (const unsigned char*)b->out.p + b->outoff[b->dev_of[i]];
}

void* cjBatchStream(const CJBatch* b) { return (void*)b->stream; }

DLManagedTensor* cjBatchDLPack(CJBatch* b, int i) {
  if (!b || !b->ready || i < 0 || i >= b->n_in || b->dev_of[i] < 0) return NULL;
  const int k = b->dev_of[i];
  const int64_t w = b->dims[5 * k], h = b->dims[5 * k + 1], c = b->dims[5 * k + 2];
  void* p = (unsigned char*)b->out.p + b->outoff[k];
  if (c == 3 && (b->out_format == CJ_OUT_PLANAR || b->out_format == CJ_OUT_NV12)) {
    const int64_t n[1] = {w * h + 2 * (int64_t)b->dims[5 * k + 3] * b->dims[5 * k + 4]};
    return cj_dl_view(p, b->device, 1, n);
  }
  const int64_t shape[3] = {h, w, 3};
  return cj_dl_view(p, b->device, c == 3 ? 3 : 2, shape);
}

long long cjBatchCopyCoefficients(CJBatch* b, int i, short* dst, long long max_blocks) {
  if (!b || !b->ready || i < 0 || i >= b->n_in || b->dev_of[i] < 0 || !dst) return PROGRAMMER_ERROR;
  const int k = b->dev_of[i];
  const CJImageDesc* dd = (const CJImageDesc*)b->h_desc.p;
  const CJImageHeader* hh = (const CJImageHeader*)b->h_hdr.p;
  const int64_t n = hh[k].total_blocks;
  if (n > max_blocks) return PROGRAMMER_ERROR;
  CJ_CUDA_TRY(cudaMemcpyAsync(dst, (const int16_t*)b->coef.p + dd[k].coef0 * 64, (size_t)n * 128,
                              cudaMemcpyDeviceToHost, b->stream),
              CUDA_MEM_ERROR);
  CJ_CUDA_TRY(cudaStreamSynchronize(b->stream), CUDA_KERNEL_LAUNCH_ERROR);
  return n;
}

int cjBatchPhaseTimes(const CJBatch* b, float* ms) {
  const CJBatchCtl* ctl = (const CJBatchCtl*)b->h_ctl.p;
  if (!ctl) return 0;
  const float total = cjBatchKernelMs(b);
  for (int k = 0; k < BT_NPHASE; k++) ms[k] = (float)((ctl->t[k + 1] - ctl->t[k]) * 1e-6);
  // the rest of the run: graph launch, control-block clear, kernel boundaries
  ms[BT_NPHASE] = total - (float)((ctl->t[BT_NPHASE] - ctl->t[0]) * 1e-6);
  return BT_NPHASE + 1;
}

void cjBatchStats(const CJBatch* b, int64_t* s) {
  const CJBatchCtl* ctl = (const CJBatchCtl*)b->h_ctl.p;
  s[0] = b->n_in;
  s[1] = b->n_dev;
  s[2] = b->grid;
  s[3] = b->nwarps;
  s[4] = b->ntiles;
  s[5] = b->nptiles;
  s[6] = ctl ? ctl->passes : 0;
  s[7] = b->blob_bytes;
  s[8] = b->out_total;
  s[9] = (int64_t)b->smem_pix;
  s[10] = b->launches;
  s[11] = b->grid_pix;
  s[12] = b->graph_launches;
  s[13] = b->graph_failures;
  s[14] = b->blocks;
  s[15] = b->scan_bytes;
}

float cjBatchKernelMs(const CJBatch* b) {
  float ms = 0.f;
  if (b->ready) cudaEventElapsedTime(&ms, b->ev0, b->ev1);
  return ms;
}

// Device time of the staged batch under the current tuning: median of
// `reps` runs after one warm-up run.
static int bt_time_config(CJBatch* b, int n, const unsigned char* blob, const int64_t* offsets,
                          const int64_t* sizes, int reps, float* ms) {
  int e = cjBatchStage(b, n, blob, offsets, sizes);
  if (!e) e = cjBatchRun(b);
  if (!e) e = cjBatchWait(b, NULL);
  std::vector<float> t;
  for (int r = 0; r < reps && !e; r++) {
    e = cjBatchRun(b);
    if (!e) e = cjBatchWait(b, NULL);
    t.push_back(cjBatchKernelMs(b));
  }
  if (e) return e;
  std::sort(t.begin(), t.end());
  *ms = t[t.size() / 2];
  return 0;
}

int cjBatchAutotune(CJBatch* b, int n, const unsigned char* blob, const int64_t* offsets,
                    const int64_t* sizes, int reps, float* best_ms, float* trials_ms, int max_trials) {
  if (!b || n <= 0 || !blob) return PROGRAMMER_ERROR;
  if (reps < 1) reps = 3;
  static const int subs[] = {512, 1024, 2048, 4096};
  static const int ctas[] = {3, 4, 5};
  int best_s = b->sub_bits, best_c = b->decode_ctas, best_t = 0;
  float best = 1e30f;
  int trial = 0;
  auto record = [&](float ms) {
    if (trials_ms && trial < max_trials) trials_ms[trial] = ms;
    trial++;
  };
  // 1. subsequence size x decode-kernel occupancy (one size for every class)
  for (int k = 0; k < CJ_SAMPLING_CLASSES; k++) b->sub_bits_class[k] = 0;
  for (int sb : subs)
    for (int c : ctas) {
      b->sub_bits = sb;
      b->decode_ctas = c;
      b->tile_cap = 0;
      float ms = 0.f;
      int e = bt_time_config(b, n, blob, offsets, sizes, reps, &ms);
      if (e) return e;
      record(ms);
      if (ms < best) {
        best = ms;
        best_s = sb;
        best_c = c;
      }
    }
  // 1b. per sampling class holding at least 1/16 of the scan bytes: other
  // sizes for that class alone, the others at their best so far
  b->sub_bits = best_s;
  b->decode_ctas = best_c;
  b->tile_cap = 0;
  int64_t cls_bytes[CJ_SAMPLING_CLASSES] = {0, 0, 0, 0, 0}, all_bytes = 0;
  {
    const CJImageHeader* hh = (const CJImageHeader*)b->h_hdr.p;  // the last stage's images
    const CJImageDesc* dd = (const CJImageDesc*)b->h_desc.p;
    for (int k = 0; k < b->n_dev; k++) {
      cls_bytes[bt_sampling_class(hh[k])] += dd[k].raw_len;
      all_bytes += dd[k].raw_len;
    }
  }
  for (int c = 0; c < CJ_SAMPLING_CLASSES; c++) {
    if (cls_bytes[c] * 16 < all_bytes) continue;
    int best_c_bits = 0;
    for (int sb : {1024, 2048, 4096, 8192, 16384}) {
      if (sb == best_s) continue;
      b->sub_bits_class[c] = sb;
      float ms = 0.f;
      int e = bt_time_config(b, n, blob, offsets, sizes, reps, &ms);
      if (e) return e;
      record(ms);
      if (ms < best) {
        best = ms;
        best_c_bits = sb;
      }
    }
    b->sub_bits_class[c] = best_c_bits;
  }
  // 2. pixel tile width at the best entropy configuration
  for (int cap : {8, 4, 2}) {
    b->tile_cap = cap;
    float ms = 0.f;
    int e = bt_time_config(b, n, blob, offsets, sizes, reps, &ms);
    if (e) return e;
    record(ms);
    if (ms < best) {
      best = ms;
      best_t = cap;
    }
  }
  b->tile_cap = best_t;
  if (best_ms) *best_ms = best;
  // leave the batch staged under the chosen tuning
  return cjBatchStage(b, n, blob, offsets, sizes);
}

}  // extern "C"

// ---------------------------------------------------------------- the drop-in reader

// decodeScanGPU's device decode (and cjReaderRedecodeDevice's): the batch
// decode kernel on the reader's one image, in the reader's grow-only
// buffers -- one cooperative launch, Huffman tables built on the device,
// fix-up passes looped on the device.  The grid is the co-resident maximum,
// cut to the image's work (destuff tiles, warp groups) for small images so
// that idle CTAs do not lengthen the grid barriers.
int cj_reader_decode(JPGReader* jpg, bool stage) {
  CJReaderDevice* d = jpg->dev;
  cudaStream_t s = d->stream;
  if (stage) {
    CJImageHeader h;
    int e = bt_fill_header(jpg, &h);
    if (e) return e;
    const int64_t n = (int64_t)(jpg->end - jpg->pos);
    static bool attrs = false;  // per process: the attribute is per function, not per device
    if (!attrs) {
      CJ_CUDA_TRY(bt_decode_attrs(), CUDA_MEM_ERROR);
      attrs = true;
    }
    int sms = 0, per_sm = 0;
    CJ_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d->device), CUDA_MEM_ERROR);
    CJ_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                    &per_sm, (const void*)bt_decode_kernel(BT_DECODE_CTAS_DEFAULT), BT_THREADS, BT_DECODE_SMEM),
                CUDA_KERNEL_LAUNCH_ERROR);
    if (per_sm < 1) return UNSUPPORTED_ERROR;
    const int cap = std::min(per_sm, BT_DECODE_CTAS_DEFAULT) * sms;
    int bpm = 0;
    for (int c = 0; c < h.nch; c++) bpm += h.comp_sx[c] * h.comp_sy[c];
    const int nh = std::min(bpm, BT_MAX_HYP);
    CJImageDesc desc;
    // the default size: 512-bit subsequences (more, shorter speculative
    // decodes: the lowest latency) when their hypothesis decodes still fit
    // in one round of the grid, else 1024 bits
    int sub = d->sub_bits;
    if (d->sub_bits_auto) {
      bt_plan_one(h, n, 512, &desc);
      sub = (int64_t)(desc.sub_cap / 32) * std::max(nh, 1) <= (int64_t)cap * BT_WARPS ? 512 : CJ_SUB_BITS_DEFAULT;
    }
    bt_plan_one(h, n, sub, &desc);
    const int nwarps = desc.sub_cap / 32;
    if (cj_dev_ensure(d->bhdr, sizeof(CJImageHeader)) || cj_dev_ensure(d->bdesc, sizeof(CJImageDesc)) ||
        cj_dev_ensure(d->params, sizeof(CJScanParams)) || cj_dev_ensure(d->status, sizeof(CJStatus)) ||
        cj_dev_ensure(d->raw, (size_t)n + 64) || cj_dev_ensure(d->data, (size_t)n + 64) ||
        cj_dev_ensure(d->tile_keep, (size_t)desc.ntiles * 4) || cj_dev_ensure(d->tile_mark, (size_t)desc.ntiles * 4) ||
        cj_dev_ensure(d->mpos, (size_t)desc.mark_cap * 4) || cj_dev_ensure(d->mcode, (size_t)desc.mark_cap) ||
        cj_dev_ensure(d->segs, (size_t)desc.seg_cap * sizeof(CJSegment)) ||
        cj_dev_ensure(d->recs, (size_t)desc.sub_cap * sizeof(CJSubRec)) ||
        cj_dev_ensure(d->ckpt, (size_t)desc.sub_cap * CJ_CKPTS * sizeof(CJCkpt)) ||
        cj_dev_ensure(d->snap, (size_t)2 * nwarps * sizeof(uint64_t)) ||
        cj_dev_ensure(d->wagg, (size_t)nwarps * sizeof(CJWarpAgg)) ||
        cj_dev_ensure(d->carry, (size_t)nwarps * sizeof(CJWarpAgg)) ||
        cj_dev_ensure(d->coef, (size_t)h.total_blocks * 128 + 128) || cj_dev_ensure(d->bctl, sizeof(CJBatchCtl)))
      return CUDA_MEM_ERROR;
    if (cj_host_ensure(d->h_bctl, sizeof(CJBatchCtl))) return OOM_ERROR;
    // MCU-phase hypotheses when their decodes fit in one round of the grid
    // (one image leaves most of the GPU idle while its settle chains run)
    d->b_nhyp = 1;
    d->b_ctas = BT_DECODE_CTAS_DEFAULT;
    const int groups = (nwarps + BT_WARPS - 1) / BT_WARPS;
    if (nh > 1 && (int64_t)nwarps * nh <= (int64_t)cap * BT_WARPS) {
      // the hypothesis variant must fit the cooperative grid: its 3-CTA
      // build (no register spills) when the grid allows, else the 4-CTA one
      const int grid_h = std::max(1, std::min(cap, std::max(desc.ntiles, groups * nh)));
      int per3 = 0, per4 = 0;
      CJ_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per3, (const void*)bt_decode_kernel(3, true),
                                                                BT_THREADS, BT_DECODE_SMEM),
                  CUDA_KERNEL_LAUNCH_ERROR);
      CJ_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                      &per4, (const void*)bt_decode_kernel(BT_DECODE_CTAS_DEFAULT, true), BT_THREADS, BT_DECODE_SMEM),
                  CUDA_KERNEL_LAUNCH_ERROR);
      const int ctas = per3 * sms >= grid_h ? 3 : (per4 * sms >= grid_h ? BT_DECODE_CTAS_DEFAULT : 0);
      if (ctas) {
        const size_t nsub = (size_t)desc.sub_cap, nrec = nsub * 2 * nh;  // hypotheses and probes
        if (cj_dev_ensure(d->hrecs, nrec * sizeof(CJSubRec)) ||
            cj_dev_ensure(d->hckpt, nrec * CJ_CKPTS * sizeof(CJCkpt)) || cj_dev_ensure(d->hmap, nsub * 16))
          return CUDA_MEM_ERROR;
        d->b_nhyp = nh;
        d->b_ctas = ctas;
      }
    }
    const int work = std::max(desc.ntiles, groups * d->b_nhyp);
    d->b_grid = std::max(1, std::min(cap, work));
    d->b_ntiles = desc.ntiles;
    d->b_nwarps = nwarps;
    d->b_nptiles = desc.nptiles;
    d->raw_len = (size_t)n;
    d->total_blocks = h.total_blocks;
    d->param_bytes = sizeof(CJImageHeader) + sizeof(CJImageDesc);
    CJ_CUDA_TRY(cudaEventRecord(d->ev_begin, s), CUDA_KERNEL_LAUNCH_ERROR);
    CJ_CUDA_TRY(cudaMemcpyAsync(d->bhdr.p, &h, sizeof(h), cudaMemcpyHostToDevice, s), CUDA_MEM_ERROR);
    CJ_CUDA_TRY(cudaMemcpyAsync(d->bdesc.p, &desc, sizeof(desc), cudaMemcpyHostToDevice, s), CUDA_MEM_ERROR);
    // (a copy from pageable memory returns once its source has been staged,
    // so the header and plan may live on this stack frame)
    if (n) CJ_CUDA_TRY(cudaMemcpyAsync(d->raw.p, jpg->pos, (size_t)n, cudaMemcpyHostToDevice, s), CUDA_MEM_ERROR);
  } else {
    CJ_CUDA_TRY(cudaEventRecord(d->ev_begin, s), CUDA_KERNEL_LAUNCH_ERROR);
  }
  CJBatchArgs a;
  memset(&a, 0, sizeof(a));
  a.hdr = (const CJImageHeader*)d->bhdr.p;
  a.desc = (const CJImageDesc*)d->bdesc.p;
  a.prm = (CJScanParams*)d->params.p;
  a.st = (CJStatus*)d->status.p;
  a.blob = (const uint8_t*)d->raw.p;
  a.data = (uint8_t*)d->data.p;
  a.tile_keep = (int32_t*)d->tile_keep.p;
  a.tile_mark = (int32_t*)d->tile_mark.p;
  a.mpos = (uint32_t*)d->mpos.p;
  a.mcode = (uint8_t*)d->mcode.p;
  a.segs = (CJSegment*)d->segs.p;
  a.recs = (CJSubRec*)d->recs.p;
  a.ckpt = (CJCkpt*)d->ckpt.p;
  a.snap0 = (uint64_t*)d->snap.p;
  a.snap1 = a.snap0 + d->b_nwarps;
  a.wagg = (CJWarpAgg*)d->wagg.p;
  a.carry = (CJWarpAgg*)d->carry.p;
  a.coef = (int16_t*)d->coef.p;
  a.ctl = (CJBatchCtl*)d->bctl.p;
  a.n = 1;
  a.ntiles = d->b_ntiles;
  a.nwarps = d->b_nwarps;
  a.nptiles = d->b_nptiles;
  a.max_passes = d->b_nwarps + 2;
  a.nhyp = d->b_nhyp;
  a.hrecs = (CJSubRec*)d->hrecs.p;
  a.hckpt = (CJCkpt*)d->hckpt.p;
  a.hmap = (uint8_t*)d->hmap.p;
  cj_profile_begin(d);
  CJ_CUDA_TRY(cudaMemsetAsync(d->bctl.p, 0, sizeof(CJBatchCtl), s), CUDA_MEM_ERROR);
  void* args[] = {&a};
  CJ_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)bt_decode_kernel(d->b_ctas, d->b_nhyp > 1),
                                          dim3(d->b_grid),
                                          dim3(BT_THREADS), args, BT_DECODE_SMEM, s),
              CUDA_KERNEL_LAUNCH_ERROR);
  cj_after_launch(d, CJ_K_DECODE_BATCH);
  CJ_CUDA_TRY(cudaEventRecord(d->ev_scan, s), CUDA_KERNEL_LAUNCH_ERROR);
  CJ_CUDA_TRY(cudaMemcpyAsync(d->h_bctl.p, d->bctl.p, sizeof(CJBatchCtl), cudaMemcpyDeviceToHost, s),
              CUDA_MEM_ERROR);
  return 0;
}

int cj_reader_decode_status(const JPGReader* jpg) {
  const CJBatchCtl* ctl = (const CJBatchCtl*)jpg->dev->h_bctl.p;
  if (!ctl || jpg->dev->progressive) return 0;  // progressive scans have no grid barriers
  if (ctl->timeout) return CUDA_KERNEL_LAUNCH_ERROR;
  if (ctl->passes > jpg->dev->b_nwarps + 2) return PROGRAMMER_ERROR;
  return 0;
}

// ---------------------------------------------------------------- no-allocation decode
//
// cjDecodeNoAlloc: the batch kernel above run on one image whose every piece
// of working memory -- compressed bytes, destuffed bytes, tables, segments,
// subsequence records, coefficient blocks, status -- lives in one statically
// sized device array, so the call itself never allocates device (or host)
// memory.  The array is held by every GPU that loads the library until the
// process exits.

#define CJ_NOALLOC_SCRATCH_BYTES (24u << 20)  // 24 MiB per device
#define CJ_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) unsigned char g_noalloc_scratch[CJ_NOALLOC_SCRATCH_BYTES];
// Device address of the array per device, set once under g_noalloc_mu; the
// host-side symbol g_noalloc_scratch is not a device address.
static std::atomic<unsigned char*> g_noalloc_ptr[CJ_NOALLOC_MAX_DEVICES];
static std::mutex g_noalloc_mu;

static size_t bt_align(size_t x) { return (x + 255) & ~(size_t)255; }

// One-time set-up on device `dev` (current): the array's device address and
// the kernels' shared-memory attributes.  Host threads calling at once wait
// for the first; a failed set-up is retried by the next call.
static unsigned char* bt_noalloc_base(int dev) {
  unsigned char* p = g_noalloc_ptr[dev].load(std::memory_order_acquire);
  if (p) return p;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  p = g_noalloc_ptr[dev].load(std::memory_order_relaxed);
  if (p) return p;
  void* addr = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
  if (e != cudaSuccess || !addr) {
    cj_note_cuda_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
    return nullptr;
  }
  e = bt_pixel_attrs();
  if (e == cudaSuccess) e = bt_decode_attrs();
  if (e != cudaSuccess) {
    cj_note_cuda_error(e, "cjDecodeNoAlloc kernel attributes", __FILE__, __LINE__);
    return nullptr;
  }
  p = (unsigned char*)addr;
  g_noalloc_ptr[dev].store(p, std::memory_order_release);
  return p;
}

extern "C" int cjDecodeNoAlloc(const unsigned char* jpeg, size_t size, unsigned char* d_out,
                               size_t out_capacity, int* width, int* height, int* channels,
                               void* stream) {
  if (!jpeg || !d_out) return PROGRAMMER_ERROR;
  int dev = 0;
  CJ_CUDA_TRY(cudaGetDevice(&dev), CUDA_MEM_ERROR);
  if (dev < 0 || dev >= CJ_NOALLOC_MAX_DEVICES) return UNSUPPORTED_ERROR;
  unsigned char* base = bt_noalloc_base(dev);
  if (!base) return CUDA_MEM_ERROR;

  // host parse on the stack
  JPGReader r;
  memset(&r, 0, sizeof(r));
  CJReaderDevice rd;
  r.dev = &rd;
  int err = cj_parse_to_scan(&r, jpeg, size);
  if (err) return err;
  CJImageHeader h;
  CJImageDesc d;
  err = bt_fill_header(&r, &h);
  if (err) return err;
  int bpm = 0;
  for (int c = 0; c < h.nch; c++) bpm += h.comp_sx[c] * h.comp_sy[c];
  const int ch = h.nch == 3 ? 3 : 1;
  const size_t out_bytes = (size_t)h.width * h.height * ch;
  if (width) *width = h.width;
  if (height) *height = h.height;
  if (channels) *channels = ch;
  if (out_capacity < out_bytes) return PROGRAMMER_ERROR;
  const int64_t scan_off = (int64_t)(r.pos - jpeg), scan_len = (int64_t)(r.end - r.pos);
  if ((uint64_t)scan_len > CJ_MAX_SCAN_BYTES) return UNSUPPORTED_ERROR;

  // plan: one image, every buffer carved out of the static array.  One image
  // alone spreads over the whole GPU only with more, shorter subsequences
  // than a batch uses: the single-image paths' 1024 bits (as openJPG), with
  // the batch's full-width pixel tiles.
  bt_plan_one(h, scan_len, CJ_SUB_BITS_DEFAULT, &d);
  d.src_off = scan_off;
  const int nwarps = d.sub_cap / 32;
  size_t off = 0;
  auto carve = [&](size_t bytes) {
    size_t o = off;
    off = bt_align(off + bytes);
    return o;
  };
  const size_t o_hdr = carve(sizeof(CJImageHeader)), o_desc = carve(sizeof(CJImageDesc));
  const size_t o_prm = carve(sizeof(CJScanParams)), o_st = carve(sizeof(CJStatus));
  const size_t o_ctl = carve(sizeof(CJBatchCtl));
  const size_t o_blob = carve(size + 64), o_data = carve((size_t)scan_len + 64);
  const size_t o_tk = carve((size_t)d.ntiles * 4), o_tm = carve((size_t)d.ntiles * 4);
  const size_t o_mpos = carve((size_t)d.mark_cap * 4), o_mcode = carve((size_t)d.mark_cap);
  const size_t o_segs = carve((size_t)d.seg_cap * sizeof(CJSegment));
  const size_t o_recs = carve((size_t)d.sub_cap * sizeof(CJSubRec));
  const size_t o_ckpt = carve((size_t)d.sub_cap * CJ_CKPTS * sizeof(CJCkpt));
  const size_t o_snap = carve((size_t)2 * nwarps * sizeof(uint64_t));
  const size_t o_wagg = carve((size_t)nwarps * sizeof(CJWarpAgg));
  const size_t o_carry = carve((size_t)nwarps * sizeof(CJWarpAgg));
  const size_t o_coef = carve((size_t)h.total_blocks * 128 + 128);
  if (off > CJ_NOALLOC_SCRATCH_BYTES) {
    fprintf(stderr,
            "libcudajpeg: cjDecodeNoAlloc: this image needs %zu bytes of working memory; the "
            "static scratch holds %u (use openJPG or the batch decoder for larger images)\n",
            off, CJ_NOALLOC_SCRATCH_BYTES);
    return UNSUPPORTED_ERROR;
  }
  CJPixGeom g;
  g.nch = h.nch;
  g.bpm = bpm;
  g.hmax = h.hmax;
  g.vmax = h.vmax;
  g.T = d.T;
  const size_t smem_pix = cj_pix_layout(&g, h.comp_sx[1], h.comp_sy[1], 2);
  const size_t smem = BT_DECODE_SMEM;
  // every check that can fail before the GPU runs anything: launch shapes
  int sms = 0, per_dec = 0, per_pix = 0;
  const bt_decode_fn dk = bt_decode_kernel(BT_DECODE_CTAS_DEFAULT);
  CJ_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), CUDA_MEM_ERROR);
  CJ_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_dec, (const void*)dk, BT_THREADS, smem),
              CUDA_KERNEL_LAUNCH_ERROR);
  const bt_pixel_fn pk = bt_pixel_kernel(CJ_PIX_IDCT_INT, CJ_OUT_RGB);
  CJ_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_pix, (const void*)pk, CJ_PIX_THREADS, smem_pix),
              CUDA_KERNEL_LAUNCH_ERROR);
  if (per_dec < 1 || per_pix < 1) return UNSUPPORTED_ERROR;
  per_dec = std::min(per_dec, BT_DECODE_CTAS_DEFAULT);

  CJBatchArgs a{};
  a.hdr = (const CJImageHeader*)(base + o_hdr);
  a.desc = (const CJImageDesc*)(base + o_desc);
  a.prm = (CJScanParams*)(base + o_prm);
  a.st = (CJStatus*)(base + o_st);
  a.blob = base + o_blob;
  a.data = base + o_data;
  a.tile_keep = (int32_t*)(base + o_tk);
  a.tile_mark = (int32_t*)(base + o_tm);
  a.mpos = (uint32_t*)(base + o_mpos);
  a.mcode = base + o_mcode;
  a.segs = (CJSegment*)(base + o_segs);
  a.recs = (CJSubRec*)(base + o_recs);
  a.ckpt = (CJCkpt*)(base + o_ckpt);
  a.snap0 = (uint64_t*)(base + o_snap);
  a.snap1 = a.snap0 + nwarps;
  a.wagg = (CJWarpAgg*)(base + o_wagg);
  a.carry = (CJWarpAgg*)(base + o_carry);
  a.coef = (int16_t*)(base + o_coef);
  a.out = d_out;
  a.ctl = (CJBatchCtl*)(base + o_ctl);
  a.n = 1;
  a.ntiles = d.ntiles;
  a.nwarps = nwarps;
  a.nptiles = d.nptiles;
  a.max_passes = nwarps + 2;
  a.wait_limit = 0;

  // From the first queued copy on, every return waits for the stream: the
  // shared array must be idle when the call returns.
  cudaStream_t s = (cudaStream_t)stream;
  auto fail = [&](cudaError_t e, const char* what, int code) {
    cj_note_cuda_error(e, what, __FILE__, __LINE__);
    cudaStreamSynchronize(s);
    cudaGetLastError();
    return code;
  };
  cudaError_t e = cudaMemcpyAsync(base + o_hdr, &h, sizeof(h), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(base + o_desc, &d, sizeof(d), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(base + o_blob, jpeg, size, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(base + o_ctl, 0, sizeof(CJBatchCtl), s);
  if (e != cudaSuccess) return fail(e, "cjDecodeNoAlloc copies", CUDA_MEM_ERROR);
  void* args[] = {&a};
  e = cudaLaunchCooperativeKernel((const void*)dk, dim3(per_dec * sms), dim3(BT_THREADS), args, smem, s);
  if (e != cudaSuccess) return fail(e, "cjDecodeNoAlloc decode kernel", CUDA_KERNEL_LAUNCH_ERROR);
  pk<<<std::min(d.nptiles, per_pix * sms), CJ_PIX_THREADS, smem_pix, s>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(e, "cjDecodeNoAlloc pixel kernel", CUDA_KERNEL_LAUNCH_ERROR);
  CJStatus st;
  CJBatchCtl ctl;
  e = cudaMemcpyAsync(&st, base + o_st, sizeof(st), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&ctl, base + o_ctl, sizeof(ctl), cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return fail(e, "cjDecodeNoAlloc status copy", CUDA_MEM_ERROR);
  CJ_CUDA_TRY(cudaStreamSynchronize(s), CUDA_KERNEL_LAUNCH_ERROR);
  if (ctl.timeout) return CUDA_KERNEL_LAUNCH_ERROR;
  if (ctl.passes > nwarps + 2) return PROGRAMMER_ERROR;
  return cj_status_error(&st);
}
