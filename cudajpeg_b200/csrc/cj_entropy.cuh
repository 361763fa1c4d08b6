// cj_entropy.cuh -- device building blocks of the entropy decode in the
// persistent batch kernel (batch.cu): destuff classification, subsequence
// lanes, speculative block decode, the warp settle loop and the cooperative
// coefficient write-out.
#pragma once
#include <limits.h>
#include <stdint.h>

#include "cj_core.h"
#include "cj_scan_util.cuh"

// 16 stuffed bytes starting at `base`, their neighbours, and what to keep.
struct CJChunk {
  uint32_t w[4];    // the 16 bytes, little-endian words
  uint32_t keep;    // bit j: byte j is entropy data
  uint32_t mark;    // bit j: byte j is the FF of an RSTn marker
  uint32_t next;    // byte after the chunk (marker code of bit 15)
  bool bad;         // an FF followed by anything but 00 / D0-D7
};

__device__ __forceinline__ uint32_t cj_byte(const CJChunk& c, int j) {
  return (c.w[j >> 2] >> (8 * (j & 3))) & 0xFF;
}

// The memory a chunk is classified from: the two aligned 16-byte words
// around its 16 bytes and the one after them, and the byte before it.  For a
// chunk that starts inside the data (base < n) the words lie below
// raw + n + 31; the callers' buffers hold at least 31 bytes past the data and
// start on a 16-byte boundary.  Loaded apart from the classification so that
// a loop can fetch its next chunk early.
struct CJChunkIn {
  uint4 lo, hi;
  uint32_t sh;    // the chunk's offset inside lo
  uint32_t prev;  // the byte before the chunk (0 at the start)
};

__device__ __forceinline__ CJChunkIn cj_chunk_load(const uint8_t* raw, int64_t n, int64_t base) {
  CJChunkIn x;
  x.lo = x.hi = make_uint4(0, 0, 0, 0);
  x.sh = 0;
  if (base < n) {
    const uintptr_t addr = (uintptr_t)(raw + base);
    const uint4* q = reinterpret_cast<const uint4*>(addr & ~(uintptr_t)15);
    x.lo = q[0];
    x.hi = q[1];
    x.sh = (uint32_t)(addr & 15);
  }
  x.prev = (base > 0 && base - 1 < n) ? raw[base - 1] : 0;
  return x;
}

// Classify a loaded chunk: its bytes come out of the two words by funnel
// shifts, whatever its alignment; bytes at or past n read as 0.
__device__ __forceinline__ CJChunk cj_classify_in(const CJChunkIn& x, int64_t n, int64_t base) {
  CJChunk c;
  c.keep = c.mark = 0;
  c.bad = false;
  c.w[0] = c.w[1] = c.w[2] = c.w[3] = 0;
  c.next = 0;
  if (base < n) {
    const uint4 lo = x.lo, hi = x.hi;
    const uint32_t sh = x.sh, bs = (sh & 3) * 8;
    uint32_t a0, a1, a2, a3, a4, a5;
    switch (sh >> 2) {
      case 0: a0 = lo.x; a1 = lo.y; a2 = lo.z; a3 = lo.w; a4 = hi.x; a5 = hi.y; break;
      case 1: a0 = lo.y; a1 = lo.z; a2 = lo.w; a3 = hi.x; a4 = hi.y; a5 = hi.z; break;
      case 2: a0 = lo.z; a1 = lo.w; a2 = hi.x; a3 = hi.y; a4 = hi.z; a5 = hi.w; break;
      default: a0 = lo.w; a1 = hi.x; a2 = hi.y; a3 = hi.z; a4 = hi.w; a5 = 0; break;
    }
    c.w[0] = __funnelshift_r(a0, a1, bs);
    c.w[1] = __funnelshift_r(a1, a2, bs);
    c.w[2] = __funnelshift_r(a2, a3, bs);
    c.w[3] = __funnelshift_r(a3, a4, bs);
    // byte 16 of the chunk: byte 0 of the next word
    const uint32_t after = __funnelshift_r(a4, a5, bs) & 0xFF;
    c.next = (base + 16 < n) ? after : 0;
    if (base + 16 > n) {
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const int64_t valid = n - (base + 4 * k);  // bytes of word k below n
        if (valid <= 0) c.w[k] = 0;
        else if (valid < 4) c.w[k] &= (1u << (8 * valid)) - 1u;
      }
    }
  }
  uint32_t prev = x.prev;
#pragma unroll
  for (int j = 0; j < 16; j++) {
    if (base + j >= n) break;
    uint32_t b = cj_byte(c, j);
    uint32_t nx = (j < 15) ? cj_byte(c, j + 1) : c.next;
    bool has_next = base + j + 1 < n;
    if (prev == 0xFF && (base + j) > 0) {
      // second byte of an FF pair: stuffing or the RSTn code, never data
      if (b != 0x00 && (b & 0xF8) != 0xD0) c.bad = true;
    } else if (b == 0xFF) {
      if (has_next && nx == 0x00) c.keep |= 1u << j;
      else if (has_next && (nx & 0xF8) == 0xD0) c.mark |= 1u << j;
      else c.bad = true;
    } else {
      c.keep |= 1u << j;
    }
    prev = b;
  }
  return c;
}

struct CJLane {
  uint64_t begin, end;   // this subsequence's bits
  uint64_t end_byte;     // its segment's end (bytes)
  int seg;
  bool head, last, active;
};

__device__ __forceinline__ CJLane cj_lane(const CJSegment* segs, int nseg, int nsub, int i,
                                          int sub_bits) {
  CJLane l;
  l.active = i < nsub;
  l.begin = l.end = l.end_byte = 0;
  l.seg = 0;
  l.head = l.last = false;
  if (!l.active) return l;
  int lo = 0, hi = nseg - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (segs[mid].first_sub <= i) lo = mid;
    else hi = mid - 1;
  }
  const CJSegment& s = segs[lo];
  int j = i - s.first_sub;
  l.seg = lo;
  l.begin = s.bit_begin + (uint64_t)j * sub_bits;
  l.end = min(s.bit_end, l.begin + (uint64_t)sub_bits);
  if (l.begin > s.bit_end) l.begin = s.bit_end;
  l.end_byte = s.bit_end >> 3;
  l.head = (j == 0);
  l.last = (j == s.nsub - 1);
  return l;
}

// Bit reader of the decode loops: the current and the next big-endian word
// and a bit offset; a 32-bit window is one funnel shift, and a word boundary
// is crossed at most once per symbol (a symbol consumes at most 31 bits).
// One more word is loaded a crossing ahead and kept as read from memory
// (byte-swapped only when it becomes the next word), so a load has several
// symbols to arrive before the window needs it.
// Bytes at or past `end_byte` read as 0xFF (the padding the reference's bit
// reader supplies).
struct CJFBits {
  const uint32_t* words;
  uint32_t wfull, end_byte, cur, nxt, raw2, wi, off;

  __device__ __forceinline__ uint32_t word(uint32_t i) const {
    return i < wfull ? cj_bswap(words[i]) : cj_word(words, i, end_byte);
  }
  // word i as stored (cj_bswap of it is word(i))
  __device__ __forceinline__ uint32_t word_raw(uint32_t i) const {
    return i < wfull ? words[i] : cj_bswap(cj_word(words, i, end_byte));
  }
  __device__ __forceinline__ void init(const uint32_t* w, uint64_t eb, uint64_t p) {
    words = w;
    end_byte = (uint32_t)eb;
    wfull = (uint32_t)(eb >> 2);
    const uint32_t w0 = (uint32_t)(p >> 5);
    off = (uint32_t)(p & 31);
    cur = word(w0);
    wi = w0 + 1;
    nxt = word(wi);
    raw2 = word_raw(wi + 1);
  }
  __device__ __forceinline__ uint32_t peek() const { return __funnelshift_l(nxt, cur, off); }
  __device__ __forceinline__ void skip(uint32_t u) {
    off += u;
    if (off >= 32) {
      off -= 32;
      cur = nxt;
      nxt = cj_bswap(raw2);
      wi++;
      raw2 = word_raw(wi + 1);
    }
  }
  __device__ __forceinline__ uint64_t pos() const { return ((uint64_t)(wi - 1) << 5) + off; }
};

// Component, DC slot and AC slot of MCU phase m (from the packed phase
// table; the per-phase arrays for MCUs of more than 10 blocks).
__device__ __forceinline__ void cj_phase(const CJScanParams& sp, int bpm, uint64_t pack, uint32_t m, int& c,
                                         uint32_t& dslot, uint32_t& aslot) {
  if (bpm <= 10) {
    const uint32_t f = (uint32_t)(pack >> (6 * m)) & 63;
    c = (int)(f & 3);
    dslot = (f >> 2) & 3;
    aslot = f >> 4;
  } else {
    c = sp.phase_comp[m];
    dslot = sp.comp_dc[c];
    aslot = sp.comp_ac[c];
  }
}

// Checkpoints of a subsequence decode: the decoder state at the first block
// boundary at or after each of CJ_CKPTS thresholds (1/4, 1/2, 3/4 of the
// subsequence): position relative to the subsequence start and MCU phase
// (pp = phase << 24 | position), blocks begun before it, DC sums before it.
// Thresholds the decode never passes get its exit state.
#define CJ_CKPTS 3
struct CJCkpt {
  uint32_t pp;
  int32_t nb, d0, d1, d2;
};

// Speculative decode of one subsequence from `start`: blocks beginning
// before the subsequence's end, their DC sums, and the state after them.
// One Huffman symbol per iteration through the decode-step tables (CJSteps):
// bits consumed, zig-zag advance and magnitude size come from one lookup, so
// DC and AC symbols of all lanes take the same instructions; a block ends
// when the position passes 62 (EOB and invalid symbols advance by >= 64).
// The DC symbol's window is kept and its difference added when the block
// ends.  Symbol for symbol this is the serial T.81 block decode
// (src/decodeScanGPU.cu:78-100): a failing block is counted and
// decoding goes on after the bits the failing symbol consumed.
//
// Checkpoints (`ck`, CJ_CKPTS of them) are written for every decode.  A
// re-decode (RESUME) from a corrected start compares each checkpoint it
// reaches with the previous decode's (`old`): when position and phase agree
// the two decodes are identical from there on, so it stops and returns the
// previous totals shifted by the difference in blocks and DC sums before that
// point (shifting the later checkpoints too).  The result equals a full
// decode from `start`.
template <bool RESUME, bool HYP = false>
__device__ __forceinline__ CJSubRec cj_spec_decode(const CJScanParams& sp, const CJSteps& T,
                                                   const uint32_t* words, const CJLane& ln, uint64_t start,
                                                   CJCkpt* __restrict__ ck,
                                                   const CJSubRec& old, uint32_t cstep,
                                                   const CJCkpt* hck = nullptr, const CJSubRec* hrec = nullptr,
                                                   int nh = 0) {
  CJFBits br;
  br.init(words, ln.end_byte, cj_state_bit(start));
  uint32_t m = cj_state_phase(start);
  const int bpm = sp.bpm;
  const uint64_t pack = sp.phase_pack;
  int c;
  uint32_t aslot, slot;
  cj_phase(sp, bpm, pack, m, c, slot, aslot);
  int k = -1, nb = 0, d0 = 0, d1 = 0, d2 = 0;
  uint32_t dcv = 0, dcst = 0;
  const uint32_t endrel = (uint32_t)(ln.end - ln.begin);
  int rem = (int)((int64_t)ln.end - (int64_t)cj_state_bit(start));
  uint32_t j = 0, thresh = cstep;
  CJSubRec r;
  r.start = start;
  // Checkpoints at the boundary `rel` bits into the subsequence; true when
  // this decode has joined the previous one (r then holds the result).
  auto checkpoint = [&](uint32_t rel, bool final) -> bool {
    while (j < CJ_CKPTS && (final || rel >= thresh)) {
      const uint32_t pp = (m << 24) | rel;
      if (RESUME && !final) {
        // checkpoints may have been written by another SM in an earlier pass
        // of the same kernel: read them from L2, never a stale L1 line
        if (__ldcg(&ck[j].pp) == pp) {
          const int dn = nb - __ldcg(&ck[j].nb), e0 = d0 - __ldcg(&ck[j].d0), e1 = d1 - __ldcg(&ck[j].d1),
                    e2 = d2 - __ldcg(&ck[j].d2);
          for (uint32_t q = j; q < CJ_CKPTS; q++) {
            ck[q].nb = __ldcg(&ck[q].nb) + dn;
            ck[q].d0 = __ldcg(&ck[q].d0) + e0;
            ck[q].d1 = __ldcg(&ck[q].d1) + e1;
            ck[q].d2 = __ldcg(&ck[q].d2) + e2;
          }
          r.exit = old.exit;
          r.nblocks = old.nblocks + dn;
          r.dc[0] = old.dc[0] + e0;
          r.dc[1] = old.dc[1] + e1;
          r.dc[2] = old.dc[2] + e2;
          return true;
        }
        // the same test against the decodes of the subsequence from its
        // first bit under the other MCU phases (hypotheses): equal position
        // and phase at a block boundary mean the two decodes coincide from
        // there on, so this decode takes that path's totals and checkpoints
        for (int h = 0; HYP && h < nh; h++) {
          const CJCkpt* hc = hck + h * CJ_CKPTS;
          if (__ldcg(&hc[j].pp) != pp) continue;
          const int dn = nb - __ldcg(&hc[j].nb), e0 = d0 - __ldcg(&hc[j].d0), e1 = d1 - __ldcg(&hc[j].d1),
                    e2 = d2 - __ldcg(&hc[j].d2);
          for (uint32_t q = j; q < CJ_CKPTS; q++)
            ck[q] = CJCkpt{__ldcg(&hc[q].pp), __ldcg(&hc[q].nb) + dn, __ldcg(&hc[q].d0) + e0,
                           __ldcg(&hc[q].d1) + e1, __ldcg(&hc[q].d2) + e2};
          r.exit = __ldcg(&hrec[h].exit);
          r.nblocks = __ldcg(&hrec[h].nblocks) + dn;
          r.dc[0] = __ldcg(&hrec[h].dc[0]) + e0;
          r.dc[1] = __ldcg(&hrec[h].dc[1]) + e1;
          r.dc[2] = __ldcg(&hrec[h].dc[2]) + e2;
          return true;
        }
      }
      ck[j] = CJCkpt{pp, nb, d0, d1, d2};
      j++;
      thresh += cstep;
    }
    return false;
  };
  if (rem > 0) {
    if (checkpoint(endrel - (uint32_t)rem, false)) return r;
    for (;;) {
      const uint32_t v = br.peek();
      const uint32_t st = cj_step(T, sp, slot, v);
      const int kn = k + (int)((st >> 5) & 127);
      const uint32_t used = (st & 31) - (kn > 63 ? (st >> 12) : 0u);
      const bool isdc = k < 0;
      dcv = isdc ? v : dcv;
      dcst = isdc ? st : dcst;
      br.skip(used);
      rem -= (int)used;
      slot = aslot;
      if (kn >= 63) {
        const uint32_t size = dcst >> 12, len = (dcst & 31) - size;
        const int dd = size ? cj_extend((dcv << len) >> (32 - size), size) : 0;
        if (c == 0) d0 += dd;
        else if (c == 1) d1 += dd;
        else d2 += dd;
        k = -1;
        nb++;
        m = (m + 1 == (uint32_t)bpm) ? 0 : m + 1;
        cj_phase(sp, bpm, pack, m, c, slot, aslot);
        if (rem <= 0) break;
        const uint32_t rel = endrel - (uint32_t)rem;
        if (rel >= thresh && checkpoint(rel, false)) return r;
      } else {
        k = kn;
      }
    }
  }
  const uint64_t pend = br.pos();
  checkpoint((uint32_t)(pend - ln.begin), true);  // thresholds not reached: the exit
  r.exit = cj_state(pend, m);
  r.nblocks = nb;
  r.dc[0] = d0;
  r.dc[1] = d1;
  r.dc[2] = d2;
  return r;
}

// Checkpoints of global lane `i` and the threshold spacing of a subsequence.
__device__ __forceinline__ CJCkpt* cj_lane_ckpts(CJCkpt* base, int64_t i) { return base + i * CJ_CKPTS; }
__device__ __forceinline__ uint32_t cj_ckpt_step(int sub_bits) { return (uint32_t)sub_bits / (CJ_CKPTS + 1); }

// Re-decode lanes whose input state (lane 0: `lane0_in`; others: the exit of
// the previous lane) differs from the state they last decoded from, until no
// lane changes.  Lane l settles after at most l+1 re-decodes.
// HYP: hck / hrec / nh are the lane's hypothesis decodes (cj_spec_decode).
template <bool HYP = false>
__device__ __forceinline__ bool cj_warp_settle(const CJScanParams& sp, const CJSteps& T, const uint32_t* words,
                                               const CJLane& ln, CJSubRec& r, uint64_t lane0_in,
                                               CJCkpt* ck, uint32_t cstep, const CJCkpt* hck = nullptr,
                                               const CJSubRec* hrec = nullptr, int nh = 0) {
  int lane = threadIdx.x & 31;
  bool dirty = false;
  for (int it = 0; it < 34; it++) {
    uint64_t pred = __shfl_up_sync(CJ_FULL, r.exit, 1);
    uint64_t want = ln.head ? r.start : (lane == 0 ? lane0_in : pred);
    bool change = ln.active && want != r.start;
    if (!__any_sync(CJ_FULL, change)) break;
    if (change) {
      r = cj_spec_decode<true, HYP>(sp, T, words, ln, want, ck, r, cstep, hck, hrec, nh);
      dirty = true;
    }
  }
  return dirty;
}

// Errors are ordered by the block they occur in; the status keeps the first
// (stored complemented so an all-zero status means "no error").
__device__ __forceinline__ void cj_raise(CJStatus* st, int64_t block, int code) {
  unsigned long long key = ((unsigned long long)block << 8) | (unsigned)code;
  atomicMax(&st->err_key, ~key);
}

__device__ __forceinline__ void cj_raise_dec(CJStatus* st, int64_t block, int code) {
  unsigned long long key = ((unsigned long long)block << 8) | (unsigned)code;
  atomicMax(&st->dec_err_key, ~key);
}

// Segmented-sum operator over (head flag, sums).
struct CJAgg5 {
  int f, n, a, b, c;
};
__device__ __forceinline__ CJAgg5 cj_op(const CJAgg5& x, const CJAgg5& y) {
  CJAgg5 r;
  r.f = x.f | y.f;
  if (y.f) {
    r.n = y.n; r.a = y.a; r.b = y.b; r.c = y.c;
  } else {
    r.n = x.n + y.n; r.a = x.a + y.a; r.b = x.b + y.b; r.c = x.c + y.c;
  }
  return r;
}

// Segmented exclusive prefix, over the lanes of a warp, of each lane's blocks
// and DC sums: from the last segment head at or before the lane, plus the
// carry from earlier warps (cn, c0..c2) when the segment began before this warp.
__device__ __forceinline__ void cj_warp_prefix(const CJSubRec& r, const CJLane& ln, int cn, int c0,
                                               int c1, int c2, int64_t* blocks, int* d0, int* d1,
                                               int* d2) {
  const int lane = threadIdx.x & 31;
  // Segmented exclusive prefix of (blocks, DC sums) over the warp.
  int s0 = r.nblocks, s1 = r.dc[0], s2 = r.dc[1], s3 = r.dc[2];
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    int t0 = __shfl_up_sync(CJ_FULL, s0, d), t1 = __shfl_up_sync(CJ_FULL, s1, d);
    int t2 = __shfl_up_sync(CJ_FULL, s2, d), t3 = __shfl_up_sync(CJ_FULL, s3, d);
    if (lane >= d) {
      s0 += t0; s1 += t1; s2 += t2; s3 += t3;
    }
  }
  unsigned heads = __ballot_sync(CJ_FULL, ln.active && ln.head);
  unsigned mine = heads & ((2u << lane) - 1u);  // heads at or before this lane
  int a = mine ? 31 - __clz(mine) : 0;
  int src = a > 0 ? a - 1 : 0;
  int b0 = __shfl_sync(CJ_FULL, s0, src), b1 = __shfl_sync(CJ_FULL, s1, src);
  int b2 = __shfl_sync(CJ_FULL, s2, src), b3 = __shfl_sync(CJ_FULL, s3, src);
  if (a == 0) b0 = b1 = b2 = b3 = 0;
  int e0 = s0 - r.nblocks - b0, e1 = s1 - r.dc[0] - b1, e2 = s2 - r.dc[1] - b2,
      e3 = s3 - r.dc[2] - b3;
  if (!mine) {
    e0 += cn; e1 += c0; e2 += c1; e3 += c2;
  }
  *blocks = e0;
  *d0 = e1;
  *d1 = e2;
  *d2 = e3;
}

// Blocks lane `ln` writes from block `first`: to its block count, or to its
// segment's last block for the segment's last lane; clamped to the segment.
__device__ __forceinline__ int64_t cj_lane_write_end(const CJLane& ln, const CJSegment& seg, const CJSubRec& r,
                                                     int64_t first) {
  const int64_t bend = seg.first_block + seg.nblocks;
  const int64_t end = ln.last ? bend : first + r.nblocks;
  return end > bend ? bend : end;
}

// Warp-cooperative write-out of 32 units (one per lane; `active` = false for
// lanes without one), symbol for symbol the serial block decode with the
// same structural checks.  Each lane builds its current block in its own
// 64-entry int16 buffer in shared memory (`wbuf` + lane * 64, all zero on
// entry and on return).  After every symbol the warp stores the blocks its
// lanes completed in that step: 8 lanes per block, 4 blocks per round, one
// 16-byte store each -- a whole 128-byte line per block instead of one
// scattered 2-byte store per coefficient -- and clears those buffers.  Blocks
// go to memory whole, so the range needs no zero fill; a unit that stops at
// an error stores its partial block (as the serial decode leaves it) and zeroes
// the rest of its range, up to `zero_end`.
__device__ __forceinline__ void cj_write_units_warp(const CJScanParams& sp, const CJSteps& T, const uint32_t* words,
                                                    const CJLane& ln, const CJSegment& seg, uint64_t start,
                                                    int64_t first_block, int dc0, int dc1, int dc2,
                                                    int16_t* __restrict__ coef, CJStatus* st, const uint8_t* zz,
                                                    uint64_t stop, int64_t zero_end, bool active, int16_t* wbuf) {
  const int lane = threadIdx.x & 31;
  int16_t* mine = wbuf + lane * 64;
  int64_t b = first_block;
  const int64_t bend = seg.first_block + seg.nblocks;
  const uint64_t seg_end = seg.bit_end;
  const int bpm = sp.bpm;
  const uint64_t pack = sp.phase_pack;
  CJFBits br;
  uint32_t m = 0, aslot = 0, slot = 0;
  int c = 0;
  if (active) {
    br.init(words, ln.end_byte, cj_state_bit(start));
    m = cj_state_phase(start);
    cj_phase(sp, bpm, pack, m, c, slot, aslot);
  }
  int k = -1;
  int32_t dd = 0;
  bool cut = false;  // stopped inside block b at an error
  // the structural checks made before every block; false = stop here
  auto block_start = [&]() -> bool {
    const uint64_t p = br.pos();
    if (p >= stop) return false;  // the next unit's first block
    if (!ln.last && p >= ln.end) return false;
    if (b >= bend) {
      if (!ln.last) cj_raise_dec(st, b, CJ_DEV_EXTRA);
      else if (seg.marker_follows) {
        if (((p + 7) >> 3) != ln.end_byte) cj_raise_dec(st, b, CJ_DEV_TRAILING);
      } else if (ln.end_byte > ((p + 7) >> 3) + 2) {
        cj_raise_dec(st, b, CJ_DEV_TRAILING);
      }
      return false;
    }
    if (seg.marker_follows && p >= seg_end) {
      cj_raise_dec(st, b, CJ_DEV_OVERRUN);
      return false;
    }
    return true;
  };
  bool run = active && block_start();
  for (;;) {
    int done = -1;  // block (of this image) to store after this step
    if (run) {
      const uint32_t v = br.peek();
      const uint32_t stp = cj_step(T, sp, slot, v);
      const uint32_t dk = (stp >> 5) & 127, size = stp >> 12, total = stp & 31;
      const int kn = k + (int)dk;
      const uint32_t len = total - size;
      const int32_t val = size ? cj_extend((v << len) >> (32 - size), size) : 0;
      if (k < 0) dd = val;
      else if (size && kn <= 63) mine[zz[kn]] = (int16_t)val;
      br.skip(total - (kn > 63 ? size : 0u));
      slot = aslot;
      if (kn < 63) {
        k = kn;
      } else if (kn > 63 && dk != CJ_STEP_EOB) {  // failing symbol: the block is cut here
        cj_raise_dec(st, b, dk == CJ_STEP_NO_CODE ? CJ_DEV_BAD_CODE : CJ_DEV_BAD_AC);
        done = (int)b;
        cut = true;
        run = false;
      } else if (seg.marker_follows && br.pos() > seg_end) {
        cj_raise_dec(st, b, CJ_DEV_OVERRUN);
        done = (int)b;
        cut = true;
        run = false;
      } else {
        int dcv;
        if (c == 0) dcv = dc0 += dd;
        else if (c == 1) dcv = dc1 += dd;
        else dcv = dc2 += dd;
        if (dcv < -32768 || dcv > 32767) {
          cj_raise_dec(st, b, CJ_DEV_DC_RANGE);
          cut = true;
          run = false;
        } else {
          mine[0] = (int16_t)dcv;
          b++;
          m = (m + 1 == (uint32_t)bpm) ? 0 : m + 1;
          cj_phase(sp, bpm, pack, m, c, slot, aslot);
          k = -1;
          run = block_start();
        }
        done = (int)(cut ? b : b - 1);
      }
    }
    unsigned mask = __ballot_sync(CJ_FULL, done >= 0);
    __syncwarp();
    while (mask) {  // warp-uniform: up to 4 blocks per round, lanes 8j..8j+7 take the j-th
      const int s0 = __ffs(mask) - 1;
      mask &= mask - 1;
      const int s1 = __ffs(mask) - 1;
      mask &= mask - 1;
      const int s2 = __ffs(mask) - 1;
      mask &= mask - 1;
      const int s3 = __ffs(mask) - 1;
      mask &= mask - 1;
      const int j = lane >> 3;
      const int src = j == 0 ? s0 : (j == 1 ? s1 : (j == 2 ? s2 : s3));
      const int bsrc = __shfl_sync(CJ_FULL, done, src < 0 ? 0 : src);
      if (src >= 0) {
        uint4* s = reinterpret_cast<uint4*>(wbuf + src * 64) + (lane & 7);
        reinterpret_cast<uint4*>(coef + (int64_t)bsrc * 64)[lane & 7] = *s;
        *s = make_uint4(0, 0, 0, 0);
      }
    }
    __syncwarp();
    if (!__any_sync(CJ_FULL, run)) break;
  }
  // blocks of the range an early stop left undecoded read as zeros
  for (int64_t x = cut ? b + 1 : b; active && x < zero_end; x++) {
    uint4* p = reinterpret_cast<uint4*>(coef + x * 64);
#pragma unroll
    for (int i = 0; i < 8; i++) p[i] = make_uint4(0, 0, 0, 0);
  }
}
