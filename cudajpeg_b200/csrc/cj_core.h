// cj_core.h -- data layouts, Huffman tables and decode steps shared by the
// entropy kernels.  Everything here is plain C++ marked __host__ __device__
// so the same code is compiled for sm_100a kernels and for host checks of
// the table builder.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define CJ_HD __host__ __device__ __forceinline__
#else
#define CJ_HD inline
#endif

// ---------------------------------------------------------------- limits
#define CJ_FAST_BITS 10          // first-level Huffman lookup width
#define CJ_MAX_BPM 32            // blocks per MCU (the standard allows 10)
#define CJ_SUB_BITS_DEFAULT 1024 // bits per speculative subsequence
#define CJ_MAX_SCAN_BYTES (256u << 20) // block / bit counters are 32-bit

// Device error codes (the reader maps them to the format.h codes)
#define CJ_DEV_OK 0
#define CJ_DEV_BAD_CODE 1        // Huffman prefix with no code (SYNTAX_ERROR)
#define CJ_DEV_BAD_AC 2          // zero-size AC symbol that is not EOB/ZRL, or run past 63
#define CJ_DEV_OVERRUN 3         // restart interval needs bits past its marker
#define CJ_DEV_TRAILING 4        // restart interval has whole bytes after its last MCU
#define CJ_DEV_MARKER 5          // bad / missing / misplaced RSTn, or other marker in scan
#define CJ_DEV_DC_RANGE 6        // DC predictor outside int16 (UNSUPPORTED_ERROR)
#define CJ_DEV_EXTRA 7           // more entropy data than MCUs
#define CJ_DEV_CAPACITY 8        // more markers / subsequences than buffers allow

// One Huffman table in canonical form.
//   fast[w >> (16 - CJ_FAST_BITS)] = (len << 8) | symbol for codes of length
//   <= CJ_FAST_BITS, else 0; longer codes are found through maxcode/valoff
//   exactly as in ITU T.81 Annex F.2.2.3 (DECODE procedure).
struct CJHuff {
  uint16_t fast[1 << CJ_FAST_BITS];
  int32_t maxcode[18];  // [l], l = 1..16: largest code of length l, -1 if none
  int32_t valoff[18];   // symbol index of code c of length l = valoff[l] + c
  uint8_t vals[256];
};

// Decode steps: the per-symbol work of the entropy decoder, tabulated.
// Entry for a Huffman table slot and the next 10 bits of the stream:
//   bits 0-4   bits the symbol consumes: code length + magnitude size
//   bits 5-11  advance of the zig-zag position: DC 1 (from -1 to 0), AC
//              run + 1, ZRL 16, EOB 64, invalid AC symbol 96, no code 97
//   bits 12-15 magnitude size (extra bits that carry the value)
// An entry consuming 0 bits is a pointer: bits 5-15 index a 64-entry
// subtable for the following 6 bits (codes of 11-16 bits), or are
// CJ_STEP_SEARCH when the table has more long-code prefixes than subtables
// (the canonical search then decodes the code).  Long codes of a canonical
// table are the last codes of the code space, so their 10-bit prefixes form
// one contiguous range [pmin, pmax]: subtable i serves prefix pmin + i.
#define CJ_STEP_SUBS 16
#define CJ_STEP_SEARCH 0x7FFu
#define CJ_STEP_EOB 64u
#define CJ_STEP_BAD_AC 96u
#define CJ_STEP_NO_CODE 97u
#define CJ_STEP_BAD (1u | (CJ_STEP_NO_CODE << 5))  // consume 1 bit, end the block
struct CJSteps {
  uint16_t pri[4][1 << CJ_FAST_BITS];
  uint16_t sub[4][CJ_STEP_SUBS][64];
};

// Per-scan parameters, built on the host after SOS and copied once.
struct alignas(16) CJScanParams {
  CJHuff huff[4];                 // DC0, DC1, AC0, AC1
  CJSteps steps;                  // the same four tables as decode steps
  int16_t qnat[4][64];            // quantisation tables, natural order
  uint8_t phase_comp[CJ_MAX_BPM]; // component of the k-th block of an MCU
  uint8_t phase_blk[CJ_MAX_BPM];  // index of that block inside its component's MCU part
  uint8_t comp_dc[3], comp_ac[3], comp_q[3];
  uint8_t comp_sx[3], comp_sy[3];
  uint8_t pad0;
  uint8_t zz[64];                 // natural-order index of zig-zag position k
  int32_t nch, bpm, mcux, mcuy;
  int32_t width, height;
  int32_t hmax, vmax, xshift, yshift; // chroma upsample shifts
  int32_t restart_interval;          // MCUs, 0 = none
  int32_t nseg_expected;             // restart intervals in the scan
  int64_t total_blocks;              // mcux*mcuy*bpm
  int32_t comp_stride[3];            // plane strides (bytes) for plane outputs
  int32_t comp_rows[3];
  // phases 0..bpm-1 of an MCU, 6 bits each: component | DC slot << 2 |
  // AC slot << 4 (valid when bpm <= 10, the standard's limit)
  uint64_t phase_pack;
};

// Component and DC / AC table slots of MCU phase m.
CJ_HD uint64_t cj_phase_pack(const CJScanParams& p) {
  uint64_t pack = 0;
  for (int m = 0; m < p.bpm && m < 10; m++) {
    const int c = p.phase_comp[m];
    pack |= (uint64_t)(c | (p.comp_dc[c] << 2) | (p.comp_ac[c] << 4)) << (6 * m);
  }
  return pack;
}

// A restart interval (or the whole scan) in the destuffed buffer.
struct CJSegment {
  uint64_t bit_begin, bit_end;   // bits in the destuffed buffer
  int64_t first_block;           // global block index of its first block
  int64_t nblocks;               // blocks it must contain
  int32_t first_sub, nsub;       // its subsequences
  int32_t marker_follows;        // an RSTn ends it: its data must end on that
                                 // byte; otherwise reads past the end give 1-bits
  int32_t pad;
};

// Decoder state at a block boundary: bit position and MCU phase.
CJ_HD uint64_t cj_state(uint64_t bit, uint32_t phase) { return (bit << 8) | phase; }
CJ_HD uint64_t cj_state_bit(uint64_t s) { return s >> 8; }
CJ_HD uint32_t cj_state_phase(uint64_t s) { return (uint32_t)(s & 0xFF); }

// One speculative subsequence: where its decode started, where it left off,
// how many blocks it began and the sum of its DC differences per component.
struct alignas(16) CJSubRec {
  uint64_t start;
  uint64_t exit;
  int32_t nblocks;
  int32_t dc[3];
};

// Per-warp aggregate used by the segmented block/DC scan.
struct alignas(16) CJWarpAgg {
  int32_t has_head;  // a segment starts inside this warp
  int32_t nblocks;   // sums over the lanes after the last segment head
  int32_t dc[3];
  int32_t pad[3];
};

// Status words the host reads back after a decode.
struct CJStatus {
  unsigned long long err_key;     // destuff / segment errors: complemented
                                  // min of (block << 8 | CJ_DEV_*), 0 = none
  unsigned long long dec_err_key; // errors of the coefficient write-out and
                                  // pixel passes (same encoding); cleared when
                                  // those passes are re-run
  int32_t unstable;           // warps whose last exit changed in the last fix-up pass
  int32_t nmarkers;           // RSTn markers found by the destuffer
  int32_t nsub;               // subsequences in use
  int32_t nseg;               // restart intervals in use
  int64_t destuffed;          // bytes after destuffing
};
#define CJ_NO_ERROR_KEY 0xFFFFFFFFFFFFFFFFull

// ---------------------------------------------------------------- bit access
CJ_HD uint32_t cj_bswap(uint32_t v) {
#ifdef __CUDA_ARCH__
  return __byte_perm(v, 0, 0x0123);
#else
  return __builtin_bswap32(v);
#endif
}

// 32-bit big-endian word `w` of the destuffed buffer; bytes at or past
// `end_byte` read as 0xFF (the padding the reference's bit reader supplies).
CJ_HD uint32_t cj_word(const uint32_t* words, uint64_t w, uint64_t end_byte) {
  uint64_t first = w * 4;
  if (first >= end_byte) return 0xFFFFFFFFu;
  uint32_t v = cj_bswap(words[w]);
  uint64_t last = first + 4;
  if (last > end_byte) v |= (1u << (8 * (uint32_t)(last - end_byte))) - 1u;
  return v;
}

// Decode one Huffman code from a left-aligned 16-bit window.  Returns
// (len << 8) | symbol, or 0 when no code of length 1..16 matches.
// Codes longer than CJ_FAST_BITS: canonical search by length.
CJ_HD uint32_t cj_huff_slow(const CJHuff& t, uint32_t win16) {
  for (int l = CJ_FAST_BITS + 1; l <= 16; l++) {
    int32_t code = (int32_t)(win16 >> (16 - l));
    if (code <= t.maxcode[l]) return ((uint32_t)l << 8) | t.vals[(t.valoff[l] + code) & 255];
  }
  return 0;
}

CJ_HD uint32_t cj_huff_decode(const CJHuff& t, uint32_t win16) {
  uint32_t e = t.fast[win16 >> (16 - CJ_FAST_BITS)];
  if (e) return e;
  return cj_huff_slow(t, win16);
}

// Decode step of a decoded (len << 8 | symbol) from a DC (ac = false) or AC table.
CJ_HD uint32_t cj_step_of(uint32_t e, bool ac) {
  if (!e) return CJ_STEP_BAD;
  const uint32_t len = e >> 8, sym = e & 255, size = sym & 15, run = sym >> 4;
  const uint32_t dk = !ac ? 1u : (size ? run + 1 : (sym == 0 ? CJ_STEP_EOB : (sym == 0xF0 ? 16u : CJ_STEP_BAD_AC)));
  return (len + size) | (dk << 5) | (size << 12);
}

// 10-bit prefixes of the codes longer than 10 bits, from the DHT counts
// (canonical assignment, T.81 Annex C); *pmin > *pmax when there are none.
CJ_HD void cj_long_prefixes(const uint8_t counts[16], int* pmin, int* pmax) {
  int code = 0;
  *pmin = 1 << CJ_FAST_BITS;
  *pmax = -1;
  for (int l = 1; l <= 16; l++) {
    const int n = counts[l - 1];
    if (l > CJ_FAST_BITS && n) {
      const int a = code >> (l - CJ_FAST_BITS), b = (code + n - 1) >> (l - CJ_FAST_BITS);
      if (a < *pmin) *pmin = a;
      if (b > *pmax) *pmax = b;
    }
    code = (code + n) << 1;
  }
}

// Primary step entry for prefix p of table t (its fast table already built).
CJ_HD uint16_t cj_step_primary(const CJHuff& t, int pmin, int pmax, int p, bool ac) {
  const uint32_t e = t.fast[p];
  if (e) return (uint16_t)cj_step_of(e, ac);
  if (p < pmin || p > pmax) return (uint16_t)CJ_STEP_BAD;
  const uint32_t i = (uint32_t)(p - pmin);
  return (uint16_t)((i < CJ_STEP_SUBS ? i : CJ_STEP_SEARCH) << 5);
}

// Entry j of subtable s (prefix pmin + s) of table t.
CJ_HD uint16_t cj_step_sub(const CJHuff& t, int pmin, int s, int j, bool ac) {
  const uint32_t win = ((uint32_t)(pmin + s) << 6) | (uint32_t)j;
  if (pmin + s >= (1 << CJ_FAST_BITS)) return (uint16_t)CJ_STEP_BAD;
  return (uint16_t)cj_step_of(cj_huff_slow(t, win), ac);
}

// The decode step for the 32-bit window v (MSB = next bit) of table `slot`,
// from step tables `T` (sp.steps or a copy of them, e.g. in shared memory).
CJ_HD uint32_t cj_step(const CJSteps& T, const CJScanParams& sp, uint32_t slot, uint32_t v) {
  uint32_t st = T.pri[slot][v >> (32 - CJ_FAST_BITS)];
  if (!(st & 31)) {
    const uint32_t i = st >> 5;
    st = i != CJ_STEP_SEARCH ? T.sub[slot][i][(v >> 16) & 63]
                             : cj_step_of(cj_huff_slow(sp.huff[slot], v >> 16), slot >= 2);
  }
  return st;
}
CJ_HD uint32_t cj_step(const CJScanParams& sp, uint32_t slot, uint32_t v) { return cj_step(sp.steps, sp, slot, v); }


// Sign extension of a `size`-bit magnitude category value (T.81 F.2.2.1).
CJ_HD int32_t cj_extend(uint32_t bits, uint32_t size) {
  return (bits < (1u << (size - 1))) ? (int32_t)bits - (int32_t)(1u << size) + 1 : (int32_t)bits;
}

// Natural-order index of zig-zag position k (T.81 figure A.6).
#define CJ_ZIGZAG_INIT                                                                  \
  {0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,  12, 19, 26, 33, 40, 48, \
   41, 34, 27, 20, 13, 6,  7,  14, 21, 28, 35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, \
   30, 37, 44, 51, 58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63}
