/*
 * jpeg_oracle.c -- CPU restatement of the reference baseline-JPEG decode path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA decoder in
 * cudajpeg_b200/: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline may load it.  Nothing in the product links against it.
 *
 * It restates, in plain single-threaded C, the algorithm of the reference
 * (jndean/CUDAjpeg) for the path it accelerates:
 *   - container / marker loop ........ src/format.cu:113-215
 *   - SOF / DHT / DQT / DRI parsing ... src/format.cu:242-442
 *   - SOS header + table remap ....... src/decodeScanGPU.cu:104-144
 *   - byte unstuffing ................. src/decodeScanGPU.cu:11-24
 *   - bit reader + Huffman decode ..... src/decodeScanGPU.cu:28-100
 *   - scan loop incl. restart markers . src/decodeScanGPU.cu:435-490
 *   - integer iDCT (row / column) ..... CPUonly/src/pixelTransformCPU.c:14-107
 *   - nearest upsample + YCbCr->RGB ... CPUonly/src/pixelTransformCPU.c:110-172
 * and adds an FP64 separable iDCT used to measure iDCT error.  Beyond the
 * reference (which rejects both, src/format.cu:191-200 and :432) it also
 * decodes progressive frames (SOF2, ITU T.81 Annex G) and 16-bit
 * quantisation tables (Pq = 1): the checker of the decoder's extensions,
 * pinned by files whose baseline twin (the same coefficients written as one
 * baseline scan) the reference decodes.
 *
 * Parity is pinned against the reference itself: oracle/Makefile compiles the
 * reference's own sources into oracle/_ref/, and tests/golden/ holds vectors
 * produced by that build (tests/golden/make_golden.py).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OR_NO_ERROR 0
#define OR_SYNTAX_ERROR 1
#define OR_UNSUPPORTED_ERROR 2
#define OR_OOM_ERROR 3
#define OR_FILE_ERROR 5

/* Natural-order index of each zig-zag position (ITU T.81 figure A.6). */
static const uint8_t kZigZagToNatural[64] = {
    0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,
    12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6,  7,  14, 21, 28,
    35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
    58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

typedef struct {
  uint8_t sym; /* run/size byte (AC) or size category (DC) */
  uint8_t len; /* code length, 0 = no code has this 16-bit prefix */
} OracleVlc;

typedef struct {
  int id, sx, sy, dq_id, dc_id, ac_id;
  int width, height, stride, rows; /* plane geometry, padded to whole MCUs */
  int dc_pred;
  int nblocks;
  int32_t *coef; /* dequantised, natural order, 64 per block, scan order */
  int32_t *coef_pos;
  int32_t *qcoef; /* progressive frames: quantised values built up scan by scan */
  uint8_t *plane; /* stride x rows */
} OracleComp;

typedef struct {
  uint8_t *buf; /* private copy of the file; unstuffing rewrites it */
  size_t size;
  uint8_t *pos, *end;
  uint32_t bits;
  int nbits;
  int width, height, nch, mcux, mcuy, hmax, vmax;
  int restart_interval;
  OracleComp comp[3];
  OracleVlc *vlc[4]; /* DC0, DC1, AC0, AC1 (table_id = (Tc<<1 | Th)) */
  uint16_t dq[4][64]; /* zig-zag order, as stored in the DQT segment */
  int progressive;    /* SOF2 */
  int eobrun;         /* progressive AC scans: blocks left in the current end-of-band run */
  uint8_t *pixels; /* RGB W*H*3, or grey W*H */
  int error;
  int scan_done;
} OracleImage;

static unsigned read16(const uint8_t *p) { return ((unsigned)p[0] << 8) | p[1]; }

/* ---------------- marker segments (src/format.cu:237-442) ---------------- */

static void skip_segment(OracleImage *im) { im->pos += read16(im->pos); }

static void parse_sof(OracleImage *im) {
  /* src/format.cu:242-354 */
  uint8_t *seg = im->pos;
  unsigned len = read16(seg);
  if (len < 9 || seg + len >= im->end) { im->error = OR_SYNTAX_ERROR; return; }
  if (seg[2] != 8) { im->error = OR_UNSUPPORTED_ERROR; return; }
  im->height = read16(seg + 3);
  im->width = read16(seg + 5);
  if (!im->width || !im->height) { im->error = OR_SYNTAX_ERROR; return; }
  im->nch = seg[7];
  if (im->nch != 1 && im->nch != 3) { im->error = OR_UNSUPPORTED_ERROR; return; }
  if (len < 8u + 3u * im->nch) { im->error = OR_SYNTAX_ERROR; return; }
  int hmax = 0, vmax = 0;
  for (int c = 0; c < im->nch; c++) {
    const uint8_t *d = seg + 8 + 3 * c;
    OracleComp *k = &im->comp[c];
    k->id = d[0];
    k->sx = d[1] >> 4;
    k->sy = d[1] & 15;
    k->dq_id = d[2];
    if (!k->sx || !k->sy || k->dq_id > 3) { im->error = OR_SYNTAX_ERROR; return; }
    if ((k->sx & (k->sx - 1)) || (k->sy & (k->sy - 1))) {
      im->error = OR_UNSUPPORTED_ERROR;
      return;
    }
    if (k->sx > hmax) hmax = k->sx;
    if (k->sy > vmax) vmax = k->sy;
  }
  if (im->nch == 1) { im->comp[0].sx = im->comp[0].sy = hmax = vmax = 1; }
  im->hmax = hmax;
  im->vmax = vmax;
  im->mcux = (im->width + 8 * hmax - 1) / (8 * hmax);
  im->mcuy = (im->height + 8 * vmax - 1) / (8 * vmax);
  for (int c = 0; c < im->nch; c++) {
    OracleComp *k = &im->comp[c];
    k->width = (im->width * k->sx + hmax - 1) / hmax;
    k->height = (im->height * k->sy + vmax - 1) / vmax;
    k->stride = im->mcux * k->sx * 8;
    k->rows = im->mcuy * k->sy * 8;
    k->dc_pred = 0;
    if ((k->width < 3 && k->sx != hmax) || (k->height < 3 && k->sy != vmax)) {
      im->error = OR_UNSUPPORTED_ERROR;
      return;
    }
    k->nblocks = im->mcux * k->sx * im->mcuy * k->sy;
    free(k->coef);
    free(k->plane);
    k->coef = (int32_t *)calloc((size_t)k->nblocks * 64, sizeof(int32_t));
    k->plane = (uint8_t *)malloc((size_t)k->stride * k->rows);
    if (!k->coef || !k->plane) { im->error = OR_OOM_ERROR; return; }
    free(k->qcoef);
    k->qcoef = NULL;
    if (im->progressive) {
      k->qcoef = (int32_t *)calloc((size_t)k->nblocks * 64, sizeof(int32_t));
      if (!k->qcoef) { im->error = OR_OOM_ERROR; return; }
    }
    k->coef_pos = k->coef;
  }
  if (im->nch == 3) {
    if (im->comp[1].width != im->comp[2].width ||
        im->comp[1].height != im->comp[2].height ||
        im->comp[0].width != im->width || im->comp[0].height != im->height) {
      im->error = OR_UNSUPPORTED_ERROR;
      return;
    }
  }
  im->pos += len;
}

static void parse_dht(OracleImage *im) {
  /* src/format.cu:357-400: canonical codes expanded into a 16-bit table */
  uint8_t *p = im->pos;
  uint8_t *seg_end = p + read16(p);
  if (seg_end > im->end) { im->error = OR_SYNTAX_ERROR; return; }
  p += 2;
  while (p < seg_end) {
    uint8_t tc_th = p[0];
    if (tc_th & 0xEC) { im->error = OR_SYNTAX_ERROR; return; }
    if (tc_th & 0x02) { im->error = OR_UNSUPPORTED_ERROR; return; }
    int slot = (tc_th | (tc_th >> 3)) & 3;
    if (!im->vlc[slot]) {
      im->vlc[slot] = (OracleVlc *)calloc(65536, sizeof(OracleVlc));
      if (!im->vlc[slot]) { im->error = OR_OOM_ERROR; return; }
    }
    OracleVlc *t = im->vlc[slot];
    const uint8_t *sym = p + 17;
    int left = 65536; /* table entries not yet owned by a code */
    int fill = 0;
    for (int l = 1; l <= 16; l++) {
      int n = p[l];
      if (!n) continue;
      if (sym + n > seg_end) { im->error = OR_SYNTAX_ERROR; return; }
      int span = 1 << (16 - l);
      left -= n * span;
      if (left < 0) { im->error = OR_SYNTAX_ERROR; return; }
      for (int i = 0; i < n; i++, sym++)
        for (int j = 0; j < span; j++, fill++) {
          t[fill].len = (uint8_t)l;
          t[fill].sym = *sym;
        }
    }
    for (; fill < 65536; fill++) t[fill].len = 0;
    p = (uint8_t *)sym;
  }
  if (p != seg_end) { im->error = OR_SYNTAX_ERROR; return; }
  im->pos = seg_end;
}

static void parse_dqt(OracleImage *im) {
  /* src/format.cu:424-442 for 8-bit tables; 16-bit tables (Pq = 1, T.81
   * B.2.4.1: 64 big-endian values), which the reference rejects, are read
   * too -- their values must stay below 2^15 */
  uint8_t *seg_end = im->pos + read16(im->pos);
  if (seg_end > im->end) { im->error = OR_SYNTAX_ERROR; return; }
  uint8_t *p = im->pos + 2;
  while (p < seg_end) {
    const int pq = p[0] >> 4, id = p[0] & 15;
    const int n = pq ? 129 : 65;
    if (pq > 1 || id > 3 || p + n > seg_end) { im->error = OR_SYNTAX_ERROR; return; }
    for (int k = 0; k < 64; k++) {
      const unsigned v = pq ? read16(p + 1 + 2 * k) : p[1 + k];
      if (v > 32767) { im->error = OR_UNSUPPORTED_ERROR; return; }
      im->dq[id][k] = (uint16_t)v;
    }
    p += n;
  }
  if (p != seg_end) { im->error = OR_SYNTAX_ERROR; return; }
  im->pos = seg_end;
}

static void parse_dri(OracleImage *im) {
  /* src/format.cu:404-421 */
  unsigned len = read16(im->pos);
  uint8_t *seg_end = im->pos + len;
  if (len < 2 || seg_end > im->end) { im->error = OR_SYNTAX_ERROR; return; }
  im->restart_interval = read16(im->pos + 2);
  im->pos = seg_end;
}

/* ---------------- entropy-coded segment (src/decodeScanGPU.cu) ---------------- */

static void unstuff(OracleImage *im) {
  /* src/decodeScanGPU.cu:11-24: drop the 00 after FF, keep FF Dn, drop other
   * bytes that follow an FF; then terminate the data with FF D9. */
  uint8_t *src = im->pos, *dst = im->pos;
  while (src < im->end) {
    uint8_t b = *src++;
    *dst++ = b;
    if (b != 0xFF) continue;
    uint8_t nxt = *src++;
    if (nxt == 0x00) continue;
    if ((nxt & 0xF8) == 0xD0) *dst++ = nxt;
  }
  im->end = dst;
  dst[0] = 0xFF;
  dst[1] = 0xD9;
}

static int show_bits(OracleImage *im, int n) {
  /* src/decodeScanGPU.cu:28-37: reads past the end return 1-bits */
  if (!n) return 0;
  while (im->nbits < n) {
    uint8_t b = (im->pos >= im->end) ? 0xFF : *im->pos++;
    im->bits = (im->bits << 8) | b;
    im->nbits += 8;
  }
  return (int)((im->bits >> (im->nbits - n)) & ((1u << n) - 1));
}

static int get_bits(OracleImage *im, int n) {
  int v = show_bits(im, n);
  im->nbits -= n;
  return v;
}

static int get_vlc(OracleImage *im, const OracleVlc *t, uint8_t *sym_out) {
  /* src/decodeScanGPU.cu:50-75 */
  OracleVlc e = t[show_bits(im, 16)];
  if (!e.len) { im->error = OR_SYNTAX_ERROR; return 0; }
  im->nbits -= e.len;
  if (sym_out) *sym_out = e.sym;
  int size = e.sym & 15;
  if (!size) return 0;
  int v = get_bits(im, size);
  if (v < (1 << (size - 1))) v += (-1 << size) + 1;
  return v;
}

static void decode_block(OracleImage *im, OracleComp *k) {
  /* src/decodeScanGPU.cu:78-100 */
  uint8_t sym = 0;
  int32_t *blk = k->coef_pos;
  const uint16_t *q = im->dq[k->dq_id];
  k->dc_pred += get_vlc(im, im->vlc[k->dc_id], NULL);
  blk[0] = k->dc_pred * q[0];
  int z = 0;
  do {
    int v = get_vlc(im, im->vlc[k->ac_id], &sym);
    if (!sym) break; /* EOB */
    if (!(sym & 15) && sym != 0xF0) { im->error = OR_SYNTAX_ERROR; return; }
    z += (sym >> 4) + 1;
    if (z > 63) { im->error = OR_SYNTAX_ERROR; return; }
    blk[kZigZagToNatural[z]] = v * q[z];
  } while (z < 63);
  k->coef_pos += 64;
}

static void decode_scan(OracleImage *im) {
  /* SOS header: src/decodeScanGPU.cu:124-144 */
  uint8_t *p = im->pos;
  unsigned hlen = read16(p);
  if (p + hlen > im->end) { im->error = OR_SYNTAX_ERROR; return; }
  p += 2;
  if (hlen < 4u + 2u * im->nch) { im->error = OR_SYNTAX_ERROR; return; }
  if (*p++ != im->nch) { im->error = OR_UNSUPPORTED_ERROR; return; }
  for (int c = 0; c < im->nch; c++, p += 2) {
    if (p[0] != im->comp[c].id) { im->error = OR_SYNTAX_ERROR; return; }
    if (p[1] & 0xEE) { im->error = OR_SYNTAX_ERROR; return; }
    im->comp[c].dc_id = p[1] >> 4;
    im->comp[c].ac_id = (p[1] & 1) | 2;
  }
  if (p[0] || p[1] != 63 || p[2]) { im->error = OR_UNSUPPORTED_ERROR; return; }
  im->pos += hlen;
  for (int c = 0; c < im->nch; c++)
    if (!im->vlc[im->comp[c].dc_id] || !im->vlc[im->comp[c].ac_id]) {
      /* the reference would read an uninitialised table here */
      im->error = OR_SYNTAX_ERROR;
      return;
    }
  unstuff(im);

  /* MCU loop with restart handling: src/decodeScanGPU.cu:456-490 (the
   * no-restart branch at :435-452 is the same loop without the marker check) */
  int ri = im->restart_interval;
  int left = ri, expect = 0;
  for (int my = 0; my < im->mcuy; my++)
    for (int mx = 0; mx < im->mcux; mx++) {
      for (int c = 0; c < im->nch; c++) {
        OracleComp *k = &im->comp[c];
        for (int b = 0; b < k->sx * k->sy; b++) {
          decode_block(im, k);
          if (im->error) return;
        }
      }
      if (ri && !(--left) && im->pos < im->end) {
        im->nbits &= 0xF8; /* byte align */
        int m = get_bits(im, 16);
        if ((m & 0xFFF8) != 0xFFD0 || (m & 7) != expect) {
          im->error = OR_SYNTAX_ERROR;
          return;
        }
        expect = (expect + 1) & 7;
        left = ri;
        for (int c = 0; c < 3; c++) im->comp[c].dc_pred = 0;
      }
    }
  im->scan_done = 1;
}

/* ---------------- progressive scans (ITU T.81 Annex G) ----------------
 *
 * Not in the reference (it rejects SOF2, src/format.cu:191-200).  Each
 * scan's entropy-coded data runs to the next marker that is not RSTn; the
 * bit reader below reads it with the FF 00 stuffing removed.  Coefficients
 * are built up in qcoef (quantised, natural order) and dequantised at EOI. */

typedef struct {
  const uint8_t *p, *end; /* stuffed bytes of the scan */
  uint32_t bits;
  int nbits;
} ProgBits;

static int pb_bit(ProgBits *b) {
  if (!b->nbits) {
    uint8_t v = 0;
    if (b->p < b->end) {
      v = *b->p++;
      if (v == 0xFF && b->p < b->end && *b->p == 0x00) b->p++;
    }
    b->bits = v;
    b->nbits = 8;
  }
  b->nbits--;
  return (b->bits >> b->nbits) & 1;
}

static int pb_bits(ProgBits *b, int n) {
  int v = 0;
  while (n--) v = (v << 1) | pb_bit(b);
  return v;
}

/* Huffman decode with the 16-bit table: bit by bit against the code lengths
 * (the table gives {len, symbol} of the code that prefixes a window). */
static int pb_huff(ProgBits *b, const OracleVlc *t, int *err) {
  int code = 0;
  for (int l = 1; l <= 16; l++) {
    code = (code << 1) | pb_bit(b);
    const OracleVlc e = t[code << (16 - l)];
    if (e.len == l) return e.sym;
  }
  *err = OR_SYNTAX_ERROR;
  return 0;
}

static int pb_extend(int v, int s) { return v < (1 << (s - 1)) ? v - (1 << s) + 1 : v; }

/* After a restart interval: skip to the byte boundary and the RSTn marker. */
static int pb_restart(ProgBits *b, int expect) {
  b->nbits = 0;
  if (b->p + 1 >= b->end || b->p[0] != 0xFF || b->p[1] != (0xD0 | expect)) return OR_SYNTAX_ERROR;
  b->p += 2;
  return 0;
}

/* One block of a progressive scan (T.81 G.1.2.1-3; the decoding procedures
 * DECODE_DC_FIRST / DC refinement / DECODE_AC_FIRST / AC refinement with
 * end-of-band runs). */
static int prog_block(OracleImage *im, ProgBits *b, OracleComp *k, int32_t *q, int ss, int se, int ah, int al) {
  int err = 0;
  if (ss == 0) {
    if (!ah) {
      const int s = pb_huff(b, im->vlc[k->dc_id], &err);
      if (err) return err;
      if (s > 11) return OR_SYNTAX_ERROR;
      k->dc_pred += s ? pb_extend(pb_bits(b, s), s) : 0;
      q[0] = k->dc_pred * (1 << al);
    } else if (pb_bit(b)) {
      q[0] |= 1 << al;
    }
    return 0;
  }
  const OracleVlc *t = im->vlc[k->ac_id];
  int kk = ss;
  if (!ah) {
    if (im->eobrun > 0) { im->eobrun--; return 0; }
    while (kk <= se) {
      const int rs = pb_huff(b, t, &err);
      if (err) return err;
      const int r = rs >> 4, s = rs & 15;
      if (s) {
        kk += r;
        if (kk > se) return OR_SYNTAX_ERROR;
        q[kZigZagToNatural[kk]] = pb_extend(pb_bits(b, s), s) * (1 << al);
        kk++;
      } else if (r == 15) {
        kk += 16;
      } else {
        im->eobrun = (1 << r) - 1;
        if (r) im->eobrun += pb_bits(b, r);
        break;
      }
    }
    return 0;
  }
  const int p1 = 1 << al, m1 = -(1 << al);
  if (im->eobrun == 0) {
    for (; kk <= se; kk++) {
      const int rs = pb_huff(b, t, &err);
      if (err) return err;
      int r = rs >> 4, s = rs & 15, val = 0;
      if (s) {
        if (s != 1) return OR_SYNTAX_ERROR;
        val = pb_bit(b) ? p1 : m1;
      } else if (r != 15) {
        im->eobrun = 1 << r;
        if (r) im->eobrun += pb_bits(b, r);
        break;
      }
      /* pass r zero-history coefficients, refining the nonzero ones met */
      while (kk <= se) {
        int32_t *c = &q[kZigZagToNatural[kk]];
        if (*c) {
          if (pb_bit(b) && !(*c & p1)) *c += *c >= 0 ? p1 : m1;
        } else if (--r < 0) {
          break;
        }
        kk++;
      }
      if (val) {
        if (kk > se) return OR_SYNTAX_ERROR;
        q[kZigZagToNatural[kk]] = val;
      }
    }
  }
  if (im->eobrun > 0) {
    /* inside an end-of-band run: correction bits of the nonzero coefficients */
    for (; kk <= se; kk++) {
      int32_t *c = &q[kZigZagToNatural[kk]];
      if (*c && pb_bit(b) && !(*c & p1)) *c += *c >= 0 ? p1 : m1;
    }
    im->eobrun--;
  }
  return 0;
}

static void decode_prog_scan(OracleImage *im) {
  /* SOS of a progressive frame (T.81 B.2.3, G.1.1.1.1) */
  uint8_t *p = im->pos;
  unsigned hlen = read16(p);
  if (p + hlen > im->end || hlen < 6) { im->error = OR_SYNTAX_ERROR; return; }
  const int ns = p[2];
  if (ns < 1 || ns > im->nch || hlen != 6u + 2u * ns) { im->error = OR_SYNTAX_ERROR; return; }
  int comps[3];
  for (int j = 0; j < ns; j++) {
    const uint8_t *d = p + 3 + 2 * j;
    int c = 0;
    while (c < im->nch && im->comp[c].id != d[0]) c++;
    if (c == im->nch || (j && c <= comps[j - 1]) || (d[1] & 0xEE)) { im->error = OR_SYNTAX_ERROR; return; }
    comps[j] = c;
    im->comp[c].dc_id = d[1] >> 4;
    im->comp[c].ac_id = (d[1] & 1) | 2;
  }
  const uint8_t *t = p + 3 + 2 * ns;
  const int ss = t[0], se = t[1], ah = t[2] >> 4, al = t[2] & 15;
  if ((ss == 0) != (se == 0) || se > 63 || ss > se || (ss && ns != 1) || al > 13 || (ah && ah != al + 1)) {
    im->error = OR_SYNTAX_ERROR;
    return;
  }
  for (int j = 0; j < ns; j++) {
    const OracleComp *k = &im->comp[comps[j]];
    if ((ss == 0 && !ah && !im->vlc[k->dc_id]) || (ss && !im->vlc[k->ac_id])) { im->error = OR_SYNTAX_ERROR; return; }
  }
  im->pos += hlen;
  /* the scan's data: up to the next marker other than RSTn */
  const uint8_t *e = im->pos;
  while (e + 1 < im->end + 2 && !(e[0] == 0xFF && e[1] != 0x00 && (e[1] & 0xF8) != 0xD0)) e++;
  ProgBits b = {im->pos, e, 0, 0};
  im->eobrun = 0;
  for (int c = 0; c < 3; c++) im->comp[c].dc_pred = 0;
  const int ri = im->restart_interval;
  int left = ri, expect = 0, err = 0;
  if (ns > 1) { /* interleaved (DC scans only): MCU order */
    for (int my = 0; my < im->mcuy && !err; my++)
      for (int mx = 0; mx < im->mcux && !err; mx++) {
        for (int j = 0; j < ns && !err; j++) {
          OracleComp *k = &im->comp[comps[j]];
          const int per = k->sx * k->sy;
          for (int w = 0; w < per && !err; w++)
            err = prog_block(im, &b, k, k->qcoef + 64 * ((size_t)(my * im->mcux + mx) * per + w), ss, se, ah, al);
        }
        if (!err && ri && !(--left) && !(my == im->mcuy - 1 && mx == im->mcux - 1)) {
          err = pb_restart(&b, expect);
          expect = (expect + 1) & 7;
          left = ri;
          im->eobrun = 0;
          for (int c = 0; c < 3; c++) im->comp[c].dc_pred = 0;
        }
      }
  } else { /* one component: its blocks in raster order, not padded to MCUs */
    OracleComp *k = &im->comp[comps[0]];
    const int bw = (k->width + 7) / 8, bh = (k->height + 7) / 8, per = k->sx * k->sy;
    for (int by = 0; by < bh && !err; by++)
      for (int bx = 0; bx < bw && !err; bx++) {
        const size_t mcu = (size_t)(by / k->sy) * im->mcux + bx / k->sx;
        const size_t blk = mcu * per + (by % k->sy) * k->sx + bx % k->sx;
        err = prog_block(im, &b, k, k->qcoef + 64 * blk, ss, se, ah, al);
        if (!err && ri && !(--left) && !(by == bh - 1 && bx == bw - 1)) {
          err = pb_restart(&b, expect);
          expect = (expect + 1) & 7;
          left = ri;
          im->eobrun = 0;
          k->dc_pred = 0;
        }
      }
  }
  if (err) { im->error = err; return; }
  im->pos = (uint8_t *)e;
  im->scan_done = 1;
}

/* Progressive frames at EOI: dequantise the built-up coefficients. */
static void prog_dequantise(OracleImage *im) {
  for (int c = 0; c < im->nch; c++) {
    OracleComp *k = &im->comp[c];
    const uint16_t *dq = im->dq[k->dq_id];
    for (size_t b = 0; b < (size_t)k->nblocks; b++)
      for (int z = 0; z < 64; z++) {
        const int n = kZigZagToNatural[z];
        k->coef[64 * b + n] = k->qcoef[64 * b + n] * dq[z];
      }
  }
}

/* ---------------- pixel stage (CPUonly/src/pixelTransformCPU.c) ---------------- */

#define W1 2841 /* 2048*sqrt(2)*cos(1*pi/16) */
#define W2 2676 /* 2048*sqrt(2)*cos(2*pi/16) */
#define W3 2408 /* 2048*sqrt(2)*cos(3*pi/16) */
#define W5 1609 /* 2048*sqrt(2)*cos(5*pi/16) */
#define W6 1108 /* 2048*sqrt(2)*cos(6*pi/16) */
#define W7 565  /* 2048*sqrt(2)*cos(7*pi/16) */

static uint8_t clip8(int x) { return x < 0 ? 0 : (x > 255 ? 255 : (uint8_t)x); }

/* One 8-point row of the fixed-point iDCT (pixelTransformCPU.c:14-57), in place.
 * The all-AC-zero shortcut of the reference gives the same result as the
 * general butterflies, so it is not restated. */
void oracle_idct_row(int32_t *d) {
  int a0 = (d[0] * 2048) + 128, a1 = d[4] * 2048, a2 = d[6], a3 = d[2];
  int a4 = d[1], a5 = d[7], a6 = d[5], a7 = d[3], t;
  t = W7 * (a4 + a5);
  a4 = t + (W1 - W7) * a4;
  a5 = t - (W1 + W7) * a5;
  t = W3 * (a6 + a7);
  a6 = t - (W3 - W5) * a6;
  a7 = t - (W3 + W5) * a7;
  t = a0 + a1;
  a0 -= a1;
  a1 = W6 * (a3 + a2);
  a2 = a1 - (W2 + W6) * a2;
  a3 = a1 + (W2 - W6) * a3;
  a1 = a4 + a6;
  a4 -= a6;
  a6 = a5 + a7;
  a5 -= a7;
  a7 = t + a3;
  t -= a3;
  a3 = a0 + a2;
  a0 -= a2;
  a2 = (181 * (a4 + a5) + 128) >> 8;
  a4 = (181 * (a4 - a5) + 128) >> 8;
  d[0] = (a7 + a1) >> 8;
  d[1] = (a3 + a2) >> 8;
  d[2] = (a0 + a4) >> 8;
  d[3] = (t + a6) >> 8;
  d[4] = (t - a6) >> 8;
  d[5] = (a0 - a4) >> 8;
  d[6] = (a3 - a2) >> 8;
  d[7] = (a7 - a1) >> 8;
}

/* One 8-point column of the fixed-point iDCT with the +128 level shift and
 * clip (pixelTransformCPU.c:60-107).  d points at row 0 of the column. */
void oracle_idct_col(const int32_t *d, uint8_t *out, int stride) {
  int a0 = (d[0] * 256) + 8192, a1 = d[32] * 256, a2 = d[48], a3 = d[16];
  int a4 = d[8], a5 = d[56], a6 = d[40], a7 = d[24], t;
  t = W7 * (a4 + a5) + 4;
  a4 = (t + (W1 - W7) * a4) >> 3;
  a5 = (t - (W1 + W7) * a5) >> 3;
  t = W3 * (a6 + a7) + 4;
  a6 = (t - (W3 - W5) * a6) >> 3;
  a7 = (t - (W3 + W5) * a7) >> 3;
  t = a0 + a1;
  a0 -= a1;
  a1 = W6 * (a3 + a2) + 4;
  a2 = (a1 - (W2 + W6) * a2) >> 3;
  a3 = (a1 + (W2 - W6) * a3) >> 3;
  a1 = a4 + a6;
  a4 -= a6;
  a6 = a5 + a7;
  a5 -= a7;
  a7 = t + a3;
  t -= a3;
  a3 = a0 + a2;
  a0 -= a2;
  a2 = (181 * (a4 + a5) + 128) >> 8;
  a4 = (181 * (a4 - a5) + 128) >> 8;
  out[0 * stride] = clip8(((a7 + a1) >> 14) + 128);
  out[1 * stride] = clip8(((a3 + a2) >> 14) + 128);
  out[2 * stride] = clip8(((a0 + a4) >> 14) + 128);
  out[3 * stride] = clip8(((t + a6) >> 14) + 128);
  out[4 * stride] = clip8(((t - a6) >> 14) + 128);
  out[5 * stride] = clip8(((a0 - a4) >> 14) + 128);
  out[6 * stride] = clip8(((a3 - a2) >> 14) + 128);
  out[7 * stride] = clip8(((a7 - a1) >> 14) + 128);
}

/* Integer iDCT of one 64-coefficient natural-order block into a plane. */
void oracle_idct_block(const int32_t *coef, uint8_t *out, int stride) {
  int32_t tmp[64];
  memcpy(tmp, coef, sizeof(tmp));
  for (int r = 0; r < 8; r++) oracle_idct_row(tmp + 8 * r);
  for (int c = 0; c < 8; c++) oracle_idct_col(tmp + c, out + c, stride);
}

/* Block b of a component, in scan order, sits at plane block (bx, by):
 * MCU m = b / (sx*sy) in raster order, then sy rows of sx blocks inside it
 * (decodeScanGPU.cu:437-447 emission order; pixelTransformGPU.cu:120-131). */
static void block_origin(const OracleImage *im, const OracleComp *k, int b, int *bx, int *by) {
  int per = k->sx * k->sy;
  int m = b / per, r = b % per;
  *bx = (m % im->mcux) * k->sx + r % k->sx;
  *by = (m / im->mcux) * k->sy + r / k->sx;
}

static void pixel_stage(OracleImage *im) {
  for (int c = 0; c < im->nch; c++) {
    OracleComp *k = &im->comp[c];
    for (int b = 0; b < k->nblocks; b++) {
      int bx, by;
      block_origin(im, k, b, &bx, &by);
      oracle_idct_block(k->coef + 64 * (size_t)b,
                        k->plane + (size_t)by * 8 * k->stride + bx * 8, k->stride);
    }
  }
  size_t npix = (size_t)im->width * im->height;
  im->pixels = (uint8_t *)malloc(npix * (im->nch == 3 ? 3 : 1));
  if (!im->pixels) { im->error = OR_OOM_ERROR; return; }
  if (im->nch == 3) {
    /* upsample factor: pixelTransformCPU.c:113-114 (double until >= image) */
    int xs = 0, ys = 0;
    while ((im->comp[1].width << xs) < im->width) xs++;
    while ((im->comp[1].height << ys) < im->height) ys++;
    const OracleComp *Y = &im->comp[0], *Cb = &im->comp[1], *Cr = &im->comp[2];
    uint8_t *o = im->pixels;
    for (int y = 0; y < im->height; y++)
      for (int x = 0; x < im->width; x++) {
        /* pixelTransformCPU.c:147-158 */
        int yy = Y->plane[(size_t)y * Y->stride + x] << 8;
        size_t ci = (size_t)(y >> ys) * Cb->stride + (x >> xs);
        int cb = Cb->plane[ci] - 128, cr = Cr->plane[ci] - 128;
        *o++ = clip8((yy + 359 * cr + 128) >> 8);
        *o++ = clip8((yy - 88 * cb - 183 * cr + 128) >> 8);
        *o++ = clip8((yy + 454 * cb + 128) >> 8);
      }
  } else {
    const OracleComp *Y = &im->comp[0];
    for (int y = 0; y < im->height; y++)
      memcpy(im->pixels + (size_t)y * im->width, Y->plane + (size_t)y * Y->stride, im->width);
  }
}

/* ---------------- public entry points (called through ctypes) ---------------- */

void oracle_free(OracleImage *im) {
  if (!im) return;
  free(im->buf);
  for (int i = 0; i < 4; i++) free(im->vlc[i]);
  for (int c = 0; c < 3; c++) { free(im->comp[c].coef); free(im->comp[c].plane); free(im->comp[c].qcoef); }
  free(im->pixels);
  free(im);
}

/* Decode a whole JPEG held in memory.  Returns the image (check *err). The
 * marker loop restates src/format.cu:159-215, including its treatment of the
 * whole remainder of the file (up to the final EOI) as the entropy data. */
OracleImage *oracle_decode(const uint8_t *data, size_t size, int *err) {
  OracleImage *im = (OracleImage *)calloc(1, sizeof(OracleImage));
  if (!im) { *err = OR_OOM_ERROR; return NULL; }
  if (size < 4 || data[0] != 0xFF || data[1] != 0xD8 || data[size - 2] != 0xFF ||
      data[size - 1] != 0xD9) {
    im->error = OR_FILE_ERROR;
    goto done;
  }
  if (size < 6) { im->error = OR_SYNTAX_ERROR; goto done; }
  im->buf = (uint8_t *)malloc(size + 4);
  if (!im->buf) { im->error = OR_OOM_ERROR; goto done; }
  memcpy(im->buf, data, size);
  im->size = size;
  im->end = im->buf + size - 2;
  im->pos = im->buf + 2;
  while (!im->error) {
    if (im->pos > im->end || im->pos[0] != 0xFF) { im->error = OR_SYNTAX_ERROR; break; }
    im->pos += 2;
    uint8_t m = im->pos[-1];
    switch (m) {
      case 0xC0: parse_sof(im); break;
      case 0xC2: im->progressive = 1; parse_sof(im); break;
      case 0xC4: parse_dht(im); break;
      case 0xDB: parse_dqt(im); break;
      case 0xDD: parse_dri(im); break;
      case 0xDA:
        if (!im->nch) { im->error = OR_SYNTAX_ERROR; break; }
        if (im->progressive) decode_prog_scan(im);
        else decode_scan(im);
        break;
      case 0xFE: skip_segment(im); break;
      case 0xD9: break;
      default:
        if ((m & 0xF0) == 0xE0) skip_segment(im);
        else im->error = OR_SYNTAX_ERROR;
    }
    if (im->error) break;
    if (im->pos[-1] == 0xD9) {
      if (!im->scan_done) { im->error = OR_SYNTAX_ERROR; break; }
      if (im->progressive) prog_dequantise(im);
      pixel_stage(im);
      break;
    }
  }
done:
  *err = im->error;
  return im;
}

/* info[0..]: width, height, nch, mcux, mcuy, restart_interval, then per
 * component c (base 6+8c): sx, sy, width, height, stride, rows, nblocks, dq_id */
void oracle_info(const OracleImage *im, int *info) {
  info[0] = im->width; info[1] = im->height; info[2] = im->nch;
  info[3] = im->mcux; info[4] = im->mcuy; info[5] = im->restart_interval;
  for (int c = 0; c < 3; c++) {
    const OracleComp *k = &im->comp[c];
    int *o = info + 6 + 8 * c;
    o[0] = k->sx; o[1] = k->sy; o[2] = k->width; o[3] = k->height;
    o[4] = k->stride; o[5] = k->rows; o[6] = k->nblocks; o[7] = k->dq_id;
  }
}

void oracle_coefs(const OracleImage *im, int c, int32_t *out) {
  memcpy(out, im->comp[c].coef, (size_t)im->comp[c].nblocks * 64 * sizeof(int32_t));
}

void oracle_plane(const OracleImage *im, int c, uint8_t *out) {
  memcpy(out, im->comp[c].plane, (size_t)im->comp[c].stride * im->comp[c].rows);
}

void oracle_pixels(const OracleImage *im, uint8_t *out) {
  memcpy(out, im->pixels, (size_t)im->width * im->height * (im->nch == 3 ? 3 : 1));
}

void oracle_dq(const OracleImage *im, uint16_t *out) { memcpy(out, im->dq, sizeof(im->dq)); }

/* Integer iDCT of n natural-order blocks (int32 dequantised) into n separate
 * 8x8 uint8 tiles: used to test the plane kernels block by block. */
void oracle_idct_blocks(const int32_t *coef, int64_t n, uint8_t *out) {
  for (int64_t b = 0; b < n; b++) oracle_idct_block(coef + 64 * b, out + 64 * b, 8);
}

/* FP64 separable orthonormal iDCT (ITU T.81 A.3.3) of n blocks, before the
 * +128 shift, rounding and clip: the exact reference for iDCT error. */
void oracle_idct_f64(const int32_t *coef, int64_t n, double *out) {
  double basis[8][8]; /* basis[u][x] = C(u)/2 cos((2x+1)u pi/16) */
  for (int u = 0; u < 8; u++)
    for (int x = 0; x < 8; x++)
      basis[u][x] = (u ? 0.5 : 0.5 / sqrt(2.0)) * cos((2 * x + 1) * u * 3.14159265358979323846 / 16.0);
  for (int64_t b = 0; b < n; b++) {
    const int32_t *f = coef + 64 * b;
    double tmp[8][8];
    for (int v = 0; v < 8; v++) /* rows: tmp[v][x] = sum_u F[v][u] basis[u][x] */
      for (int x = 0; x < 8; x++) {
        double s = 0;
        for (int u = 0; u < 8; u++) s += f[8 * v + u] * basis[u][x];
        tmp[v][x] = s;
      }
    double *o = out + 64 * b;
    for (int y = 0; y < 8; y++)
      for (int x = 0; x < 8; x++) {
        double s = 0;
        for (int v = 0; v < 8; v++) s += tmp[v][x] * basis[v][y];
        o[8 * y + x] = s;
      }
  }
}

/* ---------------- fancy (triangle) chroma upsampling ----------------
 *
 * Not part of the reference path (its upsampling is nearest replication,
 * CPUonly/src/pixelTransformCPU.c:110-127); this restates the published IJG
 * decoder's "fancy" upsampling (libjpeg jdsample.c: h2v1, h1v2 and h2v2
 * fancy upsamplers) as the checker of the decoder's optional fancy mode.
 * A factor-2 direction interpolates with weights 3/4 and 1/4 between the
 * nearer and the farther sample; each output pair alternates its rounding
 * bias (h2v1 / h1v2: +1 then +2, >> 2; h2v2: +8 then +7, >> 4 after the
 * vertical 3:1 column sums); the first and last column of a row use the
 * edge sample alone (h2v2: 4 x the column sum), the rows above the first
 * and below the last repeat them.  Other factors replicate (IJG
 * int_upsample).  `in` is a cw x ch plane (stride in_stride); `out` gets the
 * ow x oh upsampled plane (cropped from 2cw x 2ch).  A one-sample-wide
 * plane uses its sample for both neighbours. */
void oracle_fancy_upsample(const uint8_t *in, int cw, int ch, int in_stride, int xs, int ys,
                           uint8_t *out, int ow, int oh) {
  const int fancy = (xs == 1 && ys <= 1) || (xs == 0 && ys == 1);
  for (int y = 0; y < oh; y++) {
    const int r = y >> ys;
    const uint8_t *row = in + (size_t)(r < ch ? r : ch - 1) * in_stride;
    int nb = r;
    if (fancy && ys == 1) nb = (y & 1) ? (r + 1 < ch ? r + 1 : ch - 1) : (r > 0 ? r - 1 : 0);
    const uint8_t *nrow = in + (size_t)(nb < ch ? nb : ch - 1) * in_stride;
    for (int x = 0; x < ow; x++) {
      const int i = x >> xs;
      int v;
      if (!fancy) {
        v = row[i < cw ? i : cw - 1];
      } else if (xs == 0) { /* h1v2 */
        v = (3 * row[i] + nrow[i] + ((y & 1) ? 2 : 1)) >> 2;
      } else if (ys == 0) { /* h2v1 */
        if (x & 1) v = (i == cw - 1) ? row[i] : (3 * row[i] + row[i + 1] + 2) >> 2;
        else v = (i == 0) ? row[i] : (3 * row[i] + row[i - 1] + 1) >> 2;
      } else { /* h2v2 */
        const int cs = 3 * row[i] + nrow[i];
        if (x & 1) v = (i == cw - 1) ? (4 * cs + 7) >> 4 : (3 * cs + 3 * row[i + 1] + nrow[i + 1] + 7) >> 4;
        else v = (i == 0) ? (4 * cs + 8) >> 4 : (3 * cs + 3 * row[i - 1] + nrow[i - 1] + 8) >> 4;
      }
      out[(size_t)y * ow + x] = (uint8_t)v;
    }
  }
}

/* The decoded image with fancy chroma upsampling: upsampled Y, Cb, Cr
 * interleaved (ycc, may be NULL) and RGB through the reference's colour
 * transform (CPUonly/src/pixelTransformCPU.c:147-158; rgb, may be NULL).
 * Colour images only. */
void oracle_fancy(const OracleImage *im, uint8_t *ycc, uint8_t *rgb) {
  const int W = im->width, H = im->height;
  int xs = 0, ys = 0;
  while ((im->comp[1].width << xs) < W) xs++;
  while ((im->comp[1].height << ys) < H) ys++;
  uint8_t *cb = (uint8_t *)malloc((size_t)W * H), *cr = (uint8_t *)malloc((size_t)W * H);
  if (!cb || !cr) { free(cb); free(cr); return; }
  oracle_fancy_upsample(im->comp[1].plane, im->comp[1].width, im->comp[1].height, im->comp[1].stride, xs, ys, cb, W, H);
  oracle_fancy_upsample(im->comp[2].plane, im->comp[2].width, im->comp[2].height, im->comp[2].stride, xs, ys, cr, W, H);
  const OracleComp *Y = &im->comp[0];
  for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++) {
      const size_t k = (size_t)y * W + x;
      const int yv = Y->plane[(size_t)y * Y->stride + x];
      if (ycc) { ycc[3 * k] = (uint8_t)yv; ycc[3 * k + 1] = cb[k]; ycc[3 * k + 2] = cr[k]; }
      if (rgb) {
        const int yy = yv << 8, b = cb[k] - 128, r = cr[k] - 128;
        rgb[3 * k] = clip8((yy + 359 * r + 128) >> 8);
        rgb[3 * k + 1] = clip8((yy - 88 * b - 183 * r + 128) >> 8);
        rgb[3 * k + 2] = clip8((yy + 454 * b + 128) >> 8);
      }
    }
  free(cb);
  free(cr);
}
