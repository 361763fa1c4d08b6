// cj_parse.cuh -- the marker-segment parse of one JPEG file up to its scan,
// as one function that runs on the host and on the device.  The batch
// decoder runs it on the GPU, one thread per file (k_parse_headers in
// batch.cu), over the files it has already copied to the device; it yields
// the same header, scan range and error code as the host marker loop of the
// drop-in path (format.cu cj_marker_loop with stop_at_scan, scan.cu
// cj_parse_sos, progressive.cu cj_parse_prog_sos) for every file, malformed
// ones included.  The checks are the reference's (src/format.cu:113-442,
// src/decodeScanGPU.cu:124-144), cited per segment below.
#pragma once
#include <stdint.h>

#include "../../include/format.h"
#include "cj_core.h"

// What the parse of one image hands the device decode (tables as parsed,
// geometry).
struct CJImageHeader {
  uint8_t counts[4][16];    // DHT BITS per table slot
  uint8_t symbols[4][256];  // DHT HUFFVAL per table slot
  uint16_t dq[4][64];       // DQT (8- or 16-bit values), zig-zag order
  uint8_t comp_dc[3], comp_ac[3], comp_q[3], comp_sx[3], comp_sy[3];
  uint8_t nch, huff_mask, xshift, yshift, pad[4];
  int32_t mcux, mcuy, width, height, hmax, vmax, restart_interval, nseg_expected;
  int64_t total_blocks;
};

CJ_HD unsigned cj_rd16(const uint8_t* p) { return ((unsigned)p[0] << 8) | p[1]; }

// Frame state the segments build up (a fresh one per file).
struct CJParseState {
  int nch, ids[3], sx[3], sy[3], dq[3], cw[3], chh[3];
  int width, height, sxmax, symax, mcux, mcuy;
  int restart, huff_defined, progressive;
};

// SOF0 / SOF2 (src/format.cu:242-354): precision, size, components,
// power-of-two sampling, the geometry the decoder supports.
CJ_HD int cj_ps_sof(const uint8_t* buf, int64_t& pos, int64_t end, CJParseState& s) {
  if (pos > end) return SYNTAX_ERROR;
  const uint8_t* block = buf + pos;
  const unsigned block_len = cj_rd16(block);
  if (block_len < 9 || pos + block_len >= end) return SYNTAX_ERROR;
  if (block[2] != 8) return UNSUPPORTED_ERROR;
  s.height = (int)cj_rd16(block + 3);
  s.width = (int)cj_rd16(block + 5);
  if (!s.width || !s.height) return SYNTAX_ERROR;
  s.nch = block[7];
  if (s.nch != 1 && s.nch != 3) return UNSUPPORTED_ERROR;
  if (block_len < 8u + s.nch * 3u) return SYNTAX_ERROR;
  int sxm = 0, sym = 0;
  for (int i = 0; i < s.nch; i++) {
    const uint8_t* c = block + 8 + 3 * i;
    s.ids[i] = c[0];
    s.sx[i] = c[1] >> 4;
    s.sy[i] = c[1] & 0xF;
    s.dq[i] = c[2];
    if (!s.sx[i] || !s.sy[i] || s.dq[i] > 3) return SYNTAX_ERROR;
    if ((s.sx[i] & (s.sx[i] - 1)) || (s.sy[i] & (s.sy[i] - 1))) return UNSUPPORTED_ERROR;
    if (s.sx[i] > sxm) sxm = s.sx[i];
    if (s.sy[i] > sym) sym = s.sy[i];
  }
  if (s.nch == 1) s.sx[0] = s.sy[0] = sxm = sym = 1;
  s.sxmax = sxm;
  s.symax = sym;
  // the host keeps these as unsigned short (JPGReader): the same wrap
  s.mcux = (uint16_t)((s.width + 8 * sxm - 1) / (8 * sxm));
  s.mcuy = (uint16_t)((s.height + 8 * sym - 1) / (8 * sym));
  int bpm = 0;
  for (int i = 0; i < s.nch; i++) {
    s.cw[i] = (s.width * s.sx[i] + sxm - 1) / sxm;
    s.chh[i] = (s.height * s.sy[i] + sym - 1) / sym;
    if ((s.cw[i] < 3 && s.sx[i] != sxm) || (s.chh[i] < 3 && s.sy[i] != sym)) return UNSUPPORTED_ERROR;
    bpm += s.sx[i] * s.sy[i];
  }
  if (bpm > CJ_MAX_BPM) return UNSUPPORTED_ERROR;
  if (s.nch == 3 && (s.cw[1] != s.cw[2] || s.chh[1] != s.chh[2] || s.cw[0] != s.width || s.chh[0] != s.height))
    return UNSUPPORTED_ERROR;
  pos += block_len;
  return 0;
}

// DHT (src/format.cu:357-400): table class and id, code-space overflow, at
// most 256 symbols; kept in canonical (BITS, HUFFVAL) form per slot
// (DC0, DC1, AC0, AC1).
CJ_HD int cj_ps_dht(const uint8_t* buf, int64_t& pos, int64_t end, CJParseState& s, CJImageHeader* h) {
  if (pos > end) return SYNTAX_ERROR;
  const int64_t block_end = pos + cj_rd16(buf + pos);
  if (block_end > end) return SYNTAX_ERROR;
  int64_t p = pos + 2;
  while (p < block_end) {
    const unsigned val = buf[p];
    if (val & 0xEC) return SYNTAX_ERROR;
    if (val & 0x02) return UNSUPPORTED_ERROR;
    const int slot = (int)((val | (val >> 3)) & 3);
    if (p + 17 > block_end) return SYNTAX_ERROR;
    const int64_t sym = p + 17;
    int remain = 65536, nsym = 0;
    for (int l = 1; l <= 16; l++) {
      const int count = buf[p + l];
      if (!count) continue;
      if (sym + nsym + count > block_end) return SYNTAX_ERROR;
      remain -= count << (16 - l);
      if (remain < 0) return SYNTAX_ERROR;
      nsym += count;
    }
    if (nsym > 256) return UNSUPPORTED_ERROR;
    for (int l = 0; l < 16; l++) h->counts[slot][l] = buf[p + 1 + l];
    for (int k = 0; k < nsym; k++) h->symbols[slot][k] = buf[sym + k];
    s.huff_defined |= 1 << slot;
    p = sym + nsym;
  }
  if (p != block_end) return SYNTAX_ERROR;
  pos = block_end;
  return 0;
}

// DQT (src/format.cu:424-442; 16-bit tables, Pq = 1, as the host parser
// reads them, steps below 2^15).
CJ_HD int cj_ps_dqt(const uint8_t* buf, int64_t& pos, int64_t end, CJImageHeader* h) {
  if (pos > end) return SYNTAX_ERROR;
  const int64_t block_end = pos + cj_rd16(buf + pos);
  if (block_end > end) return SYNTAX_ERROR;
  int64_t p = pos + 2;
  while (p < block_end) {
    const int pq = buf[p] >> 4, id = buf[p] & 15;
    const int n = pq ? 129 : 65;
    if (pq > 1 || id > 3 || p + n > block_end) return SYNTAX_ERROR;
    for (int k = 0; k < 64; k++) {
      const unsigned v = pq ? cj_rd16(buf + p + 1 + 2 * k) : buf[p + 1 + k];
      if (v > 32767) return UNSUPPORTED_ERROR;
      h->dq[id][k] = (uint16_t)v;
    }
    p += n;
  }
  if (p != block_end) return SYNTAX_ERROR;
  pos = block_end;
  return 0;
}

// DRI (src/format.cu:404-421).
CJ_HD int cj_ps_dri(const uint8_t* buf, int64_t& pos, int64_t end, CJParseState& s) {
  if (pos > end) return SYNTAX_ERROR;
  const unsigned block_len = cj_rd16(buf + pos);
  if (block_len < 2 || pos + block_len > end) return SYNTAX_ERROR;
  if (block_len < 4) return SYNTAX_ERROR;
  s.restart = (int)cj_rd16(buf + pos + 2);
  pos += block_len;
  return 0;
}

// SOS of a progressive frame: only checked (the batch decoder takes
// baseline frames): a valid header is UNSUPPORTED_ERROR, an invalid one a
// SYNTAX_ERROR, as progressive.cu cj_parse_prog_sos decides.
CJ_HD int cj_ps_prog_sos(const uint8_t* buf, int64_t pos, int64_t end, const CJParseState& s) {
  if (pos + 2 > end) return SYNTAX_ERROR;
  const uint8_t* p = buf + pos;
  const unsigned hlen = cj_rd16(p);
  if (hlen < 6 || pos + hlen > end) return SYNTAX_ERROR;
  if (!s.nch) return SYNTAX_ERROR;
  const int ns = p[2];
  if (ns < 1 || ns > s.nch || hlen != 6u + 2u * ns) return SYNTAX_ERROR;
  int prev = -1, dc[3] = {0, 0, 0}, ac[3] = {0, 0, 0};
  for (int j = 0; j < ns; j++) {
    const uint8_t* d = p + 3 + 2 * j;
    int c = 0;
    while (c < s.nch && s.ids[c] != d[0]) c++;
    if (c == s.nch || c <= prev || (d[1] & 0xEE)) return SYNTAX_ERROR;
    prev = c;
    dc[j] = d[1] >> 4;
    ac[j] = (d[1] & 1) | 2;
  }
  const uint8_t* t = p + 3 + 2 * ns;
  const int ss = t[0], se = t[1], ah = t[2] >> 4, al = t[2] & 15;
  if ((ss == 0) != (se == 0) || se > 63 || ss > se || (ss && ns != 1) || al > 13 || (ah && ah != al + 1))
    return SYNTAX_ERROR;
  for (int j = 0; j < ns; j++) {
    const bool need_dc = ss == 0 && !ah, need_ac = ss != 0;
    if ((need_dc && !(s.huff_defined & (1 << dc[j]))) || (need_ac && !(s.huff_defined & (1 << ac[j]))))
      return SYNTAX_ERROR;
  }
  return UNSUPPORTED_ERROR;
}

// The parse of one file: the marker loop of src/format.cu:159-215 up to the
// first SOS, that SOS's check (src/decodeScanGPU.cu:124-144 for the
// component list, Ss/Se/Ah/Al; each component's own tables must be
// defined), then the header of the batch decoder.  *scan_off / *scan_len:
// the entropy-coded bytes (from after the SOS header to before the EOI).
CJ_HD int cj_parse_header(const uint8_t* buf, int64_t size, CJImageHeader* h, int64_t* scan_off,
                          int64_t* scan_len) {
  for (int k = 0; k < (int)sizeof(CJImageHeader); k++) reinterpret_cast<uint8_t*>(h)[k] = 0;
  *scan_off = *scan_len = 0;
  if (size < 4 || buf[0] != 0xFF || buf[1] != 0xD8 || buf[size - 2] != 0xFF || buf[size - 1] != 0xD9)
    return FILE_ERROR;
  if (size < 6) return SYNTAX_ERROR;
  const int64_t end = size - 2;  // the EOI marker is left out, as checked
  int64_t pos = 2;
  CJParseState s;
  s.nch = 0;
  s.restart = 0;
  s.huff_defined = 0;
  s.progressive = 0;
  s.width = s.height = s.mcux = s.mcuy = s.sxmax = s.symax = 0;
  for (;;) {
    if (pos > end || buf[pos] != 0xFF) return SYNTAX_ERROR;
    const int marker = buf[pos + 1];
    pos += 2;
    int e = 0;
    switch (marker) {
      case 0xC0: e = cj_ps_sof(buf, pos, end, s); break;
      case 0xC2:
        s.progressive = 1;
        e = cj_ps_sof(buf, pos, end, s);
        break;
      case 0xC4: e = cj_ps_dht(buf, pos, end, s, h); break;
      case 0xDB: e = cj_ps_dqt(buf, pos, end, h); break;
      case 0xDD: e = cj_ps_dri(buf, pos, end, s); break;
      case 0xDA: {
        if (s.progressive) return cj_ps_prog_sos(buf, pos, end, s);
        if (pos > end) return SYNTAX_ERROR;
        const unsigned hlen = cj_rd16(buf + pos);
        if (pos + hlen > end) return SYNTAX_ERROR;
        if (!s.nch) return SYNTAX_ERROR;
        if (hlen < 4u + 2u * s.nch) return SYNTAX_ERROR;
        const uint8_t* p = buf + pos + 2;
        if (*(p++) != s.nch) return UNSUPPORTED_ERROR;
        for (int i = 0; i < s.nch; i++, p += 2) {
          if (p[0] != s.ids[i]) return SYNTAX_ERROR;
          if (p[1] & 0xEE) return SYNTAX_ERROR;
          h->comp_dc[i] = (uint8_t)(p[1] >> 4);
          h->comp_ac[i] = (uint8_t)((p[1] & 1) | 2);
          if (!(s.huff_defined & (1 << h->comp_dc[i])) || !(s.huff_defined & (1 << h->comp_ac[i])))
            return SYNTAX_ERROR;
        }
        if (p[0] || p[1] != 63 || p[2]) return UNSUPPORTED_ERROR;
        pos += hlen;
        if (end - pos > (int64_t)CJ_MAX_SCAN_BYTES) return UNSUPPORTED_ERROR;
        *scan_off = pos;
        *scan_len = end - pos;
        // the header (batch.cu bt_fill_header on the host)
        h->huff_mask = (uint8_t)s.huff_defined;
        h->nch = (uint8_t)s.nch;
        int bpm = 0;
        for (int c = 0; c < s.nch; c++) {
          h->comp_q[c] = (uint8_t)s.dq[c];
          h->comp_sx[c] = (uint8_t)s.sx[c];
          h->comp_sy[c] = (uint8_t)s.sy[c];
          bpm += s.sx[c] * s.sy[c];
        }
        h->mcux = s.mcux;
        h->mcuy = s.mcuy;
        h->width = s.width;
        h->height = s.height;
        h->hmax = s.sxmax;
        h->vmax = s.symax;
        int xs = 0, ys = 0;
        if (s.nch == 3) {
          while ((s.cw[1] << xs) < s.width) xs++;
          while ((s.chh[1] << ys) < s.height) ys++;
        }
        h->xshift = (uint8_t)xs;
        h->yshift = (uint8_t)ys;
        h->restart_interval = s.restart;
        const int64_t mcus = (int64_t)h->mcux * h->mcuy;
        h->nseg_expected = s.restart ? (int)((mcus + s.restart - 1) / s.restart) : 1;
        h->total_blocks = mcus * bpm;
        // the pixel tile layout's geometry condition (cj_pix_check)
        if (h->comp_sx[0] != h->hmax || h->comp_sy[0] != h->vmax) return UNSUPPORTED_ERROR;
        if (h->nch == 3 && ((h->comp_sx[1] << xs) != h->hmax || (h->comp_sy[1] << ys) != h->vmax))
          return UNSUPPORTED_ERROR;
        return 0;
      }
      case 0xFE: e = pos > end ? SYNTAX_ERROR : (pos += cj_rd16(buf + pos), 0); break;
      case 0xD9: break;
      default:
        if ((marker & 0xF0) == 0xE0) e = pos > end ? SYNTAX_ERROR : (pos += cj_rd16(buf + pos), 0);
        else e = SYNTAX_ERROR;
    }
    if (e) return e;
    // a skipped segment that ran past the file: the next marker read fails
    // (checked here, so the byte before pos -- at most the EOI's last byte,
    // end + 1 -- is inside the file)
    if (pos > end + 2) return SYNTAX_ERROR;
    // EOI, or a segment that happens to end on byte 0xD9 (the reference
    // takes either as the end of the file, src/format.cu:204): before any
    // scan, a syntax error
    if (buf[pos - 1] == 0xD9) return SYNTAX_ERROR;
  }
}
