// progressive.cu -- progressive JPEG (SOF2) scans on the GPU.
//
// The reference decodes baseline frames only: SOF2 falls to its marker
// switch's SYNTAX_ERROR (src/format.cu:191-200).  Here a progressive frame
// goes through the same marker loop: every SOS (decodeScanGPU) decodes its
// scan into the int16 coefficient blocks (quantised, natural order, MCU scan
// order -- the layout of a baseline scan), scans accumulate in stream order,
// and the EOI's pixel stage is the baseline one.  Scan types follow ITU T.81
// Annex G (G.1.2): DC first (interleaved or not), DC refinement (one bit per
// block), AC first with end-of-band runs, and AC refinement with correction
// bits.  Restart intervals are independent: one thread decodes each (a scan
// without restart markers is one thread's serial decode); the host finds the
// RSTn markers and the end of the scan while it walks the markers.
#include <stdio.h>
#include <string.h>

#include <vector>

#include "../../include/decodeScanGPU.h"
#include "cj_entropy.cuh"
#include "cj_internal.h"
#include "cj_tables.h"

// The kernel's parameter block: the scan, its four Huffman tables, and the
// stuffed byte range [start, end) of each restart interval.
struct CJProgBlock {
  CJProgScan s;
  CJHuff huff[4];
};

// MSB-first bits of one interval's stuffed bytes: FF 00 reads as FF; bytes
// past the end read as 0.
struct CJProgBits {
  const uint8_t* p;
  const uint8_t* e;
  uint64_t acc;
  int n;
  __device__ __forceinline__ void fill() {
    while (n <= 56) {
      uint32_t b = 0;
      if (p < e) {
        b = *p++;
        if (b == 0xFF && p < e && *p == 0x00) p++;
      }
      acc |= (uint64_t)b << (56 - n);
      n += 8;
    }
  }
  __device__ __forceinline__ uint32_t peek16() {
    fill();
    return (uint32_t)(acc >> 48);
  }
  __device__ __forceinline__ uint32_t bits(int k) {  // k <= 16
    if (!k) return 0;
    fill();
    const uint32_t v = (uint32_t)(acc >> (64 - k));
    acc <<= k;
    n -= k;
    return v;
  }
  // Huffman symbol, or -1 when no code matches
  __device__ __forceinline__ int huff(const CJHuff& t) {
    const uint32_t e = cj_huff_decode(t, peek16());
    if (!e) return -1;
    acc <<= (e >> 8);
    n -= (int)(e >> 8);
    return (int)(e & 255);
  }
};

__device__ __forceinline__ int cj_prog_extend(uint32_t v, int s) {
  return v < (1u << (s - 1)) ? (int)v - (1 << s) + 1 : (int)v;
}

// A value into an int16 coefficient; false when it does not fit.
__device__ __forceinline__ bool cj_prog_store(int16_t* c, int v) {
  if (v < -32768 || v > 32767) return false;
  *c = (int16_t)v;
  return true;
}

// One block of the scan (T.81 G.1.2): returns 0 or a CJ_DEV_* code.
__device__ int cj_prog_block(const CJProgBlock& P, int j, CJProgBits& br, int16_t* blk, int* dc_pred,
                             int* eobrun, const uint8_t* zz) {
  const CJProgScan& S = P.s;
  if (S.ss == 0) {
    if (!S.ah) {
      const int s = br.huff(P.huff[S.dc_slot[j]]);
      if (s < 0) return CJ_DEV_BAD_CODE;
      if (s > 11) return CJ_DEV_BAD_AC;
      dc_pred[j] += s ? cj_prog_extend(br.bits(s), s) : 0;
      if (!cj_prog_store(&blk[0], dc_pred[j] * (1 << S.al))) return CJ_DEV_DC_RANGE;
    } else if (br.bits(1)) {
      blk[0] = (int16_t)(blk[0] | (1 << S.al));
    }
    return 0;
  }
  const CJHuff& t = P.huff[S.ac_slot[j]];
  int k = S.ss;
  if (!S.ah) {
    if (*eobrun > 0) {
      (*eobrun)--;
      return 0;
    }
    while (k <= S.se) {
      const int rs = br.huff(t);
      if (rs < 0) return CJ_DEV_BAD_CODE;
      const int r = rs >> 4, s = rs & 15;
      if (s) {
        k += r;
        if (k > S.se) return CJ_DEV_BAD_AC;
        if (!cj_prog_store(&blk[zz[k]], cj_prog_extend(br.bits(s), s) * (1 << S.al))) return CJ_DEV_DC_RANGE;
        k++;
      } else if (r == 15) {
        k += 16;
      } else {
        *eobrun = (1 << r) - 1;
        if (r) *eobrun += (int)br.bits(r);
        break;
      }
    }
    return 0;
  }
  const int p1 = 1 << S.al, m1 = -(1 << S.al);
  if (*eobrun == 0) {
    for (; k <= S.se; k++) {
      const int rs = br.huff(t);
      if (rs < 0) return CJ_DEV_BAD_CODE;
      int r = rs >> 4, val = 0;
      const int s = rs & 15;
      if (s) {
        if (s != 1) return CJ_DEV_BAD_AC;
        val = br.bits(1) ? p1 : m1;
      } else if (r != 15) {
        *eobrun = 1 << r;
        if (r) *eobrun += (int)br.bits(r);
        break;
      }
      // pass r zero-history coefficients, refining the nonzero ones met
      while (k <= S.se) {
        int16_t* c = &blk[zz[k]];
        if (*c) {
          if (br.bits(1) && !(*c & p1)) *c = (int16_t)(*c + (*c >= 0 ? p1 : m1));
        } else if (--r < 0) {
          break;
        }
        k++;
      }
      if (val) {
        if (k > S.se) return CJ_DEV_BAD_AC;
        blk[zz[k]] = (int16_t)val;
      }
    }
  }
  if (*eobrun > 0) {
    // inside an end-of-band run: the correction bits of the nonzero coefficients
    for (; k <= S.se; k++) {
      int16_t* c = &blk[zz[k]];
      if (*c && br.bits(1) && !(*c & p1)) *c = (int16_t)(*c + (*c >= 0 ? p1 : m1));
    }
    (*eobrun)--;
  }
  return 0;
}

__constant__ uint8_t c_prog_zz[64] = CJ_ZIGZAG_INIT;

// One thread per restart interval of the scan.
__global__ void __launch_bounds__(128) k_prog_scan(const CJProgBlock* __restrict__ blk_params,
                                                   const int64_t* __restrict__ spans, const uint8_t* __restrict__ file,
                                                   int16_t* __restrict__ coef, CJStatus* st) {
  __shared__ CJProgBlock P;
  __shared__ uint8_t zz[64];
  for (int k = threadIdx.x; k < (int)(sizeof(CJProgBlock) / 4); k += blockDim.x)
    reinterpret_cast<uint32_t*>(&P)[k] = reinterpret_cast<const uint32_t*>(blk_params)[k];
  if (threadIdx.x < 64) zz[threadIdx.x] = c_prog_zz[threadIdx.x];
  __syncthreads();
  const CJProgScan& S = P.s;
  const int iv = blockIdx.x * blockDim.x + threadIdx.x;
  if (iv >= S.nint) return;
  CJProgBits br;
  br.p = file + spans[2 * iv];
  br.e = file + spans[2 * iv + 1];
  br.acc = 0;
  br.n = 0;
  int dc_pred[3] = {0, 0, 0}, eobrun = 0;
  const int u0 = S.ri ? iv * S.ri : 0;
  const int u1 = S.ri ? min(S.nunits, u0 + S.ri) : S.nunits;
  for (int u = u0; u < u1; u++) {
    if (S.ns > 1) {  // interleaved (DC scans): an MCU of every scan component
      for (int j = 0; j < S.ns; j++)
        for (int w = 0; w < S.sx[j] * S.sy[j]; w++) {
          const int64_t b = (int64_t)u * S.bpm + S.first[j] + w;
          const int e = cj_prog_block(P, j, br, coef + b * 64, dc_pred, &eobrun, zz);
          if (e) {
            cj_raise(st, b, e);
            return;
          }
        }
    } else {  // one component: its blocks in raster order
      const int bx = u % S.bw, by = u / S.bw;
      const int64_t mcu = (int64_t)(by / S.sy[0]) * S.mcux + bx / S.sx[0];
      const int64_t b = mcu * S.bpm + S.first[0] + (by % S.sy[0]) * S.sx[0] + bx % S.sx[0];
      const int e = cj_prog_block(P, 0, br, coef + b * 64, dc_pred, &eobrun, zz);
      if (e) {
        cj_raise(st, b, e);
        return;
      }
    }
  }
}

// ---------------------------------------------------------------- host side

// Validate the SOS header of a progressive frame (T.81 B.2.3, G.1.1.1.1) at
// jpg->pos and fill `s` with the scan's components and band; on success
// jpg->pos is on the first entropy-coded byte.
int cj_parse_prog_sos(JPGReader* jpg, CJProgScan* s) {
  unsigned char* p = jpg->pos;
  if (p + 2 > jpg->end) return SYNTAX_ERROR;
  const unsigned hlen = read16(p);
  if (hlen < 6 || p + hlen > jpg->end) return SYNTAX_ERROR;
  if (!jpg->num_channels) return SYNTAX_ERROR;  // SOS before SOF
  const int ns = p[2];
  if (ns < 1 || ns > jpg->num_channels || hlen != 6u + 2u * ns) return SYNTAX_ERROR;
  memset(s, 0, sizeof(*s));
  int prev = -1;
  for (int j = 0; j < ns; j++) {
    const unsigned char* d = p + 3 + 2 * j;
    int c = 0;
    while (c < jpg->num_channels && jpg->channels[c].id != d[0]) c++;
    if (c == jpg->num_channels || c <= prev || (d[1] & 0xEE)) return SYNTAX_ERROR;
    prev = c;
    ColourChannel* ch = &jpg->channels[c];
    ch->dc_id = d[1] >> 4;
    ch->ac_id = (d[1] & 1) | 2;
    s->dc_slot[j] = ch->dc_id;
    s->ac_slot[j] = ch->ac_id;
    s->first[j] = jpg->dev->comp_first[c];
    s->sx[j] = ch->samples_x;
    s->sy[j] = ch->samples_y;
    if (ns == 1) {
      s->bw = (ch->width + 7) / 8;
      s->bh = (ch->height + 7) / 8;
    }
  }
  const unsigned char* t = p + 3 + 2 * ns;
  s->ns = ns;
  s->ss = t[0];
  s->se = t[1];
  s->ah = t[2] >> 4;
  s->al = t[2] & 15;
  if ((s->ss == 0) != (s->se == 0) || s->se > 63 || s->ss > s->se || (s->ss && ns != 1) || s->al > 13 ||
      (s->ah && s->ah != s->al + 1))
    return SYNTAX_ERROR;
  for (int j = 0; j < ns; j++) {
    const bool need_dc = s->ss == 0 && !s->ah, need_ac = s->ss != 0;
    if ((need_dc && !(jpg->huff_defined & (1 << s->dc_slot[j]))) ||
        (need_ac && !(jpg->huff_defined & (1 << s->ac_slot[j]))))
      return SYNTAX_ERROR;
  }
  jpg->pos += hlen;
  return 0;
}

// decodeScanGPU for a scan of a progressive frame: check the header, find the
// scan's restart intervals and its end (the next marker that is not RSTn),
// and queue its decode.  The first scan of the frame copies the file to the
// device and clears the coefficients.
int cj_prog_scan(JPGReader* jpg) {
  CJReaderDevice* d = jpg->dev;
  // the header first (host only, so a malformed file fails the same way
  // with or without a GPU), then the device
  for (int c = 0, k = 0; c < jpg->num_channels; c++) {
    d->comp_first[c] = k;
    k += jpg->channels[c].samples_x * jpg->channels[c].samples_y;
  }
  CJProgBlock blk;
  int err = cj_parse_prog_sos(jpg, &blk.s);
  if (err) return err;
  err = cj_gpu_init(jpg);
  if (err) return err;
  if (!d->prog_scans) cj_fill_params(jpg, (CJScanParams*)d->h_params.p);
  const CJScanParams* hp = (const CJScanParams*)d->h_params.p;
  CJProgScan& S = blk.s;
  S.bpm = hp->bpm;
  S.mcux = hp->mcux;
  S.nunits = S.ns > 1 ? hp->mcux * hp->mcuy : S.bw * S.bh;
  S.ri = jpg->restart_interval;
  S.nint = S.ri ? (S.nunits + S.ri - 1) / S.ri : 1;
  for (int slot = 0; slot < 4; slot++) {
    if (jpg->huff_defined & (1 << slot)) cj_build_huff(d->huff[slot].counts, d->huff[slot].symbols, &blk.huff[slot]);
    else memset(&blk.huff[slot], 0, sizeof(CJHuff));
  }
  // restart intervals and the end of the scan, from the stuffed bytes
  const unsigned char* base = jpg->buf;
  std::vector<int64_t> spans;
  spans.reserve(2 * (size_t)S.nint);
  spans.push_back((int64_t)(jpg->pos - base));
  unsigned char* q = jpg->pos;
  const unsigned char* lim = jpg->end;  // the EOI marker lies past it
  int expect = 0;
  for (;;) {
    q = (unsigned char*)memchr(q, 0xFF, (size_t)(lim - q));
    if (!q || q + 1 >= lim + 2) {
      q = (unsigned char*)lim;
      break;
    }
    const unsigned char m = q[1];
    if (m == 0x00) {
      q += 2;
      continue;
    }
    if ((m & 0xF8) == 0xD0) {  // RSTn: ends one interval, starts the next
      if ((m & 7) != expect || (int)(spans.size() / 2) + 1 >= S.nint) return SYNTAX_ERROR;
      expect = (expect + 1) & 7;
      spans.push_back((int64_t)(q - base));
      spans.push_back((int64_t)(q + 2 - base));
      q += 2;
      continue;
    }
    break;  // the next marker segment (or EOI)
  }
  spans.push_back((int64_t)(q - base));
  if ((int)(spans.size() / 2) != S.nint) return SYNTAX_ERROR;
  const size_t file_bytes = (size_t)(jpg->end + 2 - base);
  if (!d->prog_scans) {
    const CJScanParams* h = hp;
    d->total_blocks = h->total_blocks;
    if (cj_dev_ensure(d->raw, file_bytes + 64) || cj_dev_ensure(d->status, sizeof(CJStatus)) ||
        cj_dev_ensure(d->coef, (size_t)d->total_blocks * 128 + 128) || cj_dev_ensure(d->params, sizeof(CJScanParams)))
      return CUDA_MEM_ERROR;
    CJ_CUDA_TRY(cudaEventRecord(d->ev_begin, d->stream), CUDA_KERNEL_LAUNCH_ERROR);
    CJ_CUDA_TRY(cudaMemcpyAsync(d->raw.p, base, file_bytes, cudaMemcpyHostToDevice, d->stream), CUDA_MEM_ERROR);
    CJ_CUDA_TRY(cudaMemsetAsync(d->coef.p, 0, (size_t)d->total_blocks * 128, d->stream), CUDA_MEM_ERROR);
    CJ_CUDA_TRY(cudaMemsetAsync(d->status.p, 0, sizeof(CJStatus), d->stream), CUDA_MEM_ERROR);
    d->raw_len = file_bytes;
    d->param_bytes = 0;
    d->nkev = 0;
  }
  // the parameter block and the spans, in one stream-ordered copy: the next
  // scan's copy into the same buffer waits for this scan's kernel
  const size_t pbytes = (sizeof(CJProgBlock) + 15) & ~(size_t)15;
  const size_t bytes = pbytes + spans.size() * sizeof(int64_t);
  std::vector<uint8_t> host(bytes);
  memcpy(host.data(), &blk, sizeof(blk));
  memcpy(host.data() + pbytes, spans.data(), spans.size() * sizeof(int64_t));
  if (cj_dev_ensure(d->pscan, bytes)) return CUDA_MEM_ERROR;
  CJ_CUDA_TRY(cudaMemcpyAsync(d->pscan.p, host.data(), bytes, cudaMemcpyHostToDevice, d->stream), CUDA_MEM_ERROR);
  d->param_bytes += bytes;
  k_prog_scan<<<(S.nint + 127) / 128, 128, 0, d->stream>>>(
      (const CJProgBlock*)d->pscan.p, (const int64_t*)((const uint8_t*)d->pscan.p + pbytes),
      (const uint8_t*)d->raw.p, (int16_t*)d->coef.p, (CJStatus*)d->status.p);
  cj_after_launch(d, CJ_K_PROG_SCAN);
  CJ_CUDA_TRY(cudaGetLastError(), CUDA_KERNEL_LAUNCH_ERROR);
  d->prog_scans++;
  jpg->pos = q;  // the marker that ends the scan
  return 0;
}

// The pixel stage's parameters of a progressive frame (geometry and the
// quantisation tables; the Huffman tables are not needed after the scans),
// queued before the pixel kernel.
int cj_prog_finish(JPGReader* jpg) {
  CJReaderDevice* d = jpg->dev;
  CJScanParams* hp = (CJScanParams*)d->h_params.p;
  cj_fill_params(jpg, hp);
  CJ_CUDA_TRY(cudaMemcpyAsync(d->params.p, hp, sizeof(CJScanParams), cudaMemcpyHostToDevice, d->stream),
              CUDA_MEM_ERROR);
  CJ_CUDA_TRY(cudaEventRecord(d->ev_scan, d->stream), CUDA_KERNEL_LAUNCH_ERROR);
  return 0;
}
