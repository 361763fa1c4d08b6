// format.cu -- JPGReader lifecycle, file input, marker-segment parsing and the
// openJPG driver of libcudajpeg.  Host C++; the device work is launched from
// scan.cu (entropy decode) and pixel.cu (pixel stage).
//
// The marker loop and the segment checks follow the reference's
// src/format.cu (line numbers cited per function) so that the same files
// decode and the same malformed files are rejected with the same codes.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <new>

#include "../../include/decodeScanGPU.h"
#include "../../include/format.h"
#include "../../include/pixelTransformGPU.h"
#include "cj_internal.h"

extern "C" {

unsigned short read16(const unsigned char* pos) { return (unsigned short)((pos[0] << 8) | pos[1]); }

JPGReader* newJPGReader(void) {
  // src/format.cu:12-29.  Host state only: the GPU stream and buffers are
  // created by the first scan, so headers can be parsed without a GPU.
  JPGReader* r = (JPGReader*)calloc(1, sizeof(JPGReader));
  if (!r) return NULL;
  r->dev = new (std::nothrow) CJReaderDevice();
  if (!r->dev) {
    free(r);
    return NULL;
  }
  return r;
}

void delJPGReader(JPGReader* r) {
  // src/format.cu:32-59
  if (!r) return;
  if (r->dev) {
    cj_dev_release(r->dev);
    delete r->dev;
  }
  for (int c = 0; c < 3; c++) free(r->channels[c].working_space.mem);
  free(r);
}

void printError(JPGReader* r) {
  // src/format.cu:62-78 (same text)
  printf("Code: ");
  switch (r->error) {
    case NO_ERROR: printf("NO_ERROR"); break;
    case SYNTAX_ERROR: printf("SYNTAX_ERROR"); break;
    case UNSUPPORTED_ERROR: printf("UNSUPPORTED_ERROR"); break;
    case OOM_ERROR: printf("OOM_ERROR"); break;
    case CUDA_MEM_ERROR: printf("CUDA_MEM_ERROR"); break;
    case FILE_ERROR: printf("FILE_ERROR"); break;
    case CUDA_KERNEL_LAUNCH_ERROR: printf("CUDA_KERNEL_LAUNCH_ERROR"); break;
    case PROGRAMMER_ERROR: printf("PROGRAMMER_ERROR"); break;
    default: printf("[Unrecognised error code: %d]", r->error);
  }
  if (r->error_func) printf(" Func: %s", r->error_func);
  if (r->error_file) printf(" File: %s", r->error_file);
  if (r->error_line) printf(" Line: %d", r->error_line);
}

void writeJPG(JPGReader* r, const char* filename) {
  // src/format.cu:218-229: binary PPM (colour) or PGM (grey)
  FILE* f = fopen(filename, "wb");
  if (!f) {
    printf("Couldn't open output file %s\n", filename);
    return;
  }
  fprintf(f, "P%d\n%d %d\n255\n", (r->num_channels > 1) ? 6 : 5, r->width, r->height);
  const unsigned char* px = (r->num_channels == 1) ? r->channels[0].pixels.mem : r->pixels;
  if (px) fwrite(px, 1, (size_t)r->width * r->height * r->num_channels, f);
  fclose(f);
}

// A segment's two length bytes must lie inside the file (the reference reads
// them unchecked; a truncated file would read past its buffer).
static int seg_len_ok(JPGReader* jpg) { return jpg->pos + 2 <= jpg->end + 2; }

void skipBlock(JPGReader* jpg) {
  // src/format.cu:237-239
  if (!seg_len_ok(jpg)) THROW(SYNTAX_ERROR);
  jpg->pos += read16(jpg->pos);
}

void decodeSOF(JPGReader* jpg) {
  // src/format.cu:242-354 (checks and geometry; output buffers are sized
  // by the pixel stage)
  if (!seg_len_ok(jpg)) THROW(SYNTAX_ERROR);
  unsigned char* block = jpg->pos;
  unsigned int block_len = read16(block);
  if (block_len < 9 || block + block_len >= jpg->end) THROW(SYNTAX_ERROR);
  if (block[2] != 8) THROW(UNSUPPORTED_ERROR);
  jpg->height = read16(block + 3);
  jpg->width = read16(block + 5);
  if (!jpg->width || !jpg->height) THROW(SYNTAX_ERROR);
  jpg->num_channels = block[7];
  if (jpg->num_channels != 1 && jpg->num_channels != 3) THROW(UNSUPPORTED_ERROR);
  if (block_len < 8u + jpg->num_channels * 3u) THROW(SYNTAX_ERROR);
  block += 8;
  int sx_max = 0, sy_max = 0;
  for (int i = 0; i < jpg->num_channels; i++, block += 3) {
    ColourChannel* ch = &jpg->channels[i];
    ch->id = block[0];
    ch->samples_x = block[1] >> 4;
    ch->samples_y = block[1] & 0xF;
    ch->dq_id = block[2];
    if (!ch->samples_x || !ch->samples_y || ch->dq_id > 3) THROW(SYNTAX_ERROR);
    if ((ch->samples_x & (ch->samples_x - 1)) || (ch->samples_y & (ch->samples_y - 1)))
      THROW(UNSUPPORTED_ERROR);  // powers of two only
    if (ch->samples_x > sx_max) sx_max = ch->samples_x;
    if (ch->samples_y > sy_max) sy_max = ch->samples_y;
  }
  if (jpg->num_channels == 1) {
    jpg->channels[0].samples_x = sx_max = 1;
    jpg->channels[0].samples_y = sy_max = 1;
  }
  jpg->block_size_x = (unsigned short)(sx_max << 3);
  jpg->block_size_y = (unsigned short)(sy_max << 3);
  jpg->num_blocks_x = (unsigned short)((jpg->width + jpg->block_size_x - 1) / jpg->block_size_x);
  jpg->num_blocks_y = (unsigned short)((jpg->height + jpg->block_size_y - 1) / jpg->block_size_y);
  int bpm = 0;
  for (int i = 0; i < jpg->num_channels; i++) {
    ColourChannel* ch = &jpg->channels[i];
    ch->width = (jpg->width * ch->samples_x + sx_max - 1) / sx_max;
    ch->height = (jpg->height * ch->samples_y + sy_max - 1) / sy_max;
    ch->stride = jpg->num_blocks_x * (ch->samples_x << 3);
    ch->block_stride = jpg->num_blocks_y * (ch->samples_y << 3);
    ch->num_blocks = jpg->num_blocks_x * ch->samples_x * jpg->num_blocks_y * ch->samples_y;
    ch->dc_cumulative_val = 0;
    if ((ch->width < 3 && ch->samples_x != sx_max) || (ch->height < 3 && ch->samples_y != sy_max))
      THROW(UNSUPPORTED_ERROR);
    bpm += ch->samples_x * ch->samples_y;
  }
  // A larger MCU than the device tables hold (the standard allows 10 blocks).
  if (bpm > CJ_MAX_BPM) THROW(UNSUPPORTED_ERROR);
  if (jpg->num_channels == 3) {
    if (jpg->channels[1].width != jpg->channels[2].width ||
        jpg->channels[1].height != jpg->channels[2].height ||
        jpg->channels[0].width != jpg->width || jpg->channels[0].height != jpg->height)
      THROW(UNSUPPORTED_ERROR);
  }
  jpg->pos += block_len;
}

void decodeDHT(JPGReader* jpg) {
  // src/format.cu:357-400: the same validity checks; the table is kept in
  // canonical (BITS, HUFFVAL) form and packed for the device at SOS.
  if (!seg_len_ok(jpg)) THROW(SYNTAX_ERROR);
  unsigned char* pos = jpg->pos;
  unsigned int block_len = read16(pos);
  unsigned char* block_end = pos + block_len;
  if (block_end > jpg->end) THROW(SYNTAX_ERROR);
  pos += 2;
  while (pos < block_end) {
    unsigned char val = pos[0];
    if (val & 0xEC) THROW(SYNTAX_ERROR);
    if (val & 0x02) THROW(UNSUPPORTED_ERROR);
    int slot = (val | (val >> 3)) & 3;  // DC0, DC1, AC0, AC1
    if (pos + 17 > block_end) THROW(SYNTAX_ERROR);
    const unsigned char* sym = pos + 17;
    int remain = 65536, nsym = 0;
    for (int l = 1; l <= 16; l++) {
      int count = pos[l];
      if (!count) continue;
      if (sym + nsym + count > block_end) THROW(SYNTAX_ERROR);
      remain -= count << (16 - l);
      if (remain < 0) THROW(SYNTAX_ERROR);
      nsym += count;
    }
    // HUFFVAL holds at most 256 symbols (ITU T.81 B.2.4.2)
    if (nsym > 256) THROW(UNSUPPORTED_ERROR);
    CJHostHuff* h = &jpg->dev->huff[slot];
    memcpy(h->counts, pos + 1, 16);
    memcpy(h->symbols, sym, nsym);
    h->nsym = nsym;
    jpg->huff_defined |= 1 << slot;
    pos = (unsigned char*)sym + nsym;
  }
  if (pos != block_end) THROW(SYNTAX_ERROR);
  jpg->pos = block_end;
}

void decodeDRI(JPGReader* jpg) {
  // src/format.cu:404-421
  if (!seg_len_ok(jpg)) THROW(SYNTAX_ERROR);
  unsigned int block_len = read16(jpg->pos);
  unsigned char* block_end = jpg->pos + block_len;
  if (block_len < 2 || block_end > jpg->end) THROW(SYNTAX_ERROR);
  if (block_len < 4) THROW(SYNTAX_ERROR);  // the interval field itself
  jpg->restart_interval = read16(jpg->pos + 2);
  jpg->pos = block_end;
}

void decodeDQT(JPGReader* jpg) {
  // src/format.cu:424-442 for 8-bit tables.  16-bit tables (Pq = 1, ITU
  // T.81 B.2.4.1: 64 big-endian values), which the reference rejects through
  // its id check, are read as well; their values must stay below 2^15 (the
  // largest step the IJG encoder writes).  dq_tables keeps the reference's
  // 8-bit view (a 16-bit value saturates there); the decoder uses the
  // tables as parsed.
  if (!seg_len_ok(jpg)) THROW(SYNTAX_ERROR);
  unsigned int block_len = read16(jpg->pos);
  unsigned char* block_end = jpg->pos + block_len;
  if (block_end > jpg->end) THROW(SYNTAX_ERROR);
  unsigned char* pos = jpg->pos + 2;
  while (pos < block_end) {
    const int pq = pos[0] >> 4, id = pos[0] & 15;
    const int n = pq ? 129 : 65;
    if (pq > 1 || id > 3 || pos + n > block_end) THROW(SYNTAX_ERROR);
    for (int k = 0; k < 64; k++) {
      const unsigned v = pq ? read16(pos + 1 + 2 * k) : pos[1 + k];
      if (v > 32767) THROW(UNSUPPORTED_ERROR);
      jpg->dev->dq16[id][k] = (uint16_t)v;
      jpg->dq_tables[id][k] = (unsigned char)(v > 255 ? 255 : v);
    }
    pos += n;
  }
  if (pos != block_end) THROW(SYNTAX_ERROR);
  jpg->pos = block_end;
}

// The marker loop of src/format.cu:159-215 over a file image in memory.
// With stop_at_scan the loop returns 0 after the SOS header has been checked
// (jpg->pos = first entropy-coded byte, jpg->end = last byte before EOI)
// without launching any device work: the batch decoder's host parse.
static int cj_marker_loop(JPGReader* r, unsigned char* buf, size_t size, bool stop_at_scan) {
  r->error = NO_ERROR;
  r->error_line = 0;
  r->error_file = r->error_func = NULL;
  if (size < 4 || buf[0] != 0xFF || buf[1] != 0xD8 || buf[size - 2] != 0xFF ||
      buf[size - 1] != 0xD9)
    return r->error = FILE_ERROR;
  if (size < 6) return r->error = SYNTAX_ERROR;
  r->buf = buf;
  r->end = buf + size - 2;  // leave out the EOI marker, already checked
  r->pos = buf + 2;
  r->restart_interval = 0;
  r->num_blocks_x = r->num_blocks_y = 0;
  r->num_channels = 0;
  r->time = 0;
  r->scan_seen = 0;
  r->dev->progressive = false;
  r->dev->prog_scans = 0;
  while (!r->error) {
    if (r->pos > r->end || r->pos[0] != 0xFF) {
      r->error = SYNTAX_ERROR;
      break;
    }
    r->pos += 2;
    switch (r->pos[-1]) {
      case 0xC0: decodeSOF(r); break;
      case 0xC2:  // progressive (ITU T.81 Annex G; the reference rejects it)
        r->dev->progressive = true;
        decodeSOF(r);
        break;
      case 0xC4: decodeDHT(r); break;
      case 0xDB: decodeDQT(r); break;
      case 0xDD: decodeDRI(r); break;
      case 0xDA:
        if (stop_at_scan) {
          if (r->dev->progressive) {
            // the batch decoder takes baseline frames only: a valid
            // progressive scan is unsupported there, an invalid one a
            // syntax error as for the marker loop
            CJProgScan ps;
            int e = cj_parse_prog_sos(r, &ps);
            return r->error = e ? e : UNSUPPORTED_ERROR;
          }
          int e = cj_parse_sos(r);
          if (!e) r->scan_seen = 1;
          return r->error = e;
        }
        decodeScanGPU(r);
        break;
      case 0xFE: skipBlock(r); break;
      case 0xD9: break;
      default:
        if ((r->pos[-1] & 0xF0) == 0xE0) skipBlock(r);
        else r->error = SYNTAX_ERROR;
    }
    if (r->error) break;
    // a skipped segment that ran past the file: the next marker read fails
    // (checked here, so the byte before pos -- at most the EOI's last byte,
    // end + 1 -- is inside the file)
    if (r->pos > r->end + 2) {
      r->error = SYNTAX_ERROR;
      break;
    }
    if (r->pos[-1] == 0xD9) {
      // EOI (or a segment that happens to end on byte 0xD9, which the
      // reference also takes as the end of the file, src/format.cu:204)
      if (!r->scan_seen) {
        r->error = SYNTAX_ERROR;
        r->error_func = (char*)"openJPG: end of image before any scan";
        break;
      }
      iDCT_resample_colourTransform(r);
      break;
    }
  }
  return r->error;
}

static int cj_parse_and_decode(JPGReader* r, unsigned char* buf, size_t size) {
  return cj_marker_loop(r, buf, size, false);
}

int cj_parse_to_scan(JPGReader* r, const unsigned char* buf, size_t size) {
  int e = cj_marker_loop(r, (unsigned char*)buf, size, true);
  if (!e && !r->scan_seen) e = r->error = SYNTAX_ERROR;  // EOI before any scan
  return e;
}

int openJPGMem(JPGReader* r, const unsigned char* data, size_t size) {
  // The bytes are parsed in place and never written; for the fastest
  // host->device copy they should be in pinned memory.
  if (!r) return PROGRAMMER_ERROR;
  return cj_parse_and_decode(r, (unsigned char*)data, size);
}

int openJPG(JPGReader* r, const char* filename) {
  // src/format.cu:113-157: read the whole file, then parse it.  The file is
  // read into the reader's pinned buffer so its scan can be copied to the
  // GPU without staging.
  if (!r) return PROGRAMMER_ERROR;
  FILE* f = fopen(filename, "rb");
  if (!f) return r->error = FILE_ERROR;
  fseek(f, 0, SEEK_END);
  long size = ftell(f);
  fseek(f, 0, SEEK_SET);
  if (size <= 0) {
    fclose(f);
    return r->error = FILE_ERROR;
  }
  int err = cj_gpu_init(r);
  if (err) {
    fclose(f);
    return r->error = err;
  }
  if (cj_host_ensure(r->dev->h_file, (size_t)size + 16)) {
    fclose(f);
    return r->error = OOM_ERROR;
  }
  unsigned char* buf = (unsigned char*)r->dev->h_file.p;
  size_t got = fread(buf, 1, (size_t)size, f);
  fclose(f);
  if (got != (size_t)size) return r->error = FILE_ERROR;
  memset(buf + size, 0, 16);
  r->file_buf.mem = buf;
  r->file_buf.size = (unsigned int)size;
  r->file_buf.max_size = (unsigned int)r->dev->h_file.cap;
  return cj_parse_and_decode(r, buf, (size_t)size);
}

}  // extern "C"
