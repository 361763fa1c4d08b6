/*
 * ref_gputree_harness.cpp -- turns the reference's GPU-tree host code
 * (src/format.cu + src/decodeScanCPU.cu, compiled as host C++ against
 * ref_cuda_stub.h) into a coefficient oracle in oracle/_ref/libref_gputree.so.
 * TEST INFRASTRUCTURE ONLY.
 *
 * format.cu's marker loop calls decodeScanGPU at SOS (src/format.cu:195) and
 * iDCT_resample_colourTransform at EOI (:205).  Here decodeScanGPU points the
 * working Huffman tables at the parsed ones (what reshuffleHuffmanTables does
 * for the identity mapping, src/decodeScanGPU.cu:104-120) and runs the
 * reference's serial host decoder src/decodeScanCPU.cu:98-152, which handles
 * restart markers; the pixel step is left out, so channels[c].working_space
 * holds the reference's dequantised coefficients when openJPG returns.
 */
#include <stdint.h>
#include <string.h>

#include "format.h" /* include/format.h: JPGReader */
#include "decodeScanCPU.h"

void decodeScanGPU(JPGReader *jpg) {
  for (int i = 0; i < 4; i++) jpg->vlc_tables[i] = jpg->vlc_tables_backup[i];
  decodeScanCPU(jpg);
}

void iDCT_resample_colourTransform(JPGReader *) {}

extern "C" {
void *refgpu_new() { return newJPGReader(); }
void refgpu_del(void *r) { delJPGReader((JPGReader *)r); }
int refgpu_open(void *r, const char *path) { return openJPG((JPGReader *)r, path); }

/* info: width, height, nch, mcux, mcuy, restart_interval, then per component
 * c (base 6+4c): samples_x, samples_y, coefficient count, dq table id */
void refgpu_info(void *r, int *info) {
  JPGReader *j = (JPGReader *)r;
  info[0] = j->width;
  info[1] = j->height;
  info[2] = j->num_channels;
  info[3] = j->num_blocks_x;
  info[4] = j->num_blocks_y;
  info[5] = j->restart_interval;
  for (int c = 0; c < 3; c++) {
    info[6 + 4 * c] = j->channels[c].samples_x;
    info[7 + 4 * c] = j->channels[c].samples_y;
    info[8 + 4 * c] = (int)j->channels[c].working_space.size;
    info[9 + 4 * c] = j->channels[c].dq_id;
  }
}

void refgpu_coefs(void *r, int c, int32_t *out) {
  JPGReader *j = (JPGReader *)r;
  memcpy(out, j->channels[c].working_space.mem,
         (size_t)j->channels[c].working_space.size * sizeof(int32_t));
}
}
