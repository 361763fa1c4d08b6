/*
 * decodeScanGPU.h -- scan (entropy) decode of libcudajpeg.
 *
 * Drop-in for the reference's include/decodeScanGPU.h:6.  Called by the
 * marker loop at SOS with jpg->pos on the SOS length field; on return the
 * scan's quantised coefficients are resident on the GPU (MCU scan order,
 * int16, natural order) and jpg->pos is past the entropy-coded data.
 * Errors are reported through jpg->error like the reference (THROW).
 *
 * Unlike the reference (src/decodeScanGPU.cu:435-490, a serial host decode)
 * the whole scan is decoded on the device: destuffing and restart-marker
 * search, speculative self-synchronising Huffman decode, block/DC prefix
 * scan and the run-length / zig-zag write-out.
 */
#ifndef DECODESCANGPU_H
#define DECODESCANGPU_H

#include "format.h"

#ifdef __cplusplus
extern "C" {
#endif

void decodeScanGPU(JPGReader *jpgreader);

#ifdef __cplusplus
}
#endif
#endif /* DECODESCANGPU_H */
