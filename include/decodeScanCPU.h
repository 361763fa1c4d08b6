/*
 * decodeScanCPU.h -- drop-in for the reference's include/decodeScanCPU.h:6.
 *
 * The reference's decodeScanCPU (src/decodeScanCPU.cu:98-152) is a serial
 * host scan decoder that nothing in its own tree calls.  This library has no
 * CPU decode path: decodeScanCPU is the same device decode as decodeScanGPU
 * (same contract: called at SOS with jpg->pos on the SOS length field,
 * errors through jpg->error), so a caller that names it links and decodes
 * on the GPU.
 */
#ifndef DECODESCANCPU_H
#define DECODESCANCPU_H

#include "format.h"

#ifdef __cplusplus
extern "C" {
#endif

void decodeScanCPU(JPGReader *jpgreader);

#ifdef __cplusplus
}
#endif
#endif /* DECODESCANCPU_H */
