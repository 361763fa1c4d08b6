/*
 * pixelTransformGPU.h -- pixel stage of libcudajpeg: iDCT, chroma
 * upsampling and YCbCr->RGB.
 *
 *   reference                                        here
 *   iDCT_resample_colourTransform  pixelTransformGPU.h:17   same name: one fused
 *       kernel (dequantise + integer iDCT + nearest upsample + colour) writes
 *       RGB / grey straight from the coefficient blocks, then one D2H copy
 *   __global__ iDCT_GPU            pixelTransformGPU.h:6-10 cjIDCTPlane: C launcher
 *       of the per-component plane iDCT, in three arithmetic forms
 */
#ifndef PIXELTRANSFORMGPU_H
#define PIXELTRANSFORMGPU_H

#include "format.h"

#ifdef __cplusplus
extern "C" {
#endif

void iDCT_resample_colourTransform(JPGReader *jpg);

/* The reference's alternative final stages (include/pixelTransformGPU.h:18-20:
 * upsampling + colour on the GPU, split between GPU and host, or on the
 * host).  Here each is the same fused GPU pixel stage as
 * iDCT_resample_colourTransform: it runs that stage if the last scan's
 * pixels are still pending, and otherwise leaves the decoded image as it is.
 * There is no host pixel path. */
void upsampleAndColourTransformHybrid(JPGReader *jpg);
void upsampleAndColourTransformGPU(JPGReader *jpg);
void upsampleAndColourTransformCPU(JPGReader *jpg);

/* Arithmetic forms of cjIDCTPlane */
#define CJ_IDCT_INT 0   /* the reference's fixed-point iDCT: bit-exact */
#define CJ_IDCT_F32 1   /* FP32 separable iDCT on CUDA cores */
#define CJ_IDCT_TC 2    /* FP16 hi+lo basis on tensor cores, FP32 accumulate */

/* iDCT of one component into a padded uint8 plane.
 *   d_coef       quantised int16 blocks, natural order, MCU-interleaved scan
 *                order (the layout decodeScanGPU leaves on the device)
 *   bpm          blocks per MCU; first: index of this component's first block
 *                inside an MCU; samples_x/y: its sampling factors
 *   mcux, mcuy   MCUs across / down
 *   d_qnat       64 int16 quantisation steps, natural order
 *   d_plane      output, `stride` bytes per row, mcuy*samples_y*8 rows
 * Returns 0 or a format.h error code. */
int cjIDCTPlane(const short *d_coef, int bpm, int first, int samples_x, int samples_y,
                int mcux, int mcuy, const short *d_qnat, unsigned char *d_plane, int stride,
                int mode, void *stream);

/* Raw iDCT values (before the +128 level shift, rounding and clipping) of
 * `nblocks` quantised int16 blocks that share the quantisation table d_qnat,
 * as FP32 [nblocks][64] (row-major 8x8): the precision measurement of the
 * CJ_IDCT_F32 and CJ_IDCT_TC forms against an FP64 iDCT.  Returns 0 or a
 * format.h error code. */
int cjIDCTBlocksRaw(const short *d_coef, long long nblocks, const short *d_qnat, float *d_out,
                    int mode, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* PIXELTRANSFORMGPU_H */
