// cj_idct.cuh -- 8-point iDCT building blocks shared by the pixel and plane
// kernels.
#pragma once
#include <stdint.h>

// iDCT constants: 2048*sqrt(2)*cos(k*pi/16) (pixelTransformGPU.cu:10-15)
#define CJ_W1 2841
#define CJ_W2 2676
#define CJ_W3 2408
#define CJ_W5 1609
#define CJ_W6 1108
#define CJ_W7 565

__device__ __forceinline__ uint32_t cj_clip8(int x) { return x < 0 ? 0 : (x > 255 ? 255 : x); }

// Row pass, in place on 8 int32 values (pixelTransformGPU.cu:43-80).
__device__ __forceinline__ void cj_idct_row(int* d) {
  int x0 = (d[0] * 2048) + 128, x1 = d[4] * 2048, x2 = d[6], x3 = d[2];
  int x4 = d[1], x5 = d[7], x6 = d[5], x7 = d[3], x8;
  x8 = CJ_W7 * (x4 + x5);
  x4 = x8 + (CJ_W1 - CJ_W7) * x4;
  x5 = x8 - (CJ_W1 + CJ_W7) * x5;
  x8 = CJ_W3 * (x6 + x7);
  x6 = x8 - (CJ_W3 - CJ_W5) * x6;
  x7 = x8 - (CJ_W3 + CJ_W5) * x7;
  x8 = x0 + x1;
  x0 -= x1;
  x1 = CJ_W6 * (x3 + x2);
  x2 = x1 - (CJ_W2 + CJ_W6) * x2;
  x3 = x1 + (CJ_W2 - CJ_W6) * x3;
  x1 = x4 + x6;
  x4 -= x6;
  x6 = x5 + x7;
  x5 -= x7;
  x7 = x8 + x3;
  x8 -= x3;
  x3 = x0 + x2;
  x0 -= x2;
  x2 = (181 * (x4 + x5) + 128) >> 8;
  x4 = (181 * (x4 - x5) + 128) >> 8;
  d[0] = (x7 + x1) >> 8;
  d[1] = (x3 + x2) >> 8;
  d[2] = (x0 + x4) >> 8;
  d[3] = (x8 + x6) >> 8;
  d[4] = (x8 - x6) >> 8;
  d[5] = (x0 - x4) >> 8;
  d[6] = (x3 - x2) >> 8;
  d[7] = (x7 - x1) >> 8;
}

// Column pass with level shift and clip (pixelTransformGPU.cu:87-141).
__device__ __forceinline__ void cj_idct_col(const int* d, uint32_t* o) {
  int x0 = (d[0] * 256) + 8192, x1 = d[4] * 256, x2 = d[6], x3 = d[2];
  int x4 = d[1], x5 = d[7], x6 = d[5], x7 = d[3], x8;
  x8 = CJ_W7 * (x4 + x5) + 4;
  x4 = (x8 + (CJ_W1 - CJ_W7) * x4) >> 3;
  x5 = (x8 - (CJ_W1 + CJ_W7) * x5) >> 3;
  x8 = CJ_W3 * (x6 + x7) + 4;
  x6 = (x8 - (CJ_W3 - CJ_W5) * x6) >> 3;
  x7 = (x8 - (CJ_W3 + CJ_W5) * x7) >> 3;
  x8 = x0 + x1;
  x0 -= x1;
  x1 = CJ_W6 * (x3 + x2) + 4;
  x2 = (x1 - (CJ_W2 + CJ_W6) * x2) >> 3;
  x3 = (x1 + (CJ_W2 - CJ_W6) * x3) >> 3;
  x1 = x4 + x6;
  x4 -= x6;
  x6 = x5 + x7;
  x5 -= x7;
  x7 = x8 + x3;
  x8 -= x3;
  x3 = x0 + x2;
  x0 -= x2;
  x2 = (181 * (x4 + x5) + 128) >> 8;
  x4 = (181 * (x4 - x5) + 128) >> 8;
  o[0] = cj_clip8(((x7 + x1) >> 14) + 128);
  o[1] = cj_clip8(((x3 + x2) >> 14) + 128);
  o[2] = cj_clip8(((x0 + x4) >> 14) + 128);
  o[3] = cj_clip8(((x8 + x6) >> 14) + 128);
  o[4] = cj_clip8(((x8 - x6) >> 14) + 128);
  o[5] = cj_clip8(((x0 - x4) >> 14) + 128);
  o[6] = cj_clip8(((x3 - x2) >> 14) + 128);
  o[7] = cj_clip8(((x7 - x1) >> 14) + 128);
}


// Unpack 8 int16 coefficients (one 16-byte row) and dequantise them.
__device__ __forceinline__ void cj_unpack_dequant(uint4 raw, const int16_t* q, int* v) {
  v[0] = (int)(int16_t)(raw.x & 0xFFFF) * q[0];
  v[1] = (int)(int16_t)(raw.x >> 16) * q[1];
  v[2] = (int)(int16_t)(raw.y & 0xFFFF) * q[2];
  v[3] = (int)(int16_t)(raw.y >> 16) * q[3];
  v[4] = (int)(int16_t)(raw.z & 0xFFFF) * q[4];
  v[5] = (int)(int16_t)(raw.z >> 16) * q[5];
  v[6] = (int)(int16_t)(raw.w & 0xFFFF) * q[6];
  v[7] = (int)(int16_t)(raw.w >> 16) * q[7];
}

// FP32 8-point inverse DCT-II: o[x] = sum_u in[u] * basis[u*8 + x].
__device__ __forceinline__ void cj_idct8_f32(const int* in, const float* basis, float* o) {
#pragma unroll
  for (int x = 0; x < 8; x++) {
    float s = 0.f;
#pragma unroll
    for (int u = 0; u < 8; u++) s = fmaf((float)in[u], basis[u * 8 + x], s);
    o[x] = s;
  }
}

__device__ __forceinline__ void cj_idct8_f32f(const float* in, const float* basis, float* o) {
#pragma unroll
  for (int x = 0; x < 8; x++) {
    float s = 0.f;
#pragma unroll
    for (int u = 0; u < 8; u++) s = fmaf(in[u], basis[u * 8 + x], s);
    o[x] = s;
  }
}
