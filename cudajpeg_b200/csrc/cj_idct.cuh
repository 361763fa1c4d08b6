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

// Column pass (pixelTransformGPU.cu:87-141) up to the final >> 14: the
// samples before the +128 level shift and the clip.
__device__ __forceinline__ void cj_idct_col_s(const int* d, int* o) {
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
  o[0] = (x7 + x1) >> 14;
  o[1] = (x3 + x2) >> 14;
  o[2] = (x0 + x4) >> 14;
  o[3] = (x8 + x6) >> 14;
  o[4] = (x8 - x6) >> 14;
  o[5] = (x0 - x4) >> 14;
  o[6] = (x3 - x2) >> 14;
  o[7] = (x7 - x1) >> 14;
}

// Column pass with level shift and clip.
__device__ __forceinline__ void cj_idct_col(const int* d, uint32_t* o) {
  int s[8];
  cj_idct_col_s(d, s);
#pragma unroll
  for (int j = 0; j < 8; j++) o[j] = cj_clip8(s[j] + 128);
}

// Two column-pass samples a, b -> the bytes clip(a + 128), clip(b + 128) in
// the low half (a in the low byte): a signed saturating pack to [-128, 127]
// and a flip of each byte's top bit (s + 128 == s ^ 0x80 for a signed byte).
__device__ __forceinline__ uint32_t cj_level2(int a, int b) {
  uint32_t d;
  asm("cvt.pack.sat.s8.s32.b32 %0, %1, %2, 0;" : "=r"(d) : "r"(b), "r"(a));
  return d ^ 0x8080u;
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

// The same with the quantisation factors already widened to int32.
__device__ __forceinline__ void cj_unpack_dequant32(uint4 raw, const int* q, int* v) {
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
