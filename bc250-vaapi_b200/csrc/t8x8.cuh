// t8x8.cuh - the H.264 High-profile 8x8 luma transform's device pieces
// (the core transform pair of clause 8.5.13.2, the quantiser and scaling
// classes of flat scaling lists), shared by the stage kernels (t8x8.cu) and
// the P chain's 8x8 form (pframe.cu).
#pragma once
#include "common.cuh"

namespace b200enc {

// normAdjust8x8 (8-318) by qp % 6 and position class, and the quantiser
// multipliers of the same classes.
static __constant__ int kV8[6][6] = {{20, 18, 32, 19, 25, 24}, {22, 19, 35, 21, 28, 26}, {26, 23, 42, 24, 33, 31},
                              {28, 25, 45, 26, 35, 33}, {32, 28, 51, 30, 40, 38}, {36, 32, 58, 34, 46, 43}};
static __constant__ int kMF8[6][6] = {{13107, 11428, 20972, 12222, 16777, 15481}, {11916, 10826, 19174, 11058, 14980, 14290},
                               {10082, 8943, 15978, 9675, 12710, 11985},   {9362, 8228, 14913, 8931, 11984, 11259},
                               {8192, 7346, 13159, 7740, 10486, 9777},     {7282, 6428, 11570, 6830, 9118, 8640}};

__device__ __forceinline__ int cls8(int i, int j) {
  if ((i & 3) == 0 && (j & 3) == 0) return 0;
  if ((i & 1) && (j & 1)) return 1;
  if ((i & 3) == 2 && (j & 3) == 2) return 2;
  if (((i & 3) == 0 && (j & 1)) || ((i & 1) && (j & 3) == 0)) return 3;
  if (((i & 3) == 0 && (j & 3) == 2) || ((i & 3) == 2 && (j & 3) == 0)) return 4;
  return 5;
}

// Forward 1-D transform of eight values (the core transform whose inverse is
// 8.5.13.2).
__device__ __forceinline__ void fwd8(int (&s)[8]) {
  const int a0 = s[0] + s[7], a1 = s[1] + s[6], a2 = s[2] + s[5], a3 = s[3] + s[4];
  const int b0 = a0 + a3, b1 = a1 + a2, b2 = a0 - a3, b3 = a1 - a2;
  const int a4 = s[0] - s[7], a5 = s[1] - s[6], a6 = s[2] - s[5], a7 = s[3] - s[4];
  const int b4 = a5 + a6 + ((a4 >> 1) + a4), b5 = a4 - a7 - ((a6 >> 1) + a6);
  const int b6 = a4 + a7 - ((a5 >> 1) + a5), b7 = a5 - a6 + ((a7 >> 1) + a7);
  s[0] = b0 + b1;
  s[4] = b0 - b1;
  s[2] = b2 + (b3 >> 1);
  s[6] = (b2 >> 1) - b3;
  s[1] = b4 + (b7 >> 2);
  s[7] = (b4 >> 2) - b7;
  s[3] = b5 + (b6 >> 2);
  s[5] = b6 - (b5 >> 2);
}

// Unnormalised 8-point Walsh-Hadamard transform (butterflies, natural order
// of the butterfly network; a cost measure only).
__device__ __forceinline__ void had8(int (&v)[8]) {
#pragma unroll
  for (int h = 1; h < 8; h <<= 1)
#pragma unroll
    for (int i = 0; i < 8; i += 2 * h)
#pragma unroll
      for (int j = i; j < i + h; ++j) {
        const int a = v[j], b = v[j + h];
        v[j] = a + b;
        v[j + h] = a - b;
      }
}

// Inverse 1-D transform of eight values (8.5.13.2).
__device__ __forceinline__ void inv8(int (&d)[8]) {
  const int a0 = d[0] + d[4], a2 = d[0] - d[4];
  const int a4 = (d[2] >> 1) - d[6], a6 = (d[6] >> 1) + d[2];
  const int b0 = a0 + a6, b2 = a2 + a4, b4 = a2 - a4, b6 = a0 - a6;
  const int a1 = -d[3] + d[5] - d[7] - (d[7] >> 1);
  const int a3 = d[1] + d[7] - d[3] - (d[3] >> 1);
  const int a5 = -d[1] + d[7] + d[5] + (d[5] >> 1);
  const int a7 = d[3] + d[5] + d[1] + (d[1] >> 1);
  const int b1 = (a7 >> 2) + a1, b3 = a3 + (a5 >> 2), b5 = (a3 >> 2) - a5, b7 = a7 - (a1 >> 2);
  d[0] = b0 + b7;
  d[7] = b0 - b7;
  d[1] = b2 + b5;
  d[6] = b2 - b5;
  d[2] = b4 + b3;
  d[5] = b4 - b3;
  d[3] = b6 + b1;
  d[4] = b6 - b1;
}

// 8x8 frame zig-zag scan (raster positions), Table 8-13: CAVLC carries an 8x8
// block as four 4x4 blocks, block i taking scan positions i, i + 4, ...
static __constant__ uint8_t kZigzag8[64] = {0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,
                                            12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6,  7,  14, 21, 28,
                                            35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
                                            58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

// Position in that scan of each raster position.
static __constant__ uint8_t kZigzag8Inv[64] = {0,  1,  5,  6,  14, 15, 27, 28, 2,  4,  7,  13, 16, 26, 29, 42,
                                               3,  8,  12, 17, 25, 30, 41, 43, 9,  11, 18, 24, 31, 40, 44, 53,
                                               10, 19, 23, 32, 39, 45, 52, 54, 20, 22, 33, 38, 46, 51, 55, 60,
                                               21, 34, 37, 47, 50, 56, 59, 61, 35, 36, 48, 49, 57, 58, 62, 63};

// Quantisation of one transformed coefficient at (row i, column j).
__device__ __forceinline__ int quant8(int c, int i, int j, int rem, int sh, long long f) {
  const long long a = c < 0 ? -(long long)c : c;
  const int l = (int)((a * kMF8[rem][cls8(i, j)] + f) >> sh);
  return c < 0 ? -l : l;
}

// Scaling (8.5.13.1, flat lists) of one level at (row i, column j).
__device__ __forceinline__ int scale8(int c, int i, int j, int per, int rem) {
  const int ls = 16 * kV8[rem][cls8(i, j)];
  return per >= 6 ? (c * ls) << (per - 6) : (c * ls + (1 << (5 - per))) >> (6 - per);
}

}  // namespace b200enc
