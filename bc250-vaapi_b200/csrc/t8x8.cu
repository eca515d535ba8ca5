// t8x8.cu - the H.264 High-profile 8x8 luma transform on the GPU: forward
// integer transform + quantisation (flat scaling lists) of residual blocks,
// and scaling + inverse transform (clause 8.5.13) + the add onto the
// prediction. The reference's encoder codes 4x4 transforms only; its decoder
// carries the inverse (A1/src/h264_recon.c:158-210, h264d_idct8_add), which
// the decoder half here reproduces bit for bit.
//
// Eight threads per 8x8 block, 32 blocks per 256-thread CTA: each thread
// transforms one row in registers, the block is transposed through shared
// memory, each thread transforms one column.
#include "b200enc_internal.h"
#include "common.cuh"

namespace b200enc {

constexpr int kT8Blocks = 32;  // blocks per CTA
constexpr int kT8Pitch = 65;   // shared words per block (odd: the column pass is conflict-free)

// normAdjust8x8 (8-318) by qp % 6 and position class, and the quantiser
// multipliers of the same classes.
__constant__ int kV8[6][6] = {{20, 18, 32, 19, 25, 24}, {22, 19, 35, 21, 28, 26}, {26, 23, 42, 24, 33, 31},
                              {28, 25, 45, 26, 35, 33}, {32, 28, 51, 30, 40, 38}, {36, 32, 58, 34, 46, 43}};
__constant__ int kMF8[6][6] = {{13107, 11428, 20972, 12222, 16777, 15481}, {11916, 10826, 19174, 11058, 14980, 14290},
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

__global__ void __launch_bounds__(8 * kT8Blocks) t8_forward_kernel(const int16_t* __restrict__ res,
                                                                   int16_t* __restrict__ lev,
                                                                   unsigned long long* __restrict__ nz, int n,
                                                                   int qp, int intra) {
  __shared__ int t[kT8Blocks][kT8Pitch];
  const int g = threadIdx.x >> 3, k = threadIdx.x & 7;
  const int b = blockIdx.x * kT8Blocks + g;
  const bool on = b < n;
  int v[8];
  if (on) {  // row k
    const uint4 w = *reinterpret_cast<const uint4*>(res + (size_t)b * 64 + 8 * k);
    const uint32_t u[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      v[2 * i] = (int)(int16_t)(u[i] & 0xffffu);
      v[2 * i + 1] = (int)(int16_t)(u[i] >> 16);
    }
    fwd8(v);
#pragma unroll
    for (int i = 0; i < 8; ++i) t[g][8 * k + i] = v[i];
  }
  __syncwarp();
  unsigned long long m = 0;
  if (on) {  // column k
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = t[g][8 * i + k];
    fwd8(v);
    const int per = qp / 6, rem = qp - 6 * per, sh = 16 + per;
    const long long f = (1ll << sh) / (intra ? 3 : 6);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const long long a = v[i] < 0 ? -(long long)v[i] : v[i];
      const int l = (int)((a * kMF8[rem][cls8(i, k)] + f) >> sh);
      const int q = v[i] < 0 ? -l : l;
      t[g][8 * i + k] = q;
      if (q) m |= 1ull << (8 * i + k);
    }
  }
  __syncwarp();
  // the block's nonzero mask: OR over its eight threads
#pragma unroll
  for (int o = 1; o < 8; o <<= 1) m |= __shfl_xor_sync(0xffffffffu, m, o);
  if (on) {  // row k of levels, one 16-byte store
    uint32_t u[4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
      u[i] = ((uint32_t)t[g][8 * k + 2 * i] & 0xffffu) | ((uint32_t)t[g][8 * k + 2 * i + 1] << 16);
    *reinterpret_cast<uint4*>(lev + (size_t)b * 64 + 8 * k) = make_uint4(u[0], u[1], u[2], u[3]);
    if (nz && k == 0) nz[b] = m;
  }
}

__global__ void __launch_bounds__(8 * kT8Blocks) t8_recon_kernel(const int16_t* __restrict__ lev,
                                                                 const int32_t* __restrict__ xy,
                                                                 uint8_t* __restrict__ plane, int pitch, int n,
                                                                 int qp) {
  __shared__ int t[kT8Blocks][kT8Pitch];
  const int g = threadIdx.x >> 3, k = threadIdx.x & 7;
  const int b = blockIdx.x * kT8Blocks + g;
  const bool on = b < n;
  const int per = qp / 6, rem = qp - 6 * per;
  int v[8];
  if (on) {  // row k: scaling (8.5.13.1), then the row transform
    const uint4 w = *reinterpret_cast<const uint4*>(lev + (size_t)b * 64 + 8 * k);
    const uint32_t u[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int c = (int)(int16_t)((u[i >> 1] >> (16 * (i & 1))) & 0xffffu);
      const int ls = 16 * kV8[rem][cls8(k, i)];
      v[i] = per >= 6 ? (c * ls) << (per - 6) : (c * ls + (1 << (5 - per))) >> (6 - per);
    }
    inv8(v);
#pragma unroll
    for (int i = 0; i < 8; ++i) t[g][8 * k + i] = v[i];
  }
  __syncwarp();
  if (on) {  // column k
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = t[g][8 * i + k];
    inv8(v);
#pragma unroll
    for (int i = 0; i < 8; ++i) t[g][8 * i + k] = v[i];
  }
  __syncwarp();
  if (on) {  // row k onto the prediction
    uint8_t* p = plane + (size_t)(xy[2 * b + 1] + k) * pitch + xy[2 * b];
#pragma unroll
    for (int i = 0; i < 8; ++i) p[i] = (uint8_t)clip1(p[i] + ((t[g][8 * k + i] + 32) >> 6));
  }
}

}  // namespace b200enc

using namespace b200enc;

extern "C" int b200enc_h264_t8_forward(const int16_t* residual, int16_t* levels, unsigned long long* nz, int n,
                                       int qp, int intra, void* stream) {
  if (!residual || !levels || n < 0 || qp < 0 || qp > 51) return -1;
  if ((((uintptr_t)residual) | ((uintptr_t)levels)) & 15) return -1;
  if (n == 0) return 0;
  t8_forward_kernel<<<(n + kT8Blocks - 1) / kT8Blocks, 8 * kT8Blocks, 0, (cudaStream_t)stream>>>(
      residual, levels, nz, n, qp, intra ? 1 : 0);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int b200enc_h264_t8_recon(const int16_t* levels, const int32_t* xy, uint8_t* plane, int pitch, int n,
                                     int qp, void* stream) {
  if (!levels || !xy || !plane || n < 0 || qp < 0 || qp > 51 || pitch < 8) return -1;
  if (((uintptr_t)levels) & 15) return -1;
  if (n == 0) return 0;
  t8_recon_kernel<<<(n + kT8Blocks - 1) / kT8Blocks, 8 * kT8Blocks, 0, (cudaStream_t)stream>>>(levels, xy, plane,
                                                                                             pitch, n, qp);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
