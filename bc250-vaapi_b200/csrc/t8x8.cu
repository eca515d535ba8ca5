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
#include "t8x8.cuh"

namespace b200enc {

constexpr int kT8Blocks = 32;  // blocks per CTA
constexpr int kT8Pitch = 65;   // shared words per block (odd: the column pass is conflict-free)

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
