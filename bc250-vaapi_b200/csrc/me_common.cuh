// me_common.cuh - pieces shared by the full-search and learned-proposal
// motion estimators: byte-SIMD SAD, block reductions, and the half/quarter-pel
// refine of A1/shaders/motion_estimation.comp (:154-215 interpolation,
// :388-459 refine order), run on an integer winner whose neighbourhood the
// caller has staged in shared memory.
#pragma once
#include "common.cuh"

namespace b200enc {

__device__ __forceinline__ uint32_t sad4_acc(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t d;
  asm("vabsdiff4.u32.u32.u32.add %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
  return d;
}

template <int NT>
__device__ __forceinline__ uint32_t block_sum(uint32_t v, uint32_t* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (NT == 32) return v;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  uint32_t s = 0;
#pragma unroll
  for (int i = 0; i < NT / 32; ++i) s += red[i];
  return s;
}

template <int NT>
__device__ __forceinline__ uint32_t block_min(uint32_t v, uint32_t* red) {
  v = __reduce_min_sync(0xffffffffu, v);
  if (NT == 32) return v;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  uint32_t m = 0xffffffffu;
#pragma unroll
  for (int i = 0; i < NT / 32; ++i) m = min(m, red[i]);
  return m;
}

// Quarter-pel sample from precomputed half-pel planes, with the letters and
// averages of motion_estimation.comp:197-213.
__device__ __forceinline__ int qpel_sample(int phase, int G, int H, int M, int b, int h, int m, int s, int j) {
  switch (phase) {
    case 0: return G;
    case 1: return (G + b + 1) >> 1;
    case 2: return b;
    case 3: return (b + H + 1) >> 1;
    case 4: return (G + h + 1) >> 1;
    case 5: return (b + h + 1) >> 1;
    case 6: return (b + j + 1) >> 1;
    case 7: return (b + m + 1) >> 1;
    case 8: return h;
    case 9: return (h + j + 1) >> 1;
    case 10: return j;
    case 11: return (j + m + 1) >> 1;
    case 12: return (h + M + 1) >> 1;
    case 13: return (h + s + 1) >> 1;
    case 14: return (j + s + 1) >> 1;
    default: return (m + s + 1) >> 1;
  }
}

// The log word a search writes into MV.pad under B200ENC_ME_LOG_INTEGER:
// bit 31 set, bit 30 = zero-MV early-out, bits 8-15 = integer winner dy +
// 128, bits 0-7 = dx + 128.
__device__ __forceinline__ uint32_t me_log_word(int mx, int my, bool early) {
  return 0x80000000u | (early ? 0x40000000u : 0u) | ((uint32_t)(my + 128) << 8) | (uint32_t)(mx + 128);
}

// Candidate offsets in quarter pels, motion_estimation.comp:395-398, :435-438.
__constant__ int8_t kHalfOff[8][2] = {{2, 0}, {-2, 0}, {0, 2}, {0, -2}, {2, 2}, {2, -2}, {-2, 2}, {-2, -2}};
__constant__ int8_t kQtrOff[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {1, -1}, {-1, 1}, {-1, -1}};

// Refine planes over coordinates relative to the integer winner: columns
// -1..16 and rows -1..16 (18 x 18); raw horizontal 6-tap sums for rows
// -3..19 (23 x 18).
struct RefineShared {
  int16_t pb[18][18], ph[18][18], pj[18][18];
  int32_t hr[23][18];
  uint32_t part[8][4];
};

// Half- then quarter-pel refine around an integer winner whose integer SAD
// is int_sad. G8(rx, ry) returns the reference pel at offset (rx, ry) from
// the winner's top-left, for rx, ry in [-3, 19]. cur: the 256 current pels
// in shared memory. Every thread of the NT-thread block calls it and gets
// the same result: (*qx, *qy) the quarter-pel offset from the winner and
// the winning SAD (strict improvement only, offsets tried in table order).
template <int NT, class G8F>
__device__ __forceinline__ uint32_t qpel_refine(RefineShared& rf, G8F G8, const uint8_t* cur, uint32_t int_sad,
                                                int* qx_out, int* qy_out) {
  const int tid = threadIdx.x;
  for (int i = tid; i < 23 * 18; i += NT) {
    const int ry = i / 18 - 3, rx = i % 18 - 1;
    rf.hr[ry + 3][rx + 1] = G8(rx - 2, ry) - 5 * G8(rx - 1, ry) + 20 * G8(rx, ry) + 20 * G8(rx + 1, ry) -
                             5 * G8(rx + 2, ry) + G8(rx + 3, ry);
  }
  __syncthreads();
  for (int i = tid; i < 18 * 18; i += NT) {
    const int ry = i / 18 - 1, rx = i % 18 - 1;
    rf.pb[ry + 1][rx + 1] = (int16_t)clip1((rf.hr[ry + 3][rx + 1] + 16) >> 5);
    const int v = G8(rx, ry - 2) - 5 * G8(rx, ry - 1) + 20 * G8(rx, ry) + 20 * G8(rx, ry + 1) -
                  5 * G8(rx, ry + 2) + G8(rx, ry + 3);
    rf.ph[ry + 1][rx + 1] = (int16_t)clip1((v + 16) >> 5);
    const int j1 = rf.hr[ry + 1][rx + 1] - 5 * rf.hr[ry + 2][rx + 1] + 20 * rf.hr[ry + 3][rx + 1] +
                   20 * rf.hr[ry + 4][rx + 1] - 5 * rf.hr[ry + 5][rx + 1] + rf.hr[ry + 6][rx + 1];
    rf.pj[ry + 1][rx + 1] = (int16_t)clip1((j1 + 512) >> 10);
  }
  __syncthreads();

  // Eight candidates at once: per-thread partial SADs, then one reduction.
  auto score8 = [&](const int8_t (*off)[2], int bx, int by, uint32_t* res) {
    uint32_t p[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) p[c] = 0;
    for (int pix = tid; pix < 256; pix += NT) {
      const int x = pix & 15, y = pix >> 4;
      const int cv = cur[y * 16 + x];
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const int ox_ = bx + off[c][0], oy_ = by + off[c][1];  // quarter-pel offset from the integer winner
        const int rx = x + (ox_ >> 2), ry = y + (oy_ >> 2);
        const int phase = (oy_ & 3) * 4 + (ox_ & 3);
        const int v = qpel_sample(phase, G8(rx, ry), G8(rx + 1, ry), G8(rx, ry + 1), rf.pb[ry + 1][rx + 1],
                                  rf.ph[ry + 1][rx + 1], rf.ph[ry + 1][rx + 2], rf.pb[ry + 2][rx + 1],
                                  rf.pj[ry + 1][rx + 1]);
        p[c] += (uint32_t)abs(cv - v);
      }
    }
#pragma unroll
    for (int c = 0; c < 8; ++c) {
#pragma unroll
      for (int o2 = 16; o2 > 0; o2 >>= 1) p[c] += __shfl_xor_sync(0xffffffffu, p[c], o2);
    }
    __syncthreads();
    if ((tid & 31) == 0)
#pragma unroll
      for (int c = 0; c < 8; ++c) rf.part[c][tid >> 5] = p[c];
    __syncthreads();
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      uint32_t s = 0;
#pragma unroll
      for (int w = 0; w < NT / 32; ++w) s += rf.part[c][w];
      res[c] = s;
    }
  };

  uint32_t cs[8];
  score8(kHalfOff, 0, 0, cs);
  uint32_t bsad = int_sad;
  int hx = 0, hy = 0;
#pragma unroll
  for (int c = 0; c < 8; ++c)
    if (cs[c] < bsad) { bsad = cs[c]; hx = kHalfOff[c][0]; hy = kHalfOff[c][1]; }
  score8(kQtrOff, hx, hy, cs);
  int qx = 0, qy = 0;
#pragma unroll
  for (int c = 0; c < 8; ++c)
    if (cs[c] < bsad) { bsad = cs[c]; qx = kQtrOff[c][0]; qy = kQtrOff[c][1]; }
  *qx_out = hx + qx;
  *qy_out = hy + qy;
  return bsad;
}

}  // namespace b200enc
