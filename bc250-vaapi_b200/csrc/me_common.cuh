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

// The log word a search writes into MV.pad under B200ENC_ME_LOG_INTEGER:
// bit 31 set, bit 30 = zero-MV early-out, bits 8-15 = integer winner dy +
// 128, bits 0-7 = dx + 128.
__device__ __forceinline__ uint32_t me_log_word(int mx, int my, bool early) {
  return 0x80000000u | (early ? 0x40000000u : 0u) | ((uint32_t)(my + 128) << 8) | (uint32_t)(mx + 128);
}

// Candidate offsets in quarter pels, motion_estimation.comp:395-398, :435-438.
__constant__ int8_t kHalfOff[8][2] = {{2, 0}, {-2, 0}, {0, 2}, {0, -2}, {2, 2}, {2, -2}, {-2, 2}, {-2, -2}};
__constant__ int8_t kQtrOff[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {1, -1}, {-1, 1}, {-1, -1}};

// One 32-bit word of a reference row (4 pels from gx), with the column
// clamped to [0, RW-1] per pel when the word leaves the plane.
__device__ __forceinline__ uint32_t load_word_clamped(const uint8_t* row, int gx, int RW) {
  if (gx >= 0 && gx + 3 < RW) return __ldg(reinterpret_cast<const uint32_t*>(row + gx));
  return (uint32_t)__ldg(row + clampi(gx, 0, RW - 1)) | ((uint32_t)__ldg(row + clampi(gx + 1, 0, RW - 1)) << 8) |
         ((uint32_t)__ldg(row + clampi(gx + 2, 0, RW - 1)) << 16) |
         ((uint32_t)__ldg(row + clampi(gx + 3, 0, RW - 1)) << 24);
}

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
// With NT == 32 the caller may be one warp of a larger block: only the warp
// synchronises, and the sums come from shuffles alone.
template <int NT, class G8F>
__device__ __forceinline__ uint32_t qpel_refine(RefineShared& rf, G8F G8, const uint8_t* cur, uint32_t int_sad,
                                                int* qx_out, int* qy_out) {
  const int tid = NT == 32 ? (int)(threadIdx.x & 31) : (int)threadIdx.x;
  for (int i = tid; i < 23 * 18; i += NT) {
    const int ry = i / 18 - 3, rx = i % 18 - 1;
    rf.hr[ry + 3][rx + 1] = G8(rx - 2, ry) - 5 * G8(rx - 1, ry) + 20 * G8(rx, ry) + 20 * G8(rx + 1, ry) -
                             5 * G8(rx + 2, ry) + G8(rx + 3, ry);
  }
  if (NT == 32) __syncwarp(); else __syncthreads();
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
  if (NT == 32) __syncwarp(); else __syncthreads();

  // One quarter-pel sample at offset (rx, ry) from the winner with phase
  // (fy*4 + fx); the letters and averages of motion_estimation.comp:197-213,
  // loading only the operands the phase uses (phase is uniform per call).
  auto sample = [&](int phase, int rx, int ry) -> int {
    switch (phase) {
      case 0: return G8(rx, ry);
      case 1: return (G8(rx, ry) + rf.pb[ry + 1][rx + 1] + 1) >> 1;
      case 2: return rf.pb[ry + 1][rx + 1];
      case 3: return (rf.pb[ry + 1][rx + 1] + G8(rx + 1, ry) + 1) >> 1;
      case 4: return (G8(rx, ry) + rf.ph[ry + 1][rx + 1] + 1) >> 1;
      case 5: return (rf.pb[ry + 1][rx + 1] + rf.ph[ry + 1][rx + 1] + 1) >> 1;
      case 6: return (rf.pb[ry + 1][rx + 1] + rf.pj[ry + 1][rx + 1] + 1) >> 1;
      case 7: return (rf.pb[ry + 1][rx + 1] + rf.ph[ry + 1][rx + 2] + 1) >> 1;
      case 8: return rf.ph[ry + 1][rx + 1];
      case 9: return (rf.ph[ry + 1][rx + 1] + rf.pj[ry + 1][rx + 1] + 1) >> 1;
      case 10: return rf.pj[ry + 1][rx + 1];
      case 11: return (rf.pj[ry + 1][rx + 1] + rf.ph[ry + 1][rx + 2] + 1) >> 1;
      case 12: return (rf.ph[ry + 1][rx + 1] + G8(rx, ry + 1) + 1) >> 1;
      case 13: return (rf.ph[ry + 1][rx + 1] + rf.pb[ry + 2][rx + 1] + 1) >> 1;
      case 14: return (rf.pj[ry + 1][rx + 1] + rf.pb[ry + 2][rx + 1] + 1) >> 1;
      default: return (rf.ph[ry + 1][rx + 2] + rf.pb[ry + 2][rx + 1] + 1) >> 1;
    }
  };

  // Eight candidates, one at a time: per-thread partial SADs, then a block
  // (or warp) reduction per candidate.
  auto score8 = [&](const int8_t (*off)[2], int bx, int by, uint32_t* res) {
    for (int c = 0; c < 8; ++c) {
      const int ox_ = bx + off[c][0], oy_ = by + off[c][1];  // quarter-pel offset from the integer winner
      const int dx = ox_ >> 2, dy = oy_ >> 2, phase = (oy_ & 3) * 4 + (ox_ & 3);
      uint32_t p = 0;
      for (int pix = tid; pix < 256; pix += NT) {
        const int x = pix & 15, y = pix >> 4;
        p += (uint32_t)abs((int)cur[pix] - sample(phase, x + dx, y + dy));
      }
#pragma unroll
      for (int o2 = 16; o2 > 0; o2 >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o2);
      res[c] = p;
      if (NT > 32 && (tid & 31) == 0) rf.part[c][tid >> 5] = p;
    }
    if (NT == 32) return;
    __syncthreads();
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      uint32_t sum = 0;
#pragma unroll
      for (int w = 0; w < NT / 32; ++w) sum += rf.part[c][w];
      res[c] = sum;
    }
    __syncthreads();  // part[] is rewritten by the next call
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
