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

// ---------------------------------------------------------------------------
// The same refine for one warp, on byte-SIMD words: the half-pel planes are
// bytes (their values are clipped to 0..255), every quarter-pel sample is
// either a plane value or the rounded byte average (a + b + 1) >> 1 of two,
// which vavgu4 forms for 4 pels at once, and vabsdiff4 accumulates the SAD.
// Results are identical to qpel_refine.
struct RefineSimd {
  alignas(4) int16_t hr[23][18];  // 6-tap sums of 8-bit samples: -2550 .. 10710
  alignas(4) uint8_t pl[3][18][20];  // b, h, j at [ry+1][rx+1], ry, rx in -1..16
};

// The operands of each quarter-pel phase (fy*4+fx), motion_estimation.comp:
// 197-213: {plane, sx, sy} twice (plane 0 G, 1 b, 2 h, 3 j, -1 none); the
// sample is the first operand or the rounded average of both.
__constant__ int8_t kQpelOp[16][6] = {
    {0, 0, 0, -1, 0, 0}, {0, 0, 0, 1, 0, 0}, {1, 0, 0, -1, 0, 0}, {1, 0, 0, 0, 1, 0},
    {0, 0, 0, 2, 0, 0},  {1, 0, 0, 2, 0, 0}, {1, 0, 0, 3, 0, 0},  {1, 0, 0, 2, 1, 0},
    {2, 0, 0, -1, 0, 0}, {2, 0, 0, 3, 0, 0}, {3, 0, 0, -1, 0, 0}, {3, 0, 0, 2, 1, 0},
    {2, 0, 0, 0, 0, 1},  {2, 0, 0, 1, 0, 1}, {3, 0, 0, 1, 0, 1},  {2, 1, 0, 1, 0, 1}};

// Two words (8 pels) of a byte row starting at byte offset c of a 4-aligned row.
__device__ __forceinline__ void row8(const uint8_t* row, int c, uint32_t& w0, uint32_t& w1) {
  const uint32_t* r = reinterpret_cast<const uint32_t*>(row) + (c >> 2);
  const int sh = (c & 3) * 8;
  const uint32_t a0 = r[0], a1 = r[1], a2 = r[2];
  w0 = __funnelshift_r(a0, a1, sh);
  w1 = __funnelshift_r(a1, a2, sh);
}

// g: 4-aligned rows of the reference, gstride bytes apart; the integer
// winner's top-left pel is at row g_r0, byte g_c0 (rows g_r0-3 .. g_r0+19
// and bytes g_c0-3 .. g_c0+19+8 must be readable). cur: the 64 words of the
// current MB. Every lane of the warp returns the same result.
__device__ __forceinline__ uint32_t qpel_refine_warp_simd(RefineSimd& rf, const uint8_t* g, int gstride, int g_r0,
                                                          int g_c0, const uint32_t* cur, uint32_t int_sad,
                                                          int* qx_out, int* qy_out) {
  const int lane = threadIdx.x & 31;
  auto G8 = [&](int rx, int ry) -> int { return g[(g_r0 + ry) * gstride + g_c0 + rx]; };
  // horizontal sums, four columns (rx .. rx+3) per lane and pass: the nine
  // bytes rx-2 .. rx+6 of the row come from three word loads; the pairs of
  // 16-bit sums are stored as words (hr rows are 36 bytes, rx+1 is 0 mod 4)
  for (int i = lane; i < 23 * 5; i += 32) {
    const int q = i / 5, ry = q - 3, rx = (i - 5 * q) * 4 - 1;
    const int bo = g_c0 + rx - 2;
    const uint32_t* wp = reinterpret_cast<const uint32_t*>(g + (g_r0 + ry) * gstride) + (bo >> 2);
    const int sh = (bo & 3) * 8;
    const uint32_t a0 = wp[0], a1 = wp[1], a2 = wp[2];
    const uint32_t lo = __funnelshift_r(a0, a1, sh), hi = __funnelshift_r(a1, a2, sh);
    int e[9];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      e[k] = (int)((lo >> (8 * k)) & 0xffu);
      e[k + 4] = (int)((hi >> (8 * k)) & 0xffu);
    }
    e[8] = (int)((a2 >> sh) & 0xffu);
    int v[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) v[j] = e[j] - 5 * e[j + 1] + 20 * e[j + 2] + 20 * e[j + 3] - 5 * e[j + 4] + e[j + 5];
    uint32_t* dst = reinterpret_cast<uint32_t*>(&rf.hr[ry + 3][rx + 1]);
    dst[0] = (uint32_t)(uint16_t)v[0] | ((uint32_t)(uint16_t)v[1] << 16);
    if (rx + 3 < 17) dst[1] = (uint32_t)(uint16_t)v[2] | ((uint32_t)(uint16_t)v[3] << 16);
  }
  __syncwarp();
  for (int i = lane; i < 18 * 18; i += 32) {
    const int ry = i / 18 - 1, rx = i % 18 - 1;
    rf.pl[0][ry + 1][rx + 1] = (uint8_t)clip1((rf.hr[ry + 3][rx + 1] + 16) >> 5);
    const int v = G8(rx, ry - 2) - 5 * G8(rx, ry - 1) + 20 * G8(rx, ry) + 20 * G8(rx, ry + 1) -
                  5 * G8(rx, ry + 2) + G8(rx, ry + 3);
    rf.pl[1][ry + 1][rx + 1] = (uint8_t)clip1((v + 16) >> 5);
    const int j1 = rf.hr[ry + 1][rx + 1] - 5 * rf.hr[ry + 2][rx + 1] + 20 * rf.hr[ry + 3][rx + 1] +
                   20 * rf.hr[ry + 4][rx + 1] - 5 * rf.hr[ry + 5][rx + 1] + rf.hr[ry + 6][rx + 1];
    rf.pl[2][ry + 1][rx + 1] = (uint8_t)clip1((j1 + 512) >> 10);
  }
  __syncwarp();

  const int y = lane >> 1, half = lane & 1;
  const uint32_t c0 = cur[y * 4 + 2 * half], c1 = cur[y * 4 + 2 * half + 1];
  // operand (plane p: 0 G, 1 b, 2 h, 3 j; extra shifts sx, sy) of the lane's
  // 8 pels at integer offset (dx, dy) from the winner
  auto operand = [&](int p, int dx, int dy, int sx, int sy, uint32_t& w0, uint32_t& w1) {
    const int ry = y + dy + sy, rx = dx + sx + 8 * half;
    if (p == 0) row8(g + (g_r0 + ry) * gstride, g_c0 + rx, w0, w1);
    else row8(&rf.pl[p - 1][ry + 1][0], rx + 1, w0, w1);
  };
  auto part = [&](int ox, int oy) -> uint32_t {  // the lane's share of the SAD at quarter-pel (ox, oy)
    const int dx = ox >> 2, dy = oy >> 2, ph = (oy & 3) * 4 + (ox & 3);
    uint32_t a0, a1;
    operand(kQpelOp[ph][0], dx, dy, kQpelOp[ph][1], kQpelOp[ph][2], a0, a1);
    if (kQpelOp[ph][3] >= 0) {
      uint32_t b0, b1;
      operand(kQpelOp[ph][3], dx, dy, kQpelOp[ph][4], kQpelOp[ph][5], b0, b1);
      a0 = __vavgu4(a0, b0);
      a1 = __vavgu4(a1, b1);
    }
    return sad4_acc(a1, c1, sad4_acc(a0, c0, 0u));
  };
  // The 8 positions (bx, by) + off[c] summed over the warp together: the
  // exchanges at distances 16, 8 and 4 each hand half of the lane's partial
  // sums to its partner, so that lane L is left with position (L >> 2) & 7,
  // and two more finish its sum. Returns min over c of (SAD_c << 3 | c): the
  // smallest SAD, the earliest position among equal ones.
  // Half-pel positions (kHalfOff order) each read one plane: b at (2,0) and
  // (-2,0), h at (0,2) and (0,-2), j at the diagonals; the integer offset is
  // -1 where the quarter-pel offset is -2. Plane and offsets are constants.
  auto half_part = [&](int c) -> uint32_t {
    const int p = c < 2 ? 1 : (c < 4 ? 2 : 3);
    const int dx = (c == 1 || c == 6 || c == 7) ? -1 : 0;
    const int dy = (c == 3 || c == 5 || c == 7) ? -1 : 0;
    uint32_t a0, a1;
    operand(p, dx, dy, 0, 0, a0, a1);
    return sad4_acc(a1, c1, sad4_acc(a0, c0, 0u));
  };
  auto best8 = [&](const int8_t(*off)[2], int bx, int by) -> uint32_t {
    uint32_t v[8];
    if (off == nullptr) {
#pragma unroll
      for (int c = 0; c < 8; ++c) v[c] = half_part(c);
    } else {
#pragma unroll
      for (int c = 0; c < 8; ++c) v[c] = part(bx + off[c][0], by + off[c][1]);
    }
    const bool h16 = lane & 16, h8 = lane & 8, h4 = lane & 4;
    uint32_t w[4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
      w[i] = (h16 ? v[i + 4] : v[i]) + __shfl_xor_sync(0xffffffffu, h16 ? v[i] : v[i + 4], 16);
    uint32_t x[2];
#pragma unroll
    for (int i = 0; i < 2; ++i)
      x[i] = (h8 ? w[i + 2] : w[i]) + __shfl_xor_sync(0xffffffffu, h8 ? w[i] : w[i + 2], 8);
    uint32_t t = (h4 ? x[1] : x[0]) + __shfl_xor_sync(0xffffffffu, h4 ? x[0] : x[1], 4);
    t += __shfl_xor_sync(0xffffffffu, t, 2);
    t += __shfl_xor_sync(0xffffffffu, t, 1);
    return __reduce_min_sync(0xffffffffu, (t << 3) | (uint32_t)((lane >> 2) & 7));
  };
  uint32_t bsad = int_sad;
  int hx = 0, hy = 0;
  const uint32_t mh = best8(nullptr, 0, 0);  // the half-pel positions, kHalfOff order
  if ((mh >> 3) < bsad) {
    bsad = mh >> 3;
    hx = kHalfOff[mh & 7][0];
    hy = kHalfOff[mh & 7][1];
  }
  int qx = 0, qy = 0;
  const uint32_t mq = best8(kQtrOff, hx, hy);
  if ((mq >> 3) < bsad) {
    bsad = mq >> 3;
    qx = kQtrOff[mq & 7][0];
    qy = kQtrOff[mq & 7][1];
  }
  *qx_out = hx + qx;
  *qy_out = hy + qy;
  return bsad;
}

}  // namespace b200enc