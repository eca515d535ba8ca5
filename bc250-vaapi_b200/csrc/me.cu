// me.cu - plain full-search block motion estimation, one CTA per 16x16 MB.
//
// Reference stage: A1/shaders/motion_estimation.comp (zero-MV early-out
// :312-331, lambda cost :363, half/quarter-pel refine :388-459 with the
// 6-tap interpolation of :154-215). The reference searches a diamond; the
// plain form here is exhaustive over [-R,R]^2 with a raster tie-break (the
// CPU oracle states the exact rule) and keeps the reference's refine.
//
// B200 layout: the (2R+24)^2 reference window (search range plus the 6-tap
// reach of the refine) is staged once in shared memory; the current MB sits
// in 64 registers per thread. Thread t owns candidate column dx = t - R and
// sweeps the window rows top to bottom: each row's 16 bytes (one funnel
// shift per word off 5 aligned shared loads) feed the SADs of the 16
// candidates that use that row, accumulated in a 16-slot ring, so every
// window byte is read once per column. SAD is the byte-SIMD
// vabsdiff4-with-add; the integer path uses no tensor cores. The column
// dx = +R is scored directly, one candidate per thread, after the sweep.
#include "common.cuh"
#include "b200enc_internal.h"

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

// Candidate offsets in quarter pels, motion_estimation.comp:395-398, :435-438.
__constant__ int8_t kHalfOff[8][2] = {{2, 0}, {-2, 0}, {0, 2}, {0, -2}, {2, 2}, {2, -2}, {-2, 2}, {-2, -2}};
__constant__ int8_t kQtrOff[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {1, -1}, {-1, 1}, {-1, -1}};

template <int R>
struct MeShared {
  static constexpr int WP = 2 * R + 24;  // window side in pels
  static constexpr int WW = WP / 4;      // 32-bit words per window row
  uint32_t win[WP * WW];
  uint32_t cur[64];
  uint32_t red[8];
  uint32_t part[8][4];
  // Refine planes over coordinates relative to the integer winner:
  // columns -1..16 and rows -1..16 (18 x 18); raw horizontal 6-tap sums
  // for rows -3..19 (23 x 18).
  int16_t pb[18][18], ph[18][18], pj[18][18];
  int32_t hr[23][18];
};

template <int R>
__global__ void __launch_bounds__(2 * R) me_full_search_kernel(const uint8_t* __restrict__ cur, int cur_pitch,
                                                               const uint8_t* __restrict__ ref, int ref_pitch,
                                                               Geo g, int lambda, int zero_thresh,
                                                               MV* __restrict__ out) {
  constexpr int NT = 2 * R;
  using S = MeShared<R>;
  constexpr int WP = S::WP, WW = S::WW, SIDE = 2 * R + 1;
  __shared__ S sh;
  const int tid = threadIdx.x;
  const int mbx = blockIdx.x, mby = blockIdx.y;
  const int X = mbx * 16, Y = mby * 16;
  const int ox = X - R - 4, oy = Y - R - 4;  // window origin (multiple of 4)

  // ---- stage the reference window (clamped) and the current MB ----------
  for (int i = tid; i < WP * WW; i += NT) {
    const int row = i / WW, w = i - row * WW;
    const int gy = clampi(oy + row, 0, g.RH - 1);
    const int gx = ox + 4 * w;
    const uint8_t* rp = ref + (size_t)gy * ref_pitch;
    uint32_t v;
    if (gx >= 0 && gx + 3 < g.RW) {
      v = __ldg(reinterpret_cast<const uint32_t*>(rp + gx));
    } else {
      v = (uint32_t)__ldg(rp + clampi(gx, 0, g.RW - 1)) | ((uint32_t)__ldg(rp + clampi(gx + 1, 0, g.RW - 1)) << 8) |
          ((uint32_t)__ldg(rp + clampi(gx + 2, 0, g.RW - 1)) << 16) |
          ((uint32_t)__ldg(rp + clampi(gx + 3, 0, g.RW - 1)) << 24);
    }
    sh.win[i] = v;
  }
  for (int i = tid; i < 64; i += NT) {
    const int r = i >> 2, w = i & 3;
    const uint8_t* cp = cur + (size_t)clampi(Y + r, 0, g.H - 1) * cur_pitch;
    const int gx = X + 4 * w;
    uint32_t v;
    if (gx + 3 < g.W) {
      v = __ldg(reinterpret_cast<const uint32_t*>(cp + gx));
    } else {
      v = (uint32_t)__ldg(cp + min(gx, g.W - 1)) | ((uint32_t)__ldg(cp + min(gx + 1, g.W - 1)) << 8) |
          ((uint32_t)__ldg(cp + min(gx + 2, g.W - 1)) << 16) | ((uint32_t)__ldg(cp + min(gx + 3, g.W - 1)) << 24);
    }
    sh.cur[i] = v;
  }
  __syncthreads();

  // ---- zero-MV check (motion_estimation.comp:312-331) --------------------
  uint32_t z = 0;
  for (int i = tid; i < 64; i += NT) {
    const int r = i >> 2, w = i & 3;
    z = sad4_acc(sh.cur[i], sh.win[(R + 4 + r) * WW + (R + 4) / 4 + w], z);
  }
  const uint32_t sad0 = block_sum<NT>(z, sh.red);
  MV* o = out + (size_t)mby * g.mbw + mbx;
  if (zero_thresh >= 0 && sad0 <= (uint32_t)zero_thresh) {
    if (tid == 0) *o = MV{0, 0, sad0, 0u};
    return;
  }

  // ---- integer full search: column sweep ---------------------------------
  uint32_t cw[16][4];
#pragma unroll
  for (int r = 0; r < 16; ++r)
#pragma unroll
    for (int w = 0; w < 4; ++w) cw[r][w] = sh.cur[r * 4 + w];

  const int dx = tid - R;
  const int col = tid + 4;  // window byte column of candidate dx
  const int wb = col >> 2, shft = (col & 3) * 8;
  const uint32_t lam_dx = (uint32_t)lambda * (uint32_t)abs(dx);
  uint32_t acc[16];
#pragma unroll
  for (int s = 0; s < 16; ++s) acc[s] = 0;
  uint32_t best = 0xffffffffu;
  constexpr int G = (2 * R + 16) / 16;
  for (int gi = 0; gi < G; ++gi) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const int wrow = gi * 16 + k;
      const uint32_t* rowp = sh.win + (4 + wrow) * WW + wb;
      const uint32_t w0 = rowp[0], w1 = rowp[1], w2 = rowp[2], w3 = rowp[3], w4 = rowp[4];
      const uint32_t r0 = __funnelshift_r(w0, w1, shft), r1 = __funnelshift_r(w1, w2, shft);
      const uint32_t r2 = __funnelshift_r(w2, w3, shft), r3 = __funnelshift_r(w3, w4, shft);
#pragma unroll
      for (int r = 0; r < 16; ++r) {
        uint32_t a = acc[(k - r) & 15];
        a = sad4_acc(r0, cw[r][0], a);
        a = sad4_acc(r1, cw[r][1], a);
        a = sad4_acc(r2, cw[r][2], a);
        a = sad4_acc(r3, cw[r][3], a);
        acc[(k - r) & 15] = a;
      }
      // slot (k+1)&15 now holds the finished candidate cy = wrow - 15
      const int cy = wrow - 15;
      const int sl = (k + 1) & 15;
      if (cy >= 0) {
        const uint32_t cost = acc[sl] + lam_dx + (uint32_t)lambda * (uint32_t)abs(cy - R);
        best = min(best, (cost << 14) | (uint32_t)(cy * SIDE + tid));
      }
      acc[sl] = 0;
    }
  }
  // column dx = +R (aligned), candidates cy = tid and, for thread 0, cy = 2R
  for (int cy = tid; cy <= 2 * R; cy += NT) {
    uint32_t s = 0;
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      const uint32_t* rowp = sh.win + (4 + cy + r) * WW + (2 * R + 4) / 4;
      s = sad4_acc(rowp[0], cw[r][0], s);
      s = sad4_acc(rowp[1], cw[r][1], s);
      s = sad4_acc(rowp[2], cw[r][2], s);
      s = sad4_acc(rowp[3], cw[r][3], s);
    }
    const uint32_t cost = s + (uint32_t)lambda * (uint32_t)(R + abs(cy - R));
    best = min(best, (cost << 14) | (uint32_t)(cy * SIDE + 2 * R));
  }
  best = block_min<NT>(best, sh.red);
  const int idx = (int)(best & 0x3fffu);
  const int mx = idx % SIDE - R, my = idx / SIDE - R;
  const uint32_t int_sad = (best >> 14) - (uint32_t)lambda * (uint32_t)(abs(mx) + abs(my));

  // ---- half-pel planes around the winner --------------------------------
  const uint8_t* wb8 = reinterpret_cast<const uint8_t*>(sh.win);
  const int px0 = mx + R + 4, py0 = my + R + 4;  // window coords of the winner
  auto G8 = [&](int rx, int ry) -> int { return wb8[(py0 + ry) * WP + px0 + rx]; };
  for (int i = tid; i < 23 * 18; i += NT) {
    const int ry = i / 18 - 3, rx = i % 18 - 1;
    sh.hr[ry + 3][rx + 1] = G8(rx - 2, ry) - 5 * G8(rx - 1, ry) + 20 * G8(rx, ry) + 20 * G8(rx + 1, ry) -
                             5 * G8(rx + 2, ry) + G8(rx + 3, ry);
  }
  __syncthreads();
  for (int i = tid; i < 18 * 18; i += NT) {
    const int ry = i / 18 - 1, rx = i % 18 - 1;
    sh.pb[ry + 1][rx + 1] = (int16_t)clip1((sh.hr[ry + 3][rx + 1] + 16) >> 5);
    const int v = G8(rx, ry - 2) - 5 * G8(rx, ry - 1) + 20 * G8(rx, ry) + 20 * G8(rx, ry + 1) -
                  5 * G8(rx, ry + 2) + G8(rx, ry + 3);
    sh.ph[ry + 1][rx + 1] = (int16_t)clip1((v + 16) >> 5);
    const int j1 = sh.hr[ry + 1][rx + 1] - 5 * sh.hr[ry + 2][rx + 1] + 20 * sh.hr[ry + 3][rx + 1] +
                   20 * sh.hr[ry + 4][rx + 1] - 5 * sh.hr[ry + 5][rx + 1] + sh.hr[ry + 6][rx + 1];
    sh.pj[ry + 1][rx + 1] = (int16_t)clip1((j1 + 512) >> 10);
  }
  __syncthreads();

  // Eight candidates at once: per-thread partial SADs, then one reduction.
  auto score8 = [&](const int8_t (*off)[2], int bx, int by, uint32_t* res) {
    uint32_t p[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) p[c] = 0;
    const uint8_t* cb = reinterpret_cast<const uint8_t*>(sh.cur);
    for (int pix = tid; pix < 256; pix += NT) {
      const int x = pix & 15, y = pix >> 4;
      const int cv = cb[y * 16 + x];
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const int ox_ = bx + off[c][0], oy_ = by + off[c][1];  // quarter-pel offset from the integer winner
        const int rx = x + (ox_ >> 2), ry = y + (oy_ >> 2);
        const int phase = (oy_ & 3) * 4 + (ox_ & 3);
        const int v = qpel_sample(phase, G8(rx, ry), G8(rx + 1, ry), G8(rx, ry + 1), sh.pb[ry + 1][rx + 1],
                                  sh.ph[ry + 1][rx + 1], sh.ph[ry + 1][rx + 2], sh.pb[ry + 2][rx + 1],
                                  sh.pj[ry + 1][rx + 1]);
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
      for (int c = 0; c < 8; ++c) sh.part[c][tid >> 5] = p[c];
    __syncthreads();
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      uint32_t s = 0;
#pragma unroll
      for (int w = 0; w < NT / 32; ++w) s += sh.part[c][w];
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
  if (tid == 0) *o = MV{4 * mx + hx + qx, 4 * my + hy + qy, bsad, 0u};
}

}  // namespace b200enc

using namespace b200enc;

extern "C" int b200enc_me_full_search(const uint8_t* cur_y, int cur_pitch, const uint8_t* ref_y, int ref_pitch,
                                      int W, int H, int RW, int RH, int range, int lambda, int zero_thresh,
                                      void* mv_out, void* stream) {
  if (!cur_y || !ref_y || !mv_out || W <= 0 || H <= 0 || RW <= 0 || RH <= 0) return -1;
  if ((cur_pitch & 3) || (ref_pitch & 3) || (((uintptr_t)cur_y) & 3) || (((uintptr_t)ref_y) & 3)) return -1;
  if (lambda < 0 || lambda > 1023) return -1;
  Geo g{W, H, RW, RH, (W + 15) / 16, (H + 15) / 16};
  dim3 grid(g.mbw, g.mbh);
  cudaStream_t st = (cudaStream_t)stream;
  switch (range) {
    case 16:
      me_full_search_kernel<16><<<grid, 32, 0, st>>>(cur_y, cur_pitch, ref_y, ref_pitch, g, lambda, zero_thresh,
                                                     (MV*)mv_out);
      break;
    case 32:
      me_full_search_kernel<32><<<grid, 64, 0, st>>>(cur_y, cur_pitch, ref_y, ref_pitch, g, lambda, zero_thresh,
                                                     (MV*)mv_out);
      break;
    default:
      return -1;
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
