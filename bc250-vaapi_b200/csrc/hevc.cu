// hevc.cu - HEVC encoder primitives the reference's host RD loop calls per
// block, as batched GPU kernels:
//   H1  half-sample planes of the previous reconstruction for the motion
//       search (approach1-compute-encoder/src/hevc_enc_template.c:312-400,
//       build_hpel / hpel_pass): the whole-sample plane and the H, V and HV
//       planes of the 8-tap filter -1 4 -11 40 40 -11 4 -1, with a margin;
//   H2  8x8 CU motion search on those planes (search_sad :463, motion_search
//       :958);
//   H3  4x4 intra luma mode choice (hevc_intra_template.c:177);
//   H1-H3 at 8 bits and at 10 (Main10): the reference builds its template
//       twice (encoder_h265.c:1220-1227, hevc_intra.c), changing only the
//       sample type, the clip value, the no-neighbour fill and the search
//       SAD's scaling to eight-bit units;
//   H4  forward transform + quantisation of 4x4 (DCT-II or DST-VII) and 8x8
//       (DCT-II) residual blocks at 8 or 10 bits (hevc_intra.c:468, :565, :720);
//   H5  dequantisation + inverse transform of the same blocks
//       (hevc_intra.c:484, :586, :761).
// Arithmetic is the reference's compiled (SSE2) path: both transform passes
// round, shift and saturate to int16 exactly where its packs instructions
// do; the quantiser divides by levelScale through the same reciprocal
// multiply, which is exact over the reachable range.
#include <algorithm>

#include "b200enc_internal.h"
#include "common.cuh"

namespace b200enc {

// H.265 transform matrices and levelScale (standard constants; the decoder
// uses the same values).
__constant__ int16_t kHDct4[4][4] = {{64, 64, 64, 64}, {83, 36, -36, -83}, {64, -64, -64, 64}, {36, -83, 83, -36}};
__constant__ int16_t kHDst4[4][4] = {{29, 55, 74, 84}, {74, 74, 0, -74}, {84, -29, -74, 55}, {55, -84, 74, -29}};
__constant__ int16_t kHDct8[8][8] = {{64, 64, 64, 64, 64, 64, 64, 64},     {89, 75, 50, 18, -18, -50, -75, -89},
                                     {83, 36, -36, -83, -83, -36, 36, 83}, {75, -18, -89, -50, 50, 89, 18, -75},
                                     {64, -64, -64, 64, 64, -64, -64, 64}, {50, -89, 18, 75, -75, -18, 89, -50},
                                     {36, -83, 83, -36, -36, 83, -83, 36}, {18, -50, 75, -89, 89, -75, 50, -18}};
__constant__ int kHLevelScale[6] = {40, 45, 51, 57, 64, 72};

__device__ __forceinline__ int sat16(int v) { return v > 32767 ? 32767 : (v < -32768 ? -32768 : v); }

// Quantiser parameters of one QP: level = ((|x| << shift) + offset) >> p,
// then * m >> 32 (division by levelScale), capped at 32767, sign restored.
struct HQuant {
  int shift, p;
  uint32_t offset, m;
};

__device__ __forceinline__ HQuant hquant(int q, int shift, int round_q12) {
  HQuant h;
  h.shift = shift;
  h.p = q / 6 + 4;
  const uint32_t d = (uint32_t)kHLevelScale[q % 6];
  h.offset = (uint32_t)((((uint64_t)d << h.p) * (uint64_t)round_q12) / 12u);
  h.m = (uint32_t)((((uint64_t)1 << 32) + d - 1) / d);
  return h;
}

__device__ __forceinline__ int16_t hquant_level(int x, const HQuant& h) {
  const uint32_t mag = (uint32_t)(x < 0 ? -x : x);
  const uint32_t t = ((mag << h.shift) + h.offset) >> h.p;
  uint32_t l = (uint32_t)(((uint64_t)t * h.m) >> 32);
  if (l > 32767u) l = 32767u;
  return (int16_t)(x < 0 ? -(int)l : (int)l);
}

// Dequantisation, flat scaling list (8.6.3): level * levelScale << (q/6+4),
// rounded and shifted down by bd_shift, saturated to int16.
__device__ __forceinline__ int hdequant(int c, int q, int bd_shift) {
  const int a = q / 6 + 4, ls = kHLevelScale[q % 6];
  const int prod = c * ls;
  int v;
  if (a >= bd_shift) v = (int)((uint32_t)prod << (a - bd_shift));
  else v = (prod + (1 << (bd_shift - a - 1))) >> (bd_shift - a);
  return sat16(v);
}

// ---- 4x4 -------------------------------------------------------------------
__global__ void hevc_tq4_kernel(const int16_t* __restrict__ res, int16_t* __restrict__ out, int n, int q, int use_dst,
                                int round_q12, int s1, int qshift) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  const int16_t(*M)[4] = use_dst ? kHDst4 : kHDct4;
  int x[16];
  const int4* src = reinterpret_cast<const int4*>(res + (size_t)b * 16);
  const int4 v0 = src[0], v1 = src[1];
  const int w[8] = {v0.x, v0.y, v0.z, v0.w, v1.x, v1.y, v1.z, v1.w};
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    x[2 * i] = (int)(int16_t)(w[i] & 0xffff);
    x[2 * i + 1] = (int)(int16_t)((uint32_t)w[i] >> 16);
  }
  // an all-zero block gives all-zero levels whatever the rounding offset
  // (with a full-step offset the quantiser alone would give 1s)
  if (!(v0.x | v0.y | v0.z | v0.w | v1.x | v1.y | v1.z | v1.w)) {
    int4* dst = reinterpret_cast<int4*>(out + (size_t)b * 16);
    dst[0] = dst[1] = make_int4(0, 0, 0, 0);
    return;
  }
  int t[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      int s = 0;
#pragma unroll
      for (int r = 0; r < 4; ++r) s += M[i][r] * x[r * 4 + c];
      t[i][c] = sat16((s + (1 << (s1 - 1))) >> s1);
    }
  const HQuant h = hquant(q, qshift, round_q12);
  __align__(16) int16_t o[16];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int s = 0;
#pragma unroll
      for (int c = 0; c < 4; ++c) s += M[j][c] * t[i][c];
      o[i * 4 + j] = hquant_level(sat16((s + 128) >> 8), h);
    }
  int4* dst = reinterpret_cast<int4*>(out + (size_t)b * 16);
  dst[0] = *reinterpret_cast<const int4*>(&o[0]);
  dst[1] = *reinterpret_cast<const int4*>(&o[8]);
}

__global__ void hevc_dqit4_kernel(const int16_t* __restrict__ coeff, int16_t* __restrict__ out, int n, int q,
                                  int use_dst, int bd_shift, int s2) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  const int16_t(*M)[4] = use_dst ? kHDst4 : kHDct4;
  const int4* src = reinterpret_cast<const int4*>(coeff + (size_t)b * 16);
  const int4 v0 = src[0], v1 = src[1];
  const int w[8] = {v0.x, v0.y, v0.z, v0.w, v1.x, v1.y, v1.z, v1.w};
  int d[16];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    d[2 * i] = hdequant((int)(int16_t)(w[i] & 0xffff), q, bd_shift);
    d[2 * i + 1] = hdequant((int)(int16_t)((uint32_t)w[i] >> 16), q, bd_shift);
  }
  int g[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      int s = 0;
#pragma unroll
      for (int k = 0; k < 4; ++k) s += M[k][r] * d[k * 4 + c];
      g[r][c] = sat16((s + 64) >> 7);
    }
  __align__(16) int16_t o[16];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      int s = 0;
#pragma unroll
      for (int k = 0; k < 4; ++k) s += M[k][c] * g[r][k];
      o[r * 4 + c] = (int16_t)sat16((s + (1 << (s2 - 1))) >> s2);
    }
  int4* dst = reinterpret_cast<int4*>(out + (size_t)b * 16);
  dst[0] = *reinterpret_cast<const int4*>(&o[0]);
  dst[1] = *reinterpret_cast<const int4*>(&o[8]);
}

// ---- 8x8 -------------------------------------------------------------------
__global__ void __launch_bounds__(128) hevc_tq8_kernel(const int16_t* __restrict__ res, int16_t* __restrict__ out,
                                                       int n, int q, int round_q12, int s1, int qshift) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  int x[64];
  const int4* src = reinterpret_cast<const int4*>(res + (size_t)b * 64);
  int any = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int4 v = src[i];
    any |= v.x | v.y | v.z | v.w;
    const int w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      x[8 * i + 2 * k] = (int)(int16_t)(w[k] & 0xffff);
      x[8 * i + 2 * k + 1] = (int)(int16_t)((uint32_t)w[k] >> 16);
    }
  }
  if (!any) {  // as for 4x4: an all-zero block gives all-zero levels
    int4* dst = reinterpret_cast<int4*>(out + (size_t)b * 64);
#pragma unroll
    for (int i = 0; i < 8; ++i) dst[i] = make_int4(0, 0, 0, 0);
    return;
  }
  int t[64];  // t[i*8+c]: column c, frequency i
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      int s = 0;
#pragma unroll
      for (int r = 0; r < 8; ++r) s += kHDct8[i][r] * x[r * 8 + c];
      t[i * 8 + c] = sat16((s + (1 << (s1 - 1))) >> s1);
    }
  const HQuant h = hquant(q, qshift, round_q12);
  int4* dst = reinterpret_cast<int4*>(out + (size_t)b * 64);
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    __align__(16) int16_t o[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      int s = 0;
#pragma unroll
      for (int c = 0; c < 8; ++c) s += kHDct8[j][c] * t[i * 8 + c];
      o[j] = hquant_level(sat16((s + 256) >> 9), h);
    }
    dst[i] = *reinterpret_cast<const int4*>(o);
  }
}

__global__ void __launch_bounds__(128) hevc_dqit8_kernel(const int16_t* __restrict__ coeff, int16_t* __restrict__ out,
                                                         int n, int q, int bd_shift, int s2) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  int d[64];
  const int4* src = reinterpret_cast<const int4*>(coeff + (size_t)b * 64);
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int4 v = src[i];
    const int w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      d[8 * i + 2 * k] = hdequant((int)(int16_t)(w[k] & 0xffff), q, bd_shift);
      d[8 * i + 2 * k + 1] = hdequant((int)(int16_t)((uint32_t)w[k] >> 16), q, bd_shift);
    }
  }
  int g[64];  // g[r*8+c]
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      int s = 0;
#pragma unroll
      for (int k = 0; k < 8; ++k) s += kHDct8[k][r] * d[k * 8 + c];
      g[r * 8 + c] = sat16((s + 64) >> 7);
    }
  int4* dst = reinterpret_cast<int4*>(out + (size_t)b * 64);
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    __align__(16) int16_t o[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      int s = 0;
#pragma unroll
      for (int k = 0; k < 8; ++k) s += kHDct8[k][c] * g[r * 8 + k];
      o[c] = (int16_t)sat16((s + (1 << (s2 - 1))) >> s2);
    }
    dst[r] = *reinterpret_cast<const int4*>(o);
  }
}

// ---- half-sample planes ----------------------------------------------------
// Output tile of 32 columns x 8 rows per 256-thread block. Plane coordinates
// (r, c) are picture coordinates + margin; every reference read is clamped to
// the picture (the reference's edge extension). With Y(k) = clampY(r - M - 3 + k)
// and X(k) = clampX(c - M - 3 + k):
//   I  = ref[clampY(r - M)][clampX(c - M)]
//   H  = clip((sum_k tap[k] * ref[clampY(r - M)][X(k)] + 32) >> 6)
//   V  = clip((sum_k tap[k] * ref[Y(k)][clampX(c - M)] + 32) >> 6)
//   HV = clip((sum_k tap[k] * T(Y(k)) + 2048) >> 12),  T(y) = sum_j tap[j] * ref[y][X(j)]
constexpr int kHpTileW = 32, kHpTileH = 8;

// P: the sample type (uint8_t at 8 bits, uint16_t at 10); maxv the largest
// sample value, (1 << BitDepth) - 1 (hevc_enc_template.c:23-25).
template <typename P>
__global__ void __launch_bounds__(256) hevc_hpel_kernel(const P* __restrict__ ref, int pitch, int w, int h, int M,
                                                        P* __restrict__ pI, P* __restrict__ pH, P* __restrict__ pV,
                                                        P* __restrict__ pHV, int opitch, int rows, int cols,
                                                        int maxv) {
  __shared__ P src[kHpTileH + 7][kHpTileW + 8];
  __shared__ int32_t tsum[kHpTileH + 7][kHpTileW];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int c0 = blockIdx.x * kHpTileW, r0 = blockIdx.y * kHpTileH;
  // source rows r0-M-3 .. r0-M+kHpTileH+3, columns c0-M-3 .. c0-M+kHpTileW+4
  for (int i = threadIdx.x; i < (kHpTileH + 7) * (kHpTileW + 8); i += 256) {
    const int sr = i / (kHpTileW + 8), sc = i - sr * (kHpTileW + 8);
    const int y = clampi(r0 - M - 3 + sr, 0, h - 1), x = clampi(c0 - M - 3 + sc, 0, w - 1);
    src[sr][sc] = ref[(size_t)y * pitch + x];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < (kHpTileH + 7) * kHpTileW; i += 256) {
    const int sr = i / kHpTileW, sc = i - sr * kHpTileW;
    const P* p = &src[sr][sc];
    tsum[sr][sc] = -p[0] + 4 * p[1] - 11 * p[2] + 40 * p[3] + 40 * p[4] - 11 * p[5] + 4 * p[6] - p[7];
  }
  __syncthreads();
  const int r = r0 + ty, c = c0 + tx;
  if (r >= rows || c >= cols) return;
  const int sr = ty + 3, sc = tx + 3;  // the sample (r - M, c - M) in the staged tile
  const size_t o = (size_t)r * opitch + c;
  pI[o] = src[sr][sc];
  pH[o] = (P)clampi((tsum[sr][tx] + 32) >> 6, 0, maxv);
  const int v = -src[ty][sc] + 4 * src[ty + 1][sc] - 11 * src[ty + 2][sc] + 40 * src[ty + 3][sc] +
                40 * src[ty + 4][sc] - 11 * src[ty + 5][sc] + 4 * src[ty + 6][sc] - src[ty + 7][sc];
  pV[o] = (P)clampi((v + 32) >> 6, 0, maxv);
  const int hv = -tsum[ty][tx] + 4 * tsum[ty + 1][tx] - 11 * tsum[ty + 2][tx] + 40 * tsum[ty + 3][tx] +
                 40 * tsum[ty + 4][tx] - 11 * tsum[ty + 5][tx] + 4 * tsum[ty + 6][tx] - tsum[ty + 7][tx];
  pHV[o] = (P)clampi((hv + 2048) >> 12, 0, maxv);
}

// ---- 8x8 CU motion search -------------------------------------------------
// One warp per CU job, the reference's walk (hevc_enc_template.c:958-1043)
// step for step: every lane follows the same (uniform) control flow and the
// SADs are warp reductions, lane l scoring row l/4, columns 2(l%4), +1.
// Strides in samples. sad_shift brings a SAD back to eight-bit units (0 at
// eight bits, 2 at ten: hevc_enc_template.c:484).
template <typename P>
struct HevcSearch {
  const P* src;
  int src_pitch, w, h, M, qpel;
  const P* plane[4];
  int ppitch, sad_shift;
};

__device__ __forceinline__ int hevc_mvd_bits(int d) {
  const unsigned a = (unsigned)(d < 0 ? -d : d);
  if (a == 0) return 1;
  if (a == 1) return 3;
  return 3 + 2 * (31 - __clz((int)((a - 2) / 2 + 1))) + 2;
}

// SAD of the CU against the search planes at absolute quarter-sample
// position (qx, qy) (search_sad, hevc_enc_template.c:463): positions are
// clamped to the planes' margin; even/even reads one half-grid block, a
// position odd in x, y or both averages (rounded) the two blocks beside it.
template <typename P>
__device__ __forceinline__ uint32_t hevc_search_sad(const HevcSearch<P>& S, int cu_x, int cu_y, int qx, int qy,
                                                    int lane) {
  const int lo = -(S.M - 2) * 4;
  const int hx = (S.w - 8 + S.M - 2) * 4, hy = (S.h - 8 + S.M - 2) * 4;
  qx = qx < lo ? lo : (qx > hx ? hx : qx);
  qy = qy < lo ? lo : (qy > hy ? hy : qy);
  const int r = lane >> 2, c = (lane & 3) * 2;
  auto sample = [&](int bqx, int bqy, int dc) -> int {
    const int ph = ((bqx & 2) ? 1 : 0) + ((bqy & 2) ? 2 : 0);
    const int x = (bqx >> 2) + S.M + c + dc, y = (bqy >> 2) + S.M + r;
    return S.plane[ph][(size_t)y * S.ppitch + x];
  };
  uint32_t sad = 0;
#pragma unroll
  for (int dc = 0; dc < 2; ++dc) {
    int v;
    if (!(qx & 1) && !(qy & 1)) v = sample(qx, qy, dc);
    else if ((qx & 1) && (qy & 1)) v = (sample(qx - 1, qy - 1, dc) + sample(qx + 1, qy + 1, dc) + 1) >> 1;
    else if (qx & 1) v = (sample(qx - 1, qy, dc) + sample(qx + 1, qy, dc) + 1) >> 1;
    else v = (sample(qx, qy - 1, dc) + sample(qx, qy + 1, dc) + 1) >> 1;
    const int sv = S.src[(size_t)(cu_y + r) * S.src_pitch + cu_x + c + dc];
    sad += (uint32_t)abs(sv - v);
  }
  return __reduce_add_sync(0xffffffffu, sad) >> S.sad_shift;
}

template <typename P>
__global__ void __launch_bounds__(128) hevc_me_kernel(HevcSearch<P> S, const b200enc_hevc_me_job_t* __restrict__ jobs,
                                                      int n, b200enc_hevc_me_result_t* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int j = blockIdx.x * 4 + (threadIdx.x >> 5);
  if (j >= n) return;
  const b200enc_hevc_me_job_t job = jobs[j];
  const int cu_x = job.cu_x, cu_y = job.cu_y;
  if (cu_x < 0 || cu_y < 0 || cu_x > S.w - 8 || cu_y > S.h - 8) {  // not a CU of this picture
    if (lane == 0) {
      b200enc_hevc_me_result_t r{};
      r.sad = 0xffffffffu;
      r.cost_q8 = -1;
      out[j] = r;
    }
    return;
  }
  const int min_dx = -cu_x - 8, max_dx = S.w - cu_x, min_dy = -cu_y - 8, max_dy = S.h - cu_y;
  const int range = 64, qx0 = cu_x * 4, qy0 = cu_y * 4;
  auto mv_bits = [&](int qx, int qy) -> int {
    const int b0 = hevc_mvd_bits(qx - job.mvp[0].x) + hevc_mvd_bits(qy - job.mvp[0].y);
    const int b1 = hevc_mvd_bits(qx - job.mvp[1].x) + hevc_mvd_bits(qy - job.mvp[1].y);
    return b0 <= b1 ? b0 : b1;
  };
  auto cost = [&](int qx, int qy, uint32_t sad) -> long long {
    return (long long)sad * 256 + (long long)job.lambda_q8 * mv_bits(qx, qy);
  };
  int bx = 0, by = 0;
  long long best = 0x7fffffffffffffffll;
  uint32_t best_sad = 0;
  int seen_x[16], seen_y[16], n_seen = 0;
  const int ns = job.n_starts < 0 ? 0 : (job.n_starts > 16 ? 16 : job.n_starts);
  for (int i = 0; i < ns; ++i) {
    int dx = (job.starts[i].x + 2) >> 2, dy = (job.starts[i].y + 2) >> 2;
    dx = dx < min_dx ? min_dx : (dx > max_dx ? max_dx : dx);
    dy = dy < min_dy ? min_dy : (dy > max_dy ? max_dy : dy);
    bool dup = false;
    for (int k = 0; k < n_seen && !dup; ++k) dup = seen_x[k] == dx && seen_y[k] == dy;
    if (dup) continue;
    seen_x[n_seen] = dx;
    seen_y[n_seen++] = dy;
    const uint32_t sd = hevc_search_sad(S, cu_x, cu_y, qx0 + dx * 4, qy0 + dy * 4, lane);
    const long long c = cost(dx * 4, dy * 4, sd);
    if (c < best) { best = c; best_sad = sd; bx = dx; by = dy; }
  }
  const int cx0 = bx, cy0 = by;
  int back = -1;
  for (int step = 0; step < 32; ++step) {
    const int ddx[4] = {-1, 1, 0, 0}, ddy[4] = {0, 0, -1, 1};
    int nbx = bx, nby = by, nk = -1;
    for (int k = 0; k < 4; ++k) {
      if (k == back) continue;
      const int dx = bx + ddx[k], dy = by + ddy[k];
      if (dx < min_dx || dx > max_dx || dy < min_dy || dy > max_dy) continue;
      if (dx < cx0 - range || dx > cx0 + range || dy < cy0 - range || dy > cy0 + range) continue;
      const uint32_t sd = hevc_search_sad(S, cu_x, cu_y, qx0 + dx * 4, qy0 + dy * 4, lane);
      const long long c = cost(dx * 4, dy * 4, sd);
      if (c < best) { best = c; best_sad = sd; nbx = dx; nby = dy; nk = k; }
    }
    if (nbx == bx && nby == by) break;
    bx = nbx;
    by = nby;
    back = nk ^ 1;
  }
  int mx = bx * 4, my = by * 4;
  for (int st = 2; st >= (S.qpel ? 1 : 2); st >>= 1) {
    const int ox[8] = {-1, 0, 1, -1, 1, -1, 0, 1}, oy[8] = {-1, -1, -1, 0, 0, 1, 1, 1};
    const int c0x = mx, c0y = my;
    for (int k = 0; k < 8; ++k) {
      const int tx = c0x + ox[k] * st, ty = c0y + oy[k] * st;
      const uint32_t sd = hevc_search_sad(S, cu_x, cu_y, qx0 + tx, qy0 + ty, lane);
      const long long c = cost(tx, ty, sd);
      if (c < best) { best = c; best_sad = sd; mx = tx; my = ty; }
    }
  }
  if (lane == 0) {
    const int b0 = hevc_mvd_bits(mx - job.mvp[0].x) + hevc_mvd_bits(my - job.mvp[0].y);
    const int b1 = hevc_mvd_bits(mx - job.mvp[1].x) + hevc_mvd_bits(my - job.mvp[1].y);
    b200enc_hevc_me_result_t r;
    r.mv.x = (int16_t)mx;
    r.mv.y = (int16_t)my;
    r.mvp_idx = b1 < b0 ? 1 : 0;
    r.cost_q8 = best;
    r.sad = best_sad;
    r.pad = 0;
    out[j] = r;
  }
}

// ---- intra 4x4 luma mode choice ----------------------------------------------
// hevc_intra_template.c:20-260 (gather_neighbors, predict_from_refs,
// hevc_choose_luma_mode) with hevc_intra.c's z-scan availability: a
// neighbour is available iff it is inside the picture, at or below the
// slice's first row, and earlier in the encoder's fixed coding order (CTU
// 16x16 raster, CU 8x8 z-order, PU 4x4 z-order).
__device__ __forceinline__ long long hz_rank(int x, int y, int width) {
  const int width_ctu = (width + 15) >> 4;
  const int rx = x & 15, ry = y & 15;
  long long rank = ((long long)(y >> 4) * width_ctu + (x >> 4)) * 4 + ((ry >> 3) * 2 + (rx >> 3));
  return rank * 4 + (((ry & 7) >> 2) * 2 + ((rx & 7) >> 2));
}
__device__ __forceinline__ bool hz_avail(int nx, int ny, int width, int height, int y_min, long long cur) {
  if (nx < 0 || ny < y_min || nx >= width || ny >= height) return false;
  return hz_rank(nx, ny, width) < cur;
}

constexpr int kHModePlanar = 0, kHModeDc = 1, kHModeHor = 10, kHModeVer = 26;

__device__ __forceinline__ void hpredict(const int* left, const int* top, int corner, int mode, int maxv, int* pred) {
  if (mode == kHModePlanar) {
#pragma unroll
    for (int y = 0; y < 4; ++y)
#pragma unroll
      for (int x = 0; x < 4; ++x)
        pred[y * 4 + x] = ((3 - x) * left[y] + (x + 1) * top[4] + (3 - y) * top[x] + (y + 1) * left[4] + 4) >> 3;
  } else if (mode == kHModeDc) {
    const int dc = (left[0] + left[1] + left[2] + left[3] + top[0] + top[1] + top[2] + top[3] + 4) >> 3;
#pragma unroll
    for (int i = 0; i < 16; ++i) pred[i] = dc;
    pred[0] = (left[0] + 2 * dc + top[0] + 2) >> 2;
#pragma unroll
    for (int x = 1; x < 4; ++x) pred[x] = (top[x] + 3 * dc + 2) >> 2;
#pragma unroll
    for (int y = 1; y < 4; ++y) pred[y * 4] = (left[y] + 3 * dc + 2) >> 2;
  } else if (mode == kHModeHor) {
#pragma unroll
    for (int y = 0; y < 4; ++y)
#pragma unroll
      for (int x = 0; x < 4; ++x) pred[y * 4 + x] = left[y];
#pragma unroll
    for (int x = 0; x < 4; ++x) pred[x] = clampi(left[0] + ((top[x] - corner) >> 1), 0, maxv);
  } else {
#pragma unroll
    for (int y = 0; y < 4; ++y)
#pragma unroll
      for (int x = 0; x < 4; ++x) pred[y * 4 + x] = top[x];
#pragma unroll
    for (int y = 0; y < 4; ++y) pred[y * 4] = clampi(top[0] + ((left[y] - corner) >> 1), 0, maxv);
  }
}

// P: the sample type; bd the bit depth (8 or 10). Pitches in samples.
template <typename P>
__global__ void hevc_intra4_kernel(const P* __restrict__ src, int src_pitch, const P* __restrict__ rec,
                                   int rec_pitch, int width, int height, const int* __restrict__ jobs, int n,
                                   int* __restrict__ modes, P* __restrict__ preds, int bd) {
  const int maxv = (1 << bd) - 1;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int x0 = jobs[3 * j], y0 = jobs[3 * j + 1], y_min = jobs[3 * j + 2];
  if (x0 < 0 || y0 < 0 || x0 + 4 > width || y0 + 4 > height || (x0 & 3) || (y0 & 3)) {
    modes[j] = -1;  // not a 4x4 PU of this picture
    return;
  }
  const long long cur = hz_rank(x0, y0, width);
  const bool a_left = hz_avail(x0 - 1, y0, width, height, y_min, cur);
  const bool a_top = hz_avail(x0, y0 - 1, width, height, y_min, cur);
  const bool a_corner = hz_avail(x0 - 1, y0 - 1, width, height, y_min, cur);
  const bool a_tr = hz_avail(x0 + 4, y0 - 1, width, height, y_min, cur);
  // the substitution scan over p[-1][3..0], p[-1][-1], p[0..4][-1]
  int sv[10];
  bool sa[10];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    sa[i] = a_left;
    sv[i] = a_left ? rec[(size_t)(y0 + 3 - i) * rec_pitch + x0 - 1] : 0;
  }
  sa[4] = a_corner;
  sv[4] = a_corner ? rec[(size_t)(y0 - 1) * rec_pitch + x0 - 1] : 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    sa[5 + i] = a_top;
    sv[5 + i] = a_top ? rec[(size_t)(y0 - 1) * rec_pitch + x0 + i] : 0;
  }
  sa[9] = a_tr;
  sv[9] = a_tr ? rec[(size_t)(y0 - 1) * rec_pitch + x0 + 4] : 0;
  int first = -1;
#pragma unroll
  for (int i = 9; i >= 0; --i)
    if (sa[i]) first = i;
  if (first < 0) {
#pragma unroll
    for (int i = 0; i < 10; ++i) sv[i] = 1 << (bd - 1);  // 128 at eight bits, 512 at ten
  } else {
    const int f = sv[first];
#pragma unroll
    for (int i = 0; i < 10; ++i)
      if (i < first) sv[i] = f;
#pragma unroll
    for (int i = 1; i < 10; ++i)
      if (i > first && !sa[i]) sv[i] = sv[i - 1];
  }
  int left[5], top[5];
  left[3] = sv[0]; left[2] = sv[1]; left[1] = sv[2]; left[0] = sv[3];
  const int corner = sv[4];
  top[0] = sv[5]; top[1] = sv[6]; top[2] = sv[7]; top[3] = sv[8]; top[4] = sv[9];
  left[4] = hz_avail(x0 - 1, y0 + 4, width, height, y_min, cur) ? rec[(size_t)(y0 + 4) * rec_pitch + x0 - 1]
                                                                : left[3];
  int s[16];
#pragma unroll
  for (int y = 0; y < 4; ++y)
#pragma unroll
    for (int x = 0; x < 4; ++x) s[y * 4 + x] = src[(size_t)(y0 + y) * src_pitch + x0 + x];
  const int order[4] = {kHModePlanar, kHModeDc, kHModeHor, kHModeVer};
  int best_mode = -1, best_sad = 0;
  int best_pred[16];
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    int pr[16];
    hpredict(left, top, corner, order[m], maxv, pr);
    int sad = 0;
#pragma unroll
    for (int i = 0; i < 16; ++i) sad += abs(s[i] - pr[i]);
    if (m == 0 || sad < best_sad) {
      best_sad = sad;
      best_mode = order[m];
#pragma unroll
      for (int i = 0; i < 16; ++i) best_pred[i] = pr[i];
    }
  }
  modes[j] = best_mode;
  if (sizeof(P) == 1) {
    uint32_t w4[4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
      w4[r] = (uint32_t)best_pred[4 * r] | ((uint32_t)best_pred[4 * r + 1] << 8) |
              ((uint32_t)best_pred[4 * r + 2] << 16) | ((uint32_t)best_pred[4 * r + 3] << 24);
    *reinterpret_cast<uint4*>(preds + (size_t)j * 16) = make_uint4(w4[0], w4[1], w4[2], w4[3]);
  } else {
    uint32_t w8[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) w8[k] = (uint32_t)best_pred[2 * k] | ((uint32_t)best_pred[2 * k + 1] << 16);
    uint4* o = reinterpret_cast<uint4*>(preds + (size_t)j * 16);
    o[0] = make_uint4(w8[0], w8[1], w8[2], w8[3]);
    o[1] = make_uint4(w8[4], w8[5], w8[6], w8[7]);
  }
}

bool aligned16(const void* p) { return (((uintptr_t)p) & 15) == 0; }
int hclamp(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

}  // namespace b200enc

using namespace b200enc;

extern "C" {

int b200enc_hevc_transform_quant_4x4(const int16_t* residual, int16_t* coeff, int n, int qp, int use_dst,
                                     int round_q12, int bit_depth, void* stream) {
  if (!residual || !coeff || n < 0 || (bit_depth != 8 && bit_depth != 10)) return -1;
  if (!aligned16(residual) || !aligned16(coeff) || round_q12 < 0 || round_q12 > 12) return -1;
  if (n == 0) return 0;
  const int q = bit_depth == 8 ? hclamp(qp, 0, 51) : hclamp(qp, 0, 63);
  hevc_tq4_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(residual, coeff, n, q, use_dst ? 1 : 0,
                                                                       round_q12, bit_depth == 8 ? 1 : 3,
                                                                       bit_depth == 8 ? 5 : 7);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int b200enc_hevc_dequant_itransform_4x4(const int16_t* coeff, int16_t* residual, int n, int qp, int use_dst,
                                        int bit_depth, void* stream) {
  if (!residual || !coeff || n < 0 || (bit_depth != 8 && bit_depth != 10)) return -1;
  if (!aligned16(residual) || !aligned16(coeff)) return -1;
  // the reference clamps the 10-bit Qp' but takes the 8-bit QP as given
  if (bit_depth == 8 && (qp < 0 || qp > 51)) return -1;
  if (n == 0) return 0;
  const int q = bit_depth == 8 ? qp : hclamp(qp, 0, 63);
  hevc_dqit4_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(coeff, residual, n, q, use_dst ? 1 : 0,
                                                                         bit_depth == 8 ? 5 : 7,
                                                                         bit_depth == 8 ? 12 : 10);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int b200enc_hevc_transform_quant_8x8(const int16_t* residual, int16_t* coeff, int n, int qp, int bit_depth,
                                     int round_q12, void* stream) {
  if (!residual || !coeff || n < 0 || (bit_depth != 8 && bit_depth != 10)) return -1;
  if (!aligned16(residual) || !aligned16(coeff) || round_q12 < 0 || round_q12 > 12) return -1;
  if (n == 0) return 0;
  hevc_tq8_kernel<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(residual, coeff, n, hclamp(qp, 0, 63),
                                                                       round_q12, 3 + bit_depth - 9, bit_depth - 2);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int b200enc_hevc_dequant_itransform_8x8(const int16_t* coeff, int16_t* residual, int n, int qp, int bit_depth,
                                        void* stream) {
  if (!residual || !coeff || n < 0 || (bit_depth != 8 && bit_depth != 10)) return -1;
  if (!aligned16(residual) || !aligned16(coeff)) return -1;
  if (n == 0) return 0;
  hevc_dqit8_kernel<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(coeff, residual, n, hclamp(qp, 0, 63),
                                                                         bit_depth - 2, 20 - bit_depth);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int b200enc_hevc_build_hpel(const uint8_t* recon, int pitch, int w, int h, int margin, uint8_t* plane_i,
                            uint8_t* plane_h, uint8_t* plane_v, uint8_t* plane_hv, int plane_pitch, void* stream) {
  if (!recon || !plane_i || !plane_h || !plane_v || !plane_hv || w <= 0 || h <= 0) return -1;
  if (margin < 0 || margin > 256 || pitch < w) return -1;
  const int rows = h + 2 * margin, cols = w + 2 * margin;
  if (plane_pitch < cols) return -1;
  dim3 grid((cols + kHpTileW - 1) / kHpTileW, (rows + kHpTileH - 1) / kHpTileH);
  hevc_hpel_kernel<uint8_t><<<grid, 256, 0, (cudaStream_t)stream>>>(recon, pitch, w, h, margin, plane_i, plane_h,
                                                                    plane_v, plane_hv, plane_pitch, rows, cols, 255);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int b200enc_hevc_build_hpel_10(const uint16_t* recon, int pitch, int w, int h, int margin, uint16_t* plane_i,
                               uint16_t* plane_h, uint16_t* plane_v, uint16_t* plane_hv, int plane_pitch,
                               void* stream) {
  if (!recon || !plane_i || !plane_h || !plane_v || !plane_hv || w <= 0 || h <= 0) return -1;
  if (margin < 0 || margin > 256 || pitch < w) return -1;
  const int rows = h + 2 * margin, cols = w + 2 * margin;
  if (plane_pitch < cols) return -1;
  dim3 grid((cols + kHpTileW - 1) / kHpTileW, (rows + kHpTileH - 1) / kHpTileH);
  hevc_hpel_kernel<uint16_t><<<grid, 256, 0, (cudaStream_t)stream>>>(recon, pitch, w, h, margin, plane_i, plane_h,
                                                                     plane_v, plane_hv, plane_pitch, rows, cols,
                                                                     1023);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int b200enc_hevc_motion_search(const uint8_t* src_y, int src_pitch, int w, int h, const uint8_t* plane_i,
                               const uint8_t* plane_h, const uint8_t* plane_v, const uint8_t* plane_hv, int plane_pitch,
                               int margin, int qpel, const b200enc_hevc_me_job_t* jobs, int n,
                               b200enc_hevc_me_result_t* results, void* stream) {
  if (!src_y || !plane_i || !plane_h || !plane_v || !plane_hv || !jobs || !results || n < 0) return -1;
  if (w < 8 || h < 8 || margin < 10 || plane_pitch < w + 2 * margin || src_pitch < w) return -1;
  if (n == 0) return 0;
  HevcSearch<uint8_t> S{src_y, src_pitch, w, h, margin, qpel ? 1 : 0, {plane_i, plane_h, plane_v, plane_hv},
                        plane_pitch, 0};
  hevc_me_kernel<uint8_t><<<(n + 3) / 4, 128, 0, (cudaStream_t)stream>>>(S, jobs, n, results);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int b200enc_hevc_motion_search_10(const uint16_t* src_y, int src_pitch, int w, int h, const uint16_t* plane_i,
                                  const uint16_t* plane_h, const uint16_t* plane_v, const uint16_t* plane_hv,
                                  int plane_pitch, int margin, int qpel, const b200enc_hevc_me_job_t* jobs, int n,
                                  b200enc_hevc_me_result_t* results, void* stream) {
  if (!src_y || !plane_i || !plane_h || !plane_v || !plane_hv || !jobs || !results || n < 0) return -1;
  if (w < 8 || h < 8 || margin < 10 || plane_pitch < w + 2 * margin || src_pitch < w) return -1;
  if (n == 0) return 0;
  HevcSearch<uint16_t> S{src_y, src_pitch, w, h, margin, qpel ? 1 : 0, {plane_i, plane_h, plane_v, plane_hv},
                         plane_pitch, 2};
  hevc_me_kernel<uint16_t><<<(n + 3) / 4, 128, 0, (cudaStream_t)stream>>>(S, jobs, n, results);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int b200enc_hevc_choose_luma_mode(const uint8_t* src_y, int src_pitch, const uint8_t* recon_y, int recon_pitch,
                                  int width, int height, const int* jobs, int n, int* modes, uint8_t* preds,
                                  void* stream) {
  if (!src_y || !recon_y || !jobs || !modes || !preds || n < 0 || width < 4 || height < 4) return -1;
  if (!aligned16(preds) || src_pitch < width || recon_pitch < width) return -1;
  if (n == 0) return 0;
  hevc_intra4_kernel<uint8_t><<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(
      src_y, src_pitch, recon_y, recon_pitch, width, height, jobs, n, modes, preds, 8);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int b200enc_hevc_choose_luma_mode_10(const uint16_t* src_y, int src_pitch, const uint16_t* recon_y, int recon_pitch,
                                     int width, int height, const int* jobs, int n, int* modes, uint16_t* preds,
                                     void* stream) {
  if (!src_y || !recon_y || !jobs || !modes || !preds || n < 0 || width < 4 || height < 4) return -1;
  if (!aligned16(preds) || src_pitch < width || recon_pitch < width) return -1;
  if (n == 0) return 0;
  hevc_intra4_kernel<uint16_t><<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(
      src_y, src_pitch, recon_y, recon_pitch, width, height, jobs, n, modes, preds, 10);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// The same planes from and to host memory, for a host encoder that keeps its
// reconstruction and search planes in host buffers (the reference's
// hevc_encoder_t: prev_recon_y, hpel[4], hpel_stride). Each calling thread
// keeps its own device workspace and stream, grown to the largest picture
// it has seen; the call returns when the four planes are in `planes`.
namespace {
struct HpelWork {
  cudaStream_t st = nullptr;
  void* buf = nullptr;
  size_t bytes = 0;
  ~HpelWork() {
    if (buf) cudaFree(buf);
    if (st) cudaStreamDestroy(st);
  }
};
thread_local HpelWork t_hpel;
}  // namespace

int b200enc_hevc_build_hpel_host(const void* recon, int w, int h, int bit_depth, int margin, void* const planes[4],
                                 int plane_stride) {
  if (!recon || !planes || w <= 0 || h <= 0 || (bit_depth != 8 && bit_depth != 10)) return -1;
  if (margin < 0 || margin > 256 || plane_stride < w + 2 * margin) return -1;
  for (int i = 0; i < 4; ++i)
    if (!planes[i]) return -1;
  const size_t bps = bit_depth == 8 ? 1 : 2;
  const int rows = h + 2 * margin;
  const size_t rec_bytes = (size_t)w * h * bps, plane_bytes = (size_t)plane_stride * rows * bps;
  const size_t need = ((rec_bytes + 255) & ~(size_t)255) + 4 * ((plane_bytes + 255) & ~(size_t)255);
  HpelWork& wk = t_hpel;
  if (!wk.st && cudaStreamCreateWithFlags(&wk.st, cudaStreamNonBlocking) != cudaSuccess) return -1;
  if (wk.bytes < need) {
    if (wk.buf) cudaFree(wk.buf);
    wk.buf = nullptr;
    wk.bytes = 0;
    if (cudaMalloc(&wk.buf, need) != cudaSuccess) return -1;
    wk.bytes = need;
  }
  uint8_t* d = static_cast<uint8_t*>(wk.buf);
  uint8_t* drec = d;
  uint8_t* dp[4];
  for (int i = 0; i < 4; ++i) dp[i] = d + ((rec_bytes + 255) & ~(size_t)255) + i * ((plane_bytes + 255) & ~(size_t)255);
  if (cudaMemcpyAsync(drec, recon, rec_bytes, cudaMemcpyHostToDevice, wk.st) != cudaSuccess) return -1;
  const int rc = bit_depth == 8
                     ? b200enc_hevc_build_hpel(drec, w, w, h, margin, dp[0], dp[1], dp[2], dp[3], plane_stride, wk.st)
                     : b200enc_hevc_build_hpel_10(reinterpret_cast<const uint16_t*>(drec), w, w, h, margin,
                                                  reinterpret_cast<uint16_t*>(dp[0]),
                                                  reinterpret_cast<uint16_t*>(dp[1]),
                                                  reinterpret_cast<uint16_t*>(dp[2]),
                                                  reinterpret_cast<uint16_t*>(dp[3]), plane_stride, wk.st);
  if (rc != 0) return -1;
  for (int i = 0; i < 4; ++i)
    if (cudaMemcpyAsync(planes[i], dp[i], plane_bytes, cudaMemcpyDeviceToHost, wk.st) != cudaSuccess) return -1;
  return cudaStreamSynchronize(wk.st) == cudaSuccess ? 0 : -1;
}

int b200enc_pin_host(void* ptr, size_t bytes) {
  if (!ptr || bytes == 0) return -1;
  if (cudaHostRegister(ptr, bytes, cudaHostRegisterDefault) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  return 0;
}

int b200enc_unpin_host(void* ptr) {
  if (!ptr) return -1;
  if (cudaHostUnregister(ptr) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  return 0;
}

}  // extern "C"
