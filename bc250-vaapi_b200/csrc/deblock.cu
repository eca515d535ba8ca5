// deblock.cu - spec deblocking (H.264 clause 8.7) as a persistent wavefront.
//
// The reference shader (A1/shaders/deblock_filter.comp) filters luma only,
// treats bS 4 like bS 3, and runs all edges of a direction at once, so
// neighbouring edges race on the samples they share; no decoder reproduces
// it. This kernel reproduces the reference's C deblocker
// (A1/src/h264_deblock.c:263-368) exactly: raster-order semantics, vertical
// edges then horizontal per macroblock, luma and chroma, bS 0-4 with the
// strong filter.
//
// Raster order matters only between filtering steps whose sample footprints
// overlap. The vertical edges of (x,y) read and write only rows of
// macroblock row y, which no step of row y-1 touches; they follow the
// horizontal edges of (x-1,y). The horizontal edges of (x,y) read and change
// the bottom rows of (x,y-1), final once the vertical edges of (x+1,y-1)
// (the last step to change its right columns) are done. So rows run as a
// wavefront with a skew of one macroblock step. Luma and chroma never share
// a sample, so they are two independent wavefronts.
//
// Layout for latency (the wavefront is latency-bound: ~mbw + mbh dependent
// macroblock steps per frame):
//   * a CTA owns a group of R consecutive macroblock rows (taken by ticket,
//     so groups are only owned by running CTAs and waits cannot deadlock);
//     R luma warps + R chroma warps, one warp per row and plane kind;
//   * the group's rows (plus a 4-row / 2-row halo above) pass through a
//     ring of 16 macroblock columns in shared memory (42 KB per CTA at
//     4 rows, whatever the picture width), so deblocking CTAs leave room on
//     their SMs for other streams' kernels;
//   * row warps wait on shared-memory progress words only: a row on the row
//     above, the group's first row on the columns the IO warps have staged;
//   * two IO warps (luma, chroma) load the ring's columns ahead of the first
//     row and, once the group's last row is done with a column, write it
//     back and release it to the next group in batches (one fence, a release
//     store); two halo warps fetch each column's halo rows as soon as the
//     group above releases it; no row warp touches a global flag or fence;
//   * boundary strengths of the whole group are computed up front.
// Waits are bounded; on timeout a CTA records the error and leaves, and
// every waiter gives up as soon as it sees a recorded error.
#include <algorithm>

#include "b200enc_internal.h"
#include "common.cuh"

namespace b200enc {

// Table 8-16 / 8-17 (the same values the reference's decoder tables and its
// shader hold: A1/src/h264_dec_tables.c, A1/shaders/deblock_filter.comp:185-210).
__constant__ uint8_t kAlpha[52] = {0,  0,  0,  0,  0,  0,  0,  0,  0,  0,   0,   0,   0,   0,   0,   0,   4,  4,
                                   5,  6,  7,  8,  9,  10, 12, 13, 15, 17,  20,  22,  25,  28,  32,  36,  40, 45,
                                   50, 56, 63, 71, 80, 90, 101, 113, 127, 144, 162, 182, 203, 226, 255, 255};
__constant__ uint8_t kBeta[52] = {0, 0, 0, 0, 0, 0, 0, 0, 0,  0,  0,  0,  0,  0,  0,  0,  2,  2,
                                  2, 3, 3, 3, 3, 4, 4, 4, 6,  6,  7,  7,  8,  8,  9,  9,  10, 10,
                                  11, 11, 12, 12, 13, 13, 14, 14, 15, 15, 16, 16, 17, 17, 18, 18};
__constant__ uint8_t kTc0[52][3] = {
    {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0},  {0, 0, 0},  {0, 0, 0},
    {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0},  {0, 0, 0},  {0, 0, 1},
    {0, 0, 1}, {0, 0, 1}, {0, 0, 1}, {0, 1, 1}, {0, 1, 1}, {1, 1, 1}, {1, 1, 1},  {1, 1, 1},  {1, 1, 1},
    {1, 1, 2}, {1, 1, 2}, {1, 1, 2}, {1, 1, 2}, {1, 2, 3}, {1, 2, 3}, {2, 2, 3},  {2, 2, 4},  {2, 3, 4},
    {2, 3, 4}, {3, 3, 5}, {3, 4, 6}, {3, 4, 6}, {4, 5, 7}, {4, 5, 8}, {4, 6, 9},  {5, 7, 10}, {6, 8, 11},
    {6, 8, 13}, {7, 10, 14}, {8, 11, 16}, {9, 12, 18}, {10, 13, 20}, {11, 15, 23}, {13, 17, 25}};

// Line filters (clause 8.7.2.3 / 8.7.2.4) on samples held in registers; the
// callers unroll the edge loop, so every index is a compile-time constant.
// They are branch-free: every lane evaluates the whole filter and keeps the
// result by selection, so lanes whose edges differ in bS or in the sample
// tests never split the warp, and the dependent chain per edge stays short.
// A line with bS 0 or a failed sample test is left as it is.
//
// This encoder's boundary strengths are 4 on the macroblock edges of intra
// pictures, 3 on their internal edges and 0-2 in P pictures, so the strong
// filter is taken on a warp-uniform condition (intra picture, macroblock
// edge) and the normal filter elsewhere.
__device__ __forceinline__ void luma_normal(int p2, int& p1, int& p0, int& q0, int& q1, int q2, int bs, int alpha,
                                            int beta, int tc0) {
  const int dqp = q0 - p0;
  const bool f = (bs != 0) & (abs(dqp) < alpha) & (abs(p1 - p0) < beta) & (abs(q1 - q0) < beta);
  const bool ap = abs(p2 - p0) < beta, aq = abs(q2 - q0) < beta;
  const int tc = tc0 + (int)ap + (int)aq;
  const int delta = clampi((dqp * 4 + (p1 - q1) + 4) >> 3, -tc, tc);
  const int avg = (p0 + q0 + 1) >> 1;
  const int np1 = p1 + clampi((p2 + avg - (p1 << 1)) >> 1, -tc0, tc0);
  const int nq1 = q1 + clampi((q2 + avg - (q1 << 1)) >> 1, -tc0, tc0);
  const int np0 = clip1(p0 + delta), nq0 = clip1(q0 - delta);
  p1 = (f & ap) ? np1 : p1;
  q1 = (f & aq) ? nq1 : q1;
  p0 = f ? np0 : p0;
  q0 = f ? nq0 : q0;
}

__device__ __forceinline__ void luma_strong(int p3, int& p2, int& p1, int& p0, int& q0, int& q1, int& q2, int q3, int bs,
                                            int alpha, int beta) {
  const int d0 = abs(p0 - q0);
  const bool f = (bs != 0) & (d0 < alpha) & (abs(p1 - p0) < beta) & (abs(q1 - q0) < beta);
  const bool small = d0 < ((alpha >> 2) + 2);
  const bool sp = f & small & (abs(p2 - p0) < beta), sq = f & small & (abs(q2 - q0) < beta);
  const int a0 = (p2 + 2 * p1 + 2 * p0 + 2 * q0 + q1 + 4) >> 3;
  const int a1 = (p2 + p1 + p0 + q0 + 2) >> 2;
  const int a2 = (2 * p3 + 3 * p2 + p1 + p0 + q0 + 4) >> 3;
  const int aw = (2 * p1 + p0 + q1 + 2) >> 2;
  const int b0 = (q2 + 2 * q1 + 2 * q0 + 2 * p0 + p1 + 4) >> 3;
  const int b1 = (q2 + q1 + q0 + p0 + 2) >> 2;
  const int b2 = (2 * q3 + 3 * q2 + q1 + q0 + p0 + 4) >> 3;
  const int bw = (2 * q1 + q0 + p1 + 2) >> 2;
  p0 = sp ? a0 : (f ? aw : p0);
  p1 = sp ? a1 : p1;
  p2 = sp ? a2 : p2;
  q0 = sq ? b0 : (f ? bw : q0);
  q1 = sq ? b1 : q1;
  q2 = sq ? b2 : q2;
}

__device__ __forceinline__ void chroma_normal(int p1, int& p0, int& q0, int q1, int bs, int alpha, int beta, int tc0) {
  const int dqp = q0 - p0;
  const bool f = (bs != 0) & (abs(dqp) < alpha) & (abs(p1 - p0) < beta) & (abs(q1 - q0) < beta);
  const int tc = tc0 + 1;
  const int delta = clampi((dqp * 4 + (p1 - q1) + 4) >> 3, -tc, tc);
  const int np0 = clip1(p0 + delta), nq0 = clip1(q0 - delta);
  p0 = f ? np0 : p0;
  q0 = f ? nq0 : q0;
}

__device__ __forceinline__ void chroma_strong(int p1, int& p0, int& q0, int q1, int bs, int alpha, int beta) {
  const bool f = (bs != 0) & (abs(p0 - q0) < alpha) & (abs(p1 - p0) < beta) & (abs(q1 - q0) < beta);
  const int np0 = (2 * p1 + p0 + q1 + 2) >> 2, nq0 = (2 * q1 + q0 + p1 + 2) >> 2;
  p0 = f ? np0 : p0;
  q0 = f ? nq0 : q0;
}

__device__ __forceinline__ int tc0_for(int bs, int t1, int t2, int t3) { return bs == 1 ? t1 : (bs == 2 ? t2 : t3); }

// Filter thresholds of one picture (uniform QP): luma and chroma alpha/beta
// and tC0 for bS 1..3.
struct DbQ {
  int al, be, alc, bec, tcl1, tcl2, tcl3, tcc1, tcc2, tcc3, is_intra;
};

__device__ __forceinline__ DbQ db_q(int qp, int is_intra) {
  const int qpc = chroma_qp(qp);
  return DbQ{kAlpha[qp], kBeta[qp], kAlpha[qpc], kBeta[qpc], kTc0[qp][0], kTc0[qp][1], kTc0[qp][2],
             kTc0[qpc][0], kTc0[qpc][1], kTc0[qpc][2], is_intra};
}

// One macroblock's filtering steps on samples in shared memory, one warp per
// step, lanes 0..15 (the callers skip them when alpha or beta is 0). `bs` is
// the macroblock's 32 boundary strengths ([dir][edge][segment]).
//
// Vertical edges of a luma macroblock: lane = sample row. `row` is the
// macroblock row's first sample row, `xo` the macroblock's byte offset in it,
// `xl` the left macroblock's (used iff has_left); 20 samples from p3 of the
// left edge to q3 of the last internal edge, in registers.
__device__ __forceinline__ void luma_v_step(uint8_t* row, int sp, int xo, int xl, bool has_left, const uint8_t* bs,
                                            int lane, const DbQ& q) {
  uint8_t* rowb = row + (size_t)lane * sp;
  uint32_t* rw = reinterpret_cast<uint32_t*>(rowb + xo);
  uint32_t* lw = reinterpret_cast<uint32_t*>(rowb + xl + 12);
  int v[20];
  const uint32_t w0 = has_left ? *lw : 0u;
  const uint32_t w1 = rw[0], w2 = rw[1], w3 = rw[2], w4 = rw[3];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    v[k] = (w0 >> (8 * k)) & 255;
    v[4 + k] = (w1 >> (8 * k)) & 255;
    v[8 + k] = (w2 >> (8 * k)) & 255;
    v[12 + k] = (w3 >> (8 * k)) & 255;
    v[16 + k] = (w4 >> (8 * k)) & 255;
  }
  const int seg = lane >> 2;
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int b = bs[e * 4 + seg];
    const int i = 4 + 4 * e;
    if (q.is_intra && e == 0)
      luma_strong(v[i - 4], v[i - 3], v[i - 2], v[i - 1], v[i], v[i + 1], v[i + 2], v[i + 3], b, q.al, q.be);
    else
      luma_normal(v[i - 3], v[i - 2], v[i - 1], v[i], v[i + 1], v[i + 2], b, q.al, q.be,
                  tc0_for(b, q.tcl1, q.tcl2, q.tcl3));
  }
  uint32_t o[5];
#pragma unroll
  for (int k = 0; k < 5; ++k)
    o[k] = (uint32_t)v[4 * k] | ((uint32_t)v[4 * k + 1] << 8) | ((uint32_t)v[4 * k + 2] << 16) |
           ((uint32_t)v[4 * k + 3] << 24);
  if (has_left) *lw = o[0];
  rw[0] = o[1];
  rw[1] = o[2];
  rw[2] = o[3];
  rw[3] = o[4];
}

// Vertical edges of one chroma plane's sample row (lane = plane * 8 + row):
// chroma samples 8mx-2 .. 8mx+7 (every other byte of the NV12 row).
__device__ __forceinline__ void chroma_v_step(uint8_t* row, int sp, int xo, int xl, bool has_left, const uint8_t* bs,
                                              int lane, const DbQ& q) {
  const int pl = lane >> 3, i = lane & 7;
  uint8_t* rowb = row + (size_t)i * sp;
  uint8_t* cur = rowb + xo + pl;
  uint8_t* left = rowb + xl + pl;
  int v[10];
  v[0] = has_left ? left[12] : 0;
  v[1] = has_left ? left[14] : 0;
#pragma unroll
  for (int k = 2; k < 10; ++k) v[k] = cur[2 * (k - 2)];
  const int seg = i >> 1;
#pragma unroll
  for (int e = 0; e < 4; e += 2) {
    const int b = bs[e * 4 + seg];
    const int j = 2 + 2 * e;
    if (q.is_intra && e == 0)
      chroma_strong(v[j - 2], v[j - 1], v[j], v[j + 1], b, q.alc, q.bec);
    else
      chroma_normal(v[j - 2], v[j - 1], v[j], v[j + 1], b, q.alc, q.bec, tc0_for(b, q.tcc1, q.tcc2, q.tcc3));
  }
  if (has_left) left[14] = (uint8_t)v[1];
#pragma unroll
  for (int k = 2; k < 10; ++k) cur[2 * (k - 2)] = (uint8_t)v[k];
}

// Horizontal edges of a luma macroblock: lane = sample column, rows -4..15;
// `top` is the sample row four rows above the macroblock.
__device__ __forceinline__ void luma_h_step(uint8_t* top, int sp, int xo, const uint8_t* bs, int lane, const DbQ& q) {
  uint8_t* col = top + xo + lane;
  int v[20];
#pragma unroll
  for (int r = 0; r < 20; ++r) v[r] = col[(size_t)r * sp];
  const int seg = lane >> 2;
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int b = bs[16 + e * 4 + seg];
    const int i = 4 + 4 * e;
    if (q.is_intra && e == 0)
      luma_strong(v[i - 4], v[i - 3], v[i - 2], v[i - 1], v[i], v[i + 1], v[i + 2], v[i + 3], b, q.al, q.be);
    else
      luma_normal(v[i - 3], v[i - 2], v[i - 1], v[i], v[i + 1], v[i + 2], b, q.al, q.be,
                  tc0_for(b, q.tcl1, q.tcl2, q.tcl3));
  }
#pragma unroll
  for (int r = 1; r < 19; ++r) col[(size_t)r * sp] = (uint8_t)v[r];
}

// Horizontal edges of a chroma macroblock: lane = plane + 2 * column, rows
// -2..7; `top` is the chroma sample row two rows above the macroblock.
__device__ __forceinline__ void chroma_h_step(uint8_t* top, int sp, int xo, const uint8_t* bs, int lane,
                                              const DbQ& q) {
  const int pl = lane >> 3, i = lane & 7;
  uint8_t* col = top + xo + 2 * i + pl;
  int v[10];
#pragma unroll
  for (int r = 0; r < 10; ++r) v[r] = col[(size_t)r * sp];
  const int seg = i >> 1;
#pragma unroll
  for (int e = 0; e < 4; e += 2) {
    const int b = bs[16 + e * 4 + seg];
    const int j = 2 + 2 * e;
    if (q.is_intra && e == 0)
      chroma_strong(v[j - 2], v[j - 1], v[j], v[j + 1], b, q.alc, q.bec);
    else
      chroma_normal(v[j - 2], v[j - 1], v[j], v[j + 1], b, q.alc, q.bec, tc0_for(b, q.tcc1, q.tcc2, q.tcc3));
  }
#pragma unroll
  for (int r = 1; r < 9; ++r) col[(size_t)r * sp] = (uint8_t)v[r];
}

// Boundary strength (clause 8.7.2.1 for this encoder's macroblock kinds) of
// segment k of edge e in direction dir of macroblock mb; has_edge0 = the
// macroblock edge is filtered (a left / upper neighbour inside the picture
// being deblocked).
// Nonzero levels in the transform block holding 4x4 block b (raster) of
// macroblock mb: the 4x4 block, or with the 8x8 transform (t8[mb]) its 8x8
// block (h264_deblock.c:119-137).
__device__ __forceinline__ uint32_t db_coef(const uint32_t* __restrict__ nzm, const uint8_t* __restrict__ t8, int mb,
                                            int b) {
  const uint32_t* n = nzm + (size_t)mb * 24;
  if (!t8 || !t8[mb]) return __ldg(n + b) & 0xffffu;
  const int c = b & 10;
  return (__ldg(n + c) | __ldg(n + c + 1) | __ldg(n + c + 4) | __ldg(n + c + 5)) & 0xffffu;
}

__device__ __forceinline__ int db_bs(int k, int e, int dir, int mb, int mbw, bool has_edge0, int is_intra,
                                     const uint32_t* __restrict__ nzm, const MV* __restrict__ mvs,
                                     const uint8_t* __restrict__ t8 = nullptr) {
  if (e == 0 && !has_edge0) return 0;
  if ((e & 1) && t8 && t8[mb]) return 0;  // no luma edge inside an 8x8 transform block (h264_deblock.c:294,324)
  if (is_intra) return e == 0 ? 4 : 3;
  const int mbp = e ? mb : (dir == 0 ? mb - 1 : mb - mbw);
  const int bq = dir == 0 ? k * 4 + e : e * 4 + k;
  const int bp = e ? (dir == 0 ? bq - 1 : bq - 4) : (dir == 0 ? k * 4 + 3 : 12 + k);
  if (db_coef(nzm, t8, mbp, bp) | db_coef(nzm, t8, mb, bq)) return 2;
  if (e != 0) return 0;
  const int2 a = __ldg(reinterpret_cast<const int2*>(mvs + mbp));
  const int2 c = __ldg(reinterpret_cast<const int2*>(mvs + mb));
  return (abs(a.x - c.x) >= 4 || abs(a.y - c.y) >= 4) ? 1 : 0;
}

// Shared-memory plan of one CTA (dynamic shared memory). The group's rows
// are held as a ring of kDbRing macroblock columns (column mx in slot
// mx % kDbRing), not the whole picture width:
//   luma ring   : (16R + 4) rows x sp bytes, row 0 = picture row 16*y0 - 4
//   chroma ring : (8R + 2) rows x sp bytes (NV12), row 0 = picture row 8*y0 - 2
//   bS          : R x mbw x 32 bytes ([dir][edge][segment] per macroblock)
//   progress    : 2R words (luma rows, then chroma rows), 2 words of loaded
//                 columns (luma, chroma), 2 words of columns whose halo rows
//                 are in as well (luma, chroma)
// sp = 16*kDbRing + 4: a 4-byte skew per row keeps the 16 lanes that walk 16
// consecutive rows of one column on 16 different banks.
constexpr int kDbRing = 16;

struct DbPlan {
  int R, sp;
  size_t luma_off, chroma_off, bs_off, prog_off, bytes;
};

__host__ __device__ inline DbPlan db_plan(int mbw, int R) {
  DbPlan p;
  p.R = R;
  p.sp = 16 * kDbRing + 4;
  p.luma_off = 0;
  p.chroma_off = p.luma_off + (size_t)(16 * R + 4) * p.sp;
  p.bs_off = p.chroma_off + (size_t)(8 * R + 2) * p.sp;
  p.prog_off = (p.bs_off + (size_t)R * mbw * 32 + 15) & ~(size_t)15;
  p.bytes = p.prog_off + (2 * R + 4) * sizeof(uint32_t);
  return p;
}

// Bounded wait on a shared progress word: give up after max_wait_us
// microseconds of %globaltimer, or as soon as another CTA has recorded an
// error. Called by all 32 lanes of a warp: each poll is one broadcast
// shared load and the lanes stay converged. (Lane 0 spinning alone while the
// other lanes waited at a shuffle for its result measured ~2000 cycles more
// per wait, even when the word was already there.)
__device__ __forceinline__ bool wait_shared(const volatile uint32_t* flag, const Scratch& sc, uint32_t need,
                                            uint32_t max_wait_us, uint32_t where) {
  const uint64_t t0 = global_ns(), budget = (uint64_t)max_wait_us * 1000u;
  for (uint32_t it = 0;; ++it) {
    if (*flag >= need) return true;
    if ((it & 63) == 63) {
      if (load_acquire(sc.err()) != 0u) return false;
      if (global_ns() - t0 > budget) break;
    }
    __nanosleep(32);  // leave the issue slots to the warps doing the work
  }
  if (atomicCAS(sc.err(), 0u, kErrWaitTimeout) == 0u) atomicExch(sc.err_detail(), where);
  return false;
}

// BATCH: the group tickets (bt.ticket[1]) run over the row groups of every
// stream of a batch (bt.groups, R = bt.db_rows rows each); a group waits
// only on its own stream's rows and scratch. Dynamic shared memory is sized
// for the widest stream.
template <bool BATCH>
__global__ void deblock_kernel(int mbw_, int mbh_, int R, int qp_, int is_intra_,
                                                      const uint32_t* __restrict__ nzm_, const MV* __restrict__ mvs_,
                                                      uint8_t* rec_y_, uint8_t* rec_uv_, int rec_pitch_,
                                                      uint32_t* scratch_, uint32_t max_wait, BatchTab bt) {  // max_wait in microseconds
  extern __shared__ __align__(16) uint8_t smem[];
  __shared__ int s_group, s_abort;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nthr = blockDim.x;

  auto scol = [](int mx) { return 16 * (mx & (kDbRing - 1)); };  // byte offset of MB column mx in a ring row

  for (;;) {
    if (tid == 0) {
      s_group = (int)atomicAdd(BATCH ? bt.ticket + 1 : Scratch{scratch_}.ticket(), 1u);
      s_abort = 0;
    }
    __syncthreads();
    int mbw = mbw_, mbh = mbh_, qp = qp_, is_intra = is_intra_, rec_pitch = rec_pitch_;
    const uint32_t* nzm = nzm_;
    const MV* mvs = mvs_;
    uint8_t *rec_y = rec_y_, *rec_uv = rec_uv_;
    uint32_t* scratch = scratch_;
    int group = s_group;
    if (BATCH) {
      if (group >= bt.groups.total()) return;
      const int k = bt.groups.find(group);
      const BatchStream& st = bt.groups.stream(k);
      group -= bt.groups.prefix[k];
      mbw = st.g.mbw;
      mbh = st.g.mbh;
      qp = st.qp;
      is_intra = st.is_intra;
      nzm = st.nz;
      mvs = st.mv;
      rec_y = st.rec_y;
      rec_uv = st.rec_uv;
      rec_pitch = st.rec_pitch;
      scratch = st.scr_db;
    }
    const int y0 = group * R;
    if (y0 >= mbh) return;
    const DbPlan P = db_plan(mbw, R);
    uint8_t* ly = smem + P.luma_off;
    uint8_t* cy = smem + P.chroma_off;
    uint8_t* bsm = smem + P.bs_off;
    volatile uint32_t* prog = reinterpret_cast<volatile uint32_t*>(smem + P.prog_off);
    const Scratch sc{scratch};
    uint32_t* gprog_luma = scratch + 4;
    uint32_t* gprog_chroma = scratch + 4 + mbh;
    const DbQ q = db_q(qp, is_intra);
    const int rows = min(R, mbh - y0);
    const bool has_next = y0 + rows < mbh;

    // ---- prologue: progress words and the group's boundary strengths -----
    for (int i = tid; i < 2 * R + 4; i += nthr) prog[i] = 0u;
    for (int i = tid; i < rows * mbw * 32; i += nthr) {
      const int k = i & 3, e = (i >> 2) & 3, dir = (i >> 4) & 1, m = i >> 5;
      const int my = y0 + m / mbw, mx = m % mbw;
      bsm[i] = (uint8_t)db_bs(k, e, dir, my * mbw + mx, mbw, dir == 0 ? mx > 0 : my > 0, is_intra, nzm, mvs);
    }
    __syncthreads();

    const bool is_luma = warp < R;
    const int wr = is_luma ? warp : warp - R;  // row within the group
    const int y = y0 + wr;
    if (warp >= 2 * R + 2) {
      // ---- halo warp: luma (2R+2) or chroma (2R+3) ---------------------------
      // Fetches the halo rows above the group (the bottom rows of the group
      // above) for each staged column as soon as the group above releases
      // it, and publishes how many columns the first row may start on.
      const bool hl = warp == 2 * R + 2;
      const int halo = hl ? 4 : 2;
      uint8_t* base = hl ? ly : cy;
      const uint8_t* gplane = hl ? rec_y : rec_uv;
      const int grow = hl ? 16 * y0 - 4 : 8 * y0 - 2;  // picture row of ring row 0
      const volatile uint32_t* loaded_prog = prog + 2 * R + (hl ? 0 : 1);
      volatile uint32_t* ready_prog = prog + 2 * R + (hl ? 2 : 3);
      const uint32_t* gflag = (hl ? gprog_luma : gprog_chroma) + (y0 - 1);
      int ready = 0;
      uint32_t idle = 0;
      uint64_t t_idle = 0;
      while (ready < mbw) {
        uint32_t l = 0, g = (uint32_t)mbw;
        if (lane == 0) {
          l = *loaded_prog;
          if (y0 > 0) g = load_acquire(gflag);
        }
        l = __shfl_sync(0xffffffffu, l, 0);
        g = __shfl_sync(0xffffffffu, g, 0);
        const int upto = min((int)g, (int)l);
        if (upto > ready) {
          __threadfence_block();
          if (y0 > 0)
            for (int c = ready; c < upto; ++c)
              if (lane < halo) {
                const uint4 v = __ldcg(reinterpret_cast<const uint4*>(gplane + (size_t)(grow + lane) * rec_pitch + 16 * c));
                uint32_t* d = reinterpret_cast<uint32_t*>(base + (size_t)lane * P.sp + scol(c));
                d[0] = v.x;
                d[1] = v.y;
                d[2] = v.z;
                d[3] = v.w;
              }
          ready = upto;
          __threadfence_block();
          __syncwarp();
          if (lane == 0) *ready_prog = (uint32_t)ready;
          idle = 0;
          continue;
        }
        int stop = 0;
        if (lane == 0) {
          if (idle == 0) t_idle = global_ns();
          if ((idle & 63) == 63) {
            if (load_acquire(sc.err()) != 0u) {
              stop = 1;
            } else if (global_ns() - t_idle > (uint64_t)max_wait * 1000u) {
              if (atomicCAS(sc.err(), 0u, kErrWaitTimeout) == 0u)
                atomicExch(sc.err_detail(), (uint32_t)(y0 * mbw + ready));
              stop = 1;
            }
          }
        }
        ++idle;
        stop = __shfl_sync(0xffffffffu, stop, 0);
        if (stop) {
          s_abort = 1;
          break;
        }
        __nanosleep(128);  // off the rows' critical path: poll gently
      }
    } else if (warp >= 2 * R) {
      // ---- IO warp: luma (2R) or chroma (2R+1) -------------------------------
      // Loads the group's macroblock columns into the ring ahead of its first
      // row; once the group's last row has filtered the vertical edges of
      // macroblock c+1 (the last change to column c), writes column c back
      // (the halo rows above the group, modified by the first row's top
      // edges, included) and releases column c to the next group. Releases
      // come before loads, and only the rows the next group reads are
      // written ahead of the release's fence.
      const bool io_luma = warp == 2 * R;
      const int halo = io_luma ? 4 : 2, nrows = io_luma ? 16 * rows : 8 * rows;
      uint8_t* base = io_luma ? ly : cy;
      uint8_t* gplane = io_luma ? rec_y : rec_uv;
      const int grow0 = io_luma ? 16 * y0 : 8 * y0;  // picture row of ring row `halo`
      volatile uint32_t* loaded_prog = prog + 2 * R + (io_luma ? 0 : 1);
      const volatile uint32_t* last_prog = prog + (io_luma ? 0 : R) + (rows - 1);
      uint32_t* gflag = (io_luma ? gprog_luma : gprog_chroma) + (y0 + rows - 1);
      const int wb0 = y0 > 0 ? 1 : halo, wb1 = halo + nrows;  // ring rows written back
      int loaded = 0, evicted = 0;
      uint32_t idle = 0;
      uint64_t t_idle = 0;
      while (evicted < mbw) {
        bool did = false;
        // Releases first: they gate the next group. Columns [0, d) are
        // final (one read, broadcast: the word keeps moving).
        uint32_t d = *last_prog;
        if ((int)d > evicted) {
          __threadfence_block();
          const int nc = (int)d - evicted;
          if (has_next) {
            // the group's last `halo` rows, which the next group reads as
            // its halo, then the release; only these stores wait on the fence
            for (int t = lane; t < nc * halo; t += 32) {
              const int c = evicted + t / halo, rr = wb1 - halo + t % halo;
              const uint32_t* s4 = reinterpret_cast<const uint32_t*>(base + (size_t)rr * P.sp + scol(c));
              __stcg(reinterpret_cast<uint4*>(gplane + (size_t)(grow0 + rr - halo) * rec_pitch + 16 * c),
                     make_uint4(s4[0], s4[1], s4[2], s4[3]));
            }
            __threadfence();
            __syncwarp();
            if (lane == 0) store_release(gflag, d);
          }
          // the other rows (the next group writes its halo rows back itself,
          // so they are not written again here)
          const int wbe = has_next ? wb1 - halo : wb1;
          for (int c = evicted; c < (int)d; ++c)
            for (int rr = wb0 + lane; rr < wbe; rr += 32) {
              const uint32_t* s4 = reinterpret_cast<const uint32_t*>(base + (size_t)rr * P.sp + scol(c));
              __stcg(reinterpret_cast<uint4*>(gplane + (size_t)(grow0 + rr - halo) * rec_pitch + 16 * c),
                     make_uint4(s4[0], s4[1], s4[2], s4[3]));
            }
          evicted = (int)d;
          did = true;
        }
        // then at most two columns of loads before looking for releases again
        for (int n = 0; n < 2 && loaded < mbw && loaded - evicted < kDbRing; ++n) {
          for (int r = lane; r < nrows; r += 32) {  // one 16-byte row segment per lane
            const uint4 v = __ldcg(reinterpret_cast<const uint4*>(gplane + (size_t)(grow0 + r) * rec_pitch + 16 * loaded));
            uint32_t* w = reinterpret_cast<uint32_t*>(base + (size_t)(halo + r) * P.sp + scol(loaded));
            w[0] = v.x;
            w[1] = v.y;
            w[2] = v.z;
            w[3] = v.w;
          }
          ++loaded;
          did = true;
          __threadfence_block();
          __syncwarp();
          if (lane == 0) *loaded_prog = (uint32_t)loaded;
        }
        if (did) {
          idle = 0;
          continue;
        }
        // nothing to do until the last row moves
        int stop = 0;
        if (lane == 0) {
          if (idle == 0) t_idle = global_ns();
          if ((idle & 63) == 63) {
            if (load_acquire(sc.err()) != 0u) {
              stop = 1;
            } else if (global_ns() - t_idle > (uint64_t)max_wait * 1000u) {
              if (atomicCAS(sc.err(), 0u, kErrWaitTimeout) == 0u)
                atomicExch(sc.err_detail(), (uint32_t)((y0 + rows - 1) * mbw + evicted));
              stop = 1;
            }
          }
        }
        ++idle;
        stop = __shfl_sync(0xffffffffu, stop, 0);
        if (stop) {
          s_abort = 1;
          break;
        }
        __nanosleep(128);
      }
    } else if (wr < rows) {
      const uint8_t* bsrow = bsm + (size_t)wr * mbw * 32;
      volatile uint32_t* my_prog = prog + (is_luma ? 0 : R) + wr;
      const volatile uint32_t* up_prog = prog + (is_luma ? 0 : R) + wr - 1;
      const volatile uint32_t* loaded_prog = prog + 2 * R + (is_luma ? 0 : 1);
      const volatile uint32_t* ready_prog = prog + 2 * R + (is_luma ? 2 : 3);
      for (int mx = 0; mx < mbw; ++mx) {
        const uint32_t need = (uint32_t)(mx + 1);
        bool ok = true;
        // Vertical edges read and write only this row's own sample rows, so
        // they need nothing from the row above, only the columns staged in
        // the ring: the first row waits for them; every other row is behind
        // the row above (which waited) except at its first macroblock.
        if (wr == 0) {
          ok = wait_shared(loaded_prog, sc, need, max_wait, (uint32_t)(y * mbw + mx));
          __threadfence_block();
        } else if (mx == 0) {
          ok = wait_shared(loaded_prog, sc, 1u, max_wait, (uint32_t)(y * mbw));
          __threadfence_block();
        }
        if (!ok) {
          s_abort = 1;
          break;
        }
        __syncwarp();
        const uint8_t* bs = bsrow + mx * 32;
        if (is_luma) {
          if (q.al && q.be && lane < 16)
            luma_v_step(ly + (size_t)(4 + 16 * wr) * P.sp, P.sp, scol(mx), scol(mx - 1), mx > 0, bs, lane, q);
        } else {
          if (q.alc && q.bec && lane < 16)
            chroma_v_step(cy + (size_t)(2 + 8 * wr) * P.sp, P.sp, scol(mx), scol(mx - 1), mx > 0, bs, lane, q);
        }
        __syncwarp();
        // Macroblock mx-1's samples are final for this row now (the left
        // edge of mx was their last change).
        if (mx > 0) {
          __threadfence_block();
          __syncwarp();
          if (lane == 0) *my_prog = (uint32_t)mx;
        }
        // Horizontal edges of mx read and change the bottom rows of the
        // macroblock above, which are final once the row above has filtered
        // the vertical edges of mx+1: a skew of one macroblock step per row.
        // The first row waits for the halo rows above the group instead.
        if (wr == 0) {
          ok = wait_shared(ready_prog, sc, need, max_wait, (uint32_t)(y * mbw + mx));
          __threadfence_block();
        } else {
          ok = wait_shared(up_prog, sc, need, max_wait, (uint32_t)(y * mbw + mx));
          __threadfence_block();
        }
        if (!ok) {
          s_abort = 1;
          break;
        }
        __syncwarp();
        if (is_luma) {
          if (q.al && q.be && lane < 16) luma_h_step(ly + (size_t)(16 * wr) * P.sp, P.sp, scol(mx), bs, lane, q);
        } else {
          if (q.alc && q.bec && lane < 16) chroma_h_step(cy + (size_t)(8 * wr) * P.sp, P.sp, scol(mx), bs, lane, q);
        }
        if (mx == mbw - 1) {  // all of the row's macroblocks are final
          __syncwarp();
          __threadfence_block();
          __syncwarp();
          if (lane == 0) *my_prog = (uint32_t)mbw;
        }
      }
    }
    __syncthreads();
    if (s_abort) return;
  }
}


// ---------------------------------------------------------------------------
// Tile deblocking. Raster-order deblocking reaches only a short distance: a
// filter changes at most three samples either side of an edge and reads at
// most four, edges are four samples apart, and the value one edge hands to
// the next (its q1, read back as the next edge's p2) depends on that edge's
// own inputs only, so a change does not travel along a row or a column. As a
// result the deblocked samples of a tile of macroblocks are those of the
// raster-order deblocking of the tile with one macroblock of margin on every
// side (clipped at the picture), treated as a picture of its own (no
// filtering on the margin's outer edges). The oracle checks this against
// whole-picture deblocking on random and adversarial content, intra and
// inter, for several tile shapes (tests/test_deblock_tiles.py).
//
// So each CTA takes one tile: it loads the tile and its margin from the
// unfiltered reconstruction (`src`) into shared memory, deblocks it there in
// raster order (the row wavefront of the kernel above, one luma and one
// chroma warp per macroblock row, rows a macroblock step apart), and stores
// the tile alone to `dst`. CTAs never wait on one another; a picture is
// mbw/TW x mbh/TH independent tiles of (TW + TH + 3) dependent steps each,
// instead of one wavefront of mbw + mbh - 1 steps. `dst` must not overlap
// `src` (neighbouring tiles read each other's samples as their margin).
// ---------------------------------------------------------------------------
constexpr int kDbTileMax = 8;    // TH <= 8 (a luma and a chroma warp per region row)
constexpr int kDbTileMaxW = 16;  // TW <= 16 (the width sets shared memory only: 78 KB at 16 x 8)

struct DbTilePlan {
  int sp;  // shared-memory row stride: 16 * (TW + 2) + 4 bytes, an odd word count
  size_t luma_off, chroma_off, bs_off, prog_off, bytes;
};

__host__ __device__ inline DbTilePlan db_tile_plan(int TW, int TH) {
  DbTilePlan p;
  p.sp = 16 * (TW + 2) + 4;
  p.luma_off = 0;                                                    // 4 margin rows + 16 (TH + 2) rows
  p.chroma_off = (size_t)(16 * (TH + 2) + 4) * p.sp;                 // 2 margin rows + 8 (TH + 2) rows
  p.bs_off = p.chroma_off + (size_t)(8 * (TH + 2) + 2) * p.sp;       // [MB][dir][edge][segment]
  p.prog_off = (p.bs_off + (size_t)(TH + 2) * (TW + 2) * 32 + 15) & ~(size_t)15;
  p.bytes = p.prog_off + 2 * (TH + 2) * sizeof(uint32_t);            // progress: luma rows, chroma rows
  return p;
}

// BATCH: one CTA per tile of every stream of a batch (bt.groups counts each
// stream's tiles; bt.db_rows = TH, bt.db_cols = TW); the stream's unfiltered
// reconstruction is rec_y/rec_uv, the deblocked one goes to db_y/db_uv.
template <bool BATCH>
__global__ void __launch_bounds__(64 * (kDbTileMax + 2), 2) deblock_tile_kernel(
    int mbw_, int mbh_, int TW, int TH, int qp_, int is_intra_, const uint32_t* __restrict__ nzm_,
    const MV* __restrict__ mvs_, const uint8_t* __restrict__ t8_, const uint8_t* __restrict__ src_y_,
    const uint8_t* __restrict__ src_uv_,
    uint8_t* __restrict__ dst_y_, uint8_t* __restrict__ dst_uv_, int pitch_, uint32_t* status_, uint32_t max_wait,
    BatchTab bt) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nthr = blockDim.x;
  int mbw = mbw_, mbh = mbh_, qp = qp_, is_intra = is_intra_, pitch = pitch_;
  const uint32_t* nzm = nzm_;
  const MV* mvs = mvs_;
  const uint8_t *src_y = src_y_, *src_uv = src_uv_;
  uint8_t *dst_y = dst_y_, *dst_uv = dst_uv_;
  uint32_t* status = status_;
  int tile = blockIdx.x;
  if (BATCH) {
    if (tile >= bt.groups.total()) return;
    TW = bt.db_cols;
    TH = bt.db_rows;
    const int k = bt.groups.find(tile);
    const BatchStream& st = bt.groups.stream(k);
    tile -= bt.groups.prefix[k];
    mbw = st.g.mbw;
    mbh = st.g.mbh;
    qp = st.qp;
    is_intra = st.is_intra;
    nzm = st.nz;
    mvs = st.mv;
    src_y = st.rec_y;
    src_uv = st.rec_uv;
    dst_y = st.db_y;
    dst_uv = st.db_uv;
    pitch = st.rec_pitch;
    status = st.scr_db;
  }
  const int ntx = (mbw + TW - 1) / TW;
  const int tx = tile % ntx, ty = tile / ntx;
  const int x0 = tx * TW, y0 = ty * TH;
  if (y0 >= mbh) return;
  const int x1 = min(mbw, x0 + TW), y1 = min(mbh, y0 + TH);
  // the deblocked region: the tile and its margin, clipped at the picture
  const int rx0 = max(0, x0 - 1), ry0 = max(0, y0 - 1), rx1 = min(mbw, x1 + 1), ry1 = min(mbh, y1 + 1);
  const int RWr = rx1 - rx0, RHr = ry1 - ry0;
  const DbTilePlan P = db_tile_plan(TW, TH);
  uint8_t* ly = smem + P.luma_off;    // row 4 = picture row 16 * ry0, byte 0 = column 16 * rx0
  uint8_t* cy = smem + P.chroma_off;  // row 2 = picture row 8 * ry0
  uint8_t* bsm = smem + P.bs_off;
  volatile uint32_t* prog = reinterpret_cast<volatile uint32_t*>(smem + P.prog_off);
  const Scratch sc{status};
  const DbQ q = db_q(qp, is_intra);

  // ---- load the region, boundary strengths, progress words -----------------
  {
    const int lrows = 16 * RHr, crows = 8 * RHr, n = (lrows + crows) * RWr;
    for (int i = tid; i < n; i += nthr) {
      const int r = i / RWr, c = i - r * RWr;
      const bool lu = r < lrows;
      const int rr = lu ? r : r - lrows;
      const uint8_t* g = lu ? src_y + (size_t)(16 * ry0 + rr) * pitch + 16 * (rx0 + c)
                            : src_uv + (size_t)(8 * ry0 + rr) * pitch + 16 * (rx0 + c);
      const uint4 v = __ldg(reinterpret_cast<const uint4*>(g));
      uint32_t* d = reinterpret_cast<uint32_t*>((lu ? ly + (size_t)(4 + rr) * P.sp : cy + (size_t)(2 + rr) * P.sp) +
                                                16 * c);
      d[0] = v.x;
      d[1] = v.y;
      d[2] = v.z;
      d[3] = v.w;
    }
    // the margin rows above the region are read (never changed: the top
    // edges of the region's first row have bS 0) by its first row's
    // horizontal steps; give them defined contents
    for (int i = tid; i < 6 * (P.sp / 4); i += nthr) {
      const int r = i / (P.sp / 4), w = i - r * (P.sp / 4);
      reinterpret_cast<uint32_t*>(r < 4 ? ly + (size_t)r * P.sp : cy + (size_t)(r - 4) * P.sp)[w] = 0u;
    }
    for (int i = tid; i < RHr * RWr * 32; i += nthr) {
      const int k = i & 3, e = (i >> 2) & 3, dir = (i >> 4) & 1, m = i >> 5;
      const int lyr = m / RWr, lxr = m - lyr * RWr;
      bsm[i] = (uint8_t)db_bs(k, e, dir, (ry0 + lyr) * mbw + rx0 + lxr, mbw, dir == 0 ? lxr > 0 : lyr > 0, is_intra,
                              nzm, mvs, BATCH ? nullptr : t8_);
    }
    for (int i = tid; i < 2 * (TH + 2); i += nthr) prog[i] = 0u;
  }
  __syncthreads();

  // ---- the region's rows, one luma and one chroma warp each ----------------
  {
    const bool is_luma = warp < TH + 2;
    const int wr = is_luma ? warp : warp - (TH + 2);
    if (wr < RHr) {
      const uint8_t* bsrow = bsm + (size_t)wr * RWr * 32;
      volatile uint32_t* my_prog = prog + (is_luma ? 0 : TH + 2) + wr;
      const volatile uint32_t* up_prog = my_prog - 1;
      const bool on = is_luma ? (q.al && q.be) : (q.alc && q.bec);
      uint8_t* vrow = is_luma ? ly + (size_t)(4 + 16 * wr) * P.sp : cy + (size_t)(2 + 8 * wr) * P.sp;
      uint8_t* htop = is_luma ? ly + (size_t)(16 * wr) * P.sp : cy + (size_t)(8 * wr) * P.sp;
      for (int mx = 0; mx < RWr; ++mx) {
        const uint8_t* bs = bsrow + mx * 32;
        // vertical edges: this row's own samples only
        if (on && lane < 16) {
          if (is_luma)
            luma_v_step(vrow, P.sp, 16 * mx, 16 * (mx - 1), mx > 0, bs, lane, q);
          else
            chroma_v_step(vrow, P.sp, 16 * mx, 16 * (mx - 1), mx > 0, bs, lane, q);
        }
        __syncwarp();
        if (mx > 0) {  // macroblock mx-1 of this row is final
          __threadfence_block();
          __syncwarp();
          if (lane == 0) *my_prog = (uint32_t)mx;
        }
        // horizontal edges of mx: the row above has filtered the vertical
        // edges of mx+1 (all of its row at the last macroblock)
        if (wr > 0) {
          if (!wait_shared(up_prog, sc, (uint32_t)(mx + 1), max_wait,
                           (uint32_t)((ry0 + wr) * mbw + rx0 + mx)))
            break;
          __threadfence_block();
        }
        __syncwarp();
        if (on && lane < 16) {
          if (is_luma)
            luma_h_step(htop, P.sp, 16 * mx, bs, lane, q);
          else
            chroma_h_step(htop, P.sp, 16 * mx, bs, lane, q);
        }
        if (mx == RWr - 1) {
          __syncwarp();
          __threadfence_block();
          __syncwarp();
          if (lane == 0) *my_prog = (uint32_t)RWr;
        }
      }
    }
  }
  __syncthreads();

  // ---- store the tile (whatever a failed wait left: the status says so) -----
  {
    const int tw = x1 - x0, lrows = 16 * (y1 - y0), crows = 8 * (y1 - y0), n = (lrows + crows) * tw;
    const int ox = x0 - rx0, oy = y0 - ry0;  // the tile's macroblock offset in the region
    for (int i = tid; i < n; i += nthr) {
      const int r = i / tw, c = i - r * tw;
      const bool lu = r < lrows;
      const int rr = lu ? r : r - lrows;
      const uint32_t* s4 = reinterpret_cast<const uint32_t*>(
          (lu ? ly + (size_t)(4 + 16 * oy + rr) * P.sp : cy + (size_t)(2 + 8 * oy + rr) * P.sp) + 16 * (ox + c));
      uint8_t* g = lu ? dst_y + (size_t)(16 * y0 + rr) * pitch + 16 * (x0 + c)
                      : dst_uv + (size_t)(8 * y0 + rr) * pitch + 16 * (x0 + c);
      *reinterpret_cast<uint4*>(g) = make_uint4(s4[0], s4[1], s4[2], s4[3]);
    }
  }
}

}  // namespace b200enc

using namespace b200enc;

static constexpr uint32_t kMaxWaitUsDb = 2000000u;  // 2 s

// Rows per CTA: 4 unless the autotuner chose otherwise (one luma + one
// chroma warp each, plus two IO and two halo warps: 64R + 128 threads). The ring must hold the 2*R columns a group's rows
// span plus prefetch, so R stays well below kDbRing.
static int db_rows_per_cta(int mbw, int mbh) {
  int dev = 0, maxsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (maxsm <= 0) maxsm = 48 * 1024;
  const int tuned = b200enc_tuned(B200ENC_TUNE_DEBLOCK_ROWS);
  int R = tuned > 0 ? tuned : 4;
  while (R > 1 && db_plan(mbw, R).bytes + 64 > (size_t)maxsm) --R;
  if (R > mbh) R = mbh;
  if (db_plan(mbw, R).bytes + 64 > (size_t)maxsm) return 0;
  return R;
}

extern "C" int b200enc_deblock_launch(int mbw, int mbh, int qp, int is_intra, const uint32_t* nz, const void* mv,
                                      uint8_t* rec_y, uint8_t* rec_uv, int rec_pitch, uint32_t* scratch, int ctas,
                                      uint32_t max_wait, void* stream) {
  const int R = db_rows_per_cta(mbw, mbh);
  if (R <= 0) return -1;
  const DbPlan P = db_plan(mbw, R);
  const int groups = (mbh + R - 1) / R;
  if (ctas <= 0 || ctas > groups) ctas = groups;
  if (cudaFuncSetAttribute(deblock_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P.bytes) !=
      cudaSuccess)
    return -1;
  deblock_kernel<false><<<ctas, 64 * R + 128, P.bytes, (cudaStream_t)stream>>>(
      mbw, mbh, R, qp, is_intra, nz, (const MV*)mv, rec_y, rec_uv, rec_pitch, scratch, max_wait, BatchTab{});
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// Rows per group a batch's deblocking uses for streams up to max_mbw
// macroblocks wide (0 if none fits).
int b200enc_deblock_batch_rows(int max_mbw, int max_mbh) { return db_rows_per_cta(max_mbw, max_mbh); }

// The deblocking of every stream of a batch: `ctas` persistent CTAs over
// bt.groups (bt.db_rows rows per group; each stream's scratch zeroed and
// bt.ticket[1] = 0 by the caller).
int b200enc_deblock_batch_launch(const BatchTab& bt, int max_mbw, int ctas, uint32_t max_wait, cudaStream_t st) {
  if (ctas <= 0) return 0;
  const int R = bt.db_rows;
  if (R <= 0) return -1;
  const DbPlan P = db_plan(max_mbw, R);
  if (cudaFuncSetAttribute(deblock_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P.bytes) !=
      cudaSuccess)
    return -1;
  deblock_kernel<true><<<ctas, 64 * R + 128, P.bytes, st>>>(0, 0, R, 0, 0, nullptr, nullptr, nullptr, nullptr, 0,
                                                            nullptr, max_wait, bt);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int b200enc_deblock(int mbw, int mbh, int qp, int is_intra, const uint32_t* nz, const void* mv,
                               uint8_t* rec_y, uint8_t* rec_uv, int rec_pitch, void* scratch, size_t scratch_bytes,
                               int ctas, void* stream) {
  if (!nz || !mv || !rec_y || !rec_uv || !scratch || mbw <= 0 || mbh <= 0 || qp < 0 || qp > 51) return -1;
  if ((rec_pitch & 15) || (((uintptr_t)rec_y) & 15) || (((uintptr_t)rec_uv) & 15)) return -1;
  if (rec_pitch < mbw * 16) return -1;
  if (scratch_bytes < b200enc_wavefront_scratch_bytes(mbh)) return -1;
  if (cudaMemsetAsync(scratch, 0, b200enc_wavefront_scratch_bytes(mbh), (cudaStream_t)stream) != cudaSuccess) return -1;
  return b200enc_deblock_launch(mbw, mbh, qp, is_intra, nz, mv, rec_y, rec_uv, rec_pitch, (uint32_t*)scratch, ctas,
                                kMaxWaitUsDb, stream);
}

// Tile shape of the tile deblocking (TW x TH macroblocks): 8 x 8 unless the
// autotuner chose otherwise.
static void db_tile_shape(int* tw, int* th) {
  const int w = b200enc_tuned(B200ENC_TUNE_DEBLOCK_TILE_W), h = b200enc_tuned(B200ENC_TUNE_DEBLOCK_TILE_H);
  *tw = w > 0 ? std::min(w, kDbTileMaxW) : 8;
  *th = h > 0 ? std::min(h, kDbTileMax) : 8;
}

int b200enc_deblock_tiles_launch(int mbw, int mbh, int qp, int is_intra, const uint32_t* nz, const void* mv,
                                 const uint8_t* src_y, const uint8_t* src_uv, uint8_t* dst_y, uint8_t* dst_uv,
                                 int pitch, uint32_t* status, uint32_t max_wait, cudaStream_t stream,
                                 const uint8_t* t8) {
  int TW, TH;
  db_tile_shape(&TW, &TH);
  const DbTilePlan P = db_tile_plan(TW, TH);
  if (cudaFuncSetAttribute(deblock_tile_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P.bytes) !=
      cudaSuccess)
    return -1;
  const int tiles = ((mbw + TW - 1) / TW) * ((mbh + TH - 1) / TH);
  deblock_tile_kernel<false><<<tiles, 64 * (TH + 2), P.bytes, stream>>>(
      mbw, mbh, TW, TH, qp, is_intra, nz, (const MV*)mv, t8, src_y, src_uv, dst_y, dst_uv, pitch, status,
      max_wait, BatchTab{});
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// Tiles of a stream of mbw x mbh macroblocks under the current tile shape,
// and the shape itself (for a batch's table).
int b200enc_deblock_tile_count(int mbw, int mbh, int* tw, int* th) {
  int TW, TH;
  db_tile_shape(&TW, &TH);
  if (tw) *tw = TW;
  if (th) *th = TH;
  return ((mbw + TW - 1) / TW) * ((mbh + TH - 1) / TH);
}

// The tile deblocking of every stream of a batch: one CTA per tile
// (bt.groups over the streams' tiles, bt.db_cols x bt.db_rows each).
int b200enc_deblock_tiles_batch_launch(const BatchTab& bt, int tiles, uint32_t max_wait, cudaStream_t st) {
  if (tiles <= 0) return 0;
  const int TW = bt.db_cols, TH = bt.db_rows;
  if (TW < 1 || TH < 1 || TW > kDbTileMaxW || TH > kDbTileMax) return -1;
  const DbTilePlan P = db_tile_plan(TW, TH);
  if (cudaFuncSetAttribute(deblock_tile_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P.bytes) !=
      cudaSuccess)
    return -1;
  deblock_tile_kernel<true><<<tiles, 64 * (TH + 2), P.bytes, st>>>(0, 0, 0, 0, 0, 0, nullptr, nullptr, nullptr,
                                                                   nullptr, nullptr, nullptr, nullptr, 0, nullptr,
                                                                   max_wait, bt);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int b200enc_deblock_tiles_t8(int mbw, int mbh, int qp, int is_intra, const uint32_t* nz,
                                        const uint8_t* t8, const void* mv, const uint8_t* src_y,
                                        const uint8_t* src_uv, uint8_t* dst_y, uint8_t* dst_uv, int pitch,
                                        uint32_t* status, void* stream);

extern "C" int b200enc_deblock_tiles(int mbw, int mbh, int qp, int is_intra, const uint32_t* nz, const void* mv,
                                     const uint8_t* src_y, const uint8_t* src_uv, uint8_t* dst_y, uint8_t* dst_uv,
                                     int pitch, uint32_t* status, void* stream) {
  return b200enc_deblock_tiles_t8(mbw, mbh, qp, is_intra, nz, nullptr, mv, src_y, src_uv, dst_y, dst_uv, pitch,
                                  status, stream);
}

extern "C" int b200enc_deblock_tiles_t8(int mbw, int mbh, int qp, int is_intra, const uint32_t* nz,
                                        const uint8_t* t8, const void* mv, const uint8_t* src_y,
                                        const uint8_t* src_uv, uint8_t* dst_y, uint8_t* dst_uv, int pitch,
                                        uint32_t* status, void* stream) {
  if (!nz || !mv || !src_y || !src_uv || !dst_y || !dst_uv || !status || mbw <= 0 || mbh <= 0 || qp < 0 || qp > 51)
    return -1;
  const uintptr_t a = (uintptr_t)src_y | (uintptr_t)src_uv | (uintptr_t)dst_y | (uintptr_t)dst_uv;
  if ((pitch & 15) || (a & 15) || pitch < mbw * 16) return -1;
  // the destination planes must not overlap the source planes
  const uint8_t *s0 = src_y, *s1 = src_y + (size_t)pitch * mbh * 16, *c0 = src_uv, *c1 = src_uv + (size_t)pitch * mbh * 8;
  const uint8_t *d0 = dst_y, *d1 = dst_y + (size_t)pitch * mbh * 16, *e0 = dst_uv, *e1 = dst_uv + (size_t)pitch * mbh * 8;
  auto overlap = [](const uint8_t* a0, const uint8_t* a1, const uint8_t* b0, const uint8_t* b1) {
    return a0 < b1 && b0 < a1;
  };
  if (overlap(d0, d1, s0, s1) || overlap(d0, d1, c0, c1) || overlap(e0, e1, s0, s1) || overlap(e0, e1, c0, c1))
    return -1;
  if (cudaMemsetAsync(status, 0, 16, (cudaStream_t)stream) != cudaSuccess) return -1;
  return b200enc_deblock_tiles_launch(mbw, mbh, qp, is_intra, nz, mv, src_y, src_uv, dst_y, dst_uv, pitch, status,
                                      kMaxWaitUsDb, (cudaStream_t)stream, t8);
}
