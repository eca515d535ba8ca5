// hevc_deblock.cu - HEVC deblocking (H.265 clause 8.7.2) of one 4:2:0
// picture, in place, in two launches.
//
// Reproduces the deblocking stages of the reference decoder's loop filter
// (approach1-compute-encoder/src/hevc_filter.c:449-490 over
// hevc_filter_template.c:48-420): every vertical edge of the picture first,
// then every horizontal edge over the vertically filtered picture; luma on
// the 8x8 edge grid with the strong/weak decision of the first and last
// line of each 4-line segment, chroma on the 16-luma-sample grid where the
// boundary strength is 2; per-slice beta/tC offsets and switches, tile and
// slice boundaries, lossless (no-filter) blocks, QpY averaged across the
// edge, 8- and 10-bit samples.
//
// Two launches, as the clause orders it: all vertical edges, then all
// horizontal edges. Inside a pass the edges are independent: they sit on
// the 8-sample grid and a luma filter reads 4 and writes 3 samples either
// side (chroma: 8 chroma samples apart, reads 2, writes 1), so no edge reads
// or writes a sample another edge of the same pass writes. One thread per
// 4-line segment filters in place in global memory - no tiles, no halos,
// nothing shared between threads. (A single launch over tiles with halos
// would need the neighbours' samples as the vertical pass left them, which
// an in-place neighbour may already have overwritten.) Consecutive threads
// take consecutive segments along a row, so each warp reads and writes
// contiguous runs of the picture: ~2.5 B/px of HBM traffic per pass at
// 8 bits.
#include <cstddef>

#include "b200enc_internal.h"

// The layouts the Python bindings mirror (b200enc/__init__.py).
static_assert(sizeof(b200enc_hevc_mvf_t) == 20, "mvf record");
static_assert(sizeof(b200enc_hevc_slice_filter_t) == 8, "slice filter record");
static_assert(sizeof(b200enc_hevc_deblock_t) == 168 && offsetof(b200enc_hevc_deblock_t, edges) == 64 &&
                  offsetof(b200enc_hevc_deblock_t, qp_y) == 104 && offsetof(b200enc_hevc_deblock_t, tile_of_ctb) == 144,
              "parameter block");

namespace b200enc {

// Table 8-12 (beta' by Q = 0..51, tC' by Q = 0..53) and Table 8-10 (QpC for
// qPi = 30..43), as clause 8.7.2.5.3 / 8.7.2.5.5 and 8.6.1 give them.
__constant__ uint8_t kHdbBeta[52] = {0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  6,  7,
                                     8,  9,  10, 11, 12, 13, 14, 15, 16, 17, 18, 20, 22, 24, 26, 28, 30, 32,
                                     34, 36, 38, 40, 42, 44, 46, 48, 50, 52, 54, 56, 58, 60, 62, 64};
__constant__ uint8_t kHdbTc[54] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1,  1,  1,  1,  1,  1,  1,  1,  1,
                                   2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 5, 5, 6, 6, 7, 8, 9, 10, 11, 13, 14, 16, 18, 20, 22, 24};
__constant__ uint8_t kHdbQpC[14] = {29, 30, 31, 32, 33, 33, 34, 34, 35, 35, 36, 36, 37, 37};

constexpr int kHdbThreads = 256;

__device__ __forceinline__ int hdb_clip(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// What one edge cell asks once for both its segments (hevc_filter_template.c
// :266-296): tile and slice boundaries, the q-side slice's settings, the
// lossless sides, the averaged QpY and beta.
struct HdbEdge {
  bool on, keep_p, keep_q;
  int qp, beta, tc_offset;
};

__device__ __forceinline__ int hdb_ctb(const b200enc_hevc_deblock_t& p, int x, int y, int ctb_w) {
  return (y >> p.log2_ctb) * ctb_w + (x >> p.log2_ctb);
}

__device__ HdbEdge hdb_edge(const b200enc_hevc_deblock_t& p, int x, int y, bool vertical, int ctb_w) {
  HdbEdge r;
  r.on = false;
  const int xp = vertical ? x - 1 : x, yp = vertical ? y : y - 1;
  if (p.tile_of_ctb && !p.loop_filter_across_tiles &&
      __ldg(p.tile_of_ctb + hdb_ctb(p, xp, yp, ctb_w)) != __ldg(p.tile_of_ctb + hdb_ctb(p, x, y, ctb_w)))
    return r;
  const int sq = p.slice_of_ctb ? __ldg(p.slice_of_ctb + hdb_ctb(p, x, y, ctb_w)) : 0;
  if (sq < 0 || !p.slice_filter || sq >= p.n_slice_filter) return r;
  const b200enc_hevc_slice_filter_t f = p.slice_filter[sq];
  if (f.disabled) return r;
  if (!f.across_slices) {
    const int sp = p.slice_of_ctb ? __ldg(p.slice_of_ctb + hdb_ctb(p, xp, yp, ctb_w)) : 0;
    if (sp != sq) return r;
  }
  const int l = p.log2_min_cb, mcw = p.width >> l;
  r.keep_p = p.no_filter && __ldg(p.no_filter + (yp >> l) * mcw + (xp >> l)) != 0;
  r.keep_q = p.no_filter && __ldg(p.no_filter + (y >> l) * mcw + (x >> l)) != 0;
  if (r.keep_p && r.keep_q) return r;
  r.qp = ((int)__ldg(p.qp_y + (y >> l) * mcw + (x >> l)) + (int)__ldg(p.qp_y + (yp >> l) * mcw + (xp >> l)) + 1) >> 1;
  r.beta = (int)kHdbBeta[hdb_clip(r.qp + f.beta_offset, 0, 51)] << (p.bit_depth_luma - 8);
  r.tc_offset = f.tc_offset;
  r.on = true;
  return r;
}

// One prediction unit's motion in registers (the list index is a run-time
// value, so the arrays are selected from rather than indexed).
struct HdbMv {
  int x[2], y[2], poc[2], flag;
};

__device__ __forceinline__ HdbMv hdb_mv(const b200enc_hevc_mvf_t* m) {
  // 20-byte entries are 4-byte aligned only: five word loads
  const int* w = reinterpret_cast<const int*>(m);
  const int m0 = __ldg(w), m1 = __ldg(w + 1);  // mv[0][x, y], mv[1][x, y]
  HdbMv r;
  r.x[0] = (int16_t)(m0 & 0xffff);
  r.y[0] = (int16_t)(m0 >> 16);
  r.x[1] = (int16_t)(m1 & 0xffff);
  r.y[1] = (int16_t)(m1 >> 16);
  r.poc[0] = __ldg(w + 2);
  r.poc[1] = __ldg(w + 3);
  r.flag = __ldg(w + 4) & 0xff;
  return r;
}

__device__ __forceinline__ bool hdb_differ(const HdbMv& a, int la, const HdbMv& b, int lb) {
  const int ax = la ? a.x[1] : a.x[0], ay = la ? a.y[1] : a.y[0];
  const int bx = lb ? b.x[1] : b.x[0], by = lb ? b.y[1] : b.y[0];
  return abs(ax - bx) >= 4 || abs(ay - by) >= 4;
}

// Boundary strength of one segment, clause 8.7.2.4
// (hevc_filter_template.c:207-259).
__device__ int hdb_strength(const b200enc_hevc_deblock_t& p, int xp, int yp, int xq, int yq, bool transform_edge) {
  if (!p.mvf) return 2;
  const int ip = (yp >> 2) * p.min_pu_width + (xp >> 2), iq = (yq >> 2) * p.min_pu_width + (xq >> 2);
  const HdbMv P = hdb_mv(p.mvf + ip), Q = hdb_mv(p.mvf + iq);
  if (!P.flag || !Q.flag) return 2;
  if (transform_edge && p.cbf && (__ldg(p.cbf + ip) || __ldg(p.cbf + iq))) return 1;
  const int np = P.flag == 3 ? 2 : 1, nq = Q.flag == 3 ? 2 : 1;
  if (np != nq) return 1;
  if (np == 1) {
    const int lp = (P.flag & 1) ? 0 : 1, lq = (Q.flag & 1) ? 0 : 1;
    if ((lp ? P.poc[1] : P.poc[0]) != (lq ? Q.poc[1] : Q.poc[0])) return 1;
    return hdb_differ(P, lp, Q, lq) ? 1 : 0;
  }
  const bool same = P.poc[0] == Q.poc[0] && P.poc[1] == Q.poc[1];
  const bool crossed = P.poc[0] == Q.poc[1] && P.poc[1] == Q.poc[0];
  if (!same && !crossed) return 1;
  if (P.poc[0] != P.poc[1]) {
    if (same) return (hdb_differ(P, 0, Q, 0) || hdb_differ(P, 1, Q, 1)) ? 1 : 0;
    return (hdb_differ(P, 0, Q, 1) || hdb_differ(P, 1, Q, 0)) ? 1 : 0;
  }
  const bool straight = !(hdb_differ(P, 0, Q, 0) || hdb_differ(P, 1, Q, 1));
  const bool swapped = !(hdb_differ(P, 0, Q, 1) || hdb_differ(P, 1, Q, 0));
  return (straight || swapped) ? 0 : 1;
}

// One 4-line luma segment in shared memory (clauses 8.7.2.5.3, 8.7.2.5.6,
// 8.7.2.5.7; hevc_filter_template.c:48-140): `q` at q0 of the first line,
// `fw` from p to q, `gl` from one line to the next.
template <typename T>
__device__ void hdb_luma(T* q, int fw, int gl, int beta, int tc, bool keep_p, bool keep_q, int maxv) {
  auto P = [&](int k, int i) { return (int)q[i * gl - (k + 1) * fw]; };
  auto Q = [&](int k, int i) { return (int)q[i * gl + k * fw]; };
  const int dp0 = abs(P(2, 0) - 2 * P(1, 0) + P(0, 0)), dp3 = abs(P(2, 3) - 2 * P(1, 3) + P(0, 3));
  const int dq0 = abs(Q(2, 0) - 2 * Q(1, 0) + Q(0, 0)), dq3 = abs(Q(2, 3) - 2 * Q(1, 3) + Q(0, 3));
  const int dpq0 = dp0 + dq0, dpq3 = dp3 + dq3;
  if (dpq0 + dpq3 >= beta) return;
  const int dp = dp0 + dp3, dq = dq0 + dq3;
  const int thr = (5 * tc + 1) >> 1;
  bool strong = true;
#pragma unroll
  for (int i = 0; i < 4; i += 3) {
    const int dpq = 2 * (i == 0 ? dpq0 : dpq3);
    strong = strong && dpq < (beta >> 2) && abs(P(3, i) - P(0, i)) + abs(Q(0, i) - Q(3, i)) < (beta >> 3) &&
             abs(P(0, i) - Q(0, i)) < thr;
  }
  if (strong) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int p0 = P(0, i), p1 = P(1, i), p2 = P(2, i), p3 = P(3, i);
      const int q0 = Q(0, i), q1 = Q(1, i), q2 = Q(2, i), q3 = Q(3, i);
      T* l = q + i * gl;
      if (!keep_p) {
        l[-fw] = (T)hdb_clip((p2 + 2 * p1 + 2 * p0 + 2 * q0 + q1 + 4) >> 3, p0 - 2 * tc, p0 + 2 * tc);
        l[-2 * fw] = (T)hdb_clip((p2 + p1 + p0 + q0 + 2) >> 2, p1 - 2 * tc, p1 + 2 * tc);
        l[-3 * fw] = (T)hdb_clip((2 * p3 + 3 * p2 + p1 + p0 + q0 + 4) >> 3, p2 - 2 * tc, p2 + 2 * tc);
      }
      if (!keep_q) {
        l[0] = (T)hdb_clip((p1 + 2 * p0 + 2 * q0 + 2 * q1 + q2 + 4) >> 3, q0 - 2 * tc, q0 + 2 * tc);
        l[fw] = (T)hdb_clip((p0 + q0 + q1 + q2 + 2) >> 2, q1 - 2 * tc, q1 + 2 * tc);
        l[2 * fw] = (T)hdb_clip((p0 + q0 + q1 + 3 * q2 + 2 * q3 + 4) >> 3, q2 - 2 * tc, q2 + 2 * tc);
      }
    }
    return;
  }
  const bool touch_p1 = dp < ((beta + (beta >> 1)) >> 3), touch_q1 = dq < ((beta + (beta >> 1)) >> 3);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int p0 = P(0, i), p1 = P(1, i), p2 = P(2, i);
    const int q0 = Q(0, i), q1 = Q(1, i), q2 = Q(2, i);
    int delta = (9 * (q0 - p0) - 3 * (q1 - p1) + 8) >> 4;
    if (abs(delta) >= tc * 10) continue;
    delta = hdb_clip(delta, -tc, tc);
    T* l = q + i * gl;
    if (!keep_p) l[-fw] = (T)hdb_clip(p0 + delta, 0, maxv);
    if (!keep_q) l[0] = (T)hdb_clip(q0 - delta, 0, maxv);
    if (touch_p1 && !keep_p) {
      const int d1 = hdb_clip((((p2 + p0 + 1) >> 1) - p1 + delta) >> 1, -(tc >> 1), tc >> 1);
      l[-2 * fw] = (T)hdb_clip(p1 + d1, 0, maxv);
    }
    if (touch_q1 && !keep_q) {
      const int d1 = hdb_clip((((q2 + q0 + 1) >> 1) - q1 - delta) >> 1, -(tc >> 1), tc >> 1);
      l[fw] = (T)hdb_clip(q1 + d1, 0, maxv);
    }
  }
}

// One 4-line chroma segment (clause 8.7.2.5.5; hevc_filter_template.c:149-162).
template <typename T>
__device__ void hdb_chroma(T* q, int fw, int gl, int tc, bool keep_p, bool keep_q, int maxv) {
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    T* l = q + i * gl;
    const int p1 = l[-2 * fw], p0 = l[-fw], q0 = l[0], q1 = l[fw];
    const int delta = hdb_clip((((q0 - p0) * 4) + p1 - q1 + 4) >> 3, -tc, tc);
    if (!keep_p) l[-fw] = (T)hdb_clip(p0 + delta, 0, maxv);
    if (!keep_q) l[0] = (T)hdb_clip(q0 - delta, 0, maxv);
  }
}

// tC of one chroma plane, hevc_filter_template.c:176-181 and :322-329.
__device__ __forceinline__ int hdb_tc_chroma(const b200enc_hevc_deblock_t& p, const HdbEdge& ed, int plane) {
  const int qpi = hdb_clip(ed.qp + (plane == 0 ? p.cb_qp_offset : p.cr_qp_offset), 0, 57);
  const int qpc = qpi < 30 ? qpi : (qpi > 43 ? qpi - 6 : (int)kHdbQpC[qpi - 30]);
  return (int)kHdbTc[hdb_clip(qpc + 2 + ed.tc_offset, 0, 53)] << (p.bit_depth_chroma - 8);
}

// Vertical edges: thread = (4-row segment, 8x8 cell column); chroma with the
// first segment of a cell on the 16-sample grid (hevc_filter_template.c
// :298-335).
template <typename T>
__global__ void __launch_bounds__(kHdbThreads) hevc_deblock_v_kernel(const b200enc_hevc_deblock_t p) {
  const int ncx = p.width >> 3, nseg = p.height >> 2;
  const int idx = blockIdx.x * kHdbThreads + threadIdx.x;
  if (idx >= ncx * nseg) return;
  const int seg = idx / ncx, cx = idx - seg * ncx;
  if (cx == 0) return;  // the picture's left border is no edge
  const int ex = cx << 3, sy = seg << 2;
  const int e = __ldg(p.edges + (size_t)(sy >> 3) * p.edges_stride + cx);
  if (!(e & 1)) return;
  const int ctb_w = (p.width + (1 << p.log2_ctb) - 1) >> p.log2_ctb;
  const HdbEdge ed = hdb_edge(p, ex, sy & ~7, true, ctb_w);
  if (!ed.on) return;
  const int bs = hdb_strength(p, ex - 1, sy, ex, sy, (e & 4) != 0);
  if (!bs) return;
  const int maxv = (int)(sizeof(T) == 1 ? 255 : 1023);
  const int tc = (int)kHdbTc[hdb_clip(ed.qp + 2 * (bs - 1) + ed.tc_offset, 0, 53)] << (p.bit_depth_luma - 8);
  T* Y = reinterpret_cast<T*>(p.plane[0]);
  hdb_luma<T>(Y + (size_t)sy * p.stride[0] + ex, 1, p.stride[0], ed.beta, tc, ed.keep_p, ed.keep_q, maxv);
  if (bs != 2 || (ex & 15) || (sy & 7)) return;
#pragma unroll
  for (int pl = 0; pl < 2; ++pl) {
    const int tcc = hdb_tc_chroma(p, ed, pl);
    if (!tcc) continue;
    T* C = reinterpret_cast<T*>(p.plane[1 + pl]);
    hdb_chroma<T>(C + (size_t)(sy >> 1) * p.stride[1 + pl] + (ex >> 1), 1, p.stride[1 + pl], tcc, ed.keep_p,
                  ed.keep_q, maxv);
  }
}

// Horizontal edges: thread = (8x8 cell row, 4-column segment); chroma with
// the first segment of a cell on the 16-row grid.
template <typename T>
__global__ void __launch_bounds__(kHdbThreads) hevc_deblock_h_kernel(const b200enc_hevc_deblock_t p) {
  const int nsx = p.width >> 2, ncy = p.height >> 3;
  const int idx = blockIdx.x * kHdbThreads + threadIdx.x;
  if (idx >= nsx * ncy) return;
  const int cy = idx / nsx, s = idx - cy * nsx;
  if (cy == 0) return;  // nor is its top border
  const int ey = cy << 3, sx = s << 2;
  const int e = __ldg(p.edges + (size_t)cy * p.edges_stride + (sx >> 3));
  if (!(e & 2)) return;
  const int ctb_w = (p.width + (1 << p.log2_ctb) - 1) >> p.log2_ctb;
  const HdbEdge ed = hdb_edge(p, sx & ~7, ey, false, ctb_w);
  if (!ed.on) return;
  const int bs = hdb_strength(p, sx, ey - 1, sx, ey, (e & 8) != 0);
  if (!bs) return;
  const int maxv = (int)(sizeof(T) == 1 ? 255 : 1023);
  const int tc = (int)kHdbTc[hdb_clip(ed.qp + 2 * (bs - 1) + ed.tc_offset, 0, 53)] << (p.bit_depth_luma - 8);
  T* Y = reinterpret_cast<T*>(p.plane[0]);
  hdb_luma<T>(Y + (size_t)ey * p.stride[0] + sx, p.stride[0], 1, ed.beta, tc, ed.keep_p, ed.keep_q, maxv);
  if (bs != 2 || (ey & 15) || (sx & 7)) return;
#pragma unroll
  for (int pl = 0; pl < 2; ++pl) {
    const int tcc = hdb_tc_chroma(p, ed, pl);
    if (!tcc) continue;
    T* C = reinterpret_cast<T*>(p.plane[1 + pl]);
    hdb_chroma<T>(C + (size_t)(ey >> 1) * p.stride[1 + pl] + (sx >> 1), p.stride[1 + pl], 1, tcc, ed.keep_p,
                  ed.keep_q, maxv);
  }
}

}  // namespace b200enc

using namespace b200enc;

extern "C" int b200enc_hevc_deblock(const b200enc_hevc_deblock_t* p, void* stream) {
  if (!p) return -1;
  const b200enc_hevc_deblock_t& q = *p;
  if (q.bit_depth_luma != 8 && q.bit_depth_luma != 10) return -1;
  if (q.bit_depth_chroma < 8 || q.bit_depth_chroma > q.bit_depth_luma) return -1;
  if (q.width <= 0 || q.height <= 0 || (q.width & 7) || (q.height & 7)) return -1;
  if (q.log2_ctb < 4 || q.log2_ctb > 6 || q.log2_min_cb < 3 || q.log2_min_cb > q.log2_ctb) return -1;
  if ((q.width & ((1 << q.log2_min_cb) - 1)) || (q.height & ((1 << q.log2_min_cb) - 1))) return -1;
  if (!q.plane[0] || !q.plane[1] || !q.plane[2] || !q.edges || !q.qp_y) return -1;
  if (q.stride[0] < q.width || q.stride[1] < q.width / 2 || q.stride[2] < q.width / 2) return -1;
  if (q.edges_stride < q.width / 8) return -1;
  if ((q.mvf || q.cbf) && q.min_pu_width < q.width / 4) return -1;
  if (((uintptr_t)q.mvf & 3) || ((uintptr_t)q.slice_filter & 3)) return -1;
  if (q.slice_filter && q.n_slice_filter <= 0) return -1;
  const int nv = (q.width >> 3) * (q.height >> 2), nh = (q.width >> 2) * (q.height >> 3);
  const cudaStream_t st = (cudaStream_t)stream;
  if (q.bit_depth_luma == 8) {
    hevc_deblock_v_kernel<uint8_t><<<(nv + kHdbThreads - 1) / kHdbThreads, kHdbThreads, 0, st>>>(q);
    hevc_deblock_h_kernel<uint8_t><<<(nh + kHdbThreads - 1) / kHdbThreads, kHdbThreads, 0, st>>>(q);
  } else {
    hevc_deblock_v_kernel<uint16_t><<<(nv + kHdbThreads - 1) / kHdbThreads, kHdbThreads, 0, st>>>(q);
    hevc_deblock_h_kernel<uint16_t><<<(nh + kHdbThreads - 1) / kHdbThreads, kHdbThreads, 0, st>>>(q);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
