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
// 4-line segment filters in place in global memory - no tiles, no halos -
// one lane per line, the segment's four lanes sharing the decision through
// warp shuffles. (A single launch over tiles with halos
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

__device__ __forceinline__ HdbEdge hdb_edge(const b200enc_hevc_deblock_t& p, int x, int y, bool vertical, int ctb_w) {
  // Every map read is issued before any of them is looked at (one round
  // trip instead of a chain); only the slice settings wait for the slice id.
  const int xp = vertical ? x - 1 : x, yp = vertical ? y : y - 1;
  const int cq = hdb_ctb(p, x, y, ctb_w), cp = hdb_ctb(p, xp, yp, ctb_w);
  const int l = p.log2_min_cb, mcw = p.width >> l;
  const int bq = (y >> l) * mcw + (x >> l), bp = (yp >> l) * mcw + (xp >> l);
  const int tq = p.tile_of_ctb ? __ldg(p.tile_of_ctb + cq) : 0, tp = p.tile_of_ctb ? __ldg(p.tile_of_ctb + cp) : 0;
  const int sq = p.slice_of_ctb ? __ldg(p.slice_of_ctb + cq) : 0, sp = p.slice_of_ctb ? __ldg(p.slice_of_ctb + cp) : 0;
  const bool nq = p.no_filter && __ldg(p.no_filter + bq) != 0, np = p.no_filter && __ldg(p.no_filter + bp) != 0;
  const int qq = __ldg(p.qp_y + bq), qp = __ldg(p.qp_y + bp);
  HdbEdge r;
  r.on = false;
  if (!p.loop_filter_across_tiles && tp != tq) return r;
  if (sq < 0 || !p.slice_filter || sq >= p.n_slice_filter) return r;
  const b200enc_hevc_slice_filter_t f = p.slice_filter[sq];
  if (f.disabled) return r;
  if (!f.across_slices && sp != sq) return r;
  r.keep_p = np;
  r.keep_q = nq;
  if (np && nq) return r;
  r.qp = (qq + qp + 1) >> 1;
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

// One line of a 4-line luma segment (clauses 8.7.2.5.3, 8.7.2.5.6,
// 8.7.2.5.7; hevc_filter_template.c:48-140). The four lanes 4k..4k+3 of a
// warp hold the segment's four lines; the decisions read lines 0 and 3 only,
// so those lanes' figures are shuffled to the other two. `q` points at this
// line's q0 and `fw` steps from p to q. Every lane of the warp calls it
// (the shuffles); `inside` says the segment lies in the picture (its
// samples may be read), `act` that it is filtered.
template <typename T>
__device__ __forceinline__ void hdb_luma_line(T* q, int fw, bool inside, bool act, int beta, int tc, bool keep_p,
                                              bool keep_q, int maxv) {
  int p3 = 0, p2 = 0, p1 = 0, p0 = 0, q0 = 0, q1 = 0, q2 = 0, q3 = 0;
  if (inside) {  // the samples of an edge position in the picture, whether or not it is filtered
    p3 = q[-4 * fw];
    p2 = q[-3 * fw];
    p1 = q[-2 * fw];
    p0 = q[-fw];
    q0 = q[0];
    q1 = q[fw];
    q2 = q[2 * fw];
    q3 = q[3 * fw];
  }
  const int dp = abs(p2 - 2 * p1 + p0), dq = abs(q2 - 2 * q1 + q0);
  const int flat = abs(p3 - p0) + abs(q0 - q3), step = abs(p0 - q0);
  const int l0 = (threadIdx.x & 31) & ~3, l3 = l0 + 3;
  const int dp0 = __shfl_sync(0xffffffffu, dp, l0), dp3 = __shfl_sync(0xffffffffu, dp, l3);
  const int dq0 = __shfl_sync(0xffffffffu, dq, l0), dq3 = __shfl_sync(0xffffffffu, dq, l3);
  const int fl0 = __shfl_sync(0xffffffffu, flat, l0), fl3 = __shfl_sync(0xffffffffu, flat, l3);
  const int st0 = __shfl_sync(0xffffffffu, step, l0), st3 = __shfl_sync(0xffffffffu, step, l3);
  if (!act) return;
  const int dpq0 = dp0 + dq0, dpq3 = dp3 + dq3;
  if (dpq0 + dpq3 >= beta) return;
  const int thr = (5 * tc + 1) >> 1;
  const bool strong = 2 * dpq0 < (beta >> 2) && fl0 < (beta >> 3) && st0 < thr && 2 * dpq3 < (beta >> 2) &&
                      fl3 < (beta >> 3) && st3 < thr;
  if (strong) {
    if (!keep_p) {
      q[-fw] = (T)hdb_clip((p2 + 2 * p1 + 2 * p0 + 2 * q0 + q1 + 4) >> 3, p0 - 2 * tc, p0 + 2 * tc);
      q[-2 * fw] = (T)hdb_clip((p2 + p1 + p0 + q0 + 2) >> 2, p1 - 2 * tc, p1 + 2 * tc);
      q[-3 * fw] = (T)hdb_clip((2 * p3 + 3 * p2 + p1 + p0 + q0 + 4) >> 3, p2 - 2 * tc, p2 + 2 * tc);
    }
    if (!keep_q) {
      q[0] = (T)hdb_clip((p1 + 2 * p0 + 2 * q0 + 2 * q1 + q2 + 4) >> 3, q0 - 2 * tc, q0 + 2 * tc);
      q[fw] = (T)hdb_clip((p0 + q0 + q1 + q2 + 2) >> 2, q1 - 2 * tc, q1 + 2 * tc);
      q[2 * fw] = (T)hdb_clip((p0 + q0 + q1 + 3 * q2 + 2 * q3 + 4) >> 3, q2 - 2 * tc, q2 + 2 * tc);
    }
    return;
  }
  int delta = (9 * (q0 - p0) - 3 * (q1 - p1) + 8) >> 4;
  if (abs(delta) >= tc * 10) return;
  delta = hdb_clip(delta, -tc, tc);
  const int side = (beta + (beta >> 1)) >> 3;
  if (!keep_p) {
    q[-fw] = (T)hdb_clip(p0 + delta, 0, maxv);
    if (dp0 + dp3 < side)
      q[-2 * fw] = (T)hdb_clip(p1 + hdb_clip((((p2 + p0 + 1) >> 1) - p1 + delta) >> 1, -(tc >> 1), tc >> 1), 0, maxv);
  }
  if (!keep_q) {
    q[0] = (T)hdb_clip(q0 - delta, 0, maxv);
    if (dq0 + dq3 < side)
      q[fw] = (T)hdb_clip(q1 + hdb_clip((((q2 + q0 + 1) >> 1) - q1 - delta) >> 1, -(tc >> 1), tc >> 1), 0, maxv);
  }
}

// One line of a chroma segment (clause 8.7.2.5.5; hevc_filter_template.c
// :149-162): no decision, so nothing crosses lanes.
template <typename T>
__device__ __forceinline__ void hdb_chroma_line(T* q, int fw, int tc, bool keep_p, bool keep_q, int maxv) {
  const int p1 = q[-2 * fw], p0 = q[-fw], q0 = q[0], q1 = q[fw];
  const int delta = hdb_clip((((q0 - p0) * 4) + p1 - q1 + 4) >> 3, -tc, tc);
  if (!keep_p) q[-fw] = (T)hdb_clip(p0 + delta, 0, maxv);
  if (!keep_q) q[0] = (T)hdb_clip(q0 - delta, 0, maxv);
}

// tC of one chroma plane, hevc_filter_template.c:176-181 and :322-329.
__device__ __forceinline__ int hdb_tc_chroma(const b200enc_hevc_deblock_t& p, const HdbEdge& ed, int plane) {
  const int qpi = hdb_clip(ed.qp + (plane == 0 ? p.cb_qp_offset : p.cr_qp_offset), 0, 57);
  const int qpc = qpi < 30 ? qpi : (qpi > 43 ? qpi - 6 : (int)kHdbQpC[qpi - 30]);
  return (int)kHdbTc[hdb_clip(qpc + 2 + ed.tc_offset, 0, 53)] << (p.bit_depth_chroma - 8);
}

// Vertical edges: four lanes per (4-row segment, 8x8 cell column), one per
// row; chroma with the first segment of a cell on the 16-sample grid, one
// chroma row per lane (hevc_filter_template.c:298-335).
template <typename T>
__global__ void __launch_bounds__(kHdbThreads) hevc_deblock_v_kernel(const b200enc_hevc_deblock_t p) {
  const int ncx = p.width >> 3, nseg = p.height >> 2;
  const int g = blockIdx.x * kHdbThreads + threadIdx.x, sid = g >> 2, line = g & 3;
  int ex = 0, sy = 0, bs = 0;
  bool inside = false;
  HdbEdge ed;
  ed.on = false;
  if (sid < ncx * nseg) {
    const int seg = sid / ncx, cx = sid - seg * ncx;
    ex = cx << 3;
    sy = seg << 2;
    inside = cx > 0;
    const int e = inside ? __ldg(p.edges + (size_t)(sy >> 3) * p.edges_stride + cx) : 0;
    if (inside) {
      const int ctb_w = (p.width + (1 << p.log2_ctb) - 1) >> p.log2_ctb;
      ed = hdb_edge(p, ex, sy & ~7, true, ctb_w);
      const int b = hdb_strength(p, ex - 1, sy, ex, sy, (e & 4) != 0);
      bs = ((e & 1) && ed.on) ? b : 0;
    }
  }
  const int maxv = (int)(sizeof(T) == 1 ? 255 : 1023);
  const int tc = bs ? (int)kHdbTc[hdb_clip(ed.qp + 2 * (bs - 1) + ed.tc_offset, 0, 53)] << (p.bit_depth_luma - 8) : 0;
  T* Y = reinterpret_cast<T*>(p.plane[0]);
  hdb_luma_line<T>(Y + (size_t)(sy + line) * p.stride[0] + ex, 1, inside, bs != 0, ed.beta, tc, ed.keep_p, ed.keep_q,
                   maxv);
  if (bs != 2 || (ex & 15) || (sy & 7)) return;
#pragma unroll
  for (int pl = 0; pl < 2; ++pl) {
    const int tcc = hdb_tc_chroma(p, ed, pl);
    if (!tcc) continue;
    T* C = reinterpret_cast<T*>(p.plane[1 + pl]);
    hdb_chroma_line<T>(C + (size_t)((sy >> 1) + line) * p.stride[1 + pl] + (ex >> 1), 1, tcc, ed.keep_p, ed.keep_q,
                       maxv);
  }
}

// Horizontal edges: four lanes per (8x8 cell row, 4-column segment), one
// per column; chroma with the first segment of a cell on the 16-row grid.
template <typename T>
__global__ void __launch_bounds__(kHdbThreads) hevc_deblock_h_kernel(const b200enc_hevc_deblock_t p) {
  const int nsx = p.width >> 2, ncy = p.height >> 3;
  const int g = blockIdx.x * kHdbThreads + threadIdx.x, sid = g >> 2, line = g & 3;
  int ey = 0, sx = 0, bs = 0;
  bool inside = false;
  HdbEdge ed;
  ed.on = false;
  if (sid < nsx * ncy) {
    const int cy = sid / nsx, s = sid - cy * nsx;
    ey = cy << 3;
    sx = s << 2;
    inside = cy > 0;
    const int e = inside ? __ldg(p.edges + (size_t)cy * p.edges_stride + (sx >> 3)) : 0;
    if (inside) {
      const int ctb_w = (p.width + (1 << p.log2_ctb) - 1) >> p.log2_ctb;
      ed = hdb_edge(p, sx & ~7, ey, false, ctb_w);
      const int b = hdb_strength(p, sx, ey - 1, sx, ey, (e & 8) != 0);
      bs = ((e & 2) && ed.on) ? b : 0;
    }
  }
  const int maxv = (int)(sizeof(T) == 1 ? 255 : 1023);
  const int tc = bs ? (int)kHdbTc[hdb_clip(ed.qp + 2 * (bs - 1) + ed.tc_offset, 0, 53)] << (p.bit_depth_luma - 8) : 0;
  T* Y = reinterpret_cast<T*>(p.plane[0]);
  hdb_luma_line<T>(Y + (size_t)ey * p.stride[0] + sx + line, p.stride[0], inside, bs != 0, ed.beta, tc, ed.keep_p,
                   ed.keep_q, maxv);
  if (bs != 2 || (ey & 15) || (sx & 7)) return;
#pragma unroll
  for (int pl = 0; pl < 2; ++pl) {
    const int tcc = hdb_tc_chroma(p, ed, pl);
    if (!tcc) continue;
    T* C = reinterpret_cast<T*>(p.plane[1 + pl]);
    hdb_chroma_line<T>(C + (size_t)(ey >> 1) * p.stride[1 + pl] + (sx >> 1) + line, p.stride[1 + pl], tcc, ed.keep_p,
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
  const int nv = 4 * (q.width >> 3) * (q.height >> 2), nh = 4 * (q.width >> 2) * (q.height >> 3);  // lanes
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
