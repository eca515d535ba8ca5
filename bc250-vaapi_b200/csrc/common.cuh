// common.cuh - shared device helpers for the b200enc kernels (sm_100a).
//
// Integer arithmetic of the H.264 compute-encoder stages, written for warp
// execution: a 4x4 transform block is owned by a quad of lanes (one lane per
// row), quads exchange rows/columns through shared memory, and every table
// lives in __constant__ memory. The math is the reference's
// (A1 = approach1-compute-encoder):
//   forward 4x4     A1/shaders/dct_transform.comp:34-73
//   AC quant        A1/shaders/quantize.comp:151-225
//   dequant/inverse A1/shaders/reconstruct.comp:124-177
//   DC paths        A1/src/encoder_h264.c:653-797, reconstruct.comp:179-299
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace b200enc {

struct MV {
  int32_t mvx, mvy;  // quarter-pel
  uint32_t sad, pad;
};
static_assert(sizeof(MV) == 16, "MV must match the reference's 16-byte gpu_mv_t");

// Geometry of one frame. Source reads clamp to (W, H); reference/recon reads
// clamp to (RW, RH) and recon writes stop there. RW/RH = W/H is the
// reference shaders' behaviour; RW/RH = coded size is a conforming decoder's.
struct Geo {
  int W, H, RW, RH, mbw, mbh;
};

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
__device__ __forceinline__ int clip1(int v) { return clampi(v, 0, 255); }

__device__ __forceinline__ int chroma_qp(int qpy) {
  // A1/shaders/quantize.comp:182-187 (Table 8-15, offset 0)
  if (qpy < 30) return qpy;
  const int i = qpy - 30;
  const int t = i < 22 ? i : 21;
  switch (t) {
    case 0: return 29; case 1: return 30; case 2: return 31; case 3: return 32; case 4: return 32;
    case 5: return 33; case 6: return 34; case 7: return 34; case 8: return 35; case 9: return 35;
    case 10: return 36; case 11: return 36; case 12: return 37; case 13: return 37; case 14: return 37;
    case 15: return 38; case 16: return 38; case 17: return 38; default: return 39;
  }
}

// Position class of raster index p in a 4x4 block: 0 both even, 1 both odd,
// 2 mixed (A1/shaders/quantize.comp:160-168).
__device__ __forceinline__ int pos_type(int p) {
  const int r = (p >> 2) & 1, c = p & 1;
  return (r & c) ? 1 : ((r | c) ? 2 : 0);
}

// MF (A1/shaders/quantize.comp:151-158), V (A1/shaders/reconstruct.comp:
// 124-131) and the DC level scale (reconstruct.comp:92), indexed
// [qp%6][position class].
static __constant__ int kMF[6][3] = {{13107, 5243, 8066}, {11916, 4660, 7490}, {10082, 4194, 6554},
                                     {9362, 3647, 5825},  {8192, 3355, 5243},  {7282, 2893, 4559}};
static __constant__ int kV[6][3] = {{10, 16, 13}, {11, 18, 14}, {13, 20, 16},
                                    {14, 23, 18}, {16, 25, 20}, {18, 29, 23}};
static __constant__ int kDcLs[6] = {160, 176, 208, 224, 256, 288};

__device__ __forceinline__ int mf_of(int rem, int pt) { return kMF[rem][pt]; }
__device__ __forceinline__ int v_of(int rem, int pt) { return kV[rem][pt]; }
__device__ __forceinline__ int dc_ls(int rem) { return kDcLs[rem]; }

// Quantizer constants for one QP, computed once per thread: the MF and V
// entries of the QP's row are held in registers, so a coefficient's
// constant is a selection on its position class rather than a
// constant-memory load whose address differs from lane to lane.
struct QP {
  int per, rem, f_shift, f;  // f = rounding offset of the AC quantizer
  int mf0, mf1, mf2, v0, v1, v2;
};
__device__ __forceinline__ QP make_qp(int qp, bool intra) {
  QP q;
  q.per = qp / 6;
  q.rem = qp - 6 * q.per;
  q.f_shift = 15 + q.per;
  q.f = (1 << q.f_shift) / (intra ? 3 : 6);
  q.mf0 = mf_of(q.rem, 0);
  q.mf1 = mf_of(q.rem, 1);
  q.mf2 = mf_of(q.rem, 2);
  q.v0 = v_of(q.rem, 0);
  q.v1 = v_of(q.rem, 1);
  q.v2 = v_of(q.rem, 2);
  return q;
}
__device__ __forceinline__ int qp_mf(const QP& q, int pt) { return pt == 0 ? q.mf0 : (pt == 1 ? q.mf1 : q.mf2); }
__device__ __forceinline__ int qp_v(const QP& q, int pt) { return pt == 0 ? q.v0 : (pt == 1 ? q.v1 : q.v2); }

__device__ __forceinline__ int quant_ac(int c, int pos, const QP& q) {
  const int a = c < 0 ? -c : c;
  const int l = (a * qp_mf(q, pos_type(pos)) + q.f) >> q.f_shift;
  return c < 0 ? -l : l;
}
__device__ __forceinline__ int dequant_ac(int level, int pos, const QP& q) {
  const int scale = 16 * qp_v(q, pos_type(pos));
  if (q.per >= 4) return (level * scale) << (q.per - 4);
  return (level * scale + (1 << (3 - q.per))) >> (4 - q.per);
}

__device__ __forceinline__ int quantize_dc(int v, const QP& q) {
  // A1/src/encoder_h264.c:653-709 (luma and chroma bodies are identical)
  const int ls = dc_ls(q.rem);
  const int a = v < 0 ? -v : v;
  int num, den;
  if (q.per >= 5) { num = a; den = ls << (q.per - 5); }
  else { num = a << (5 - q.per); den = ls; }
  const int l = (num + den / 2) / den;
  return v < 0 ? -l : l;
}
__device__ __forceinline__ int dequant_dc_luma(int f, const QP& q) {
  const int ls = dc_ls(q.rem);
  if (q.per >= 6) return (f * ls) << (q.per - 6);
  return (f * ls + (1 << (5 - q.per))) >> (6 - q.per);
}
__device__ __forceinline__ int dequant_dc_chroma(int f, const QP& q) {
  const int ls = dc_ls(q.rem);
  if (q.per >= 5) return (f * ls) << (q.per - 5);
  return (f * ls) >> (5 - q.per);
}

// 1-D forward butterfly (dct_transform.comp:45-53).
__device__ __forceinline__ void fwd4(int& x0, int& x1, int& x2, int& x3) {
  const int a0 = x0 + x3, a1 = x1 + x2, a2 = x1 - x2, a3 = x0 - x3;
  x0 = a0 + a1;
  x1 = (a3 << 1) + a2;
  x2 = a0 - a1;
  x3 = a3 - (a2 << 1);
}
// 1-D inverse butterfly (reconstruct.comp:168-169).
__device__ __forceinline__ void inv4(int& x0, int& x1, int& x2, int& x3) {
  const int z0 = x0 + x2, z1 = x0 - x2, z2 = (x1 >> 1) - x3, z3 = x1 + (x3 >> 1);
  x0 = z0 + z3;
  x1 = z1 + z2;
  x2 = z1 - z2;
  x3 = z0 - z3;
}

// Slice index of macroblock mb (A1/shaders/residual_predict.comp:163-171).
__device__ __forceinline__ uint32_t slice_of(uint32_t mb, uint32_t total, uint32_t ns) {
  if (ns <= 1u || total == 0u) return 0u;
  uint32_t s = (mb * ns) / total;
  if (s >= ns) s = ns - 1u;
  while (s + 1u < ns && ((s + 1u) * total) / ns <= mb) s++;
  while (s > 0u && (s * total) / ns > mb) s--;
  return s;
}

// ---------------------------------------------------------------------------
// Quad (4-lane) transform block pipeline.
//
// Lane `r` of a quad (lanes 4q .. 4q+3 of a warp) owns row r of one 4x4
// block. Rows become columns by a register transpose over the quad (two
// shuffle stages), so no shared memory and no barrier is involved; every lane
// of the warp must call these together.
// ---------------------------------------------------------------------------

// 4x4 transpose across the quad: on entry lane r holds row r (x[i] = M[r][i]),
// on return column r (x[i] = M[i][r]). Stage 1 swaps the off-diagonal 2x2
// blocks between lanes r and r^2, stage 2 the off-diagonal elements of each
// 2x2 block between lanes r and r^1.
__device__ __forceinline__ void quad_transpose(int x[4], int r) {
  const unsigned full = 0xffffffffu;
  const bool hi = (r & 2) != 0;
  int s0 = hi ? x[0] : x[2], s1 = hi ? x[1] : x[3];
  s0 = __shfl_xor_sync(full, s0, 2);
  s1 = __shfl_xor_sync(full, s1, 2);
  if (hi) { x[0] = s0; x[1] = s1; } else { x[2] = s0; x[3] = s1; }
  const bool odd = (r & 1) != 0;
  int t0 = odd ? x[0] : x[1], t1 = odd ? x[2] : x[3];
  t0 = __shfl_xor_sync(full, t0, 1);
  t1 = __shfl_xor_sync(full, t1, 1);
  if (odd) { x[0] = t0; x[2] = t1; } else { x[1] = t0; x[3] = t1; }
}

// Forward 4x4 of the residual row x[0..3] held by lane r. Returns column r
// of the coefficients: c[i] = coef[i][r]. Rows then columns, like
// dct_transform.comp; the forward transform is exact so order is moot.
__device__ __forceinline__ void quad_forward(int x[4], int r) {
  fwd4(x[0], x[1], x[2], x[3]);
  quad_transpose(x, r);
  fwd4(x[0], x[1], x[2], x[3]);
}

// Inverse 4x4 of the dequantized row d[0..3] (lane r holds row r, +32 already
// on d[0][0]); returns column r of the residual: out[i] = res[i][r]
// (reconstruct.comp:162-177: rows first, then columns, >>6).
__device__ __forceinline__ void quad_inverse(int d[4], int r) {
  inv4(d[0], d[1], d[2], d[3]);
  quad_transpose(d, r);
  inv4(d[0], d[1], d[2], d[3]);
  d[0] >>= 6;
  d[1] >>= 6;
  d[2] >>= 6;
  d[3] >>= 6;
}

// Error codes written by the wavefront kernels' bounded waits.
enum : uint32_t {
  kErrNone = 0,
  kErrWaitTimeout = 1,
};

__device__ __forceinline__ void store_release(uint32_t* flag, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(flag), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t load_acquire(const uint32_t* flag) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(flag) : "memory");
  return v;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Scratch layout of the wavefront kernels (one region per launch):
//   [0] ticket counter, [1] error code, [2] error detail, [3] reserved,
//   [4 .. 4+mbh) per-row progress (luma rows for deblocking, the only rows
//   of the intra wavefront), [4+mbh .. 4+2*mbh) chroma-row progress of the
//   deblocking wavefront.
struct Scratch {
  uint32_t* base;
  __device__ uint32_t* ticket() const { return base; }
  __device__ uint32_t* err() const { return base + 1; }
  __device__ uint32_t* err_detail() const { return base + 2; }
  __device__ uint32_t* progress(int row) const { return base + 4 + row; }
};
inline size_t scratch_words(int mbh) { return 4 + 2 * (size_t)mbh; }

// ---------------------------------------------------------------------------
// Batched steps (batch.cu): one frame of each of many streams, of uneven
// sizes, through one launch per stage. Each stage walks the items of one
// set of streams laid end to end (the P streams' macroblocks, the I
// streams' macroblock rows, every stream's deblocking tiles); an item
// finds its stream by binary search over the set's prefix sums.
// ---------------------------------------------------------------------------
struct BatchStream {
  Geo g;
  int qp, is_intra, num_slices, intra_flags;
  int lambda, zero_thresh, has_hist;
  const uint8_t *cur_y, *cur_uv;
  int cur_pitch;
  const uint8_t *ref_y, *ref_uv;  // the previous reconstruction (P frames)
  uint8_t *rec_y, *rec_uv;        // this frame's reconstruction
  int rec_pitch;                  // of both reconstructions
  int16_t* levels;
  int32_t* dc;
  uint32_t *nz, *pred_mode;
  MV* mv;             // this frame's field
  const MV* mv_prev;  // the previous P frame's field (the learned form's history)
  uint32_t *scr_intra, *scr_db;  // wavefront scratch (scratch_words(mbh) words each)
  uint8_t *db_y, *db_uv;          // the deblocked reconstruction (tile deblocking; not rec_y/rec_uv)
};

struct BatchSet {
  const BatchStream* st;  // every stream of the batch
  const int* idx;         // [n] the set's streams
  const int* prefix;      // [n + 1] item offsets
  int n;
  __device__ __forceinline__ int total() const { return n > 0 ? prefix[n] : 0; }
  // position k in the set of the stream holding `item` (0 <= item < total())
  __device__ __forceinline__ int find(int item) const {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (prefix[mid] <= item) lo = mid;
      else hi = mid - 1;
    }
    return lo;
  }
  __device__ __forceinline__ const BatchStream& stream(int k) const { return st[idx[k]]; }
};

struct BatchTab {
  BatchSet p_mbs;   // macroblocks of the streams coding a P frame (the compact P index); each
                    // stream's range is padded to a multiple of 16 items, the padding items
                    // (local index >= the stream's macroblock count) do no work
  BatchSet i_rows;  // macroblock rows of the streams coding an I frame
  BatchSet groups;  // deblocking tiles of every stream
  MV* mvc;          // motion vectors by compact P index
  uint32_t* ticket; // [0] intra rows, [1] deblocking groups
  int db_rows;      // macroblock rows per deblocking group (tile deblocking: tile height)
  int db_cols;      // tile deblocking: tile width in macroblocks
};

}  // namespace b200enc
