// cavlc.cu - CAVLC slice data (H.264 clause 7.3.4 / 9.2) on the GPU.
//
// The reference's host encoder entropy-codes a picture's slices after the
// GPU stages (A1/src/encoder_h264.c:3128-3290 for CAVLC): I slices code every
// macroblock as I16x16 (encode_mb_i16x16, :1120), P slices skip the
// macroblocks that qualify (:3236-3255) and code the others as mb_skip_run +
// P_L0_16x16 (encode_mb_p16x16, :1248). Nothing in that loop is sequential
// except two things: each block's nC is the neighbours' TotalCoeff, and each
// coded macroblock is preceded by the run of skipped macroblocks before it.
// Both are known up front: TotalCoeff is the number of nonzero levels the
// block codes, and the skip decision depends only on the macroblock's own
// levels and the vectors around it. So the slice data is built in four
// launches over the picture's staged outputs (levels, DC, nz masks, modes,
// vectors), all in device memory:
//   1. cavlc_info_kernel: per macroblock, the skip decision, coded block
//      pattern and every coded block's TotalCoeff;
//   2. cavlc_mb_kernel: per macroblock, its header and residual bits (one
//      warp per macroblock, a lane per block, into a private region of the
//      scratch);
//   3. cavlc_slice_kernel: per slice (one CTA), the skip runs and every
//      coded macroblock's bit offset (two block-wide scans), the slice's
//      length; it zeroes the slice's output words;
//   4. cavlc_pack_kernel: each coded macroblock ORs ue(skip run) and its
//      bits into the slice at its offset; each slice's first thread writes
//      the caller's slice header bits, the trailing skip run and
//      rbsp_trailing_bits;
// then cavlc_bytes_kernel turns the MSB-first words into stream bytes. The
// output is each slice's RBSP (header + slice data + trailing bits), ready
// for emulation prevention and a NAL header, bit for bit the reference's.
#include <algorithm>

#include "b200enc_internal.h"
#include "cavlc_core.h"
#include "common.cuh"
#include "t8x8.cuh"

namespace b200enc {

using namespace b200cavlc;

constexpr int kCavlcMbWords = 640;  // 2560 bytes of bits per macroblock at most (the reference's CAVLC allowance)
constexpr int kCavlcMaxSlices = 16;
constexpr int kCavlcScanThreads = 1024;

// spec luma block index (8x8 quadrants, then 4x4 within) -> block column / row
__constant__ int8_t kBlkX4[16] = {0, 1, 0, 1, 2, 3, 2, 3, 0, 1, 0, 1, 2, 3, 2, 3};
__constant__ int8_t kBlkY4[16] = {0, 0, 1, 1, 0, 0, 1, 1, 2, 2, 3, 3, 2, 2, 3, 3};
__device__ __forceinline__ int spec_blk(int y4, int x4) { return ((y4 >> 1) << 3) | ((x4 >> 1) << 2) | ((y4 & 1) << 1) | (x4 & 1); }

// Per-slice header bits (MSB first) of a launch, passed by value.
struct CavlcHdr {
  uint32_t bits[kCavlcMaxSlices][4];
  int len[kCavlcMaxSlices];
};

struct CavlcArgs {
  int mbw, mbh, qp, is_intra, ns, quality;
  int t8;  // P macroblocks code their luma with the 8x8 transform (levels in 8x8 raster order)
  const uint8_t* t8f;  // NULL, or per macroblock: 0 = this one codes 4x4 blocks after all
  const int16_t* levels;
  const int32_t* dc;
  const uint32_t* nz;
  const uint32_t* pred_mode;
  const MV* mv;
  // scratch
  uint32_t* info;    // [mbs] bit 0 skipped, bits 1..4 luma cbp quadrants (P) / bit 1 any luma AC (I), bits 8..9 cbp_chroma
  uint8_t* tcs;      // [mbs][24] TotalCoeff of the coded blocks (luma in spec order, Cb, Cr; 0 when not coded)
  uint32_t* nbits;   // [mbs] bits of the macroblock (header + residual, no skip run)
  uint32_t* words;   // [mbs][kCavlcMbWords]
  uint32_t* off;     // [mbs] bit offset of a coded macroblock's skip run in its slice
  uint32_t* run;     // [mbs] skip run before a coded macroblock (0xffffffff: none, I slices)
  uint32_t* sl;      // [kCavlcMaxSlices * 4] per slice: total bits, trailing run, overflow, bytes
  uint32_t* err;     // [1] nonzero: a macroblock's bits outgrew its region
  // output
  uint8_t* out;
  uint32_t slice_cap;  // bytes per slice region (multiple of 4)
  uint32_t* out_bytes; // [ns]
  uint8_t* out_copy;   // where the stream bytes go (out itself, or e.g. mapped page-locked host memory)
};

__device__ __forceinline__ uint32_t slice_start(uint32_t s, uint32_t total, uint32_t ns) {
  return (uint32_t)(((uint64_t)s * total) / ns);
}

// Neighbour macroblock (dx, dy) of (mbx, mby) inside the picture and the
// slice that starts at `start` (encoder_h264.c:948-958).
__device__ __forceinline__ bool nb_ok(int mbx, int mby, int dx, int dy, int mbw, uint32_t start, int* nb) {
  const int x = mbx + dx, y = mby + dy;
  if (x < 0 || y < 0 || x >= mbw) return false;
  *nb = y * mbw + x;
  return (uint32_t)*nb >= start;
}

__device__ __forceinline__ int median3(int a, int b, int c) {
  return a + b + c - min(a, min(b, c)) - max(a, max(b, c));
}

// 8.4.1.3 median predictor as the reference derives it (encoder_h264.c:974-1000).
__device__ void mv_pred(const MV* mv, int mbx, int mby, int mbw, uint32_t start, int* px, int* py) {
  int na, nbb, nc;
  const bool a = nb_ok(mbx, mby, -1, 0, mbw, start, &na);
  const bool b = nb_ok(mbx, mby, 0, -1, mbw, start, &nbb);
  bool c = nb_ok(mbx, mby, 1, -1, mbw, start, &nc);
  if (!c) c = nb_ok(mbx, mby, -1, -1, mbw, start, &nc);
  if (!b && !c && a) {
    *px = mv[na].mvx;
    *py = mv[na].mvy;
    return;
  }
  const int ax = a ? mv[na].mvx : 0, ay = a ? mv[na].mvy : 0;
  const int bx = b ? mv[nbb].mvx : 0, by = b ? mv[nbb].mvy : 0;
  const int cx = c ? mv[nc].mvx : 0, cy = c ? mv[nc].mvy : 0;
  *px = median3(ax, bx, cx);
  *py = median3(ay, by, cy);
}

// 8.4.1.1 P_Skip predictor (encoder_h264.c:1036-1051): zero when the left or
// upper neighbour is missing or has a zero vector.
__device__ void skip_pred(const MV* mv, int mbx, int mby, int mbw, uint32_t start, int* px, int* py) {
  int na, nbb;
  const bool a = nb_ok(mbx, mby, -1, 0, mbw, start, &na);
  const bool b = nb_ok(mbx, mby, 0, -1, mbw, start, &nbb);
  if (!a || !b || (mv[na].mvx == 0 && mv[na].mvy == 0) || (mv[nbb].mvx == 0 && mv[nbb].mvy == 0)) {
    *px = 0;
    *py = 0;
    return;
  }
  mv_pred(mv, mbx, mby, mbw, start, px, py);
}

// Chroma DC of one plane: the 2x2 Hadamard of the four raw DC terms
// (encoder_h264.c:791-797).
__device__ __forceinline__ void chroma_dc(const int32_t* d, int out[4]) {
  out[0] = d[0] + d[1] + d[2] + d[3];
  out[1] = d[0] - d[1] + d[2] - d[3];
  out[2] = d[0] + d[1] - d[2] - d[3];
  out[3] = d[0] - d[1] - d[2] + d[3];
}

__device__ __forceinline__ bool any_nz(const uint32_t* nzm, int b0, int b1, uint32_t mask) {
  uint32_t a = 0;
  for (int b = b0; b < b1; ++b) a |= nzm[b];
  return (a & mask) != 0;
}

// ---- 1. per macroblock: skip, coded block pattern, TotalCoeff ------------------
__global__ void __launch_bounds__(128) cavlc_info_kernel(CavlcArgs a) {
  const int mb = blockIdx.x * blockDim.x + threadIdx.x;
  const int mbs = a.mbw * a.mbh;
  if (mb >= mbs) return;
  const int mbx = mb % a.mbw, mby = mb / a.mbw;
  const uint32_t* nzm = a.nz + (size_t)mb * 24;
  const int32_t* dcm = a.dc + (size_t)mb * 24;
  uint8_t* tc = a.tcs + (size_t)mb * 24;
  const QP qc = make_qp(chroma_qp(a.qp), a.is_intra != 0);
  int cb[4], cr[4];
  chroma_dc(dcm + 16, cb);
  chroma_dc(dcm + 20, cr);
  bool cdc_raw_nz = false, cdc_nz = false;
  for (int i = 0; i < 4; ++i) {
    cdc_raw_nz |= (cb[i] != 0) | (cr[i] != 0);
    cdc_nz |= (quantize_dc(cb[i], qc) != 0) | (quantize_dc(cr[i], qc) != 0);
  }
  const bool cac_nz = any_nz(nzm, 16, 24, 0xfffeu);
  const int cbp_c = cac_nz ? 2 : (cdc_nz ? 1 : 0);
  uint32_t info = (uint32_t)cbp_c << 8;
  if (a.is_intra) {
    const bool lac = any_nz(nzm, 0, 16, 0xfffeu);
    info |= lac ? 2u : 0u;
    for (int b = 0; b < 16; ++b)
      tc[b] = lac ? (uint8_t)__popc(nzm[kBlkY4[b] * 4 + kBlkX4[b]] & 0xfffeu) : 0;
  } else {
    // P_Skip (encoder_h264.c:3236-3255): no luma level, a zero chroma DC
    // Hadamard and no chroma AC level, and the vector on the skip predictor
    const uint32_t start = slice_start(slice_of(mb, mbs, a.ns), mbs, a.ns);
    const bool zl = !any_nz(nzm, 0, 16, 0xffffu);
    bool zc = !cdc_raw_nz && !cac_nz;
    if (a.quality >= 5 && zl && !zc && abs(a.dc[mb * 2 + 0]) <= 1 && abs(a.dc[mb * 2 + 1]) <= 1) zc = true;
    int px, py;
    skip_pred(a.mv, mbx, mby, a.mbw, start, &px, &py);
    const bool skip = zl && zc && a.mv[mb].mvx == px && a.mv[mb].mvy == py;
    if (skip) {
      info = 1u;
      for (int b = 0; b < 24; ++b) tc[b] = 0;
    } else {
      for (int q = 0; q < 4; ++q) {
        uint32_t m = 0;
        for (int s = 0; s < 4; ++s) m |= nzm[kBlkY4[4 * q + s] * 4 + kBlkX4[4 * q + s]];
        if (m & 0xffffu) info |= 2u << q;
      }
      for (int b = 0; b < 16; ++b)
        tc[b] = (info >> (1 + (b >> 2)) & 1u) ? (uint8_t)__popc(nzm[kBlkY4[b] * 4 + kBlkX4[b]] & 0xffffu) : 0;
    }
  }
  if (!(info & 1u))
    for (int k = 0; k < 8; ++k) tc[16 + k] = cbp_c == 2 ? (uint8_t)__popc(nzm[16 + k] & 0xfffeu) : 0;
  a.info[mb] = info;
}

// nC of luma block b (spec order) from the TotalCoeff of its left and upper
// neighbours (encoder_h264.c:800-821).
__device__ int luma_nc(const uint8_t* tcs, int mb, int mbx, int mby, int mbw, uint32_t start, int b) {
  const int x4 = kBlkX4[b], y4 = kBlkY4[b];
  int na = -1, nb = -1, n;
  if (x4 > 0) na = tcs[mb * 24 + spec_blk(y4, x4 - 1)];
  else if (nb_ok(mbx, mby, -1, 0, mbw, start, &n)) na = tcs[n * 24 + spec_blk(y4, 3)];
  if (y4 > 0) nb = tcs[mb * 24 + spec_blk(y4 - 1, x4)];
  else if (nb_ok(mbx, mby, 0, -1, mbw, start, &n)) nb = tcs[n * 24 + spec_blk(3, x4)];
  if (na >= 0 && nb >= 0) return (na + nb + 1) >> 1;
  return na >= 0 ? na : (nb >= 0 ? nb : 0);
}

// nC of chroma AC block k (raster in its 2x2 grid) of the plane whose
// TotalCoeffs start at entry o (encoder_h264.c:823-841).
__device__ int chroma_nc(const uint8_t* tcs, int mb, int mbx, int mby, int mbw, uint32_t start, int o, int k) {
  const int x2 = k & 1, y2 = k >> 1;
  int na = -1, nb = -1, n;
  if (x2 > 0) na = tcs[mb * 24 + o + y2 * 2];
  else if (nb_ok(mbx, mby, -1, 0, mbw, start, &n)) na = tcs[n * 24 + o + y2 * 2 + 1];
  if (y2 > 0) nb = tcs[mb * 24 + o + x2];
  else if (nb_ok(mbx, mby, 0, -1, mbw, start, &n)) nb = tcs[n * 24 + o + 2 + x2];
  if (na >= 0 && nb >= 0) return (na + nb + 1) >> 1;
  return na >= 0 ? na : (nb >= 0 ? nb : 0);
}

// Prediction modes the decoder can form at the slice and picture edges
// (h264_sanitize_i16_mode / _chroma_mode, encoder_h264.c:919-946).
__device__ __forceinline__ int sanitize_i16(int m, bool top, bool left) {
  if (!top && !left) return 2;                              // DC
  if (!top && (m == 0 || m == 3)) return left ? 1 : 2;      // vertical, plane -> horizontal or DC
  if (!left && (m == 1 || m == 3)) return top ? 0 : 2;      // horizontal, plane -> vertical or DC
  return m;
}
__device__ __forceinline__ int sanitize_chroma(int m, bool top, bool left) {
  if (!top && !left) return 0;                              // DC
  if (!top && (m == 2 || m == 3)) return left ? 1 : 0;      // vertical, plane -> horizontal or DC
  if (!left && (m == 1 || m == 3)) return top ? 2 : 0;      // horizontal, plane -> vertical or DC
  return m;
}

// The luma DC block of an I16x16 macroblock: Hadamard of the 16 raw DC
// terms with the reference's rounding, quantised, transposed
// (h264_intra16_luma_dc_transform, encoder_h264.c:711-789).
__device__ void luma_dc_levels(const int32_t* d, const QP& q, int16_t out[16]) {
  int t[16], n[16];
  for (int i = 0; i < 4; ++i) {
    const int s01 = d[i * 4 + 0] + d[i * 4 + 1], d01 = d[i * 4 + 0] - d[i * 4 + 1];
    const int s23 = d[i * 4 + 2] + d[i * 4 + 3], d23 = d[i * 4 + 2] - d[i * 4 + 3];
    t[0 * 4 + i] = s01 + s23;
    t[1 * 4 + i] = s01 - s23;
    t[2 * 4 + i] = d01 - d23;
    t[3 * 4 + i] = d01 + d23;
  }
  for (int i = 0; i < 4; ++i) {
    const int s01 = t[i * 4 + 0] + t[i * 4 + 1], d01 = t[i * 4 + 0] - t[i * 4 + 1];
    const int s23 = t[i * 4 + 2] + t[i * 4 + 3], d23 = t[i * 4 + 2] - t[i * 4 + 3];
    n[i * 4 + 0] = quantize_dc((s01 + s23 + 1) >> 1, q);
    n[i * 4 + 1] = quantize_dc((s01 - s23 + 1) >> 1, q);
    n[i * 4 + 2] = quantize_dc((d01 - d23 + 1) >> 1, q);
    n[i * 4 + 3] = quantize_dc((d01 + d23 + 1) >> 1, q);
  }
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) out[r * 4 + c] = (int16_t)n[c * 4 + r];
}

// ---- 2. per macroblock: header and residual bits --------------------------------
// One warp per macroblock; each lane writes one syntax element group into its
// own bit buffer, in the order the reference writes them: lane 0 the header,
// 1 the I16x16 luma DC block, 2..17 the luma blocks (spec order), 18 and 19 the
// chroma DC blocks, 20..27 the chroma AC blocks (Cb then Cr). A warp scan of
// the lanes' lengths places them; the lanes OR their words into the warp's
// shared copy of the macroblock's region, which is then stored.
constexpr int kCavlcLaneWords = 24;  // one block: at most 16 escaped levels (~36 bits each) + tokens
constexpr int kCavlcMbWarps = 4;

__global__ void __launch_bounds__(32 * kCavlcMbWarps) cavlc_mb_kernel(CavlcArgs a) {
  __shared__ uint32_t shw[kCavlcMbWarps][kCavlcMbWords];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  const int mb = blockIdx.x * kCavlcMbWarps + wi;
  const int mbs = a.mbw * a.mbh;
  if (mb >= mbs) return;
  const uint32_t info = a.info[mb];
  if (info & 1u) {  // skipped: its run is counted by the slice pass
    if (lane == 0) a.nbits[mb] = 0;
    return;
  }
  const int mbx = mb % a.mbw, mby = mb / a.mbw;
  const uint32_t start = slice_start(slice_of(mb, mbs, a.ns), mbs, a.ns);
  const int16_t* lv = a.levels + (size_t)mb * 384;
  const int32_t* dcm = a.dc + (size_t)mb * 24;
  const int cbp_c = (int)((info >> 8) & 3u);
  const bool intra = a.is_intra != 0;
  uint32_t lw[kCavlcLaneWords];
  BitW b;
  bw_init(b, lw, kCavlcLaneWords);
  if (lane == 0) {
    if (intra) {
      int n;
      const bool left = nb_ok(mbx, mby, -1, 0, a.mbw, start, &n), top = nb_ok(mbx, mby, 0, -1, a.mbw, start, &n);
      const uint32_t pm = a.pred_mode[mb];
      put_i16_header(b, sanitize_i16((int)(pm & 3u), top, left), sanitize_chroma((int)((pm >> 2) & 3u), top, left),
                     cbp_c, (int)((info >> 1) & 1u));
    } else {
      int px, py;
      mv_pred(a.mv, mbx, mby, a.mbw, start, &px, &py);
      put_p16_header(b, a.mv[mb].mvx - px, a.mv[mb].mvy - py, (int)((info >> 1) & 15u) | (cbp_c << 4),
                     a.t8, !a.t8f || a.t8f[mb]);
    }
  } else if (lane == 1) {
    if (intra) {
      int16_t ldc[16];
      luma_dc_levels(dcm, make_qp(a.qp, true), ldc);
      put_4x4(b, ldc, false, luma_nc(a.tcs, mb, mbx, mby, a.mbw, start, 0));
    }
  } else if (lane < 18) {
    const int k = lane - 2;
    const bool coded = intra ? ((info >> 1) & 1u) : ((info >> (1 + (k >> 2))) & 1u);
    if (coded && a.t8 && !intra && (!a.t8f || a.t8f[mb])) {
      // 8x8 block k >> 2 as its 4x4 block k & 3: scan positions (k & 3) + 4j (7.3.5.3.2)
      int sc[16];
      const int16_t* l8 = lv + 64 * (k >> 2);
      for (int j = 0; j < 16; ++j) sc[j] = l8[kZigzag8[4 * j + (k & 3)]];
      put_block(b, sc, 16, nc_class(luma_nc(a.tcs, mb, mbx, mby, a.mbw, start, k)));
    } else if (coded) {
      put_4x4(b, lv + (kBlkY4[k] * 4 + kBlkX4[k]) * 16, intra, luma_nc(a.tcs, mb, mbx, mby, a.mbw, start, k));
    }
  } else if (lane < 20) {
    if (cbp_c >= 1) {
      const QP qc = make_qp(chroma_qp(a.qp), intra);
      int c[4];
      chroma_dc(dcm + 16 + 4 * (lane - 18), c);
      for (int i = 0; i < 4; ++i) c[i] = quantize_dc(c[i], qc);
      put_block(b, c, 4, 4);
    }
  } else if (lane < 28) {
    if (cbp_c == 2) {
      const int p = (lane - 20) >> 2, k = (lane - 20) & 3;
      put_4x4(b, lv + (16 + 4 * p + k) * 16, true, chroma_nc(a.tcs, mb, mbx, mby, a.mbw, start, 16 + 4 * p, k));
    }
  }
  bw_flush(b);
  // place the lanes' bits one after another
  const uint32_t len = b.pos;
  uint32_t off = len;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, off, o);
    if (lane >= o) off += y;
  }
  const uint32_t total = __shfl_sync(0xffffffffu, off, 31);
  off -= len;
  const bool over = __any_sync(0xffffffffu, b.over) || total > 32u * kCavlcMbWords;
  if (over) {
    if (lane == 0) {
      atomicExch(a.err, 1u);
      a.nbits[mb] = 0;
    }
    return;
  }
  uint32_t* sw = shw[wi];
  const uint32_t nw = (total + 31u) >> 5;
  for (uint32_t k = lane; k < nw; k += 32) sw[k] = 0u;
  __syncwarp();
  for (uint32_t k = 0; 32u * k < len; ++k) {
    const int m = (int)min(32u, len - 32u * k);
    const uint32_t v = lw[k] >> (32 - m), left = m < 32 ? v << (32 - m) : v;
    const uint32_t pos = off + 32u * k, wd = pos >> 5, sh = pos & 31u;
    atomicOr(sw + wd, left >> sh);
    if (sh + (uint32_t)m > 32u) atomicOr(sw + wd + 1, left << (32u - sh));
  }
  __syncwarp();
  uint32_t* dst = a.words + (size_t)mb * kCavlcMbWords;
  for (uint32_t k = lane; k < nw; k += 32) dst[k] = sw[k];
  if (lane == 0) a.nbits[mb] = total;
}

// ---- 3. per slice: skip runs, offsets, length --------------------------------------
// A chunk of consecutive macroblocks seen from the run of skipped macroblocks:
// `has` a coded one, R = the skips after its last coded macroblock (or all
// of its macroblocks when none is coded). Chunks compose left to right.
struct RunState {
  uint32_t has, r;
};
__device__ __forceinline__ RunState run_then(RunState a, RunState b) {
  return b.has ? b : RunState{a.has, a.r + b.r};
}

// Exclusive block-wide scans over kCavlcScanThreads threads (32 warps).
__device__ RunState scan_run(RunState v, RunState* sh, RunState* total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  RunState x = v;
  for (int o = 1; o < 32; o <<= 1) {
    RunState y{__shfl_up_sync(0xffffffffu, x.has, o), __shfl_up_sync(0xffffffffu, x.r, o)};
    if (lane >= o) x = run_then(y, x);
  }
  if (lane == 31) sh[w] = x;
  __syncthreads();
  if (w == 0) {
    RunState t = sh[lane];
    for (int o = 1; o < 32; o <<= 1) {
      RunState y{__shfl_up_sync(0xffffffffu, t.has, o), __shfl_up_sync(0xffffffffu, t.r, o)};
      if (lane >= o) t = run_then(y, t);
    }
    sh[lane] = t;  // inclusive over warps
  }
  __syncthreads();
  RunState before = w > 0 ? sh[w - 1] : RunState{0u, 0u};
  RunState xin{__shfl_up_sync(0xffffffffu, x.has, 1), __shfl_up_sync(0xffffffffu, x.r, 1)};
  if (lane > 0) before = run_then(before, xin);
  *total = sh[31];
  __syncthreads();
  return before;
}

__device__ uint32_t scan_sum(uint32_t v, uint32_t* sh, uint32_t* total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[w] = x;
  __syncthreads();
  if (w == 0) {
    uint32_t t = sh[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    sh[lane] = t;
  }
  __syncthreads();
  const uint32_t r = (w > 0 ? sh[w - 1] : 0u) + x - v;
  *total = sh[31];
  __syncthreads();
  return r;
}

// OR n <= 32 bits (the low n of v) into MSB-first words at bit position pos.
__device__ __forceinline__ void or_bits(uint32_t* dst, uint32_t pos, uint32_t v, int n, bool atomic) {
  if (n <= 0) return;
  const uint32_t left = n < 32 ? v << (32 - n) : v;  // left-aligned
  const uint32_t k = pos >> 5, sh = pos & 31u;
  const uint32_t hi = left >> sh;
  if (atomic) atomicOr(dst + k, hi);
  else dst[k] |= hi;
  if (sh + (uint32_t)n > 32u) {
    const uint32_t lo = left << (32u - sh);
    if (atomic) atomicOr(dst + k + 1, lo);
    else dst[k + 1] |= lo;
  }
}

__global__ void __launch_bounds__(kCavlcScanThreads) cavlc_slice_kernel(CavlcArgs a, CavlcHdr h) {
  __shared__ RunState shr[32];
  __shared__ uint32_t shs[32];
  const int s = blockIdx.x, t = threadIdx.x;
  const uint32_t mbs = (uint32_t)(a.mbw * a.mbh);
  const uint32_t m0 = slice_start(s, mbs, a.ns), m1 = slice_start(s + 1, mbs, a.ns);
  const uint32_t per = (m1 - m0 + kCavlcScanThreads - 1) / kCavlcScanThreads;
  const uint32_t i0 = min(m1, m0 + t * per), i1 = min(m1, i0 + per);
  // this thread's chunk: leading skips, skips after its last coded
  // macroblock, the bits of its coded macroblocks but the first one's run
  // (I slices have no mb_skip_run: every macroblock is coded, runs are 0 bits)
  const bool runs = !a.is_intra;
  uint32_t lead = 0, tail = 0, inner = 0, has = 0;
  for (uint32_t mb = i0; mb < i1; ++mb) {
    if (a.info[mb] & 1u) {
      if (has) ++tail;
      else ++lead;
    } else {
      inner += (has && runs ? (uint32_t)ue_bits(tail) : 0u) + a.nbits[mb];
      tail = 0;
      has = 1;
    }
  }
  RunState all;
  const RunState in = scan_run(RunState{has, has ? tail : lead}, shr, &all);
  const uint32_t mine = has ? (runs ? (uint32_t)ue_bits(in.r + lead) : 0u) + inner : 0u;
  uint32_t data = 0;
  const uint32_t base = (uint32_t)h.len[s] + scan_sum(mine, shs, &data);
  const uint32_t trail = all.r;  // skips after the slice's last coded macroblock
  const uint32_t bits = (uint32_t)h.len[s] + data + (trail ? (uint32_t)ue_bits(trail) : 0u) + 1u;
  const uint32_t bytes = (bits + 7u) >> 3;
  const bool fits = bytes <= a.slice_cap && *a.err == 0u;
  // offsets and runs of the coded macroblocks
  uint32_t pos = base, run = in.r;
  for (uint32_t mb = i0; mb < i1; ++mb) {
    if (a.info[mb] & 1u) {
      ++run;
    } else {
      a.off[mb] = pos;
      a.run[mb] = runs ? run : 0xffffffffu;
      pos += (runs ? (uint32_t)ue_bits(run) : 0u) + a.nbits[mb];
      run = 0;
    }
  }
  uint32_t* dst = reinterpret_cast<uint32_t*>(a.out + (size_t)s * a.slice_cap);
  const uint32_t nw = (bytes + 3u) >> 2;
  if (fits)
    for (uint32_t k = t; k < nw; k += kCavlcScanThreads) dst[k] = 0u;
  __syncthreads();
  if (t == 0) {
    a.sl[4 * s + 0] = bits;
    a.sl[4 * s + 1] = trail;
    a.sl[4 * s + 2] = fits ? 0u : 1u;
    a.out_bytes[s] = fits ? bytes : 0xffffffffu;
    if (fits) {
      for (int k = 0; k < 4 && 32 * k < h.len[s]; ++k)
        or_bits(dst, 32u * k, h.bits[s][k] >> (32 - min(32, h.len[s] - 32 * k)), min(32, h.len[s] - 32 * k), false);
      uint32_t p = (uint32_t)h.len[s] + data;
      if (trail) {  // mb_skip_run of the slice's last macroblocks
        const int l = ilog2(trail + 1u);
        or_bits(dst, p + (uint32_t)l, trail + 1u, l + 1, false);
        p += (uint32_t)(2 * l + 1);
      }
      or_bits(dst, p, 1u, 1, false);  // rbsp_stop_one_bit; the alignment zeros are the cleared words
    }
  }
}

// ---- 4. place each coded macroblock's bits -------------------------------------
__global__ void __launch_bounds__(128) cavlc_pack_kernel(CavlcArgs a) {
  const int mb = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t mbs = (uint32_t)(a.mbw * a.mbh);
  if (mb >= (int)mbs || (a.info[mb] & 1u)) return;
  const uint32_t s = slice_of((uint32_t)mb, mbs, (uint32_t)a.ns);
  if (a.sl[4 * s + 2]) return;  // the slice did not fit
  uint32_t* dst = reinterpret_cast<uint32_t*>(a.out + (size_t)s * a.slice_cap);
  const uint32_t run = a.run[mb];
  uint32_t p = a.off[mb];
  if (run != 0xffffffffu) {  // mb_skip_run (P slices)
    const int l = ilog2(run + 1u);
    or_bits(dst, p + (uint32_t)l, run + 1u, l + 1, true);
    p += (uint32_t)(2 * l + 1);
  }
  const uint32_t n = a.nbits[mb];
  const uint32_t* w = a.words + (size_t)mb * kCavlcMbWords;
  for (uint32_t k = 0; 32u * k < n; ++k) {
    const int m = (int)min(32u, n - 32u * k);
    or_bits(dst, p + 32u * k, w[k] >> (32 - m), m, true);
  }
}

// MSB-first words -> stream bytes (in place, or into out_copy: only the
// slice's bytes cross to a host mapping).
__global__ void cavlc_bytes_kernel(CavlcArgs a) {
  const int s = blockIdx.y;
  const uint32_t nb = a.sl[4 * s + 2] ? 0xffffffffu : (a.sl[4 * s + 0] + 7u) >> 3;
  if (nb == 0xffffffffu) return;
  const uint32_t* src = reinterpret_cast<const uint32_t*>(a.out + (size_t)s * a.slice_cap);
  uint32_t* dst = reinterpret_cast<uint32_t*>(a.out_copy + (size_t)s * a.slice_cap);
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < (nb + 3u) >> 2; k += gridDim.x * blockDim.x)
    dst[k] = __byte_perm(src[k], 0u, 0x0123);
}

}  // namespace b200enc

using namespace b200enc;

namespace {

struct CavlcLayout {
  size_t info, tcs, nbits, words, off, run, sl, err, bytes;
};

size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }

CavlcLayout cavlc_layout(int mbw, int mbh) {
  const size_t mbs = (size_t)mbw * mbh;
  CavlcLayout l;
  l.err = 0;
  l.sl = 256;
  l.info = l.sl + up256(kCavlcMaxSlices * 16);
  l.tcs = l.info + up256(mbs * 4);
  l.nbits = l.tcs + up256(mbs * 24);
  l.off = l.nbits + up256(mbs * 4);
  l.run = l.off + up256(mbs * 4);
  l.words = l.run + up256(mbs * 4);
  l.bytes = l.words + mbs * kCavlcMbWords * 4;
  return l;
}

}  // namespace

extern "C" size_t b200enc_cavlc_scratch_bytes(int mbw, int mbh) {
  if (mbw <= 0 || mbh <= 0) return 0;
  return cavlc_layout(mbw, mbh).bytes;
}

extern "C" int b200enc_cavlc_slices(const b200enc_cavlc_t* p, void* stream) {
  if (!p || p->mbw <= 0 || p->mbh <= 0 || p->qp < 0 || p->qp > 51 || p->num_slices < 1 ||
      p->num_slices > kCavlcMaxSlices || p->num_slices > p->mbw * p->mbh)
    return -1;
  if (!p->levels || !p->dc || !p->nz || !p->mv || (p->is_intra && !p->pred_mode) || !p->out || !p->out_bytes ||
      !p->scratch)
    return -1;
  if ((p->slice_cap & 3) || p->slice_cap < 4 || (((uintptr_t)p->out) & 3) || (((uintptr_t)p->out_copy) & 3) ||
      (((uintptr_t)p->scratch) & 255))
    return -1;
  const CavlcLayout L = cavlc_layout(p->mbw, p->mbh);
  if (p->scratch_bytes < L.bytes) return -1;
  CavlcHdr h{};
  for (int s = 0; s < p->num_slices; ++s) {
    const int n = p->header_bits ? p->header_bits[s] : 0;
    if (n < 0 || n > 128 || (n > 0 && !p->header)) return -1;
    h.len[s] = n;
    for (int k = 0; k < 4; ++k) {
      uint32_t w = 0;
      for (int j = 0; j < 4; ++j) w = (w << 8) | (n > 0 ? p->header[16 * s + 4 * k + j] : 0u);
      h.bits[s][k] = w;
    }
  }
  uint8_t* sc = static_cast<uint8_t*>(p->scratch);
  CavlcArgs a;
  a.mbw = p->mbw;
  a.mbh = p->mbh;
  a.qp = p->qp;
  a.is_intra = p->is_intra ? 1 : 0;
  a.ns = p->num_slices;
  a.quality = p->quality_level;
  a.t8 = p->transform8x8 ? 1 : 0;
  a.t8f = p->t8_flags;
  a.levels = p->levels;
  a.dc = p->dc;
  a.nz = p->nz;
  a.pred_mode = p->pred_mode;
  a.mv = static_cast<const MV*>(p->mv);
  a.info = reinterpret_cast<uint32_t*>(sc + L.info);
  a.tcs = sc + L.tcs;
  a.nbits = reinterpret_cast<uint32_t*>(sc + L.nbits);
  a.words = reinterpret_cast<uint32_t*>(sc + L.words);
  a.off = reinterpret_cast<uint32_t*>(sc + L.off);
  a.run = reinterpret_cast<uint32_t*>(sc + L.run);
  a.sl = reinterpret_cast<uint32_t*>(sc + L.sl);
  a.err = reinterpret_cast<uint32_t*>(sc + L.err);
  a.out = p->out;
  a.slice_cap = (uint32_t)std::min<size_t>(p->slice_cap, 0xfffffffcu);
  a.out_bytes = p->out_bytes;
  a.out_copy = p->out_copy ? p->out_copy : p->out;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int mbs = p->mbw * p->mbh;
  if (cudaMemsetAsync(a.err, 0, 4, st) != cudaSuccess) return -1;
  cavlc_info_kernel<<<(mbs + 127) / 128, 128, 0, st>>>(a);
  cavlc_mb_kernel<<<(mbs + kCavlcMbWarps - 1) / kCavlcMbWarps, 32 * kCavlcMbWarps, 0, st>>>(a);
  cavlc_slice_kernel<<<p->num_slices, kCavlcScanThreads, 0, st>>>(a, h);
  cavlc_pack_kernel<<<(mbs + 127) / 128, 128, 0, st>>>(a);
  cavlc_bytes_kernel<<<dim3(16, p->num_slices), 256, 0, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
