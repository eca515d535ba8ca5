// pframe.cu - fused P-macroblock chain: motion-compensated prediction,
// residual, forward 4x4, AC quant + nonzero masks, chroma DC Hadamard,
// dequant, inverse 4x4 and reconstruction, one CTA (3 warps) per MB.
//
// Reference stages, which run as five separate dispatches with int32
// residual/pred/coeff buffers round-tripping through memory:
//   A1/shaders/residual_predict.comp:417-434, :576-635 (luma qpel MC, chroma
//   eighth-pel MC), dct_transform.comp:75-98, quantize.comp:189-225,
//   reconstruct.comp:318-442.
// Here nothing but the frame planes, the MV and the staged outputs touch
// HBM: the prediction lives in shared memory, each 4x4 block is owned by a
// quad of lanes (one row each) and all 24 blocks of the MB sit in its 3
// warps, so the chroma DC exchange stays inside warp 2.
#include "b200enc_internal.h"
#include "common.cuh"
#include "t8x8.cuh"

namespace b200enc {

struct PShared {
  // Reference and source rows staged as 16-byte units. The luma patch row r
  // holds reference row iy0-2+r from column lxa (16-aligned) on; the patch
  // origin (ix0-2, iy0-2) is at byte lo of row 0. The chroma patch (NV12
  // pairs) starts at byte cxa (16-aligned); chroma sample (ixc, iyc) is at
  // byte co of row 0.
  alignas(16) uint8_t lp[21][48];
  alignas(16) uint8_t cp[9][32];
  alignas(16) uint8_t src[16][16];   // current luma
  alignas(16) uint8_t srcc[8][16];   // current chroma (NV12 pairs)
  int16_t pred[24][16];    // prediction per block, raster within block
  int16_t res[24][16];     // residual
  alignas(16) int16_t lev[24][16];  // quantized levels (for the coalesced store)
  int32_t cdc[8];          // pre-quant chroma DC coefficients
  int32_t dcval[8];        // dequantized chroma DC per chroma block
  alignas(16) uint8_t ry[16][16];  // reconstructed luma
  alignas(16) uint8_t ruv[8][16];  // reconstructed chroma (NV12)
  int32_t t8[4][65];               // 8x8 luma transform: the four blocks between their row and column passes
  int32_t cost[3];                 // 4x4 (two warps' halves) and 8x8 Hadamard costs of the luma residual
};

// Horizontal / vertical 6-tap raw sums on a staged patch `p` (row pitch ps)
// whose element (0, 0) is reference sample (ix0-2, iy0-2).
__device__ __forceinline__ int hraw_p(const uint8_t* p, int ps, int x, int y) {
  // centred between integer columns x and x+1 of row y
  const uint8_t* r = p + (y + 2) * ps;
  return r[x] - 5 * r[x + 1] + 20 * r[x + 2] + 20 * r[x + 3] - 5 * r[x + 4] + r[x + 5];
}
__device__ __forceinline__ int vraw_p(const uint8_t* p, int ps, int x, int y) {
  const uint8_t* c = p + x + 2;
  return c[y * ps] - 5 * c[(y + 1) * ps] + 20 * c[(y + 2) * ps] + 20 * c[(y + 3) * ps] - 5 * c[(y + 4) * ps] +
         c[(y + 5) * ps];
}

// Luma quarter-pel sample (residual_predict.comp:263-298) for block-relative
// pixel (x, y) whose integer anchor is patch (x+2, y+2).
__device__ __forceinline__ int mc_luma(const uint8_t* p, int ps, int x, int y, int fx, int fy) {
  auto at = [&](int xx, int yy) { return (int)p[yy * ps + xx]; };
  const int G = at(x + 2, y + 2);
  if (!(fx | fy)) return G;
  const int phase = fy * 4 + fx;
  auto B = [&](int xx, int yy) { return clip1((hraw_p(p, ps, xx, yy) + 16) >> 5); };
  auto Hh = [&](int xx, int yy) { return clip1((vraw_p(p, ps, xx, yy) + 16) >> 5); };
  auto J = [&]() {
    const int j1 = hraw_p(p, ps, x, y - 2) - 5 * hraw_p(p, ps, x, y - 1) + 20 * hraw_p(p, ps, x, y) +
                   20 * hraw_p(p, ps, x, y + 1) - 5 * hraw_p(p, ps, x, y + 2) + hraw_p(p, ps, x, y + 3);
    return clip1((j1 + 512) >> 10);
  };
  switch (phase) {
    case 1: return (G + B(x, y) + 1) >> 1;
    case 2: return B(x, y);
    case 3: return (B(x, y) + at(x + 3, y + 2) + 1) >> 1;
    case 4: return (G + Hh(x, y) + 1) >> 1;
    case 5: return (B(x, y) + Hh(x, y) + 1) >> 1;
    case 6: return (B(x, y) + J() + 1) >> 1;
    case 7: return (B(x, y) + Hh(x + 1, y) + 1) >> 1;
    case 8: return Hh(x, y);
    case 9: return (Hh(x, y) + J() + 1) >> 1;
    case 10: return J();
    case 11: return (J() + Hh(x + 1, y) + 1) >> 1;
    case 12: return (Hh(x, y) + at(x + 2, y + 3) + 1) >> 1;
    case 13: return (Hh(x, y) + B(x, y + 1) + 1) >> 1;
    case 14: return (J() + B(x, y + 1) + 1) >> 1;
    default: return (Hh(x + 1, y) + B(x, y + 1) + 1) >> 1;
  }
}

// Stages sixteen bytes of a row, `gx` 16-aligned, into `dst` (shared,
// 16-aligned): one vector load where the bytes lie inside [0, lim) of a row
// whose base is 16-byte aligned (`vec`), else byte loads of the clamped
// columns. `pair` selects NV12 chroma clamping: byte b of the row is
// component b&1 of sample clamp(b>>1, 0, lim/2-1).
__device__ __forceinline__ void stage16_clamped(uint8_t* dst, const uint8_t* row, int gx, int lim, bool vec,
                                                bool pair) {
  if (vec && gx >= 0 && gx + 16 <= lim) {
    *reinterpret_cast<uint4*>(dst) = __ldg(reinterpret_cast<const uint4*>(row + gx));
    return;
  }
#pragma unroll 1
  for (int j = 0; j < 16; ++j) {
    const int b = gx + j;
    const int c = pair ? 2 * clampi(b >> 1, 0, (lim >> 1) - 1) + (b & 1) : clampi(b, 0, lim - 1);
    dst[j] = __ldg(row + c);
  }
}

// One CTA holds blockDim.y macroblocks of a row (the autotuner's tile
// shape: 1, 2 or 4), 96 threads (three warps) each; a macroblock's shared
// state is its slice of the dynamic shared memory. BATCH: one CTA per P
// macroblock of a batch (compact index blockIdx.x), which finds its stream,
// takes its vector from the batch's compact field and stores it into the
// stream's own field.
template <bool BATCH>
__global__ void __launch_bounds__(384, 4) p_mb_kernel(const uint8_t* __restrict__ cur_y_, const uint8_t* __restrict__ cur_uv_,
                                                  int cur_pitch_, const uint8_t* __restrict__ ref_y_,
                                                  const uint8_t* __restrict__ ref_uv_, int ref_pitch_, Geo g_, int qp_,
                                                  const MV* __restrict__ mvs, int16_t* __restrict__ levels_,
                                                  int32_t* __restrict__ dc_, uint32_t* __restrict__ nzm_,
                                                  uint32_t* __restrict__ pred_mode_, uint8_t* __restrict__ rec_y_,
                                                  uint8_t* __restrict__ rec_uv_, int rec_pitch_, BatchTab bt,
                                                  int t8 = 0, uint8_t* __restrict__ t8_flags = nullptr) {
  extern __shared__ __align__(16) uint8_t p_smem[];
  PShared& s = reinterpret_cast<PShared*>(p_smem)[threadIdx.y];
  const int tid = threadIdx.x;
  const uint8_t *cur_y = cur_y_, *cur_uv = cur_uv_, *ref_y = ref_y_, *ref_uv = ref_uv_;
  int cur_pitch = cur_pitch_, ref_pitch = ref_pitch_, qp = qp_, rec_pitch = rec_pitch_;
  Geo g = g_;
  int16_t* levels = levels_;
  int32_t* dc = dc_;
  uint32_t *nzm = nzm_, *pred_mode = pred_mode_;
  uint8_t *rec_y = rec_y_, *rec_uv = rec_uv_;
  bool active;
  int mbx, mby, mb;
  MV mv;
  if (BATCH) {
    const int ci = blockIdx.x;
    const int k = bt.p_mbs.find(ci);
    const BatchStream& st = bt.p_mbs.stream(k);
    mb = ci - bt.p_mbs.prefix[k];
    g = st.g;
    if (mb >= g.mbw * g.mbh) return;  // padding of the compact index (uniform over the CTA)
    mby = mb / g.mbw;
    mbx = mb - mby * g.mbw;
    active = true;
    cur_y = st.cur_y;
    cur_uv = st.cur_uv;
    cur_pitch = st.cur_pitch;
    ref_y = st.ref_y;
    ref_uv = st.ref_uv;
    ref_pitch = rec_pitch = st.rec_pitch;
    qp = st.qp;
    levels = st.levels;
    dc = st.dc;
    nzm = st.nz;
    pred_mode = st.pred_mode;
    rec_y = st.rec_y;
    rec_uv = st.rec_uv;
    mv = bt.mvc[ci];
    if (tid == 0) st.mv[mb] = mv;
  } else {
    // a tile reaching past the right edge computes a copy of the last
    // macroblock and stores nothing
    const int mbx_t = blockIdx.x * blockDim.y + threadIdx.y;
    active = mbx_t < g.mbw;
    mbx = active ? mbx_t : g.mbw - 1;
    mby = blockIdx.y;
    mb = mby * g.mbw + mbx;
    mv = mvs[mb];
  }
  const int X = mbx * 16, Y = mby * 16, Xc = X >> 1, Yc = Y >> 1;
  const int ix0 = X + (mv.mvx >> 2), iy0 = Y + (mv.mvy >> 2), fx = mv.mvx & 3, fy = mv.mvy & 3;
  const int ixc = Xc + (mv.mvx >> 3), iyc = Yc + (mv.mvy >> 3), fxc = mv.mvx & 7, fyc = mv.mvy & 7;
  const int cmx = g.RW / 2 - 1, cmy = g.RH / 2 - 1;

  // ---- stage reference patches and the source (16-byte units) -----------
  // Units: 0..62 luma patch (21 rows x 3), 63..80 chroma patch (9 x 2),
  // 81..96 source luma rows, 97..104 source chroma rows. Reads clamp to
  // (RW, RH) for the reference and (W, H) for the source, per sample, as the
  // byte-wise reference stages do; the vector path is taken where no clamp
  // applies.
  const int lxa = (ix0 - 2) & ~15, lo = (ix0 - 2) - lxa;
  const int cxa = (2 * ixc) & ~15, co = 2 * ixc - cxa;
  const bool rvec = ((ref_pitch & 15) == 0) && ((reinterpret_cast<uintptr_t>(ref_y) & 15) == 0) &&
                    ((reinterpret_cast<uintptr_t>(ref_uv) & 15) == 0);
  const bool cvec = ((cur_pitch & 15) == 0) && ((reinterpret_cast<uintptr_t>(cur_y) & 15) == 0) &&
                    ((reinterpret_cast<uintptr_t>(cur_uv) & 15) == 0);
  for (int u = tid; u < 105; u += 96) {
    if (u < 63) {
      const int r = u / 3, q = u - 3 * r;
      const uint8_t* row = ref_y + (size_t)clampi(iy0 - 2 + r, 0, g.RH - 1) * ref_pitch;
      stage16_clamped(&s.lp[r][16 * q], row, lxa + 16 * q, g.RW, rvec, false);
    } else if (u < 81) {
      const int r = (u - 63) >> 1, q = (u - 63) & 1;
      const uint8_t* row = ref_uv + (size_t)clampi(iyc + r, 0, cmy) * ref_pitch;
      stage16_clamped(&s.cp[r][16 * q], row, cxa + 16 * q, 2 * (g.RW / 2), rvec, true);
    } else if (u < 97) {
      const int r = u - 81;
      const uint8_t* row = cur_y + (size_t)clampi(Y + r, 0, g.H - 1) * cur_pitch;
      stage16_clamped(&s.src[r][0], row, X, g.W, cvec, false);
    } else {
      const int r = u - 97;
      const uint8_t* row = cur_uv + (size_t)clampi(Yc + r, 0, g.H / 2 - 1) * cur_pitch;
      stage16_clamped(&s.srcc[r][0], row, 2 * Xc, 2 * (g.W / 2), cvec, true);
    }
  }
  __syncthreads();

  // ---- prediction + residual --------------------------------------------
  const uint8_t* lpp = &s.lp[0][lo];
  for (int i = tid; i < 256; i += 96) {
    const int x = i & 15, y = i >> 4;
    const int pv = mc_luma(lpp, 48, x, y, fx, fy);
    const int src = s.src[y][x];
    const int blk = (y >> 2) * 4 + (x >> 2), pos = (y & 3) * 4 + (x & 3);
    s.pred[blk][pos] = (int16_t)pv;
    s.res[blk][pos] = (int16_t)(src - pv);
  }
  for (int i = tid; i < 128; i += 96) {
    const int pl = i >> 6, x = i & 7, y = (i >> 3) & 7;
    const int A = s.cp[y][co + 2 * x + pl], B = s.cp[y][co + 2 * x + 2 + pl];
    const int C = s.cp[y + 1][co + 2 * x + pl], D = s.cp[y + 1][co + 2 * x + 2 + pl];
    const int pv = ((8 - fxc) * (8 - fyc) * A + fxc * (8 - fyc) * B + (8 - fxc) * fyc * C + fxc * fyc * D + 32) >> 6;
    const int src = s.srcc[y][2 * x + pl];
    const int blk = 16 + 4 * pl + (y >> 2) * 2 + (x >> 2), pos = (y & 3) * 4 + (x & 3);
    s.pred[blk][pos] = (int16_t)pv;
    s.res[blk][pos] = (int16_t)(src - pv);
  }
  __syncthreads();

  // ---- 4x4 or 8x8 luma transform (t8 = 2: chosen per macroblock) --------
  // The residual's cost under each size, on the scale of a SAD: 4x4 blocks
  // (sum |H4 R H4|) / 2 - quads of warps 0-1, row r of block b, the column
  // pass across the quad by shuffles - and 8x8 blocks (sum |H8 R H8| + 2) / 4
  // - warp 2, eight lanes per block, transposed through s.t8. H4 and H8 are
  // unnormalised Walsh-Hadamard matrices; any row order gives the same sums.
  bool use8 = t8 == 1;
  if (t8 == 2) {
    if (tid < 64) {
      const int bb = tid >> 2, rr = tid & 3;
      int h[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) h[i] = s.res[bb][4 * rr + i];
      const int a0 = h[0] + h[1], a1 = h[0] - h[1], a2 = h[2] + h[3], a3 = h[2] - h[3];
      h[0] = a0 + a2;
      h[1] = a1 + a3;
      h[2] = a0 - a2;
      h[3] = a1 - a3;
      int sum = 0;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int o1 = __shfl_xor_sync(0xffffffffu, h[i], 1);
        const int u = (rr & 1) ? o1 - h[i] : h[i] + o1;
        const int o2 = __shfl_xor_sync(0xffffffffu, u, 2);
        const int w = (rr & 2) ? o2 - u : u + o2;
        sum += abs(w);
      }
      sum += __shfl_xor_sync(0xffffffffu, sum, 1);
      sum += __shfl_xor_sync(0xffffffffu, sum, 2);
      int c = rr == 0 ? sum >> 1 : 0;
#pragma unroll
      for (int o = 4; o < 32; o <<= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
      if ((tid & 31) == 0) s.cost[tid >> 5] = c;
    } else {
      const int ln = tid - 64, qq = ln >> 3, kk = ln & 7, ox = 8 * (qq & 1), oy = 8 * (qq >> 1);
      int v[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const int xx = ox + c, yy = oy + kk;
        v[c] = s.res[(yy >> 2) * 4 + (xx >> 2)][(yy & 3) * 4 + (xx & 3)];
      }
      had8(v);
#pragma unroll
      for (int c = 0; c < 8; ++c) s.t8[qq][8 * kk + c] = v[c];
      __syncwarp();
#pragma unroll
      for (int i = 0; i < 8; ++i) v[i] = s.t8[qq][8 * i + kk];
      had8(v);
      int sum = 0;
#pragma unroll
      for (int i = 0; i < 8; ++i) sum += abs(v[i]);
#pragma unroll
      for (int o = 1; o < 8; o <<= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
      int c = kk == 0 ? (sum + 2) >> 2 : 0;
      c += __shfl_xor_sync(0xffffffffu, c, 8);
      c += __shfl_xor_sync(0xffffffffu, c, 16);
      if (ln == 0) s.cost[2] = c;
    }
    __syncthreads();
    use8 = s.cost[2] < s.cost[0] + s.cost[1];
  }

  // ---- forward + quant: quad (b, r) owns row r of block b ---------------
  // (with the 8x8 luma transform, warp 0 codes the four 8x8 luma blocks
  // instead and warp 1 has no luma block; chroma is the same)
  const int b = tid >> 2, r = tid & 3;
  const bool luma = b < 16;
  const bool quad = !(use8 && luma);
  const QP q = make_qp(luma ? qp : chroma_qp(qp), false);
  int x[4];
  if (quad) {
#pragma unroll
    for (int i = 0; i < 4; ++i) x[i] = s.res[b][4 * r + i];
    quad_forward(x, r);  // x[i] = coef[i][r]
    uint32_t nz = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int pos = 4 * i + r;
      const int l = quant_ac(x[i], pos, q);
      s.lev[b][pos] = (int16_t)clampi(l, -32768, 32767);
      nz |= (l != 0 ? 1u : 0u) << pos;
    }
    nz |= __shfl_xor_sync(0xffffffffu, nz, 1);
    nz |= __shfl_xor_sync(0xffffffffu, nz, 2);
    if (r == 0) {
      if (active) {
        nzm[(size_t)mb * 24 + b] = nz;
        dc[(size_t)mb * 24 + b] = x[0];
      }
      if (!luma) s.cdc[b - 16] = x[0];
    }
  }
  // 8x8 luma (warp 0): block q8 = tid >> 3 (raster of the four), thread k8
  // owns its row k8, then its column k8. Levels in raster order at
  // lev[0..255] (block q8 at 64 * q8); the nz word of 4x4 block 4 * q8 + i
  // (spec order) holds the nonzero mask of the 16 levels CAVLC codes as that
  // block: 8x8 scan positions i, i + 4, ... (7.3.5.3.2).
  const int q8 = tid >> 3, k8 = tid & 7, qx = 8 * (q8 & 1), qy = 8 * (q8 >> 1);
  const int per8 = qp / 6, rem8 = qp - 6 * per8;
  if (use8 && tid < 32) {
    auto res_at = [&](int xx, int yy) { return (int)s.res[(yy >> 2) * 4 + (xx >> 2)][(yy & 3) * 4 + (xx & 3)]; };
    int v[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) v[c] = res_at(qx + c, qy + k8);
    fwd8(v);
#pragma unroll
    for (int c = 0; c < 8; ++c) s.t8[q8][8 * k8 + c] = v[c];
    __syncwarp();
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = s.t8[q8][8 * i + k8];
    fwd8(v);
    const int sh = 16 + per8;
    const long long f = (1ll << sh) / 6;  // inter rounding
    uint32_t m[4] = {0u, 0u, 0u, 0u};
    int16_t* lev8 = &s.lev[0][0] + 64 * q8;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int l = quant8(v[i], i, k8, rem8, sh, f);
      lev8[8 * i + k8] = (int16_t)clampi(l, -32768, 32767);
      const int z = kZigzag8Inv[8 * i + k8];
      m[z & 3] |= (l != 0 ? 1u : 0u) << (z >> 2);
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      m[j] |= __shfl_xor_sync(0xffffffffu, m[j], 1);
      m[j] |= __shfl_xor_sync(0xffffffffu, m[j], 2);
      m[j] |= __shfl_xor_sync(0xffffffffu, m[j], 4);
    }
    if (k8 == 0 && active) {
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        // spec block 4 * q8 + i -> raster: quadrant origin (qx / 4, qy / 4) + (i & 1, i >> 1)
        const int rb = (qy / 4 + (i >> 1)) * 4 + qx / 4 + (i & 1);
        nzm[(size_t)mb * 24 + rb] = m[i];
        dc[(size_t)mb * 24 + rb] = 0;
      }
    }
  }
  __syncwarp();
  // chroma DC Hadamard + quant + inverse + dequant (reconstruct.comp:393-414),
  // warp 2 only: lanes of block 16 (Cb) and block 20 (Cr)
  if (!luma && r == 0 && ((b - 16) & 3) == 0) {
    const int pl = (b - 16) >> 2;
    const int c0 = s.cdc[4 * pl], c1 = s.cdc[4 * pl + 1], c2 = s.cdc[4 * pl + 2], c3 = s.cdc[4 * pl + 3];
    const int l0 = quantize_dc(c0 + c1 + c2 + c3, q), l1 = quantize_dc(c0 - c1 + c2 - c3, q);
    const int l2 = quantize_dc(c0 + c1 - c2 - c3, q), l3 = quantize_dc(c0 - c1 - c2 + c3, q);
    s.dcval[4 * pl + 0] = dequant_dc_chroma(l0 + l1 + l2 + l3, q);
    s.dcval[4 * pl + 1] = dequant_dc_chroma(l0 - l1 + l2 - l3, q);
    s.dcval[4 * pl + 2] = dequant_dc_chroma(l0 + l1 - l2 - l3, q);
    s.dcval[4 * pl + 3] = dequant_dc_chroma(l0 - l1 - l2 + l3, q);
  }
  __syncwarp();

  // ---- dequant + inverse + recon ----------------------------------------
  if (use8 && tid < 32) {  // 8x8 luma: scaling + inverse (8.5.13) onto the prediction
    const int16_t* lev8 = &s.lev[0][0] + 64 * q8;
    int v[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) v[c] = scale8(lev8[8 * k8 + c], k8, c, per8, rem8);
    inv8(v);
#pragma unroll
    for (int c = 0; c < 8; ++c) s.t8[q8][8 * k8 + c] = v[c];
    __syncwarp();
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = s.t8[q8][8 * i + k8];
    inv8(v);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int yy = qy + i, xx = qx + k8;
      s.ry[yy][xx] = (uint8_t)clip1(s.pred[(yy >> 2) * 4 + (xx >> 2)][(yy & 3) * 4 + (xx & 3)] + ((v[i] + 32) >> 6));
    }
  }
  int d[4];
  if (quad) {
#pragma unroll
    for (int i = 0; i < 4; ++i) d[i] = dequant_ac(s.lev[b][4 * r + i], 4 * r + i, q);
    if (r == 0) {
      if (!luma) d[0] = s.dcval[b - 16];
      d[0] += 32;
    }
    quad_inverse(d, r);  // d[i] = res[i][r]
  }
  if (quad && luma) {
    const int bx = b & 3, by = b >> 2;
#pragma unroll
    for (int i = 0; i < 4; ++i) s.ry[4 * by + i][4 * bx + r] = (uint8_t)clip1(s.pred[b][4 * i + r] + d[i]);
  } else if (quad) {
    const int pl = (b - 16) >> 2, sub = (b - 16) & 3;
#pragma unroll
    for (int i = 0; i < 4; ++i)
      s.ruv[4 * (sub >> 1) + i][2 * (4 * (sub & 1) + r) + pl] = (uint8_t)clip1(s.pred[b][4 * i + r] + d[i]);
  }
  __syncthreads();

  // ---- coalesced stores ---------------------------------------------------
  if (!active) return;
  if (tid < 48) {
    reinterpret_cast<uint4*>(levels + (size_t)mb * 384)[tid] = reinterpret_cast<const uint4*>(&s.lev[0][0])[tid];
  } else if (tid < 64) {
    const int row = tid - 48, gy = Y + row;
    if (gy < g.RH) {
      uint8_t* dst = rec_y + (size_t)gy * rec_pitch + X;
      if (X + 16 <= g.RW) {
        *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(s.ry[row]);
      } else {
        for (int c = 0; c < 16 && X + c < g.RW; ++c) dst[c] = s.ry[row][c];
      }
    }
  } else if (tid < 72) {
    const int row = tid - 64, gy = Yc + row;
    if (gy <= cmy) {
      uint8_t* dst = rec_uv + (size_t)gy * rec_pitch + 2 * Xc;
      if (Xc + 8 <= cmx + 1) {
        *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(s.ruv[row]);
      } else {
        for (int c = 0; c < 8 && Xc + c <= cmx; ++c) {
          dst[2 * c] = s.ruv[row][2 * c];
          dst[2 * c + 1] = s.ruv[row][2 * c + 1];
        }
      }
    }
  } else if (tid == 72) {
    pred_mode[mb] = 2u;  // residual_predict.comp:422
    if (t8_flags) t8_flags[mb] = use8 ? 1u : 0u;
  }
}

}  // namespace b200enc

using namespace b200enc;

extern "C" int b200enc_p_frame_t8(const uint8_t* cur_y, const uint8_t* cur_uv, int cur_pitch, const uint8_t* ref_y,
                                  const uint8_t* ref_uv, int ref_pitch, int W, int H, int RW, int RH, int qp,
                                  const void* mv, int16_t* levels, int32_t* dc, uint32_t* nz, uint32_t* pred_mode,
                                  uint8_t* rec_y, uint8_t* rec_uv, int rec_pitch, int t8, uint8_t* t8_flags,
                                  void* stream);

extern "C" int b200enc_p_frame(const uint8_t* cur_y, const uint8_t* cur_uv, int cur_pitch, const uint8_t* ref_y,
                               const uint8_t* ref_uv, int ref_pitch, int W, int H, int RW, int RH, int qp,
                               const void* mv, int16_t* levels, int32_t* dc, uint32_t* nz, uint32_t* pred_mode,
                               uint8_t* rec_y, uint8_t* rec_uv, int rec_pitch, void* stream) {
  return b200enc_p_frame_t8(cur_y, cur_uv, cur_pitch, ref_y, ref_uv, ref_pitch, W, H, RW, RH, qp, mv, levels, dc,
                            nz, pred_mode, rec_y, rec_uv, rec_pitch, 0, nullptr, stream);
}

extern "C" int b200enc_p_frame_t8(const uint8_t* cur_y, const uint8_t* cur_uv, int cur_pitch, const uint8_t* ref_y,
                                  const uint8_t* ref_uv, int ref_pitch, int W, int H, int RW, int RH, int qp,
                                  const void* mv, int16_t* levels, int32_t* dc, uint32_t* nz, uint32_t* pred_mode,
                                  uint8_t* rec_y, uint8_t* rec_uv, int rec_pitch, int t8, uint8_t* t8_flags,
                                  void* stream) {
  if (t8 < 0 || t8 > 2) return -1;
  if (!cur_y || !cur_uv || !ref_y || !ref_uv || !mv || !levels || !dc || !nz || !pred_mode || !rec_y || !rec_uv)
    return -1;
  if (qp < 0 || qp > 51 || W <= 0 || H <= 0 || RW <= 1 || RH <= 1) return -1;
  if ((rec_pitch & 15) || (((uintptr_t)rec_y) & 15) || (((uintptr_t)rec_uv) & 15) || (((uintptr_t)levels) & 15))
    return -1;
  if ((ref_pitch & 1) || (((uintptr_t)ref_uv) & 1)) return -1;
  Geo g{W, H, RW, RH, (W + 15) / 16, (H + 15) / 16};
  const int T = b200enc_tuned(B200ENC_TUNE_PCHAIN_MBS_PER_CTA) > 0 ? b200enc_tuned(B200ENC_TUNE_PCHAIN_MBS_PER_CTA) : 1;
  p_mb_kernel<false><<<dim3((g.mbw + T - 1) / T, g.mbh), dim3(96, T), T * sizeof(PShared), (cudaStream_t)stream>>>(
      cur_y, cur_uv, cur_pitch, ref_y, ref_uv, ref_pitch, g, qp, (const MV*)mv, levels, dc, nz, pred_mode, rec_y,
      rec_uv, rec_pitch, BatchTab{}, t8, t8_flags);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// The P chain of every P macroblock of a batch (n = the compact P count).
int b200enc_p_frame_batch_launch(const BatchTab& bt, int n, cudaStream_t st) {
  if (n <= 0) return 0;
  p_mb_kernel<true><<<n, dim3(96, 1), sizeof(PShared), st>>>(nullptr, nullptr, 0, nullptr, nullptr, 0, Geo{}, 0,
                                                             nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                                             nullptr, 0, bt);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
