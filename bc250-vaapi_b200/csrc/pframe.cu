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

namespace b200enc {

struct PShared {
  uint8_t lp[21][24];      // luma reference patch, origin (ix0-2, iy0-2)
  uint8_t cp[9][20];       // chroma reference patch (NV12 pairs), 9 x 9
  int16_t pred[24][16];    // prediction per block, raster within block
  int16_t res[24][16];     // residual
  int32_t tsm[24][16];     // transpose scratch per block
  alignas(16) int16_t lev[24][16];  // quantized levels (for the coalesced store)
  int32_t cdc[8];          // pre-quant chroma DC coefficients
  int32_t dcval[8];        // dequantized chroma DC per chroma block
  alignas(16) uint8_t ry[16][16];  // reconstructed luma
  alignas(16) uint8_t ruv[8][16];  // reconstructed chroma (NV12)
};

__device__ __forceinline__ int hraw_p(const uint8_t (*lp)[24], int x, int y) {
  // horizontal 6-tap centred between integer columns x and x+1 of row y
  const uint8_t* r = lp[y + 2];
  return r[x] - 5 * r[x + 1] + 20 * r[x + 2] + 20 * r[x + 3] - 5 * r[x + 4] + r[x + 5];
}
__device__ __forceinline__ int vraw_p(const uint8_t (*lp)[24], int x, int y) {
  return lp[y][x + 2] - 5 * lp[y + 1][x + 2] + 20 * lp[y + 2][x + 2] + 20 * lp[y + 3][x + 2] -
         5 * lp[y + 4][x + 2] + lp[y + 5][x + 2];
}

// Luma quarter-pel sample (residual_predict.comp:263-298) for block-relative
// pixel (x, y) whose integer anchor is patch (x+2, y+2).
__device__ __forceinline__ int mc_luma(const uint8_t (*lp)[24], int x, int y, int fx, int fy) {
  const int G = lp[y + 2][x + 2];
  if (!(fx | fy)) return G;
  const int phase = fy * 4 + fx;
  auto B = [&](int xx, int yy) { return clip1((hraw_p(lp, xx, yy) + 16) >> 5); };
  auto Hh = [&](int xx, int yy) { return clip1((vraw_p(lp, xx, yy) + 16) >> 5); };
  auto J = [&]() {
    const int j1 = hraw_p(lp, x, y - 2) - 5 * hraw_p(lp, x, y - 1) + 20 * hraw_p(lp, x, y) +
                   20 * hraw_p(lp, x, y + 1) - 5 * hraw_p(lp, x, y + 2) + hraw_p(lp, x, y + 3);
    return clip1((j1 + 512) >> 10);
  };
  switch (phase) {
    case 1: return (G + B(x, y) + 1) >> 1;
    case 2: return B(x, y);
    case 3: return (B(x, y) + lp[y + 2][x + 3] + 1) >> 1;
    case 4: return (G + Hh(x, y) + 1) >> 1;
    case 5: return (B(x, y) + Hh(x, y) + 1) >> 1;
    case 6: return (B(x, y) + J() + 1) >> 1;
    case 7: return (B(x, y) + Hh(x + 1, y) + 1) >> 1;
    case 8: return Hh(x, y);
    case 9: return (Hh(x, y) + J() + 1) >> 1;
    case 10: return J();
    case 11: return (J() + Hh(x + 1, y) + 1) >> 1;
    case 12: return (Hh(x, y) + lp[y + 3][x + 2] + 1) >> 1;
    case 13: return (Hh(x, y) + B(x, y + 1) + 1) >> 1;
    case 14: return (J() + B(x, y + 1) + 1) >> 1;
    default: return (Hh(x + 1, y) + B(x, y + 1) + 1) >> 1;
  }
}

__global__ void __launch_bounds__(96) p_mb_kernel(const uint8_t* __restrict__ cur_y, const uint8_t* __restrict__ cur_uv,
                                                  int cur_pitch, const uint8_t* __restrict__ ref_y,
                                                  const uint8_t* __restrict__ ref_uv, int ref_pitch, Geo g, int qp,
                                                  const MV* __restrict__ mvs, int16_t* __restrict__ levels,
                                                  int32_t* __restrict__ dc, uint32_t* __restrict__ nzm,
                                                  uint32_t* __restrict__ pred_mode, uint8_t* __restrict__ rec_y,
                                                  uint8_t* __restrict__ rec_uv, int rec_pitch) {
  __shared__ PShared s;
  const int tid = threadIdx.x;
  const int mbx = blockIdx.x, mby = blockIdx.y, mb = mby * g.mbw + mbx;
  const int X = mbx * 16, Y = mby * 16, Xc = X >> 1, Yc = Y >> 1;
  const MV mv = mvs[mb];
  const int ix0 = X + (mv.mvx >> 2), iy0 = Y + (mv.mvy >> 2), fx = mv.mvx & 3, fy = mv.mvy & 3;
  const int ixc = Xc + (mv.mvx >> 3), iyc = Yc + (mv.mvy >> 3), fxc = mv.mvx & 7, fyc = mv.mvy & 7;
  const int cmx = g.RW / 2 - 1, cmy = g.RH / 2 - 1;

  // ---- stage reference patches (clamped) --------------------------------
  for (int i = tid; i < 21 * 21; i += 96) {
    const int py = i / 21, px = i - py * 21;
    s.lp[py][px] = __ldg(ref_y + (size_t)clampi(iy0 - 2 + py, 0, g.RH - 1) * ref_pitch + clampi(ix0 - 2 + px, 0, g.RW - 1));
  }
  for (int i = tid; i < 9 * 9; i += 96) {
    const int py = i / 9, px = i - py * 9;
    const uint16_t v = __ldg(reinterpret_cast<const uint16_t*>(ref_uv + (size_t)clampi(iyc + py, 0, cmy) * ref_pitch +
                                                               2 * clampi(ixc + px, 0, cmx)));
    s.cp[py][2 * px] = (uint8_t)(v & 0xff);
    s.cp[py][2 * px + 1] = (uint8_t)(v >> 8);
  }
  __syncthreads();

  // ---- prediction + residual --------------------------------------------
  for (int i = tid; i < 256; i += 96) {
    const int x = i & 15, y = i >> 4;
    const int pv = mc_luma(s.lp, x, y, fx, fy);
    const int src = __ldg(cur_y + (size_t)clampi(Y + y, 0, g.H - 1) * cur_pitch + clampi(X + x, 0, g.W - 1));
    const int blk = (y >> 2) * 4 + (x >> 2), pos = (y & 3) * 4 + (x & 3);
    s.pred[blk][pos] = (int16_t)pv;
    s.res[blk][pos] = (int16_t)(src - pv);
  }
  for (int i = tid; i < 128; i += 96) {
    const int pl = i >> 6, x = i & 7, y = (i >> 3) & 7;
    const int A = s.cp[y][2 * x + pl], B = s.cp[y][2 * x + 2 + pl];
    const int C = s.cp[y + 1][2 * x + pl], D = s.cp[y + 1][2 * x + 2 + pl];
    const int pv = ((8 - fxc) * (8 - fyc) * A + fxc * (8 - fyc) * B + (8 - fxc) * fyc * C + fxc * fyc * D + 32) >> 6;
    const int src = __ldg(cur_uv + (size_t)clampi(Yc + y, 0, g.H / 2 - 1) * cur_pitch + 2 * clampi(Xc + x, 0, g.W / 2 - 1) + pl);
    const int blk = 16 + 4 * pl + (y >> 2) * 2 + (x >> 2), pos = (y & 3) * 4 + (x & 3);
    s.pred[blk][pos] = (int16_t)pv;
    s.res[blk][pos] = (int16_t)(src - pv);
  }
  __syncthreads();

  // ---- forward + quant: quad (b, r) owns row r of block b ---------------
  const int b = tid >> 2, r = tid & 3;
  const bool luma = b < 16;
  const QP q = make_qp(luma ? qp : chroma_qp(qp), false);
  int x[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) x[i] = s.res[b][4 * r + i];
  quad_forward(x, r, s.tsm[b]);  // x[i] = coef[i][r]
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
    nzm[(size_t)mb * 24 + b] = nz;
    dc[(size_t)mb * 24 + b] = x[0];
    if (!luma) s.cdc[b - 16] = x[0];
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
  int d[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) d[i] = dequant_ac(s.lev[b][4 * r + i], 4 * r + i, q);
  if (r == 0) {
    if (!luma) d[0] = s.dcval[b - 16];
    d[0] += 32;
  }
  quad_inverse(d, r, s.tsm[b]);  // d[i] = res[i][r]
  if (luma) {
    const int bx = b & 3, by = b >> 2;
#pragma unroll
    for (int i = 0; i < 4; ++i) s.ry[4 * by + i][4 * bx + r] = (uint8_t)clip1(s.pred[b][4 * i + r] + d[i]);
  } else {
    const int pl = (b - 16) >> 2, sub = (b - 16) & 3;
#pragma unroll
    for (int i = 0; i < 4; ++i)
      s.ruv[4 * (sub >> 1) + i][2 * (4 * (sub & 1) + r) + pl] = (uint8_t)clip1(s.pred[b][4 * i + r] + d[i]);
  }
  __syncthreads();

  // ---- coalesced stores ---------------------------------------------------
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
  }
}

}  // namespace b200enc

using namespace b200enc;

extern "C" int b200enc_p_frame(const uint8_t* cur_y, const uint8_t* cur_uv, int cur_pitch, const uint8_t* ref_y,
                               const uint8_t* ref_uv, int ref_pitch, int W, int H, int RW, int RH, int qp,
                               const void* mv, int16_t* levels, int32_t* dc, uint32_t* nz, uint32_t* pred_mode,
                               uint8_t* rec_y, uint8_t* rec_uv, int rec_pitch, void* stream) {
  if (!cur_y || !cur_uv || !ref_y || !ref_uv || !mv || !levels || !dc || !nz || !pred_mode || !rec_y || !rec_uv)
    return -1;
  if (qp < 0 || qp > 51 || W <= 0 || H <= 0 || RW <= 1 || RH <= 1) return -1;
  if ((rec_pitch & 15) || (((uintptr_t)rec_y) & 15) || (((uintptr_t)rec_uv) & 15) || (((uintptr_t)levels) & 15))
    return -1;
  if ((ref_pitch & 1) || (((uintptr_t)ref_uv) & 1)) return -1;
  Geo g{W, H, RW, RH, (W + 15) / 16, (H + 15) / 16};
  p_mb_kernel<<<dim3(g.mbw, g.mbh), 96, 0, (cudaStream_t)stream>>>(cur_y, cur_uv, cur_pitch, ref_y, ref_uv, ref_pitch,
                                                                   g, qp, (const MV*)mv, levels, dc, nz, pred_mode,
                                                                   rec_y, rec_uv, rec_pitch);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
