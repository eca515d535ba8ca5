// deblock.cu - spec deblocking (H.264 clause 8.7) as a persistent wavefront.
//
// The reference shader (A1/shaders/deblock_filter.comp) filters luma only,
// treats bS 4 like bS 3, and runs all edges of a direction at once, so
// neighbouring edges race on the samples they share; no decoder reproduces
// it. This kernel reproduces the reference's C deblocker
// (A1/src/h264_deblock.c:263-368) exactly: macroblocks in raster order
// semantics, vertical edges then horizontal, luma and chroma, bS 0-4 with
// the strong filter.
//
// Raster order matters only between macroblocks whose sample footprints
// overlap: (x-1,y), (x-1,y-1), (x,y-1) and (x+1,y-1) before (x,y). So each
// CTA (one warp) takes a macroblock row by ticket and, before macroblock x,
// waits until row y-1 has published progress >= min(x+2, mbw): the
// classic 2-macroblock-skew wavefront, which gives the raster result.
// Waits are bounded exactly as in the intra kernel.
//
// Per macroblock the warp stages a 20x20 luma tile (4-sample halo left and
// above) and the matching 10x20-byte NV12 chroma tile in shared memory;
// lanes 0-15 filter one luma line each and lanes 16-31 one chroma line
// (8 Cb + 8 Cr), first along rows across the vertical edges, then along
// columns across the horizontal ones.
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

constexpr int kTP = 20;  // tile pitch in bytes (luma and NV12 chroma)

// One luma line across one edge (clause 8.7.2.3 / 8.7.2.4).
__device__ __forceinline__ void filt_luma(uint8_t* q, int d, int bs, int alpha, int beta, int tc0) {
  const int p0 = q[-d], p1 = q[-2 * d], p2 = q[-3 * d], q0 = q[0], q1 = q[d], q2 = q[2 * d];
  if (abs(p0 - q0) >= alpha || abs(p1 - p0) >= beta || abs(q1 - q0) >= beta) return;
  const bool ap = abs(p2 - p0) < beta, aq = abs(q2 - q0) < beta;
  if (bs == 4) {
    const int p3 = q[-4 * d], q3 = q[3 * d];
    const bool small = abs(p0 - q0) < ((alpha >> 2) + 2);
    if (ap && small) {
      q[-d] = (uint8_t)((p2 + 2 * p1 + 2 * p0 + 2 * q0 + q1 + 4) >> 3);
      q[-2 * d] = (uint8_t)((p2 + p1 + p0 + q0 + 2) >> 2);
      q[-3 * d] = (uint8_t)((2 * p3 + 3 * p2 + p1 + p0 + q0 + 4) >> 3);
    } else {
      q[-d] = (uint8_t)((2 * p1 + p0 + q1 + 2) >> 2);
    }
    if (aq && small) {
      q[0] = (uint8_t)((q2 + 2 * q1 + 2 * q0 + 2 * p0 + p1 + 4) >> 3);
      q[d] = (uint8_t)((q2 + q1 + q0 + p0 + 2) >> 2);
      q[2 * d] = (uint8_t)((2 * q3 + 3 * q2 + q1 + q0 + p0 + 4) >> 3);
    } else {
      q[0] = (uint8_t)((2 * q1 + q0 + p1 + 2) >> 2);
    }
    return;
  }
  const int tc = tc0 + (ap ? 1 : 0) + (aq ? 1 : 0);
  const int delta = clampi(((q0 - p0) * 4 + (p1 - q1) + 4) >> 3, -tc, tc);
  if (ap) q[-2 * d] = (uint8_t)(p1 + clampi((p2 + ((p0 + q0 + 1) >> 1) - (p1 << 1)) >> 1, -tc0, tc0));
  if (aq) q[d] = (uint8_t)(q1 + clampi((q2 + ((p0 + q0 + 1) >> 1) - (q1 << 1)) >> 1, -tc0, tc0));
  q[-d] = (uint8_t)clip1(p0 + delta);
  q[0] = (uint8_t)clip1(q0 - delta);
}

// One chroma line (p1/q1 are never written).
__device__ __forceinline__ void filt_chroma(uint8_t* q, int d, int bs, int alpha, int beta, int tc0) {
  const int p0 = q[-d], p1 = q[-2 * d], q0 = q[0], q1 = q[d];
  if (abs(p0 - q0) >= alpha || abs(p1 - p0) >= beta || abs(q1 - q0) >= beta) return;
  if (bs == 4) {
    q[-d] = (uint8_t)((2 * p1 + p0 + q1 + 2) >> 2);
    q[0] = (uint8_t)((2 * q1 + q0 + p1 + 2) >> 2);
    return;
  }
  const int tc = tc0 + 1;
  const int delta = clampi(((q0 - p0) * 4 + (p1 - q1) + 4) >> 3, -tc, tc);
  q[-d] = (uint8_t)clip1(p0 + delta);
  q[0] = (uint8_t)clip1(q0 - delta);
}

struct DShared {
  alignas(16) uint8_t yt[20][kTP];
  alignas(16) uint8_t ct[10][kTP];
  uint8_t bsv[4][4];  // [edge][segment] vertical
  uint8_t bsh[4][4];  // [edge][segment] horizontal
  int row, abort_flag;
};

__global__ void __launch_bounds__(32) deblock_kernel(int mbw, int mbh, int qp, int is_intra,
                                                     const uint32_t* __restrict__ nzm, const MV* __restrict__ mvs,
                                                     uint8_t* rec_y, uint8_t* rec_uv, int rec_pitch,
                                                     uint32_t* scratch, uint32_t max_wait) {
  __shared__ DShared s;
  const Scratch sc{scratch};
  const int lane = threadIdx.x;
  const int qpc = chroma_qp(qp);
  const int al = kAlpha[qp], be = kBeta[qp], alc = kAlpha[qpc], bec = kBeta[qpc];
  const bool luma_on = al && be, chroma_on = alc && bec;

  for (;;) {
    if (lane == 0) {
      s.row = (int)atomicAdd(sc.ticket(), 1u);
      s.abort_flag = 0;
    }
    __syncwarp();
    const int my = s.row;
    if (my >= mbh) return;
    for (int mx = 0; mx < mbw; ++mx) {
      const int mb = my * mbw + mx;
      if (lane == 0 && my > 0) {
        const uint32_t need = (uint32_t)min(mx + 2, mbw);
        const uint32_t* pf = sc.progress(my - 1);
        bool ok = false;
        for (uint32_t it = 0; it < max_wait; ++it) {
          if (load_acquire(pf) >= need) { ok = true; break; }
          if (load_acquire(sc.err()) != 0u) break;
          if (it > 4) __nanosleep(32);
        }
        if (!ok) {
          if (atomicCAS(sc.err(), 0u, kErrWaitTimeout) == 0u) atomicExch(sc.err_detail(), 0x80000000u | (uint32_t)mb);
          s.abort_flag = 1;
        }
      }
      __syncwarp();
      if (s.abort_flag) return;

      // ---- stage tiles (L2 reads: neighbours were written by other CTAs) ----
      const int x0 = mx * 16 - 4;  // tile byte column origin (luma and NV12 chroma)
      for (int i = lane; i < 20 * 5; i += 32) {
        const int r = i / 5, w = i - r * 5, gy = my * 16 - 4 + r, gx = x0 + 4 * w;
        uint32_t v = 0;
        if (gy >= 0 && gx >= 0) v = __ldcg(reinterpret_cast<const uint32_t*>(rec_y + (size_t)gy * rec_pitch + gx));
        reinterpret_cast<uint32_t*>(s.yt[r])[w] = v;
      }
      for (int i = lane; i < 10 * 5; i += 32) {
        const int r = i / 5, w = i - r * 5, gy = my * 8 - 2 + r, gx = x0 + 4 * w;
        uint32_t v = 0;
        if (gy >= 0 && gx >= 0) v = __ldcg(reinterpret_cast<const uint32_t*>(rec_uv + (size_t)gy * rec_pitch + gx));
        reinterpret_cast<uint32_t*>(s.ct[r])[w] = v;
      }
      // ---- boundary strengths (clause 8.7.2.1) -------------------------
      {
        const int dir = lane >> 4, e = (lane >> 2) & 3, k = lane & 3;
        int bs = 0;
        const bool has_p = e > 0 || (dir == 0 ? mx > 0 : my > 0);
        if (has_p) {
          if (is_intra) {
            bs = e == 0 ? 4 : 3;
          } else {
            const int mbp = e ? mb : (dir == 0 ? mb - 1 : mb - mbw);
            const int bq = dir == 0 ? k * 4 + e : e * 4 + k;
            const int bp = e ? (dir == 0 ? bq - 1 : bq - 4) : (dir == 0 ? k * 4 + 3 : 12 + k);
            if ((__ldg(nzm + (size_t)mbp * 24 + bp) | __ldg(nzm + (size_t)mb * 24 + bq)) & 0xffffu) {
              bs = 2;
            } else if (e == 0) {
              const MV a = mvs[mbp], c = mvs[mb];
              bs = (abs(a.mvx - c.mvx) >= 4 || abs(a.mvy - c.mvy) >= 4) ? 1 : 0;
            }
          }
        }
        if (dir == 0) s.bsv[e][k] = (uint8_t)bs;
        else s.bsh[e][k] = (uint8_t)bs;
      }
      __syncwarp();

      // ---- vertical edges, left to right -------------------------------
      if (lane < 16) {
        if (luma_on) {
          uint8_t* line = s.yt[4 + lane];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int bs = s.bsv[e][lane >> 2];
            if (bs) filt_luma(line + 4 + 4 * e, 1, bs, al, be, bs < 4 ? kTc0[qp][bs - 1] : 0);
          }
        }
      } else if (chroma_on) {
        const int j = lane - 16, pl = j >> 3, i = j & 7;
        uint8_t* line = s.ct[2 + i];
#pragma unroll
        for (int e = 0; e < 4; e += 2) {
          const int bs = s.bsv[e][i >> 1];
          if (bs) filt_chroma(line + 2 * (2 + 2 * e) + pl, 2, bs, alc, bec, bs < 4 ? kTc0[qpc][bs - 1] : 0);
        }
      }
      __syncwarp();
      // ---- horizontal edges, top to bottom -----------------------------
      if (lane < 16) {
        if (luma_on) {
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int bs = s.bsh[e][lane >> 2];
            if (bs) filt_luma(&s.yt[4 + 4 * e][4 + lane], kTP, bs, al, be, bs < 4 ? kTc0[qp][bs - 1] : 0);
          }
        }
      } else if (chroma_on) {
        const int j = lane - 16, pl = j >> 3, i = j & 7;
#pragma unroll
        for (int e = 0; e < 4; e += 2) {
          const int bs = s.bsh[e][i >> 1];
          if (bs) filt_chroma(&s.ct[2 + 2 * e][2 * (2 + i) + pl], kTP, bs, alc, bec, bs < 4 ? kTc0[qpc][bs - 1] : 0);
        }
      }
      __syncwarp();

      // ---- write back everything but the unused top-left corner ---------
      for (int i = lane; i < 20 * 5; i += 32) {
        const int r = i / 5, w = i - r * 5, gy = my * 16 - 4 + r, gx = x0 + 4 * w;
        if (gy < 0 || gx < 0 || (r < 4 && w == 0)) continue;
        __stcg(reinterpret_cast<uint32_t*>(rec_y + (size_t)gy * rec_pitch + gx), reinterpret_cast<const uint32_t*>(s.yt[r])[w]);
      }
      for (int i = lane; i < 10 * 5; i += 32) {
        const int r = i / 5, w = i - r * 5, gy = my * 8 - 2 + r, gx = x0 + 4 * w;
        if (gy < 0 || gx < 0 || (r < 2 && w == 0)) continue;
        __stcg(reinterpret_cast<uint32_t*>(rec_uv + (size_t)gy * rec_pitch + gx), reinterpret_cast<const uint32_t*>(s.ct[r])[w]);
      }
      __threadfence();
      __syncwarp();
      if (lane == 0) store_release(sc.progress(my), (uint32_t)(mx + 1));
    }
  }
}

}  // namespace b200enc

using namespace b200enc;

static constexpr uint32_t kMaxWaitPollsDb = 1u << 22;

extern "C" int b200enc_deblock_launch(int mbw, int mbh, int qp, int is_intra, const uint32_t* nz, const void* mv,
                                      uint8_t* rec_y, uint8_t* rec_uv, int rec_pitch, uint32_t* scratch, int ctas,
                                      uint32_t max_wait, void* stream) {
  if (ctas <= 0 || ctas > mbh) ctas = mbh;
  deblock_kernel<<<ctas, 32, 0, (cudaStream_t)stream>>>(mbw, mbh, qp, is_intra, nz, (const MV*)mv, rec_y, rec_uv,
                                                        rec_pitch, scratch, max_wait);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int b200enc_deblock(int mbw, int mbh, int qp, int is_intra, const uint32_t* nz, const void* mv,
                               uint8_t* rec_y, uint8_t* rec_uv, int rec_pitch, void* scratch, size_t scratch_bytes,
                               int ctas, void* stream) {
  if (!nz || !mv || !rec_y || !rec_uv || !scratch || mbw <= 0 || mbh <= 0 || qp < 0 || qp > 51) return -1;
  if ((rec_pitch & 3) || (((uintptr_t)rec_y) & 3) || (((uintptr_t)rec_uv) & 3)) return -1;
  if (rec_pitch < mbw * 16) return -1;
  if (scratch_bytes < b200enc_wavefront_scratch_bytes(mbh)) return -1;
  if (cudaMemsetAsync(scratch, 0, b200enc_wavefront_scratch_bytes(mbh), (cudaStream_t)stream) != cudaSuccess) return -1;
  return b200enc_deblock_launch(mbw, mbh, qp, is_intra, nz, mv, rec_y, rec_uv, rec_pitch, (uint32_t*)scratch, ctas,
                                kMaxWaitPollsDb, stream);
}
