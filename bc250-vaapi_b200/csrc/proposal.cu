// proposal.cu - the learned motion-proposal network: candidate preparation,
// BF16 forward/backward on the tcgen05 GEMM, loss, Adam, candidate selection
// and exact integer re-scoring with the plain search's refine.
//
// The reference has no learned part; this stands in for most of the
// exhaustive search of me.cu. Per MB:
//   candidates  c0 = the previous frame's co-located MV, c1..c8 its eight
//               neighbours (raster order of the 3x3 block), c9 = zero; each
//               rounded to integer pels, clamped to [-(R-2), R-2]
//   features    exact SAD at every candidate, candidate offsets, duplicate
//               flags, the previous frame's SADs, block gradients
//   network     input 2 x 16x16 (current luma, residual against c0), four
//               2x2 stride-2 convolutions of 32 channels (16x16 -> 1x1), then
//               fc 96 -> 64 -> 16: logits of the 10 candidates and "none"
//               (the full-search winner is within +-2 pels of no candidate),
//               a no-residual logit, 4 unused
//   decision    the 4 most probable distinct candidates; if their summed
//               probability is under the confidence threshold the MB falls
//               back to full search, otherwise every integer MV within +-2 of
//               them is scored exactly with the full search's cost and
//               tie-break key, and the winner gets the same half/quarter-pel
//               refine. Whenever the full-search winner is inside those
//               windows the result equals the plain search's bit for bit.
//
// Layout: conv rows are kept in Morton order inside each MB (row m of layer
// l covers grid cell (x, y) with x = even bits of m, y = odd bits), so the
// four rows of every 2x2 patch are consecutive and each 2x2 stride-2
// convolution is a plain GEMM over the previous output viewed as
// [rows/4][4*channels]; the backward pass needs no im2col or col2im either.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "me_common.cuh"
#include "proposal.cuh"

namespace b200enc {

// ---------------------------------------------------------------------------
// Preparation: candidates, their SADs, the network input and side features.
// 64 threads (two warps) per MB.
// ---------------------------------------------------------------------------
// Word i (0..7) of an 8-word register window, by selects (no local memory).
__device__ __forceinline__ uint32_t pick8(const uint32_t (&w)[8], int i) {
  const uint32_t lo = (i & 2) ? ((i & 1) ? w[3] : w[2]) : ((i & 1) ? w[1] : w[0]);
  const uint32_t hi = (i & 2) ? ((i & 1) ? w[7] : w[6]) : ((i & 1) ? w[5] : w[4]);
  return (i & 4) ? hi : lo;
}

// BATCH: one CTA per compact P macroblock of a batch (the buffers of b are
// indexed by that compact index); geometry, planes, history and the early-out
// threshold come from the macroblock's stream.
template <bool BATCH>
__global__ void __launch_bounds__(64) lp_prepare_kernel(const uint8_t* __restrict__ cur_, int cur_pitch_,
                                                        const uint8_t* __restrict__ ref_, int ref_pitch_, Geo g_,
                                                        const MV* __restrict__ prev_, int R, int zero_thresh_,
                                                        LpBuf b, BatchTab bt) {
  __shared__ uint32_t scw[64];   // current MB, 16 rows x 4 words (clamped to W, H)
  __shared__ uint32_t rfw[64];   // reference block at candidate 0
  __shared__ int scx[kCand], scy[kCand];
  __shared__ uint32_t ssad[kCand], sprev[9];
  __shared__ uint32_t sgrad[2][2];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int mb = blockIdx.x;  // index of the buffers of b
  const uint8_t* cur = cur_;
  const uint8_t* ref = ref_;
  int cur_pitch = cur_pitch_, ref_pitch = ref_pitch_, zero_thresh = zero_thresh_;
  Geo g = g_;
  const MV* prev = prev_;
  int lmb = mb;  // the macroblock within its frame
  if (BATCH) {
    const int k = bt.p_mbs.find(mb);
    const BatchStream& st = bt.p_mbs.stream(k);
    lmb = mb - bt.p_mbs.prefix[k];
    g = st.g;
    if (lmb >= g.mbw * g.mbh) {
      // padding of the compact index: the zero inputs a tile's rows past the
      // end of a frame have, and an early-out state so nothing selects it
      *reinterpret_cast<uint4*>(b.x0 + ((size_t)mb * 64 + tid) * 8) = make_uint4(0u, 0u, 0u, 0u);
      b.f[(size_t)mb * kFIn + 32 + tid] = __float2bfloat16_rn(0.f);
      if (tid < kCand) {
        b.cand[mb * kCand + tid] = 0;
        b.cand_sad[mb * kCand + tid] = 0u;
      }
      if (tid == 0) b.state[mb] = kStEarly;
      return;
    }
    cur = st.cur_y;
    cur_pitch = st.cur_pitch;
    ref = st.ref_y;
    ref_pitch = st.rec_pitch;
    zero_thresh = st.zero_thresh;
    prev = st.has_hist ? st.mv_prev : nullptr;
  }
  const int mby = lmb / g.mbw, mbx = lmb - mby * g.mbw;
  const int X = mbx * 16, Y = mby * 16;
  {
    const int r = tid >> 2, w = tid & 3;
    const uint8_t* cp = cur + (size_t)clampi(Y + r, 0, g.H - 1) * cur_pitch;
    const int gx = X + 4 * w;
    uint32_t v;
    if (gx + 3 < g.W) {
      v = __ldg(reinterpret_cast<const uint32_t*>(cp + gx));
    } else {
      v = (uint32_t)__ldg(cp + min(gx, g.W - 1)) | ((uint32_t)__ldg(cp + min(gx + 1, g.W - 1)) << 8) |
          ((uint32_t)__ldg(cp + min(gx + 2, g.W - 1)) << 16) | ((uint32_t)__ldg(cp + min(gx + 3, g.W - 1)) << 24);
    }
    scw[tid] = v;
  }
  if (tid < kCand) {
    int cx = 0, cy = 0;
    if (tid < 9 && prev) {
      const int nx = clampi(mbx + kNb[tid][0], 0, g.mbw - 1), ny = clampi(mby + kNb[tid][1], 0, g.mbh - 1);
      const MV m = prev[ny * g.mbw + nx];
      cx = clampi((m.mvx + 2) >> 2, -(R - 2), R - 2);
      cy = clampi((m.mvy + 2) >> 2, -(R - 2), R - 2);
      sprev[tid] = m.sad;
    } else if (tid < 9) {
      sprev[tid] = 0;
    }
    scx[tid] = cx;
    scy[tid] = cy;
    ssad[tid] = 0;
  }
  __syncthreads();

  // exact SAD at each candidate: one warp per candidate, two lanes per
  // reference row (lane pair h = 0, 1 scores the row's bytes 8h .. 8h+7),
  // summed over the warp by shuffles. Where the plane's base and pitch are
  // 16-byte aligned and the row's 32-byte aligned window lies inside the
  // picture, each lane loads one 16-byte half of the window and the pair
  // swaps halves: one load instruction covers 16 rows, where five word loads
  // per row touched ~5x the L1 wavefronts. Other rows take clamped word
  // loads (the same bytes).
  {
    const bool vec = ((ref_pitch & 15) == 0) && ((reinterpret_cast<uintptr_t>(ref) & 15) == 0);
    const int r = lane >> 1, h = lane & 1;
    for (int c = warp; c < kCand; c += 2) {
      const int x0 = X + scx[c];
      const uint8_t* rp = ref + (size_t)clampi(Y + r + scy[c], 0, g.RH - 1) * ref_pitch;
      const int x16 = x0 & ~15;
      uint32_t w0, w1, w2;  // the words at (x0 & ~3) + 8h + 0, 4, 8
      int shft;
      if (vec && x16 >= 0 && x16 + 32 <= g.RW) {  // warp-uniform
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(rp + x16 + 16 * h));
        const uint32_t o0 = __shfl_xor_sync(0xffffffffu, v.x, 1), o1 = __shfl_xor_sync(0xffffffffu, v.y, 1);
        const uint32_t o2 = __shfl_xor_sync(0xffffffffu, v.z, 1), o3 = __shfl_xor_sync(0xffffffffu, v.w, 1);
        const uint32_t win[8] = {h ? o0 : v.x, h ? o1 : v.y, h ? o2 : v.z, h ? o3 : v.w,
                                 h ? v.x : o0, h ? v.y : o1, h ? v.z : o2, h ? v.w : o3};
        const int q = ((x0 - x16) >> 2) + 2 * h;  // 0..5
        w0 = pick8(win, q);
        w1 = pick8(win, q + 1);
        w2 = pick8(win, q + 2);
        shft = (x0 & 3) * 8;
      } else {
        const int xa = x0 & ~3;
        w0 = load_word_clamped(rp, xa + 8 * h, g.RW);
        w1 = load_word_clamped(rp, xa + 8 * h + 4, g.RW);
        w2 = load_word_clamped(rp, xa + 8 * h + 8, g.RW);
        shft = (x0 - xa) * 8;
      }
      const uint32_t rv0 = __funnelshift_r(w0, w1, shft), rv1 = __funnelshift_r(w1, w2, shft);
      uint32_t sad = sad4_acc(rv0, scw[r * 4 + 2 * h], 0u);
      sad = sad4_acc(rv1, scw[r * 4 + 2 * h + 1], sad);
      if (c == 0) {
        rfw[r * 4 + 2 * h] = rv0;
        rfw[r * 4 + 2 * h + 1] = rv1;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) sad += __shfl_xor_sync(0xffffffffu, sad, o);
      if (lane == 0) ssad[c] = sad;
    }
  }
  // block gradients: sum |horizontal| and |vertical| neighbour differences
  {
    const uint8_t* sc = reinterpret_cast<const uint8_t*>(scw);
    uint32_t gh = 0, gv = 0;
    for (int i = tid; i < 256; i += 64) {
      const int y = i >> 4, x = i & 15;
      if (x < 15) gh += (uint32_t)abs((int)sc[i] - (int)sc[i + 1]);
      if (y < 15) gv += (uint32_t)abs((int)sc[i] - (int)sc[i + 16]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      gh += __shfl_xor_sync(0xffffffffu, gh, o);
      gv += __shfl_xor_sync(0xffffffffu, gv, o);
    }
    if (lane == 0) {
      sgrad[warp][0] = gh;
      sgrad[warp][1] = gv;
    }
  }
  __syncthreads();

  uint32_t dup = 0;
  uint32_t smin = 0xffffffffu;
  for (int c = 0; c < kCand; ++c) {
    for (int d = 0; d < c; ++d)
      if (scx[d] == scx[c] && scy[d] == scy[c]) {
        dup |= 1u << c;
        break;
      }
    smin = min(smin, ssad[c]);
  }
  const bool early = zero_thresh >= 0 && ssad[9] <= (uint32_t)zero_thresh;

  // network input: row m (Morton cell (ox, oy) of the 8x8 grid) holds the
  // 2x2 pels (dy, dx) x (current, residual against c0) at k = (dy*2+dx)*2+ch
  {
    const uint8_t* sc = reinterpret_cast<const uint8_t*>(scw);
    const uint8_t* r0 = reinterpret_cast<const uint8_t*>(rfw);
    const int m = tid, ox = morton_x(m), oy = morton_y(m);
    __align__(16) __nv_bfloat16 v[8];
#pragma unroll
    for (int dy = 0; dy < 2; ++dy)
#pragma unroll
      for (int dx = 0; dx < 2; ++dx) {
        const int i = (2 * oy + dy) * 16 + 2 * ox + dx;
        const int cv = sc[i], rv = r0[i];
        v[(dy * 2 + dx) * 2 + 0] = __float2bfloat16_rn((float)(cv - 128) * 0.015625f);
        v[(dy * 2 + dx) * 2 + 1] = __float2bfloat16_rn((float)(cv - rv) * 0.015625f);
      }
    *reinterpret_cast<uint4*>(b.x0 + ((size_t)mb * 64 + m) * 8) = *reinterpret_cast<const uint4*>(v);
  }
  // side features (64), columns 32..95 of the fc1 input row
  {
    const int t = tid;
    float f = 0.f;
    if (t < 10) f = (float)min(ssad[t], 32767u) * (1.f / 4096.f);
    else if (t < 20) f = (float)min(ssad[t - 10] - smin, 32767u) * (1.f / 4096.f);
    else if (t < 30) f = (float)(scx[t - 20] - scx[0]) * 0.125f;
    else if (t < 40) f = (float)(scy[t - 30] - scy[0]) * 0.125f;
    else if (t < 50) f = (dup >> (t - 40)) & 1u ? 1.f : 0.f;
    else if (t < 59) f = (float)min(sprev[t - 50], 32767u) * (1.f / 4096.f);
    else if (t == 59) f = (float)abs(scx[0]) * 0.03125f;
    else if (t == 60) f = (float)abs(scy[0]) * 0.03125f;
    else if (t == 61) f = (float)(sgrad[0][0] + sgrad[1][0]) / 7680.f;
    else if (t == 62) f = (float)(sgrad[0][1] + sgrad[1][1]) / 7680.f;
    else f = prev ? 0.f : 1.f;
    b.f[(size_t)mb * kFIn + 32 + t] = __float2bfloat16_rn(f);
  }
  if (tid < kCand) {
    b.cand[mb * kCand + tid] = (scy[tid] << 16) | (scx[tid] & 0xffff);
    b.cand_sad[mb * kCand + tid] = ssad[tid];
  }
  if (tid == 0) b.state[mb] = (early ? kStEarly : 0u) | (prev ? 0u : kStNoHist) | (dup << 8);
}

__global__ void lp_select_kernel(int mbs, LpBuf b, int mode, float param, int lambda, MV* __restrict__ mv_out) {
  const int mb = blockIdx.x * blockDim.x + threadIdx.x;
  if (mb >= mbs) return;
  float z[kOut];
  if (mode == 1)
    for (int j = 0; j < kOut; ++j) z[j] = b.logits[(size_t)mb * kOut + j];
  lp_select_one(mb, mbs, b, mode, param, lambda, z, mv_out);
}

// ---------------------------------------------------------------------------
// Exact re-scoring of the selected candidates' +-2 windows, then the refine.
// 64 threads per MB, persistent over the learned list.
// ---------------------------------------------------------------------------
// One warp per MB, four independent warps per block; every warp walks the
// learned list on its own and synchronises only itself.
// Candidate k's patch covers rows cy-5 .. cy+21 and 32 bytes starting
// exactly at byte X+cx-5 (the staging shifts each row into place): the +-2
// search window plus the refine's -3..+19 reach around any winner inside
// that window, so the refine reads no global memory. With the row starting
// at that byte, integer offset ox of the window begins at byte 3+ox of every
// patch row whatever the candidate, so the search's byte shifts are
// compile-time constants. One lane scores a whole row of the window (the 5
// offsets at one oy) from three 64-bit loads of the patch row and one
// 128-bit load of the current row per macroblock row. Rows are kPatchStride
// = 10 words apart (8 used) and candidates kCandWords = 274 words: the 20
// lanes' 64-bit loads of one instruction then fall on distinct banks in
// each half-warp phase.
constexpr int kPatchRows = 27, kPatchStride = 10, kCandWords = 274;  // 8 words used per row
struct RescoreWarp {
  alignas(16) uint32_t patch[4 * kCandWords];
  alignas(16) uint32_t cur[64];
  int ccx[4], ccy[4];
  RefineSimd rf;
};

// BATCH: the listed macroblocks are compact P indices of a batch; each
// takes its stream's geometry, planes and lambda, and its vector goes to
// mv_out at the compact index.
template <bool BATCH>
__global__ void __launch_bounds__(128) lp_rescore_kernel(const uint8_t* __restrict__ cur_, int cur_pitch_,
                                                         const uint8_t* __restrict__ ref_, int ref_pitch_, Geo g_,
                                                         int R, int lambda_, int mbs, LpBuf b,
                                                         MV* __restrict__ mv_out, BatchTab bt) {
  __shared__ RescoreWarp shw[4];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  RescoreWarp& sh = shw[wid];
  const int n = b.counters[0];
  const int SIDE = 2 * R + 1;
  for (int li = blockIdx.x * 4 + wid; li < n; li += gridDim.x * 4) {
    const int mb = b.lists[li];
    const uint8_t* cur = cur_;
    const uint8_t* ref = ref_;
    int cur_pitch = cur_pitch_, ref_pitch = ref_pitch_, lambda = lambda_;
    Geo g = g_;
    int lmb = mb;
    if (BATCH) {
      const int k = bt.p_mbs.find(mb);
      const BatchStream& st = bt.p_mbs.stream(k);
      lmb = mb - bt.p_mbs.prefix[k];
      g = st.g;
      cur = st.cur_y;
      cur_pitch = st.cur_pitch;
      ref = st.ref_y;
      ref_pitch = st.rec_pitch;
      lambda = st.lambda;
    }
    const int mby = lmb / g.mbw, mbx = lmb - mby * g.mbw;
    const int X = mbx * 16, Y = mby * 16;
    const uint32_t sel = b.sel[mb];
    int valid = 0;
    if (lane < 4) {
      const int c = (int)((sel >> (8 * lane)) & 0xffu);
      if (c < kCand) {
        const int32_t p = b.cand[mb * kCand + c];
        sh.ccx[lane] = cand_x(p);
        sh.ccy[lane] = cand_y(p);
        valid = 1;
      }
    }
    // selected candidates occupy the low slots (the selection fills them in order)
    const int nk = __popc(__ballot_sync(0xffffffffu, valid) & 0xfu);
    __syncwarp();
    const bool ref_vec = ((ref_pitch & 15) == 0) && ((reinterpret_cast<uintptr_t>(ref) & 15) == 0);
    // stage the current MB (clamped to W, H) and the candidate patches
    for (int i = lane; i < 64; i += 32) {
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
    // one patch row (8 words from s = X+cx-5) per lane and pass: three
    // 16-byte loads from s & ~15 where the 48 bytes lie inside the row of a
    // 16-byte aligned plane, else the clamped word loads from s & ~3; the
    // words are then shifted by (s & 3) bytes into place
    for (int t = lane; t < nk * kPatchRows; t += 32) {
      const int k = t / kPatchRows, r = t - k * kPatchRows;
      const int s0 = X + sh.ccx[k] - 5, xa16 = s0 & ~15, sft = (s0 & 3) * 8;
      const uint8_t* rp = ref + (size_t)clampi(Y + sh.ccy[k] - 5 + r, 0, g.RH - 1) * ref_pitch;
      uint32_t* dst = sh.patch + k * kCandWords + r * kPatchStride;
      uint32_t v[9];
      if (ref_vec && xa16 >= 0 && xa16 + 48 <= g.RW) {
        const uint4 a = __ldg(reinterpret_cast<const uint4*>(rp + xa16));
        const uint4 b2 = __ldg(reinterpret_cast<const uint4*>(rp + xa16 + 16));
        const uint4 c = __ldg(reinterpret_cast<const uint4*>(rp + xa16 + 32));
        const uint32_t u[12] = {a.x, a.y, a.z, a.w, b2.x, b2.y, b2.z, b2.w, c.x, c.y, c.z, c.w};
        switch ((s0 - xa16) >> 2) {  // word w of the aligned row is u[q + w]
          case 0:
#pragma unroll
            for (int w = 0; w < 9; ++w) v[w] = u[w];
            break;
          case 1:
#pragma unroll
            for (int w = 0; w < 9; ++w) v[w] = u[w + 1];
            break;
          case 2:
#pragma unroll
            for (int w = 0; w < 9; ++w) v[w] = u[w + 2];
            break;
          default:
#pragma unroll
            for (int w = 0; w < 9; ++w) v[w] = u[w + 3];
            break;
        }
      } else {
#pragma unroll
        for (int w = 0; w < 9; ++w) v[w] = load_word_clamped(rp, (s0 & ~3) + 4 * w, g.RW);
      }
#pragma unroll
      for (int w = 0; w < 8; w += 2)
        *reinterpret_cast<uint2*>(dst + w) =
            make_uint2(__funnelshift_r(v[w], v[w + 1], sft), __funnelshift_r(v[w + 1], v[w + 2], sft));
    }
    __syncwarp();

    // the 25 integer offsets of each candidate: lane k*5+oy scores the row
    // of offsets (ox = 0..4, oy) of candidate k
    uint32_t best = 0xffffffffu;
    if (lane < nk * 5) {
      const int k = lane / 5, oy = lane - 5 * k;
      const uint32_t* prow = sh.patch + k * kCandWords + (oy + 3) * kPatchStride;
      uint32_t s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0;
#pragma unroll 4
      for (int r = 0; r < 16; ++r) {
        const uint2 p0 = *reinterpret_cast<const uint2*>(prow + r * kPatchStride);
        const uint2 p1 = *reinterpret_cast<const uint2*>(prow + r * kPatchStride + 2);
        const uint2 p2 = *reinterpret_cast<const uint2*>(prow + r * kPatchStride + 4);
        const uint4 c = *reinterpret_cast<const uint4*>(sh.cur + 4 * r);
        const uint32_t u0 = p0.x, u1 = p0.y, u2 = p1.x, u3 = p1.y, u4 = p2.x, u5 = p2.y;
        s0 = sad4_acc(__funnelshift_r(u0, u1, 24), c.x, s0);  // ox 0: bytes 3..18
        s0 = sad4_acc(__funnelshift_r(u1, u2, 24), c.y, s0);
        s0 = sad4_acc(__funnelshift_r(u2, u3, 24), c.z, s0);
        s0 = sad4_acc(__funnelshift_r(u3, u4, 24), c.w, s0);
        s1 = sad4_acc(u1, c.x, s1);  // ox 1: bytes 4..19
        s1 = sad4_acc(u2, c.y, s1);
        s1 = sad4_acc(u3, c.z, s1);
        s1 = sad4_acc(u4, c.w, s1);
        s2 = sad4_acc(__funnelshift_r(u1, u2, 8), c.x, s2);  // ox 2: bytes 5..20
        s2 = sad4_acc(__funnelshift_r(u2, u3, 8), c.y, s2);
        s2 = sad4_acc(__funnelshift_r(u3, u4, 8), c.z, s2);
        s2 = sad4_acc(__funnelshift_r(u4, u5, 8), c.w, s2);
        s3 = sad4_acc(__funnelshift_r(u1, u2, 16), c.x, s3);  // ox 3: bytes 6..21
        s3 = sad4_acc(__funnelshift_r(u2, u3, 16), c.y, s3);
        s3 = sad4_acc(__funnelshift_r(u3, u4, 16), c.z, s3);
        s3 = sad4_acc(__funnelshift_r(u4, u5, 16), c.w, s3);
        s4 = sad4_acc(__funnelshift_r(u1, u2, 24), c.x, s4);  // ox 4: bytes 7..22
        s4 = sad4_acc(__funnelshift_r(u2, u3, 24), c.y, s4);
        s4 = sad4_acc(__funnelshift_r(u3, u4, 24), c.z, s4);
        s4 = sad4_acc(__funnelshift_r(u4, u5, 24), c.w, s4);
      }
      const int dy = sh.ccy[k] - 2 + oy, dx0 = sh.ccx[k] - 2;
      const uint32_t sads[5] = {s0, s1, s2, s3, s4};
#pragma unroll
      for (int ox = 0; ox < 5; ++ox) {
        const int dx = dx0 + ox;
        const uint32_t cost = sads[ox] + (uint32_t)lambda * (uint32_t)(abs(dx) + abs(dy));
        best = min(best, (cost << 14) | (uint32_t)((dy + R) * SIDE + (dx + R)));
      }
    }
    best = __reduce_min_sync(0xffffffffu, best);
    const int idx = (int)(best & 0x3fffu);
    const int mx = idx % SIDE - R, my = idx / SIDE - R;
    const uint32_t int_sad = (best >> 14) - (uint32_t)lambda * (uint32_t)(abs(mx) + abs(my));

    // the refine reads the patch of the first candidate whose window holds
    // the winner (clamped like the full search's window)
    int kw = 0;
    for (int k = nk - 1; k >= 0; --k)
      if (abs(mx - sh.ccx[k]) <= 2 && abs(my - sh.ccy[k]) <= 2) kw = k;
    const uint8_t* pb8 = reinterpret_cast<const uint8_t*>(sh.patch + kw * kCandWords);
    const int row0 = my - (sh.ccy[kw] - 5), col0 = mx - sh.ccx[kw] + 5;
    int qx, qy;
    const uint32_t bsad =
        qpel_refine_warp_simd(sh.rf, pb8, kPatchStride * 4, row0, col0, sh.cur, int_sad, &qx, &qy);
    if (lane == 0) mv_out[mb] = MV{4 * mx + qx, 4 * my + qy, bsad, 0u};
    __syncwarp();  // the warp's shared memory is restaged for its next MB
  }
}

// ---------------------------------------------------------------------------
// Training: labels, loss + logit gradient, ReLU backward, bias sums, Adam.
// ---------------------------------------------------------------------------
// Target of an MB from the full search's log word (B200ENC_ME_LOG_INTEGER):
// the set (bit mask over the 11 classes) of distinct candidates whose +-2
// window holds the integer winner, or {10} ("none") if there is none;
// early-outs and MBs without history get weight 0. The no-residual target
// is 1 iff all 24 nz words of the plain encode are 0.
__global__ void lp_label_kernel(int mbs, LpBuf b, const MV* __restrict__ logged, const uint32_t* __restrict__ nz,
                                int* __restrict__ label, float* __restrict__ norez, float* __restrict__ weight) {
  const int mb = blockIdx.x * blockDim.x + threadIdx.x;
  if (mb >= mbs) return;
  const uint32_t st = b.state[mb];
  const uint32_t w = logged[mb].pad;
  const bool valid = (w >> 31) && !((w >> 30) & 1u) && !(st & (kStEarly | kStNoHist));
  int lab = 0;
  if (valid) {
    const int dx = (int)(w & 0xffu) - 128, dy = (int)((w >> 8) & 0xffu) - 128;
    const uint32_t dup = (st >> 8) & 0x3ffu;
    for (int c = 0; c < kCand; ++c) {
      if ((dup >> c) & 1u) continue;
      const int32_t p = b.cand[mb * kCand + c];
      if (abs(dx - cand_x(p)) <= 2 && abs(dy - cand_y(p)) <= 2) lab |= 1 << c;
    }
  }
  if (lab == 0) lab = 1 << (kClasses - 1);
  bool zero_res = true;
  if (nz)
    for (int k = 0; k < 24; ++k) zero_res = zero_res && nz[mb * 24 + k] == 0u;
  label[mb] = lab;
  norez[mb] = zero_res ? 1.f : 0.f;
  weight[mb] = valid ? 1.f : 0.f;
  if (valid) atomicAdd(&b.counters[2], 1);
}

// Mean over valid samples of -log(probability mass of the target set under
// the 11-way masked softmax) + 0.5 BCE(no-residual); writes dLoss/dlogits
// (p_j - [j in set] p_j / P_set for the set term) as BF16 and adds the loss
// sum to *loss.
__global__ void lp_loss_kernel(int mbs, LpBuf b, const int* __restrict__ label, const float* __restrict__ norez,
                               const float* __restrict__ weight, __nv_bfloat16* __restrict__ g5,
                               float* __restrict__ loss) {
  const int mb = blockIdx.x * blockDim.x + threadIdx.x;
  if (mb >= mbs) return;
  const float nval = (float)max(b.counters[2], 1);
  const float w = weight[mb] / nval;
  const uint32_t dup = (b.state[mb] >> 8) & 0x3ffu;
  float z[kClasses], p[kClasses];
  for (int j = 0; j < kClasses; ++j) z[j] = b.logits[(size_t)mb * kOut + j];
  masked_softmax(z, dup, p);
  const uint32_t y = (uint32_t)label[mb];
  float pset = 0.f;
  for (int j = 0; j < kClasses; ++j)
    if ((y >> j) & 1u) pset += p[j];
  pset = fmaxf(pset, 1e-30f);
  const float zs = b.logits[(size_t)mb * kOut + 11];
  const float ps = 1.f / (1.f + expf(-zs));
  const float t = norez[mb];
  __nv_bfloat16* gr = g5 + (size_t)mb * kOut;
  for (int j = 0; j < kClasses; ++j)
    gr[j] = __float2bfloat16_rn(w * (p[j] - (((y >> j) & 1u) ? p[j] / pset : 0.f)));
  gr[11] = __float2bfloat16_rn(w * 0.5f * (ps - t));
  for (int j = 12; j < kOut; ++j) gr[j] = __float2bfloat16_rn(0.f);
  if (weight[mb] > 0.f) {
    // softplus forms of -log p_y and the BCE
    const float ce = -logf(pset);
    const float bce = fmaxf(zs, 0.f) - zs * t + log1pf(expf(-fabsf(zs)));
    atomicAdd(loss, w * (ce + 0.5f * bce));
  }
}

// G[r][c] = bf16(dA[r*lda + c] * (Y[r*ldy + c] > 0)), c < C
__global__ void lp_relu_bwd_kernel(long long rows, int C, const float* __restrict__ dA, int lda,
                                   const __nv_bfloat16* __restrict__ Y, int ldy, __nv_bfloat16* __restrict__ G) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * C) return;
  const long long r = i / C;
  const int c = (int)(i - r * C);
  const float y = __bfloat162float(Y[r * ldy + c]);
  G[i] = __float2bfloat16_rn(y > 0.f ? dA[r * lda + c] : 0.f);
}

// out[c] += sum over rows of G[r][c] (G is [rows][C] BF16)
__global__ void lp_colsum_kernel(long long rows, int C, const __nv_bfloat16* __restrict__ G, float* __restrict__ out) {
  const int c = threadIdx.x % C;
  const int lanes = blockDim.x / C;
  const int sub = threadIdx.x / C;
  if (sub >= lanes) return;
  float s = 0.f;
  for (long long r = (long long)blockIdx.x * lanes + sub; r < rows; r += (long long)gridDim.x * lanes)
    s += __bfloat162float(G[r * C + c]);
  atomicAdd(out + c, s);
}

__global__ void lp_adam_kernel(int n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                               float* __restrict__ v, __nv_bfloat16* __restrict__ pb, float lr_t, float b1, float b2,
                               float eps) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float pi = p[i] - lr_t * mi / (sqrtf(vi) + eps);
  p[i] = pi;
  pb[i] = __float2bfloat16_rn(pi);
}

__global__ void lp_to_bf16_kernel(int n, const float* __restrict__ p, __nv_bfloat16* __restrict__ pb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) pb[i] = __float2bfloat16_rn(p[i]);
}

// ---------------------------------------------------------------------------
// Host runtime
// ---------------------------------------------------------------------------
struct Proposal {
  int max_mbs = 0;
  float *params = nullptr, *grads = nullptr, *adam_m = nullptr, *adam_v = nullptr;
  __nv_bfloat16* wb = nullptr;
  uint8_t* w8 = nullptr;  // FP8 weights + scales (lp_net8_launch), rebuilt when w8_stale
  bool w8_stale = true;
  LpBuf b{};
  uint32_t* err = nullptr;
  // the fallback full search runs on a side stream, concurrently with the
  // re-scoring of the learned MBs (disjoint MBs of the same MV field)
  cudaStream_t side = nullptr;
  cudaEvent_t ev_sel = nullptr, ev_fb = nullptr;
  // training buffers (allocated on first use)
  bool train_ready = false;
  int *label = nullptr;
  float *norez = nullptr, *weight = nullptr, *loss = nullptr;
  __nv_bfloat16 *g5 = nullptr, *g4 = nullptr, *g3 = nullptr, *g2 = nullptr, *g1 = nullptr, *g0 = nullptr;
  float *da5 = nullptr, *da4 = nullptr, *da3 = nullptr, *da2 = nullptr, *da1 = nullptr;
  std::vector<void*> allocs;

  template <class T>
  bool alloc(T** p, size_t count) {
    void* q = nullptr;
    if (cudaMalloc(&q, count * sizeof(T) + 16) != cudaSuccess) return false;
    allocs.push_back(q);
    *p = static_cast<T*>(q);
    return true;
  }
  ~Proposal() {
    if (side) cudaStreamSynchronize(side);
    for (void* p : allocs) cudaFree(p);
    if (ev_sel) cudaEventDestroy(ev_sel);
    if (ev_fb) cudaEventDestroy(ev_fb);
    if (side) cudaStreamDestroy(side);
  }
  bool init(int mbs) {
    max_mbs = mbs;
    const size_t B = (size_t)mbs;
    return alloc(&params, kParams) && alloc(&grads, kParams) && alloc(&adam_m, kParams) && alloc(&adam_v, kParams) &&
           alloc(&wb, kParams) && alloc(&w8, kNet8PackBytes) && alloc(&b.x0, B * 64 * 8) && alloc(&b.y1, B * 64 * 32) && alloc(&b.y2, B * 16 * 32) &&
           alloc(&b.y3, B * 4 * 32) && alloc(&b.f, B * kFIn) && alloc(&b.h, B * 64) && alloc(&b.logits, B * kOut) &&
           alloc(&b.cand, B * kCand) && alloc(&b.cand_sad, B * kCand) && alloc(&b.state, B) && alloc(&b.sel, B) &&
           alloc(&b.p_norez, B) && alloc(&b.lists, 2 * B) && alloc(&b.counters, 8) && alloc(&err, 1) &&
           cudaMemset(params, 0, kParams * 4) == cudaSuccess && cudaMemset(adam_m, 0, kParams * 4) == cudaSuccess &&
           cudaMemset(adam_v, 0, kParams * 4) == cudaSuccess && cudaMemset(wb, 0, kParams * 2) == cudaSuccess &&
           cudaMemset(b.counters, 0, 32) == cudaSuccess && cudaMemset(err, 0, 4) == cudaSuccess &&
           cudaMemset(b.f, 0, B * kFIn * 2) == cudaSuccess &&
           cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking) == cudaSuccess &&
           cudaEventCreateWithFlags(&ev_sel, cudaEventDisableTiming) == cudaSuccess &&
           cudaEventCreateWithFlags(&ev_fb, cudaEventDisableTiming) == cudaSuccess;
  }
  bool init_train() {
    if (train_ready) return true;
    const size_t B = (size_t)max_mbs;
    train_ready = alloc(&label, B) && alloc(&norez, B) && alloc(&weight, B) && alloc(&loss, 1) &&
                  alloc(&g5, B * kOut) && alloc(&g4, B * 64) && alloc(&g3, B * 32) && alloc(&g2, B * 128) &&
                  alloc(&g1, B * 512) && alloc(&g0, B * 2048) && alloc(&da5, B * 64) && alloc(&da4, B * kFIn) &&
                  alloc(&da3, B * 128) && alloc(&da2, B * 512) && alloc(&da1, B * 2048) &&
                  cudaMemset(loss, 0, 4) == cudaSuccess;
    return train_ready;
  }
  const __nv_bfloat16* W(int l) const { return wb + layer_woff(l); }
  const float* bias(int l) const { return params + layer_boff(l); }
  float* gW(int l) const { return grads + layer_woff(l); }
  float* gb(int l) const { return grads + layer_boff(l); }
};

// SHA-256 (FIPS 180-4) for checkpoint integrity.
struct Sha256 {
  uint32_t h[8] = {0x6a09e667u, 0xbb67ae85u, 0x3c6ef372u, 0xa54ff53au, 0x510e527fu, 0x9b05688cu, 0x1f83d9abu, 0x5be0cd19u};
  uint8_t buf[64];
  size_t nbuf = 0;
  uint64_t total = 0;
  static uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }
  void block(const uint8_t* p) {
    static const uint32_t k[64] = {
        0x428a2f98u, 0x71374491u, 0xb5c0fbcfu, 0xe9b5dba5u, 0x3956c25bu, 0x59f111f1u, 0x923f82a4u, 0xab1c5ed5u,
        0xd807aa98u, 0x12835b01u, 0x243185beu, 0x550c7dc3u, 0x72be5d74u, 0x80deb1feu, 0x9bdc06a7u, 0xc19bf174u,
        0xe49b69c1u, 0xefbe4786u, 0x0fc19dc6u, 0x240ca1ccu, 0x2de92c6fu, 0x4a7484aau, 0x5cb0a9dcu, 0x76f988dau,
        0x983e5152u, 0xa831c66du, 0xb00327c8u, 0xbf597fc7u, 0xc6e00bf3u, 0xd5a79147u, 0x06ca6351u, 0x14292967u,
        0x27b70a85u, 0x2e1b2138u, 0x4d2c6dfcu, 0x53380d13u, 0x650a7354u, 0x766a0abbu, 0x81c2c92eu, 0x92722c85u,
        0xa2bfe8a1u, 0xa81a664bu, 0xc24b8b70u, 0xc76c51a3u, 0xd192e819u, 0xd6990624u, 0xf40e3585u, 0x106aa070u,
        0x19a4c116u, 0x1e376c08u, 0x2748774cu, 0x34b0bcb5u, 0x391c0cb3u, 0x4ed8aa4au, 0x5b9cca4fu, 0x682e6ff3u,
        0x748f82eeu, 0x78a5636fu, 0x84c87814u, 0x8cc70208u, 0x90befffau, 0xa4506cebu, 0xbef9a3f7u, 0xc67178f2u};
    uint32_t w[64];
    for (int i = 0; i < 16; ++i)
      w[i] = (uint32_t)p[4 * i] << 24 | (uint32_t)p[4 * i + 1] << 16 | (uint32_t)p[4 * i + 2] << 8 | p[4 * i + 3];
    for (int i = 16; i < 64; ++i) {
      const uint32_t s0 = rotr(w[i - 15], 7) ^ rotr(w[i - 15], 18) ^ (w[i - 15] >> 3);
      const uint32_t s1 = rotr(w[i - 2], 17) ^ rotr(w[i - 2], 19) ^ (w[i - 2] >> 10);
      w[i] = w[i - 16] + s0 + w[i - 7] + s1;
    }
    uint32_t a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5], g = h[6], hh = h[7];
    for (int i = 0; i < 64; ++i) {
      const uint32_t t1 = hh + (rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25)) + ((e & f) ^ (~e & g)) + k[i] + w[i];
      const uint32_t t2 = (rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22)) + ((a & b) ^ (a & c) ^ (b & c));
      hh = g; g = f; f = e; e = d + t1; d = c; c = b; b = a; a = t1 + t2;
    }
    h[0] += a; h[1] += b; h[2] += c; h[3] += d; h[4] += e; h[5] += f; h[6] += g; h[7] += hh;
  }
  void update(const uint8_t* p, size_t n) {
    total += n;
    while (n) {
      const size_t take = std::min(n, 64 - nbuf);
      memcpy(buf + nbuf, p, take);
      nbuf += take; p += take; n -= take;
      if (nbuf == 64) { block(buf); nbuf = 0; }
    }
  }
  void finish(uint8_t out[32]) {
    const uint64_t bits = total * 8;
    const uint8_t one = 0x80, zero = 0;
    update(&one, 1);
    while (nbuf != 56) update(&zero, 1);
    uint8_t len[8];
    for (int i = 0; i < 8; ++i) len[i] = (uint8_t)(bits >> (56 - 8 * i));
    update(len, 8);
    for (int i = 0; i < 8; ++i)
      for (int j = 0; j < 4; ++j) out[4 * i + j] = (uint8_t)(h[i] >> (24 - 8 * j));
  }
};

static int splits_for(long long k) {
  const long long chunks = (k + 63) / 64;
  long long s = chunks / 16;
  return (int)(s < 1 ? 1 : (s > 255 ? 255 : s));
}

#define LP_TRY(x) \
  do {            \
    if ((x) != 0) return -1; \
  } while (0)

static int lp_forward(Proposal* P, int mbs, cudaStream_t st) {
  const long long B = mbs;
  const int relu_bf = B200ENC_GEMM_RELU | B200ENC_GEMM_OUT_BF16;
  void* s = (void*)st;
  LP_TRY(b200enc_gemm_bf16((int)(B * 64), 32, 8, P->b.x0, 8, 1, P->W(0), 8, 1, (float*)P->b.y1, 32, P->bias(0),
                           relu_bf, P->err, s));
  LP_TRY(b200enc_gemm_bf16((int)(B * 16), 32, 128, P->b.y1, 128, 1, P->W(1), 128, 1, (float*)P->b.y2, 32,
                           P->bias(1), relu_bf, P->err, s));
  LP_TRY(b200enc_gemm_bf16((int)(B * 4), 32, 128, P->b.y2, 128, 1, P->W(2), 128, 1, (float*)P->b.y3, 32, P->bias(2),
                           relu_bf, P->err, s));
  LP_TRY(b200enc_gemm_bf16((int)B, 32, 128, P->b.y3, 128, 1, P->W(3), 128, 1, (float*)P->b.f, kFIn, P->bias(3),
                           relu_bf, P->err, s));
  LP_TRY(b200enc_gemm_bf16((int)B, 64, kFIn, P->b.f, kFIn, 1, P->W(4), kFIn, 1, (float*)P->b.h, 64, P->bias(4),
                           relu_bf, P->err, s));
  LP_TRY(b200enc_gemm_bf16((int)B, kOut, 64, P->b.h, 64, 1, P->W(5), 64, 1, P->b.logits, kOut, P->bias(5), 0, P->err,
                           s));
  return 0;
}

// Gradient of one layer given its BF16 output gradient G [rows][out]:
// dW += G^T A (split K over the rows), db += column sums of G, and, when dA
// is non-null, dA = G W (FP32, [rows][in]).
static int lp_layer_bwd(Proposal* P, int l, long long rows, const __nv_bfloat16* G, const __nv_bfloat16* A, int lda,
                        float* dA, cudaStream_t st) {
  const int in = layer_in(l), out = layer_out(l);
  void* s = (void*)st;
  LP_TRY(b200enc_gemm_bf16(out, in, (int)rows, G, 1, out, A, 1, lda, P->gW(l), in, nullptr,
                           B200ENC_GEMM_SPLITK(splits_for(rows)), P->err, s));
  const int lanes = 256 / out;
  long long blocks = (rows + lanes * 64 - 1) / (lanes * 64);
  if (blocks > 1184) blocks = 1184;
  if (blocks < 1) blocks = 1;
  lp_colsum_kernel<<<(int)blocks, lanes * out, 0, st>>>(rows, out, G, P->gb(l));
  if (dA) LP_TRY(b200enc_gemm_bf16((int)rows, in, out, G, out, 1, P->W(l), 1, in, dA, in, nullptr, 0, P->err, s));
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

static void relu_bwd(long long rows, int C, const float* dA, int lda, const __nv_bfloat16* Y, int ldy,
                     __nv_bfloat16* G, cudaStream_t st) {
  const long long n = rows * C;
  lp_relu_bwd_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(rows, C, dA, lda, Y, ldy, G);
}

static int lp_backward(Proposal* P, int mbs, cudaStream_t st) {
  const long long B = mbs;
  if (cudaMemsetAsync(P->grads, 0, kParams * 4, st) != cudaSuccess) return -1;
  lp_loss_kernel<<<(mbs + 127) / 128, 128, 0, st>>>(mbs, P->b, P->label, P->norez, P->weight, P->g5, P->loss);
  LP_TRY(lp_layer_bwd(P, 5, B, P->g5, P->b.h, 64, P->da5, st));
  relu_bwd(B, 64, P->da5, 64, P->b.h, 64, P->g4, st);
  LP_TRY(lp_layer_bwd(P, 4, B, P->g4, P->b.f, kFIn, P->da4, st));
  relu_bwd(B, 32, P->da4, kFIn, P->b.f, kFIn, P->g3, st);
  LP_TRY(lp_layer_bwd(P, 3, B, P->g3, P->b.y3, 128, P->da3, st));
  relu_bwd(B * 4, 32, P->da3, 32, P->b.y3, 32, P->g2, st);
  LP_TRY(lp_layer_bwd(P, 2, B * 4, P->g2, P->b.y2, 128, P->da2, st));
  relu_bwd(B * 16, 32, P->da2, 32, P->b.y2, 32, P->g1, st);
  LP_TRY(lp_layer_bwd(P, 1, B * 16, P->g1, P->b.y1, 128, P->da1, st));
  relu_bwd(B * 64, 32, P->da1, 32, P->b.y1, 32, P->g0, st);
  LP_TRY(lp_layer_bwd(P, 0, B * 64, P->g0, P->b.x0, 8, nullptr, st));
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace b200enc

using namespace b200enc;

extern "C" {

int b200enc_proposal_num_params(void) { return kParams; }

void* b200enc_proposal_create(int max_mbs) {
  if (max_mbs <= 0 || max_mbs > (1 << 20)) return nullptr;
  Proposal* P = new (std::nothrow) Proposal();
  if (!P) return nullptr;
  if (!P->init(max_mbs)) {
    delete P;
    return nullptr;
  }
  return P;
}

void b200enc_proposal_destroy(void* h) { delete static_cast<Proposal*>(h); }

int b200enc_proposal_set_params(void* h, const float* host_params, int n) {
  Proposal* P = static_cast<Proposal*>(h);
  if (!P || !host_params || n != kParams) return -1;
  if (cudaMemcpy(P->params, host_params, kParams * 4, cudaMemcpyHostToDevice) != cudaSuccess) return -1;
  P->w8_stale = true;
  lp_to_bf16_kernel<<<(kParams + 255) / 256, 256>>>(kParams, P->params, P->wb);
  return cudaDeviceSynchronize() == cudaSuccess ? 0 : -1;
}

// Loads the parameters of a checkpoint file written by b200enc.proposal
// (magic "B2PN", version 1, little-endian header n/step/meta length/has-Adam,
// meta JSON, FP32 parameters, optional Adam moments, SHA-256 trailer).
// Returns -2 on a checksum or format mismatch, -1 on I/O or device errors.
int b200enc_proposal_load(void* h, const char* path) {
  Proposal* P = static_cast<Proposal*>(h);
  if (!P || !path) return -1;
  FILE* f = fopen(path, "rb");
  if (!f) return -1;
  std::vector<uint8_t> data;
  uint8_t tmp[65536];
  size_t n;
  while ((n = fread(tmp, 1, sizeof(tmp), f)) > 0) data.insert(data.end(), tmp, tmp + n);
  fclose(f);
  if (data.size() < 24 + 32) return -2;
  const size_t body = data.size() - 32;
  Sha256 sh;
  sh.update(data.data(), body);
  uint8_t dig[32];
  sh.finish(dig);
  if (memcmp(dig, data.data() + body, 32) != 0 || memcmp(data.data(), "B2PN", 4) != 0) return -2;
  uint32_t hdr[5];
  memcpy(hdr, data.data() + 4, 20);
  if (hdr[0] != 1 || hdr[1] != (uint32_t)kParams) return -2;
  const size_t off = 24 + (size_t)hdr[3];
  if (off + (size_t)kParams * 4 > body) return -2;
  std::vector<float> params(kParams);
  memcpy(params.data(), data.data() + off, (size_t)kParams * 4);
  return b200enc_proposal_set_params(h, params.data(), kParams);
}

int b200enc_proposal_get_params(void* h, float* host_params, int n) {
  Proposal* P = static_cast<Proposal*>(h);
  if (!P || !host_params || n != kParams) return -1;
  return cudaMemcpy(host_params, P->params, kParams * 4, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -1;
}

int b200enc_proposal_prepare(void* h, const uint8_t* cur_y, int cur_pitch, const uint8_t* ref_y, int ref_pitch,
                             int W, int H, int RW, int RH, const void* prev_mv, int range, int zero_thresh,
                             void* stream) {
  Proposal* P = static_cast<Proposal*>(h);
  if (!P || !cur_y || !ref_y || W <= 0 || H <= 0 || RW <= 0 || RH <= 0) return -1;
  if (range != 16 && range != 32) return -1;
  Geo g{W, H, RW, RH, (W + 15) / 16, (H + 15) / 16};
  const int mbs = g.mbw * g.mbh;
  if (mbs > P->max_mbs) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  if (cudaMemsetAsync(P->b.counters, 0, 32, st) != cudaSuccess) return -1;
  lp_prepare_kernel<false><<<mbs, 64, 0, st>>>(cur_y, cur_pitch, ref_y, ref_pitch, g, (const MV*)prev_mv, range,
                                               zero_thresh, P->b, BatchTab{});
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int b200enc_proposal_forward(void* h, int mbs, void* stream) {
  Proposal* P = static_cast<Proposal*>(h);
  if (!P || mbs <= 0 || mbs > P->max_mbs) return -1;
  return lp_forward(P, mbs, (cudaStream_t)stream);
}

int b200enc_proposal_labels(void* h, int mbs, const void* logged_mv, const uint32_t* nz, void* stream) {
  Proposal* P = static_cast<Proposal*>(h);
  if (!P || mbs <= 0 || mbs > P->max_mbs || !logged_mv || !P->init_train()) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  lp_label_kernel<<<(mbs + 127) / 128, 128, 0, st>>>(mbs, P->b, (const MV*)logged_mv, nz, P->label, P->norez,
                                                     P->weight);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int b200enc_proposal_backward(void* h, int mbs, void* stream) {
  Proposal* P = static_cast<Proposal*>(h);
  if (!P || mbs <= 0 || mbs > P->max_mbs || !P->init_train()) return -1;
  return lp_backward(P, mbs, (cudaStream_t)stream);
}

int b200enc_proposal_adam(void* h, float lr, float beta1, float beta2, float eps, int step, void* stream) {
  Proposal* P = static_cast<Proposal*>(h);
  if (!P || step < 1) return -1;
  const double c1 = 1.0 - std::pow((double)beta1, step), c2 = 1.0 - std::pow((double)beta2, step);
  const float lr_t = (float)(lr * std::sqrt(c2) / c1);
  P->w8_stale = true;
  lp_adam_kernel<<<(kParams + 255) / 256, 256, 0, (cudaStream_t)stream>>>(kParams, P->params, P->grads, P->adam_m,
                                                                         P->adam_v, P->wb, lr_t, beta1, beta2, eps);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int b200enc_proposal_train_step(void* h, int mbs, float lr, int step, void* stream) {
  if (b200enc_proposal_forward(h, mbs, stream) != 0) return -1;
  if (b200enc_proposal_backward(h, mbs, stream) != 0) return -1;
  return b200enc_proposal_adam(h, lr, 0.9f, 0.999f, 1e-8f, step, stream);
}

int b200enc_proposal_me(void* h, const uint8_t* cur_y, int cur_pitch, const uint8_t* ref_y, int ref_pitch, int W,
                        int H, int RW, int RH, const void* prev_mv, int range, int lambda, int zero_thresh, int mode,
                        float param, void* mv_out, void* stream) {
  Proposal* P = static_cast<Proposal*>(h);
  if (!P || !mv_out || (mode < 1 || mode > 3)) return -1;
  if (!prev_mv)  // no motion history: the plain search
    return b200enc_me_full_search(cur_y, cur_pitch, ref_y, ref_pitch, W, H, RW, RH, range, lambda, zero_thresh,
                                  mv_out, stream);
  if (lambda < 0 || lambda > 1023) return -1;
  if ((cur_pitch & 3) || (ref_pitch & 3) || (((uintptr_t)cur_y) & 3) || (((uintptr_t)ref_y) & 3)) return -1;
  if (b200enc_proposal_prepare(h, cur_y, cur_pitch, ref_y, ref_pitch, W, H, RW, RH, prev_mv, range, zero_thresh,
                               stream) != 0)
    return -1;
  Geo g{W, H, RW, RH, (W + 15) / 16, (H + 15) / 16};
  const int mbs = g.mbw * g.mbh;
  cudaStream_t st = (cudaStream_t)stream;
  if (mode == 1) {
    if (lp_net_launch(mbs, P->b, P->wb, P->params, param, lambda, (MV*)mv_out, P->err, st) != 0) return -1;
  } else if (mode == 3) {
    if (lp_net8_launch(mbs, P->b, P->params, P->w8, &P->w8_stale, param, lambda, (MV*)mv_out, P->err, st) != 0)
      return -1;
  } else {
    lp_select_kernel<<<(mbs + 127) / 128, 128, 0, st>>>(mbs, P->b, mode, param, lambda, (MV*)mv_out);
  }
  // fork: the fallback full search on the side stream, the re-scoring here
  if (cudaEventRecord(P->ev_sel, st) != cudaSuccess || cudaStreamWaitEvent(P->side, P->ev_sel, 0) != cudaSuccess)
    return -1;
  const int rc = b200enc_me_full_search_ex(cur_y, cur_pitch, ref_y, ref_pitch, W, H, RW, RH, range, lambda,
                                           zero_thresh, mv_out, P->b.lists + mbs, P->b.counters + 1, mbs, 0,
                                           (void*)P->side);
  int sms = 148, dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int per_sm = b200enc_tuned(B200ENC_TUNE_RESCORE_CTAS_PER_SM) > 0 ? b200enc_tuned(B200ENC_TUNE_RESCORE_CTAS_PER_SM) : 8;
  lp_rescore_kernel<false><<<std::max(1, std::min((mbs + 3) / 4, per_sm * sms)), 128, 0, st>>>(
      cur_y, cur_pitch, ref_y, ref_pitch, g, range, lambda, mbs, P->b, (MV*)mv_out, BatchTab{});
  // join
  if (cudaEventRecord(P->ev_fb, P->side) != cudaSuccess || cudaStreamWaitEvent(st, P->ev_fb, 0) != cudaSuccess)
    return -1;
  return (rc == 0 && cudaGetLastError() == cudaSuccess) ? 0 : -1;
}

// Device pointers of the runtime's tensors, for tests and the training
// driver: 0 params f32, 1 grads f32, 2 x0, 3 y1, 4 y2, 5 y3, 6 f, 7 h (bf16),
// 8 logits f32, 9 cand, 10 cand_sad, 11 state, 12 sel, 13 p_norez,
// 14 lists, 15 counters, 16 label, 17 norez target, 18 weight, 19 loss, 20 err.
int b200enc_proposal_tensor(void* h, int which, void** ptr, size_t* bytes) {
  Proposal* P = static_cast<Proposal*>(h);
  if (!P || !ptr || !bytes) return -1;
  const size_t B = (size_t)P->max_mbs;
  if (which >= 16 && !P->init_train()) return -1;
  switch (which) {
    case 0: *ptr = P->params; *bytes = kParams * 4; break;
    case 1: *ptr = P->grads; *bytes = kParams * 4; break;
    case 2: *ptr = P->b.x0; *bytes = B * 64 * 8 * 2; break;
    case 3: *ptr = P->b.y1; *bytes = B * 64 * 32 * 2; break;
    case 4: *ptr = P->b.y2; *bytes = B * 16 * 32 * 2; break;
    case 5: *ptr = P->b.y3; *bytes = B * 4 * 32 * 2; break;
    case 6: *ptr = P->b.f; *bytes = B * kFIn * 2; break;
    case 7: *ptr = P->b.h; *bytes = B * 64 * 2; break;
    case 8: *ptr = P->b.logits; *bytes = B * kOut * 4; break;
    case 9: *ptr = P->b.cand; *bytes = B * kCand * 4; break;
    case 10: *ptr = P->b.cand_sad; *bytes = B * kCand * 4; break;
    case 11: *ptr = P->b.state; *bytes = B * 4; break;
    case 12: *ptr = P->b.sel; *bytes = B * 4; break;
    case 13: *ptr = P->b.p_norez; *bytes = B * 4; break;
    case 14: *ptr = P->b.lists; *bytes = 2 * B * 4; break;
    case 15: *ptr = P->b.counters; *bytes = 32; break;
    case 16: *ptr = P->label; *bytes = B * 4; break;
    case 17: *ptr = P->norez; *bytes = B * 4; break;
    case 18: *ptr = P->weight; *bytes = B * 4; break;
    case 19: *ptr = P->loss; *bytes = 4; break;
    case 20: *ptr = P->err; *bytes = 4; break;
    default: return -1;
  }
  return 0;
}

}  // extern "C"

// The learned form over every P macroblock of a batch (n = the compact P
// count; modes 1 and 3): preparation, the network with its selection, the
// fallback full search (list mode, side stream) and the re-scoring, as
// b200enc_proposal_me does for one frame; every vector lands in bt.mvc.
int b200enc_proposal_me_batch(void* h, const BatchTab& bt, int n, int range, int lambda, int mode, float param,
                              cudaStream_t st) {
  Proposal* P = static_cast<Proposal*>(h);
  if (!P || n <= 0 || n > P->max_mbs || (mode != 1 && mode != 3) || (range != 16 && range != 32)) return -1;
  if (cudaMemsetAsync(P->b.counters, 0, 32, st) != cudaSuccess) return -1;
  lp_prepare_kernel<true><<<n, 64, 0, st>>>(nullptr, 0, nullptr, 0, Geo{}, nullptr, range, 0, P->b, bt);
  if (mode == 1) {
    if (lp_net_launch(n, P->b, P->wb, P->params, param, lambda, bt.mvc, P->err, st) != 0) return -1;
  } else {
    if (lp_net8_launch(n, P->b, P->params, P->w8, &P->w8_stale, param, lambda, bt.mvc, P->err, st) != 0) return -1;
  }
  int sms = 148, dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaEventRecord(P->ev_sel, st) != cudaSuccess || cudaStreamWaitEvent(P->side, P->ev_sel, 0) != cudaSuccess)
    return -1;
  const int fb_sm = b200enc_tuned(B200ENC_TUNE_FALLBACK_CTAS_PER_SM) > 0 ? b200enc_tuned(B200ENC_TUNE_FALLBACK_CTAS_PER_SM) : 8;
  const int rc = b200enc_me_batch_launch(bt, range, P->b.lists + n, P->b.counters + 1, std::min(n, fb_sm * sms),
                                         P->side);
  const int rs_sm = b200enc_tuned(B200ENC_TUNE_RESCORE_CTAS_PER_SM) > 0 ? b200enc_tuned(B200ENC_TUNE_RESCORE_CTAS_PER_SM) : 8;
  lp_rescore_kernel<true><<<std::max(1, std::min((n + 3) / 4, rs_sm * sms)), 128, 0, st>>>(
      nullptr, 0, nullptr, 0, Geo{}, range, 0, n, P->b, bt.mvc, bt);
  if (cudaEventRecord(P->ev_fb, P->side) != cudaSuccess || cudaStreamWaitEvent(st, P->ev_fb, 0) != cudaSuccess)
    return -1;
  return (rc == 0 && cudaGetLastError() == cudaSuccess) ? 0 : -1;
}

