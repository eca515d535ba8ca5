// proposal.cuh - shared definitions of the learned motion-proposal kernels
// (proposal.cu: preparation, training, re-scoring; proposal_infer.cu: the
// fused inference network): network shape, parameter layout, the per-frame
// buffers and the candidate selection rule.
#pragma once
#include <cuda_bf16.h>

#include "b200enc_internal.h"
#include "common.cuh"

namespace b200enc {

constexpr int kCand = 10;
constexpr int kClasses = 11;  // candidates + none
constexpr int kOut = 16;
constexpr int kFeat = 64;
constexpr int kFIn = 96;  // fc1 input: 32 conv features + 64 side features
static_assert(kFIn == 32 + kFeat, "fc1 input = conv features + side features");
constexpr int kLayers = 6;
__host__ __device__ constexpr int layer_in(int l) { return l == 0 ? 8 : (l < 4 ? 128 : (l == 4 ? kFIn : 64)); }
__host__ __device__ constexpr int layer_out(int l) { return l < 4 ? 32 : (l == 4 ? 64 : kOut); }
__host__ __device__ constexpr int layer_woff(int l) {
  return l == 0 ? 0 : layer_woff(l - 1) + layer_out(l - 1) * layer_in(l - 1) + layer_out(l - 1);
}
__host__ __device__ constexpr int layer_boff(int l) { return layer_woff(l) + layer_out(l) * layer_in(l); }
constexpr int kParams = layer_boff(kLayers - 1) + layer_out(kLayers - 1);

// per-MB state word
constexpr uint32_t kStEarly = 1u, kStNoHist = 2u;  // dup mask in bits 8..17

__constant__ int8_t kNb[9][2] = {{0, 0}, {-1, -1}, {0, -1}, {1, -1}, {-1, 0}, {1, 0}, {-1, 1}, {0, 1}, {1, 1}};

struct LpBuf {
  __nv_bfloat16 *x0, *y1, *y2, *y3, *f, *h;
  float* logits;
  int32_t* cand;      // [mbs][10] packed (cy << 16) | (cx & 0xffff)
  uint32_t* cand_sad;  // [mbs][10]
  uint32_t* state;     // [mbs]
  uint32_t* sel;       // [mbs] 4 x int8 candidate indices (-1 unused)
  float* p_norez;      // [mbs]
  int* lists;          // learned [mbs], fallback [mbs]
  int* counters;       // [0] learned, [1] fallback, [2] valid training samples, [3] early-outs
};

__device__ __forceinline__ int morton_x(int m) { return (m & 1) | ((m >> 1) & 2) | ((m >> 2) & 4); }
__device__ __forceinline__ int morton_y(int m) { return ((m >> 1) & 1) | ((m >> 2) & 2) | ((m >> 3) & 4); }

__device__ __forceinline__ int cand_x(int32_t p) { return (int)(int16_t)(p & 0xffff); }
__device__ __forceinline__ int cand_y(int32_t p) { return p >> 16; }

__device__ __forceinline__ void masked_softmax(const float* z, uint32_t dup, float* p) {
  float mx = -INFINITY;
  for (int j = 0; j < kClasses; ++j)
    if (!((dup >> j) & 1u)) mx = fmaxf(mx, z[j]);
  float s = 0.f;
  for (int j = 0; j < kClasses; ++j) {
    p[j] = ((dup >> j) & 1u) ? 0.f : expf(z[j] - mx);
    s += p[j];
  }
  const float inv = 1.f / s;
  for (int j = 0; j < kClasses; ++j) p[j] *= inv;
}

// mode 1: the network's 4 most probable distinct candidates, falling back
// when their probability sum is under `param`. mode 2 (no network): the 4
// distinct candidates of lowest exact cost (SAD + lambda * |c|), falling
// back when that lowest cost exceeds param * 256 (param < 0: never).
__device__ __forceinline__ void lp_select_one(int mb, int mbs, const LpBuf& b, int mode, float param, int lambda,
                                              const float* logits, MV* __restrict__ mv_out) {
  const uint32_t st = b.state[mb];
  if (st & kStEarly) {
    mv_out[mb] = MV{0, 0, b.cand_sad[mb * kCand + 9], 0u};
    atomicAdd(&b.counters[3], 1);
    b.sel[mb] = 0xffffffffu;
    return;
  }
  if (st & kStNoHist) {
    b.lists[mbs + atomicAdd(&b.counters[1], 1)] = mb;
    b.sel[mb] = 0xffffffffu;
    return;
  }
  const uint32_t dup = (st >> 8) & 0x3ffu;
  float p[kClasses];
  const bool heuristic = mode == 2;
  uint32_t min_cost = 0xffffffffu;
  if (heuristic) {
    for (int c = 0; c < kCand; ++c) {
      const int32_t q = b.cand[mb * kCand + c];
      const uint32_t cost = b.cand_sad[mb * kCand + c] + (uint32_t)lambda * (uint32_t)(abs(cand_x(q)) + abs(cand_y(q)));
      p[c] = -(float)cost;
      min_cost = min(min_cost, cost);
    }
    p[kCand] = -INFINITY;
  } else {
    masked_softmax(logits, dup, p);
    b.p_norez[mb] = 1.f / (1.f + expf(-logits[11]));
  }
  uint32_t chosen = dup, sel = 0xffffffffu;
  float conf = 0.f;
  for (int k = 0; k < 4; ++k) {
    int best = -1;
    for (int c = 0; c < kCand; ++c)
      if (!((chosen >> c) & 1u) && (best < 0 || p[c] > p[best])) best = c;
    if (best < 0) break;
    chosen |= 1u << best;
    conf += p[best];
    sel = (sel & ~(0xffu << (8 * k))) | ((uint32_t)best << (8 * k));
  }
  b.sel[mb] = sel;
  const bool fall = heuristic ? (param >= 0.f && (float)min_cost > param * 256.f) : (conf < param);
  if (fall) {
    b.lists[mbs + atomicAdd(&b.counters[1], 1)] = mb;
  } else {
    b.lists[atomicAdd(&b.counters[0], 1)] = mb;
  }
}

// lp_select_one in mode 1 for the MBs mb0 .. mb0+nmb-1 of a network tile,
// lane i taking MB mb0+i (nmb <= 32), called by all 32 lanes of a warp.
// `st` is the lane's MB state word (read ahead by the caller). The same
// selection; the list appends are aggregated to one atomic per list per
// warp (the order inside a list is not meaningful).
__device__ __forceinline__ void lp_select_warp(int mb0, int nmb, int mbs, const LpBuf& b, float param,
                                               const float* logits, uint32_t st, MV* __restrict__ mv_out) {
  const int lane = threadIdx.x & 31;
  const bool act = lane < nmb;
  const int mb = mb0 + lane;
  const bool early = act && (st & kStEarly);
  bool fall = false;
  if (act && !early) {
    uint32_t sel = 0xffffffffu;
    if (st & kStNoHist) {
      fall = true;
    } else {
      const uint32_t dup = (st >> 8) & 0x3ffu;
      float p[kClasses];
      masked_softmax(logits, dup, p);
      b.p_norez[mb] = 1.f / (1.f + expf(-logits[11]));
      uint32_t chosen = dup;
      float conf = 0.f;
      for (int k = 0; k < 4; ++k) {
        int best = -1;
        for (int c = 0; c < kCand; ++c)
          if (!((chosen >> c) & 1u) && (best < 0 || p[c] > p[best])) best = c;
        if (best < 0) break;
        chosen |= 1u << best;
        conf += p[best];
        sel = (sel & ~(0xffu << (8 * k))) | ((uint32_t)best << (8 * k));
      }
      fall = conf < param;
    }
    b.sel[mb] = sel;
  }
  if (early) {
    mv_out[mb] = MV{0, 0, b.cand_sad[mb * kCand + 9], 0u};
    b.sel[mb] = 0xffffffffu;
  }
  const bool learn = act && !early && !fall;
  const uint32_t m_early = __ballot_sync(0xffffffffu, early), m_fall = __ballot_sync(0xffffffffu, fall),
                 m_learn = __ballot_sync(0xffffffffu, learn);
  int base_f = 0, base_l = 0;
  if (lane == 0) {
    if (m_early) atomicAdd(&b.counters[3], __popc(m_early));
    if (m_fall) base_f = atomicAdd(&b.counters[1], __popc(m_fall));
    if (m_learn) base_l = atomicAdd(&b.counters[0], __popc(m_learn));
  }
  base_f = __shfl_sync(0xffffffffu, base_f, 0);
  base_l = __shfl_sync(0xffffffffu, base_l, 0);
  const uint32_t below = (1u << lane) - 1u;
  if (fall) b.lists[mbs + base_f + __popc(m_fall & below)] = mb;
  if (learn) b.lists[base_l + __popc(m_learn & below)] = mb;
}

// The fused inference network + selection (proposal_infer.cu): logits of
// every MB into b.logits, selection as lp_select_one(mode 1, conf).
int lp_net_launch(int mbs, const LpBuf& b, const __nv_bfloat16* wb, const float* params, float conf, int lambda,
                  MV* mv_out, uint32_t* err, cudaStream_t st);
// The same in FP8 E4M3 (proposal_infer8.cu). `w8` (kNet8PackBytes) holds the
// E4M3 weights and their scales, quantised from the FP32 master parameters
// on `st` first when *stale (then cleared).
constexpr int kNet8PackBytes = 20480 + 6 * 64 * 4;
int lp_net8_launch(int mbs, const LpBuf& b, const float* params, uint8_t* w8, bool* stale, float conf, int lambda,
                   MV* mv_out, uint32_t* err, cudaStream_t st);

}  // namespace b200enc
