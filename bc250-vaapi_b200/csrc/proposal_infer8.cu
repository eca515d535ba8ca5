// proposal_infer8.cu - the motion-proposal network's inference in FP8 (E4M3)
// on the tcgen05 tensor cores (kind::f8f6f4, FP32 accumulation), as one
// persistent kernel with the candidate selection fused into its last
// epilogue. The network is trained in BF16 (proposal.cu, tc_gemm.cu); this
// is its FP8 inference form, selected by b200enc_proposal_me mode 3.
//
// Quantisation (the CPU oracle, oracle/proposal_ref.py forward_fp8, follows
// the same arithmetic step for step):
//   * weights: one scale per output channel, s_w = amax_k |W[n][k]| / 448,
//     W8 = E4M3(W * (448 / amax)), from the FP32 master parameters, by a
//     one-CTA pass whenever they have changed (the runtime marks the pack
//     stale on set_params and on each Adam step); each CTA copies the pack;
//   * activations: one scale per 16-MB tile and layer input, s = amax / 448
//     over the tile, A8 = E4M3(A * (448 / amax)) - the network input, each
//     hidden layer's output after bias and ReLU, and the fc1 input (the c4
//     output and the side features together);
//   * epilogues: y = max(fma(acc, s_in * s_w[n], b[n]), 0) in FP32; the
//     logits are fma(acc, s_in * s_w[n], b[n]).
// E4M3 conversion rounds to nearest even and saturates at +-448.
//
// Shape of the work as in proposal_infer.cu (Morton conv rows, 2x2 stride-2
// convs as plain GEMMs), with 8-bit operands: one MMA consumes K = 32, the
// canonical layout's core-matrix rows hold 16 elements, and the operand
// tiles take half the shared memory (~105 KB per CTA instead of 168 KB), so
// two CTAs share an SM.
// Each hidden epilogue makes two passes over TMEM: the first finds the
// tile's maximum (warp max, one shared atomic per warp), a barrier
// publishes it, the second quantises and stores - so no thread holds its
// values across the barrier.
#include <cuda_fp8.h>

#include <cstddef>

#include "me_common.cuh"
#include "proposal.cuh"
#include "umma.cuh"

namespace b200enc {

constexpr int kNet8TileMbs = 16;
// 8 warps (two per TMEM lane quadrant) and ~105 KB of shared memory: two
// CTAs fit on an SM (registers, shared memory and TMEM's 512 columns), so
// one CTA's epilogues run while the other waits on its MMAs.
constexpr int kNet8Threads = 256;
constexpr int kNet8Wpq = kNet8Threads / 128;  // warps per TMEM lane quadrant

struct Net8Smem {
  // weights as B operands (8-bit canonical, rows = N)
  alignas(128) uint8_t w1[32 * 32];  // K 8 padded to 32 with zeros
  alignas(128) uint8_t w2[32 * 128];
  alignas(128) uint8_t w3[32 * 128];
  alignas(128) uint8_t w4[32 * 128];
  alignas(128) uint8_t wf1[64 * 96];
  alignas(128) uint8_t wf2[16 * 64];
  // activations as A operands (8-bit canonical, 128-row tiles)
  alignas(128) uint8_t x0[8][128 * 32];  // also a4 [128 x 128] once c1 has consumed it
  alignas(128) uint8_t a2[2][128 * 128];  // also hd [128 x 64] once c2 has consumed it
  alignas(128) uint8_t a3[128 * 128];     // also f [128 x 96] once c3 has consumed it
  float sw[6][64];                        // weight scales per layer and output channel
  float b1[32], b2[32], b3[32], b4[32], bf1[64], bf2[16];
  uint32_t amax[8];                       // the tile's maximum per layer input (float bits, >= 0)
  uint64_t bar;
  uint32_t tmem;
  int failed;
};

__device__ __forceinline__ uint8_t to_e4m3(float v) {
  return (uint8_t)__nv_cvt_float_to_fp8(v, __NV_SATFINITE, __NV_E4M3);
}

// Scale pair of a maximum: multiply by `inv` to quantise, by `s` to undo it.
__device__ __forceinline__ void e4m3_scale(float amax, float& inv, float& s) {
  if (amax > 0.f) {
    inv = 448.f / amax;
    s = amax / 448.f;
  } else {
    inv = 1.f;
    s = 1.f;
  }
}

// Warp maximum of non-negative values, folded into *slot (float bits of a
// non-negative float order like the floats).
__device__ __forceinline__ void warp_amax(uint32_t* slot, float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) atomicMax(slot, __float_as_uint(v));
}

// Stages one layer's FP32 weights W[N][K] (row-major at `src`) as E4M3 into
// the canonical tile `dst` of N rows and Kp >= K columns (zero padded), with
// the per-channel scale into `sw`. One warp per output channel.
__device__ void stage_w8(const float* __restrict__ src, int N, int K, int Kp, uint8_t* dst, float* sw) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int n = warp; n < N; n += kNet8Threads / 32) {
    float m = 0.f;
    for (int k = lane; k < K; k += 32) m = fmaxf(m, fabsf(src[n * K + k]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    float inv, s;
    e4m3_scale(m, inv, s);
    if (lane == 0) sw[n] = s;
    for (int k = lane; k < Kp; k += 32) dst[canon_off8(n, k, N)] = k < K ? to_e4m3(src[n * K + k] * inv) : (uint8_t)0;
  }
}

// 16 consecutive channels of one output row as E4M3, one 16-byte store.
__device__ __forceinline__ void store16_e4m3(uint8_t* dst, const float (&y)[16], float inv) {
  uint32_t w[4];
#pragma unroll
  for (int j = 0; j < 4; ++j)
    w[j] = (uint32_t)to_e4m3(y[4 * j] * inv) | ((uint32_t)to_e4m3(y[4 * j + 1] * inv) << 8) |
           ((uint32_t)to_e4m3(y[4 * j + 2] * inv) << 16) | ((uint32_t)to_e4m3(y[4 * j + 3] * inv) << 24);
  *reinterpret_cast<uint4*>(dst) = make_uint4(w[0], w[1], w[2], w[3]);
}

// Bias + ReLU of 16 channels ch0.. of one accumulator row, dequantised by
// s_in * s_w[ch].
__device__ __forceinline__ void epi16(const uint32_t (&acc)[16], float s_in, const float* sw, const float* bias,
                                      float (&y)[16]) {
#pragma unroll
  for (int i = 0; i < 16; ++i) y[i] = fmaxf(fmaf(__uint_as_float(acc[i]), s_in * sw[i], bias[i]), 0.f);
}

__device__ __forceinline__ float max16(const float (&y)[16]) {
  float m = 0.f;
#pragma unroll
  for (int i = 0; i < 16; ++i) m = fmaxf(m, y[i]);
  return m;
}

// The weight pack in global memory: the six E4M3 tiles in Net8Smem's order
// (w1 .. wf2, contiguous) and the per-channel scales.
struct W8Pack {
  uint8_t w[20480];
  float sw[6][64];
};
static_assert(sizeof(W8Pack) == kNet8PackBytes, "weight pack");
static_assert(offsetof(Net8Smem, w2) == 1024 && offsetof(Net8Smem, w3) == 5120 && offsetof(Net8Smem, w4) == 9216 &&
                  offsetof(Net8Smem, wf1) == 13312 && offsetof(Net8Smem, wf2) == 19456 &&
                  offsetof(Net8Smem, x0) == 20480,
              "the weight tiles are contiguous at the start of Net8Smem");

// Quantises the FP32 parameters into the pack (one CTA; once per parameter
// change).
__global__ void __launch_bounds__(kNet8Threads) lp_quant8_kernel(const float* __restrict__ params, uint8_t* w8) {
  W8Pack& pk = *reinterpret_cast<W8Pack*>(w8);
  stage_w8(params + layer_woff(0), 32, 8, 32, pk.w + 0, pk.sw[0]);
  stage_w8(params + layer_woff(1), 32, 128, 128, pk.w + 1024, pk.sw[1]);
  stage_w8(params + layer_woff(2), 32, 128, 128, pk.w + 5120, pk.sw[2]);
  stage_w8(params + layer_woff(3), 32, 128, 128, pk.w + 9216, pk.sw[3]);
  stage_w8(params + layer_woff(4), 64, 96, 96, pk.w + 13312, pk.sw[4]);
  stage_w8(params + layer_woff(5), 16, 64, 64, pk.w + 19456, pk.sw[5]);
}

__device__ __forceinline__ float bf16_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t w) { return __uint_as_float(w & 0xffff0000u); }

__global__ void __launch_bounds__(kNet8Threads, 2) lp_net8_kernel(int mbs, LpBuf b, const float* __restrict__ params,
                                                         const uint8_t* __restrict__ w8, float param, int lambda,
                                                         MV* __restrict__ mv_out, uint32_t* __restrict__ err) {
  extern __shared__ __align__(128) uint8_t smem_raw[];
  Net8Smem& s = *reinterpret_cast<Net8Smem*>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int quad = warp & 3, wq = warp >> 2;  // TMEM lane quadrant, warp index within it

  // ---- E4M3 weights with per-channel scales (the pack), biases, once per CTA
  {
    const uint4* src = reinterpret_cast<const uint4*>(w8);
    uint4* dst = reinterpret_cast<uint4*>(s.w1);
    for (int i = tid; i < 20480 / 16; i += kNet8Threads) dst[i] = src[i];
    const float* sws = reinterpret_cast<const W8Pack*>(w8)->sw[0];
    for (int i = tid; i < 6 * 64; i += kNet8Threads) (&s.sw[0][0])[i] = sws[i];
  }
  if (tid < 32) {
    s.b1[tid] = params[layer_boff(0) + tid];
    s.b2[tid] = params[layer_boff(1) + tid];
    s.b3[tid] = params[layer_boff(2) + tid];
    s.b4[tid] = params[layer_boff(3) + tid];
  }
  if (tid < 64) s.bf1[tid] = params[layer_boff(4) + tid];
  if (tid < 16) s.bf2[tid] = params[layer_boff(5) + tid];
  if (tid < 8) s.amax[tid] = 0u;
  if (warp == 0) tmem_alloc(&s.tmem, 256);
  if (tid == 0) {
    mbar_init(&s.bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s.failed = 0;
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s.tmem;
  uint32_t phase = 0;
  constexpr uint64_t kWaitNs = 2000000000ull;

  const uint32_t a_x0 = smem_u32(s.x0), a_a2 = smem_u32(s.a2), a_a3 = smem_u32(s.a3);
  const uint32_t a_w1 = smem_u32(s.w1), a_w2 = smem_u32(s.w2), a_w3 = smem_u32(s.w3), a_w4 = smem_u32(s.w4);
  const uint32_t a_wf1 = smem_u32(s.wf1), a_wf2 = smem_u32(s.wf2);
  uint8_t* a4 = &s.x0[0][0];
  uint8_t* hd = &s.a2[0][0];
  uint8_t* fin = s.a3;  // fc1 input: c4 outputs (columns 0..31) + side features (32..95)
  const uint32_t a_a4 = a_x0, a_hd = a_a2, a_f = a_a3;

  auto sync_mma = [&]() -> bool {  // one layer's MMAs done (all threads)
    if (!mbar_wait(&s.bar, phase, kWaitNs)) s.failed = 1;
    phase ^= 1;
    tc_fence_after();
    __syncthreads();
    return s.failed == 0;
  };
  auto publish = [&]() {  // generic smem writes and TMEM reads done -> next MMAs
    tmem_wait_ld();
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
  };
  auto scale_of = [&](int l, float& inv, float& sc) { e4m3_scale(__uint_as_float(s.amax[l]), inv, sc); };

  const int ntiles = (mbs + kNet8TileMbs - 1) / kNet8TileMbs;
  // the next tile's inputs are loaded into registers while the current one
  // computes: 1024 network rows (8 BF16 each, two per thread) and the 16 x 8
  // chunks of side features (threads 0..127)
  constexpr int kRowsPerThread = kNet8TileMbs * 64 / kNet8Threads;
  uint4 pre_x[kRowsPerThread], pre_f = make_uint4(0, 0, 0, 0);
  uint32_t pre_st = 0u;  // warp 0: the MB state words the selection reads
  auto prefetch = [&](int tile) {
    const int mb0 = tile * kNet8TileMbs, nmb = min(kNet8TileMbs, mbs - mb0);
#pragma unroll
    for (int i = 0; i < kRowsPerThread; ++i) {
      const int R = tid + i * kNet8Threads;
      pre_x[i] = (R >> 6) < nmb ? *reinterpret_cast<const uint4*>(b.x0 + ((size_t)mb0 * 64 + R) * 8)
                                : make_uint4(0, 0, 0, 0);
    }
    if (warp == 0) pre_st = lane < nmb ? b.state[mb0 + lane] : 0u;
    if (tid < 128) {
      const int m = tid >> 3, c8 = tid & 7;
      pre_f = m < nmb ? *reinterpret_cast<const uint4*>(b.f + (size_t)(mb0 + m) * kFIn + 32 + c8 * 8)
                      : make_uint4(0, 0, 0, 0);
    }
  };
  if ((int)blockIdx.x < ntiles) prefetch(blockIdx.x);
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int mb0 = tile * kNet8TileMbs;
    const int nmb = min(kNet8TileMbs, mbs - mb0);
    uint4 cur_x[kRowsPerThread];
#pragma unroll
    for (int i = 0; i < kRowsPerThread; ++i) cur_x[i] = pre_x[i];
    const uint4 cur_f = pre_f;  // waits in registers until c3 has freed a3
    const uint32_t cur_st = pre_st;
    if (tile + (int)gridDim.x < ntiles) prefetch(tile + gridDim.x);

    // ---- network input: the tile's maximum, then E4M3 rows ----------------
    {
      float m = 0.f;
#pragma unroll
      for (int i = 0; i < kRowsPerThread; ++i) {
        const uint32_t w[4] = {cur_x[i].x, cur_x[i].y, cur_x[i].z, cur_x[i].w};
#pragma unroll
        for (int j = 0; j < 4; ++j) m = fmaxf(m, fmaxf(fabsf(bf16_lo(w[j])), fabsf(bf16_hi(w[j]))));
      }
      warp_amax(&s.amax[0], m);
    }
    __syncthreads();
    float inv0, s0;
    scale_of(0, inv0, s0);
#pragma unroll
    for (int i = 0; i < kRowsPerThread; ++i) {
      const int R = tid + i * kNet8Threads;
      uint8_t* t = s.x0[R >> 7];
      const uint32_t w[4] = {cur_x[i].x, cur_x[i].y, cur_x[i].z, cur_x[i].w};
      uint32_t q[2];
#pragma unroll
      for (int j = 0; j < 2; ++j)
        q[j] = (uint32_t)to_e4m3(bf16_lo(w[2 * j]) * inv0) | ((uint32_t)to_e4m3(bf16_hi(w[2 * j]) * inv0) << 8) |
               ((uint32_t)to_e4m3(bf16_lo(w[2 * j + 1]) * inv0) << 16) |
               ((uint32_t)to_e4m3(bf16_hi(w[2 * j + 1]) * inv0) << 24);
      *reinterpret_cast<uint4*>(t + canon_off8(R & 127, 0, 128)) = make_uint4(q[0], q[1], 0u, 0u);
      *reinterpret_cast<uint4*>(t + canon_off8(R & 127, 16, 128)) = make_uint4(0u, 0u, 0u, 0u);
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();

    // ---- c1: 8 tiles of 128 rows, K 32 (8 used), N 32 ---------------------
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int t = 0; t < 8; ++t)
        umma_f8(tmem + 32 * t, canon_desc8(a_x0 + t * (128 * 32), 128, 0), canon_desc8(a_w1, 32, 0),
                umma_idesc_e4m3(128, 32), 0u);
      umma_commit(&s.bar);
    }
    if (!sync_mma()) break;
    {  // pass 1: the tile's maximum (8 tiles x 2 channel halves per quadrant, 4 warps each)
      float m = 0.f;
      for (int job = wq; job < 16; job += kNet8Wpq) {
        const int t = job >> 1, h = job & 1;
        uint32_t v[16];
        float y[16];
        tmem_row16(tmem, quad, 32 * t + 16 * h, v);
        epi16(v, s0, s.sw[0] + 16 * h, s.b1 + 16 * h, y);
        m = fmaxf(m, max16(y));
      }
      warp_amax(&s.amax[1], m);
    }
    __syncthreads();
    float inv1, s1;
    scale_of(1, inv1, s1);
    for (int job = wq; job < 16; job += kNet8Wpq) {  // pass 2: E4M3 conv rows -> a2 (row R/4, K (R%4)*32 + ch)
      const int t = job >> 1, h = job & 1;
      uint32_t v[16];
      float y[16];
      tmem_row16(tmem, quad, 32 * t + 16 * h, v);
      epi16(v, s0, s.sw[0] + 16 * h, s.b1 + 16 * h, y);
      const int R = 128 * t + 32 * quad + lane, q = R >> 2, j = R & 3;
      store16_e4m3(s.a2[q >> 7] + canon_off8(q & 127, j * 32 + 16 * h, 128), y, inv1);
    }
    publish();

    // ---- c2: 2 tiles x 4 K steps -------------------------------------------
    if (tid == 0) {
      tc_fence_after();
      for (int t = 0; t < 2; ++t)
#pragma unroll
        for (int ks = 0; ks < 4; ++ks)
          umma_f8(tmem + 32 * t, canon_desc8(a_a2 + t * (128 * 128), 128, 32 * ks), canon_desc8(a_w2, 32, 32 * ks),
                  umma_idesc_e4m3(128, 32), ks > 0 ? 1u : 0u);
      umma_commit(&s.bar);
    }
    if (!sync_mma()) break;
    {  // 2 tiles x 2 halves per quadrant
      float m = 0.f;
      for (int job = wq; job < 4; job += kNet8Wpq) {
        const int t2 = job >> 1, h2 = job & 1;
        uint32_t v[16];
        float y[16];
        tmem_row16(tmem, quad, 32 * t2 + 16 * h2, v);
        epi16(v, s1, s.sw[1] + 16 * h2, s.b2 + 16 * h2, y);
        m = fmaxf(m, max16(y));
      }
      warp_amax(&s.amax[2], m);
    }
    __syncthreads();
    float inv2, s2;
    scale_of(2, inv2, s2);
    for (int job = wq; job < 4; job += kNet8Wpq) {
      const int t2 = job >> 1, h2 = job & 1;
      uint32_t v[16];
      float y[16];
      tmem_row16(tmem, quad, 32 * t2 + 16 * h2, v);
      epi16(v, s1, s.sw[1] + 16 * h2, s.b2 + 16 * h2, y);
      const int R = 128 * t2 + 32 * quad + lane, q = R >> 2, j = R & 3;
      store16_e4m3(s.a3 + canon_off8(q, j * 32 + 16 * h2, 128), y, inv2);
    }
    publish();

    // ---- c3 (64 valid rows) ------------------------------------------------
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int ks = 0; ks < 4; ++ks)
        umma_f8(tmem, canon_desc8(a_a3, 128, 32 * ks), canon_desc8(a_w3, 32, 32 * ks), umma_idesc_e4m3(128, 32),
                ks > 0 ? 1u : 0u);
      umma_commit(&s.bar);
    }
    if (!sync_mma()) break;
    const bool c3w = quad < 2 && wq < 2;  // rows 0..63: quadrants 0, 1; two halves
    if (c3w) {
      uint32_t v[16];
      float y[16];
      tmem_row16(tmem, quad, 16 * wq, v);
      epi16(v, s2, s.sw[2] + 16 * wq, s.b3 + 16 * wq, y);
      warp_amax(&s.amax[3], max16(y));
    }
    __syncthreads();
    float inv3, s3;
    scale_of(3, inv3, s3);
    if (c3w) {
      uint32_t v[16];
      float y[16];
      tmem_row16(tmem, quad, 16 * wq, v);
      epi16(v, s2, s.sw[2] + 16 * wq, s.b3 + 16 * wq, y);
      const int R = 32 * quad + lane, q = R >> 2, j = R & 3;
      store16_e4m3(a4 + canon_off8(q, j * 32 + 16 * wq, 128), y, inv3);
    }
    publish();

    // ---- c4 (16 valid rows) -> fc1 input with the side features -------------
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int ks = 0; ks < 4; ++ks)
        umma_f8(tmem, canon_desc8(a_a4, 128, 32 * ks), canon_desc8(a_w4, 32, 32 * ks), umma_idesc_e4m3(128, 32),
                ks > 0 ? 1u : 0u);
      umma_commit(&s.bar);
    }
    if (!sync_mma()) break;
    const bool c4w = quad == 0 && wq < 2;  // rows 0..15, two halves of the 32 channels
    float fv[8];
    {
      const uint32_t w[4] = {cur_f.x, cur_f.y, cur_f.z, cur_f.w};
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        fv[2 * j] = bf16_lo(w[j]);
        fv[2 * j + 1] = bf16_hi(w[j]);
      }
    }
    {
      float m = 0.f;
      if (c4w) {
        uint32_t v[16];
        float y[16];
        tmem_row16(tmem, 0, 16 * wq, v);
        epi16(v, s3, s.sw[3] + 16 * wq, s.b4 + 16 * wq, y);
        if (lane < 16) m = max16(y);
      }
      if (tid < 128)
#pragma unroll
        for (int j = 0; j < 8; ++j) m = fmaxf(m, fabsf(fv[j]));
      warp_amax(&s.amax[4], m);
    }
    __syncthreads();
    float inv4, s4;
    scale_of(4, inv4, s4);
    if (c4w) {
      uint32_t v[16];
      float y[16];
      tmem_row16(tmem, 0, 16 * wq, v);
      epi16(v, s3, s.sw[3] + 16 * wq, s.b4 + 16 * wq, y);
      if (lane < 16) store16_e4m3(fin + canon_off8(lane, 16 * wq, 128), y, inv4);
    }
    if (tid < 128) {
      uint32_t q[2];
#pragma unroll
      for (int j = 0; j < 2; ++j)
        q[j] = (uint32_t)to_e4m3(fv[4 * j] * inv4) | ((uint32_t)to_e4m3(fv[4 * j + 1] * inv4) << 8) |
               ((uint32_t)to_e4m3(fv[4 * j + 2] * inv4) << 16) | ((uint32_t)to_e4m3(fv[4 * j + 3] * inv4) << 24);
      *reinterpret_cast<uint2*>(fin + canon_off8(tid >> 3, 32 + (tid & 7) * 8, 128)) = make_uint2(q[0], q[1]);
    }
    publish();

    // ---- fc1 (K 96, N 64) ------------------------------------------------------
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int ks = 0; ks < 3; ++ks)
        umma_f8(tmem, canon_desc8(a_f, 128, 32 * ks), canon_desc8(a_wf1, 64, 32 * ks), umma_idesc_e4m3(128, 64),
                ks > 0 ? 1u : 0u);
      umma_commit(&s.bar);
    }
    if (!sync_mma()) break;
    if (quad == 0) {  // rows 0..15, 64 channels in blocks of 16 over quadrant 0's warps
      float m = 0.f;
      for (int blk = wq; blk < 4; blk += kNet8Wpq) {
        uint32_t v[16];
        float y[16];
        tmem_row16(tmem, 0, 16 * blk, v);
        epi16(v, s4, s.sw[4] + 16 * blk, s.bf1 + 16 * blk, y);
        if (lane < 16) m = fmaxf(m, max16(y));
      }
      warp_amax(&s.amax[5], m);
    }
    __syncthreads();
    float inv5, s5;
    scale_of(5, inv5, s5);
    if (quad == 0)
      for (int blk = wq; blk < 4; blk += kNet8Wpq) {
        uint32_t v[16];
        float y[16];
        tmem_row16(tmem, 0, 16 * blk, v);
        epi16(v, s4, s.sw[4] + 16 * blk, s.bf1 + 16 * blk, y);
        if (lane < 16) store16_e4m3(hd + canon_off8(lane, 16 * blk, 128), y, inv5);
      }
    publish();

    // ---- fc2 (K 64, N 16) -> logits -> selection ------------------------------
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int ks = 0; ks < 2; ++ks)
        umma_f8(tmem, canon_desc8(a_hd, 128, 32 * ks), canon_desc8(a_wf2, 16, 32 * ks), umma_idesc_e4m3(128, 16),
                ks > 0 ? 1u : 0u);
      umma_commit(&s.bar);
    }
    if (!sync_mma()) break;
    if (warp == 0) {
      uint32_t v[16];
      tmem_ld16(tmem, v);
      tmem_wait_ld();
      float z[kOut];
#pragma unroll
      for (int j = 0; j < kOut; ++j) z[j] = fmaf(__uint_as_float(v[j]), s5 * s.sw[5][j], s.bf2[j]);
      if (lane < nmb) {
        float4* lo = reinterpret_cast<float4*>(b.logits + (size_t)(mb0 + lane) * kOut);
#pragma unroll
        for (int j = 0; j < 4; ++j) lo[j] = make_float4(z[4 * j], z[4 * j + 1], z[4 * j + 2], z[4 * j + 3]);
      }
      lp_select_warp(mb0, nmb, mbs, b, param, z, cur_st, mv_out);
    }
    if (tid < 8) s.amax[tid] = 0u;  // every read of this tile's maxima is behind the barriers above
    publish();
  }
  if (s.failed && tid == 0 && err) atomicExch(err, 1u);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 256);
}

int lp_net8_launch(int mbs, const LpBuf& b, const float* params, uint8_t* w8, bool* stale, float conf, int lambda,
                   MV* mv_out, uint32_t* err, cudaStream_t st) {
  if (*stale) {
    lp_quant8_kernel<<<1, kNet8Threads, 0, st>>>(params, w8);
    if (cudaGetLastError() != cudaSuccess) return -1;
    *stale = false;
  }
  static_assert(sizeof(Net8Smem) <= 227 * 1024, "FP8 network exceeds shared memory");
  const int smem = (int)sizeof(Net8Smem);
  if (cudaFuncSetAttribute(lp_net8_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
    return -1;
  int sms = 148;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int ntiles = (mbs + kNet8TileMbs - 1) / kNet8TileMbs;
  lp_net8_kernel<<<std::min(ntiles, 2 * sms), kNet8Threads, smem, st>>>(mbs, b, params, w8, conf, lambda, mv_out,
                                                                       err);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace b200enc
