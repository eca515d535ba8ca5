// proposal_infer.cu - the motion-proposal network's inference as one
// persistent kernel on the tcgen05 tensor cores, with the candidate
// selection fused into its last epilogue.
//
// One CTA per SM (168 KB of shared memory), 16 warps, looping over tiles of
// 16 MBs. The BF16 weights of all six layers are staged once per CTA as
// UMMA B operands. Per tile every layer is a handful of M=128 MMAs into
// TMEM, issued by one thread and committed to an mbarrier; the epilogue
// (warp w reads TMEM lanes 32(w%4).. = rows; the four warps of a lane
// quadrant split the column blocks between them) adds the bias, applies ReLU,
// rounds to BF16 and writes the next layer's A operand directly in the
// canonical K-major layout. Because conv rows are in Morton order inside
// each MB, the four rows of every 2x2 stride-2 patch are consecutive: output
// row R of a conv layer becomes row R/4, K-offset (R%4)*32 of the next
// layer's operand. Arithmetic is the unfused path's (BF16 operands, FP32
// accumulation in the same K order, bias + ReLU in FP32, BF16 outputs).
//
//   c1  x0 [1024 x 16(8)] . w1 -> 8 tiles of 128 rows, N=32
//   c2  a2 [ 256 x 128]   . w2 -> 2 tiles, N=32
//   c3  a3 [  64 x 128]   . w3 -> 1 tile (64 rows used)
//   c4  a4 [  16 x 128]   . w4 -> 1 tile (16 rows used)
//   fc1 f  [  16 x 96 ]   . wf1 -> N=64
//   fc2 hd [  16 x 64 ]   . wf2 -> N=16 logits -> selection
#include <cuda_bf16.h>

#include "me_common.cuh"
#include "proposal.cuh"
#include "umma.cuh"

namespace b200enc {

constexpr int kNetTileMbs = 16;

struct NetSmem {
  // weights as B operands (canonical, rows = N)
  alignas(128) uint16_t w1[32 * 16];  // K 8 padded to 16 with zeros
  alignas(128) uint16_t w2[32 * 128];
  alignas(128) uint16_t w3[32 * 128];
  alignas(128) uint16_t w4[32 * 128];
  alignas(128) uint16_t wf1[64 * 96];
  alignas(128) uint16_t wf2[16 * 64];
  // activations as A operands (canonical, 128-row tiles)
  alignas(128) uint16_t x0[8][128 * 16];  // also a4 [128 x 128] once c1 has consumed it
  alignas(128) uint16_t a2[2][128 * 128];  // also hd [128 x 64] once c2 has consumed it
  alignas(128) uint16_t a3[128 * 128];  // also f [128 x 96] once c3 has consumed it
  float b1[32], b2[32], b3[32], b4[32], bf1[64], bf2[16];
  uint64_t bar;
  uint32_t tmem;
  int failed;
};

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&v);
}

// Bias + ReLU + BF16 of 8 consecutive channels, stored as one 16-byte chunk.
__device__ __forceinline__ void store8_relu(uint16_t* dst, const uint32_t* acc, const float* bias) {
  float x[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) x[i] = fmaxf(__uint_as_float(acc[i]) + bias[i], 0.f);
  uint4 v;
  v.x = pack_bf16x2(x[0], x[1]);
  v.y = pack_bf16x2(x[2], x[3]);
  v.z = pack_bf16x2(x[4], x[5]);
  v.w = pack_bf16x2(x[6], x[7]);
  *reinterpret_cast<uint4*>(dst) = v;
}


// Writes channels ch0 .. ch0+15 of conv output row R into the next layer's
// operand tile set `dst` (128-row tiles of K=128): row R/4, K offset
// (R%4)*32 + ch0.
__device__ __forceinline__ void store_conv_row16(uint16_t* dst_tiles, int R, int ch0, const uint32_t (&v)[16],
                                                 const float* bias) {
  const int q = R >> 2, j = R & 3;
  uint16_t* tile = dst_tiles + (size_t)(q >> 7) * (128 * 128);
  store8_relu(tile + canon_off(q & 127, j * 32 + ch0, 128), &v[0], bias + ch0);
  store8_relu(tile + canon_off(q & 127, j * 32 + ch0 + 8, 128), &v[8], bias + ch0 + 8);
}

constexpr int kNetThreads = 512;

__global__ void __launch_bounds__(kNetThreads, 1) lp_net_kernel(int mbs, LpBuf b, const __nv_bfloat16* __restrict__ wb,
                                                       const float* __restrict__ params, float param, int lambda,
                                                       MV* __restrict__ mv_out, uint32_t* __restrict__ err) {
  extern __shared__ __align__(128) uint8_t smem_raw[];
  NetSmem& s = *reinterpret_cast<NetSmem*>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int quad = warp & 3, wq = warp >> 2;  // TMEM lane quadrant, warp index within it (0..3)
  const uint16_t* w16 = reinterpret_cast<const uint16_t*>(wb);

  // ---- weights and biases, once per CTA --------------------------------
  for (int i = tid; i < 32 * 16; i += kNetThreads) {
    const int n = i >> 4, k = i & 15;
    s.w1[canon_off(n, k, 32)] = k < 8 ? w16[layer_woff(0) + n * 8 + k] : (uint16_t)0;
  }
  for (int i = tid; i < 32 * 128; i += kNetThreads) {
    const int n = i >> 7, k = i & 127;
    s.w2[canon_off(n, k, 32)] = w16[layer_woff(1) + i];
    s.w3[canon_off(n, k, 32)] = w16[layer_woff(2) + i];
    s.w4[canon_off(n, k, 32)] = w16[layer_woff(3) + i];
  }
  for (int i = tid; i < 64 * 96; i += kNetThreads) s.wf1[canon_off(i / 96, i % 96, 64)] = w16[layer_woff(4) + i];
  for (int i = tid; i < 16 * 64; i += kNetThreads) s.wf2[canon_off(i >> 6, i & 63, 16)] = w16[layer_woff(5) + i];
  if (tid < 32) {
    s.b1[tid] = params[layer_boff(0) + tid];
    s.b2[tid] = params[layer_boff(1) + tid];
    s.b3[tid] = params[layer_boff(2) + tid];
    s.b4[tid] = params[layer_boff(3) + tid];
  }
  if (tid < 64) s.bf1[tid] = params[layer_boff(4) + tid];
  if (tid < 16) s.bf2[tid] = params[layer_boff(5) + tid];
  if (warp == 0) tmem_alloc(&s.tmem, 256);
  if (tid == 0) {
    mbar_init(&s.bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s.failed = 0;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s.tmem;
  uint32_t phase = 0;
  constexpr uint64_t kWaitNs = 2000000000ull;

  const uint32_t a_x0 = smem_u32(s.x0), a_a2 = smem_u32(s.a2), a_a3 = smem_u32(s.a3);
  const uint32_t a_w1 = smem_u32(s.w1), a_w2 = smem_u32(s.w2), a_w3 = smem_u32(s.w3), a_w4 = smem_u32(s.w4);
  const uint32_t a_wf1 = smem_u32(s.wf1), a_wf2 = smem_u32(s.wf2);
  uint16_t* a4 = &s.x0[0][0];
  uint16_t* hd = &s.a2[0][0];
  uint16_t* fin = s.a3;  // fc1 input: c4 outputs (columns 0..31) + side features (32..95)
  const uint32_t a_a4 = a_x0, a_hd = a_a2, a_f = a_a3;

  // one layer: issue, commit, wait (all threads); false if the wait gave up
  auto sync_mma = [&]() -> bool {
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

  const int ntiles = (mbs + kNetTileMbs - 1) / kNetTileMbs;
  // The next tile's inputs are loaded into registers while the current tile
  // computes: 1024 network rows (16 B each, two per thread) and the 16 x 8
  // chunks of side features (threads 0..127).
  constexpr int kRowsPerThread = kNetTileMbs * 64 / kNetThreads;
  uint4 pre_x[kRowsPerThread], pre_f = make_uint4(0, 0, 0, 0);
  uint32_t pre_st = 0u;  // warp 0: the MB state words the selection reads
  auto prefetch = [&](int tile) {
    const int mb0 = tile * kNetTileMbs, nmb = min(kNetTileMbs, mbs - mb0);
#pragma unroll
    for (int i = 0; i < kRowsPerThread; ++i) {
      const int R = tid + i * kNetThreads;
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
    const int mb0 = tile * kNetTileMbs;
    const int nmb = min(kNetTileMbs, mbs - mb0);
    const uint32_t cur_st = pre_st;
    // ---- inputs: network rows (both K chunks) and side features ---------
#pragma unroll
    for (int i = 0; i < kRowsPerThread; ++i) {
      const int R = tid + i * kNetThreads;
      uint16_t* t = s.x0[R >> 7];
      *reinterpret_cast<uint4*>(t + canon_off(R & 127, 0, 128)) = pre_x[i];
      *reinterpret_cast<uint4*>(t + canon_off(R & 127, 8, 128)) = make_uint4(0, 0, 0, 0);
    }
    // the side features wait in registers until c3 has freed a3
    const uint4 cur_f = pre_f;
    if (tile + (int)gridDim.x < ntiles) prefetch(tile + gridDim.x);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();

    // ---- c1 ---------------------------------------------------------------
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int t = 0; t < 8; ++t)
        umma_bf16(tmem + 32 * t, canon_desc(a_x0 + t * (128 * 16 * 2), 128, 0), canon_desc(a_w1, 32, 0),
                  umma_idesc_bf16(128, 32), 0u);
      umma_commit(&s.bar);
    }
    if (!sync_mma()) break;
    // 8 tiles x 2 channel halves per lane quadrant, 4 warps per quadrant
    for (int job = wq; job < 16; job += 4) {
      const int t = job >> 1, h = job & 1;
      uint32_t v[16];
      tmem_row16(tmem, quad, 32 * t + 16 * h, v);
      store_conv_row16(&s.a2[0][0], 128 * t + 32 * quad + lane, 16 * h, v, s.b1);
    }
    publish();

    // ---- c2 ---------------------------------------------------------------
    if (tid == 0) {
      tc_fence_after();
      for (int t = 0; t < 2; ++t)
#pragma unroll
        for (int ks = 0; ks < 8; ++ks)
          umma_bf16(tmem + 32 * t, canon_desc(a_a2 + t * (128 * 128 * 2), 128, 16 * ks), canon_desc(a_w2, 32, 16 * ks),
                    umma_idesc_bf16(128, 32), ks > 0 ? 1u : 0u);
      umma_commit(&s.bar);
    }
    if (!sync_mma()) break;
    {  // 2 tiles x 2 halves per quadrant: one job per warp
      const int t = wq >> 1, h = wq & 1;
      uint32_t v[16];
      tmem_row16(tmem, quad, 32 * t + 16 * h, v);
      store_conv_row16(s.a3, 128 * t + 32 * quad + lane, 16 * h, v, s.b2);
    }
    publish();

    // ---- c3 (64 valid rows) -----------------------------------------------
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int ks = 0; ks < 8; ++ks)
        umma_bf16(tmem, canon_desc(a_a3, 128, 16 * ks), canon_desc(a_w3, 32, 16 * ks), umma_idesc_bf16(128, 32),
                  ks > 0 ? 1u : 0u);
      umma_commit(&s.bar);
    }
    if (!sync_mma()) break;
    if (quad < 2 && wq < 2) {  // rows 0..63: quadrants 0, 1; two halves
      uint32_t v[16];
      tmem_row16(tmem, quad, 16 * wq, v);
      store_conv_row16(a4, 32 * quad + lane, 16 * wq, v, s.b3);
    }
    publish();

    // ---- c4 (16 valid rows) -> fc1 input columns 0..31 ---------------------
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int ks = 0; ks < 8; ++ks)
        umma_bf16(tmem, canon_desc(a_a4, 128, 16 * ks), canon_desc(a_w4, 32, 16 * ks), umma_idesc_bf16(128, 32),
                  ks > 0 ? 1u : 0u);
      umma_commit(&s.bar);
    }
    if (!sync_mma()) break;
    if (tid < 128) *reinterpret_cast<uint4*>(fin + canon_off(tid >> 3, 32 + (tid & 7) * 8, 128)) = cur_f;
    if (quad == 0 && wq < 2) {  // rows 0..15, two halves of the 32 channels
      uint32_t v[16];
      tmem_row16(tmem, 0, 16 * wq, v);
      if (lane < 16) {
        store8_relu(fin + canon_off(lane, 16 * wq, 128), &v[0], s.b4 + 16 * wq);
        store8_relu(fin + canon_off(lane, 16 * wq + 8, 128), &v[8], s.b4 + 16 * wq + 8);
      }
    }
    publish();

    // ---- fc1 (N=64) ----------------------------------------------------------
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int ks = 0; ks < 6; ++ks)
        umma_bf16(tmem, canon_desc(a_f, 128, 16 * ks), canon_desc(a_wf1, 64, 16 * ks), umma_idesc_bf16(128, 64),
                  ks > 0 ? 1u : 0u);
      umma_commit(&s.bar);
    }
    if (!sync_mma()) break;
    if (quad == 0) {  // rows 0..15, 64 channels: 16 per warp of quadrant 0
      uint32_t v[16];
      tmem_row16(tmem, 0, 16 * wq, v);
      if (lane < 16) {
        store8_relu(hd + canon_off(lane, 16 * wq, 128), &v[0], s.bf1 + 16 * wq);
        store8_relu(hd + canon_off(lane, 16 * wq + 8, 128), &v[8], s.bf1 + 16 * wq + 8);
      }
    }
    publish();

    // ---- fc2 (N=16) -> logits -> selection ----------------------------------
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int ks = 0; ks < 4; ++ks)
        umma_bf16(tmem, canon_desc(a_hd, 128, 16 * ks), canon_desc(a_wf2, 16, 16 * ks), umma_idesc_bf16(128, 16),
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
      for (int j = 0; j < kOut; ++j) z[j] = __uint_as_float(v[j]) + s.bf2[j];
      if (lane < nmb) {
        float4* lo = reinterpret_cast<float4*>(b.logits + (size_t)(mb0 + lane) * kOut);
#pragma unroll
        for (int j = 0; j < 4; ++j) lo[j] = make_float4(z[4 * j], z[4 * j + 1], z[4 * j + 2], z[4 * j + 3]);
      }
      lp_select_warp(mb0, nmb, mbs, b, param, z, cur_st, mv_out);
    }
    publish();
  }
  if (s.failed && tid == 0 && err) atomicExch(err, 1u);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 256);
}

int lp_net_launch(int mbs, const LpBuf& b, const __nv_bfloat16* wb, const float* params, float conf, int lambda,
                  MV* mv_out, uint32_t* err, cudaStream_t st) {
  static_assert(sizeof(NetSmem) <= 227 * 1024, "fused network exceeds shared memory");
  const int smem = (int)sizeof(NetSmem);
  if (cudaFuncSetAttribute(lp_net_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess) return -1;
  int sms = 148;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int ntiles = (mbs + kNetTileMbs - 1) / kNetTileMbs;
  lp_net_kernel<<<std::min(ntiles, sms), kNetThreads, smem, st>>>(mbs, b, wb, params, conf, lambda, mv_out, err);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace b200enc
