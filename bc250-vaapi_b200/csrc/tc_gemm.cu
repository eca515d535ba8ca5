// tc_gemm.cu - BF16 GEMM on the 5th-generation tensor cores (tcgen05).
//
// The one dense contraction in this project is the learned motion-proposal
// network (convolutions as GEMMs over batches of macroblocks, forward and
// backward). This kernel computes
//     C[m][n] = epilogue( sum_k A(m,k) * B(n,k) )
// with A and B BF16 read through arbitrary (row, k) strides, so transposed
// operands of the backward pass need no copies, FP32 accumulation in tensor
// memory, and an epilogue of optional FP32 accumulate-into-C, bias and ReLU.
//
// Split K (grid z > 1) gives each z slice a range of 64-wide K chunks and
// adds the slices' FP32 partial products into C with atomics, for the weight
// gradients of the backward pass, whose reduction runs over every sample.
//
// Per CTA: a 128 x BN output tile, 4 warps. For each 64-wide K chunk the
// threads stage A (128 x 64) and B (BN x 64) in shared memory in the
// canonical K-major no-swizzle UMMA layout (8-row x 16-byte core matrices,
// rows of a core matrix 16 B apart, 8-row groups 128 B apart, K chunks of 8
// elements (BN or 128) x 16 B apart), one elected thread issues four
// tcgen05.mma (M=128, K=16) and commits them to an mbarrier; the next chunk's
// staging waits on that barrier. The accumulator lives in TMEM (lane = row,
// column = n) and is read back with tcgen05.ld 32x32b by each warp for its
// 32 rows.
#include <cuda_bf16.h>

#include "b200enc_internal.h"
#include "umma.cuh"

namespace b200enc {

constexpr int kTcM = 128, kTcK = 64;

template <int BN>
struct TcShared {
  alignas(128) uint16_t a[kTcM * kTcK];  // 16 KB
  alignas(128) uint16_t b[BN * kTcK];
  uint64_t bar;
  uint32_t tmem;
  int failed;
};

// Loads the first kw (a multiple of 16, at most 64) columns of one K chunk
// of an operand (rows x kw) into the canonical layout: element (r, kk) at
// ((kk/8) * rows/8 + r/8) * 64 + (r%8) * 8 + kk%8.
__device__ __forceinline__ void stage_chunk(uint16_t* dst, int rows, int kw, const __nv_bfloat16* src, long long rs,
                                            long long ks, int r0, int rmax, int k0, int kmax) {
  const int total = rows * kw;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    const int kk = i % kw, r = i / kw;  // consecutive threads walk k: coalesced for K-contiguous sources
    const int gr = r0 + r, gk = k0 + kk;
    uint16_t v = 0;
    if (gr < rmax && gk < kmax) v = __bfloat16_as_ushort(src[(long long)gr * rs + (long long)gk * ks]);
    dst[((kk >> 3) * (rows >> 3) + (r >> 3)) * 64 + (r & 7) * 8 + (kk & 7)] = v;
  }
}

template <int BN>
__global__ void __launch_bounds__(128) tc_gemm_kernel(int M, int N, int K, const __nv_bfloat16* __restrict__ A,
                                                      long long a_rs, long long a_ks, const __nv_bfloat16* __restrict__ B,
                                                      long long b_rs, long long b_ks, float* __restrict__ C, long long ldc,
                                                      const float* __restrict__ bias, int flags,
                                                      uint32_t* __restrict__ err) {
  constexpr uint32_t kCols = BN <= 32 ? 32 : (BN <= 64 ? 64 : (BN <= 128 ? 128 : 256));
  extern __shared__ __align__(128) uint8_t smem_raw[];
  TcShared<BN>& s = *reinterpret_cast<TcShared<BN>*>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * kTcM, n0 = blockIdx.y * BN;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s.tmem)),
                 "r"(kCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 0) {
    mbar_init(&s.bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s.failed = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s.tmem;
  constexpr uint32_t idesc = umma_idesc_bf16(kTcM, BN);

  // split K: blockIdx.z takes chunks [c_begin, c_end) and adds its partial
  // product into C atomically
  const int splits = gridDim.z;
  const int nchunks_all = (K + kTcK - 1) / kTcK;
  const int per = (nchunks_all + splits - 1) / splits;
  const int c_begin = blockIdx.z * per, c_end = min(nchunks_all, c_begin + per);
  uint32_t phase = 0;
  for (int c = c_begin; c < c_end; ++c) {
    if (c > c_begin) {
      // the MMAs reading the previous chunk must be done before restaging
      if (!mbar_wait(&s.bar, phase, 2000000000ull)) s.failed = 1;
      phase ^= 1;
    }
    const int ksteps = min(kTcK, K - c * kTcK + 15) / 16;  // 16-wide MMA steps holding real K
    stage_chunk(s.a, kTcM, ksteps * 16, A, a_rs, a_ks, m0, M, c * kTcK, K);
    stage_chunk(s.b, BN, ksteps * 16, B, b_rs, b_ks, n0, N, c * kTcK, K);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (s.failed) break;
    if (threadIdx.x == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (int k = 0; k < ksteps; ++k) {
        // K step k covers the core-matrix chunks 2k and 2k+1
        const uint64_t da = umma_desc(smem_u32(s.a) + (uint32_t)(2 * k * (kTcM / 8) * 128), kTcM * 16, 128);
        const uint64_t db = umma_desc(smem_u32(s.b) + (uint32_t)(2 * k * (BN / 8) * 128), BN * 16, 128);
        const uint32_t acc = (c > c_begin || k > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
            "l"(da), "l"(db), "r"(idesc), "r"(acc)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&s.bar))
                   : "memory");
    }
  }
  const bool any = c_end > c_begin;
  if (any && !s.failed && !mbar_wait(&s.bar, phase, 2000000000ull)) s.failed = 1;
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

  if (any && !s.failed) {
    // epilogue: warp w owns TMEM lanes (= rows) 32w .. 32w+31
    const int row = m0 + warp * 32 + lane;
#pragma unroll
    for (int cb = 0; cb < BN; cb += 16) {
      uint32_t v[16];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)cb;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (row < M) {
        if (splits > 1) {
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int col = n0 + cb + j;
            if (col < N) atomicAdd(C + (long long)row * ldc + col, __uint_as_float(v[j]));
          }
        } else {
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int col = n0 + cb + j;
            if (col >= N) continue;
            float x = __uint_as_float(v[j]);
            if (flags & B200ENC_GEMM_OUT_BF16) {
              __nv_bfloat16* dst = reinterpret_cast<__nv_bfloat16*>(C) + (long long)row * ldc + col;
              if (flags & B200ENC_GEMM_ACCUMULATE) x += __bfloat162float(*dst);
              if (bias) x += bias[col];
              if ((flags & B200ENC_GEMM_RELU) && x < 0.f) x = 0.f;
              *dst = __float2bfloat16_rn(x);
            } else {
              float* dst = C + (long long)row * ldc + col;
              if (flags & B200ENC_GEMM_ACCUMULATE) x += *dst;
              if (bias) x += bias[col];
              if ((flags & B200ENC_GEMM_RELU) && x < 0.f) x = 0.f;
              *dst = x;
            }
          }
        }
      }
    }
  } else if (threadIdx.x == 0 && err) {
    atomicExch(err, 1u);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
  }
}

template <int BN>
static int launch_tc(int M, int N, int K, const void* A, long long a_rs, long long a_ks, const void* B,
                     long long b_rs, long long b_ks, float* C, long long ldc, const float* bias, int flags,
                     uint32_t* err, cudaStream_t st) {
  const size_t smem = sizeof(TcShared<BN>) + 128;
  if (cudaFuncSetAttribute(tc_gemm_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return -1;
  const int splits = (flags >> 16) & 0xFF;
  dim3 grid((M + kTcM - 1) / kTcM, (N + BN - 1) / BN, splits > 1 ? splits : 1);
  tc_gemm_kernel<BN><<<grid, 128, smem, st>>>(M, N, K, (const __nv_bfloat16*)A, a_rs, a_ks,
                                              (const __nv_bfloat16*)B, b_rs, b_ks, C, ldc, bias, flags, err);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace b200enc

using namespace b200enc;

extern "C" int b200enc_gemm_bf16(int M, int N, int K, const void* A, long long a_rs, long long a_ks, const void* B,
                                 long long b_rs, long long b_ks, float* C, long long ldc, const float* bias, int flags,
                                 uint32_t* err, void* stream) {
  if (M <= 0 || N <= 0 || K <= 0 || !A || !B || !C) return -1;
  const int splits = (flags >> 16) & 0xFF;
  // split-K adds FP32 partial products atomically: no per-element epilogue
  if (splits > 1 && (flags & (B200ENC_GEMM_OUT_BF16 | B200ENC_GEMM_RELU | B200ENC_GEMM_ACCUMULATE) || bias))
    return -1;
  cudaStream_t st = (cudaStream_t)stream;
  if (N <= 32) return launch_tc<32>(M, N, K, A, a_rs, a_ks, B, b_rs, b_ks, C, ldc, bias, flags, err, st);
  if (N <= 64) return launch_tc<64>(M, N, K, A, a_rs, a_ks, B, b_rs, b_ks, C, ldc, bias, flags, err, st);
  return launch_tc<128>(M, N, K, A, a_rs, a_ks, B, b_rs, b_ks, C, ldc, bias, flags, err, st);
}
