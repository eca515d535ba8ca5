// me.cu - plain full-search block motion estimation, one CTA per 16x16 MB.
//
// Reference stage: A1/shaders/motion_estimation.comp (zero-MV early-out
// :312-331, lambda cost :363, half/quarter-pel refine :388-459 with the
// 6-tap interpolation of :154-215). The reference searches a diamond; the
// plain form here is exhaustive over [-R,R]^2 with a raster tie-break (the
// CPU oracle states the exact rule) and keeps the reference's refine.
//
// B200 layout: the (2R+24)^2 reference window (search range plus the 6-tap
// reach of the refine) is staged once in shared memory, by one 2-D TMA load
// (cp.async.bulk.tensor, no multicast) of a box that starts on the 16-byte
// boundary 12 bytes left of the window when the window lies inside the
// reference plane, by clamped word loads into the same layout at the
// picture edges and in batched steps; the current MB sits
// in 64 registers per thread. Thread t owns candidate column dx = t - R and
// sweeps the window rows top to bottom: each row's 16 bytes (one funnel
// shift per word off 5 aligned shared loads) feed the SADs of the 16
// candidates that use that row, accumulated in a 16-slot ring, so every
// window byte is read once per column. SAD is the byte-SIMD
// vabsdiff4-with-add; the integer path uses no tensor cores. The column
// dx = +R is scored directly, one candidate per thread, after the sweep.
#include <cuda.h>

#include <algorithm>
#include <cstring>

#include "b200enc_internal.h"
#include "me_common.cuh"
#include "umma.cuh"

namespace b200enc {

template <int R>
struct MeShared {
  static constexpr int WP = 2 * R + 24;                   // window side in pels
  static constexpr int WW = WP / 4;                       // 32-bit words of a window row
  static constexpr int OFF = 3;                           // window column 0 sits 12 bytes into a staged row
  static constexpr int BW = (4 * OFF + WP + 15) / 16 * 16;  // staged row: the TMA box width in bytes
  static constexpr int WS = BW / 4;                       // 32-bit words per staged row
  alignas(128) uint32_t win[WP * WS];
  uint32_t cur[64];
  uint32_t red[8];
  uint64_t bar;  // TMA completion
  RefineShared rf;
};
static_assert(MeShared<16>::BW == 80 && MeShared<32>::BW == 112, "box widths");

// Where a CTA's macroblocks come from (MODE): 0 one CTA per MB of one frame;
// 1 a persistent grid over a list of that frame's MBs; 2 a persistent grid
// over every P macroblock of a batch; 3 over a list of compact batch P
// indices (the learned form's fallback in a batch). The search itself is
// the same in all four.
enum : int { kMeGrid = 0, kMeList = 1, kMeBatch = 2, kMeBatchList = 3 };

// Error word of launches given no scratch word (b200enc_me_wait_errors).
__device__ uint32_t g_me_wait_err;

template <int R, int MODE>
__global__ void __launch_bounds__(2 * R) me_full_search_kernel(const uint8_t* __restrict__ cur_, int cur_pitch_,
                                                               const uint8_t* __restrict__ ref_, int ref_pitch_,
                                                               Geo g_, int lambda_, int zero_thresh_,
                                                               MV* __restrict__ out_, const int* __restrict__ mb_list,
                                                               const int* __restrict__ mb_count, int flags,
                                                               BatchTab bt, const __grid_constant__ CUtensorMap tmap,
                                                               int use_tma, uint32_t* err) {
  constexpr int NT = 2 * R;
  using S = MeShared<R>;
  constexpr int WP = S::WP, WW = S::WW, WS = S::WS, OFF = S::OFF, SIDE = 2 * R + 1;
  constexpr uint64_t kWaitNs = 2000000000ull;
  __shared__ S sh;
  const int tid = threadIdx.x;
  // the map describes this launch's single reference plane; batched steps
  // read one plane per stream and stage with loads
  const bool tma_ok = (MODE == kMeGrid || MODE == kMeList) && use_tma;
  uint32_t phase = 0;
  if (tma_ok) {
    if (tid == 0) {
      mbar_init(&sh.bar, 1);
      fence_async_smem();
    }
    __syncthreads();
  }
  const int n_items = MODE == kMeGrid ? 1 : (MODE == kMeBatch ? bt.p_mbs.total() : *mb_count);
  for (int item = MODE == kMeGrid ? 0 : (int)blockIdx.x; item < n_items; item += MODE == kMeGrid ? 1 : (int)gridDim.x) {
  int mbx = blockIdx.x, mby = blockIdx.y;
  const uint8_t* cur = cur_;
  const uint8_t* ref = ref_;
  int cur_pitch = cur_pitch_, ref_pitch = ref_pitch_, lambda = lambda_, zero_thresh = zero_thresh_;
  Geo g = g_;
  MV* o;
  if (MODE == kMeList) {
    const int mb = mb_list[item];
    mby = mb / g.mbw;
    mbx = mb - mby * g.mbw;
  }
  if (MODE == kMeBatch || MODE == kMeBatchList) {
    const int ci = MODE == kMeBatch ? item : mb_list[item];
    const int k = bt.p_mbs.find(ci);
    const BatchStream& st = bt.p_mbs.stream(k);
    const int local = ci - bt.p_mbs.prefix[k];
    g = st.g;
    mby = local / g.mbw;
    mbx = local - mby * g.mbw;
    cur = st.cur_y;
    cur_pitch = st.cur_pitch;
    ref = st.ref_y;
    ref_pitch = st.rec_pitch;
    lambda = st.lambda;
    zero_thresh = st.zero_thresh;
    o = bt.mvc + ci;
  } else {
    o = out_ + (size_t)mby * g.mbw + mbx;
  }
  if (MODE != kMeGrid) {
    if (tma_ok) fence_async_smem();  // this thread's accesses of the window precede the next TMA write
    __syncthreads();                 // the previous item's shared memory is no longer read
  }
  if ((MODE == kMeBatch || MODE == kMeBatchList) && mby >= g.mbh) continue;  // padding of the compact index
  const int X = mbx * 16, Y = mby * 16;
  const int ox = X - R - 4, oy = Y - R - 4;  // window origin (multiple of 4)

  // ---- stage the reference window and the current MB --------------------
  // A window inside the plane needs no clamping: one TMA box of WP rows of
  // BW bytes from column ox - 12 (a multiple of 16: ox = X - R - 4 with X a
  // multiple of 16 and R 16 or 32); the bytes either side of the window in
  // the box are never read.
  const bool tma = tma_ok && ox >= 0 && ox + WP <= g.RW && oy >= 0 && oy + WP <= g.RH;
  if (tma) {
    if (tid == 0) {
      mbar_arrive_expect_tx(&sh.bar, (uint32_t)(S::BW * WP));
      tma_load_2d(sh.win, &tmap, ox - 4 * OFF, oy, &sh.bar);
    }
  } else {
    for (int i = tid; i < WP * WW; i += NT) {
      const int row = i / WW, w = i - row * WW;
      const int gy = clampi(oy + row, 0, g.RH - 1);
      sh.win[row * WS + OFF + w] = load_word_clamped(ref + (size_t)gy * ref_pitch, ox + 4 * w, g.RW);
    }
  }
  for (int i = tid; i < 64; i += NT) {
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
  bool waited = true;
  if (tma) {
    waited = mbar_wait(&sh.bar, phase, kWaitNs);
    phase ^= 1u;
  }
  if (__syncthreads_or(!waited)) {
    // the window never arrived: report, give the copy one more bounded
    // wait, leave this CTA's remaining macroblocks unwritten
    if (tid == 0) {
      uint32_t* e = err ? err : &g_me_wait_err;
      if (atomicCAS(e, 0u, kErrWaitTimeout) == 0u && err) atomicExch(err + 1, (uint32_t)(mby * g.mbw + mbx));
      *o = MV{0, 0, 0xffffffffu, 0u};
      mbar_wait(&sh.bar, phase ^ 1u, kWaitNs);
    }
    return;
  }

  // ---- zero-MV check (motion_estimation.comp:312-331) --------------------
  uint32_t z = 0;
  for (int i = tid; i < 64; i += NT) {
    const int r = i >> 2, w = i & 3;
    z = sad4_acc(sh.cur[i], sh.win[(R + 4 + r) * WS + OFF + (R + 4) / 4 + w], z);
  }
  const uint32_t sad0 = block_sum<NT>(z, sh.red);
  if (zero_thresh >= 0 && sad0 <= (uint32_t)zero_thresh) {
    if (tid == 0) *o = MV{0, 0, sad0, (flags & B200ENC_ME_LOG_INTEGER) ? me_log_word(0, 0, true) : 0u};
    continue;
  }

  // ---- integer full search: column sweep ---------------------------------
  uint32_t cw[16][4];
#pragma unroll
  for (int r = 0; r < 16; ++r)
#pragma unroll
    for (int w = 0; w < 4; ++w) cw[r][w] = sh.cur[r * 4 + w];

  const int dx = tid - R;
  const int col = tid + 4;  // window byte column of candidate dx
  const int wb = col >> 2, shft = (col & 3) * 8;
  const uint32_t lam_dx = (uint32_t)lambda * (uint32_t)abs(dx);
  uint32_t acc[16];
#pragma unroll
  for (int s = 0; s < 16; ++s) acc[s] = 0;
  uint32_t best = 0xffffffffu;
  constexpr int G = (2 * R + 16) / 16;
  for (int gi = 0; gi < G; ++gi) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const int wrow = gi * 16 + k;
      const uint32_t* rowp = sh.win + (4 + wrow) * WS + OFF + wb;
      const uint32_t w0 = rowp[0], w1 = rowp[1], w2 = rowp[2], w3 = rowp[3], w4 = rowp[4];
      const uint32_t r0 = __funnelshift_r(w0, w1, shft), r1 = __funnelshift_r(w1, w2, shft);
      const uint32_t r2 = __funnelshift_r(w2, w3, shft), r3 = __funnelshift_r(w3, w4, shft);
#pragma unroll
      for (int r = 0; r < 16; ++r) {
        uint32_t a = acc[(k - r) & 15];
        a = sad4_acc(r0, cw[r][0], a);
        a = sad4_acc(r1, cw[r][1], a);
        a = sad4_acc(r2, cw[r][2], a);
        a = sad4_acc(r3, cw[r][3], a);
        acc[(k - r) & 15] = a;
      }
      // slot (k+1)&15 now holds the finished candidate cy = wrow - 15
      const int cy = wrow - 15;
      const int sl = (k + 1) & 15;
      if (cy >= 0) {
        const uint32_t cost = acc[sl] + lam_dx + (uint32_t)lambda * (uint32_t)abs(cy - R);
        best = min(best, (cost << 14) | (uint32_t)(cy * SIDE + tid));
      }
      acc[sl] = 0;
    }
  }
  // column dx = +R (aligned), candidates cy = tid and, for thread 0, cy = 2R
  for (int cy = tid; cy <= 2 * R; cy += NT) {
    uint32_t s = 0;
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      const uint32_t* rowp = sh.win + (4 + cy + r) * WS + OFF + (2 * R + 4) / 4;
      s = sad4_acc(rowp[0], cw[r][0], s);
      s = sad4_acc(rowp[1], cw[r][1], s);
      s = sad4_acc(rowp[2], cw[r][2], s);
      s = sad4_acc(rowp[3], cw[r][3], s);
    }
    const uint32_t cost = s + (uint32_t)lambda * (uint32_t)(R + abs(cy - R));
    best = min(best, (cost << 14) | (uint32_t)(cy * SIDE + 2 * R));
  }
  best = block_min<NT>(best, sh.red);
  const int idx = (int)(best & 0x3fffu);
  const int mx = idx % SIDE - R, my = idx / SIDE - R;
  const uint32_t int_sad = (best >> 14) - (uint32_t)lambda * (uint32_t)(abs(mx) + abs(my));

  // ---- half/quarter-pel refine around the winner -------------------------
  const uint8_t* wb8 = reinterpret_cast<const uint8_t*>(sh.win) + 4 * OFF;
  const int px0 = mx + R + 4, py0 = my + R + 4;  // window coords of the winner
  auto G8 = [&](int rx, int ry) -> int { return wb8[(py0 + ry) * S::BW + px0 + rx]; };
  int qx, qy;
  const uint32_t bsad =
      qpel_refine<NT>(sh.rf, G8, reinterpret_cast<const uint8_t*>(sh.cur), int_sad, &qx, &qy);
  if (tid == 0)
    *o = MV{4 * mx + qx, 4 * my + qy, bsad, (flags & B200ENC_ME_LOG_INTEGER) ? me_log_word(mx, my, false) : 0u};
  }
}

}  // namespace b200enc

using namespace b200enc;

namespace {

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = []() -> EncodeTiledFn {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

// Tensor map of a reference luma plane (RW x RH bytes, `pitch` apart) whose
// box is one search window of range R: MeShared<R>::BW bytes by WP rows.
// False when TMA cannot describe the plane (base or pitch not 16-byte
// aligned, a plane smaller than the box), the plane is not device memory
// (page-locked or managed host memory is staged with loads), or staging by
// TMA is tuned off; the kernel then stages every window with loads.
template <int R>
bool window_map(CUtensorMap* m, const uint8_t* ref, int pitch, int RW, int RH) {
  using S = MeShared<R>;
  memset(m, 0, sizeof(*m));
  if (b200enc_tuned(B200ENC_TUNE_ME_STAGE) == 1) return false;
  if ((reinterpret_cast<uintptr_t>(ref) & 15) || (pitch & 15) || RW < S::BW || RH < S::WP) return false;
  cudaPointerAttributes pa;
  if (cudaPointerGetAttributes(&pa, ref) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (pa.type != cudaMemoryTypeDevice) return false;
  EncodeTiledFn fn = encode_tiled();
  if (!fn) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)RW, (cuuint64_t)RH};
  const cuuint64_t strides[1] = {(cuuint64_t)pitch};
  const cuuint32_t box[2] = {(cuuint32_t)S::BW, (cuuint32_t)S::WP};
  const cuuint32_t estr[2] = {1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<uint8_t*>(ref), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int R>
void launch_frame(dim3 grid, bool list, const uint8_t* cur_y, int cur_pitch, const uint8_t* ref_y, int ref_pitch,
                  const Geo& g, int lambda, int zero_thresh, MV* out, const int* mb_list, const int* mb_count,
                  int flags, uint32_t* err, cudaStream_t st) {
  CUtensorMap map;
  const int use_tma = window_map<R>(&map, ref_y, ref_pitch, g.RW, g.RH) ? 1 : 0;
  const BatchTab none{};
  if (list)
    me_full_search_kernel<R, kMeList><<<grid, 2 * R, 0, st>>>(cur_y, cur_pitch, ref_y, ref_pitch, g, lambda,
                                                              zero_thresh, out, mb_list, mb_count, flags, none, map,
                                                              use_tma, err);
  else
    me_full_search_kernel<R, kMeGrid><<<grid, 2 * R, 0, st>>>(cur_y, cur_pitch, ref_y, ref_pitch, g, lambda,
                                                              zero_thresh, out, mb_list, mb_count, flags, none, map,
                                                              use_tma, err);
}

}  // namespace

// b200enc_me_full_search_ex with the error word of a wavefront scratch
// region: a window copy that never completes sets err[0] (kErrWaitTimeout)
// and err[1] (the macroblock). err == nullptr: the library's own word, read
// by b200enc_me_wait_errors.
int b200enc_me_full_search_err(const uint8_t* cur_y, int cur_pitch, const uint8_t* ref_y, int ref_pitch, int W,
                               int H, int RW, int RH, int range, int lambda, int zero_thresh, void* mv_out,
                               const int* mb_list, const int* mb_count, int list_capacity, int flags, uint32_t* err,
                               cudaStream_t st) {
  if (!cur_y || !ref_y || !mv_out || W <= 0 || H <= 0 || RW <= 0 || RH <= 0) return -1;
  if ((cur_pitch & 3) || (ref_pitch & 3) || (((uintptr_t)cur_y) & 3) || (((uintptr_t)ref_y) & 3)) return -1;
  if (lambda < 0 || lambda > 1023) return -1;
  if ((mb_list == nullptr) != (mb_count == nullptr)) return -1;
  Geo g{W, H, RW, RH, (W + 15) / 16, (H + 15) / 16};
  if (mb_list && (list_capacity <= 0 || list_capacity > g.mbw * g.mbh)) return -1;
  int sms = 148, dev = 0;
  if (mb_list && cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // list mode: a persistent grid of up to 8 CTAs per SM (or the tuned
  // count) walks the list
  const int per_sm = b200enc_tuned(B200ENC_TUNE_FALLBACK_CTAS_PER_SM) > 0 ? b200enc_tuned(B200ENC_TUNE_FALLBACK_CTAS_PER_SM) : 8;
  dim3 grid = mb_list ? dim3(std::min(list_capacity, per_sm * sms)) : dim3(g.mbw, g.mbh);
  const bool list = mb_list != nullptr;
  switch (range) {
    case 16:
      launch_frame<16>(grid, list, cur_y, cur_pitch, ref_y, ref_pitch, g, lambda, zero_thresh, (MV*)mv_out, mb_list,
                       mb_count, flags, err, st);
      break;
    case 32:
      launch_frame<32>(grid, list, cur_y, cur_pitch, ref_y, ref_pitch, g, lambda, zero_thresh, (MV*)mv_out, mb_list,
                       mb_count, flags, err, st);
      break;
    default:
      return -1;
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int b200enc_me_full_search_ex(const uint8_t* cur_y, int cur_pitch, const uint8_t* ref_y, int ref_pitch,
                                         int W, int H, int RW, int RH, int range, int lambda, int zero_thresh,
                                         void* mv_out, const int* mb_list, const int* mb_count, int list_capacity,
                                         int flags, void* stream) {
  return b200enc_me_full_search_err(cur_y, cur_pitch, ref_y, ref_pitch, W, H, RW, RH, range, lambda, zero_thresh,
                                    mv_out, mb_list, mb_count, list_capacity, flags, nullptr, (cudaStream_t)stream);
}

extern "C" int b200enc_me_full_search(const uint8_t* cur_y, int cur_pitch, const uint8_t* ref_y, int ref_pitch,
                                      int W, int H, int RW, int RH, int range, int lambda, int zero_thresh,
                                      void* mv_out, void* stream) {
  return b200enc_me_full_search_ex(cur_y, cur_pitch, ref_y, ref_pitch, W, H, RW, RH, range, lambda, zero_thresh,
                                   mv_out, nullptr, nullptr, 0, 0, stream);
}

extern "C" int b200enc_me_wait_errors(int clear) {
  uint32_t v = 0;
  if (cudaMemcpyFromSymbol(&v, g_me_wait_err, 4) != cudaSuccess) return -1;
  if (clear && v) {
    const uint32_t zero = 0;
    if (cudaMemcpyToSymbol(g_me_wait_err, &zero, 4) != cudaSuccess) return -1;
  }
  return (int)v;
}

// Batched full search: every P macroblock of a batch (list == nullptr: a
// persistent grid of `ctas` CTAs over the compact P index), or the compact
// indices of a list (the learned form's fallback). MVs go to bt.mvc.
int b200enc_me_batch_launch(const BatchTab& bt, int range, const int* list, const int* count, int ctas,
                            cudaStream_t st) {
  if (ctas <= 0) return -1;
  CUtensorMap none;
  memset(&none, 0, sizeof(none));
  switch (range) {
    case 16:
      if (list)
        me_full_search_kernel<16, kMeBatchList><<<ctas, 32, 0, st>>>(nullptr, 0, nullptr, 0, Geo{}, 0, 0, nullptr,
                                                                     list, count, 0, bt, none, 0, nullptr);
      else
        me_full_search_kernel<16, kMeBatch><<<ctas, 32, 0, st>>>(nullptr, 0, nullptr, 0, Geo{}, 0, 0, nullptr, nullptr,
                                                                 nullptr, 0, bt, none, 0, nullptr);
      break;
    case 32:
      if (list)
        me_full_search_kernel<32, kMeBatchList><<<ctas, 64, 0, st>>>(nullptr, 0, nullptr, 0, Geo{}, 0, 0, nullptr,
                                                                     list, count, 0, bt, none, 0, nullptr);
      else
        me_full_search_kernel<32, kMeBatch><<<ctas, 64, 0, st>>>(nullptr, 0, nullptr, 0, Geo{}, 0, 0, nullptr, nullptr,
                                                                 nullptr, 0, bt, none, 0, nullptr);
      break;
    default:
      return -1;
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
