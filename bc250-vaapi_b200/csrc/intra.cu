// intra.cu - I-frame intra wavefront as ONE persistent kernel.
//
// Reference: A1/shaders/intra_wavefront.comp:398-756, dispatched once per
// anti-diagonal with a barrier between dispatches (A1/src/gpu_compute.c:
// 3238-3249: 187 dispatches for a 1080p frame). An I16x16 macroblock needs
// only its left, top and top-left neighbours' reconstruction, so here each
// CTA takes a whole macroblock row by ticket (atomicAdd; a ticket is only
// taken by a running CTA, so rows are always owned by resident CTAs and the
// wait below cannot deadlock whatever the grid size), walks it left to
// right, and before macroblock x waits until row y-1 has published
// progress > x. Waits are bounded: on timeout the CTA records an error in
// the scratch and returns; every waiter also gives up as soon as it sees a
// recorded error.
//
// Within a macroblock the work is the reference's, laid out for warps:
// three compute warps, each 4x4 block owned by a lane quad (luma blocks in
// warps 0-1, chroma in warp 2), the 4x4 luma DC Hadamard as butterfly
// stages over 16 lanes. Two more warps keep the row-to-row handoff off the
// compute warps' path: a loader warp waits for the row above's progress
// and fetches the next macroblocks' top lines into a two-slot buffer ahead
// of use, and a publisher warp stores each macroblock's levels and
// reconstruction (kept in two-slot shared buffers), fences them and
// publishes the row's progress, while the compute warps go on with the
// next macroblock. The
// compute warps synchronise among themselves with a named barrier (96
// threads); the five warps meet only at the start and end of a row.
#include "b200enc_internal.h"
#include "common.cuh"

namespace b200enc {

struct IShared {
  int top[16], left[16], corner;
  alignas(16) uint8_t topv[2][16];  // row Y-1 from X (luma), raw; slot mbx & 1 (loader warp)
  alignas(16) uint8_t topc[2][16];  // row Yc-1 from 2*Xc (NV12 pairs), raw
  int prev_top15;                   // byte 15 of the previous MB's topv: the corner of this MB
  int top_ready;                    // top lines loaded for MBs < top_ready (loader)
  int top_used;                     // top-line slots of MBs < top_used consumed (compute)
  int stored;                       // levels and reconstruction of MBs < stored complete (compute)
  int published;                    // progress published for MBs < published (publisher)
  int tuv[2][8], luv[2][8];
  int sad[4][3];
  int dcv, pa, pb, pc;
  int row;
  int abort_flag;
  int16_t src[16][16];
  int16_t srcc[2][8][8];
  int cpred[8];                     // chroma DC predictor of blocks 16..23
  alignas(16) int16_t lev[2][24][16];  // slot mbx & 1: written by the compute warps, stored by the publisher
  int32_t ldc[16];     // pre-quant luma DC coefficients (block raster)
  int32_t ldl[16];     // quantized luma DC (natural order)
  int32_t ldcval[16];  // dequantized luma DC per block
  int32_t cdc[8];
  int32_t cdcval[8];
  alignas(16) uint8_t ry[2][16][16];  // slot mbx & 1 (the next MB's left neighbour, the publisher's source)
  alignas(16) uint8_t ruv[2][8][16];
};

__device__ __forceinline__ int hsign(int row, int idx) {
  // sign of element idx in row `row` of the butterfly used by
  // luma_dc_hadamard (A1/src/encoder_h264.c:711-730): rows
  // [+ + + +], [+ + - -], [+ - - +], [+ - + -]
  const int m = row == 0 ? 0x0 : (row == 1 ? 0xC : (row == 2 ? 0x6 : 0xA));
  return ((m >> idx) & 1) ? -1 : 1;
}

// BATCH: the row tickets (bt.ticket[0]) run over the rows of every stream
// of a batch that codes an I frame; a row waits on its own stream's
// progress words (that stream's scratch). Tickets are taken in order and a
// row only waits on an earlier row of its stream, so every wait is on a row
// some running CTA owns.
template <bool BATCH>
__global__ void __launch_bounds__(160, 1) i_frame_kernel(const uint8_t* __restrict__ cur_y_,
                                                     const uint8_t* __restrict__ cur_uv_, int cur_pitch_, Geo g_,
                                                     int qp_, int num_slices_, int16_t* __restrict__ levels_,
                                                     int32_t* __restrict__ dc_, uint32_t* __restrict__ nzm_,
                                                     uint32_t* __restrict__ pred_mode_, MV* __restrict__ mvs_,
                                                     uint8_t* rec_y_, uint8_t* rec_uv_, int rec_pitch_,
                                                     uint32_t* scratch_, uint32_t max_wait, int flags_, BatchTab bt) {
  __shared__ IShared s;
  const int tid = threadIdx.x;
  const int b = tid >> 2, r = tid & 3;
  const bool luma = b < 16;

  // the compute warps' barrier (named barrier 1, warps 0-2)
  auto csync = []() { asm volatile("bar.sync 1, 96;" ::: "memory"); };
  auto vload = [](const int& w) { return *reinterpret_cast<const volatile int*>(&w); };
  // acquire load of a shared word: orders this thread's later accesses
  // after it without waiting for its earlier ones (a fence would wait for
  // the source prefetch in flight)
  auto aload = [](const int& w) {
    int v;
    asm volatile("ld.acquire.cta.shared::cta.b32 %0, [%1];" : "=r"(v)
                 : "r"(static_cast<uint32_t>(__cvta_generic_to_shared(&w)))
                 : "memory");
    return v;
  };
  // release of a shared word: a block-scope fence, then the store. The
  // compute warps' writer is kSyncTid, a thread that never stores to global
  // memory, so its fence has nothing in flight to wait for.
  auto vstore = [](int& w, int v) {
    __threadfence_block();
    *reinterpret_cast<volatile int*>(&w) = v;
  };
  constexpr int kSyncTid = 73;  // warp 2, quad row 1: no global stores, only the source prefetch

  for (;;) {
    if (tid == 0) {
      s.row = (int)atomicAdd(BATCH ? bt.ticket : Scratch{scratch_}.ticket(), 1u);
      s.abort_flag = 0;
      s.top_ready = s.top_used = s.stored = s.published = 0;
    }
    __syncthreads();
    const uint8_t *cur_y = cur_y_, *cur_uv = cur_uv_;
    int cur_pitch = cur_pitch_, qp = qp_, num_slices = num_slices_, rec_pitch = rec_pitch_, flags = flags_;
    Geo g = g_;
    int16_t* levels = levels_;
    int32_t* dc = dc_;
    uint32_t *nzm = nzm_, *pred_mode = pred_mode_, *scratch = scratch_;
    MV* mvs = mvs_;
    uint8_t *rec_y = rec_y_, *rec_uv = rec_uv_;
    int mby = s.row;
    if (BATCH) {
      if (mby >= bt.i_rows.total()) return;
      const int k = bt.i_rows.find(mby);
      const BatchStream& st = bt.i_rows.stream(k);
      mby -= bt.i_rows.prefix[k];
      g = st.g;
      cur_y = st.cur_y;
      cur_uv = st.cur_uv;
      cur_pitch = st.cur_pitch;
      qp = st.qp;
      num_slices = st.num_slices;
      flags = st.intra_flags;
      levels = st.levels;
      dc = st.dc;
      nzm = st.nz;
      pred_mode = st.pred_mode;
      mvs = st.mv;
      rec_y = st.rec_y;
      rec_uv = st.rec_uv;
      rec_pitch = st.rec_pitch;
      scratch = st.scr_intra;
    } else if (mby >= g.mbh) {
      return;
    }
    const Scratch sc{scratch};
    const QP ql = make_qp(qp, true), qc = make_qp(chroma_qp(qp), true);
    const QP& q = luma ? ql : qc;
    const int rmx = g.RW - 1, rmy = g.RH - 1, cmx = g.RW / 2 - 1, cmy = g.RH / 2 - 1;
    const bool src_vec = ((cur_pitch & 3) == 0) && ((reinterpret_cast<uintptr_t>(cur_y) & 3) == 0) &&
                         ((reinterpret_cast<uintptr_t>(cur_uv) & 3) == 0);
    // Source words of macroblock mbx: thread t < 64 holds luma row t/4, word
    // t%4; threads 64..95 chroma row (t-64)/4, word (t-64)%4 (NV12 pairs).
    // Read one macroblock ahead, off the row's dependency chain.
    auto src_word = [&](int mbx_) -> uint32_t {
      const int Xs = mbx_ * 16, Ys = mby * 16;
      if (tid < 64) {
        const int row = tid >> 2, gx = Xs + 4 * (tid & 3);
        const uint8_t* rp = cur_y + (size_t)clampi(Ys + row, 0, g.H - 1) * cur_pitch;
        if (src_vec && gx + 4 <= g.W) return __ldg(reinterpret_cast<const uint32_t*>(rp + gx));
        uint32_t w = 0;
        for (int k = 0; k < 4; ++k) w |= (uint32_t)__ldg(rp + clampi(gx + k, 0, g.W - 1)) << (8 * k);
        return w;
      }
      const int i = tid - 64, row = i >> 2, pair = (Xs >> 1) + 2 * (i & 3);
      const uint8_t* rp = cur_uv + (size_t)clampi((Ys >> 1) + row, 0, g.H / 2 - 1) * cur_pitch;
      if (src_vec && pair + 2 <= g.W / 2) return __ldg(reinterpret_cast<const uint32_t*>(rp + 2 * pair));
      uint32_t w = 0;
      for (int k = 0; k < 4; ++k) w |= (uint32_t)__ldg(rp + 2 * clampi(pair + (k >> 1), 0, g.W / 2 - 1) + (k & 1)) << (8 * k);
      return w;
    };
    const uint64_t budget = (uint64_t)max_wait * 1000u;  // max_wait in microseconds
    // Bounded wait of one lane on a shared word (written by another warp of
    // this CTA after a block-scope fence): false on timeout (error recorded)
    // or when a wait elsewhere in the CTA gave up. The acquire load orders
    // this thread's later reads after the writer's earlier writes.
    auto wait_local = [&](const int& w, int need, uint32_t where) -> bool {
      const uint64_t t0 = global_ns();
      for (uint32_t it = 0;; ++it) {
        if (aload(w) >= need) return true;
        if (vload(s.abort_flag)) return false;
        if ((it & 15) == 15 && global_ns() - t0 > budget) {
          if (atomicCAS(sc.err(), 0u, kErrWaitTimeout) == 0u) atomicExch(sc.err_detail(), where);
          vstore(s.abort_flag, 1);
          return false;
        }
        if (it > 16) __nanosleep(32);
      }
    };
    if (tid >= 96) {
      const int lane = tid & 31;
      if (tid < 128) {
        // ---- loader warp: the row above's bottom lines, ahead of use -------
        if (lane == 0) {
          if (mby == 0) {
            vstore(s.top_ready, g.mbw);  // no top neighbour: nothing to load
          } else {
            const uint32_t* pf_row = sc.progress(mby - 1);
            for (int m = 0; m < g.mbw; ++m) {
              const int X = m * 16, Y = mby * 16, Yc = Y >> 1;
              const uint64_t t0 = global_ns();
              bool ok = false;
              for (uint32_t it = 0;; ++it) {
                if (load_acquire(pf_row) >= (uint32_t)(m + 1)) { ok = true; break; }
                if (load_acquire(sc.err()) != 0u || vload(s.abort_flag)) break;
                if ((it & 15) == 15 && global_ns() - t0 > budget) {
                  if (atomicCAS(sc.err(), 0u, kErrWaitTimeout) == 0u)
                    atomicExch(sc.err_detail(), (uint32_t)(mby * g.mbw + m));
                  break;
                }
                if (it > 16) __nanosleep(32);
              }
              // the slot's previous macroblock (m - 2) has been read
              if (!ok || !wait_local(s.top_used, m - 1, (uint32_t)(mby * g.mbw + m))) {
                vstore(s.abort_flag, 1);
                break;
              }
              // 16-byte lines: row Y-1 from X, chroma row Yc-1 from 2*Xc
              // (inside the picture's coded width; clamping applies when they
              // are read)
              *reinterpret_cast<uint4*>(s.topv[m & 1]) =
                  __ldcg(reinterpret_cast<const uint4*>(rec_y + (size_t)(Y - 1) * rec_pitch + X));
              *reinterpret_cast<uint4*>(s.topc[m & 1]) =
                  __ldcg(reinterpret_cast<const uint4*>(rec_uv + (size_t)(Yc - 1) * rec_pitch + X));
              vstore(s.top_ready, m + 1);
            }
          }
        }
      } else {
        // ---- publisher warp: the macroblock's levels and reconstruction to
        //      memory, fence, progress ----------------------------------------
        // The row below reads only each macroblock's bottom luma and chroma
        // lines (and, through its corner, those of the macroblock before);
        // every lane fences its own stores and lane 0 publishes after the
        // warp has met, so the progress word follows them.
        for (int m = 0; m < g.mbw; ++m) {
          int go = 0;
          if (lane == 0) go = wait_local(s.stored, m + 1, (uint32_t)(mby * g.mbw + m)) ? 1 : 0;
          if (!__shfl_sync(0xffffffffu, go, 0)) break;
          __syncwarp();           // orders lane 0's acquire before the other lanes' reads
          (void)aload(s.stored);  // and each lane acquires the word lane 0 saw
          const int sl = m & 1, X = m * 16, Y = mby * 16, Yc = Y >> 1, mbi = mby * g.mbw + m;
          for (int i = lane; i < 48; i += 32)
            reinterpret_cast<uint4*>(levels + (size_t)mbi * 384)[i] = reinterpret_cast<const uint4*>(&s.lev[sl][0][0])[i];
          if (lane < 16) {
            const int gy = Y + lane;
            if (gy <= rmy) {
              uint8_t* dst = rec_y + (size_t)gy * rec_pitch + X;
              if (X + 16 <= g.RW) __stcg(reinterpret_cast<uint4*>(dst), *reinterpret_cast<const uint4*>(s.ry[sl][lane]));
              else
                for (int c = 0; c < 16 && X + c < g.RW; ++c) dst[c] = s.ry[sl][lane][c];
            }
          } else if (lane < 24) {
            const int row = lane - 16, gy = Yc + row;
            if (gy <= cmy) {
              uint8_t* dst = rec_uv + (size_t)gy * rec_pitch + X;
              if ((X >> 1) + 8 <= cmx + 1) __stcg(reinterpret_cast<uint4*>(dst), *reinterpret_cast<const uint4*>(s.ruv[sl][row]));
              else
                for (int c = 0; c < 8 && (X >> 1) + c <= cmx; ++c) {
                  dst[2 * c] = s.ruv[sl][row][2 * c];
                  dst[2 * c + 1] = s.ruv[sl][row][2 * c + 1];
                }
            }
          }
          __threadfence();
          __syncwarp();
          if (lane == 0) {
            store_release(sc.progress(mby), (uint32_t)(m + 1));
            vstore(s.published, m + 1);
          }
        }
      }
      __syncthreads();  // the row's end: all five warps
      if (s.abort_flag) return;
      continue;
    }

    uint32_t pf = src_word(0);
    for (int mbx = 0; mbx < g.mbw; ++mbx) {
      const int mb = mby * g.mbw + mbx, X = mbx * 16, Y = mby * 16, Xc = X >> 1, Yc = Y >> 1;
      const uint32_t total = (uint32_t)(g.mbw * g.mbh);
      const uint32_t sl = slice_of((uint32_t)mb, total, (uint32_t)num_slices);
      const bool top_exists = mby > 0, left_exists = mbx > 0;
      const bool top_av = top_exists && slice_of((uint32_t)(mb - g.mbw), total, (uint32_t)num_slices) == sl;
      const bool left_av = left_exists && slice_of((uint32_t)(mb - 1), total, (uint32_t)num_slices) == sl;
      // Plane also predicts from the top-left sample; with the corner check
      // it needs the top-left macroblock in this slice as well (the
      // reference shader checks only top and left).
      const bool plane_av = top_av && left_av &&
                            (!(flags & B200ENC_INTRA_CORNER_CHECK) ||
                             slice_of((uint32_t)(mb - g.mbw - 1), total, (uint32_t)num_slices) == sl);
      // ---- this MB's source (prefetched), the next MB's source requested --
      {
        const uint32_t w = pf;
        if (tid < 64) {
          const int row = tid >> 2, c0 = 4 * (tid & 3);
#pragma unroll
          for (int k = 0; k < 4; ++k) s.src[row][c0 + k] = (int16_t)((w >> (8 * k)) & 255u);
        } else {
          const int i = tid - 64, row = i >> 2, x0 = 2 * (i & 3);
          s.srcc[0][row][x0] = (int16_t)(w & 255u);
          s.srcc[1][row][x0] = (int16_t)((w >> 8) & 255u);
          s.srcc[0][row][x0 + 1] = (int16_t)((w >> 16) & 255u);
          s.srcc[1][row][x0 + 1] = (int16_t)(w >> 24);
        }
        if (mbx + 1 < g.mbw) pf = src_word(mbx + 1);
      }
      const int slot = mbx & 1;  // this MB's top-line, level and reconstruction slots
      // ---- left and corner neighbours: this CTA's own previous MB --------
      // (still in s.ry / s.ruv; rows past the clamp limit read its last row,
      // as the clamped reads of the reference do)
      if (tid < 16) {
        s.left[tid] = left_exists ? s.ry[slot ^ 1][min(tid, rmy - Y)][15] : 128;
      } else if (tid < 32) {
        const int i = tid - 16, pl = i >> 3, k = i & 7;
        s.luv[pl][k] = left_av ? s.ruv[slot ^ 1][min(k, cmy - Yc)][14 + pl] : 128;
      } else if (tid == 32) {
        s.corner = (top_exists && left_exists) ? s.prev_top15 : 128;
      }
      // ---- the top neighbour's bottom lines, loaded ahead by the loader ---
      if (tid == kSyncTid) {
        if (mby > 0) wait_local(s.top_ready, mbx + 1, (uint32_t)mb);
        wait_local(s.published, mbx - 1, (uint32_t)mb);  // the slots of MB mbx - 2 are stored
      }
      csync();
      if (vload(s.abort_flag)) break;

      // ---- top lines, I16x16 candidates (intra_wavefront.comp:454-476),
      //      chroma DC predictors --------------------------------------------
      // Warp 0 spreads the luma top line and forms the candidate sums from
      // registers and shuffles (lane sums without divergence: every lane
      // loads, lanes outside a term contribute 0); warp 2 spreads the chroma
      // top line and forms the chroma DC predictors (intra_wavefront.comp:
      // 612-641).
      if (tid < 32) {
        const int t = tid & 15, k = tid & 7;
        const int tv = top_exists ? s.topv[slot][min(t, rmx - X)] : 128;
        const int lv = s.left[t];
        if (tid < 16) s.top[tid] = tv;
        const int t6 = __shfl_sync(0xffffffffu, tv, (6 - k) & 15), t8 = __shfl_sync(0xffffffffu, tv, 8 + k);
        const int lt = k <= 6 ? t6 : s.corner, la = k <= 6 ? s.left[6 - k] : s.corner;
        const int st = __reduce_add_sync(0xffffffffu, tid < 16 ? tv : 0);
        const int sl2 = __reduce_add_sync(0xffffffffu, tid < 16 ? lv : 0);
        const int hterm = __reduce_add_sync(0xffffffffu, tid < 8 ? (k + 1) * (t8 - lt) : 0);
        const int vterm = __reduce_add_sync(0xffffffffu, tid < 8 ? (k + 1) * (s.left[8 + k] - la) : 0);
        const int t15 = __shfl_sync(0xffffffffu, tv, 15);
        if (tid == 0) {
          int dcv;
          if (top_av && left_av) dcv = (st + sl2 + 16) >> 5;
          else if (top_av) dcv = (st + 8) >> 4;
          else if (left_av) dcv = (sl2 + 8) >> 4;
          else dcv = 128;
          s.dcv = dcv;
          if (plane_av) {
            s.pa = 16 * (s.left[15] + t15);
            s.pb = (5 * hterm + 32) >> 6;
            s.pc = (5 * vterm + 32) >> 6;
          } else {
            s.pa = s.pb = s.pc = 0;
          }
          s.prev_top15 = s.topv[slot][15];  // read by the next MB's corner, after the barriers below
        }
      } else if (tid >= 64 && tid < 80) {
        const int i = tid - 64, pl = i >> 3, k = i & 7;
        s.tuv[pl][k] = top_av ? s.topc[slot][2 * min(k, cmx - Xc) + pl] : 128;
        __syncwarp(0x0000ffffu);
        if (i < 8) {
          const int pl2 = i >> 2, sub = i & 3;
          const int t0 = s.tuv[pl2][0] + s.tuv[pl2][1] + s.tuv[pl2][2] + s.tuv[pl2][3];
          const int t1 = s.tuv[pl2][4] + s.tuv[pl2][5] + s.tuv[pl2][6] + s.tuv[pl2][7];
          const int l0 = s.luv[pl2][0] + s.luv[pl2][1] + s.luv[pl2][2] + s.luv[pl2][3];
          const int l1 = s.luv[pl2][4] + s.luv[pl2][5] + s.luv[pl2][6] + s.luv[pl2][7];
          int v;
          if (sub == 0) v = (top_av && left_av) ? (t0 + l0 + 4) >> 3 : top_av ? (t0 + 2) >> 2 : left_av ? (l0 + 2) >> 2 : 128;
          else if (sub == 1) v = top_av ? (t1 + 2) >> 2 : left_av ? (l0 + 2) >> 2 : 128;
          else if (sub == 2) v = left_av ? (l1 + 2) >> 2 : top_av ? (t0 + 2) >> 2 : 128;
          else v = (top_av && left_av) ? (t1 + l1 + 4) >> 3 : top_av ? (t1 + 2) >> 2 : left_av ? (l1 + 2) >> 2 : 128;
          s.cpred[i] = v;  // the predictor of chroma block 16 + i
        }
      }
      csync();
      // the top-line slot has been read by both warps: free it for MB mbx + 2
      if (tid == kSyncTid) vstore(s.top_used, mbx + 1);

      // ---- the four I16x16 SADs -----------------------------------------
      {
        uint32_t sdc = 0, sv = 0, shh = 0, spl = 0;
        for (int i = tid; i < 256; i += 96) {
          const int x = i & 15, y = i >> 4, v = s.src[y][x];
          sdc += (uint32_t)abs(v - s.dcv);
          if (top_av) sv += (uint32_t)abs(v - s.top[x]);
          if (left_av) shh += (uint32_t)abs(v - s.left[y]);
          if (plane_av) spl += (uint32_t)abs(v - clip1((s.pa + s.pb * (x - 7) + s.pc * (y - 7) + 16) >> 5));
        }
        sdc = __reduce_add_sync(0xffffffffu, sdc);
        sv = __reduce_add_sync(0xffffffffu, sv);
        shh = __reduce_add_sync(0xffffffffu, shh);
        spl = __reduce_add_sync(0xffffffffu, spl);
        if ((tid & 31) == 0) {
          s.sad[0][tid >> 5] = (int)sdc;
          s.sad[1][tid >> 5] = (int)sv;
          s.sad[2][tid >> 5] = (int)shh;
          s.sad[3][tid >> 5] = (int)spl;
        }
      }
      csync();
      // ---- mode decision, taken by every thread from the same sums --------
      int mode;
      {
        const uint32_t sdc = s.sad[0][0] + s.sad[0][1] + s.sad[0][2], sv = s.sad[1][0] + s.sad[1][1] + s.sad[1][2];
        const uint32_t shh = s.sad[2][0] + s.sad[2][1] + s.sad[2][2], spl = s.sad[3][0] + s.sad[3][1] + s.sad[3][2];
        uint32_t best = sdc;
        mode = 2;
        if (top_av && sv < best) { best = sv; mode = 0; }
        if (left_av && shh < best) { best = shh; mode = 1; }
        if (plane_av && spl < best) { best = spl; mode = 3; }
      }
      if (tid == 0) {
        pred_mode[mb] = (uint32_t)mode;  // chroma mode bits 2-3 = 0 (DC)
        mvs[mb] = MV{0, 0, 0u, 0u};
      }
      // The prediction of this thread's block row, formed where it is used
      // (residual and reconstruction) instead of being stored: luma sample
      // (x, y) of the chosen mode, or the chroma block's DC predictor.
      const int dcv = s.dcv, pa = s.pa, pb = s.pb, pc = s.pc;
      auto luma_pred = [&](int x, int y) -> int {
        if (mode == 0) return s.top[x];
        if (mode == 1) return s.left[y];
        if (mode == 3) return clip1((pa + pb * (x - 7) + pc * (y - 7) + 16) >> 5);
        return dcv;
      };
      int pred_row[4];
      if (luma) {
        const int bx = b & 3, by = b >> 2;
#pragma unroll
        for (int i = 0; i < 4; ++i) pred_row[i] = luma_pred(4 * bx + i, 4 * by + r);
      } else {
        const int pv = s.cpred[b - 16];
#pragma unroll
        for (int i = 0; i < 4; ++i) pred_row[i] = pv;
      }

      // ---- forward + AC quant (position 0 is carried by the DC paths) ----
      int x[4];
      if (luma) {
        const int bx = b & 3, by = b >> 2;
#pragma unroll
        for (int i = 0; i < 4; ++i) x[i] = s.src[4 * by + r][4 * bx + i] - pred_row[i];
      } else {
        const int pl = (b - 16) >> 2, sub = (b - 16) & 3;
#pragma unroll
        for (int i = 0; i < 4; ++i) x[i] = s.srcc[pl][4 * (sub >> 1) + r][4 * (sub & 1) + i] - pred_row[i];
      }
      quad_forward(x, r);  // x[i] = coef[i][r]
      uint32_t nz = 0;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int pos = 4 * i + r;
        const int l = pos == 0 ? 0 : quant_ac(x[i], pos, q);
        s.lev[slot][b][pos] = (int16_t)clampi(l, -32768, 32767);
        nz |= (l != 0 ? 1u : 0u) << pos;
      }
      nz |= __shfl_xor_sync(0xffffffffu, nz, 1);
      nz |= __shfl_xor_sync(0xffffffffu, nz, 2);
      if (r == 0) {
        nzm[(size_t)mb * 24 + b] = nz;
        dc[(size_t)mb * 24 + b] = x[0];
        if (luma) s.ldc[b] = x[0];
        else s.cdc[b - 16] = x[0];
      }
      csync();

      // ---- DC paths ----------------------------------------------------
      // The luma DC transform (A1/src/encoder_h264.c:711-730) is a 2-D
      // Hadamard: out[i][k] = sum_ab h_k(a) h_i(b) in[a][b] (+1 >> 1 forward).
      // Lanes t = 4a + b of warp 0 hold in[a][b]; two butterfly stages along
      // b (xor 1, 2) and two along a (xor 4, 8) leave lane 4q + p with the
      // sum for the Walsh rows (p, q) in sequency order; h's rows are those
      // rows permuted (row 0 <- 0, 1 <- 2, 2 <- 3, 3 <- 1), so lane 4q + p
      // holds out[i][k] with i = kRow[p], k = kRow[q]. Integer sums: exact in
      // any order.
      auto dc_hadamard = [&](int v) -> int {
#pragma unroll
        for (int m = 1; m <= 8; m <<= 1) {
          const int o = __shfl_xor_sync(0x0000ffffu, v, m);
          v = (tid & m) ? o - v : v + o;
        }
        return v;
      };
      if (tid < 16) {
        const int row_of[4] = {0, 3, 1, 2};  // sequency index -> row of h
        const int i = row_of[tid & 3], k = row_of[tid >> 2];
        const int sum = dc_hadamard(s.ldc[tid]);
        s.ldl[4 * i + k] = quantize_dc((sum + 1) >> 1, ql);
      } else if (tid >= 64 && tid < 72) {
        // chroma DC of one plane per 4 lanes: lane o quantises Hadamard output
        // o, then forms inverse output o from the group's four levels
        const int j = tid - 64, pl = j >> 2, o = j & 3;
        const int c0 = s.cdc[4 * pl], c1 = s.cdc[4 * pl + 1], c2 = s.cdc[4 * pl + 2], c3 = s.cdc[4 * pl + 3];
        const int sb = (o & 1) ? -1 : 1, sc2 = (o & 2) ? -1 : 1;  // signs of c1/c3 and c2/c3
        const int lo = quantize_dc(c0 + sb * c1 + sc2 * c2 + sb * sc2 * c3, qc);
        const int g0 = __shfl_sync(0x000000ffu, lo, 4 * pl), g1 = __shfl_sync(0x000000ffu, lo, 4 * pl + 1);
        const int g2 = __shfl_sync(0x000000ffu, lo, 4 * pl + 2), g3 = __shfl_sync(0x000000ffu, lo, 4 * pl + 3);
        s.cdcval[4 * pl + o] = dequant_dc_chroma(g0 + sb * g1 + sc2 * g2 + sb * sc2 * g3, qc);
      }
      __syncwarp();
      if (tid < 16) {
        const int row_of[4] = {0, 3, 1, 2};
        const int i = row_of[tid & 3], k = row_of[tid >> 2];
        const int f = dc_hadamard(s.ldl[tid]);
        s.ldcval[4 * i + k] = dequant_dc_luma(f, ql);
      }
      csync();

      // ---- dequant + inverse + recon -----------------------------------
      int d[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) d[i] = dequant_ac(s.lev[slot][b][4 * r + i], 4 * r + i, q);
      if (r == 0) d[0] = (luma ? s.ldcval[b] : s.cdcval[b - 16]) + 32;
      quad_inverse(d, r);  // d[i] = res[i][r]: column r of the block
      if (luma) {
        const int bx = b & 3, by = b >> 2;
#pragma unroll
        for (int i = 0; i < 4; ++i)
          s.ry[slot][4 * by + i][4 * bx + r] = (uint8_t)clip1(luma_pred(4 * bx + r, 4 * by + i) + d[i]);
      } else {
        const int pl = (b - 16) >> 2, sub = (b - 16) & 3;
        const int pv = pred_row[0];
#pragma unroll
        for (int i = 0; i < 4; ++i)
          s.ruv[slot][4 * (sub >> 1) + i][2 * (4 * (sub & 1) + r) + pl] = (uint8_t)clip1(pv + d[i]);
      }
      csync();
      if (tid == kSyncTid) vstore(s.stored, mbx + 1);
    }
    __syncthreads();  // the row's end: all five warps
    if (s.abort_flag) return;
  }
}

}  // namespace b200enc

using namespace b200enc;

extern "C" size_t b200enc_wavefront_scratch_bytes(int mbh) { return scratch_words(mbh < 1 ? 1 : mbh) * sizeof(uint32_t); }

extern "C" int b200enc_wavefront_status(const void* scratch, void* stream) {
  if (!scratch) return -1;
  uint32_t e = 0;
  if (cudaMemcpyAsync(&e, (const uint32_t*)scratch + 1, sizeof(e), cudaMemcpyDeviceToHost, (cudaStream_t)stream) !=
      cudaSuccess)
    return -1;
  if (cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) return -1;
  return e == 0 ? 0 : 1;
}

// Time budget of one progress wait before a wavefront CTA gives up.
static constexpr uint32_t kMaxWaitUs = 2000000u;  // 2 s

extern "C" int b200enc_i_frame_launch(const uint8_t* cur_y, const uint8_t* cur_uv, int cur_pitch, int W, int H,
                                      int RW, int RH, int qp, int num_slices, int16_t* levels, int32_t* dc,
                                      uint32_t* nz, uint32_t* pred_mode, void* mv, uint8_t* rec_y, uint8_t* rec_uv,
                                      int rec_pitch, uint32_t* scratch, int ctas, uint32_t max_wait, int flags,
                                      void* stream) {
  Geo g{W, H, RW, RH, (W + 15) / 16, (H + 15) / 16};
  if (ctas <= 0) ctas = b200enc_tuned(B200ENC_TUNE_INTRA_CTAS);
  if (ctas <= 0) ctas = g.mbh;
  if (ctas > g.mbh) ctas = g.mbh;
  i_frame_kernel<false><<<ctas, 160, 0, (cudaStream_t)stream>>>(cur_y, cur_uv, cur_pitch, g, qp, num_slices, levels, dc,
                                                              nz, pred_mode, (MV*)mv, rec_y, rec_uv, rec_pitch,
                                                              scratch, max_wait, flags, BatchTab{});
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// The intra wavefront of every I-frame stream of a batch: `ctas` persistent
// CTAs over bt.i_rows (each stream's scratch zeroed and bt.ticket[0] = 0 by
// the caller).
int b200enc_i_frame_batch_launch(const BatchTab& bt, int ctas, uint32_t max_wait, cudaStream_t st) {
  if (ctas <= 0) return 0;
  i_frame_kernel<true><<<ctas, 160, 0, st>>>(nullptr, nullptr, 0, Geo{}, 0, 1, nullptr, nullptr, nullptr, nullptr,
                                            nullptr, nullptr, nullptr, 0, nullptr, max_wait, 0, bt);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int b200enc_i_frame(const uint8_t* cur_y, const uint8_t* cur_uv, int cur_pitch, int W, int H, int RW,
                               int RH, int qp, int num_slices, int16_t* levels, int32_t* dc, uint32_t* nz,
                               uint32_t* pred_mode, void* mv, uint8_t* rec_y, uint8_t* rec_uv, int rec_pitch,
                               void* scratch, size_t scratch_bytes, int ctas, int flags, void* stream) {
  if (!cur_y || !cur_uv || !levels || !dc || !nz || !pred_mode || !mv || !rec_y || !rec_uv || !scratch) return -1;
  if (qp < 0 || qp > 51 || W <= 0 || H <= 0 || RW <= 1 || RH <= 1 || num_slices < 1) return -1;
  if ((rec_pitch & 15) || (((uintptr_t)rec_y) & 15) || (((uintptr_t)rec_uv) & 15) || (((uintptr_t)levels) & 15))
    return -1;
  const int mbh = (H + 15) / 16;
  if (scratch_bytes < b200enc_wavefront_scratch_bytes(mbh)) return -1;
  if (cudaMemsetAsync(scratch, 0, b200enc_wavefront_scratch_bytes(mbh), (cudaStream_t)stream) != cudaSuccess) return -1;
  return b200enc_i_frame_launch(cur_y, cur_uv, cur_pitch, W, H, RW, RH, qp, num_slices, levels, dc, nz, pred_mode, mv,
                                rec_y, rec_uv, rec_pitch, (uint32_t*)scratch, ctas, kMaxWaitUs, flags, stream);
}
