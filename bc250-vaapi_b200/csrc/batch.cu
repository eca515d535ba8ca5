// batch.cu - many concurrent streams of uneven frame sizes through one launch
// per stage, each step (one frame of every stream) optionally replayed as a
// captured CUDA graph.
//
// The reference runs one Vulkan queue per VA context, one frame at a time
// (approach1-compute-encoder/src/gpu_compute.h:246-250). Here a batch owns
// the state of N streams (reconstructions, outputs, motion history,
// wavefront scratch, all in one device arena) and a step enqueues, on the
// batch's CUDA stream:
//   stream table H2D (one pinned copy), scratch clear (one memset),
//   ME over every P macroblock of every P stream (full search, or the
//   learned form: preparation, network, fallback search, re-scoring),
//   the P chain over the same macroblocks,
//   the intra wavefront over every I stream's macroblock rows,
//   the tile deblocking over every stream's tiles (out of place, into the
//   buffer of the previous reconstruction),
//   status words D2H.
// Every stage kernel is the single-frame kernel's body behind a stream
// lookup (binary search of the item in the set's prefix sums), so each
// stream's outputs equal what a single-stream context computes from the same
// frames.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <dlfcn.h>
#include <string>
#include <vector>

#include "b200enc_internal.h"
#include "common.cuh"

namespace {

using namespace b200enc;

constexpr uint32_t kBatchMaxWaitUs = 2000000u;

size_t up(size_t v, size_t a) { return (v + a - 1) / a * a; }
int pad16(int mbs) { return (mbs + 15) & ~15; }

struct StreamState {
  int W, H, mbw, mbh, pitch;
  size_t rec_bytes;
  uint8_t* rec[2];
  int cur;  // rec[cur] is the latest reconstruction
  bool has_recon, has_hist;
  int16_t* levels;
  int32_t* dc;
  uint32_t *nz, *pred_mode;
  MV* mv[2];
  int mv_cur;  // mv[mv_cur] is the latest field
  uint32_t *scr_intra, *scr_db;
};

// Device table layout (one allocation, mirrored by two pinned host copies):
//   BatchStream[n] | idx p[n] i[n] g[n] | prefix p[n+1] i[n+1] g[n+1] | status
struct TableLayout {
  size_t streams, idx_p, idx_i, idx_g, pre_p, pre_i, pre_g, bytes;
  explicit TableLayout(int n) {
    streams = 0;
    idx_p = up(sizeof(BatchStream) * n, 16);
    idx_i = idx_p + 4 * (size_t)n;
    idx_g = idx_i + 4 * (size_t)n;
    pre_p = up(idx_g + 4 * (size_t)n, 16);
    pre_i = pre_p + 4 * (size_t)(n + 1);
    pre_g = pre_i + 4 * (size_t)(n + 1);
    bytes = up(pre_g + 4 * (size_t)(n + 1), 256);
  }
};

struct Batch {
  int n = 0, range = 32, me_mode = 0, deblock = 1, device = 0, sms = 148;
  float conf = 0.9f;
  cudaStream_t stream = nullptr;
  std::vector<StreamState> ss;
  uint8_t* arena = nullptr;
  uint32_t* scratch = nullptr;  // every stream's two scratch regions + 2 tickets, contiguous
  size_t scratch_words = 0;
  uint32_t* status_host = nullptr;
  MV* mvc = nullptr;
  int total_mbs = 0, max_mbw = 0, max_mbh = 0;
  int db_tw = 8, db_th = 8;  // tile deblocking's tile shape, read from the tune table at each step
  TableLayout lay{1};
  uint8_t* dtab = nullptr;
  uint8_t* htab[2] = {nullptr, nullptr};
  cudaEvent_t htab_free[2] = {nullptr, nullptr};
  int htab_next = 0;
  void* prop = nullptr;
  bool graph = false;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t done = nullptr;
  bool pending = false;
  long graph_updates = 0, graph_instantiations = 0;
};

std::string weights_path() {
  Dl_info info;
  if (dladdr((void*)&weights_path, &info) && info.dli_fname) {
    std::string p = info.dli_fname;
    const size_t cut = p.find_last_of('/');
    p = (cut == std::string::npos) ? std::string(".") : p.substr(0, cut);
    return p + "/../b200enc/data/proposal_h264.b2pn";
  }
  return "proposal_h264.b2pn";
}

void destroy(Batch* b) {
  if (!b) return;
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->prop) b200enc_proposal_destroy(b->prop);
  cudaFree(b->arena);
  cudaFree(b->dtab);
  for (int i = 0; i < 2; ++i) {
    cudaFreeHost(b->htab[i]);
    if (b->htab_free[i]) cudaEventDestroy(b->htab_free[i]);
  }
  cudaFreeHost(b->status_host);
  if (b->done) cudaEventDestroy(b->done);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

// Everything one step enqueues, on b->stream (captured in graph mode).
// np/ni/ng: streams in the P, I and deblocking sets; n_p, n_irows, n_groups:
// their item counts.
int enqueue_step(Batch* b, const uint8_t* htab, int np, int ni, int ng, int n_p, int n_irows, int n_groups) {
  cudaStream_t st = b->stream;
  int rc = 0;
  rc |= cudaMemcpyAsync(b->dtab, htab, b->lay.bytes, cudaMemcpyHostToDevice, st) != cudaSuccess;
  rc |= cudaMemsetAsync(b->scratch, 0, b->scratch_words * 4, st) != cudaSuccess;
  BatchTab bt;
  const BatchStream* sd = reinterpret_cast<const BatchStream*>(b->dtab + b->lay.streams);
  auto set = [&](size_t idx, size_t pre, int n) {
    return BatchSet{sd, reinterpret_cast<const int*>(b->dtab + idx), reinterpret_cast<const int*>(b->dtab + pre), n};
  };
  const int kp = np, ki = ni, kg = ng;
  bt.p_mbs = set(b->lay.idx_p, b->lay.pre_p, kp);
  bt.i_rows = set(b->lay.idx_i, b->lay.pre_i, ki);
  bt.groups = set(b->lay.idx_g, b->lay.pre_g, kg);
  bt.mvc = b->mvc;
  bt.ticket = b->scratch + (b->scratch_words - 2);
  bt.db_rows = b->db_th;
  bt.db_cols = b->db_tw;
  if (n_p > 0) {
    if (b->me_mode == 0)
      rc |= b200enc_me_batch_launch(bt, b->range, nullptr, nullptr, n_p, st) != 0;
    else
      rc |= b200enc_proposal_me_batch(b->prop, bt, n_p, b->range, 5, b->me_mode, b->conf, st) != 0;
    rc |= b200enc_p_frame_batch_launch(bt, n_p, st) != 0;
  }
  if (n_irows > 0) rc |= b200enc_i_frame_batch_launch(bt, n_irows, kBatchMaxWaitUs, st) != 0;
  if (b->deblock && n_groups > 0)
    rc |= b200enc_deblock_tiles_batch_launch(bt, n_groups, kBatchMaxWaitUs, st) != 0;
  // status: error words of every stream's two scratch regions
  rc |= cudaMemcpyAsync(b->status_host, b->scratch, b->scratch_words * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess;
  return rc ? -1 : 0;
}

}  // namespace

extern "C" {

void* b200enc_batch_create(int n_streams, const int* widths, const int* heights, int search_range, int me_mode,
                           float conf, int deblock) {
  if (n_streams <= 0 || n_streams > 4096 || !widths || !heights) return nullptr;
  if ((search_range != 16 && search_range != 32) || (me_mode != 0 && me_mode != 1 && me_mode != 3)) return nullptr;
  Batch* b = new Batch();
  b->n = n_streams;
  b->range = search_range;
  b->me_mode = me_mode;
  b->conf = conf;
  b->deblock = deblock ? 1 : 0;
  if (cudaGetDevice(&b->device) != cudaSuccess ||
      cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) != cudaSuccess) {
    destroy(b);
    return nullptr;
  }
  b->ss.resize(n_streams);
  size_t bytes = 0, scr_words = 0;
  for (int s = 0; s < n_streams; ++s) {
    StreamState& t = b->ss[s];
    if (widths[s] <= 0 || heights[s] <= 0 || (widths[s] & 1) || (heights[s] & 1)) {
      destroy(b);
      return nullptr;
    }
    t.W = widths[s];
    t.H = heights[s];
    t.mbw = (t.W + 15) / 16;
    t.mbh = (t.H + 15) / 16;
    t.pitch = (int)up((size_t)t.mbw * 16, 128);
    t.rec_bytes = (size_t)t.pitch * t.mbh * 16 * 3 / 2;
    const size_t mbs = (size_t)t.mbw * t.mbh;
    bytes += 2 * up(t.rec_bytes, 256) + up(mbs * 768, 256) + 2 * up(mbs * 96, 256) + up(mbs * 4, 256) +
             2 * up(mbs * 16, 256);
    scr_words += 2 * scratch_words(t.mbh);
    b->total_mbs += pad16((int)mbs);  // the compact P index, tile-aligned per stream
    b->max_mbw = std::max(b->max_mbw, t.mbw);
    b->max_mbh = std::max(b->max_mbh, t.mbh);
  }
  b->scratch_words = scr_words + 2;  // + the two tickets
  bytes += up(b->scratch_words * 4, 256) + up((size_t)b->total_mbs * 16, 256);
  b->lay = TableLayout(n_streams);
  if (cudaMalloc(&b->arena, bytes) != cudaSuccess ||
      cudaMalloc(&b->dtab, b->lay.bytes) != cudaSuccess ||
      cudaMallocHost(&b->htab[0], b->lay.bytes) != cudaSuccess ||
      cudaMallocHost(&b->htab[1], b->lay.bytes) != cudaSuccess ||
      cudaMallocHost(&b->status_host, b->scratch_words * 4) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->htab_free[0], cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->htab_free[1], cudaEventDisableTiming) != cudaSuccess) {
    destroy(b);
    return nullptr;
  }
  uint8_t* p = b->arena;
  auto take = [&](size_t n) {
    uint8_t* q = p;
    p += up(n, 256);
    return q;
  };
  b->scratch = reinterpret_cast<uint32_t*>(take(b->scratch_words * 4));
  b->mvc = reinterpret_cast<MV*>(take((size_t)b->total_mbs * 16));
  uint32_t* sw = b->scratch;
  for (StreamState& t : b->ss) {
    const size_t mbs = (size_t)t.mbw * t.mbh;
    t.rec[0] = take(t.rec_bytes);
    t.rec[1] = take(t.rec_bytes);
    t.levels = reinterpret_cast<int16_t*>(take(mbs * 768));
    t.dc = reinterpret_cast<int32_t*>(take(mbs * 96));
    t.nz = reinterpret_cast<uint32_t*>(take(mbs * 96));
    t.pred_mode = reinterpret_cast<uint32_t*>(take(mbs * 4));
    t.mv[0] = reinterpret_cast<MV*>(take(mbs * 16));
    t.mv[1] = reinterpret_cast<MV*>(take(mbs * 16));
    t.scr_intra = sw;
    sw += scratch_words(t.mbh);
    t.scr_db = sw;
    sw += scratch_words(t.mbh);
    t.cur = 0;
    t.mv_cur = 0;
    t.has_recon = t.has_hist = false;
  }
  cudaMemsetAsync(b->arena, 0, bytes, b->stream);
  if (me_mode != 0) {
    b->prop = b200enc_proposal_create(b->total_mbs);
    if (!b->prop || b200enc_proposal_load(b->prop, weights_path().c_str()) != 0) {
      destroy(b);
      return nullptr;
    }
  }
  if (cudaStreamSynchronize(b->stream) != cudaSuccess) {
    destroy(b);
    return nullptr;
  }
  return b;
}

void b200enc_batch_destroy(void* h) { destroy(static_cast<Batch*>(h)); }

void* b200enc_batch_stream(void* h) {
  Batch* b = static_cast<Batch*>(h);
  return b ? (void*)b->stream : nullptr;
}

int b200enc_batch_set_graph(void* h, int enable) {
  Batch* b = static_cast<Batch*>(h);
  if (!b) return -1;
  b->graph = enable != 0;
  return 0;
}

int b200enc_batch_encode(void* h, const b200enc_batch_frame_t* frames) {
  Batch* b = static_cast<Batch*>(h);
  if (!b || !frames) return -1;
  // validate before touching any state
  for (int s = 0; s < b->n; ++s) {
    const b200enc_batch_frame_t& f = frames[s];
    const StreamState& t = b->ss[s];
    if (!f.y || !f.uv || (f.pitch & 3) || f.pitch < t.W || f.qp < 0 || f.qp > 51 || f.num_slices < 1) return -1;
    if ((((uintptr_t)f.y) & 3) || (((uintptr_t)f.uv) & 3)) return -1;
    if (!f.is_intra && !t.has_recon) return -1;  // a stream starts with an I frame
  }
  // the host table buffer of two steps ago must have been copied
  uint8_t* ht = b->htab[b->htab_next];
  cudaEventSynchronize(b->htab_free[b->htab_next]);
  BatchStream* hs = reinterpret_cast<BatchStream*>(ht + b->lay.streams);
  int* ip = reinterpret_cast<int*>(ht + b->lay.idx_p);
  int* ii = reinterpret_cast<int*>(ht + b->lay.idx_i);
  int* ig = reinterpret_cast<int*>(ht + b->lay.idx_g);
  int* pp = reinterpret_cast<int*>(ht + b->lay.pre_p);
  int* pi = reinterpret_cast<int*>(ht + b->lay.pre_i);
  int* pg = reinterpret_cast<int*>(ht + b->lay.pre_g);
  int np = 0, ni = 0, ng = 0, n_p = 0, n_irows = 0, n_groups = 0;
  pp[0] = pi[0] = pg[0] = 0;
  b200enc_deblock_tile_count(1, 1, &b->db_tw, &b->db_th);
  for (int s = 0; s < b->n; ++s) {
    const b200enc_batch_frame_t& f = frames[s];
    StreamState& t = b->ss[s];
    BatchStream& d = hs[s];
    memset(&d, 0, sizeof(d));
    d.g = Geo{t.W, t.H, t.mbw * 16, t.mbh * 16, t.mbw, t.mbh};
    d.qp = f.qp;
    d.is_intra = f.is_intra ? 1 : 0;
    d.num_slices = f.num_slices;
    d.intra_flags = B200ENC_INTRA_CORNER_CHECK;
    d.lambda = 5;
    d.zero_thresh = 512;
    d.has_hist = (!f.is_intra && t.has_hist) ? 1 : 0;
    d.cur_y = f.y;
    d.cur_uv = f.uv;
    d.cur_pitch = f.pitch;
    const size_t luma = (size_t)t.pitch * t.mbh * 16;
    d.ref_y = t.rec[t.cur];
    d.ref_uv = t.rec[t.cur] + luma;
    d.rec_y = t.rec[t.cur ^ 1];
    d.rec_uv = t.rec[t.cur ^ 1] + luma;
    d.rec_pitch = t.pitch;
    d.levels = t.levels;
    d.dc = t.dc;
    d.nz = t.nz;
    d.pred_mode = t.pred_mode;
    d.mv = t.mv[t.mv_cur ^ 1];
    d.mv_prev = t.mv[t.mv_cur];
    d.scr_intra = t.scr_intra;
    d.scr_db = t.scr_db;
    // deblocked out of place into the previous reconstruction, which the
    // step's ME and P chain have read before the deblocking launch
    d.db_y = t.rec[t.cur];
    d.db_uv = t.rec[t.cur] + luma;
    const int mbs = t.mbw * t.mbh;
    if (f.is_intra) {
      ii[ni] = s;
      pi[ni + 1] = pi[ni] + t.mbh;
      ++ni;
      n_irows += t.mbh;
    } else {
      // each P stream's range starts on a network tile (16 macroblocks), so
      // the FP8 network's per-tile activation scales see the same macroblocks
      // as in a single-stream run; the padding macroblocks are skipped
      ip[np] = s;
      pp[np + 1] = pp[np] + pad16(mbs);
      ++np;
      n_p += pad16(mbs);
    }
    const int groups = b200enc_deblock_tile_count(t.mbw, t.mbh, nullptr, nullptr);
    ig[ng] = s;
    pg[ng + 1] = pg[ng] + groups;
    ++ng;
    n_groups += groups;
  }
  // pad the prefixes past each set's end with its total (find() never reads them)
  for (int k = np + 1; k <= b->n; ++k) pp[k] = pp[np];
  for (int k = ni + 1; k <= b->n; ++k) pi[k] = pi[ni];
  for (int k = ng + 1; k <= b->n; ++k) pg[k] = pg[ng];
  int rc = 0;
  if (b->graph) {
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return -1;
    rc = enqueue_step(b, ht, np, ni, ng, n_p, n_irows, n_groups);
    if (cudaStreamEndCapture(b->stream, &g) != cudaSuccess || !g) return -1;
    if (rc == 0) {
      bool updated = false;
      if (b->exec) {
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(b->exec, g, &info) == cudaSuccess) {
          updated = true;
          ++b->graph_updates;
        } else {
          cudaGetLastError();
          cudaGraphExecDestroy(b->exec);
          b->exec = nullptr;
        }
      }
      if (!updated) {
        if (cudaGraphInstantiate(&b->exec, g, 0) != cudaSuccess) rc = -1;
        else ++b->graph_instantiations;
      }
      if (rc == 0 && cudaGraphLaunch(b->exec, b->stream) != cudaSuccess) rc = -1;
    }
    cudaGraphDestroy(g);
  } else {
    rc = enqueue_step(b, ht, np, ni, ng, n_p, n_irows, n_groups);
  }
  if (rc != 0) return -1;
  cudaEventRecord(b->htab_free[b->htab_next], b->stream);
  b->htab_next ^= 1;
  cudaEventRecord(b->done, b->stream);
  b->pending = true;
  for (int s = 0; s < b->n; ++s) {
    StreamState& t = b->ss[s];
    if (!b->deblock) t.cur ^= 1;  // deblocked: the reconstruction is back in rec[cur]
    t.mv_cur ^= 1;
    t.has_recon = true;
    t.has_hist = !frames[s].is_intra;
  }
  return 0;
}

int b200enc_batch_sync(void* h) {
  Batch* b = static_cast<Batch*>(h);
  if (!b) return -1;
  if (!b->pending) return 0;
  if (cudaEventSynchronize(b->done) != cudaSuccess) return -1;
  b->pending = false;
  // a wavefront that gave up leaves its stream's frame incomplete
  for (const StreamState& t : b->ss) {
    const size_t oi = (size_t)(t.scr_intra - b->scratch), od = (size_t)(t.scr_db - b->scratch);
    if (b->status_host[oi + 1] | b->status_host[od + 1]) return -1;
  }
  return 0;
}

int b200enc_batch_outputs(void* h, int s, void** levels, void** dc, void** nz, void** pred_mode, void** mv,
                          void** rec_y, void** rec_uv, int* rec_pitch) {
  Batch* b = static_cast<Batch*>(h);
  if (!b || s < 0 || s >= b->n) return -1;
  const StreamState& t = b->ss[s];
  if (levels) *levels = t.levels;
  if (dc) *dc = t.dc;
  if (nz) *nz = t.nz;
  if (pred_mode) *pred_mode = t.pred_mode;
  if (mv) *mv = t.mv[t.mv_cur];
  if (rec_y) *rec_y = t.rec[t.cur];
  if (rec_uv) *rec_uv = t.rec[t.cur] + (size_t)t.pitch * t.mbh * 16;
  if (rec_pitch) *rec_pitch = t.pitch;
  return 0;
}

int b200enc_batch_graph_stats(void* h, long* instantiations, long* updates) {
  Batch* b = static_cast<Batch*>(h);
  if (!b) return -1;
  if (instantiations) *instantiations = b->graph_instantiations;
  if (updates) *updates = b->graph_updates;
  return 0;
}

}  // extern "C"
