// gpu_compute_abi.cu - the reference's gpu_compute_* boundary on CUDA.
//
// Replaces approach1-compute-encoder/src/gpu_compute.c's encode half (Vulkan
// context, buffers, per-frame stage recording :2922-3365, double-buffered
// submit/fence/staging :3523-3798). One context = one CUDA stream; a frame is
// ME -> P chain or intra wavefront -> deblock -> staging copies, enqueued
// back to back with no host round trip; end_picture records the slot's
// event and sync_slot waits on it (bounded) and checks the wavefront status
// word that was staged with the outputs.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <utility>

#include "../../include/gpu_compute.h"
#include "b200enc_internal.h"

namespace {

constexpr uint32_t kWavefrontMaxWaitUs = 2000000u;  // 2 s per progress wait

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

struct Slot {
  int16_t* levels = nullptr;
  int32_t* dc = nullptr;
  uint32_t* pred_mode = nullptr;
  b200enc_mv_t* mv = nullptr;
  uint32_t* nz = nullptr;
  uint32_t* status = nullptr;  // wavefront error words (intra, deblock)
  cudaEvent_t start = nullptr, done = nullptr;
  bool pending = false;
  // GPU entropy coding: the slice RBSPs (no header) the GPU wrote into this
  // page-locked, device-mapped memory, and their byte counts
  uint8_t* slices = nullptr;
  uint32_t* slice_bytes = nullptr;
  int num_slices = 0;
};

struct Shadow {
  uint8_t* host = nullptr;
  size_t size = 0;
};

struct Impl {
  int device = 0;
  cudaStream_t stream = nullptr;
  int W = 0, H = 0, mbw = 0, mbh = 0, RW = 0, RH = 0;
  int pitch = 0;        // recon pitch
  size_t rec_bytes = 0;  // one NV12 recon buffer
  uint8_t* rec[2] = {nullptr, nullptr};
  int cur = 0;  // rec[cur] is the latest reconstruction
  int16_t* d_levels = nullptr;
  int32_t* d_dc = nullptr;
  uint32_t* d_nz = nullptr;
  uint32_t* d_pred_mode = nullptr;
  b200enc_mv_t* d_mv = nullptr;
  uint32_t* d_scratch = nullptr;  // two wavefront scratch regions
  size_t scratch_words = 0;
  Slot slot[2];
  int submitted = 0;
  double last_latency_ms = 0.0;
  // parameters
  int range = 16, lambda = -1, zero_thresh = 512, clamp_coded = 1, deblock = -1;
  int intra_flags = B200ENC_INTRA_CORNER_CHECK;
  // learned proposal (me_mode 1: network, 2: candidates only, 3: network in FP8)
  int me_mode = 0;
  float conf = 0.9f;
  std::string weights;
  void* prop = nullptr;
  int prop_mbs = 0;
  b200enc_mv_t* d_mv_prev = nullptr;
  bool mv_hist = false;  // d_mv holds the previous P frame's field
  bool last_learned = false;  // the last P frame ran b200enc_proposal_me
  std::map<void*, Shadow> shadows;
  std::map<void*, size_t> registered;  // caller buffers this context page-locked
  // Per-stage timing (the reference's BC250_PERF_STATS timestamps,
  // gpu_compute.c:50-67): a ring of event sets, one per frame, folded into
  // running sums when completed.
  bool perf = false;
  static constexpr int kRing = 64, kMarks = 5;  // start, ME, chain, deblock, staging
  cudaEvent_t ev[kRing][kMarks] = {};
  bool ev_intra[kRing] = {};
  int ev_head = 0, ev_count = 0;
  double stage_ms[2][4] = {};  // [intra][me, chain, deblock, staging]
  long stage_frames[2] = {0, 0};
  // GPU entropy coding (b200enc_ctx_set_entropy): 0 off, 1 CAVLC slice data
  // beside the staged outputs, 2 CAVLC slice data instead of the staged
  // levels, DC, nz masks and modes
  int entropy = 0, quality = 4;
  void* d_cavlc = nullptr;     // b200enc_cavlc_scratch_bytes
  size_t cavlc_bytes = 0;
  uint8_t* d_slices = nullptr;  // the slices' bit words
  size_t slices_bytes = 0;
};

Impl* impl_of(const gpu_context_t* ctx) { return ctx ? static_cast<Impl*>(ctx->impl) : nullptr; }

int env_int(const char* name, int dflt) {
  const char* v = getenv(name);
  return (v && *v) ? atoi(v) : dflt;
}
bool fast_mode() {
  const char* fm = getenv("BC250_FAST_MODE");
  return fm && (strcmp(fm, "1") == 0 || strcmp(fm, "true") == 0);
}

void free_frame_buffers(Impl* m) {
  cudaFree(m->rec[0]);
  cudaFree(m->rec[1]);
  cudaFree(m->d_levels);
  cudaFree(m->d_dc);
  cudaFree(m->d_nz);
  cudaFree(m->d_pred_mode);
  cudaFree(m->d_mv);
  cudaFree(m->d_mv_prev);
  cudaFree(m->d_scratch);
  cudaFree(m->d_cavlc);
  cudaFree(m->d_slices);
  m->d_cavlc = nullptr;
  m->d_slices = nullptr;
  m->cavlc_bytes = m->slices_bytes = 0;
  if (m->prop) b200enc_proposal_destroy(m->prop);
  m->prop = nullptr;
  m->prop_mbs = 0;
  m->d_mv_prev = nullptr;
  m->mv_hist = false;
  m->rec[0] = m->rec[1] = nullptr;
  m->d_levels = nullptr;
  m->d_dc = nullptr;
  m->d_nz = m->d_pred_mode = nullptr;
  m->d_mv = nullptr;
  m->d_scratch = nullptr;
  for (Slot& s : m->slot) {
    cudaFreeHost(s.levels);
    cudaFreeHost(s.dc);
    cudaFreeHost(s.pred_mode);
    cudaFreeHost(s.mv);
    cudaFreeHost(s.nz);
    cudaFreeHost(s.status);
    cudaFreeHost(s.slices);
    cudaFreeHost(s.slice_bytes);
    s.slices = nullptr;
    s.slice_bytes = nullptr;
    s.levels = nullptr;
    s.dc = nullptr;
    s.pred_mode = s.nz = s.status = nullptr;
    s.mv = nullptr;
  }
  m->W = m->H = 0;
}

// (Re)allocates every per-size buffer; mirrors allocate_encoding_buffers()
// of the reference (gpu_compute.c:2931-2952).
int ensure_buffers(gpu_context_t* ctx, Impl* m, int W, int H) {
  if (m->W == W && m->H == H && m->rec[0]) return 0;
  cudaStreamSynchronize(m->stream);
  free_frame_buffers(m);
  m->W = W;
  m->H = H;
  m->mbw = (W + 15) / 16;
  m->mbh = (H + 15) / 16;
  m->pitch = (int)align_up((size_t)m->mbw * 16, 128);
  const size_t luma = (size_t)m->pitch * m->mbh * 16;
  m->rec_bytes = luma + luma / 2;
  const size_t mbs = (size_t)m->mbw * m->mbh;
  m->scratch_words = align_up(b200enc_wavefront_scratch_bytes(m->mbh) / 4, 64);
  bool ok = cudaMalloc(&m->rec[0], m->rec_bytes) == cudaSuccess && cudaMalloc(&m->rec[1], m->rec_bytes) == cudaSuccess &&
            cudaMalloc(&m->d_levels, mbs * 384 * 2) == cudaSuccess && cudaMalloc(&m->d_dc, mbs * 24 * 4) == cudaSuccess &&
            cudaMalloc(&m->d_nz, mbs * 24 * 4) == cudaSuccess && cudaMalloc(&m->d_pred_mode, mbs * 4) == cudaSuccess &&
            cudaMalloc(&m->d_mv, mbs * 16) == cudaSuccess && cudaMalloc(&m->d_mv_prev, mbs * 16) == cudaSuccess &&
            cudaMalloc(&m->d_scratch, m->scratch_words * 2 * 4) == cudaSuccess;
  for (Slot& s : m->slot) {
    ok = ok && cudaMallocHost(&s.levels, mbs * 384 * 2) == cudaSuccess &&
         cudaMallocHost(&s.dc, mbs * 24 * 4) == cudaSuccess && cudaMallocHost(&s.pred_mode, mbs * 4) == cudaSuccess &&
         cudaMallocHost(&s.mv, mbs * 16) == cudaSuccess && cudaMallocHost(&s.nz, mbs * 24 * 4) == cudaSuccess &&
         cudaMallocHost(&s.status, 16) == cudaSuccess;
  }
  if (!ok) {
    free_frame_buffers(m);
    return -1;
  }
  cudaMemsetAsync(m->rec[0], 0, m->rec_bytes, m->stream);
  cudaMemsetAsync(m->rec[1], 0, m->rec_bytes, m->stream);
  cudaMemsetAsync(m->d_mv, 0, mbs * 16, m->stream);
  for (Slot& s : m->slot) memset(s.status, 0, 16);
  m->cur = 0;
  ctx->has_recon_frame = false;
  ctx->frame_width = (uint32_t)W;
  ctx->frame_height = (uint32_t)H;
  return 0;
}

void publish_recon(gpu_context_t* ctx, Impl* m) {
  uint8_t* y = m->rec[m->cur];
  ctx->recon_image.y_plane = ctx->recon_image.y_view = y;
  ctx->recon_image.uv_plane = ctx->recon_image.uv_view = y + (size_t)m->pitch * m->mbh * 16;
  ctx->recon_image.width = (uint32_t)m->W;
  ctx->recon_image.height = (uint32_t)m->H;
  ctx->recon_image.pitch = (uint32_t)m->pitch;
  ctx->recon_image.format = GPU_IMAGE_NV12;
  ctx->recon_memory.memory = y;
  ctx->recon_memory.size = m->rec_bytes;
}

void perf_fold_one(Impl* m) {
  const int i = (m->ev_head - m->ev_count + Impl::kRing) % Impl::kRing;
  cudaEventSynchronize(m->ev[i][Impl::kMarks - 1]);
  const int k = m->ev_intra[i] ? 1 : 0;
  for (int s = 0; s < 4; ++s) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, m->ev[i][s], m->ev[i][s + 1]) == cudaSuccess) m->stage_ms[k][s] += ms;
  }
  m->stage_frames[k]++;
  m->ev_count--;
}

void perf_mark(Impl* m, int mark) {
  if (m->perf) cudaEventRecord(m->ev[m->ev_head][mark], m->stream);
}

// Bounded wait on an event: BC250_GPU_TIMEOUT_MS (0 or unset = unbounded),
// the reference's fence-wait budget (gpu_compute.c:2829-2843).
int wait_event(cudaEvent_t ev) {
  const int budget_ms = env_int("BC250_GPU_TIMEOUT_MS", 0);
  if (budget_ms <= 0) return cudaEventSynchronize(ev) == cudaSuccess ? 0 : -1;
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    const cudaError_t e = cudaEventQuery(ev);
    if (e == cudaSuccess) return 0;
    if (e != cudaErrorNotReady) return -1;
    if (std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(budget_ms)) return -1;
    std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
}

// The packaged network parameters: <dir of libb200enc.so>/../b200enc/data/.
std::string default_weights() {
  Dl_info info;
  if (dladdr((void*)&default_weights, &info) && info.dli_fname) {
    std::string p = info.dli_fname;
    const size_t cut = p.find_last_of('/');
    p = (cut == std::string::npos) ? std::string(".") : p.substr(0, cut);
    return p + "/../b200enc/data/proposal_h264.b2pn";
  }
  return "proposal_h264.b2pn";
}

// Creates the proposal runtime for the current frame size and loads the
// parameters; 0, -1 on allocation failure, -2 on a missing or bad file.
int ensure_proposal(Impl* m) {
  const int mbs = m->mbw * m->mbh;
  if (m->prop && m->prop_mbs == mbs) return 0;
  if (m->prop) b200enc_proposal_destroy(m->prop);
  m->prop = b200enc_proposal_create(mbs);
  m->prop_mbs = mbs;
  if (!m->prop) return -1;
  if (m->me_mode == 2) return 0;  // the candidate search without the network needs no parameters
  const std::string path = m->weights.empty() ? default_weights() : m->weights;
  const int rc = b200enc_proposal_load(m->prop, path.c_str());
  if (rc != 0) {
    b200enc_proposal_destroy(m->prop);
    m->prop = nullptr;
    m->prop_mbs = 0;
    return rc == -2 ? -2 : -1;
  }
  return 0;
}

// Slice capacity of one slice region for a frame of `mbs` macroblocks in
// `ns` slices: the reference's CAVLC allowance (2560 bytes per macroblock,
// encoder_h264.c:3083-3086) for the largest slice, plus its header slack.
size_t slice_cap_of(size_t mbs, int ns) { return align_up(((mbs + ns - 1) / ns) * 2560 + 4096, 256); }

// Buffers of the GPU entropy coder, allocated on first use (every slot's
// region holds 16 slices of the largest size).
int ensure_entropy(Impl* m) {
  if (m->d_cavlc) return 0;
  const size_t mbs = (size_t)m->mbw * m->mbh;
  m->cavlc_bytes = b200enc_cavlc_scratch_bytes(m->mbw, m->mbh);
  m->slices_bytes = 16 * slice_cap_of(mbs, 16) + mbs * 2560;
  bool ok = cudaMalloc(&m->d_cavlc, m->cavlc_bytes) == cudaSuccess &&
            cudaMalloc(&m->d_slices, m->slices_bytes) == cudaSuccess;
  for (Slot& s : m->slot)
    ok = ok && cudaHostAlloc(&s.slices, m->slices_bytes, cudaHostAllocMapped) == cudaSuccess &&
         cudaHostAlloc(&s.slice_bytes, 16 * sizeof(uint32_t), cudaHostAllocMapped) == cudaSuccess;
  if (!ok) {
    cudaFree(m->d_cavlc);
    cudaFree(m->d_slices);
    m->d_cavlc = nullptr;
    m->d_slices = nullptr;
    for (Slot& s : m->slot) {
      cudaFreeHost(s.slices);
      cudaFreeHost(s.slice_bytes);
      s.slices = nullptr;
      s.slice_bytes = nullptr;
    }
    return -1;
  }
  return 0;
}

// The whole hot path of one frame, enqueued on the context stream.
int encode_frame(gpu_context_t* ctx, Impl* m, const uint8_t* y, const uint8_t* uv, int src_pitch, int W, int H, int qp,
                 int is_intra, int num_slices, int me_mode, const gpu_mv_t* cpu_mvs, bool stage) {
  if (qp < 0 || qp > 51 || W <= 0 || H <= 0) return -1;
  if (ensure_buffers(ctx, m, W, H) != 0) return -1;
  if (num_slices < 1) num_slices = 1;
  const int RW = m->clamp_coded ? m->mbw * 16 : W, RH = m->clamp_coded ? m->mbh * 16 : H;
  const size_t luma = (size_t)m->pitch * m->mbh * 16, mbs = (size_t)m->mbw * m->mbh;
  Slot& sl = m->slot[ctx->current_buf];
  cudaEventRecord(sl.start, m->stream);
  if (m->perf) {
    if (m->ev_count == Impl::kRing) perf_fold_one(m);
    m->ev_intra[m->ev_head] = is_intra != 0;
  }
  perf_mark(m, 0);
  // reference for P: the latest recon, or the input itself before any
  // reconstruction exists (gpu_compute.c:3008-3015)
  const bool have_ref = ctx->has_recon_frame;
  const uint8_t* ref_y = have_ref ? m->rec[m->cur] : y;
  const uint8_t* ref_uv = have_ref ? m->rec[m->cur] + luma : uv;
  const int ref_pitch = have_ref ? m->pitch : src_pitch;
  const int ref_RW = have_ref ? RW : W, ref_RH = have_ref ? RH : H;
  uint8_t* out_y = m->rec[m->cur ^ 1];
  uint8_t* out_uv = out_y + luma;
  uint32_t* scr0 = m->d_scratch;
  uint32_t* scr1 = m->d_scratch + m->scratch_words;
  int rc = 0;
  if (is_intra) {
    m->mv_hist = false;
    m->last_learned = false;
    perf_mark(m, 1);  // intra frames have no ME stage
    rc |= cudaMemsetAsync(scr0, 0, m->scratch_words * 4, m->stream) == cudaSuccess ? 0 : -1;
    rc |= b200enc_i_frame_launch(y, uv, src_pitch, W, H, RW, RH, qp, num_slices, m->d_levels, m->d_dc, m->d_nz,
                                 m->d_pred_mode, m->d_mv, out_y, out_uv, m->pitch, scr0, 0, kWavefrontMaxWaitUs,
                                 m->intra_flags, m->stream);
  } else {
    if (cpu_mvs) {
      // caller-supplied MVs replace Stage 2 (gpu_compute.c:3078-3092)
      memcpy(sl.mv, cpu_mvs, mbs * 16);
      rc |= cudaMemcpyAsync(m->d_mv, sl.mv, mbs * 16, cudaMemcpyHostToDevice, m->stream) == cudaSuccess ? 0 : -1;
    } else {
      m->last_learned = false;
      const int lambda = m->lambda >= 0 ? m->lambda : (me_mode == 1 ? 8 : 5);
      if (m->me_mode != 0 && have_ref && m->mv_hist) {
        // the learned form fails loudly without its parameters
        if (ensure_proposal(m) != 0) return -1;
        // the previous frame's field becomes the history, the other buffer
        // takes this frame's (work already enqueued on the stream that reads
        // either buffer runs first)
        std::swap(m->d_mv, m->d_mv_prev);
        rc |= b200enc_proposal_me(m->prop, y, src_pitch, ref_y, ref_pitch, W, H, ref_RW, ref_RH, m->d_mv_prev,
                                  m->range, lambda, m->zero_thresh, m->me_mode, m->conf, m->d_mv, m->stream);
        m->last_learned = true;
      } else {
        // a window copy that never completes lands in the frame's status
        // (the intra scratch's error word, unused by P frames)
        rc |= b200enc_me_full_search_err(y, src_pitch, ref_y, ref_pitch, W, H, ref_RW, ref_RH, m->range, lambda,
                                         m->zero_thresh, m->d_mv, nullptr, nullptr, 0, 0, scr0 + 1, m->stream);
      }
    }
    m->mv_hist = have_ref;
    perf_mark(m, 1);
    rc |= b200enc_p_frame(y, uv, src_pitch, ref_y, ref_uv, ref_pitch, W, H, RW, RH, qp, m->d_mv, m->d_levels, m->d_dc,
                          m->d_nz, m->d_pred_mode, out_y, out_uv, m->pitch, m->stream);
  }
  perf_mark(m, 2);
  const bool db = m->deblock >= 0 ? m->deblock != 0 : !fast_mode();
  if (db) {
    // Deblocked as independent tiles from the unfiltered reconstruction
    // into the other buffer: the previous reconstruction, which nothing
    // reads once the P chain (or the intra wavefront) has run.
    rc |= cudaMemsetAsync(scr1, 0, m->scratch_words * 4, m->stream) == cudaSuccess ? 0 : -1;
    uint8_t* db_y = m->rec[m->cur];
    rc |= b200enc_deblock_tiles_launch(m->mbw, m->mbh, qp, is_intra, m->d_nz, m->d_mv, out_y, out_uv, db_y,
                                       db_y + luma, m->pitch, scr1, kWavefrontMaxWaitUs, m->stream);
  }
  perf_mark(m, 3);
  sl.num_slices = 0;
  if (m->entropy) {
    // the slice data of every slice, written by the GPU straight into the
    // slot's mapped host memory (only the bytes of the slices cross the bus)
    if (ensure_entropy(m) != 0) return -1;
    b200enc_cavlc_t cp{};
    cp.mbw = m->mbw;
    cp.mbh = m->mbh;
    cp.qp = qp;
    cp.is_intra = is_intra ? 1 : 0;
    cp.num_slices = std::min(num_slices, 16);
    cp.quality_level = m->quality;
    cp.levels = m->d_levels;
    cp.dc = m->d_dc;
    cp.nz = m->d_nz;
    cp.pred_mode = m->d_pred_mode;
    cp.mv = m->d_mv;
    cp.out = m->d_slices;
    cp.slice_cap = slice_cap_of(mbs, cp.num_slices);
    uint8_t* dev_slices = nullptr;
    uint32_t* dev_bytes = nullptr;
    rc |= cudaHostGetDevicePointer((void**)&dev_slices, sl.slices, 0) == cudaSuccess ? 0 : -1;
    rc |= cudaHostGetDevicePointer((void**)&dev_bytes, sl.slice_bytes, 0) == cudaSuccess ? 0 : -1;
    cp.out_copy = dev_slices;
    cp.out_bytes = dev_bytes;
    cp.scratch = m->d_cavlc;
    cp.scratch_bytes = m->cavlc_bytes;
    if (rc == 0) rc |= b200enc_cavlc_slices(&cp, m->stream);
    sl.num_slices = cp.num_slices;
  }
  if (stage) {
    cudaStream_t st = m->stream;
    if (m->entropy != 2) {
      rc |= cudaMemcpyAsync(sl.levels, m->d_levels, mbs * 768, cudaMemcpyDeviceToHost, st) == cudaSuccess ? 0 : -1;
      rc |= cudaMemcpyAsync(sl.dc, m->d_dc, mbs * 96, cudaMemcpyDeviceToHost, st) == cudaSuccess ? 0 : -1;
      rc |= cudaMemcpyAsync(sl.pred_mode, m->d_pred_mode, mbs * 4, cudaMemcpyDeviceToHost, st) == cudaSuccess ? 0 : -1;
      rc |= cudaMemcpyAsync(sl.nz, m->d_nz, mbs * 96, cudaMemcpyDeviceToHost, st) == cudaSuccess ? 0 : -1;
    }
    rc |= cudaMemcpyAsync(sl.mv, m->d_mv, mbs * 16, cudaMemcpyDeviceToHost, st) == cudaSuccess ? 0 : -1;
    rc |= cudaMemcpyAsync(sl.status, scr0 + 1, 4, cudaMemcpyDeviceToHost, st) == cudaSuccess ? 0 : -1;
    rc |= cudaMemcpyAsync(sl.status + 1, scr1 + 1, 4, cudaMemcpyDeviceToHost, st) == cudaSuccess ? 0 : -1;
  }
  perf_mark(m, 4);
  if (m->perf) {
    m->ev_head = (m->ev_head + 1) % Impl::kRing;
    m->ev_count++;
  }
  if (rc != 0) return -1;
  if (!db) m->cur ^= 1;  // deblocked: the latest reconstruction is back in rec[cur]
  ctx->has_recon_frame = true;
  publish_recon(ctx, m);
  return 0;
}

std::string dump_dir() {
  const char* d = getenv("BC250_DUMP_DIR");
  if (d && *d) return d;
  const char* x = getenv("XDG_RUNTIME_DIR");
  return std::string(x && *x ? x : "/tmp") + "/bc250_dump_frames";
}

}  // namespace

extern "C" {

int bc250_gpu_init(bc250_gpu_context_t* ctx) {
  if (!ctx) return -1;
  memset(ctx, 0, sizeof(*ctx));
  Impl* m = new Impl();
  int dev = env_int("B200ENC_DEVICE", -1);
  if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) dev = 0;
  if (cudaSetDevice(dev) != cudaSuccess || cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete m;
    return -1;
  }
  m->device = dev;
  for (Slot& s : m->slot) {
    if (cudaEventCreate(&s.start) != cudaSuccess || cudaEventCreate(&s.done) != cudaSuccess) {
      delete m;
      return -1;
    }
  }
  const int r = env_int("B200ENC_SEARCH_RANGE", 16);
  m->range = (r == 32) ? 32 : 16;
  const char* cl = getenv("B200ENC_RECON_CLAMP");
  m->clamp_coded = (cl && strcmp(cl, "visible") == 0) ? 0 : 1;
  const char* ip = getenv("B200ENC_INTRA_PLANE");
  m->intra_flags = (ip && strcmp(ip, "shader") == 0) ? 0 : B200ENC_INTRA_CORNER_CHECK;
  const char* me = getenv("B200ENC_ME");
  if (me && strcmp(me, "learned") == 0) m->me_mode = 1;
  if (me && strcmp(me, "candidates") == 0) m->me_mode = 2;
  if (me && strcmp(me, "learned_fp8") == 0) m->me_mode = 3;
  const char* wp = getenv("B200ENC_PROPOSAL_WEIGHTS");
  if (wp && *wp) m->weights = wp;
  const char* cf = getenv("B200ENC_PROPOSAL_CONF");
  if (cf && *cf) m->conf = (float)atof(cf);
  ctx->impl = m;
  return 0;
}

void bc250_gpu_destroy(bc250_gpu_context_t* ctx) {
  Impl* m = impl_of(ctx);
  if (!m) return;
  cudaStreamSynchronize(m->stream);
  free_frame_buffers(m);
  for (auto& kv : m->shadows) cudaFreeHost(kv.second.host);
  for (auto& kv : m->registered) cudaHostUnregister(kv.first);
  for (Slot& s : m->slot) {
    cudaEventDestroy(s.start);
    cudaEventDestroy(s.done);
  }
  for (auto& row : m->ev)
    for (cudaEvent_t e : row)
      if (e) cudaEventDestroy(e);
  cudaStreamDestroy(m->stream);
  delete m;
  ctx->impl = nullptr;
}

int gpu_compute_init(gpu_context_t* ctx) { return bc250_gpu_init(ctx); }
void gpu_compute_terminate(gpu_context_t* ctx) { bc250_gpu_destroy(ctx); }

int gpu_compute_create_image(gpu_context_t* ctx, int width, int height, int format, gpu_image_t* image,
                             gpu_memory_t* memory) {
  Impl* m = impl_of(ctx);
  if (!m || !image || !memory || width <= 0 || height <= 0) return -1;
  const int bpp = format == GPU_IMAGE_P010 ? 2 : 1;
  const size_t pitch = align_up((size_t)align_up(width, 16) * bpp, 128);
  const size_t rows = align_up(height, 16);
  const size_t bytes = pitch * rows + pitch * rows / 2;
  void* p = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) return -1;
  cudaMemsetAsync(p, 0, bytes, m->stream);
  memset(image, 0, sizeof(*image));
  image->y_plane = image->y_view = p;
  image->uv_plane = image->uv_view = (uint8_t*)p + pitch * rows;
  image->width = (uint32_t)width;
  image->height = (uint32_t)height;
  image->format = format;
  image->pitch = (uint32_t)pitch;
  memory->memory = p;
  memory->size = bytes;
  memory->mapped_ptr = nullptr;
  return 0;
}

void gpu_compute_destroy_image(gpu_context_t* ctx, gpu_image_t image, gpu_memory_t memory) {
  Impl* m = impl_of(ctx);
  if (!m || !memory.memory) return;
  cudaStreamSynchronize(m->stream);
  auto it = m->shadows.find(memory.memory);
  if (it != m->shadows.end()) {
    cudaFreeHost(it->second.host);
    m->shadows.erase(it);
  }
  (void)image;
  cudaFree(memory.memory);
}

int gpu_compute_get_nv12_layout(gpu_context_t* ctx, gpu_image_t* image, gpu_memory_t memory,
                                gpu_nv12_layout_t* layout) {
  if (!ctx || !image || !layout || !image->y_plane) return -1;
  layout->y_pitch = image->pitch;
  layout->y_offset = (uint64_t)((uint8_t*)image->y_plane - (uint8_t*)memory.memory);
  layout->uv_pitch = image->pitch;
  layout->uv_offset = (uint64_t)((uint8_t*)image->uv_plane - (uint8_t*)memory.memory);
  layout->total_size = memory.size;
  return 0;
}

uint8_t* gpu_compute_map_surface(gpu_context_t* ctx, gpu_image_t* image, gpu_memory_t memory,
                                 gpu_nv12_layout_t* layout, bool* unmap) {
  Impl* m = impl_of(ctx);
  if (unmap) *unmap = false;
  if (!m || !image || !memory.memory || memory.size == 0) return nullptr;
  Shadow& sh = m->shadows[memory.memory];
  if (sh.size != memory.size) {
    cudaFreeHost(sh.host);
    sh.host = nullptr;
    if (cudaMallocHost(&sh.host, memory.size) != cudaSuccess) {
      m->shadows.erase(memory.memory);
      return nullptr;
    }
    sh.size = memory.size;
  }
  if (cudaMemcpyAsync(sh.host, memory.memory, memory.size, cudaMemcpyDeviceToHost, m->stream) != cudaSuccess ||
      cudaStreamSynchronize(m->stream) != cudaSuccess)
    return nullptr;
  if (layout) gpu_compute_get_nv12_layout(ctx, image, memory, layout);
  if (unmap) *unmap = true;
  return sh.host;
}

void gpu_compute_unmap_surface(gpu_context_t* ctx, gpu_memory_t memory, bool unmap) {
  Impl* m = impl_of(ctx);
  if (!m || !unmap || !memory.memory) return;
  auto it = m->shadows.find(memory.memory);
  if (it == m->shadows.end()) return;
  cudaMemcpyAsync(memory.memory, it->second.host, it->second.size, cudaMemcpyHostToDevice, m->stream);
  cudaStreamSynchronize(m->stream);
}

int gpu_compute_upload_nv12(gpu_context_t* ctx, gpu_image_t* image, gpu_memory_t memory, const uint8_t* y_plane,
                            int y_pitch, const uint8_t* uv_plane, int uv_pitch, int width, int height) {
  Impl* m = impl_of(ctx);
  (void)memory;
  if (!m || !image || !image->y_plane || !y_plane || !uv_plane || width <= 0 || height <= 0) return -1;
  if ((uint32_t)width > image->width || (uint32_t)height > image->height) return -1;
  if (cudaMemcpy2DAsync(image->y_plane, image->pitch, y_plane, y_pitch, width, height, cudaMemcpyHostToDevice,
                        m->stream) != cudaSuccess ||
      cudaMemcpy2DAsync(image->uv_plane, image->pitch, uv_plane, uv_pitch, width, height / 2,
                        cudaMemcpyHostToDevice, m->stream) != cudaSuccess)
    return -1;
  // Host buffers the caller may reuse on return: unless both planes are
  // page-locked (cudaMallocHost, or b200enc_host_register: then stream
  // order is enough), wait for the copy.
  cudaPointerAttributes a{}, b{};
  if (cudaPointerGetAttributes(&a, y_plane) != cudaSuccess || a.type != cudaMemoryTypeHost ||
      cudaPointerGetAttributes(&b, uv_plane) != cudaSuccess || b.type != cudaMemoryTypeHost) {
    cudaGetLastError();
    return cudaStreamSynchronize(m->stream) == cudaSuccess ? 0 : -1;
  }
  return 0;
}

int gpu_compute_download_nv12(gpu_context_t* ctx, gpu_image_t* image, gpu_memory_t memory, uint8_t* y_plane,
                              int y_pitch, uint8_t* uv_plane, int uv_pitch, int width, int height) {
  Impl* m = impl_of(ctx);
  (void)memory;
  if (!m || !image || !image->y_plane || !y_plane || !uv_plane || width <= 0 || height <= 0) return -1;
  if (cudaMemcpy2DAsync(y_plane, y_pitch, image->y_plane, image->pitch, width, height, cudaMemcpyDeviceToHost,
                        m->stream) != cudaSuccess ||
      cudaMemcpy2DAsync(uv_plane, uv_pitch, image->uv_plane, image->pitch, width, height / 2,
                        cudaMemcpyDeviceToHost, m->stream) != cudaSuccess)
    return -1;
  return cudaStreamSynchronize(m->stream) == cudaSuccess ? 0 : -1;
}

void gpu_compute_copy_from_wc(void* dst, const void* src, size_t n) { memcpy(dst, src, n); }

int gpu_compute_wait_for_image_ready_host(gpu_context_t* ctx, gpu_memory_t memory) {
  (void)ctx;
  (void)memory;
  return 0;
}

int gpu_compute_cpu_read_safe(gpu_context_t* ctx) {
  Impl* m = impl_of(ctx);
  if (!m) return 1;
  for (Slot& s : m->slot)
    if (s.pending && cudaEventQuery(s.done) == cudaErrorNotReady) return 0;
  return 1;
}

FILE* bc250_debug_dump_open(const char* name, const char* what) {
  (void)what;
  if (!name || strchr(name, '/')) return nullptr;
  const std::string dir = dump_dir();
  mkdir(dir.c_str(), 0700);
  const std::string path = dir + "/" + name;
  const int fd = open(path.c_str(), O_WRONLY | O_CREAT | O_TRUNC | O_NOFOLLOW | O_CLOEXEC, 0600);
  if (fd < 0) return nullptr;
  FILE* f = fdopen(fd, "wb");
  if (!f) close(fd);
  return f;
}

int gpu_compute_begin_picture(gpu_context_t* ctx, gpu_image_t render_target) {
  Impl* m = impl_of(ctx);
  (void)render_target;
  if (!m) return -1;
  Slot& s = m->slot[ctx->current_buf];
  if (s.pending && wait_event(s.done) != 0) return -1;
  return 0;
}

int gpu_compute_dispatch_encode_ext(gpu_context_t* ctx, gpu_image_t rt, int width, int height, int qp, int is_intra,
                                    int num_slices, int me_mode, const gpu_mv_t* cpu_mvs) {
  Impl* m = impl_of(ctx);
  if (!m || !rt.y_plane || !rt.uv_plane || rt.format != GPU_IMAGE_NV12) return -1;
  return encode_frame(ctx, m, (const uint8_t*)rt.y_plane, (const uint8_t*)rt.uv_plane, (int)rt.pitch, width, height,
                      qp, is_intra, num_slices, me_mode, cpu_mvs, true);
}

int gpu_compute_dispatch_encode(gpu_context_t* ctx, gpu_image_t rt, int width, int height, int qp, int is_intra,
                                int num_slices) {
  return gpu_compute_dispatch_encode_ext(ctx, rt, width, height, qp, is_intra, num_slices, 0, nullptr);
}

int gpu_compute_dispatch_me_only(gpu_context_t* ctx, gpu_image_t rt, int width, int height) {
  Impl* m = impl_of(ctx);
  if (!m || !rt.y_plane || rt.format != GPU_IMAGE_NV12) return -1;
  if (ensure_buffers(ctx, m, width, height) != 0) return -1;
  const bool have_ref = ctx->has_recon_frame;
  const int RW = m->clamp_coded ? m->mbw * 16 : width, RH = m->clamp_coded ? m->mbh * 16 : height;
  Slot& sl = m->slot[ctx->current_buf];
  cudaEventRecord(sl.start, m->stream);
  const uint8_t* ref = have_ref ? m->rec[m->cur] : (const uint8_t*)rt.y_plane;
  if (b200enc_me_full_search((const uint8_t*)rt.y_plane, (int)rt.pitch, ref, have_ref ? m->pitch : (int)rt.pitch, width,
                             height, have_ref ? RW : width, have_ref ? RH : height, m->range,
                             m->lambda >= 0 ? m->lambda : 5, m->zero_thresh, m->d_mv, m->stream) != 0)
    return -1;
  const size_t mbs = (size_t)m->mbw * m->mbh;
  return cudaMemcpyAsync(sl.mv, m->d_mv, mbs * 16, cudaMemcpyDeviceToHost, m->stream) == cudaSuccess ? 0 : -1;
}

double gpu_compute_get_last_latency_ms(const gpu_context_t* ctx) {
  Impl* m = impl_of(ctx);
  return m ? m->last_latency_ms : 0.0;
}

int gpu_compute_end_picture(gpu_context_t* ctx) {
  Impl* m = impl_of(ctx);
  if (!m) return -1;
  Slot& s = m->slot[ctx->current_buf];
  if (cudaEventRecord(s.done, m->stream) != cudaSuccess) return -1;
  s.pending = true;
  m->submitted = ctx->current_buf;
  ctx->current_buf ^= 1;
  ctx->frames_submitted++;
  return 0;
}

int gpu_compute_submitted_slot(gpu_context_t* ctx) {
  Impl* m = impl_of(ctx);
  return m ? m->submitted : 0;
}

int gpu_compute_sync_slot(gpu_context_t* ctx, int slot) {
  Impl* m = impl_of(ctx);
  if (!m || slot < 0 || slot > 1) return -1;
  Slot& s = m->slot[slot];
  if (!s.pending) return 0;
  if (wait_event(s.done) != 0) return -1;
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, s.start, s.done) == cudaSuccess) m->last_latency_ms = ms;
  // a wavefront that gave up leaves its frame incomplete
  if (s.status && (s.status[0] | s.status[1])) return -1;
  return 0;
}

int gpu_compute_sync(gpu_context_t* ctx) { return gpu_compute_sync_slot(ctx, gpu_compute_submitted_slot(ctx)); }

#define B200_GETTER(fn, field, bytes_per_mb)                                               \
  int fn(gpu_context_t* ctx, int slot, void** data, size_t* size) {                        \
    Impl* m = impl_of(ctx);                                                                \
    if (!m || slot < 0 || slot > 1 || !data || !size || !m->slot[slot].field) return -1;   \
    *data = m->slot[slot].field;                                                           \
    *size = (size_t)m->mbw * m->mbh * (bytes_per_mb);                                      \
    return 0;                                                                              \
  }
B200_GETTER(gpu_compute_get_quant_staging_data_slot, levels, 768)
B200_GETTER(gpu_compute_get_dc_staging_data_slot, dc, 96)
B200_GETTER(gpu_compute_get_pred_mode_staging_data_slot, pred_mode, 4)
B200_GETTER(gpu_compute_get_mv_staging_data_slot, mv, 16)
B200_GETTER(gpu_compute_get_nz_staging_data_slot, nz, 96)
#undef B200_GETTER

int gpu_compute_get_quant_staging_data(gpu_context_t* c, void** d, size_t* n) {
  return gpu_compute_get_quant_staging_data_slot(c, gpu_compute_submitted_slot(c), d, n);
}
int gpu_compute_get_staging_data(gpu_context_t* c, void** d, size_t* n) { return gpu_compute_get_quant_staging_data(c, d, n); }
int gpu_compute_release_staging_data(gpu_context_t* c) { return c ? 0 : -1; }
int gpu_compute_get_dc_staging_data(gpu_context_t* c, void** d, size_t* n) {
  return gpu_compute_get_dc_staging_data_slot(c, gpu_compute_submitted_slot(c), d, n);
}
int gpu_compute_get_pred_mode_staging_data(gpu_context_t* c, void** d, size_t* n) {
  return gpu_compute_get_pred_mode_staging_data_slot(c, gpu_compute_submitted_slot(c), d, n);
}
int gpu_compute_get_mv_staging_data(gpu_context_t* c, void** d, size_t* n) {
  return gpu_compute_get_mv_staging_data_slot(c, gpu_compute_submitted_slot(c), d, n);
}
int gpu_compute_get_nz_staging_data(gpu_context_t* c, void** d, size_t* n) {
  return gpu_compute_get_nz_staging_data_slot(c, gpu_compute_submitted_slot(c), d, n);
}

void gpu_compute_debug_dump_recon(gpu_context_t* ctx, int width, int height) {
  Impl* m = impl_of(ctx);
  const char* on = getenv("BC250_DUMP_RECON_FRAMES");
  if (!m || !on || strcmp(on, "1") != 0 || !m->rec[0] || width <= 0 || height <= 0) return;
  char name[64];
  snprintf(name, sizeof(name), "recon_%05u.nv12", ctx->frames_submitted);
  FILE* f = bc250_debug_dump_open(name, "BC250_DUMP_RECON_FRAMES");
  if (!f) return;
  const size_t luma = (size_t)m->pitch * m->mbh * 16;
  uint8_t* host = (uint8_t*)malloc(m->rec_bytes);
  if (host && cudaMemcpy(host, m->rec[m->cur], m->rec_bytes, cudaMemcpyDeviceToHost) == cudaSuccess) {
    for (int r = 0; r < height; ++r) fwrite(host + (size_t)r * m->pitch, 1, width, f);
    for (int r = 0; r < height / 2; ++r) fwrite(host + luma + (size_t)r * m->pitch, 1, width, f);
  }
  free(host);
  fclose(f);
}

int b200enc_ctx_configure(gpu_context_t* ctx, int search_range, int lambda, int zero_thresh, int recon_clamp_coded,
                          int deblock) {
  Impl* m = impl_of(ctx);
  if (!m || (search_range != 16 && search_range != 32) || lambda > 1023) return -1;
  m->range = search_range;
  m->lambda = lambda;
  m->zero_thresh = zero_thresh;
  if (m->clamp_coded != (recon_clamp_coded ? 1 : 0)) ctx->has_recon_frame = false;
  m->clamp_coded = recon_clamp_coded ? 1 : 0;
  m->deblock = deblock;
  return 0;
}

int b200enc_ctx_set_me(gpu_context_t* ctx, int mode, const char* weights, float conf) {
  Impl* m = impl_of(ctx);
  if (!m || mode < 0 || mode > 3) return -1;
  cudaStreamSynchronize(m->stream);
  m->me_mode = mode;
  m->weights = weights ? weights : "";
  m->conf = conf;
  if (m->prop) {
    b200enc_proposal_destroy(m->prop);
    m->prop = nullptr;
    m->prop_mbs = 0;
  }
  if (mode != 0 && m->mbw > 0) return ensure_proposal(m);
  if ((mode == 1 || mode == 3) && m->mbw == 0) {  // check the checkpoint now, before the first frame
    void* probe = b200enc_proposal_create(1);
    if (!probe) return -1;
    const int rc = b200enc_proposal_load(probe, (m->weights.empty() ? default_weights() : m->weights).c_str());
    b200enc_proposal_destroy(probe);
    return rc;
  }
  return 0;
}

int b200enc_ctx_set_entropy(gpu_context_t* ctx, int mode, int quality_level) {
  Impl* m = impl_of(ctx);
  if (!m || mode < 0 || mode > 2 || quality_level < 1 || quality_level > 7) return -1;
  m->entropy = mode;
  m->quality = quality_level;
  return 0;
}

namespace {

// Appends bits MSB first to a byte stream, inserting emulation_prevention_
// three_byte (7.4.1: after two zero bytes, a byte <= 3 is preceded by 0x03;
// the reference's bs_rbsp_to_ebsp, bitstream.c:233-250, does the same).
struct NalOut {
  uint8_t* p;
  size_t cap, n = 0;
  int zeros = 0;
  uint64_t acc = 0;
  int nacc = 0;
  bool over = false;
  void byte(uint8_t b) {
    if (zeros == 2 && b <= 3) {
      raw(3);
      zeros = 0;
    }
    raw(b);
    zeros = b == 0 ? zeros + 1 : 0;
  }
  void raw(uint8_t b) {
    if (n < cap) p[n] = b;
    else over = true;
    ++n;
  }
  void put(int bits, uint32_t v) {  // bits <= 32
    if (bits <= 0) return;
    if (bits < 32) v &= (1u << bits) - 1u;
    acc = (acc << bits) | v;
    nacc += bits;
    while (nacc >= 8) {
      nacc -= 8;
      byte((uint8_t)(acc >> nacc));
    }
    acc &= nacc ? ((1ull << nacc) - 1ull) : 0ull;
  }
};

}  // namespace

int b200enc_ctx_slice_nals(gpu_context_t* ctx, int slot, const uint8_t* headers, const int* header_bits,
                           int nal_ref_idc, int nal_unit_type, uint8_t* out, size_t cap, size_t* written) {
  Impl* m = impl_of(ctx);
  if (!m || slot < 0 || slot > 1 || !out || !written || nal_ref_idc < 0 || nal_ref_idc > 3 || nal_unit_type < 1 ||
      nal_unit_type > 31)
    return -1;
  Slot& sl = m->slot[slot];
  if (!sl.slices || sl.num_slices <= 0) return -1;
  if (gpu_compute_sync_slot(ctx, slot) != 0) return -1;
  NalOut o{out, cap};
  for (int s = 0; s < sl.num_slices; ++s) {
    const uint32_t nb = sl.slice_bytes[s];
    if (nb == 0xffffffffu || nb == 0) return -1;
    const int hb = header_bits ? header_bits[s] : 0;
    if (hb < 0 || hb > 128 || (hb > 0 && !headers)) return -1;
    // start code and NAL header (never escaped), then the RBSP: the caller's
    // header bits, the slice data (the GPU's RBSP up to its stop bit), the
    // stop bit and the alignment zeros
    o.raw(0);
    o.raw(0);
    o.raw(0);
    o.raw(1);
    o.raw((uint8_t)((nal_ref_idc << 5) | nal_unit_type));
    o.zeros = 0;
    const uint8_t* h = headers ? headers + 16 * s : nullptr;
    for (int k = 0; k < hb; k += 8) o.put(std::min(8, hb - k), (uint32_t)(h[k >> 3] >> (8 - std::min(8, hb - k))));
    const uint8_t* d = sl.slices + (size_t)s * slice_cap_of((size_t)m->mbw * m->mbh, sl.num_slices);
    const uint8_t last = d[nb - 1];
    const int data_bits_last = 7 - __builtin_ctz(last);  // bits before the stop bit in the last byte
    for (uint32_t k = 0; k + 1 < nb; ++k) o.put(8, d[k]);
    o.put(data_bits_last, (uint32_t)(last >> (8 - data_bits_last)));
    o.put(1, 1u);
    if (o.nacc) o.put(8 - o.nacc, 0u);
  }
  *written = o.n;
  return o.over ? -1 : 0;
}

int b200enc_ctx_me_stats(gpu_context_t* ctx, int* learned, int* fallback, int* early) {
  Impl* m = impl_of(ctx);
  if (!m) return -1;
  int c[4] = {0, 0, 0, 0};
  if (m->prop && m->last_learned) {
    void* ptr = nullptr;
    size_t n = 0;
    if (b200enc_proposal_tensor(m->prop, 15, &ptr, &n) != 0) return -1;
    if (cudaMemcpyAsync(c, ptr, sizeof(c), cudaMemcpyDeviceToHost, m->stream) != cudaSuccess) return -1;
    if (cudaStreamSynchronize(m->stream) != cudaSuccess) return -1;
  }
  if (learned) *learned = c[0];
  if (fallback) *fallback = c[1];
  if (early) *early = c[3];
  return 0;
}

void* b200enc_ctx_stream(gpu_context_t* ctx) {
  Impl* m = impl_of(ctx);
  return m ? (void*)m->stream : nullptr;
}

int b200enc_ctx_recon(gpu_context_t* ctx, void** y, void** uv, int* pitch) {
  Impl* m = impl_of(ctx);
  if (!m || !m->rec[0] || !y || !uv || !pitch) return -1;
  *y = m->rec[m->cur];
  *uv = m->rec[m->cur] + (size_t)m->pitch * m->mbh * 16;
  *pitch = m->pitch;
  return 0;
}

int b200enc_ctx_device_outputs(gpu_context_t* ctx, void** levels, void** dc, void** nz, void** pred_mode, void** mv) {
  Impl* m = impl_of(ctx);
  if (!m || !m->d_levels) return -1;
  if (levels) *levels = m->d_levels;
  if (dc) *dc = m->d_dc;
  if (nz) *nz = m->d_nz;
  if (pred_mode) *pred_mode = m->d_pred_mode;
  if (mv) *mv = m->d_mv;
  return 0;
}

int b200enc_ctx_encode_device(gpu_context_t* ctx, const uint8_t* y, const uint8_t* uv, int pitch, int width,
                              int height, int qp, int is_intra, int num_slices, int stage_outputs) {
  Impl* m = impl_of(ctx);
  if (!m || !y || !uv || (pitch & 3)) return -1;
  return encode_frame(ctx, m, y, uv, pitch, width, height, qp, is_intra, num_slices, 0, nullptr, stage_outputs != 0);
}

int b200enc_host_register(gpu_context_t* ctx, void* ptr, size_t bytes) {
  Impl* m = impl_of(ctx);
  if (!m || !ptr || bytes == 0 || m->registered.count(ptr)) return -1;
  if (cudaHostRegister(ptr, bytes, cudaHostRegisterDefault) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  m->registered[ptr] = bytes;
  return 0;
}

int b200enc_host_unregister(gpu_context_t* ctx, void* ptr) {
  Impl* m = impl_of(ctx);
  if (!m || !ptr) return -1;
  auto it = m->registered.find(ptr);
  if (it == m->registered.end()) return -1;
  // copies from the buffer may still be queued
  cudaStreamSynchronize(m->stream);
  m->registered.erase(it);
  return cudaHostUnregister(ptr) == cudaSuccess ? 0 : -1;
}

int b200enc_ctx_perf(gpu_context_t* ctx, int enable) {
  Impl* m = impl_of(ctx);
  if (!m) return -1;
  if (enable && !m->ev[0][0]) {
    for (auto& row : m->ev)
      for (cudaEvent_t& e : row)
        if (cudaEventCreate(&e) != cudaSuccess) return -1;
  }
  cudaStreamSynchronize(m->stream);
  while (m->ev_count > 0) perf_fold_one(m);
  m->perf = enable != 0;
  memset(m->stage_ms, 0, sizeof(m->stage_ms));
  m->stage_frames[0] = m->stage_frames[1] = 0;
  return 0;
}

int b200enc_ctx_perf_read(gpu_context_t* ctx, int intra, double* me_ms, double* chain_ms, double* deblock_ms,
                          double* staging_ms, long* frames) {
  Impl* m = impl_of(ctx);
  if (!m) return -1;
  cudaStreamSynchronize(m->stream);
  while (m->ev_count > 0) perf_fold_one(m);
  const int k = intra ? 1 : 0;
  if (me_ms) *me_ms = m->stage_ms[k][0];
  if (chain_ms) *chain_ms = m->stage_ms[k][1];
  if (deblock_ms) *deblock_ms = m->stage_ms[k][2];
  if (staging_ms) *staging_ms = m->stage_ms[k][3];
  if (frames) *frames = m->stage_frames[k];
  return 0;
}

}  // extern "C"
