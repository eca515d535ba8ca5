// noalloc.cu - deblocking for callers that cannot allocate device memory.
//
// The deblocking wavefront needs a little scratch (a row ticket, an error
// word and two progress words per macroblock row). b200enc_deblock takes
// that scratch from the caller, which means the caller has to have
// allocated it. Some callers cannot: an encode thread on a real-time path
// (a game-streaming server's per-frame encode, or a VA-API EndPicture that
// runs under the driver lock) must not call cudaMalloc, whose implicit
// device-wide synchronisation and unbounded latency would stall every
// stream on the GPU; and a plug-in whose host budgets device memory at
// start-up may not add allocations afterwards. This file gives them a
// variant whose scratch lives in a fixed, file-scope device array that the
// module brings with it, so the call itself allocates nothing.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstdio>
#include <mutex>

#include "b200enc_internal.h"

namespace {

// Largest frame the static scratch covers: 512 macroblock rows (8192 luma
// rows). Words: ticket, error, detail, reserved + luma and chroma progress.
constexpr int kNoAllocMaxMbRows = 512;
constexpr size_t kNoAllocScratchWords = 4 + 2 * (size_t)kNoAllocMaxMbRows;  // 4112 bytes

// One copy per CUDA context that loads this library's module (the primary
// context of each device, for ordinary runtime-API callers); it stays
// resident until that context is destroyed. Every call in a context shares it.
static __device__ __align__(256) uint32_t g_deblock_scratch[kNoAllocScratchWords];

// Device addresses already looked up, keyed by the driver's context ID. The
// ID is unique for the life of the process: a context created after
// cudaDeviceReset, or a caller's own driver-API context on the same device,
// gets a new ID and so a fresh lookup, never the address of a context that
// is gone or belongs to someone else.
constexpr int kCacheEntries = 16;
struct CacheEntry {
  unsigned long long ctx_id;
  uint32_t* addr;
};
std::mutex g_mu;
CacheEntry g_cache[kCacheEntries] = {};
int g_cache_next = 0;
PFN_cuCtxGetCurrent_v4000 g_ctx_current = nullptr;
PFN_cuCtxGetId_v12000 g_ctx_id = nullptr;

// ID of the context current on this thread, 0 if none is (or the driver
// entry points are unavailable).
unsigned long long current_context_id() {
  if (!g_ctx_current || !g_ctx_id) {
    void* f1 = nullptr;
    void* f2 = nullptr;
    cudaDriverEntryPointQueryResult q1, q2;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
        cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) != cudaSuccess ||
        q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess)
      return 0;
    g_ctx_current = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(f1);
    g_ctx_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(f2);
  }
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (g_ctx_current(&c) != CUDA_SUCCESS || !c || g_ctx_id(c, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Device address of the scratch in the current context. In host code the
// array's name is only a host-side stand-in, so the address has to come from
// cudaGetSymbolAddress, with the device current; it is looked up once per
// context and cached under the context's ID.
uint32_t* scratch_in_current_context() {
  std::lock_guard<std::mutex> lock(g_mu);
  unsigned long long id = current_context_id();
  if (id != 0) {
    for (const CacheEntry& e : g_cache)
      if (e.ctx_id == id) return e.addr;
  }
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_deblock_scratch);  // makes the primary context current if none is
  if (e != cudaSuccess || !p) {
    int dev = -1;
    cudaGetDevice(&dev);
    fprintf(stderr, "[b200enc] b200enc_deblock_noalloc: cudaGetSymbolAddress failed on device %d: %s\n", dev,
            cudaGetErrorString(e));
    return nullptr;
  }
  if (id == 0) id = current_context_id();
  if (id != 0) {
    g_cache[g_cache_next] = CacheEntry{id, static_cast<uint32_t*>(p)};
    g_cache_next = (g_cache_next + 1) % kCacheEntries;
  }
  return static_cast<uint32_t*>(p);
}

}  // namespace

extern "C" int b200enc_deblock_noalloc(int mbw, int mbh, int qp, int is_intra, const uint32_t* nz, const void* mv,
                                       uint8_t* rec_y, uint8_t* rec_uv, int rec_pitch, void* stream) {
  if (mbh > kNoAllocMaxMbRows) {
    fprintf(stderr,
            "[b200enc] b200enc_deblock_noalloc: %d macroblock rows exceed the built-in scratch (max %d rows, "
            "%d luma lines); use b200enc_deblock with caller scratch\n",
            mbh, kNoAllocMaxMbRows, 16 * kNoAllocMaxMbRows);
    return -2;
  }
  if (!nz || !mv || !rec_y || !rec_uv || mbw <= 0 || mbh <= 0 || qp < 0 || qp > 51) return -1;
  if ((rec_pitch & 15) || (((uintptr_t)rec_y) & 15) || (((uintptr_t)rec_uv) & 15) || rec_pitch < mbw * 16)
    return -1;
  uint32_t* scratch = scratch_in_current_context();
  if (!scratch) return -1;
  // The array keeps whatever the previous call left: the ticket, error and
  // progress words this frame uses must start at zero.
  const size_t words = 4 + 2 * (size_t)mbh;
  if (cudaMemsetAsync(scratch, 0, words * sizeof(uint32_t), (cudaStream_t)stream) != cudaSuccess) return -1;
  return b200enc_deblock_launch(mbw, mbh, qp, is_intra, nz, mv, rec_y, rec_uv, rec_pitch, scratch, 0, 2000000u,
                                stream);
}

extern "C" int b200enc_deblock_noalloc_status(uint32_t* status_host, void* stream) {
  if (!status_host) return -1;
  uint32_t* scratch = scratch_in_current_context();
  if (!scratch) return -1;
  // word 1 of the scratch layout is the error code
  return cudaMemcpyAsync(status_host, scratch + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                         (cudaStream_t)stream) == cudaSuccess
             ? 0
             : -1;
}
