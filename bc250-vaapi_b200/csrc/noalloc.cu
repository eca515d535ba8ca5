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
#include <cstdio>
#include <mutex>

#include "b200enc_internal.h"

namespace {

// Largest frame the static scratch covers: 512 macroblock rows (8192 luma
// rows). Words: ticket, error, detail, reserved + luma and chroma progress.
constexpr int kNoAllocMaxMbRows = 512;
constexpr size_t kNoAllocScratchWords = 4 + 2 * (size_t)kNoAllocMaxMbRows;  // 4112 bytes

// One copy per device that loads this library; it stays resident until the
// process exits. Every call on a device shares it.
static __device__ __align__(256) uint32_t g_deblock_scratch[kNoAllocScratchWords];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
uint32_t* g_addr[kMaxDevices] = {};

// Device address of the scratch on the current device. In host code the
// array's name is only a host-side stand-in, so the address has to come from
// cudaGetSymbolAddress, once per device, with that device current.
uint32_t* scratch_on_current_device() {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_deblock_scratch);
    if (e != cudaSuccess || !p) {
      fprintf(stderr, "[b200enc] b200enc_deblock_noalloc: cudaGetSymbolAddress failed on device %d: %s\n", dev,
              cudaGetErrorString(e));
      return nullptr;
    }
    g_addr[dev] = static_cast<uint32_t*>(p);
  }
  return g_addr[dev];
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
  uint32_t* scratch = scratch_on_current_device();
  if (!scratch) return -1;
  // The array keeps whatever the previous call left: the ticket, error and
  // progress words this frame uses must start at zero.
  const size_t words = 4 + 2 * (size_t)mbh;
  if (cudaMemsetAsync(scratch, 0, words * sizeof(uint32_t), (cudaStream_t)stream) != cudaSuccess) return -1;
  return b200enc_deblock_launch(mbw, mbh, qp, is_intra, nz, mv, rec_y, rec_uv, rec_pitch, scratch, 0, 2000000u,
                                stream);
}
