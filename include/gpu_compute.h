/*
 * gpu_compute.h - drop-in replacement of the reference compute encoder's GPU
 * boundary (approach1-compute-encoder/src/gpu_compute.h), backed by CUDA on
 * a B200 instead of Vulkan.
 *
 * The reference's host encoder (src/encoder_h264.c) compiles unchanged
 * against this header and links against libb200enc.so: it imports exactly
 * the entry points marked [encoder] below. Types keep the reference's names
 * and the fields the encoder touches (gpu_image_t.y_plane,
 * gpu_memory_t.memory, the context's has_recon_frame / recon_image /
 * recon_memory / any_surface_exported); handles that were Vulkan objects are
 * now device pointers, and VK_NULL_HANDLE means NULL.
 *
 * Conventions kept from the reference: int returns are 0 on success and -1
 * on failure, nothing aborts; two staging slots (double buffering); staging
 * pointers stay valid until that slot is submitted again; layouts per
 * gpu_compute.h:575-648 of the reference (see include/b200enc.h).
 *
 * Environment knobs read by the library:
 *   BC250_FAST_MODE=1          skip deblocking (reference semantics)
 *   BC250_GPU_TIMEOUT_MS=N     bound the waits in begin_picture/sync_slot
 *   BC250_DUMP_RECON_FRAMES=1  debug_dump_recon writes NV12 to BC250_DUMP_DIR
 *   B200ENC_SEARCH_RANGE=16|32 integer full-search range (default 16)
 *   B200ENC_RECON_CLAMP=coded|visible  where reference reads clamp
 *                              (default coded = what a decoder does)
 *   B200ENC_INTRA_PLANE=shader the reference shader's Plane availability
 *                              (default: also require the top-left slice)
 */
#ifndef GPU_COMPUTE_H
#define GPU_COMPUTE_H

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifndef VK_NULL_HANDLE
#define VK_NULL_HANDLE NULL
#endif

#define GPU_IMAGE_NV12 0
#define GPU_IMAGE_P010 1

/* Reference: gpu_compute.h:17-45 (VkImage/VkImageView pair per plane). */
typedef struct {
    void *y_plane;          /* device pointer to luma; NULL = no image */
    void *y_view;           /* == y_plane (source compatibility) */
    void *uv_plane;         /* device pointer to interleaved CbCr */
    void *uv_view;          /* == uv_plane */
    uint32_t width;
    uint32_t height;
    int current_layout;     /* unused, kept for source compatibility */
    int format;             /* GPU_IMAGE_NV12 or GPU_IMAGE_P010 */
    uint32_t pitch;         /* bytes per row, both planes */
} gpu_image_t;

/* Reference: gpu_compute.h:47-51 (VkDeviceMemory). */
typedef struct {
    void *memory;           /* device allocation base; NULL = none */
    size_t size;
    void *mapped_ptr;       /* host shadow while mapped */
} gpu_memory_t;

/* Reference: gpu_compute.h:55-62. */
typedef struct {
    uint32_t y_pitch;
    uint64_t y_offset;
    uint32_t uv_pitch;
    uint64_t uv_offset;
    uint64_t total_size;
} gpu_nv12_layout_t;

/* Reference: gpu_compute.h:575-579. */
typedef struct {
    int32_t mvx, mvy;
    uint32_t sad;
    uint32_t _pad;
} gpu_mv_t;

/* Reference: gpu_compute.h:64-352 (caller-allocated, library-filled). */
typedef struct bc250_gpu_context {
    gpu_image_t recon_image;    /* latest reconstruction (next reference) */
    gpu_memory_t recon_memory;
    bool has_recon_frame;
    bool any_surface_exported;  /* always false: no dma-buf export here */
    uint32_t frame_width;
    uint32_t frame_height;
    uint32_t frames_submitted;
    int current_buf;
    void *impl;                 /* library-owned CUDA state */
} bc250_gpu_context_t;

typedef bc250_gpu_context_t gpu_context_t;

/* ---- lifecycle (reference gpu_compute.h:357-377) ---------------------- */
int bc250_gpu_init(bc250_gpu_context_t *ctx);
void bc250_gpu_destroy(bc250_gpu_context_t *ctx);
int gpu_compute_init(gpu_context_t *ctx);
void gpu_compute_terminate(gpu_context_t *ctx);

/* ---- surfaces (reference gpu_compute.h:380-443) ----------------------- */
int gpu_compute_create_image(gpu_context_t *ctx, int width, int height, int format,
                             gpu_image_t *image, gpu_memory_t *memory);
void gpu_compute_destroy_image(gpu_context_t *ctx, gpu_image_t image, gpu_memory_t memory);
int gpu_compute_get_nv12_layout(gpu_context_t *ctx, gpu_image_t *image, gpu_memory_t memory,
                                gpu_nv12_layout_t *layout);
/* [encoder] reference :393-397. Returns a host copy of the surface (both
 * planes at layout offsets); *unmap says whether unmap must be called,
 * which writes the host copy back. */
uint8_t *gpu_compute_map_surface(gpu_context_t *ctx, gpu_image_t *image, gpu_memory_t memory,
                                 gpu_nv12_layout_t *layout, bool *unmap);
void gpu_compute_unmap_surface(gpu_context_t *ctx, gpu_memory_t memory, bool unmap);
int gpu_compute_upload_nv12(gpu_context_t *ctx, gpu_image_t *image, gpu_memory_t memory,
                            const uint8_t *y_plane, int y_pitch,
                            const uint8_t *uv_plane, int uv_pitch, int width, int height);
int gpu_compute_download_nv12(gpu_context_t *ctx, gpu_image_t *image, gpu_memory_t memory,
                              uint8_t *y_plane, int y_pitch,
                              uint8_t *uv_plane, int uv_pitch, int width, int height);
/* [encoder] reference :439. */
void gpu_compute_copy_from_wc(void *dst, const void *src, size_t n);
/* [encoder] reference :538: no foreign producers here, returns 0. */
int gpu_compute_wait_for_image_ready_host(gpu_context_t *ctx, gpu_memory_t memory);
/* [encoder] reference :553: 1 when no submitted frame is still running. */
int gpu_compute_cpu_read_safe(gpu_context_t *ctx);
/* [encoder] reference :559. */
FILE *bc250_debug_dump_open(const char *name, const char *what);

/* ---- picture encoding (reference gpu_compute.h:582-648) --------------- */
/* [encoder] Waits (bounded by BC250_GPU_TIMEOUT_MS) until the current
 * slot's previous frame is done. */
int gpu_compute_begin_picture(gpu_context_t *ctx, gpu_image_t render_target);
int gpu_compute_dispatch_encode(gpu_context_t *ctx, gpu_image_t render_target, int width, int height,
                                int qp, int is_intra, int num_slices);
/* [encoder] Enqueues the whole hot path of one frame: full-search ME (P,
 * unless cpu_mvs is given: then those MVs are uploaded instead), the fused P
 * chain or the intra wavefront, deblocking (unless BC250_FAST_MODE=1), and
 * the staging copies of levels/dc/pred_mode/mv/nz into the current slot.
 * me_mode 1 = the reference's fast mode (lambda 8 instead of 5). */
int gpu_compute_dispatch_encode_ext(gpu_context_t *ctx, gpu_image_t render_target, int width, int height,
                                    int qp, int is_intra, int num_slices, int me_mode,
                                    const gpu_mv_t *cpu_mvs);
/* ME only into the MV staging of the current slot (reference :594). */
int gpu_compute_dispatch_me_only(gpu_context_t *ctx, gpu_image_t render_target, int width, int height);
/* [encoder] */
double gpu_compute_get_last_latency_ms(const gpu_context_t *ctx);
/* [encoder] Marks the frame submitted and flips slots. */
int gpu_compute_end_picture(gpu_context_t *ctx);
int gpu_compute_sync(gpu_context_t *ctx);
/* [encoder] */
int gpu_compute_submitted_slot(gpu_context_t *ctx);
/* [encoder] Waits for `slot`; -1 on timeout or if a wavefront wait gave up
 * (the caller then emits an all-skip frame, reference encoder_h264.h:60-64). */
int gpu_compute_sync_slot(gpu_context_t *ctx, int slot);
/* [encoder] x5 */
int gpu_compute_get_quant_staging_data_slot(gpu_context_t *ctx, int slot, void **data, size_t *size);
int gpu_compute_get_dc_staging_data_slot(gpu_context_t *ctx, int slot, void **data, size_t *size);
int gpu_compute_get_pred_mode_staging_data_slot(gpu_context_t *ctx, int slot, void **data, size_t *size);
int gpu_compute_get_mv_staging_data_slot(gpu_context_t *ctx, int slot, void **data, size_t *size);
int gpu_compute_get_nz_staging_data_slot(gpu_context_t *ctx, int slot, void **data, size_t *size);
int gpu_compute_get_staging_data(gpu_context_t *ctx, void **data, size_t *size);
int gpu_compute_release_staging_data(gpu_context_t *ctx);
int gpu_compute_get_quant_staging_data(gpu_context_t *ctx, void **data, size_t *size);
int gpu_compute_get_dc_staging_data(gpu_context_t *ctx, void **data, size_t *size);
int gpu_compute_get_pred_mode_staging_data(gpu_context_t *ctx, void **data, size_t *size);
int gpu_compute_get_mv_staging_data(gpu_context_t *ctx, void **data, size_t *size);
int gpu_compute_get_nz_staging_data(gpu_context_t *ctx, void **data, size_t *size);
/* [encoder] No-op unless BC250_DUMP_RECON_FRAMES=1. */
void gpu_compute_debug_dump_recon(gpu_context_t *ctx, int width, int height);

/* ---- B200 extensions (no reference counterpart) ------------------------ */
/* Search range (16 or 32), lambda override (-1 keeps 5/8 per me_mode),
 * zero-MV threshold (<0 disables, reference 512), recon clamp (1 coded,
 * 0 visible), deblock (1 on, 0 off, -1 per BC250_FAST_MODE). */
int b200enc_ctx_configure(gpu_context_t *ctx, int search_range, int lambda, int zero_thresh,
                          int recon_clamp_coded, int deblock);
/* The CUDA stream the context enqueues on (cudaStream_t as void*). */
void *b200enc_ctx_stream(gpu_context_t *ctx);
/* Device pointers of the latest reconstruction (coded size, NV12). */
int b200enc_ctx_recon(gpu_context_t *ctx, void **y, void **uv, int *pitch);
/* Device pointers of the per-frame outputs (same layouts as staging). */
int b200enc_ctx_device_outputs(gpu_context_t *ctx, void **levels, void **dc, void **nz,
                               void **pred_mode, void **mv);
/* One frame from device planes already in HBM (no gpu_image_t needed);
 * stage_outputs = 0 skips the device-to-host staging copies. */
int b200enc_ctx_encode_device(gpu_context_t *ctx, const uint8_t *y, const uint8_t *uv, int pitch,
                              int width, int height, int qp, int is_intra, int num_slices,
                              int stage_outputs);

/* Motion estimation form of P frames: mode 0 = plain full search (default),
 * 1 = learned proposal (b200enc_proposal_me) with the network parameters of
 * checkpoint `weights` (NULL: the packaged proposal_h264.b2pn next to the
 * library's b200enc package) and confidence threshold conf, 2 = the same
 * candidate search without the network, falling back when the best
 * candidate's cost per pel exceeds conf (conf < 0: never), 3 = mode 1 with
 * the network's inference in FP8 E4M3. The first P frame
 * after an I frame, and any P frame without a previous MV field, uses the
 * full search. Env: B200ENC_ME=learned|candidates|learned_fp8, B200ENC_PROPOSAL_WEIGHTS,
 * B200ENC_PROPOSAL_CONF. Returns -2 if the checkpoint is missing or bad. */
int b200enc_ctx_set_me(gpu_context_t *ctx, int mode, const char *weights, float conf);
/* Learned-form counters of the last P frame: MBs re-scored from the network's
 * candidates, MBs that fell back to the full search, zero-MV early-outs
 * (synchronises the context stream). */
int b200enc_ctx_me_stats(gpu_context_t *ctx, int *learned, int *fallback, int *early);
/* Entropy coding on the GPU (no reference counterpart: the reference codes
 * slices on the host, encoder_h264.c:3128-3290, 57 % of a 1440p frame by its
 * DEVLOG). mode 1: every dispatched frame also gets its CAVLC slice data
 * coded on the GPU (b200enc_cavlc_slices) into the slot's page-locked
 * memory, beside the usual staging; mode 2: the same, and the slot's levels,
 * DC, nz and mode staging copies are skipped (a caller that does not run the
 * host entropy coder: ~8 MB less over the bus per 1080p frame); 0 (default):
 * off. quality_level is the host encoder's (1..7, default 4; its P_Skip rule
 * changes at >= 5). */
int b200enc_ctx_set_entropy(gpu_context_t *ctx, int mode, int quality_level);
/* The Annex B NAL units of a slot's slices (after gpu_compute_end_picture;
 * waits for the slot like gpu_compute_sync_slot): for each slice a 4-byte
 * start code, the NAL header (nal_ref_idc, nal_unit_type), then the RBSP -
 * the caller's slice header (header_bits[s] bits, MSB first, from
 * headers + 16 * s) followed by the GPU's slice data and rbsp_trailing_bits -
 * with emulation prevention (7.4.1), as the reference's encoder assembles
 * its slices (encoder_h264.c:3429-3470). The bytes go to out (cap bytes);
 * *written gets their count. Returns 0, or -1 (entropy mode off, bad
 * arguments, a slice that outgrew its region, cap too small). */
int b200enc_ctx_slice_nals(gpu_context_t *ctx, int slot, const uint8_t *headers, const int *header_bits,
                           int nal_ref_idc, int nal_unit_type, uint8_t *out, size_t cap, size_t *written);

/* Per-stage GPU timing with CUDA events, the equivalent of the reference's
 * BC250_PERF_STATS timestamps (gpu_compute.c:50-67). enable resets the
 * sums. perf_read synchronises the stream and returns, for P (intra = 0) or
 * I (intra = 1) frames, the summed milliseconds of ME, the P chain or intra
 * wavefront, deblocking and the staging copies, and the frame count. */
int b200enc_ctx_perf(gpu_context_t *ctx, int enable);
int b200enc_ctx_perf_read(gpu_context_t *ctx, int intra, double *me_ms, double *chain_ms,
                          double *deblock_ms, double *staging_ms, long *frames);

/* Surface ingest without a staging copy. The reference uploads and downloads
 * NV12 through host-visible Vulkan memory (gpu_compute.c:2551, :2699); here
 * a caller's own frame buffers (a decoder's output pool, a capture ring) are
 * page-locked once with b200enc_host_register, after which
 * gpu_compute_upload_nv12 from them is one asynchronous DMA per plane on the
 * context stream, ordered before the next dispatch, with no copy through a
 * bounce buffer and no wait in the call (the caller must not rewrite the
 * buffer until a frame submitted after the upload has been synced).
 * Unregistered pageable buffers still work, synchronously. Registration is
 * process-wide; b200enc_host_unregister (or bc250_gpu_destroy, for what this
 * context registered) undoes it. 0 / -1 (already registered, or the driver
 * refused). */
int b200enc_host_register(gpu_context_t *ctx, void *ptr, size_t bytes);
int b200enc_host_unregister(gpu_context_t *ctx, void *ptr);

#ifdef __cplusplus
}
#endif
#endif /* GPU_COMPUTE_H */
