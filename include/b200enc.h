/*
 * b200enc.h - stage-level C-ABI of the B200 compute-encoder hot path.
 *
 * Every pointer argument named *_y, *_uv, levels, dc, nz, pred_mode, mv,
 * rec_* and scratch is DEVICE memory; `stream` is a cudaStream_t passed as
 * void* (NULL = legacy default stream). Planes are 8-bit: luma with a byte
 * pitch, chroma NV12-interleaved (CbCr pairs) with the same pitch. Each call
 * only enqueues work and returns 0, or -1 when an argument is rejected or the
 * launch fails; nothing here allocates. Output layouts are the reference's
 * staging layouts (approach1-compute-encoder/src/gpu_compute.h:575-648):
 *   levels    int16 [mbs][24][16]  (blocks 0-15 luma raster, 16-19 Cb, 20-23 Cr;
 *                                   positions raster within the 4x4 block)
 *   dc        int32 [mbs][24]      pre-quantisation coefficient 0 of each block
 *   nz        uint32[mbs][24]      bit p set iff levels[..][p] != 0
 *   pred_mode uint32[mbs]          I16x16 mode in bits 0-1, chroma mode bits 2-3
 *   mv        b200enc_mv_t[mbs]    quarter-pel MV + SAD, 16 bytes
 * Geometry: W x H is the visible frame (source reads clamp to it); RW x RH is
 * where reference/recon reads clamp and recon writes stop. RW,RH = W,H is the
 * reference shaders' behaviour; RW,RH = 16*ceil(W/16), 16*ceil(H/16) is what
 * a conforming H.264 decoder reconstructs (identical when W, H are multiples
 * of 16). Recon planes must be allocated at the coded size.
 */
#ifndef B200ENC_H
#define B200ENC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int32_t mvx, mvy; /* quarter-pel, points into the reference */
    uint32_t sad;
    uint32_t pad;
} b200enc_mv_t;

/* Plain full-search ME over [-range, range]^2 (range 16 or 32), cost
 * SAD + lambda*(|dx|+|dy|), then the 8 half-pel and 8 quarter-pel refines.
 * Replaces Stage 2, approach1-compute-encoder/shaders/motion_estimation.comp:278-469
 * (dispatched at src/gpu_compute.c:3094-3103). zero_thresh < 0 disables the
 * zero-MV early-out (the reference uses 512). Pitches and plane bases must be
 * multiples of 4. */
int b200enc_me_full_search(const uint8_t *cur_y, int cur_pitch,
                           const uint8_t *ref_y, int ref_pitch,
                           int W, int H, int RW, int RH,
                           int range, int lambda, int zero_thresh,
                           void *mv_out, void *stream);

/* The same search over a device list of MB indices (raster mby*mbw+mbx):
 * mb_list[0 .. *mb_count) with *mb_count <= list_capacity (device words,
 * written by an earlier kernel, so the host never reads the count); only
 * listed MBs' mv_out entries are written. mb_list == mb_count == NULL
 * searches every MB. flags B200ENC_ME_LOG_INTEGER writes the integer winner
 * into mv.pad: bit 31 set, bit 30 = zero-MV early-out, bits 8-15 dy+128,
 * bits 0-7 dx+128 (the qpel refine can move the MV up to 3/4 pel, so the
 * integer winner is not recoverable from mvx, mvy); used to log training
 * labels for the motion-proposal network. No reference counterpart. */
#define B200ENC_ME_LOG_INTEGER 1
int b200enc_me_full_search_ex(const uint8_t *cur_y, int cur_pitch,
                              const uint8_t *ref_y, int ref_pitch,
                              int W, int H, int RW, int RH,
                              int range, int lambda, int zero_thresh,
                              void *mv_out, const int *mb_list, const int *mb_count,
                              int list_capacity, int flags, void *stream);

/* The full search stages each reference window with one TMA copy when the
 * window lies inside the plane (base and pitch 16-byte aligned); the wait
 * for it is bounded (2 s). A copy that never completes leaves the MB's
 * mv_out entry {0, 0, sad 0xffffffff} and sets a sticky device word: this
 * returns it (0 none, 1 wait timeout, -1 on a CUDA error), clearing it when
 * `clear` is non-zero. Contexts (gpu_compute.h) report it through the
 * frame's status instead. */
int b200enc_me_wait_errors(int clear);

/* Fused P-frame chain given MVs: MC prediction, residual, forward 4x4, AC
 * quant (inter rounding), nz masks, chroma DC, dequant, inverse, recon.
 * Replaces residual_predict.comp (P path) + dct_transform.comp +
 * quantize.comp + reconstruct.comp (src/gpu_compute.c:3121-3183). rec pitch
 * and rec/levels bases must be multiples of 16. */
int b200enc_p_frame(const uint8_t *cur_y, const uint8_t *cur_uv, int cur_pitch,
                    const uint8_t *ref_y, const uint8_t *ref_uv, int ref_pitch,
                    int W, int H, int RW, int RH, int qp, const void *mv,
                    int16_t *levels, int32_t *dc, uint32_t *nz, uint32_t *pred_mode,
                    uint8_t *rec_y, uint8_t *rec_uv, int rec_pitch, void *stream);

/* Bytes of scratch the wavefront kernels (intra, deblock) need for a frame
 * of mbh macroblock rows: a ticket, an error word and two progress words per
 * row (luma and chroma wavefronts). The scratch must be zeroed before each launch; the *_frame calls
 * below do that themselves on `stream`. */
size_t b200enc_wavefront_scratch_bytes(int mbh);

/* Intra flag: Intra16x16 Plane also requires the top-left macroblock to be
 * in the current slice (Plane predicts from p[-1,-1], so a decoder needs it).
 * Without the flag the decision is the reference shader's
 * (shaders/intra_wavefront.comp:463-497 checks only top and left), which can
 * pick Plane across a slice that starts at the top neighbour; the reference
 * host encoder then writes a non-conforming stream that decoders
 * reconstruct differently. The gpu_compute_* layer sets the flag unless
 * B200ENC_INTRA_PLANE=shader. */
#define B200ENC_INTRA_CORNER_CHECK 1

/* I-frame intra wavefront: I16x16 4-mode decision from reconstructed
 * neighbours, chroma DC prediction, full transform/quant/DC/recon chain per
 * macroblock, in a persistent kernel whose CTAs take macroblock rows by
 * ticket and wait (bounded) on per-row progress words for the top
 * neighbour. Replaces the per-diagonal dispatch loop over
 * shaders/intra_wavefront.comp (src/gpu_compute.c:3217-3251). Writes
 * mv[] = 0. rec planes are read and written in place. */
int b200enc_i_frame(const uint8_t *cur_y, const uint8_t *cur_uv, int cur_pitch,
                    int W, int H, int RW, int RH, int qp, int num_slices,
                    int16_t *levels, int32_t *dc, uint32_t *nz, uint32_t *pred_mode, void *mv,
                    uint8_t *rec_y, uint8_t *rec_uv, int rec_pitch,
                    void *scratch, size_t scratch_bytes, int ctas, int flags, void *stream);

/* Spec deblocking (H.264 clause 8.7) of the coded picture, luma and chroma,
 * bS 0-4 with the strong filter, for this encoder's macroblock kinds
 * (all-I16x16 or all-P16x16/P_Skip frames, uniform QP, idc 0, zero
 * offsets). Macroblocks run as a wavefront (left neighbour and top-right
 * neighbour first), which reproduces raster order exactly. Replaces
 * shaders/deblock_filter.comp (src/gpu_compute.c:3261-3290), whose
 * luma-only, no-strong-filter approximation a decoder does not reproduce. */
int b200enc_deblock(int mbw, int mbh, int qp, int is_intra,
                    const uint32_t *nz, const void *mv,
                    uint8_t *rec_y, uint8_t *rec_uv, int rec_pitch,
                    void *scratch, size_t scratch_bytes, int ctas, void *stream);

/* The same deblocking (identical output), from an unfiltered reconstruction
 * src_y/src_uv to a separate destination dst_y/dst_uv (same pitch; the
 * destination planes must not overlap the source planes), as independent
 * tiles: each tile of TW x TH macroblocks (8 x 8 unless tuned,
 * B200ENC_TUNE_DEBLOCK_TILE_W/_H) is deblocked in raster order together with
 * one macroblock of margin on every side and stored alone, which reproduces
 * the whole picture's raster order on the tile. Replaces the same shader
 * dispatch as b200enc_deblock (src/gpu_compute.c:3261-3290). `status` is 16
 * bytes of device memory, zeroed here; word 1 is nonzero if a wait inside a
 * tile gave up. Pitch and bases must be multiples of 16. */
int b200enc_deblock_tiles(int mbw, int mbh, int qp, int is_intra,
                          const uint32_t *nz, const void *mv,
                          const uint8_t *src_y, const uint8_t *src_uv,
                          uint8_t *dst_y, uint8_t *dst_uv, int pitch,
                          uint32_t *status, void *stream);

/* The two wavefront kernels with a caller-prepared scratch (NOT cleared
 * here) and an explicit time bound, in microseconds, on each progress wait.
 * For callers that manage the scratch themselves, and for tests of the
 * bounded wait (a scratch whose ticket starts past the first row (group)
 * leaves it unowned, so every wait on it gives up after max_wait us and
 * records error 1). */
int b200enc_i_frame_launch(const uint8_t *cur_y, const uint8_t *cur_uv, int cur_pitch,
                           int W, int H, int RW, int RH, int qp, int num_slices,
                           int16_t *levels, int32_t *dc, uint32_t *nz, uint32_t *pred_mode, void *mv,
                           uint8_t *rec_y, uint8_t *rec_uv, int rec_pitch,
                           uint32_t *scratch, int ctas, uint32_t max_wait, int flags, void *stream);
int b200enc_deblock_launch(int mbw, int mbh, int qp, int is_intra, const uint32_t *nz, const void *mv,
                           uint8_t *rec_y, uint8_t *rec_uv, int rec_pitch,
                           uint32_t *scratch, int ctas, uint32_t max_wait, void *stream);

/* b200enc_deblock for callers that cannot allocate device memory. No
 * counterpart in the reference. A real-time encode thread (a streaming
 * server's per-frame encode, a VA-API EndPicture under the driver lock) must
 * not call cudaMalloc, which synchronises the whole device and can stall for
 * milliseconds, and a plug-in whose device memory is budgeted at start-up may
 * not allocate later; neither can provide the scratch b200enc_deblock wants.
 * This variant uses a fixed scratch array built into the library (4112
 * bytes per device, resident until the process exits) and allocates nothing;
 * the caller still passes the planes, nz and MVs.
 *   - Limit: mbh <= 512 macroblock rows (frames up to 8192 lines); larger
 *     frames return -2 with a message on stderr. Bad arguments return -1.
 *   - The first call in each CUDA context (the device's primary context for
 *     runtime-API callers; a new one after cudaDeviceReset) looks up the
 *     array's device address (cudaGetSymbolAddress, with that device
 *     current) and caches it under the context's ID; make that first call
 *     before any stream capture.
 *   - Every call on a device shares the one array and zeroes the part it
 *     uses on `stream` before launching: calls whose work overlaps on the GPU
 *     (two streams at once) race on it and must be serialised by the caller.
 * Status: b200enc_deblock_noalloc_status enqueues, on `stream` after the
 * call, a copy of the built-in array's error word into *status_host (0, or
 * 1 when a bounded wait gave up: only if the GPU stopped running the
 * kernel's CTAs for 2 s; the picture is then partly filtered); the word is
 * valid once the stream has reached it. It allocates nothing: a page-locked
 * *status_host keeps the copy asynchronous. 0 / -1. */
int b200enc_deblock_noalloc(int mbw, int mbh, int qp, int is_intra,
                            const uint32_t *nz, const void *mv,
                            uint8_t *rec_y, uint8_t *rec_uv, int rec_pitch, void *stream);
int b200enc_deblock_noalloc_status(uint32_t *status_host, void *stream);

/* ---- Multi-stream batches (no reference counterpart: the reference runs one
 * Vulkan queue per VA context, approach1-compute-encoder/src/gpu_compute.h
 * :246-250) ----------------------------------------------------------------
 * A batch holds n streams of their own frame sizes (even widths and
 * heights). b200enc_batch_encode codes one frame of every stream with one
 * launch per stage over all of them: ME over every P macroblock of every P
 * stream (me_mode 0 full search, 1 learned form with BF16 inference, 3 with
 * FP8), the P chain over the same macroblocks, the intra wavefront over
 * every I stream's macroblock rows, and the deblocking wavefront (deblock !=
 * 0) over every stream's row groups. Each stream's outputs and
 * reconstruction equal a single-stream context's (b200enc_ctx_*, same
 * search range, lambda 5, zero-MV threshold 512, clamping at the coded size,
 * the intra corner check) given the same frames, QPs and frame kinds.
 * Sources are device NV12 planes (pitch a multiple of 4, at least the
 * width); a stream's first frame must be intra. Work is enqueued on the
 * batch's stream (b200enc_batch_stream); b200enc_batch_sync waits and
 * returns -1 if a wavefront gave up. With b200enc_batch_set_graph(b, 1)
 * each step is captured as a CUDA graph and launched, the executable graph
 * updated in place while the step's shape stays the same. Outputs
 * (b200enc_batch_outputs: levels, dc, nz, pred_mode, mv and the
 * reconstruction of the latest step, in the single-frame layouts) stay
 * valid until the next encode. */
typedef struct {
    const uint8_t *y, *uv; /* device NV12 */
    int pitch;             /* bytes */
    int qp;                /* 0..51 */
    int is_intra;
    int num_slices;        /* >= 1 */
} b200enc_batch_frame_t;
void *b200enc_batch_create(int n_streams, const int *widths, const int *heights, int search_range, int me_mode,
                           float conf, int deblock);
void b200enc_batch_destroy(void *b);
void *b200enc_batch_stream(void *b);
int b200enc_batch_set_graph(void *b, int enable);
int b200enc_batch_encode(void *b, const b200enc_batch_frame_t *frames);
int b200enc_batch_sync(void *b);
int b200enc_batch_outputs(void *b, int s, void **levels, void **dc, void **nz, void **pred_mode, void **mv,
                          void **rec_y, void **rec_uv, int *rec_pitch);
/* Graph instantiations and in-place updates so far. */
int b200enc_batch_graph_stats(void *b, long *instantiations, long *updates);

/* Launch parameters picked by the autotuner (no reference counterpart: the
 * reference's dispatch sizes are fixed in gpu_compute.c). Each changes how
 * a kernel's work is laid out, never its results. 0 = the built-in default.
 * The table is process-wide; B200ENC_TUNE_FILE (a file of "name value"
 * lines, as b200enc_tune_name spells the names) is loaded before the first
 * launch. */
#define B200ENC_TUNE_DEBLOCK_ROWS 0         /* macroblock rows per deblocking CTA, 1..6 (default 4) */
#define B200ENC_TUNE_PCHAIN_MBS_PER_CTA 1   /* macroblocks per P-chain CTA, 1, 2 or 4 (default 1) */
#define B200ENC_TUNE_RESCORE_CTAS_PER_SM 2  /* learned re-scoring grid, CTAs per SM, 1..16 (default 8) */
#define B200ENC_TUNE_FALLBACK_CTAS_PER_SM 3 /* fallback full-search grid, CTAs per SM, 1..16 (default 8) */
#define B200ENC_TUNE_INTRA_CTAS 4           /* intra wavefront CTAs (rows in flight), >= 1 (default: one per row) */
#define B200ENC_TUNE_ME_STAGE 5             /* full-search window staging: 1 word loads, 2 TMA (default TMA) */
#define B200ENC_TUNE_DEBLOCK_TILE_W 6       /* tile deblocking: tile width in macroblocks, 1..16 (default 8) */
#define B200ENC_TUNE_DEBLOCK_TILE_H 7       /* tile deblocking: tile height in macroblocks, 1..8 (default 8) */
#define B200ENC_TUNE_COUNT 8
/* Sets a knob (0 restores the default); -1 for an unknown key or a value
 * out of range. */
int b200enc_tune_set(int key, int value);
/* Current value of a knob (0 = default), -1 for an unknown key. */
int b200enc_tune_get(int key);
/* The knob's name in tune files, NULL for an unknown key. */
const char *b200enc_tune_name(int key);
/* Loads "name value" lines; returns the number of knobs set, -1 if the file
 * cannot be read. */
int b200enc_tune_load(const char *path);

/* BF16 GEMM on the tcgen05 tensor cores with FP32 accumulation in tensor
 * memory: C[m][n] (row pitch ldc floats) = epilogue(sum_k A(m,k) * B(n,k)),
 * where A(m,k) = A[m*a_rs + k*a_ks] and B(n,k) = B[n*b_rs + k*b_ks] (BF16,
 * element strides, so transposed operands need no copy). Epilogue flags:
 * ACCUMULATE adds the existing C, then bias[n] (if bias != NULL), then RELU
 * clamps at zero, then OUT_BF16 stores BF16 instead of FP32. `err` (device word, may be NULL) is set to 1 if an
 * mbarrier wait gave up. Used by the motion-proposal network; no reference
 * counterpart (the reference has no dense contraction). */
#define B200ENC_GEMM_ACCUMULATE 1
#define B200ENC_GEMM_RELU 2
#define B200ENC_GEMM_OUT_BF16 4 /* C is BF16 (ldc in elements), rounded to nearest even */
/* Split the K reduction over n CTAs (2..255) that add FP32 partial products
 * into C atomically (C += A.B^T); excludes bias, RELU, ACCUMULATE, OUT_BF16. */
#define B200ENC_GEMM_SPLITK(n) ((n) << 16)
int b200enc_gemm_bf16(int M, int N, int K, const void *A, long long a_rs, long long a_ks,
                      const void *B, long long b_rs, long long b_ks, float *C, long long ldc,
                      const float *bias, int flags, uint32_t *err, void *stream);

/* ---- Learned motion proposal (no reference counterpart) -----------------
 * A small network ranks ten integer MV candidates per MB (the previous
 * frame's co-located MV, its 8 neighbours, zero) from the current 16x16 luma,
 * the residual at the co-located MV and the candidates' exact SADs; the top
 * four distinct candidates' +-2 pel windows are searched exactly with the
 * full search's cost, tie-break and half/quarter-pel refine, and MBs whose
 * top-4 probability is under conf_thresh take the full search. Where the
 * full-search winner lies inside the chosen windows the MV equals
 * b200enc_me_full_search's. A handle owns the parameters (FP32 master + BF16
 * copy), the activations for up to max_mbs MBs, and (on first training use)
 * the gradients and Adam state. Calls on one handle are stream-ordered and
 * must not overlap. */
int b200enc_proposal_num_params(void);
void *b200enc_proposal_create(int max_mbs);
void b200enc_proposal_destroy(void *h);
int b200enc_proposal_set_params(void *h, const float *host_params, int n);
int b200enc_proposal_get_params(void *h, float *host_params, int n);
/* Parameters from a checkpoint file (b200enc.proposal.save_checkpoint format,
 * SHA-256 verified): 0, -1 on I/O or device error, -2 on a bad file. */
int b200enc_proposal_load(void *h, const char *path);
/* Candidates, their SADs, the network input and side features for every MB
 * of a frame; prev_mv = the previous frame's b200enc_mv_t field (NULL: no
 * history). Resets the handle's counters. */
int b200enc_proposal_prepare(void *h, const uint8_t *cur_y, int cur_pitch, const uint8_t *ref_y, int ref_pitch,
                             int W, int H, int RW, int RH, const void *prev_mv, int range, int zero_thresh,
                             void *stream);
int b200enc_proposal_forward(void *h, int mbs, void *stream);
/* Training targets from a full search logged with B200ENC_ME_LOG_INTEGER on
 * the same frame (and, optionally, the plain encode's nz words). */
int b200enc_proposal_labels(void *h, int mbs, const void *logged_mv, const uint32_t *nz, void *stream);
/* Loss gradient through every layer (after forward); gradients overwrite. */
int b200enc_proposal_backward(void *h, int mbs, void *stream);
int b200enc_proposal_adam(void *h, float lr, float beta1, float beta2, float eps, int step, void *stream);
/* forward + backward + Adam (beta 0.9, 0.999, eps 1e-8), step counts from 1 */
int b200enc_proposal_train_step(void *h, int mbs, float lr, int step, void *stream);
/* Motion estimation of one frame in the learned form; prev_mv NULL runs the
 * full search. Same geometry, range, lambda, zero_thresh, mv_out and
 * alignment rules as b200enc_me_full_search. mode 1: the network ranks the
 * candidates and MBs whose top-4 probability is under `param` fall back to
 * the full search. mode 2, the baseline the network is measured against:
 * the 4 distinct candidates of lowest exact cost, falling back when that
 * cost exceeds param * 256 (param < 0: never). mode 3: mode 1 with the
 * network run in FP8 E4M3 on the tensor cores (per-channel weight scales,
 * per-tile activation scales; the BF16-trained parameters are quantised on
 * the fly). */
int b200enc_proposal_me(void *h, const uint8_t *cur_y, int cur_pitch, const uint8_t *ref_y, int ref_pitch,
                        int W, int H, int RW, int RH, const void *prev_mv, int range, int lambda,
                        int zero_thresh, int mode, float param, void *mv_out, void *stream);
/* Device pointer and size of an internal tensor (index list in proposal.cu). */
int b200enc_proposal_tensor(void *h, int which, void **ptr, size_t *bytes);

/* ---- HEVC encoder primitives ----------------------------------------------
 * Batched versions of the per-block routines the reference's HEVC host
 * encoder calls in its RD loop; arrays are device memory, 16-byte aligned,
 * blocks stored row-major back to back (16 or 64 int16 each). Results equal
 * the reference's compiled (SSE2) routines bit for bit. */
/* Forward 4x4 DCT-II (use_dst 0) or DST-VII (use_dst 1) + quantisation of n
 * residual blocks; replaces hevc_transform_quant_4x4 (8-bit, QP clamped to
 * 0..51) and hevc_transform_quant_4x4_10 (10-bit, Qp' clamped to 0..63),
 * approach1-compute-encoder/src/hevc_intra.c:468, :565. round_q12 in 0..12. */
int b200enc_hevc_transform_quant_4x4(const int16_t *residual, int16_t *coeff, int n, int qp, int use_dst,
                                     int round_q12, int bit_depth, void *stream);
/* Dequantisation + inverse 4x4; replaces hevc_dequant_itransform_4x4 and
 * _4x4_10 (hevc_intra.c:484, :586). 8-bit QP must be 0..51. */
int b200enc_hevc_dequant_itransform_4x4(const int16_t *coeff, int16_t *residual, int n, int qp, int use_dst,
                                        int bit_depth, void *stream);
/* Forward 8x8 DCT-II + quantisation (Qp' clamped to 0..63); replaces
 * hevc_transform_quant_8x8 (hevc_intra.c:720). */
int b200enc_hevc_transform_quant_8x8(const int16_t *residual, int16_t *coeff, int n, int qp, int bit_depth,
                                     int round_q12, void *stream);
/* Dequantisation + inverse 8x8; replaces hevc_dequant_itransform_8x8
 * (hevc_intra.c:761). */
int b200enc_hevc_dequant_itransform_8x8(const int16_t *coeff, int16_t *residual, int n, int qp, int bit_depth,
                                        void *stream);
/* The motion search's sample planes of an 8-bit reconstruction (w x h,
 * pitch): whole-sample I and half-sample H, V, HV (8-tap -1 4 -11 40 40 -11
 * 4 -1), each (h + 2*margin) x (w + 2*margin) with plane_pitch, picture
 * edges extended; replaces build_hpel / hpel_pass,
 * approach1-compute-encoder/src/hevc_enc_template.c:219-400 (margin 16 there). */
int b200enc_hevc_build_hpel(const uint8_t *recon, int pitch, int w, int h, int margin, uint8_t *plane_i,
                            uint8_t *plane_h, uint8_t *plane_v, uint8_t *plane_hv, int plane_pitch, void *stream);
/* The same planes of a 10-bit (Main10) reconstruction: samples 0..1023 in
 * 16-bit words, pitches in samples, half-sample values clipped at 1023;
 * replaces build_hpel_10, the BIT_DEPTH 10 instance of the same template
 * (approach1-compute-encoder/src/encoder_h265.c:1220-1227, called at :1571). */
int b200enc_hevc_build_hpel_10(const uint16_t *recon, int pitch, int w, int h, int margin, uint16_t *plane_i,
                               uint16_t *plane_h, uint16_t *plane_v, uint16_t *plane_hv, int plane_pitch,
                               void *stream);

/* b200enc_hevc_build_hpel(_10) from and to host memory, for a host encoder
 * that keeps its reconstruction and planes in host buffers: recon is w x h
 * samples (pitch w; bytes at 8 bits, 16-bit words at 10), planes[4] (I, H,
 * V, HV) each (h + 2*margin) rows of plane_stride samples; replaces the
 * reference's build_hpel_8 / build_hpel_10 on its hevc_encoder_t
 * (approach1-compute-encoder/src/hevc_enc_template.c:390-397). Uses a
 * per-thread device workspace and stream; returns when the planes are in
 * host memory. 0 / -1. */
int b200enc_hevc_build_hpel_host(const void *recon, int w, int h, int bit_depth, int margin, void *const planes[4],
                                 int plane_stride);

/* Page-locks a long-lived host buffer (cudaHostRegister) so that the copies
 * of b200enc_hevc_build_hpel_host to and from it run as DMA without a
 * bounce copy; b200enc_unpin_host undoes it and must run before the buffer
 * is freed. 0 / -1 (already pinned, or the driver refused: copies then stay
 * pageable and correct). */
int b200enc_pin_host(void *ptr, size_t bytes);
int b200enc_unpin_host(void *ptr);

/* Motion search of 8x8 CUs against the planes of b200enc_hevc_build_hpel
 * (8-bit), one job per CU: the reference's motion_search
 * (approach1-compute-encoder/src/hevc_enc_template.c:958-1043, with
 * search_sad :463) step for step: every starting point at the nearest whole
 * sample, a downhill walk (at most 32 steps, within +-64 of the best start,
 * at most 8 samples past the picture), then half- and (qpel != 0)
 * quarter-sample refinement; cost = SAD * 256 + lambda_q8 * the MVD bits to
 * the cheaper predictor. The CU must lie inside the w x h picture (cu_x <=
 * w-8, cu_y <= h-8; a job outside gets sad 0xffffffff and cost -1);
 * margin >= 10 (16 in the reference). Jobs and results are device arrays. */
typedef struct {
    int16_t x, y; /* quarter samples */
} b200enc_hevc_mv_t;
typedef struct {
    int32_t cu_x, cu_y;             /* luma position of the CU */
    b200enc_hevc_mv_t mvp[2];        /* the two AMVP predictors */
    b200enc_hevc_mv_t starts[16];    /* starting points */
    int32_t n_starts;                /* 0..16 */
    int32_t lambda_q8;
} b200enc_hevc_me_job_t;
typedef struct {
    b200enc_hevc_mv_t mv;
    int32_t mvp_idx;                 /* the cheaper predictor */
    int64_t cost_q8;
    uint32_t sad;
    uint32_t pad;
} b200enc_hevc_me_result_t;
int b200enc_hevc_motion_search(const uint8_t *src_y, int src_pitch, int w, int h, const uint8_t *plane_i,
                               const uint8_t *plane_h, const uint8_t *plane_v, const uint8_t *plane_hv,
                               int plane_pitch, int margin, int qpel, const b200enc_hevc_me_job_t *jobs, int n,
                               b200enc_hevc_me_result_t *results, void *stream);
/* The same search on 10-bit (Main10) source and planes (16-bit words,
 * pitches in samples); SADs are brought back to eight-bit units (>> 2)
 * before they are costed, as motion_search_10 / search_sad_10 do
 * (approach1-compute-encoder/src/hevc_enc_template.c:484). */
int b200enc_hevc_motion_search_10(const uint16_t *src_y, int src_pitch, int w, int h, const uint16_t *plane_i,
                                  const uint16_t *plane_h, const uint16_t *plane_v, const uint16_t *plane_hv,
                                  int plane_pitch, int margin, int qpel, const b200enc_hevc_me_job_t *jobs, int n,
                                  b200enc_hevc_me_result_t *results, void *stream);

/* Intra 4x4 luma mode choice of n PUs whose neighbours are already final in
 * recon_y (8-bit): jobs = n x {x0, y0, y_min} (PU position, multiple of 4;
 * first picture row of its slice). For each PU the reference's
 * hevc_choose_luma_mode (approach1-compute-encoder/src/hevc_intra_template.c
 * :177, neighbours :26-117 with the z-scan availability of hevc_intra.c:95-120):
 * Planar, DC, horizontal, vertical by SAD, first best kept; modes[j] = the
 * mode (0, 1, 10, 26), -1 for a position that is not a PU of the picture;
 * preds = n x 16 predicted samples (16-byte aligned). */
int b200enc_hevc_choose_luma_mode(const uint8_t *src_y, int src_pitch, const uint8_t *recon_y, int recon_pitch,
                                  int width, int height, const int *jobs, int n, int *modes, uint8_t *preds,
                                  void *stream);
/* The same choice on 10-bit (Main10) samples (16-bit words, pitches in
 * samples): no-neighbour fill 512, edge filters clipped at 1023; preds =
 * n x 16 samples (16-byte aligned); replaces hevc_choose_luma_mode_10
 * (approach1-compute-encoder/src/hevc_intra.h:152). */
int b200enc_hevc_choose_luma_mode_10(const uint16_t *src_y, int src_pitch, const uint16_t *recon_y,
                                     int recon_pitch, int width, int height, const int *jobs, int n, int *modes,
                                     uint16_t *preds, void *stream);

/* HEVC deblocking (H.265 8.7.2) of one 4:2:0 picture, in place: every
 * vertical edge of the picture, then every horizontal edge over what the
 * vertical pass left. Replaces the deblocking stages of the reference's
 * hevcd_loop_filters (approach1-compute-encoder/src/hevc_filter.c:449-490,
 * stages 0 and 1 = deblock_row over one_direction,
 * hevc_filter_template.c:48-420); SAO is not part of it. The maps are the
 * decoder's (hevc_dec_internal.h:56-70, 133-148, 214-235), in device
 * memory: */
typedef struct {
    int16_t mv[2][2];                /* [list][x, y], quarter samples */
    int32_t ref_poc[2];              /* the picture each list points at */
    uint8_t pred_flag;               /* 0 intra, 1 list 0, 2 list 1, 3 both */
    uint8_t pad[3];
} b200enc_hevc_mvf_t;                /* 20 bytes, one per 4x4 */
typedef struct {
    int16_t beta_offset, tc_offset;  /* slice_beta/tc_offset_div2 * 2 */
    uint8_t disabled;                /* slice_deblocking_filter_disabled_flag */
    uint8_t across_slices;           /* slice_loop_filter_across_slices_enabled_flag */
    uint8_t pad[2];
} b200enc_hevc_slice_filter_t;
typedef struct {
    void *plane[3];                  /* Y, Cb, Cr: uint8 at 8 bits, uint16 at 10 */
    int stride[3];                   /* in samples */
    int width, height;               /* luma samples, multiples of 8 and of the min CB */
    int bit_depth_luma, bit_depth_chroma;  /* 8 or 10 (luma decides the sample type) */
    int log2_ctb, log2_min_cb;
    /* per 8x8 cell, edges_stride >= width/8 cells a row: bit 0 a block
     * boundary on its left edge, bit 1 on its top edge, bit 2 / bit 3 that
     * left / top edge is a transform block edge; cells at x >= width are
     * not read */
    const uint8_t *edges;
    int edges_stride;
    const b200enc_hevc_mvf_t *mvf;   /* per 4x4, min_pu_width a row; NULL: bS 2 on every edge */
    const uint8_t *cbf;              /* per 4x4 (luma residual present), or NULL */
    int min_pu_width;
    const int8_t *qp_y;              /* QpY per min coding block, width >> log2_min_cb a row */
    const uint8_t *no_filter;        /* per min coding block (lossless), or NULL */
    const int32_t *slice_of_ctb;     /* per CTB in raster order, or NULL (all slice 0) */
    const b200enc_hevc_slice_filter_t *slice_filter;  /* n_slice_filter entries; NULL filters nothing */
    int n_slice_filter;
    const int32_t *tile_of_ctb;      /* per CTB in raster order, or NULL (one tile) */
    int loop_filter_across_tiles;
    int cb_qp_offset, cr_qp_offset;  /* pps_cb/cr_qp_offset */
} b200enc_hevc_deblock_t;
/* The parameter block itself is host memory. Returns 0, or -1 for a
 * parameter out of range or a launch failure. */
int b200enc_hevc_deblock(const b200enc_hevc_deblock_t *p, void *stream);

/* Reads the error word a wavefront launch left in its scratch (synchronises
 * `stream`): 0 = fine, 1 = a bounded wait gave up (the frame's output is
 * incomplete and must not be used), -1 = the read failed. */
int b200enc_wavefront_status(const void *scratch, void *stream);

/* b200enc_p_frame with the 8x8 luma transform (High profile,
 * transform_size_8x8_flag): t8 = 0 is b200enc_p_frame, 1 codes the luma of
 * every macroblock as four 8x8 blocks instead of sixteen 4x4 ones, 2 chooses
 * per macroblock - the 8x8 transform when the residual's 8x8 Hadamard cost,
 * sum over the four 8x8 blocks of (sum |H8 R H8| + 2) >> 2, is below its 4x4
 * one, sum over the sixteen 4x4 blocks of (sum |H4 R H4|) >> 1. t8_flags
 * (device [mbs], may be NULL) gets each macroblock's choice, the input of
 * b200enc_deblock_tiles_t8 and b200enc_cavlc_t.t8_flags. Chroma unchanged. Levels: the four 8x8 luma blocks in raster order
 * at levels[mb][0..255] (block q at 64 q, raster within), chroma at
 * [256..383] as before; the nz word of 4x4 block 4q + i (spec order) holds
 * the nonzero mask of the 16 levels CAVLC codes as that block (8x8 scan
 * positions i, i + 4, ..., 7.3.5.3.2). No reference counterpart (the
 * reference's encoder codes 4x4 only); its decoder reconstructs the same
 * pictures from such levels. */
int b200enc_p_frame_t8(const uint8_t *cur_y, const uint8_t *cur_uv, int cur_pitch,
                       const uint8_t *ref_y, const uint8_t *ref_uv, int ref_pitch,
                       int W, int H, int RW, int RH, int qp, const void *mv,
                       int16_t *levels, int32_t *dc, uint32_t *nz, uint32_t *pred_mode,
                       uint8_t *rec_y, uint8_t *rec_uv, int rec_pitch, int t8, uint8_t *t8_flags,
                       void *stream);

/* H.264 High-profile 8x8 luma transform (transform_size_8x8_flag). No
 * counterpart in the reference's encoder, which codes 4x4 transforms only;
 * the decoder half is its decoder's h264d_idct8_add (src/h264_recon.c:191).
 * b200enc_h264_t8_forward: forward integer transform and quantisation (flat
 * scaling lists; intra rounding 1/3 or inter 1/6) of n residual blocks,
 * int16 [n][64] raster, into levels int16 [n][64]; nz[n] (may be NULL) gets
 * each block's nonzero mask (bit p = level p != 0). Both arrays 16-byte
 * aligned. b200enc_h264_t8_recon: scaling (clause 8.5.13.1, flat lists),
 * inverse transform (8.5.13.2) and the add with clipping onto the 8x8
 * prediction at plane + xy[i][1] * pitch + xy[i][0], replaced by the
 * reconstruction (blocks must not overlap). Device pointers; asynchronous on
 * `stream`; -1 for bad arguments. */
int b200enc_h264_t8_forward(const int16_t *residual, int16_t *levels, unsigned long long *nz, int n, int qp,
                            int intra, void *stream);
int b200enc_h264_t8_recon(const int16_t *levels, const int32_t *xy, uint8_t *plane, int pitch, int n, int qp,
                          void *stream);
/* b200enc_deblock_tiles with 8x8-transform macroblocks: t8[mb] nonzero marks
 * a macroblock coded with transform_size_8x8_flag (its odd internal luma
 * edges are not filtered, the coefficient test of a boundary strength looks
 * at its 8x8 blocks: src/h264_deblock.c:119-137, 294, 324); t8 device memory
 * [mbw * mbh] or NULL. */
int b200enc_deblock_tiles_t8(int mbw, int mbh, int qp, int is_intra, const uint32_t *nz, const uint8_t *t8,
                             const void *mv, const uint8_t *src_y, const uint8_t *src_uv, uint8_t *dst_y,
                             uint8_t *dst_uv, int pitch, uint32_t *status, void *stream);

/* CAVLC slice data on the GPU: every slice of one picture coded exactly as
 * the reference's host encoder codes it (its CAVLC macroblock loop,
 * src/encoder_h264.c:3128-3290: I16x16 macroblocks in I slices, P_Skip runs
 * and P_L0_16x16 macroblocks in P slices, residual blocks by src/cavlc.c),
 * from the picture's staged outputs already in device memory (levels, DC,
 * nz masks, prediction modes, vectors: the layouts of include/gpu_compute.h).
 * Each slice's output is its RBSP: the caller's slice header bits (up to 128,
 * MSB first, 16 bytes per slice in `header`; none when header_bits is NULL),
 * the slice data, then rbsp_trailing_bits - ready for emulation prevention
 * and a NAL header. quality_level is the host encoder's (its P_Skip rule
 * changes at >= 5). out_bytes[s] is 0xffffffff when slice s outgrew
 * slice_cap (or a macroblock outgrew 2560 bytes). Asynchronous on `stream`;
 * returns -1 for bad arguments. No reference counterpart as a GPU routine:
 * it takes the host's entropy loop (DEVLOG: 57 % of a 1440p frame) off the
 * host. */
typedef struct {
    int mbw, mbh, qp, is_intra, num_slices, quality_level;
    const int16_t *levels;       /* device [mbs][24][16] */
    const int32_t *dc;           /* device [mbs][24] raw DC terms */
    const uint32_t *nz;          /* device [mbs][24] */
    const uint32_t *pred_mode;   /* device [mbs] (I slices) */
    const void *mv;              /* device [mbs] gpu_mv_t */
    const uint8_t *header;       /* host [num_slices][16] or NULL */
    const int *header_bits;      /* host [num_slices] (0..128) or NULL */
    uint8_t *out;                /* device: slice s at out + s * slice_cap */
    size_t slice_cap;            /* bytes per slice, a multiple of 4 */
    uint32_t *out_bytes;         /* device [num_slices] */
    uint8_t *out_copy;           /* NULL: the bytes end in `out`; else the bytes go here (same layout; `out` is
                                    then work space), e.g. page-locked host memory mapped for the device, so
                                    only each slice's bytes cross the bus */
    void *scratch;               /* device, 256-byte aligned */
    size_t scratch_bytes;        /* >= b200enc_cavlc_scratch_bytes(mbw, mbh) */
    int transform8x8;            /* P slices of a picture parameter set with transform_8x8_mode_flag: every
                                    macroblock with coded luma carries transform_size_8x8_flag, and its luma uses
                                    the 8x8 transform (levels and nz words as b200enc_p_frame_t8 leaves them) */
    const uint8_t *t8_flags;     /* NULL, or device [mbs]: with transform8x8, the per-macroblock choice of
                                    b200enc_p_frame_t8 (t8 = 2); 0 marks a 4x4 macroblock */
} b200enc_cavlc_t;
size_t b200enc_cavlc_scratch_bytes(int mbw, int mbh);
int b200enc_cavlc_slices(const b200enc_cavlc_t *p, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* B200ENC_H */
