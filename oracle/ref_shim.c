/*
 * ref_shim.c - thin C wrappers around the reference's OWN C functions,
 * compiled together with the reference sources (in place, read-only) into
 * oracle/_ref/libh264ref.so by oracle/Makefile. TEST INFRASTRUCTURE ONLY:
 * it exists so the tests can pin the CPU restatement (oracle.c) against the
 * reference's code, and so bench.py can time the reference's C/AVX2 SAD as
 * the CPU baseline. Nothing here is part of the product library.
 *
 * Wrapped reference entry points:
 *   h264d_deblock_picture  A1/src/h264_deblock.c:349 (also with 8x8-transform macroblocks)
 *   h264d_mc_fetch_luma / h264d_mc_luma    A1/src/h264_mc.c:278
 *   h264d_mc_fetch_chroma / h264d_mc_chroma A1/src/h264_mc.c:344
 *   h264d_dequant_build / h264d_idct4_add   A1/src/h264_recon.c:113
 *   h264d_idct8_add         A1/src/h264_recon.c:191
 *   cpu_simd_sad_16x16     A1/src/cpu_simd_me.c:136
 *   cpu_simd_me_search_frame A1/src/cpu_simd_me.c:275
 *   h264_intra16_luma_dc_transform A1/src/encoder_h264.c:775
 */
#include <stdlib.h>
#include <string.h>

#include "cpu_simd_me.h"
#include "decoder_h264.h"
#include "encoder_h264.h"
#include "h264_deblock.h"
#include "h264_mc.h"
#include "h264_recon.h"

#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    int32_t mvx, mvy;
    uint32_t sad, pad;
} shim_mv_t;

/* Deblock an NV12 picture through the reference decoder's filter, with the
 * macroblock description this encoder emits (all I16x16 or all P16x16 with
 * one reference picture, uniform QP, idc 0, zero offsets). */
/* The same with the 8x8 transform in the macroblocks whose t8 byte is set
 * (NULL: none), as the decoder's transform_size_8x8_flag. */
int refshim_deblock_nv12_t8(int mbw, int mbh, int qp, int is_intra,
                            const uint32_t *nz, const uint8_t *t8, const shim_mv_t *mv,
                            uint8_t *y, uint8_t *uv, int pitch)
{
    const int n = mbw * mbh, cw = mbw * 8, ch = mbh * 8;
    h264d_mb_t *mbs = calloc((size_t)n, sizeof(*mbs));
    uint8_t *sl = calloc((size_t)n, 1);
    uint8_t *cb = malloc((size_t)cw * ch), *cr = malloc((size_t)cw * ch);
    if (!mbs || !sl || !cb || !cr) { free(mbs); free(sl); free(cb); free(cr); return -1; }
    for (int i = 0; i < n; i++) {
        h264d_mb_t *m = &mbs[i];
        m->type = is_intra ? H264D_MB_I_16x16 : H264D_MB_P_16x16;
        m->intra = (uint8_t)(is_intra ? 1 : 0);
        m->qpy = (int8_t)qp;
        m->transform8x8 = (uint8_t)(t8 && t8[i] ? 1 : 0);
        for (int p = 0; p < 4; p++) {
            m->ref[0][p] = is_intra ? -1 : 0;
            m->ref[1][p] = -1;
            m->ref_idx[0][p] = is_intra ? -1 : 0;
            m->ref_idx[1][p] = -1;
        }
        for (int b = 0; b < 16; b++) {
            m->mv[0][b][0] = (int16_t)(is_intra ? 0 : mv[i].mvx);
            m->mv[0][b][1] = (int16_t)(is_intra ? 0 : mv[i].mvy);
            m->nnz[0][b] = (uint8_t)__builtin_popcount(nz[(size_t)i * 24 + b] & 0xffffu);
        }
    }
    for (int r = 0; r < ch; r++)
        for (int c = 0; c < cw; c++) {
            cb[r * cw + c] = uv[(size_t)r * pitch + 2 * c];
            cr[r * cw + c] = uv[(size_t)r * pitch + 2 * c + 1];
        }
    h264d_deblock_params_t prm = {0, 0, 0};
    h264d_deblock_picture(y, pitch, cb, cr, cw, mbw, mbh, mbs, sl, &prm, 0, 0);
    for (int r = 0; r < ch; r++)
        for (int c = 0; c < cw; c++) {
            uv[(size_t)r * pitch + 2 * c] = cb[r * cw + c];
            uv[(size_t)r * pitch + 2 * c + 1] = cr[r * cw + c];
        }
    free(mbs); free(sl); free(cb); free(cr);
    return 0;
}

int refshim_deblock_nv12(int mbw, int mbh, int qp, int is_intra,
                         const uint32_t *nz, const shim_mv_t *mv,
                         uint8_t *y, uint8_t *uv, int pitch)
{
    return refshim_deblock_nv12_t8(mbw, mbh, qp, is_intra, nz, NULL, mv, y, uv, pitch);
}

/* A w x h luma prediction at quarter-pel position (qx, qy) of the top-left
 * sample, through the reference decoder's MC (edge replication at the plane
 * size). */
void refshim_mc_luma(const uint8_t *plane, int pitch, int pw, int ph,
                     int qx, int qy, int w, int h, uint8_t *dst, int dst_stride)
{
    uint8_t tmp[(64 + 6) * (64 + 6)];
    int s = 0;
    const uint8_t *src = h264d_mc_fetch_luma(tmp, &s, plane, pitch, pw, ph, qx >> 2, qy >> 2, w, h);
    h264d_mc_luma(dst, dst_stride, src, s, w, h, qx & 3, qy & 3);
}

/* Same for one chroma plane of an NV12 picture, eighth-pel (ex, ey). */
void refshim_mc_chroma_nv12(const uint8_t *uv, int pitch, int cw, int chh, int plane,
                            int ex, int ey, int w, int h, uint8_t *dst, int dst_stride)
{
    uint8_t *sep = malloc((size_t)cw * chh);
    uint8_t tmp[(64 + 1) * (64 + 1)];
    int s = 0;
    if (!sep) return;
    for (int r = 0; r < chh; r++)
        for (int c = 0; c < cw; c++) sep[r * cw + c] = uv[(size_t)r * pitch + 2 * c + plane];
    const uint8_t *src = h264d_mc_fetch_chroma(tmp, &s, sep, cw, cw, chh, ex >> 3, ey >> 3, w, h);
    h264d_mc_chroma(dst, dst_stride, src, s, w, h, ex & 7, ey & 7);
    free(sep);
}

/* Scaling (flat lists) + inverse transform + add, reference decoder. */
void refshim_idct4_add(uint8_t *dst, int stride, int16_t block[16], int qp, int dc_ready)
{
    static uint8_t flat4[6][16], flat8[6][64];
    static int init;
    if (!init) { memset(flat4, 16, sizeof(flat4)); memset(flat8, 16, sizeof(flat8)); init = 1; }
    h264d_dequant_t dq;
    memset(&dq, 0, sizeof(dq));
    h264d_dequant_build(&dq, qp, flat4, flat8);
    h264d_idct4_add(dst, stride, block, dq.d4[0], qp, dc_ready != 0);
}

/* 8x8: the reference decoder's scaling (flat lists) and inverse transform,
 * added to dst (h264d_idct8_add, A1/src/h264_recon.c:191). */
void refshim_idct8_add(uint8_t *dst, int stride, int16_t block[64], int qp)
{
    static uint8_t flat4[6][16], flat8[6][64];
    static int init;
    if (!init) { memset(flat4, 16, sizeof(flat4)); memset(flat8, 16, sizeof(flat8)); init = 1; }
    h264d_dequant_t dq;
    memset(&dq, 0, sizeof(dq));
    h264d_dequant_build(&dq, qp, flat4, flat8);
    h264d_idct8_add(dst, stride, block, dq.d8[0], qp);
}

uint32_t refshim_sad16(const uint8_t *a, int pa, const uint8_t *b, int pb)
{
    return cpu_simd_sad_16x16(a, pa, b, pb);
}

int refshim_cpu_me(const uint8_t *src, int sp, const uint8_t *ref, int rp, int w, int h,
                   int radius, int threads, shim_mv_t *out)
{
    cpu_simd_me_config_t cfg;
    cpu_simd_me_config_init(&cfg, (uint32_t)w, (uint32_t)h);
    cfg.search_radius = (uint32_t)radius;
    cfg.num_threads = threads;
    return cpu_simd_me_search_frame(src, sp, ref, rp, (uint32_t)w, (uint32_t)h, (gpu_mv_t *)out, &cfg);
}

void refshim_intra16_luma_dc(const int dc_in[16], int qp, int dc_out[16], int pre[16])
{
    int m[4][4];
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++) m[r][c] = dc_in[r * 4 + c];
    h264_intra16_luma_dc_transform(m, qp, dc_out, pre);
}

/*
 * The plain full-search integer stage at the reference's own SAD speed:
 * every candidate of [-R,R]^2 scored by the reference's AVX2
 * cpu_simd_sad_16x16, cost SAD + lambda*(|dx|+|dy|), raster tie-break, on a
 * reference plane padded by edge replication (which is the clamp). Used as
 * the timed CPU baseline of the ME stage and, since it reaches the same
 * decision by independent code, as a cross-check of oracle.c's search.
 * mb rows [row0, row1) only, so a bounded sample can be timed.
 */
int refshim_full_search_int(const uint8_t *cur, int cp, int W, int H,
                            const uint8_t *ref, int rp, int RW, int RH,
                            int mbw, int row0, int row1, int R, int lambda, int threads,
                            int32_t *out_dx, int32_t *out_dy, uint32_t *out_sad)
{
    const int pad = R + 16 + 4;
    const int PW = RW + 2 * pad, PH = RH + 2 * pad;
    uint8_t *pr = malloc((size_t)PW * PH);
    if (!pr) return -1;
    for (int y = 0; y < PH; y++) {
        int sy = y - pad; sy = sy < 0 ? 0 : (sy >= RH ? RH - 1 : sy);
        for (int x = 0; x < PW; x++) {
            int sx = x - pad; sx = sx < 0 ? 0 : (sx >= RW ? RW - 1 : sx);
            pr[(size_t)y * PW + x] = ref[(size_t)sy * rp + sx];
        }
    }
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 1) collapse(2)
#endif
    for (int mby = row0; mby < row1; mby++)
        for (int mbx = 0; mbx < mbw; mbx++) {
            uint8_t cb[256];
            for (int y = 0; y < 16; y++)
                for (int x = 0; x < 16; x++) {
                    int sy = mby * 16 + y, sx = mbx * 16 + x;
                    sy = sy >= H ? H - 1 : sy; sx = sx >= W ? W - 1 : sx;
                    cb[y * 16 + x] = cur[(size_t)sy * cp + sx];
                }
            uint32_t best_key = 0xffffffffu, best_sad = 0;
            const int side = 2 * R + 1;
            for (int dy = -R; dy <= R; dy++)
                for (int dx = -R; dx <= R; dx++) {
                    const uint8_t *p = pr + (size_t)(pad + mby * 16 + dy) * PW + pad + mbx * 16 + dx;
                    uint32_t s = cpu_simd_sad_16x16(cb, 16, p, PW);
                    uint32_t cost = s + (uint32_t)lambda * (uint32_t)(abs(dx) + abs(dy));
                    uint32_t key = (cost << 14) | (uint32_t)((dy + R) * side + dx + R);
                    if (key < best_key) { best_key = key; best_sad = s; }
                }
            int idx = (int)(best_key & 0x3fff), mb = mby * mbw + mbx;
            out_dx[mb] = idx % side - R;
            out_dy[mb] = idx / side - R;
            out_sad[mb] = best_sad;
        }
    free(pr);
    return 0;
}

/* The GPU entry points encoder_h264.c imports, stubbed "no GPU" so the
 * reference host encoder links into this test library; every one reports
 * failure, which sends the reference down its GPU-free paths. */
int gpu_compute_begin_picture(gpu_context_t *c, gpu_image_t i) { (void)c; (void)i; return -1; }
int gpu_compute_dispatch_encode_ext(gpu_context_t *c, gpu_image_t i, int w, int h, int qp, int intra, int ns,
                                    int mode, const gpu_mv_t *m)
{ (void)c; (void)i; (void)w; (void)h; (void)qp; (void)intra; (void)ns; (void)mode; (void)m; return -1; }
int gpu_compute_end_picture(gpu_context_t *c) { (void)c; return -1; }
int gpu_compute_submitted_slot(gpu_context_t *c) { (void)c; return 0; }
int gpu_compute_sync_slot(gpu_context_t *c, int s) { (void)c; (void)s; return -1; }
#define SHIM_GETTER(name) \
    int name(gpu_context_t *c, int s, void **d, size_t *n) { (void)c; (void)s; *d = NULL; *n = 0; return -1; }
SHIM_GETTER(gpu_compute_get_quant_staging_data_slot)
SHIM_GETTER(gpu_compute_get_dc_staging_data_slot)
SHIM_GETTER(gpu_compute_get_pred_mode_staging_data_slot)
SHIM_GETTER(gpu_compute_get_mv_staging_data_slot)
SHIM_GETTER(gpu_compute_get_nz_staging_data_slot)
double gpu_compute_get_last_latency_ms(const gpu_context_t *c) { (void)c; return 0.0; }
int gpu_compute_cpu_read_safe(gpu_context_t *c) { (void)c; return 1; }
uint8_t *gpu_compute_map_surface(gpu_context_t *c, gpu_image_t *i, gpu_memory_t m, gpu_nv12_layout_t *l, bool *u)
{ (void)c; (void)i; (void)m; (void)l; if (u) *u = false; return NULL; }
void gpu_compute_unmap_surface(gpu_context_t *c, gpu_memory_t m, bool u) { (void)c; (void)m; (void)u; }
int gpu_compute_wait_for_image_ready_host(gpu_context_t *c, gpu_memory_t m) { (void)c; (void)m; return 0; }
void gpu_compute_copy_from_wc(void *d, const void *s, size_t n) { memcpy(d, s, n); }
void gpu_compute_debug_dump_recon(gpu_context_t *c, int w, int h) { (void)c; (void)w; (void)h; }
FILE *bc250_debug_dump_open(const char *name, const char *what) { (void)name; (void)what; return NULL; }
int gpu_compute_upload_nv12(gpu_context_t *c, gpu_image_t *i, gpu_memory_t m, const uint8_t *y, int yp,
                            const uint8_t *uv, int uvp, int w, int h)
{ (void)c; (void)i; (void)m; (void)y; (void)yp; (void)uv; (void)uvp; (void)w; (void)h; return -1; }
