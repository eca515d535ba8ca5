/*
 * cpu_boundary.c - the gpu_compute_* boundary (include/gpu_compute.h)
 * implemented on the CPU with the oracle (oracle.c). TEST INFRASTRUCTURE
 * ONLY: linked with the reference's unchanged host encoder into
 * oracle/_ref/libh264enc_cpu.so so the encode -> decode round trip of the
 * reference pipeline can be checked on a machine without a GPU. "Device"
 * pointers are host pointers here.
 */
#include <stdlib.h>
#include <string.h>

#include "../include/gpu_compute.h"
#include "oracle.h"

typedef struct {
    int W, H, mbw, mbh, pitch;
    uint8_t *rec[2];
    int cur;
    int16_t *levels[2];
    int32_t *dc[2];
    uint32_t *pred_mode[2];
    orc_mv_t *mv[2];
    uint32_t *nz[2];
    int submitted;
} cpu_impl_t;

static cpu_impl_t *impl(const gpu_context_t *c) { return c ? (cpu_impl_t *)c->impl : NULL; }

int bc250_gpu_init(bc250_gpu_context_t *ctx)
{
    if (!ctx) return -1;
    memset(ctx, 0, sizeof(*ctx));
    ctx->impl = calloc(1, sizeof(cpu_impl_t));
    return ctx->impl ? 0 : -1;
}

static void free_bufs(cpu_impl_t *m)
{
    for (int i = 0; i < 2; i++) {
        free(m->rec[i]); free(m->levels[i]); free(m->dc[i]); free(m->pred_mode[i]); free(m->mv[i]); free(m->nz[i]);
        m->rec[i] = NULL; m->levels[i] = NULL; m->dc[i] = NULL; m->pred_mode[i] = NULL; m->mv[i] = NULL; m->nz[i] = NULL;
    }
}

void bc250_gpu_destroy(bc250_gpu_context_t *ctx)
{
    cpu_impl_t *m = impl(ctx);
    if (!m) return;
    free_bufs(m);
    free(m);
    ctx->impl = NULL;
}

int gpu_compute_create_image(gpu_context_t *ctx, int w, int h, int format, gpu_image_t *img, gpu_memory_t *mem)
{
    (void)ctx;
    int pitch = (w + 15) / 16 * 16, rows = (h + 15) / 16 * 16;
    size_t bytes = (size_t)pitch * rows * 3 / 2;
    uint8_t *p = calloc(1, bytes);
    if (!p) return -1;
    memset(img, 0, sizeof(*img));
    img->y_plane = img->y_view = p;
    img->uv_plane = img->uv_view = p + (size_t)pitch * rows;
    img->width = (uint32_t)w; img->height = (uint32_t)h; img->format = format; img->pitch = (uint32_t)pitch;
    mem->memory = p; mem->size = bytes; mem->mapped_ptr = NULL;
    return 0;
}

void gpu_compute_destroy_image(gpu_context_t *ctx, gpu_image_t image, gpu_memory_t memory)
{
    (void)ctx; (void)image;
    free(memory.memory);
}

int gpu_compute_upload_nv12(gpu_context_t *ctx, gpu_image_t *img, gpu_memory_t mem, const uint8_t *y, int yp,
                            const uint8_t *uv, int uvp, int w, int h)
{
    (void)ctx; (void)mem;
    for (int r = 0; r < h; r++) memcpy((uint8_t *)img->y_plane + (size_t)r * img->pitch, y + (size_t)r * yp, (size_t)w);
    for (int r = 0; r < h / 2; r++)
        memcpy((uint8_t *)img->uv_plane + (size_t)r * img->pitch, uv + (size_t)r * uvp, (size_t)w);
    return 0;
}

int gpu_compute_begin_picture(gpu_context_t *ctx, gpu_image_t rt) { (void)rt; return impl(ctx) ? 0 : -1; }

int gpu_compute_dispatch_encode_ext(gpu_context_t *ctx, gpu_image_t rt, int w, int h, int qp, int is_intra,
                                    int num_slices, int me_mode, const gpu_mv_t *cpu_mvs)
{
    cpu_impl_t *m = impl(ctx);
    if (!m) return -1;
    if (m->W != w || m->H != h) {
        free_bufs(m);
        m->W = w; m->H = h; m->mbw = (w + 15) / 16; m->mbh = (h + 15) / 16; m->pitch = m->mbw * 16;
        size_t mbs = (size_t)m->mbw * m->mbh;
        for (int i = 0; i < 2; i++) {
            m->rec[i] = calloc((size_t)m->pitch * m->mbh * 24, 1);
            m->levels[i] = calloc(mbs * 384, 2); m->dc[i] = calloc(mbs * 24, 4); m->pred_mode[i] = calloc(mbs, 4);
            m->mv[i] = calloc(mbs, 16); m->nz[i] = calloc(mbs * 24, 4);
        }
        m->cur = 0;
        ctx->has_recon_frame = false;
    }
    const int slot = ctx->current_buf;
    const size_t luma = (size_t)m->pitch * m->mbh * 16;
    orc_frame_t f = {w, h, m->mbw * 16, m->mbh * 16, m->mbw, m->mbh, qp, num_slices < 1 ? 1 : num_slices,
                     ORC_INTRA_CORNER_CHECK};
    orc_me_params_t p = {16, me_mode == 1 ? 8 : 5, 512};
    orc_out_t o = {m->levels[slot], m->dc[slot], m->nz[slot], m->pred_mode[slot], m->mv[slot]};
    const uint8_t *ref = ctx->has_recon_frame ? m->rec[m->cur] : (const uint8_t *)rt.y_plane;
    const int rp = ctx->has_recon_frame ? m->pitch : (int)rt.pitch;
    uint8_t *out = m->rec[m->cur ^ 1];
    /* a reference taken from the input surface has its own uv offset */
    const uint8_t *ref_uv = ctx->has_recon_frame ? ref + luma : (const uint8_t *)rt.uv_plane;
    if (cpu_mvs && !is_intra) {
        memcpy(o.mv, cpu_mvs, (size_t)m->mbw * m->mbh * 16);
        orc_p_frame(&f, rt.y_plane, rt.uv_plane, (int)rt.pitch, ref, ref_uv, rp, o.mv, &o, out, out + luma, m->pitch);
        orc_deblock_frame(m->mbw, m->mbh, qp, 0, o.nz, o.mv, out, out + luma, m->pitch);
    } else {
        orc_encode_frame(&f, &p, is_intra, 1, rt.y_plane, rt.uv_plane, (int)rt.pitch, ref, ref_uv, rp, &o, out,
                         out + luma, m->pitch);
    }
    m->cur ^= 1;
    ctx->has_recon_frame = true;
    ctx->recon_image.y_plane = ctx->recon_image.y_view = m->rec[m->cur];
    ctx->recon_image.uv_plane = ctx->recon_image.uv_view = m->rec[m->cur] + luma;
    ctx->recon_image.pitch = (uint32_t)m->pitch;
    ctx->recon_image.width = (uint32_t)w; ctx->recon_image.height = (uint32_t)h;
    ctx->recon_memory.memory = m->rec[m->cur];
    ctx->recon_memory.size = luma * 3 / 2;
    ctx->frame_width = (uint32_t)w; ctx->frame_height = (uint32_t)h;
    return 0;
}

int gpu_compute_end_picture(gpu_context_t *ctx)
{
    cpu_impl_t *m = impl(ctx);
    if (!m) return -1;
    m->submitted = ctx->current_buf;
    ctx->current_buf ^= 1;
    ctx->frames_submitted++;
    return 0;
}

int gpu_compute_submitted_slot(gpu_context_t *ctx) { cpu_impl_t *m = impl(ctx); return m ? m->submitted : 0; }
int gpu_compute_sync_slot(gpu_context_t *ctx, int slot) { (void)slot; return impl(ctx) ? 0 : -1; }

#define CPU_GETTER(fn, field, per_mb) \
    int fn(gpu_context_t *ctx, int slot, void **d, size_t *n) \
    { cpu_impl_t *m = impl(ctx); if (!m || slot < 0 || slot > 1) return -1; \
      *d = m->field[slot]; *n = (size_t)m->mbw * m->mbh * (per_mb); return 0; }
CPU_GETTER(gpu_compute_get_quant_staging_data_slot, levels, 768)
CPU_GETTER(gpu_compute_get_dc_staging_data_slot, dc, 96)
CPU_GETTER(gpu_compute_get_pred_mode_staging_data_slot, pred_mode, 4)
CPU_GETTER(gpu_compute_get_mv_staging_data_slot, mv, 16)
CPU_GETTER(gpu_compute_get_nz_staging_data_slot, nz, 96)

double gpu_compute_get_last_latency_ms(const gpu_context_t *ctx) { (void)ctx; return 0.0; }
int gpu_compute_cpu_read_safe(gpu_context_t *ctx) { (void)ctx; return 1; }
uint8_t *gpu_compute_map_surface(gpu_context_t *ctx, gpu_image_t *img, gpu_memory_t mem, gpu_nv12_layout_t *l, bool *u)
{
    (void)ctx;
    if (l) {
        l->y_pitch = img->pitch; l->y_offset = 0; l->uv_pitch = img->pitch;
        l->uv_offset = (uint64_t)((uint8_t *)img->uv_plane - (uint8_t *)img->y_plane); l->total_size = mem.size;
    }
    if (u) *u = false;
    return (uint8_t *)img->y_plane;
}
void gpu_compute_unmap_surface(gpu_context_t *ctx, gpu_memory_t mem, bool u) { (void)ctx; (void)mem; (void)u; }
int gpu_compute_wait_for_image_ready_host(gpu_context_t *ctx, gpu_memory_t mem) { (void)ctx; (void)mem; return 0; }
void gpu_compute_copy_from_wc(void *d, const void *s, size_t n) { memcpy(d, s, n); }
void gpu_compute_debug_dump_recon(gpu_context_t *ctx, int w, int h) { (void)ctx; (void)w; (void)h; }
FILE *bc250_debug_dump_open(const char *name, const char *what) { (void)name; (void)what; return NULL; }

/* The reconstruction the boundary keeps as the next reference (coded size). */
int cpu_boundary_recon(gpu_context_t *ctx, void **y, void **uv, int *pitch)
{
    cpu_impl_t *m = impl(ctx);
    if (!m || !m->rec[0]) return -1;
    *y = m->rec[m->cur];
    *uv = m->rec[m->cur] + (size_t)m->pitch * m->mbh * 16;
    *pitch = m->pitch;
    return 0;
}
