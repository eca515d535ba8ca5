/*
 * hevc_shim.c - TEST INFRASTRUCTURE ONLY. Compiles the reference's HEVC
 * host encoder where it lies (approach1-compute-encoder/src/encoder_h265.c,
 * included, with its hevc_enc_template.c) so the tests can call the static
 * primitive the B200 kernels replace, and stubs the two gpu_compute_* entry
 * points the encoder imports but these tests never reach (hevc_link_stubs.c
 * has the rest). The public transform/quant functions come from the
 * reference's hevc_intra.c, linked in as is.
 */
#include "encoder_h265.c"

int gpu_compute_download_nv12(gpu_context_t *ctx, gpu_image_t *image, gpu_memory_t memory, uint8_t *y_plane,
                              int y_pitch, uint8_t *uv_plane, int uv_pitch, int width, int height)
{
    (void)ctx; (void)image; (void)memory; (void)y_plane; (void)y_pitch; (void)uv_plane; (void)uv_pitch;
    (void)width; (void)height;
    return -1;
}
FILE *bc250_debug_dump_open(const char *name, const char *what) { (void)name; (void)what; return NULL; }

/* build_hpel (hevc_enc_template.c:390) of the 8-bit encoder on a w x h
 * reconstruction (pitch w): the whole-sample plane and the three half-sample
 * planes, (h + 2*16) rows x (w + 2*16) columns each, into planes[4] with
 * that width as pitch. Returns the margin. */
int refshim_hevc_build_hpel(const uint8_t *recon, int w, int h, uint8_t *planes[4])
{
    struct hevc_encoder enc;
    memset(&enc, 0, sizeof(enc));
    enc.coded_width = (uint32_t)w;
    enc.coded_height = (uint32_t)h;
    enc.bit_depth = 8;
    enc.prev_recon_y = (void *)recon;
    enc.hpel_stride = w + 2 * HPEL_MARGIN;
    for (int i = 0; i < 4; i++) enc.hpel[i] = planes[i];
    enc.hpel_tmp = malloc((size_t)enc.hpel_stride * (h + 2 * HPEL_MARGIN + 7) * sizeof(int32_t));
    if (!enc.hpel_tmp) return -1;
    enc.pool = NULL;
    enc.threads = 1;
    build_hpel_8(&enc);
    free(enc.hpel_tmp);
    return HPEL_MARGIN;
}

/* motion_search (hevc_enc_template.c:958) of the 8-bit encoder for one 8x8
 * CU: the search planes as build_hpel leaves them (pitch w + 2*16), the
 * source picture (pitch w), quarter-sample refinement on or off. Writes the
 * vector, the predictor index, the cost (q8) and the SAD. */
void refshim_hevc_motion_search(uint8_t *planes[4], const uint8_t *src, int w, int h, int qpel, int cu_x, int cu_y,
                                const int16_t mvp[4], const int16_t *starts, int n_starts, int lambda_q8,
                                int16_t mv_out[2], int *mvp_idx, int64_t *cost_q8, uint32_t *sad)
{
    struct hevc_encoder enc;
    memset(&enc, 0, sizeof(enc));
    enc.coded_width = (uint32_t)w;
    enc.coded_height = (uint32_t)h;
    enc.bit_depth = 8;
    enc.hpel_stride = w + 2 * HPEL_MARGIN;
    for (int i = 0; i < 4; i++) enc.hpel[i] = planes[i];
    enc.src_y = (void *)src;
    enc.qpel = qpel != 0;
    hevc_mv_t p[2] = {{mvp[0], mvp[1]}, {mvp[2], mvp[3]}};
    hevc_mv_t st[16];
    for (int i = 0; i < n_starts && i < 16; i++) {
        st[i].x = starts[2 * i];
        st[i].y = starts[2 * i + 1];
    }
    hevc_mv_t m = motion_search_8(&enc, cu_x, cu_y, p, st, n_starts, lambda_q8, mvp_idx, cost_q8, sad);
    mv_out[0] = m.x;
    mv_out[1] = m.y;
}

/* build_hpel_10, the 10-bit (Main10) instance of the same template
 * (encoder_h265.c:1220-1227): 16-bit samples, pitches in samples. */
int refshim_hevc_build_hpel_10(const uint16_t *recon, int w, int h, uint16_t *planes[4])
{
    struct hevc_encoder enc;
    memset(&enc, 0, sizeof(enc));
    enc.coded_width = (uint32_t)w;
    enc.coded_height = (uint32_t)h;
    enc.bit_depth = 10;
    enc.prev_recon_y = (void *)recon;
    enc.hpel_stride = w + 2 * HPEL_MARGIN;
    for (int i = 0; i < 4; i++) enc.hpel[i] = planes[i];
    enc.hpel_tmp = malloc((size_t)enc.hpel_stride * (h + 2 * HPEL_MARGIN + 7) * sizeof(int32_t));
    if (!enc.hpel_tmp) return -1;
    enc.pool = NULL;
    enc.threads = 1;
    build_hpel_10(&enc);
    free(enc.hpel_tmp);
    return HPEL_MARGIN;
}

/* motion_search_10 for one 8x8 CU on 10-bit planes and source. */
void refshim_hevc_motion_search_10(uint16_t *planes[4], const uint16_t *src, int w, int h, int qpel, int cu_x,
                                   int cu_y, const int16_t mvp[4], const int16_t *starts, int n_starts,
                                   int lambda_q8, int16_t mv_out[2], int *mvp_idx, int64_t *cost_q8, uint32_t *sad)
{
    struct hevc_encoder enc;
    memset(&enc, 0, sizeof(enc));
    enc.coded_width = (uint32_t)w;
    enc.coded_height = (uint32_t)h;
    enc.bit_depth = 10;
    enc.hpel_stride = w + 2 * HPEL_MARGIN;
    for (int i = 0; i < 4; i++) enc.hpel[i] = planes[i];
    enc.src_y = (void *)src;
    enc.qpel = qpel != 0;
    hevc_mv_t p[2] = {{mvp[0], mvp[1]}, {mvp[2], mvp[3]}};
    hevc_mv_t st[16];
    for (int i = 0; i < n_starts && i < 16; i++) {
        st[i].x = starts[2 * i];
        st[i].y = starts[2 * i + 1];
    }
    hevc_mv_t m = motion_search_10(&enc, cu_x, cu_y, p, st, n_starts, lambda_q8, mvp_idx, cost_q8, sad);
    mv_out[0] = m.x;
    mv_out[1] = m.y;
}
