/*
 * hevc_hpel_binding.c - binds the reference HEVC encoder's half-sample
 * planes to the GPU.
 *
 * The reference's host HEVC encoder (approach1-compute-encoder/src/
 * encoder_h265.c) builds the motion search's four sample planes of the
 * previous reconstruction once per P picture (build_hpel_8 / build_hpel_10,
 * hevc_enc_template.c:390-397, called from encode_core at encoder_h265.c
 * :1570-1572) in two passes over its worker pool. A maintainer compiles this
 * file instead of encoder_h265.c: it includes that file unchanged and routes
 * its worker_pool_for calls through b200_pool_for, which hands the first
 * pass of a plane build to b200enc_hevc_build_hpel_host (all four planes,
 * bit-identical to the reference's) and skips the second; every other
 * worker_pool_for call of the encoder goes to the reference's pool as
 * before. The encoder's bitstream is therefore byte for byte the reference's.
 *
 * There is no host fallback: if the GPU call fails, the failure is reported
 * on stderr and counted (b200_hevc_hpel_stats), and that picture's planes
 * keep their previous contents, so its motion search is worse but the
 * stream stays decodable (the encoder reconstructs from its own
 * predictions).
 *
 * The encoder's two reconstruction buffers (they swap every picture) and
 * its four plane buffers are page-locked at its first GPU picture
 * (b200enc_pin_host), so the uploads and read-backs run as DMA straight
 * from and into them; hevc_encoder_destroy, wrapped here, unlocks them
 * before the reference's destroy frees them.
 */
#include <pthread.h>
#include <stdio.h>

#include "worker_pool.h"

static void b200_pool_for(worker_pool_t *p, int count, int chunk, void (*fn)(void *arg, int begin, int end),
                          void *arg, int n);
#define worker_pool_for b200_pool_for
#define hevc_encoder_destroy b200_ref_hevc_encoder_destroy
#include "encoder_h265.c"
#undef hevc_encoder_destroy
#undef worker_pool_for

#include "b200enc.h"

static long g_gpu_pictures, g_failed_pictures;

/* Encoders whose buffers are page-locked, and which of them. */
#define B200_MAX_PINNED_ENCODERS 64
static struct {
    const hevc_encoder_t *enc;
    void *ptr[6];
    int n;
} g_pinned[B200_MAX_PINNED_ENCODERS];
static pthread_mutex_t g_pinned_lock = PTHREAD_MUTEX_INITIALIZER;

static void b200_pin_encoder(hevc_encoder_t *enc, int ten)
{
    pthread_mutex_lock(&g_pinned_lock);
    int free_slot = -1;
    for (int i = 0; i < B200_MAX_PINNED_ENCODERS; i++) {
        if (g_pinned[i].enc == enc) {
            pthread_mutex_unlock(&g_pinned_lock);
            return;
        }
        if (!g_pinned[i].enc && free_slot < 0) free_slot = i;
    }
    if (free_slot >= 0) {
        const size_t bps = ten ? 2 : 1;
        const size_t luma = (size_t)enc->coded_width * enc->coded_height * bps;
        const size_t plane = (size_t)enc->hpel_stride * (enc->coded_height + 2 * HPEL_MARGIN) * bps;
        void *const bufs[6] = { enc->recon_y, enc->prev_recon_y, enc->hpel[0], enc->hpel[1], enc->hpel[2],
                                enc->hpel[3] };
        const size_t sizes[6] = { luma, luma, plane, plane, plane, plane };
        g_pinned[free_slot].enc = enc;
        g_pinned[free_slot].n = 0;
        for (int i = 0; i < 6; i++)
            if (b200enc_pin_host(bufs[i], sizes[i]) == 0) g_pinned[free_slot].ptr[g_pinned[free_slot].n++] = bufs[i];
    }
    pthread_mutex_unlock(&g_pinned_lock);
}

void hevc_encoder_destroy(hevc_encoder_t *encoder)
{
    if (encoder) {
        pthread_mutex_lock(&g_pinned_lock);
        for (int i = 0; i < B200_MAX_PINNED_ENCODERS; i++)
            if (g_pinned[i].enc == encoder) {
                for (int k = 0; k < g_pinned[i].n; k++) b200enc_unpin_host(g_pinned[i].ptr[k]);
                g_pinned[i].enc = NULL;
                g_pinned[i].n = 0;
            }
        pthread_mutex_unlock(&g_pinned_lock);
    }
    b200_ref_hevc_encoder_destroy(encoder);
}

void b200_hevc_hpel_stats(long *gpu_pictures, long *failed_pictures)
{
    if (gpu_pictures) *gpu_pictures = g_gpu_pictures;
    if (failed_pictures) *failed_pictures = g_failed_pictures;
}

static void b200_pool_for(worker_pool_t *p, int count, int chunk, void (*fn)(void *arg, int begin, int end),
                          void *arg, int n)
{
    if (fn == hpel_rows_8 || fn == hpel_rows_10) {
        const int ten = fn == hpel_rows_10;
        hevc_encoder_t *enc = ten ? ((const hpel_job_t_10 *)arg)->enc : ((const hpel_job_t_8 *)arg)->enc;
        const int pass = ten ? ((const hpel_job_t_10 *)arg)->pass : ((const hpel_job_t_8 *)arg)->pass;
        if (pass == 1) {
            b200_pin_encoder(enc, ten);
            void *const planes[4] = { enc->hpel[0], enc->hpel[1], enc->hpel[2], enc->hpel[3] };
            if (b200enc_hevc_build_hpel_host(enc->prev_recon_y, (int)enc->coded_width, (int)enc->coded_height,
                                             ten ? 10 : 8, HPEL_MARGIN, planes, enc->hpel_stride) == 0) {
                __atomic_add_fetch(&g_gpu_pictures, 1, __ATOMIC_RELAXED);
            } else {
                __atomic_add_fetch(&g_failed_pictures, 1, __ATOMIC_RELAXED);
                fprintf(stderr, "[b200enc] b200enc_hevc_build_hpel_host failed: this picture's search planes are stale\n");
            }
        }
        return;  /* pass 2: the GPU built all four planes in pass 1 */
    }
    worker_pool_for(p, count, chunk, fn, arg, n);
}
