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
 */
#include <stdio.h>

#include "worker_pool.h"

static void b200_pool_for(worker_pool_t *p, int count, int chunk, void (*fn)(void *arg, int begin, int end),
                          void *arg, int n);
#define worker_pool_for b200_pool_for
#include "encoder_h265.c"
#undef worker_pool_for

#include "b200enc.h"

static long g_gpu_pictures, g_failed_pictures;

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
