/*
 * hevc_link_stubs.c - TEST INFRASTRUCTURE ONLY. Entry points the reference's
 * HEVC encoder links against but never reaches on the paths tested here:
 * the libx265 fallback (libx265 is not installed) and the decoder's row
 * wait (hevc_wpp.c), which hevc_mc.c references for decoder-side motion
 * compensation. Linked into every build of the reference encoder in
 * oracle/_ref (the CPU build and the GPU-bound one).
 */
#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#include "encoder_x265.h"

hevc_x265_t *hevc_x265_create(void) { return NULL; }
int hevc_x265_encode(hevc_x265_t *x, const hevc_x265_config_t *cfg, const uint8_t *y, int y_stride,
                     const uint8_t *uv, int uv_stride, bool force_idr, int frame_qp, uint8_t *out,
                     size_t out_cap)
{
    (void)x; (void)cfg; (void)y; (void)y_stride; (void)uv; (void)uv_stride; (void)force_idr;
    (void)frame_qp; (void)out; (void)out_cap;
    return -1;
}
void hevc_x265_destroy(hevc_x265_t *x) { (void)x; }
void hevcd_await_rows(const void *g, int rows) { (void)g; (void)rows; }
