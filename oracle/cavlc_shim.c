/*
 * cavlc_shim.c - the reference's CAVLC slice data writer on the CPU, for the
 * GPU entropy coder's parity tests. TEST INFRASTRUCTURE ONLY: compiled with
 * the reference sources (read in place) into oracle/_ref/libcavlcref.so by
 * oracle/Makefile; nothing here is part of the product library.
 *
 * The reference's host encoder writes a slice's macroblock layer inline in
 * h264_encoder_encode_frame (A1/src/encoder_h264.c:3128-3290): I slices code
 * every macroblock with encode_mb_i16x16 (:1120), P slices decide P_Skip per
 * macroblock (zero luma levels, zero chroma DC Hadamard and AC levels, the
 * vector equal to the 8.4.1.1 skip predictor; :3236-3255) and code the rest
 * with mb_skip_run + encode_mb_p16x16 (:1248), the residual blocks through
 * cavlc.c. Those functions are static, so this file includes encoder_h264.c
 * (unchanged) and restates only that loop around them, calling the
 * reference's own functions for every bit it writes.
 */
#include "encoder_h264.c"

/* Slice data of macroblocks [start_mb, end_mb) of one picture, written from
 * bit 0 of `out` (no slice header) and closed by rbsp_trailing_bits, as the
 * reference's CAVLC path writes it. levels/dc/nz/pred_modes/mvs are the
 * staging layouts of include/gpu_compute.h. Returns the byte count, -1 if
 * `cap` bytes did not hold it. */
int refshim_cavlc_slice_data(int mbw, int mbh, int qp, int is_idr, int quality_level, int start_mb, int end_mb,
                             const int16_t *levels, const int32_t *dc, const uint32_t *nz,
                             const uint32_t *pred_modes, const gpu_mv_t *mvs, uint8_t *out, int cap)
{
    const int total = mbw * mbh;
    uint8_t (*nzl)[16] = calloc((size_t)total, 16);
    uint8_t (*nzb)[4] = calloc((size_t)total, 4);
    uint8_t (*nzr)[4] = calloc((size_t)total, 4);
    if (!nzl || !nzb || !nzr) { free(nzl); free(nzb); free(nzr); return -1; }
    nc_ctx_t nc = {
        .nz_luma = nzl, .nz_cb = nzb, .nz_cr = nzr,
        .width_in_mbs = (uint32_t)mbw, .start_mb = (uint32_t)start_mb, .nz_mask = nz,
    };
    const int *dcs = (const int *)dc;
    bitstream_t bs;
    bs_init(&bs, out, (size_t)cap);
    if (is_idr) {
        for (uint32_t mb = (uint32_t)start_mb; mb < (uint32_t)end_mb; mb++)
            encode_mb_i16x16(&bs, levels, dcs, pred_modes, mb, mb % (uint32_t)mbw, mb / (uint32_t)mbw, &nc, qp);
    } else {
        uint32_t run = 0;
        for (uint32_t mb = (uint32_t)start_mb; mb < (uint32_t)end_mb; mb++) {
            const uint32_t mbx = mb % (uint32_t)mbw, mby = mb / (uint32_t)mbw;
            bool zl = mb_has_any_luma_nonzero(levels, nz, mb) == 0;
            bool zc = mb_has_any_chroma_nonzero(levels, dcs, nz, mb) == 0;
            if (quality_level >= 5 && zl && !zc && abs(dcs[mb * 2 + 0]) <= 1 && abs(dcs[mb * 2 + 1]) <= 1) zc = true;
            int px, py;
            skip_mv_predictor(mvs, mbx, mby, nc.width_in_mbs, nc.start_mb, &px, &py);
            const bool skip = zl && zc && mvs[mb].mvx == px && mvs[mb].mvy == py;
            if (skip) {
                run++;
                memset(nc.nz_luma[mb], 0, 16);
                memset(nc.nz_cb[mb], 0, 4);
                memset(nc.nz_cr[mb], 0, 4);
            } else {
                cavlc_write_p_skip_run(&bs, run);
                run = 0;
                encode_mb_p16x16(&bs, levels, dcs, mvs, mb, mbx, mby, &nc, qp);
            }
        }
        if (run > 0) cavlc_write_p_skip_run(&bs, run);
    }
    cavlc_write_slice_trailing_bits(&bs);
    bs_flush(&bs);
    free(nzl); free(nzb); free(nzr);
    if (bs.overflow) return -1;
    return (int)bs_bytes_written(&bs);
}
