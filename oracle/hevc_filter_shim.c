/*
 * hevc_filter_shim.c - TEST INFRASTRUCTURE ONLY. Drives the reference
 * decoder's loop filter (approach1-compute-encoder/src/hevc_filter.c and
 * its hevc_filter_template.c, compiled where they lie) over one picture
 * described by the same parameter block as b200enc_hevc_deblock
 * (include/b200enc.h), so the GPU deblocking can be compared with it
 * sample for sample. SAO stays off (no SAO parameters are set), so
 * hevcd_loop_filters runs exactly its two deblocking stages.
 */
#include "hevc_dec_internal.h"

#include <stdlib.h>
#include <string.h>

#include "../include/b200enc.h"

/* The decoder's thread pool lives in its wavefront file, which these tests
 * do not link: without a pool the filter starts threads of its own
 * (hevc_filter.c:464-480). */
hevcd_pool_t *hevcd_pool_for(hevcd_t *d)
{
    (void)d;
    return NULL;
}

/* Same parameter block as the GPU entry point, with host pointers. */
int refshim_hevc_deblock(const b200enc_hevc_deblock_t *p)
{
    if (!p || (p->bit_depth_luma != 8 && p->bit_depth_luma != 10)) return -1;
    hevc_sps_t sps;
    hevc_pps_t pps;
    hevcd_t d;
    memset(&sps, 0, sizeof sps);
    memset(&pps, 0, sizeof pps);
    memset(&d, 0, sizeof d);

    sps.chroma_format_idc = 1;
    sps.width = p->width;
    sps.height = p->height;
    sps.bit_depth_luma = p->bit_depth_luma;
    sps.bit_depth_chroma = p->bit_depth_chroma;
    sps.log2_min_cb = p->log2_min_cb;
    sps.log2_ctb = p->log2_ctb;
    sps.ctb_size = 1 << p->log2_ctb;
    sps.ctb_width = (p->width + sps.ctb_size - 1) >> p->log2_ctb;
    sps.ctb_height = (p->height + sps.ctb_size - 1) >> p->log2_ctb;
    sps.ctb_count = sps.ctb_width * sps.ctb_height;
    sps.min_cb_width = p->width >> p->log2_min_cb;
    sps.min_cb_height = p->height >> p->log2_min_cb;
    pps.cb_qp_offset = p->cb_qp_offset;
    pps.cr_qp_offset = p->cr_qp_offset;
    pps.loop_filter_across_tiles = p->loop_filter_across_tiles != 0;

    d.sps = &sps;
    d.pps = &pps;
    for (int c = 0; c < 3; c++) {
        d.plane[c] = (uint8_t *)p->plane[c];
        d.stride[c] = p->stride[c];
    }
    d.n_planes = 3;
    d.edges = (uint8_t *)p->edges;
    d.edges_stride = p->edges_stride;
    d.n_edges = (size_t)p->edges_stride * ((p->height + 7) / 8);
    d.min_pu_width = p->min_pu_width;
    d.min_pu_height = (p->height + 3) / 4;
    d.cbf_map = (uint8_t *)p->cbf;
    d.n_cbf = p->cbf ? (size_t)p->min_pu_width * d.min_pu_height : 0;
    d.qp_y_map = (int8_t *)p->qp_y;
    d.n_qp = (size_t)sps.min_cb_width * sps.min_cb_height;
    d.no_filter = (uint8_t *)p->no_filter;
    d.n_no_filter = p->no_filter ? d.n_qp : 0;
    d.slice_of_ctb = (int32_t *)p->slice_of_ctb;
    d.n_slice_map = p->slice_of_ctb ? (size_t)sps.ctb_count : 0;

    hevcd_slice_filter_t *sf = NULL;
    if (p->slice_filter && p->n_slice_filter > 0) {
        sf = calloc((size_t)p->n_slice_filter, sizeof *sf);
        if (!sf) return -1;
        for (int i = 0; i < p->n_slice_filter; i++) {
            sf[i].beta_offset = p->slice_filter[i].beta_offset;
            sf[i].tc_offset = p->slice_filter[i].tc_offset;
            sf[i].disabled = p->slice_filter[i].disabled;
            sf[i].across_slices = p->slice_filter[i].across_slices;
        }
    }
    d.slice_filter = sf;
    d.n_slice_filter = sf ? (size_t)p->n_slice_filter : 0;

    /* Tiles: a raster-order tile id per CTB, handed over with the identity
     * as tile scan, which is all hevcd_tile_at reads. */
    int32_t *ident = NULL;
    if (p->tile_of_ctb) {
        ident = malloc((size_t)sps.ctb_count * sizeof *ident);
        if (!ident) {
            free(sf);
            return -1;
        }
        int n_tiles = 1;
        for (int i = 0; i < sps.ctb_count; i++) {
            ident[i] = i;
            if (p->tile_of_ctb[i] + 1 > n_tiles) n_tiles = p->tile_of_ctb[i] + 1;
        }
        d.rs_to_ts = ident;
        d.ts_to_rs = ident;
        d.tile_of_ts = (int32_t *)p->tile_of_ctb;
        d.n_tile_map = (size_t)sps.ctb_count;
        d.n_tiles = n_tiles;
    } else {
        d.n_tiles = 1;
    }

    /* The decoder's motion field type: same values, its own layout. */
    hevcd_mvf_t *mvf = NULL;
    if (p->mvf) {
        const size_t n = (size_t)p->min_pu_width * d.min_pu_height;
        mvf = calloc(n, sizeof *mvf);
        if (!mvf) {
            free(sf);
            free(ident);
            return -1;
        }
        for (size_t i = 0; i < n; i++) {
            memcpy(mvf[i].mv, p->mvf[i].mv, sizeof mvf[i].mv);
            mvf[i].ref_poc[0] = p->mvf[i].ref_poc[0];
            mvf[i].ref_poc[1] = p->mvf[i].ref_poc[1];
            mvf[i].pred_flag = p->mvf[i].pred_flag;
        }
    }
    d.mvf = mvf;

    hevcd_loop_filters(&d);

    free(mvf);
    free(ident);
    free(sf);
    return 0;
}
