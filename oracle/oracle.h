/*
 * oracle.h - CPU restatement of the reference compute encoder's hot-path
 * stages, used ONLY as the test checker (tests/, __graft_entry__.smoke(),
 * bench.py's cpu_baseline leg). Nothing in the product library links or
 * calls this code; the CUDA path fails loudly when its extension is absent.
 *
 * Each function cites the reference file:line it follows (paths relative to
 * the reference project root, A1 = approach1-compute-encoder).
 *
 * Parity pinning: the restatement is checked against (a) the reference's own
 * C functions compiled from its sources into oracle/_ref (h264_deblock.c,
 * h264_mc.c, h264_recon.c, cpu_simd_me.c, encoder_h264.c's exported DC
 * transform) and (b) the reference tests' golden vectors
 * (A1/tests/test_encode.c:60-96, A1/tests/test_cpu_simd_me.c:16-106).
 *
 * Plane conventions shared with the CUDA library:
 *   - luma: 8-bit, row pitch `pitch` bytes.
 *   - chroma: NV12 interleaved CbCr, row pitch `pitch` bytes (W/2 pairs).
 *   - source reads clamp to the visible size (W, H); reference/recon reads
 *     clamp to (RW, RH) and recon writes are bounded by (RW, RH). RW/RH equal
 *     to W/H reproduces the reference shaders exactly; RW/RH equal to the
 *     coded size (16*mbw, 16*mbh) is what a conforming decoder does.
 */
#ifndef B200ENC_ORACLE_H
#define B200ENC_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int32_t mvx, mvy; /* quarter-pel */
    uint32_t sad;
    uint32_t pad;
} orc_mv_t;

typedef struct {
    int W, H;      /* visible size: source clamp */
    int RW, RH;    /* recon/reference clamp and recon write bound */
    int mbw, mbh;
    int qp;
    int num_slices;
    int flags;     /* ORC_INTRA_CORNER_CHECK: Plane also needs the top-left MB's slice */
} orc_frame_t;

/* Intra16x16 Plane predicts from p[-1,-1] too, so a conforming encoder only
 * picks it when the top-left macroblock is available. The reference shader
 * only checks top and left (A1/shaders/intra_wavefront.comp:463, :486, :497),
 * which lets it pick Plane across a slice boundary that starts at the top
 * neighbour; with this flag the top-left slice is checked as well. */
#define ORC_INTRA_CORNER_CHECK 1

typedef struct {
    int range;        /* integer search range R: dx, dy in [-R, R] */
    int lambda;       /* motion cost weight per integer pel of |dx|+|dy| */
    int zero_thresh;  /* SAD(0,0) <= zero_thresh ends the search; < 0 disables */
} orc_me_params_t;

/* Per-frame outputs, reference staging layout (A1/src/gpu_compute.h:575-648). */
typedef struct {
    int16_t  *levels;    /* [mbs][24][16] */
    int32_t  *dc;        /* [mbs][24] */
    uint32_t *nz;        /* [mbs][24] */
    uint32_t *pred_mode; /* [mbs] */
    orc_mv_t *mv;        /* [mbs] */
} orc_out_t;

int  orc_chroma_qp(int qpy);
uint32_t orc_slice_of(uint32_t mb, uint32_t total_mbs, uint32_t num_slices);
void orc_forward_4x4(const int in[16], int out[16]);
void orc_inverse_4x4(int d[16], int r[16]);
int  orc_quant_ac(int coeff, int pos, int qp, int intra);
int  orc_dequant_ac(int level, int pos, int qp);
void orc_luma_dc_hadamard_fwd(const int in[16], int out[16]);
void orc_luma_dc_hadamard_inv(const int in[16], int out[16]);
void orc_chroma_dc_hadamard(const int in[4], int out[4]);
int  orc_quantize_dc_luma(int v, int qp);
int  orc_quantize_dc_chroma(int v, int qp);
int  orc_dequant_dc_luma(int f, int qp);
int  orc_dequant_dc_chroma(int f, int qp);
/* Spec-order I16x16 DC as handed to CAVLC (transposed), test_encode.c:60-96. */
void orc_intra16_luma_dc_transform(const int dc_in[16], int qp, int dc_out[16], int pre[16]);

int  orc_interp_luma_qpel(const uint8_t *ref, int pitch, int RW, int RH, int qx, int qy);
int  orc_interp_chroma(const uint8_t *ref_uv, int pitch, int RW, int RH, int plane, int ex, int ey);
uint32_t orc_sad16(const uint8_t *a, int pa, const uint8_t *b, int pb);

/* Plain full-search ME for one frame. */
void orc_me_frame(const orc_frame_t *f, const orc_me_params_t *p,
                  const uint8_t *cur_y, int cur_pitch,
                  const uint8_t *ref_y, int ref_pitch, orc_mv_t *mv);

/* Half- then quarter-pel refine of the plain search around integer winner
 * (imx, imy) whose integer SAD is int_sad; writes mvx, mvy, sad, pad = 0. */
void orc_me_refine(const orc_frame_t *f, const uint8_t *cur_y, int cur_pitch, const uint8_t *ref_y, int ref_pitch,
                   int mbx, int mby, int imx, int imy, uint32_t int_sad, orc_mv_t *o);

/* The plain search's selection key minimised over the integer MVs of the
 * rectangle [x0,x1] x [y0,y1] (inside [-R,R]^2); key >> 14 = SAD + lambda
 * cost, key & 0x3fff = (dy+R)*(2R+1) + dx+R. */
uint32_t orc_me_rect_key(const orc_frame_t *f, const orc_me_params_t *p, const uint8_t *cur_y, int cur_pitch,
                         const uint8_t *ref_y, int ref_pitch, int mbx, int mby, int x0, int y0, int x1, int y1);

/* P-frame predict + transform + quant + DC + dequant + recon, given MVs. */
void orc_p_frame(const orc_frame_t *f,
                 const uint8_t *cur_y, const uint8_t *cur_uv, int cur_pitch,
                 const uint8_t *ref_y, const uint8_t *ref_uv, int ref_pitch,
                 const orc_mv_t *mv, orc_out_t *out,
                 uint8_t *rec_y, uint8_t *rec_uv, int rec_pitch);

/* I-frame intra wavefront (run in raster order, which respects the
 * diagonal dependency), writing recon in place. */
void orc_i_frame(const orc_frame_t *f,
                 const uint8_t *cur_y, const uint8_t *cur_uv, int cur_pitch,
                 orc_out_t *out, uint8_t *rec_y, uint8_t *rec_uv, int rec_pitch);

/* The same macroblocks in a caller-given order (raster indices); orc_i_frame
 * is the raster order. Returns -1 for a macroblock outside the picture. For
 * checking that a parallel schedule keeps the raster order's result. */
int orc_i_frame_steps(const orc_frame_t *f,
                      const uint8_t *cur_y, const uint8_t *cur_uv, int cur_pitch,
                      orc_out_t *out, uint8_t *rec_y, uint8_t *rec_uv, int rec_pitch,
                      const int32_t *order, int n);

/* Spec deblocking (H.264 8.7) of the coded picture (16*mbw x 16*mbh) for
 * the macroblock kinds this encoder emits: all-intra (I16x16) frames or
 * all-inter (P16x16 / P_Skip, one reference) frames, uniform QP,
 * disable_deblocking_filter_idc = 0, zero filter offsets. */
void orc_deblock_frame(int mbw, int mbh, int qp, int is_intra,
                       const uint32_t *nz, const orc_mv_t *mv,
                       uint8_t *rec_y, uint8_t *rec_uv, int rec_pitch);

/* The same filtering as steps applied in a caller-given order, steps[i] =
 * 2 * mb + dir (dir 0: the macroblock's vertical edges, 1: its horizontal
 * edges); orc_deblock_frame is the raster order 0, 1, 2, 3, ... Returns -1
 * for a step outside the picture. For checking that a parallel schedule
 * keeps the raster order's result. */
/* orc_deblock_frame with the 8x8 transform in the macroblocks whose t8 byte
 * is nonzero (t8 NULL: none): their odd luma edges are not filtered and the
 * coefficient test of a boundary strength looks at the 8x8 block. */
void orc_deblock_frame_t8(int mbw, int mbh, int qp, int is_intra, const uint32_t *nz, const uint8_t *t8,
                          const orc_mv_t *mv, uint8_t *ry, uint8_t *ruv, int rp);
int orc_deblock_steps(int mbw, int mbh, int qp, int is_intra,
                      const uint32_t *nz, const orc_mv_t *mv,
                      uint8_t *rec_y, uint8_t *rec_uv, int rec_pitch,
                      const int32_t *steps, int nsteps);

/* One whole frame of the hot path: ME (P only) -> P or I chain -> deblock. */
void orc_encode_frame(const orc_frame_t *f, const orc_me_params_t *p, int is_intra, int deblock,
                      const uint8_t *cur_y, const uint8_t *cur_uv, int cur_pitch,
                      const uint8_t *ref_y, const uint8_t *ref_uv, int ref_pitch,
                      orc_out_t *out, uint8_t *rec_y, uint8_t *rec_uv, int rec_pitch);

/* Threads for the oracle's parallel loops (full search, P chain). */
void orc_set_threads(int n);

#ifdef __cplusplus
}
#endif

/* H.264 High profile 8x8 transform: forward integer transform and
 * quantisation with flat scaling lists (the encoder side), and scaling,
 * inverse transform and the add onto a prediction (clause 8.5.13, the
 * decoder side, pinned to the reference decoder's h264d_idct8_add).
 * Coefficients and levels in raster order. */
/* The P chain with the 8x8 luma transform (High profile; no counterpart in
 * the reference's encoder): t8 = 0 is orc_p_frame, 1 codes every
 * macroblock's luma as four 8x8 blocks, 2 chooses per macroblock
 * (orc_t8_choose). An 8x8 block's levels are raster over the four 16-level
 * slots of its quadrant; the nz word of each of its 4x4 blocks is the mask of
 * the 16 levels CAVLC codes as that block; t8_flags (may be NULL) gets each
 * macroblock's choice. */
void orc_p_frame_t8(const orc_frame_t *f,
                    const uint8_t *cur_y, const uint8_t *cur_uv, int cur_pitch,
                    const uint8_t *ref_y, const uint8_t *ref_uv, int ref_pitch,
                    const orc_mv_t *mv, orc_out_t *out,
                    uint8_t *rec_y, uint8_t *rec_uv, int rec_pitch, int t8, uint8_t *t8_flags);
/* 1 when a macroblock's luma residual (int [16][16] raster) costs less under
 * the 8x8 transform than under the 4x4 one. */
int orc_t8_choose(const int res[256]);
void orc_fwd_quant8(const int16_t res[64], int16_t lev[64], int qp, int intra);
void orc_dequant_idct8_add(const int16_t lev[64], uint8_t *dst, int stride, int qp);

#endif
