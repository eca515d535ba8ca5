/*
 * oracle.c - CPU restatement of the reference compute encoder's hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline leg. The product library never links it.
 *
 * Citations are reference paths (A1 = approach1-compute-encoder). The GLSL
 * shaders cannot run anywhere here (no Vulkan), so their integer math is
 * restated in C; the decoder-side pieces follow the reference's own C and
 * are cross-checked against it (compiled from its sources into oracle/_ref).
 */
#include "oracle.h"

#include <omp.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline int clip1(int v) { return clampi(v, 0, 255); }
static inline int iabs(int v) { return v < 0 ? -v : v; }

/* ---------------------------------------------------------------- tables */

/* MF, A1/shaders/quantize.comp:151-158; columns [both even, both odd, mixed]. */
static const int MF[6][3] = {
    {13107, 5243, 8066}, {11916, 4660, 7490}, {10082, 4194, 6554},
    {9362, 3647, 5825},  {8192, 3355, 5243},  {7282, 2893, 4559}};
/* V, A1/shaders/reconstruct.comp:124-131 (same column convention). */
static const int VT[6][3] = {
    {10, 16, 13}, {11, 18, 14}, {13, 20, 16}, {14, 23, 18}, {16, 25, 20}, {18, 29, 23}};
/* A1/shaders/reconstruct.comp:92 = A1/src/encoder_h264.c DC_LEVEL_SCALE0. */
static const int DC_LS[6] = {160, 176, 208, 224, 256, 288};

static inline int pos_type(int idx)
{
    /* A1/shaders/quantize.comp:160-168 */
    int r = idx >> 2, c = idx & 3;
    if (!(r & 1) && !(c & 1)) return 0;
    if ((r & 1) && (c & 1)) return 1;
    return 2;
}

int orc_chroma_qp(int qpy)
{
    /* A1/shaders/quantize.comp:182-187 (Table 8-15 with offset 0) */
    static const int t[22] = {29, 30, 31, 32, 32, 33, 34, 34, 35, 35, 36,
                              36, 37, 37, 37, 38, 38, 38, 39, 39, 39, 39};
    if (qpy < 30) return qpy;
    int i = qpy - 30;
    return t[i < 22 ? i : 21];
}

uint32_t orc_slice_of(uint32_t mb, uint32_t total, uint32_t ns)
{
    /* A1/shaders/residual_predict.comp:163-171 */
    if (ns <= 1 || total == 0) return 0;
    uint32_t s = (mb * ns) / total;
    if (s >= ns) s = ns - 1;
    while (s + 1 < ns && ((s + 1) * total) / ns <= mb) s++;
    while (s > 0 && (s * total) / ns > mb) s--;
    return s;
}

/* ------------------------------------------------------------ transforms */

void orc_forward_4x4(const int in[16], int out[16])
{
    /* A1/shaders/dct_transform.comp:34-73: rows then columns. */
    int m[16];
    for (int i = 0; i < 4; i++) {
        const int *p = in + 4 * i;
        int a0 = p[0] + p[3], a1 = p[1] + p[2], a2 = p[1] - p[2], a3 = p[0] - p[3];
        m[4 * i + 0] = a0 + a1;
        m[4 * i + 1] = (a3 << 1) + a2;
        m[4 * i + 2] = a0 - a1;
        m[4 * i + 3] = a3 - (a2 << 1);
    }
    for (int j = 0; j < 4; j++) {
        int p0 = m[j], p1 = m[4 + j], p2 = m[8 + j], p3 = m[12 + j];
        int a0 = p0 + p3, a1 = p1 + p2, a2 = p1 - p2, a3 = p0 - p3;
        out[j] = a0 + a1;
        out[4 + j] = (a3 << 1) + a2;
        out[8 + j] = a0 - a1;
        out[12 + j] = a3 - (a2 << 1);
    }
}

void orc_inverse_4x4(int d[16], int r[16])
{
    /* A1/shaders/reconstruct.comp:162-177 (+32 on DC, rows, columns, >>6). */
    int t[16];
    d[0] += 32;
    for (int i = 0; i < 4; i++) {
        const int *p = d + 4 * i;
        int z0 = p[0] + p[2], z1 = p[0] - p[2], z2 = (p[1] >> 1) - p[3], z3 = p[1] + (p[3] >> 1);
        t[4 * i + 0] = z0 + z3;
        t[4 * i + 1] = z1 + z2;
        t[4 * i + 2] = z1 - z2;
        t[4 * i + 3] = z0 - z3;
    }
    for (int j = 0; j < 4; j++) {
        int p0 = t[j], p1 = t[4 + j], p2 = t[8 + j], p3 = t[12 + j];
        int z0 = p0 + p2, z1 = p0 - p2, z2 = (p1 >> 1) - p3, z3 = p1 + (p3 >> 1);
        r[j] = (z0 + z3) >> 6;
        r[4 + j] = (z1 + z2) >> 6;
        r[8 + j] = (z1 - z2) >> 6;
        r[12 + j] = (z0 - z3) >> 6;
    }
}

int orc_quant_ac(int coeff, int pos, int qp, int intra)
{
    /* A1/shaders/quantize.comp:203-221 */
    int per = qp / 6, rem = qp % 6;
    int f = (1 << (15 + per)) / (intra ? 3 : 6);
    int a = iabs(coeff);
    int level = (a * MF[rem][pos_type(pos)] + f) >> (15 + per);
    return coeff < 0 ? -level : level;
}

int orc_dequant_ac(int level, int pos, int qp)
{
    /* A1/shaders/reconstruct.comp:148-154 */
    int per = qp / 6, rem = qp % 6;
    int scale = 16 * VT[rem][pos_type(pos)];
    if (per >= 4) return (level * scale) << (per - 4);
    return (level * scale + (1 << (3 - per))) >> (4 - per);
}

void orc_luma_dc_hadamard_fwd(const int in[16], int out[16])
{
    /* A1/src/encoder_h264.c:711-730 (= reconstruct.comp:181-194) */
    int t[16];
    for (int i = 0; i < 4; i++) {
        int s01 = in[4 * i] + in[4 * i + 1], d01 = in[4 * i] - in[4 * i + 1];
        int s23 = in[4 * i + 2] + in[4 * i + 3], d23 = in[4 * i + 2] - in[4 * i + 3];
        t[i] = s01 + s23;
        t[4 + i] = s01 - s23;
        t[8 + i] = d01 - d23;
        t[12 + i] = d01 + d23;
    }
    for (int i = 0; i < 4; i++) {
        int s01 = t[4 * i] + t[4 * i + 1], d01 = t[4 * i] - t[4 * i + 1];
        int s23 = t[4 * i + 2] + t[4 * i + 3], d23 = t[4 * i + 2] - t[4 * i + 3];
        out[4 * i + 0] = (s01 + s23 + 1) >> 1;
        out[4 * i + 1] = (s01 - s23 + 1) >> 1;
        out[4 * i + 2] = (d01 - d23 + 1) >> 1;
        out[4 * i + 3] = (d01 + d23 + 1) >> 1;
    }
}

void orc_luma_dc_hadamard_inv(const int in[16], int out[16])
{
    /* A1/shaders/reconstruct.comp:201-213: same butterflies, no >>1. */
    int t[16];
    for (int i = 0; i < 4; i++) {
        int s01 = in[4 * i] + in[4 * i + 1], d01 = in[4 * i] - in[4 * i + 1];
        int s23 = in[4 * i + 2] + in[4 * i + 3], d23 = in[4 * i + 2] - in[4 * i + 3];
        t[i] = s01 + s23;
        t[4 + i] = s01 - s23;
        t[8 + i] = d01 - d23;
        t[12 + i] = d01 + d23;
    }
    for (int i = 0; i < 4; i++) {
        int s01 = t[4 * i] + t[4 * i + 1], d01 = t[4 * i] - t[4 * i + 1];
        int s23 = t[4 * i + 2] + t[4 * i + 3], d23 = t[4 * i + 2] - t[4 * i + 3];
        out[4 * i + 0] = s01 + s23;
        out[4 * i + 1] = s01 - s23;
        out[4 * i + 2] = d01 - d23;
        out[4 * i + 3] = d01 + d23;
    }
}

void orc_chroma_dc_hadamard(const int c[4], int o[4])
{
    /* A1/src/encoder_h264.c:791-797 */
    o[0] = c[0] + c[1] + c[2] + c[3];
    o[1] = c[0] - c[1] + c[2] - c[3];
    o[2] = c[0] + c[1] - c[2] - c[3];
    o[3] = c[0] - c[1] - c[2] + c[3];
}

static int quantize_dc_common(int v, int qp)
{
    /* A1/src/encoder_h264.c:653-678 and :687-709 (identical bodies; int64
     * there, int32 here is exact for 8-bit residual ranges). */
    int per = qp / 6, rem = qp % 6;
    long long ls = DC_LS[rem], av = v < 0 ? -(long long)v : v, num, den;
    if (per >= 5) { num = av; den = ls << (per - 5); }
    else { num = av << (5 - per); den = ls; }
    long long level = (num + den / 2) / den;
    return (int)(v < 0 ? -level : level);
}
int orc_quantize_dc_luma(int v, int qp) { return quantize_dc_common(v, qp); }
int orc_quantize_dc_chroma(int v, int qp) { return quantize_dc_common(v, qp); }

int orc_dequant_dc_luma(int f, int qp)
{
    /* A1/shaders/reconstruct.comp:285-291 */
    int per = qp / 6, ls = DC_LS[qp % 6];
    if (per >= 6) return (f * ls) << (per - 6);
    return (f * ls + (1 << (5 - per))) >> (6 - per);
}

int orc_dequant_dc_chroma(int f, int qp)
{
    /* A1/shaders/reconstruct.comp:293-299 */
    int per = qp / 6, ls = DC_LS[qp % 6];
    if (per >= 5) return (f * ls) << (per - 5);
    return (f * ls) >> (5 - per);
}

void orc_intra16_luma_dc_transform(const int dc_in[16], int qp, int dc_out[16], int pre[16])
{
    /* A1/src/encoder_h264.c:775-789: Hadamard, quantize, hand CAVLC the
     * transpose. */
    int raw[16], nat[16];
    orc_luma_dc_hadamard_fwd(dc_in, raw);
    for (int i = 0; i < 16; i++) nat[i] = orc_quantize_dc_luma(raw[i], qp);
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++) dc_out[4 * r + c] = nat[4 * c + r];
    if (pre) memcpy(pre, nat, sizeof(nat));
}

/* ---------------------------------------------------------- interpolation */

static inline int refY(const uint8_t *ref, int pitch, int RW, int RH, int x, int y)
{
    return ref[(size_t)clampi(y, 0, RH - 1) * pitch + clampi(x, 0, RW - 1)];
}

static int hraw(const uint8_t *r, int p, int RW, int RH, int x, int y)
{
    return refY(r, p, RW, RH, x - 2, y) - 5 * refY(r, p, RW, RH, x - 1, y) + 20 * refY(r, p, RW, RH, x, y) +
           20 * refY(r, p, RW, RH, x + 1, y) - 5 * refY(r, p, RW, RH, x + 2, y) + refY(r, p, RW, RH, x + 3, y);
}
static int vraw(const uint8_t *r, int p, int RW, int RH, int x, int y)
{
    return refY(r, p, RW, RH, x, y - 2) - 5 * refY(r, p, RW, RH, x, y - 1) + 20 * refY(r, p, RW, RH, x, y) +
           20 * refY(r, p, RW, RH, x, y + 1) - 5 * refY(r, p, RW, RH, x, y + 2) + refY(r, p, RW, RH, x, y + 3);
}

int orc_interp_luma_qpel(const uint8_t *ref, int p, int RW, int RH, int qx, int qy)
{
    /* A1/shaders/motion_estimation.comp:180-215 (= residual_predict.comp:263-298) */
    int ix = qx >> 2, iy = qy >> 2, fx = qx & 3, fy = qy & 3;
    int G = refY(ref, p, RW, RH, ix, iy);
    if (!fx && !fy) return G;
    int H = refY(ref, p, RW, RH, ix + 1, iy);
    int M = refY(ref, p, RW, RH, ix, iy + 1);
    int b = clip1((hraw(ref, p, RW, RH, ix, iy) + 16) >> 5);
    int h = clip1((vraw(ref, p, RW, RH, ix, iy) + 16) >> 5);
    int m = clip1((vraw(ref, p, RW, RH, ix + 1, iy) + 16) >> 5);
    int s = clip1((hraw(ref, p, RW, RH, ix, iy + 1) + 16) >> 5);
    int j1 = hraw(ref, p, RW, RH, ix, iy - 2) - 5 * hraw(ref, p, RW, RH, ix, iy - 1) +
             20 * hraw(ref, p, RW, RH, ix, iy) + 20 * hraw(ref, p, RW, RH, ix, iy + 1) -
             5 * hraw(ref, p, RW, RH, ix, iy + 2) + hraw(ref, p, RW, RH, ix, iy + 3);
    int j = clip1((j1 + 512) >> 10);
#define QAVG(a, c) (((a) + (c) + 1) >> 1)
    switch (fy * 4 + fx) {
    case 1: return QAVG(G, b);
    case 2: return b;
    case 3: return QAVG(b, H);
    case 4: return QAVG(G, h);
    case 5: return QAVG(b, h);
    case 6: return QAVG(b, j);
    case 7: return QAVG(b, m);
    case 8: return h;
    case 9: return QAVG(h, j);
    case 10: return j;
    case 11: return QAVG(j, m);
    case 12: return QAVG(h, M);
    case 13: return QAVG(h, s);
    case 14: return QAVG(j, s);
    default: return QAVG(m, s);
    }
#undef QAVG
}

int orc_interp_chroma(const uint8_t *uv, int p, int RW, int RH, int plane, int ex, int ey)
{
    /* A1/shaders/residual_predict.comp:613-630; (ex, ey) in 1/8 chroma pel. */
    int mx = RW / 2 - 1, my = RH / 2 - 1;
    int ix = ex >> 3, iy = ey >> 3, fx = ex & 7, fy = ey & 7;
    int x0 = clampi(ix, 0, mx), x1 = clampi(ix + 1, 0, mx);
    int y0 = clampi(iy, 0, my), y1 = clampi(iy + 1, 0, my);
    int A = uv[(size_t)y0 * p + 2 * x0 + plane], B = uv[(size_t)y0 * p + 2 * x1 + plane];
    int C = uv[(size_t)y1 * p + 2 * x0 + plane], D = uv[(size_t)y1 * p + 2 * x1 + plane];
    return ((8 - fx) * (8 - fy) * A + fx * (8 - fy) * B + (8 - fx) * fy * C + fx * fy * D + 32) >> 6;
}

uint32_t orc_sad16(const uint8_t *a, int pa, const uint8_t *b, int pb)
{
    uint32_t s = 0;
    for (int y = 0; y < 16; y++)
        for (int x = 0; x < 16; x++) s += (uint32_t)iabs(a[y * pa + x] - b[y * pb + x]);
    return s;
}

/* -------------------------------------------------------------------- ME */

static void load_cur_mb(const orc_frame_t *f, const uint8_t *cur, int pitch, int mbx, int mby, int out[256])
{
    for (int y = 0; y < 16; y++)
        for (int x = 0; x < 16; x++)
            out[y * 16 + x] = cur[(size_t)clampi(mby * 16 + y, 0, f->H - 1) * pitch +
                                  clampi(mbx * 16 + x, 0, f->W - 1)];
}

static uint32_t sad_qpel(const orc_frame_t *f, const int cur[256], const uint8_t *ref, int rp,
                         int X, int Y, int mvx, int mvy)
{
    uint32_t s = 0;
    for (int y = 0; y < 16; y++)
        for (int x = 0; x < 16; x++)
            s += (uint32_t)iabs(cur[y * 16 + x] -
                                orc_interp_luma_qpel(ref, rp, f->RW, f->RH, (X + x) * 4 + mvx, (Y + y) * 4 + mvy));
    return s;
}

static const int HALF_OFF[8][2] = {{2, 0}, {-2, 0}, {0, 2}, {0, -2}, {2, 2}, {2, -2}, {-2, 2}, {-2, -2}};
static const int QTR_OFF[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {1, -1}, {-1, 1}, {-1, -1}};

void orc_me_refine(const orc_frame_t *f, const uint8_t *cur_y, int cp, const uint8_t *ref_y, int rp,
                   int mbx, int mby, int imx, int imy, uint32_t int_sad, orc_mv_t *o)
{
    /* Steps 3-4 of the plain search below, for a given integer winner. */
    int cur[256];
    load_cur_mb(f, cur_y, cp, mbx, mby, cur);
    const int X = mbx * 16, Y = mby * 16;
    int bx = imx * 4, by = imy * 4;
    uint32_t best = int_sad;
    int hx = 0, hy = 0;
    for (int c = 0; c < 8; c++) {
        uint32_t s = sad_qpel(f, cur, ref_y, rp, X, Y, bx + HALF_OFF[c][0], by + HALF_OFF[c][1]);
        if (s < best) { best = s; hx = HALF_OFF[c][0]; hy = HALF_OFF[c][1]; }
    }
    bx += hx; by += hy;
    int qx = 0, qy = 0;
    for (int c = 0; c < 8; c++) {
        uint32_t s = sad_qpel(f, cur, ref_y, rp, X, Y, bx + QTR_OFF[c][0], by + QTR_OFF[c][1]);
        if (s < best) { best = s; qx = QTR_OFF[c][0]; qy = QTR_OFF[c][1]; }
    }
    o->mvx = bx + qx;
    o->mvy = by + qy;
    o->sad = best;
    o->pad = 0;
}

uint32_t orc_me_rect_key(const orc_frame_t *f, const orc_me_params_t *p, const uint8_t *cur_y, int cp,
                         const uint8_t *ref_y, int rp, int mbx, int mby, int x0, int y0, int x1, int y1)
{
    /* The plain search's key (cost << 14 | raster index over [-R,R]^2)
     * minimised over the integer MVs of [x0,x1] x [y0,y1] only. */
    const int R = p->range, side = 2 * R + 1, X = mbx * 16, Y = mby * 16;
    int cur[256];
    load_cur_mb(f, cur_y, cp, mbx, mby, cur);
    uint32_t best_key = 0xffffffffu;
    for (int dy = y0; dy <= y1; dy++)
        for (int dx = x0; dx <= x1; dx++) {
            uint32_t s = 0;
            for (int y = 0; y < 16; y++)
                for (int x = 0; x < 16; x++)
                    s += (uint32_t)iabs(cur[y * 16 + x] - refY(ref_y, rp, f->RW, f->RH, X + x + dx, Y + y + dy));
            uint32_t cost = s + (uint32_t)p->lambda * (uint32_t)(iabs(dx) + iabs(dy));
            uint32_t key = (cost << 14) | (uint32_t)((dy + R) * side + (dx + R));
            if (key < best_key) best_key = key;
        }
    return best_key;
}

/* Edge-replicated copy of the reference luma: sample (x, y) of the copy at
 * pad[(y + P) * pp + x + P] equals refY(ref, rp, RW, RH, x, y) for every x in
 * [-P, RW+P), y in [-P, RH+P), so the search reads it without clamps. */
static uint8_t *pad_ref(const orc_frame_t *f, const uint8_t *ref_y, int rp, int P, int *pp)
{
    const int pw = f->RW + 2 * P, ph = f->RH + 2 * P;
    uint8_t *pad = (uint8_t *)malloc((size_t)pw * ph);
    if (!pad) return NULL;
    for (int y = 0; y < ph; y++)
        for (int x = 0; x < pw; x++) pad[(size_t)y * pw + x] = (uint8_t)refY(ref_y, rp, f->RW, f->RH, x - P, y - P);
    *pp = pw;
    return pad;
}

/* SAD of the 16x16 block cur (contiguous rows) against r (pitch rp). */
static inline uint32_t sad16_u8(const uint8_t *cur, const uint8_t *r, int rp)
{
    uint32_t s = 0;
    for (int y = 0; y < 16; y++) {
        const uint8_t *a = cur + 16 * y, *b = r + (size_t)y * rp;
        for (int x = 0; x < 16; x++) s += (uint32_t)iabs((int)a[x] - (int)b[x]);
    }
    return s;
}

void orc_me_frame(const orc_frame_t *f, const orc_me_params_t *p,
                  const uint8_t *cur_y, int cp, const uint8_t *ref_y, int rp, orc_mv_t *mv)
{
    /*
     * Plain full search (the reference has no exhaustive search; this is the
     * plain form's definition, built from A1/shaders/motion_estimation.comp):
     *   1. SAD at (0,0); if <= zero_thresh, MV (0,0) with that SAD (:312-331).
     *   2. Every integer (dx,dy) in [-R,R]^2, cost = SAD + lambda*(|dx|+|dy|)
     *      (:363); lowest cost wins, ties go to the first in raster order
     *      (dy outer, dx inner).
     *   3. Eight half-pel offsets around the winner, exact 6-tap SAD, strict
     *      improvement over the winner's integer SAD, in :395-398 order.
     *   4. Eight quarter-pel offsets around that, same rule (:435-438).
     * Reference samples are read clamped to (RW, RH) (refY); steps 1-2 read
     * them from an edge-replicated copy, which holds the same values, and the
     * macroblock rows run in parallel (each MB is independent).
     */
    const int R = p->range, side = 2 * R + 1, P = R + 16;
    int pp = 0;
    uint8_t *pad = pad_ref(f, ref_y, rp, P, &pp);
    if (!pad) return;
#pragma omp parallel for schedule(dynamic, 1)
    for (int mby = 0; mby < f->mbh; mby++) {
        int cur[256];
        uint8_t cur8[256];
        for (int mbx = 0; mbx < f->mbw; mbx++) {
            const int X = mbx * 16, Y = mby * 16;
            orc_mv_t *o = &mv[mby * f->mbw + mbx];
            load_cur_mb(f, cur_y, cp, mbx, mby, cur);
            for (int i = 0; i < 256; i++) cur8[i] = (uint8_t)cur[i];
            const uint8_t *at = pad + (size_t)(Y + P) * pp + (X + P);
            const uint32_t sad0 = sad16_u8(cur8, at, pp);
            if (p->zero_thresh >= 0 && sad0 <= (uint32_t)p->zero_thresh) {
                o->mvx = o->mvy = 0;
                o->sad = sad0;
                o->pad = 0;
                continue;
            }
            uint32_t best_key = 0xffffffffu, best_sad = 0;
            for (int dy = -R; dy <= R; dy++)
                for (int dx = -R; dx <= R; dx++) {
                    const uint32_t s = sad16_u8(cur8, at + (ptrdiff_t)dy * pp + dx, pp);
                    uint32_t cost = s + (uint32_t)p->lambda * (uint32_t)(iabs(dx) + iabs(dy));
                    uint32_t key = (cost << 14) | (uint32_t)((dy + R) * side + (dx + R));
                    if (key < best_key) { best_key = key; best_sad = s; }
                }
            int idx = (int)(best_key & 0x3fff);
            orc_me_refine(f, cur_y, cp, ref_y, rp, mbx, mby, idx % side - R, idx / side - R, best_sad, o);
        }
    }
    free(pad);
}

/* ------------------------------------------------------- P-frame chain */

static void store_rec_luma(const orc_frame_t *f, uint8_t *rec, int rp, int X, int Y, int blk, const int v[16])
{
    int ox = X + (blk & 3) * 4, oy = Y + (blk >> 2) * 4;
    for (int p = 0; p < 16; p++) {
        int x = ox + (p & 3), y = oy + (p >> 2);
        if (x < f->RW && y < f->RH) rec[(size_t)y * rp + x] = (uint8_t)v[p];
    }
}

static void store_rec_chroma(const orc_frame_t *f, uint8_t *rec_uv, int rp, int Xc, int Yc, int sub,
                             const int cb[16], const int cr[16])
{
    int ox = Xc + (sub & 1) * 4, oy = Yc + (sub >> 1) * 4;
    int mx = f->RW / 2 - 1, my = f->RH / 2 - 1;
    for (int p = 0; p < 16; p++) {
        int x = ox + (p & 3), y = oy + (p >> 2);
        if (x > mx || y > my) continue;
        rec_uv[(size_t)y * rp + 2 * x] = (uint8_t)cb[p];
        rec_uv[(size_t)y * rp + 2 * x + 1] = (uint8_t)cr[p];
    }
}

static inline int srcY(const orc_frame_t *f, const uint8_t *s, int p, int x, int y)
{
    return s[(size_t)clampi(y, 0, f->H - 1) * p + clampi(x, 0, f->W - 1)];
}
static inline int srcC(const orc_frame_t *f, const uint8_t *s, int p, int plane, int x, int y)
{
    return s[(size_t)clampi(y, 0, f->H / 2 - 1) * p + 2 * clampi(x, 0, f->W / 2 - 1) + plane];
}

/* Chroma DC + recon for the 8 chroma blocks of one MB, shared by the P and
 * I paths (A1/shaders/reconstruct.comp:383-441, intra_wavefront.comp:706-755). */
static void chroma_recon(const orc_frame_t *f, int qpc, const int coef[24][16], const int lev[24][16],
                         const int pred[24][16], uint8_t *rec_uv, int rp, int Xc, int Yc)
{
    int rec[2][4][16];
    for (int pl = 0; pl < 2; pl++) {
        int din[4], raw[4], lv[4], fv[4];
        for (int b = 0; b < 4; b++) din[b] = coef[16 + 4 * pl + b][0];
        orc_chroma_dc_hadamard(din, raw);
        for (int i = 0; i < 4; i++) lv[i] = orc_quantize_dc_chroma(raw[i], qpc);
        orc_chroma_dc_hadamard(lv, fv);
        for (int sub = 0; sub < 4; sub++) {
            int blk = 16 + 4 * pl + sub, d[16], r[16];
            d[0] = orc_dequant_dc_chroma(fv[sub], qpc);
            for (int p = 1; p < 16; p++) d[p] = orc_dequant_ac(lev[blk][p], p, qpc);
            orc_inverse_4x4(d, r);
            for (int p = 0; p < 16; p++) rec[pl][sub][p] = clip1(pred[blk][p] + r[p]);
        }
    }
    for (int sub = 0; sub < 4; sub++) store_rec_chroma(f, rec_uv, rp, Xc, Yc, sub, rec[0][sub], rec[1][sub]);
}

/* H.264 8x8 frame zig-zag scan (Table 8-13): scan position -> raster 8y+x,
 * built by walking the anti-diagonals, up-right on even ones and down-left
 * on odd ones. */
static void zigzag8(int zz[64])
{
    int n = 0;
    for (int d = 0; d < 15; d++) {
        const int lo = d > 7 ? d - 7 : 0, hi = d < 7 ? d : 7;
        for (int k = hi; k >= lo; k--) {
            const int x = (d & 1) ? k : d - k, y = d - x;
            zz[n++] = 8 * y + x;
        }
    }
}

/* Sum of |coefficients| of the 2-D Walsh-Hadamard transform of an n x n
 * block (n = 4 or 8), raster int. */
static int hadamard_abs(const int *blk, int n)
{
    int t[64];
    for (int i = 0; i < n * n; i++) t[i] = blk[i];
    for (int pass = 0; pass < 2; pass++)
        for (int line = 0; line < n; line++)
            for (int h = 1; h < n; h <<= 1)
                for (int i = 0; i < n; i += 2 * h)
                    for (int j = i; j < i + h; j++) {
                        int *a = pass ? &t[j * n + line] : &t[line * n + j];
                        int *b = pass ? &t[(j + h) * n + line] : &t[line * n + j + h];
                        const int u = *a, v = *b;
                        *a = u + v;
                        *b = u - v;
                    }
    int s = 0;
    for (int i = 0; i < n * n; i++) s += abs(t[i]);
    return s;
}

int orc_t8_choose(const int res[256])
{
    /* The luma residual's cost under each transform size, both on the scale
     * of a sum of absolute differences: 4x4 blocks (sum |H4 R H4|) / 2,
     * 8x8 blocks (sum |H8 R H8| + 2) / 4 (H4, H8 unnormalised Walsh-Hadamard
     * matrices); the 8x8 transform when its cost is lower. */
    int c4 = 0, c8 = 0, b[64];
    for (int by = 0; by < 4; by++)
        for (int bx = 0; bx < 4; bx++) {
            for (int i = 0; i < 16; i++) b[i] = res[(4 * by + (i >> 2)) * 16 + 4 * bx + (i & 3)];
            c4 += hadamard_abs(b, 4) >> 1;
        }
    for (int q = 0; q < 4; q++) {
        for (int i = 0; i < 64; i++) b[i] = res[(8 * (q >> 1) + (i >> 3)) * 16 + 8 * (q & 1) + (i & 7)];
        c8 += (hadamard_abs(b, 8) + 2) >> 2;
    }
    return c8 < c4;
}

void orc_p_frame(const orc_frame_t *f,
                 const uint8_t *cur_y, const uint8_t *cur_uv, int cp,
                 const uint8_t *ref_y, const uint8_t *ref_uv, int rfp,
                 const orc_mv_t *mv, orc_out_t *out,
                 uint8_t *rec_y, uint8_t *rec_uv, int rp)
{
    orc_p_frame_t8(f, cur_y, cur_uv, cp, ref_y, ref_uv, rfp, mv, out, rec_y, rec_uv, rp, 0, NULL);
}

void orc_p_frame_t8(const orc_frame_t *f,
                    const uint8_t *cur_y, const uint8_t *cur_uv, int cp,
                    const uint8_t *ref_y, const uint8_t *ref_uv, int rfp,
                    const orc_mv_t *mv, orc_out_t *out,
                    uint8_t *rec_y, uint8_t *rec_uv, int rp, int t8, uint8_t *t8_flags)
{
    /* A1/shaders/residual_predict.comp:417-434 (luma MC), :576-635 (chroma
     * MC), dct_transform.comp:75-98, quantize.comp:189-225 (inter f = 1/6),
     * reconstruct.comp:318-442 (P luma has no DC split, :358-363). */
    /* Macroblocks are independent (each reads the reference and writes only
     * its own outputs and reconstruction): the rows run in parallel. */
    const int qp = f->qp, qpc = orc_chroma_qp(qp);
#pragma omp parallel for schedule(dynamic, 1)
    for (int mby = 0; mby < f->mbh; mby++)
        for (int mbx = 0; mbx < f->mbw; mbx++) {
            const int mb = mby * f->mbw + mbx, X = mbx * 16, Y = mby * 16, Xc = X / 2, Yc = Y / 2;
            const int mvx = mv[mb].mvx, mvy = mv[mb].mvy;
            int res[24][16], pred[24][16], coef[24][16], lev[24][16];
            for (int py = 0; py < 16; py++)
                for (int px = 0; px < 16; px++) {
                    int blk = (py >> 2) * 4 + (px >> 2), pos = (py & 3) * 4 + (px & 3);
                    int pv = orc_interp_luma_qpel(ref_y, rfp, f->RW, f->RH, (X + px) * 4 + mvx, (Y + py) * 4 + mvy);
                    pred[blk][pos] = pv;
                    res[blk][pos] = srcY(f, cur_y, cp, X + px, Y + py) - pv;
                }
            for (int pl = 0; pl < 2; pl++)
                for (int sub = 0; sub < 4; sub++)
                    for (int pos = 0; pos < 16; pos++) {
                        int blk = 16 + 4 * pl + sub;
                        int xo = (sub & 1) * 4 + (pos & 3), yo = (sub >> 1) * 4 + (pos >> 2);
                        int pv = orc_interp_chroma(ref_uv, rfp, f->RW, f->RH, pl, (Xc + xo) * 8 + mvx, (Yc + yo) * 8 + mvy);
                        pred[blk][pos] = pv;
                        res[blk][pos] = srcC(f, cur_uv, cp, pl, Xc + xo, Yc + yo) - pv;
                    }
            /* 8x8 luma (High profile, clause 8.5.13; no counterpart in the
             * reference's encoder): t8 = 1 always, 2 by orc_t8_choose. */
            int use8 = t8 == 1;
            if (t8 == 2) {
                int r16[256];
                for (int p = 0; p < 256; p++)
                    r16[p] = res[((p >> 6) << 2) + ((p & 15) >> 2)][(((p >> 4) & 3) << 2) + (p & 3)];
                use8 = orc_t8_choose(r16);
            }
            if (t8_flags) t8_flags[mb] = (uint8_t)use8;
            if (use8) {
                int zz[64];
                zigzag8(zz);
                for (int q8 = 0; q8 < 4; q8++) {
                    const int qx = 8 * (q8 & 1), qy = 8 * (q8 >> 1);
                    int16_t r8[64], l8[64];
                    uint8_t p8[64];
                    for (int i = 0; i < 64; i++) {
                        const int xx = qx + (i & 7), yy = qy + (i >> 3);
                        const int blk = (yy >> 2) * 4 + (xx >> 2), pos = (yy & 3) * 4 + (xx & 3);
                        r8[i] = (int16_t)res[blk][pos];
                        p8[i] = (uint8_t)pred[blk][pos];
                    }
                    orc_fwd_quant8(r8, l8, qp, 0);
                    /* raster levels over the quadrant's four 16-level slots */
                    for (int i = 0; i < 64; i++) out->levels[(size_t)mb * 384 + 64 * q8 + i] = l8[i];
                    /* CAVLC codes the 8x8 block as four 4x4 blocks: block i
                     * of the quadrant (spec order) holds scan positions
                     * i, i + 4, ... (7.3.5.3.2); its nz word is their mask */
                    for (int i = 0; i < 4; i++) {
                        uint32_t m = 0;
                        for (int j = 0; j < 16; j++)
                            if (l8[zz[4 * j + i]]) m |= 1u << j;
                        const int rb = (qy / 4 + (i >> 1)) * 4 + qx / 4 + (i & 1);
                        out->nz[(size_t)mb * 24 + rb] = m;
                        out->dc[(size_t)mb * 24 + rb] = 0;
                    }
                    orc_dequant_idct8_add(l8, p8, 8, qp);
                    for (int i = 0; i < 64; i++) {
                        const int xx = qx + (i & 7), yy = qy + (i >> 3);
                        if (X + xx < f->RW && Y + yy < f->RH) rec_y[(size_t)(Y + yy) * rp + X + xx] = p8[i];
                    }
                }
            }
            for (int b = use8 ? 16 : 0; b < 24; b++) {
                int q = b < 16 ? qp : qpc;
                uint32_t nz = 0;
                orc_forward_4x4(res[b], coef[b]);
                for (int p = 0; p < 16; p++) {
                    lev[b][p] = orc_quant_ac(coef[b][p], p, q, 0);
                    out->levels[((size_t)mb * 24 + b) * 16 + p] = (int16_t)clampi(lev[b][p], -32768, 32767);
                    if (lev[b][p]) nz |= 1u << p;
                }
                out->nz[(size_t)mb * 24 + b] = nz;
                out->dc[(size_t)mb * 24 + b] = coef[b][0];
            }
            out->pred_mode[mb] = 2; /* residual_predict.comp:422 */
            for (int b = 0; b < (use8 ? 0 : 16); b++) {
                int d[16], r[16], v[16];
                for (int p = 0; p < 16; p++) d[p] = orc_dequant_ac(lev[b][p], p, qp);
                orc_inverse_4x4(d, r);
                for (int p = 0; p < 16; p++) v[p] = clip1(pred[b][p] + r[p]);
                store_rec_luma(f, rec_y, rp, X, Y, b, v);
            }
            chroma_recon(f, qpc, coef, lev, pred, rec_uv, rp, Xc, Yc);
        }
}

/* ------------------------------------------------------- I-frame chain */

/* One macroblock of the I frame (A1/shaders/intra_wavefront.comp:398-756):
 * the I16x16 decision from the reconstructed left, top and top-left
 * neighbours, the chain, and its reconstruction into rec. */
static void i_mb(const orc_frame_t *f, const uint8_t *cur_y, const uint8_t *cur_uv, int cp, orc_out_t *out,
                 uint8_t *rec_y, uint8_t *rec_uv, int rp, int mbx, int mby)
{
    const int qp = f->qp, qpc = orc_chroma_qp(qp);
    const uint32_t total = (uint32_t)(f->mbw * f->mbh);
    const int rmx = f->RW - 1, rmy = f->RH - 1, cmx = f->RW / 2 - 1, cmy = f->RH / 2 - 1;
    const int mb = mby * f->mbw + mbx, X = mbx * 16, Y = mby * 16, Xc = X / 2, Yc = Y / 2;
    const uint32_t sl = orc_slice_of((uint32_t)mb, total, (uint32_t)f->num_slices);
    const int top_exists = mby > 0, left_exists = mbx > 0;
    const int top_av = top_exists && orc_slice_of((uint32_t)(mb - f->mbw), total, (uint32_t)f->num_slices) == sl;
    const int left_av = left_exists && orc_slice_of((uint32_t)(mb - 1), total, (uint32_t)f->num_slices) == sl;
    const int plane_av = top_av && left_av &&
        (!(f->flags & ORC_INTRA_CORNER_CHECK) ||
         orc_slice_of((uint32_t)(mb - f->mbw - 1), total, (uint32_t)f->num_slices) == sl);
    int top[16], left[16], corner;
    for (int i = 0; i < 16; i++) {
        top[i] = top_exists ? rec_y[(size_t)clampi(Y - 1, 0, rmy) * rp + clampi(X + i, 0, rmx)] : 128;
        left[i] = left_exists ? rec_y[(size_t)clampi(Y + i, 0, rmy) * rp + clampi(X - 1, 0, rmx)] : 128;
    }
    corner = (top_exists && left_exists) ? rec_y[(size_t)clampi(Y - 1, 0, rmy) * rp + clampi(X - 1, 0, rmx)] : 128;
    int st = 0, sl_ = 0;
    for (int i = 0; i < 16; i++) { st += top[i]; sl_ += left[i]; }
    int dcv;
    if (top_av && left_av) dcv = (st + sl_ + 16) >> 5;
    else if (top_av) dcv = (st + 8) >> 4;
    else if (left_av) dcv = (sl_ + 8) >> 4;
    else dcv = 128;
    int pa = 0, pb = 0, pc = 0;
    if (plane_av) {
        int Hs = 0, Vs = 0;
        for (int k = 0; k < 8; k++) {
            int l = (6 - k >= 0) ? top[6 - k] : corner;
            Hs += (k + 1) * (top[8 + k] - l);
            int a = (6 - k >= 0) ? left[6 - k] : corner;
            Vs += (k + 1) * (left[8 + k] - a);
        }
        pa = 16 * (left[15] + top[15]);
        pb = (5 * Hs + 32) >> 6;
        pc = (5 * Vs + 32) >> 6;
    }
    int src[256];
    for (int y = 0; y < 16; y++)
        for (int x = 0; x < 16; x++) src[y * 16 + x] = srcY(f, cur_y, cp, X + x, Y + y);
    uint32_t sdc = 0, sv = 0, sh = 0, spl = 0;
    for (int y = 0; y < 16; y++)
        for (int x = 0; x < 16; x++) {
            int s = src[y * 16 + x];
            sdc += (uint32_t)iabs(s - dcv);
            if (top_av) sv += (uint32_t)iabs(s - top[x]);
            if (left_av) sh += (uint32_t)iabs(s - left[y]);
            if (plane_av) spl += (uint32_t)iabs(s - clip1((pa + pb * (x - 7) + pc * (y - 7) + 16) >> 5));
        }
    uint32_t best = sdc;
    int mode = 2;
    if (top_av && sv < best) { best = sv; mode = 0; }
    if (left_av && sh < best) { best = sh; mode = 1; }
    if (plane_av && spl < best) { best = spl; mode = 3; }
    out->pred_mode[mb] = (uint32_t)mode;
    out->mv[mb].mvx = out->mv[mb].mvy = 0;
    out->mv[mb].sad = out->mv[mb].pad = 0;

    int res[24][16], pred[24][16], coef[24][16], lev[24][16];
    for (int y = 0; y < 16; y++)
        for (int x = 0; x < 16; x++) {
            int pv;
            if (mode == 0) pv = top[x];
            else if (mode == 1) pv = left[y];
            else if (mode == 3) pv = clip1((pa + pb * (x - 7) + pc * (y - 7) + 16) >> 5);
            else pv = dcv;
            int blk = (y >> 2) * 4 + (x >> 2), pos = (y & 3) * 4 + (x & 3);
            pred[blk][pos] = pv;
            res[blk][pos] = src[y * 16 + x] - pv;
        }
    int dcin[16];
    for (int b = 0; b < 16; b++) {
        uint32_t nz = 0;
        orc_forward_4x4(res[b], coef[b]);
        out->dc[(size_t)mb * 24 + b] = coef[b][0];
        dcin[b] = coef[b][0];
        lev[b][0] = 0;
        out->levels[((size_t)mb * 24 + b) * 16] = 0;
        for (int p = 1; p < 16; p++) {
            lev[b][p] = orc_quant_ac(coef[b][p], p, qp, 1);
            out->levels[((size_t)mb * 24 + b) * 16 + p] = (int16_t)clampi(lev[b][p], -32768, 32767);
            if (lev[b][p]) nz |= 1u << p;
        }
        out->nz[(size_t)mb * 24 + b] = nz;
    }
    int raw[16], dl[16], fv[16];
    orc_luma_dc_hadamard_fwd(dcin, raw);
    for (int b = 0; b < 16; b++) dl[b] = orc_quantize_dc_luma(raw[b], qp);
    orc_luma_dc_hadamard_inv(dl, fv);
    for (int b = 0; b < 16; b++) {
        int d[16], r[16], v[16];
        d[0] = orc_dequant_dc_luma(fv[b], qp);
        for (int p = 1; p < 16; p++) d[p] = orc_dequant_ac(lev[b][p], p, qp);
        orc_inverse_4x4(d, r);
        for (int p = 0; p < 16; p++) v[p] = clip1(pred[b][p] + r[p]);
        store_rec_luma(f, rec_y, rp, X, Y, b, v);
    }
    /* Chroma: DC prediction from recon neighbours gated on slice
     * availability (intra_wavefront.comp:601-642). */
    for (int pl = 0; pl < 2; pl++) {
        int tu[8], lu[8];
        for (int i = 0; i < 8; i++) {
            tu[i] = top_av ? rec_uv[(size_t)clampi(Yc - 1, 0, cmy) * rp + 2 * clampi(Xc + i, 0, cmx) + pl] : 128;
            lu[i] = left_av ? rec_uv[(size_t)clampi(Yc + i, 0, cmy) * rp + 2 * clampi(Xc - 1, 0, cmx) + pl] : 128;
        }
        int t0 = tu[0] + tu[1] + tu[2] + tu[3], t1 = tu[4] + tu[5] + tu[6] + tu[7];
        int l0 = lu[0] + lu[1] + lu[2] + lu[3], l1 = lu[4] + lu[5] + lu[6] + lu[7];
        int dcp[4];
        if (top_av && left_av) dcp[0] = (t0 + l0 + 4) >> 3;
        else if (top_av) dcp[0] = (t0 + 2) >> 2;
        else if (left_av) dcp[0] = (l0 + 2) >> 2;
        else dcp[0] = 128;
        if (top_av) dcp[1] = (t1 + 2) >> 2;
        else if (left_av) dcp[1] = (l0 + 2) >> 2;
        else dcp[1] = 128;
        if (left_av) dcp[2] = (l1 + 2) >> 2;
        else if (top_av) dcp[2] = (t0 + 2) >> 2;
        else dcp[2] = 128;
        if (top_av && left_av) dcp[3] = (t1 + l1 + 4) >> 3;
        else if (top_av) dcp[3] = (t1 + 2) >> 2;
        else if (left_av) dcp[3] = (l1 + 2) >> 2;
        else dcp[3] = 128;
        for (int sub = 0; sub < 4; sub++) {
            int blk = 16 + 4 * pl + sub;
            uint32_t nz = 0;
            for (int pos = 0; pos < 16; pos++) {
                int xo = (sub & 1) * 4 + (pos & 3), yo = (sub >> 1) * 4 + (pos >> 2);
                pred[blk][pos] = dcp[sub];
                res[blk][pos] = srcC(f, cur_uv, cp, pl, Xc + xo, Yc + yo) - dcp[sub];
            }
            orc_forward_4x4(res[blk], coef[blk]);
            out->dc[(size_t)mb * 24 + blk] = coef[blk][0];
            lev[blk][0] = 0;
            out->levels[((size_t)mb * 24 + blk) * 16] = 0;
            for (int p = 1; p < 16; p++) {
                lev[blk][p] = orc_quant_ac(coef[blk][p], p, qpc, 1);
                out->levels[((size_t)mb * 24 + blk) * 16 + p] = (int16_t)clampi(lev[blk][p], -32768, 32767);
                if (lev[blk][p]) nz |= 1u << p;
            }
            out->nz[(size_t)mb * 24 + blk] = nz;
        }
    }
    chroma_recon(f, qpc, coef, lev, pred, rec_uv, rp, Xc, Yc);
}

void orc_i_frame(const orc_frame_t *f,
                 const uint8_t *cur_y, const uint8_t *cur_uv, int cp,
                 orc_out_t *out, uint8_t *rec_y, uint8_t *rec_uv, int rp)
{
    /* Raster order visits every macroblock after its left, top and top-left
     * neighbours, which is all the diagonal schedule
     * (A1/src/gpu_compute.c:3238-3249) guarantees. */
    for (int mby = 0; mby < f->mbh; mby++)
        for (int mbx = 0; mbx < f->mbw; mbx++) i_mb(f, cur_y, cur_uv, cp, out, rec_y, rec_uv, rp, mbx, mby);
}

int orc_i_frame_steps(const orc_frame_t *f,
                      const uint8_t *cur_y, const uint8_t *cur_uv, int cp,
                      orc_out_t *out, uint8_t *rec_y, uint8_t *rec_uv, int rp,
                      const int32_t *order, int n)
{
    /* The same macroblocks in the caller's order (raster indices). */
    for (int i = 0; i < n; i++) {
        if (order[i] < 0 || order[i] >= f->mbw * f->mbh) return -1;
        i_mb(f, cur_y, cur_uv, cp, out, rec_y, rec_uv, rp, order[i] % f->mbw, order[i] / f->mbw);
    }
    return 0;
}

/* --------------------------------------------------------------- deblock */

/* Table 8-16/8-17 values; the same numbers the reference's decoder tables
 * carry (A1/src/h264_dec_tables.c) and its shader restates
 * (A1/shaders/deblock_filter.comp:185-210). */
static const uint8_t ALPHA[52] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 4, 4, 5, 6, 7, 8, 9, 10, 12, 13,
                                  15, 17, 20, 22, 25, 28, 32, 36, 40, 45, 50, 56, 63, 71, 80, 90, 101, 113, 127,
                                  144, 162, 182, 203, 226, 255, 255};
static const uint8_t BETA[52] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4,
                                 6, 6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13, 14, 14, 15, 15, 16, 16,
                                 17, 17, 18, 18};
static const uint8_t TC0[52][3] = {
    {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0},
    {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 1},
    {0, 0, 1}, {0, 0, 1}, {0, 0, 1}, {0, 1, 1}, {0, 1, 1}, {1, 1, 1}, {1, 1, 1}, {1, 1, 1}, {1, 1, 1},
    {1, 1, 2}, {1, 1, 2}, {1, 1, 2}, {1, 1, 2}, {1, 2, 3}, {1, 2, 3}, {2, 2, 3}, {2, 2, 4}, {2, 3, 4},
    {2, 3, 4}, {3, 3, 5}, {3, 4, 6}, {3, 4, 6}, {4, 5, 7}, {4, 5, 8}, {4, 6, 9}, {5, 7, 10}, {6, 8, 11},
    {6, 8, 13}, {7, 10, 14}, {8, 11, 16}, {9, 12, 18}, {10, 13, 20}, {11, 15, 23}, {13, 17, 25}};

static void filt_luma(uint8_t *q, int d, int bs, int alpha, int beta, int tc0)
{
    /* Clause 8.7.2.3 / 8.7.2.4 (A1/src/h264_deblock.c:31-88). */
    int p0 = q[-d], p1 = q[-2 * d], p2 = q[-3 * d], q0 = q[0], q1 = q[d], q2 = q[2 * d];
    if (iabs(p0 - q0) >= alpha || iabs(p1 - p0) >= beta || iabs(q1 - q0) >= beta) return;
    int ap = iabs(p2 - p0) < beta, aq = iabs(q2 - q0) < beta;
    if (bs == 4) {
        int p3 = q[-4 * d], q3 = q[3 * d];
        int small = iabs(p0 - q0) < ((alpha >> 2) + 2);
        if (ap && small) {
            q[-d] = (uint8_t)((p2 + 2 * p1 + 2 * p0 + 2 * q0 + q1 + 4) >> 3);
            q[-2 * d] = (uint8_t)((p2 + p1 + p0 + q0 + 2) >> 2);
            q[-3 * d] = (uint8_t)((2 * p3 + 3 * p2 + p1 + p0 + q0 + 4) >> 3);
        } else {
            q[-d] = (uint8_t)((2 * p1 + p0 + q1 + 2) >> 2);
        }
        if (aq && small) {
            q[0] = (uint8_t)((q2 + 2 * q1 + 2 * q0 + 2 * p0 + p1 + 4) >> 3);
            q[d] = (uint8_t)((q2 + q1 + q0 + p0 + 2) >> 2);
            q[2 * d] = (uint8_t)((2 * q3 + 3 * q2 + q1 + q0 + p0 + 4) >> 3);
        } else {
            q[0] = (uint8_t)((2 * q1 + q0 + p1 + 2) >> 2);
        }
        return;
    }
    int tc = tc0 + ap + aq;
    int delta = clampi(((q0 - p0) * 4 + (p1 - q1) + 4) >> 3, -tc, tc);
    if (ap) q[-2 * d] = (uint8_t)(p1 + clampi((p2 + ((p0 + q0 + 1) >> 1) - (p1 << 1)) >> 1, -tc0, tc0));
    if (aq) q[d] = (uint8_t)(q1 + clampi((q2 + ((p0 + q0 + 1) >> 1) - (q1 << 1)) >> 1, -tc0, tc0));
    q[-d] = (uint8_t)clip1(p0 + delta);
    q[0] = (uint8_t)clip1(q0 - delta);
}

static void filt_chroma(uint8_t *q, int d, int bs, int alpha, int beta, int tc0)
{
    /* A1/src/h264_deblock.c:92-119: p1/q1 never written. */
    int p0 = q[-d], p1 = q[-2 * d], q0 = q[0], q1 = q[d];
    if (iabs(p0 - q0) >= alpha || iabs(p1 - p0) >= beta || iabs(q1 - q0) >= beta) return;
    if (bs == 4) {
        q[-d] = (uint8_t)((2 * p1 + p0 + q1 + 2) >> 2);
        q[0] = (uint8_t)((2 * q1 + q0 + p1 + 2) >> 2);
        return;
    }
    int tc = tc0 + 1;
    int delta = clampi(((q0 - p0) * 4 + (p1 - q1) + 4) >> 3, -tc, tc);
    q[-d] = (uint8_t)clip1(p0 + delta);
    q[0] = (uint8_t)clip1(q0 - delta);
}

/* Whether the transform block holding 4x4 block b (raster) of macroblock mb
 * has a coefficient: the 4x4 block, or with the 8x8 transform the 8x8 block
 * whose four 4x4 blocks are ORed (A1/src/h264_deblock.c:119-137). */
static int has_coef(const uint32_t *nz, const uint8_t *t8, int mb, int b)
{
    if (!t8 || !t8[mb]) return (nz[(size_t)mb * 24 + b] & 0xffff) != 0;
    const int c = b & 10;
    return ((nz[(size_t)mb * 24 + c] | nz[(size_t)mb * 24 + c + 1] | nz[(size_t)mb * 24 + c + 4] |
             nz[(size_t)mb * 24 + c + 5]) & 0xffff) != 0;
}

static int bs_of(int is_intra, int mb_edge, const uint32_t *nz, const uint8_t *t8, const orc_mv_t *mv, int mbp,
                 int bp, int mbq, int bq)
{
    /* Clause 8.7.2.1 for this encoder's macroblock kinds
     * (A1/src/h264_deblock.c:139-210). */
    if (is_intra) return mb_edge ? 4 : 3;
    if (has_coef(nz, t8, mbp, bp) || has_coef(nz, t8, mbq, bq)) return 2;
    if (iabs(mv[mbp].mvx - mv[mbq].mvx) >= 4 || iabs(mv[mbp].mvy - mv[mbq].mvy) >= 4) return 1;
    return 0;
}

/* One filtering step of macroblock mb: its vertical edges (dir 0, left to
 * right) or its horizontal edges (dir 1, top to bottom), luma and chroma
 * (A1/src/h264_deblock.c:263-347). Uniform QP so qPav = QP. */
static void deblock_step(int mbw, int qp, int is_intra, const uint32_t *nz, const uint8_t *t8, const orc_mv_t *mv,
                         uint8_t *ry, uint8_t *ruv, int rp, int mb, int dir)
{
    const int qpc = orc_chroma_qp(qp);
    const int a = ALPHA[qp], b = BETA[qp], ac = ALPHA[qpc], bc = BETA[qpc];
    const int my = mb / mbw, mx = mb % mbw;
    uint8_t *py = ry + (size_t)my * 16 * rp + mx * 16;
    uint8_t *pc = ruv + (size_t)my * 8 * rp + mx * 16;
    for (int e = 0; e < 4; e++) {
        if (e == 0 && (dir == 0 ? mx == 0 : my == 0)) continue;
        /* 8x8 transform: no luma edge inside the 8x8 blocks (h264_deblock.c:294,324) */
        if ((e & 1) && t8 && t8[mb]) continue;
        int mbp = e ? mb : (dir == 0 ? mb - 1 : mb - mbw);
        for (int k = 0; k < 4; k++) {
            int bq = dir == 0 ? k * 4 + e : e * 4 + k;
            int bp = e ? (dir == 0 ? bq - 1 : bq - 4) : (dir == 0 ? k * 4 + 3 : 12 + k);
            int bs = bs_of(is_intra, e == 0, nz, t8, mv, mbp, bp, mb, bq);
            if (!bs) continue;
            if (a && b) {
                int tc0 = bs < 4 ? TC0[qp][bs - 1] : 0;
                for (int i = 0; i < 4; i++) {
                    uint8_t *q = dir == 0 ? py + (size_t)(k * 4 + i) * rp + e * 4
                                          : py + (size_t)(e * 4) * rp + k * 4 + i;
                    filt_luma(q, dir == 0 ? 1 : rp, bs, a, b, tc0);
                }
            }
            if ((e == 0 || e == 2) && ac && bc) {
                int tc0 = bs < 4 ? TC0[qpc][bs - 1] : 0;
                for (int pl = 0; pl < 2; pl++)
                    for (int i = 0; i < 2; i++) {
                        uint8_t *q = dir == 0 ? pc + (size_t)(k * 2 + i) * rp + 2 * (e * 2) + pl
                                              : pc + (size_t)(e * 2) * rp + 2 * (k * 2 + i) + pl;
                        filt_chroma(q, dir == 0 ? 2 : rp, bs, ac, bc, tc0);
                    }
            }
        }
    }
}

void orc_deblock_frame_t8(int mbw, int mbh, int qp, int is_intra, const uint32_t *nz, const uint8_t *t8,
                          const orc_mv_t *mv, uint8_t *ry, uint8_t *ruv, int rp)
{
    for (int mb = 0; mb < mbw * mbh; mb++) {
        deblock_step(mbw, qp, is_intra, nz, t8, mv, ry, ruv, rp, mb, 0);
        deblock_step(mbw, qp, is_intra, nz, t8, mv, ry, ruv, rp, mb, 1);
    }
}

void orc_deblock_frame(int mbw, int mbh, int qp, int is_intra, const uint32_t *nz, const orc_mv_t *mv,
                       uint8_t *ry, uint8_t *ruv, int rp)
{
    /* Macroblocks in raster order; per macroblock the vertical edges left
     * to right, then the horizontal edges top to bottom (clause 8.7,
     * A1/src/h264_deblock.c:263-347). */
    for (int mb = 0; mb < mbw * mbh; mb++) {
        deblock_step(mbw, qp, is_intra, nz, NULL, mv, ry, ruv, rp, mb, 0);
        deblock_step(mbw, qp, is_intra, nz, NULL, mv, ry, ruv, rp, mb, 1);
    }
}

int orc_deblock_steps(int mbw, int mbh, int qp, int is_intra, const uint32_t *nz, const orc_mv_t *mv, uint8_t *ry,
                      uint8_t *ruv, int rp, const int32_t *steps, int nsteps)
{
    /* The same steps in the caller's order: steps[i] = 2 * mb + dir. */
    for (int i = 0; i < nsteps; i++) {
        const int mb = steps[i] >> 1, dir = steps[i] & 1;
        if (steps[i] < 0 || mb >= mbw * mbh) return -1;
        deblock_step(mbw, qp, is_intra, nz, NULL, mv, ry, ruv, rp, mb, dir);
    }
    return 0;
}

/* ------------------------------------------------------------ one frame */

void orc_encode_frame(const orc_frame_t *f, const orc_me_params_t *p, int is_intra, int deblock,
                      const uint8_t *cur_y, const uint8_t *cur_uv, int cp,
                      const uint8_t *ref_y, const uint8_t *ref_uv, int rfp,
                      orc_out_t *out, uint8_t *rec_y, uint8_t *rec_uv, int rp)
{
    /* Stage order of A1/src/gpu_compute.c:2922-3365: ME, then the P chain or
     * the intra wavefront, then deblocking. */
    if (is_intra) {
        orc_i_frame(f, cur_y, cur_uv, cp, out, rec_y, rec_uv, rp);
    } else {
        orc_me_frame(f, p, cur_y, cp, ref_y, rfp, out->mv);
        orc_p_frame(f, cur_y, cur_uv, cp, ref_y, ref_uv, rfp, out->mv, out, rec_y, rec_uv, rp);
    }
    if (deblock) orc_deblock_frame(f->mbw, f->mbh, f->qp, is_intra, out->nz, out->mv, rec_y, rec_uv, rp);
}

/* Threads the parallel loops above may use (OpenMP); 0 leaves the default. */
void orc_set_threads(int n)
{
    if (n > 0) omp_set_num_threads(n);
}

/* ------------------------------------------------ 8x8 transform (High) */

/* Forward 8x8 integer transform, one dimension: the published core transform
 * whose inverse is clause 8.5.13.2 (the encoder side of
 * transform_size_8x8_flag; the reference's encoder has none, its decoder
 * the inverse, A1/src/h264_recon.c:158-189). */
static void fwd8_1d(int32_t *d, int st)
{
    const int32_t s0 = d[0], s1 = d[st], s2 = d[2 * st], s3 = d[3 * st];
    const int32_t s4 = d[4 * st], s5 = d[5 * st], s6 = d[6 * st], s7 = d[7 * st];
    const int32_t a0 = s0 + s7, a1 = s1 + s6, a2 = s2 + s5, a3 = s3 + s4;
    const int32_t b0 = a0 + a3, b1 = a1 + a2, b2 = a0 - a3, b3 = a1 - a2;
    const int32_t a4 = s0 - s7, a5 = s1 - s6, a6 = s2 - s5, a7 = s3 - s4;
    const int32_t b4 = a5 + a6 + ((a4 >> 1) + a4);
    const int32_t b5 = a4 - a7 - ((a6 >> 1) + a6);
    const int32_t b6 = a4 + a7 - ((a5 >> 1) + a5);
    const int32_t b7 = a5 - a6 + ((a7 >> 1) + a7);
    d[0] = b0 + b1;
    d[4 * st] = b0 - b1;
    d[2 * st] = b2 + (b3 >> 1);
    d[6 * st] = (b2 >> 1) - b3;
    d[st] = b4 + (b7 >> 2);
    d[7 * st] = (b4 >> 2) - b7;
    d[3 * st] = b5 + (b6 >> 2);
    d[5 * st] = b6 - (b5 >> 2);
}

/* Position class of raster position p of an 8x8 block (the six classes of
 * normAdjust8x8, clause 8.5.9 (8-318)). */
static int cls8(int p)
{
    const int i = p >> 3, j = p & 7;
    if ((i & 3) == 0 && (j & 3) == 0) return 0;
    if ((i & 1) && (j & 1)) return 1;
    if ((i & 3) == 2 && (j & 3) == 2) return 2;
    if (((i & 3) == 0 && (j & 1)) || ((i & 1) && (j & 3) == 0)) return 3;
    if (((i & 3) == 0 && (j & 3) == 2) || ((i & 3) == 2 && (j & 3) == 0)) return 4;
    return 5;
}

/* normAdjust8x8 v[qp % 6][class] (8-318), the decoder's dequantisation
 * factor / 16 under flat scaling lists, and the encoder's quantisation
 * multipliers MF8 = round(2^22 / (v * norm)) of the same classes. */
static const int V8[6][6] = {{20, 18, 32, 19, 25, 24}, {22, 19, 35, 21, 28, 26}, {26, 23, 42, 24, 33, 31},
                             {28, 25, 45, 26, 35, 33}, {32, 28, 51, 30, 40, 38}, {36, 32, 58, 34, 46, 43}};
static const int MF8[6][6] = {{13107, 11428, 20972, 12222, 16777, 15481}, {11916, 10826, 19174, 11058, 14980, 14290},
                              {10082, 8943, 15978, 9675, 12710, 11985},   {9362, 8228, 14913, 8931, 11984, 11259},
                              {8192, 7346, 13159, 7740, 10486, 9777},     {7282, 6428, 11570, 6830, 9118, 8640}};

void orc_fwd_quant8(const int16_t res[64], int16_t lev[64], int qp, int intra)
{
    int32_t t[64];
    for (int n = 0; n < 64; n++) t[n] = res[n];
    for (int r = 0; r < 8; r++) fwd8_1d(t + 8 * r, 1);
    for (int c = 0; c < 8; c++) fwd8_1d(t + c, 8);
    const int per = qp / 6, rem = qp % 6, sh = 16 + per;
    const int64_t f = ((int64_t)1 << sh) / (intra ? 3 : 6);
    for (int n = 0; n < 64; n++) {
        const int64_t a = t[n] < 0 ? -(int64_t)t[n] : t[n];
        const int64_t l = (a * MF8[rem][cls8(n)] + f) >> sh;
        lev[n] = (int16_t)(t[n] < 0 ? -l : l);
    }
}

/* Scaling (8.5.13.1, flat lists), the inverse transform (8.5.13.2) and the
 * add with clipping, onto the 8x8 prediction at dst. */
void orc_dequant_idct8_add(const int16_t lev[64], uint8_t *dst, int stride, int qp)
{
    int32_t t[64];
    const int per = qp / 6, rem = qp % 6;
    for (int n = 0; n < 64; n++) {
        const int32_t ls = 16 * V8[rem][cls8(n)];
        t[n] = per >= 6 ? (lev[n] * ls) << (per - 6) : (lev[n] * ls + (1 << (5 - per))) >> (6 - per);
    }
    for (int pass = 0; pass < 2; pass++)
        for (int k = 0; k < 8; k++) {
            int32_t *d = pass == 0 ? t + 8 * k : t + k;
            const int st = pass == 0 ? 1 : 8;
            const int32_t a0 = d[0] + d[4 * st], a2 = d[0] - d[4 * st];
            const int32_t a4 = (d[2 * st] >> 1) - d[6 * st], a6 = (d[6 * st] >> 1) + d[2 * st];
            const int32_t b0 = a0 + a6, b2 = a2 + a4, b4 = a2 - a4, b6 = a0 - a6;
            const int32_t a1 = -d[3 * st] + d[5 * st] - d[7 * st] - (d[7 * st] >> 1);
            const int32_t a3 = d[st] + d[7 * st] - d[3 * st] - (d[3 * st] >> 1);
            const int32_t a5 = -d[st] + d[7 * st] + d[5 * st] + (d[5 * st] >> 1);
            const int32_t a7 = d[3 * st] + d[5 * st] + d[st] + (d[st] >> 1);
            const int32_t b1 = (a7 >> 2) + a1, b3 = a3 + (a5 >> 2), b5 = (a3 >> 2) - a5, b7 = a7 - (a1 >> 2);
            d[0] = b0 + b7;
            d[7 * st] = b0 - b7;
            d[st] = b2 + b5;
            d[6 * st] = b2 - b5;
            d[2 * st] = b4 + b3;
            d[5 * st] = b4 - b3;
            d[3 * st] = b6 + b1;
            d[4 * st] = b6 - b1;
        }
    for (int y = 0; y < 8; y++)
        for (int x = 0; x < 8; x++) {
            const int v = dst[y * stride + x] + ((t[y * 8 + x] + 32) >> 6);
            dst[y * stride + x] = (uint8_t)(v < 0 ? 0 : (v > 255 ? 255 : v));
        }
}
