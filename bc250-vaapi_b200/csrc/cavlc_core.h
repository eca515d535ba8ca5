// cavlc_core.h - CAVLC (H.264 clause 9.2) for the macroblock kinds this
// encoder codes: the code tables and the writers of one residual block and
// of the I16x16 / P16x16 macroblock headers, as used by the GPU entropy
// coder (cavlc.cu, one thread per macroblock). Written for device and host
// compilers alike (`CAVLC_HD`): cavlc.cu instantiates it for the GPU, and the
// test build compiles the same file on the host to check it against the
// reference's writer without a GPU.
//
// The bits are those of the reference's host writer (A1/src/cavlc.c:353-801
// and the macroblock headers at :75-160): the same tables (the spec's), the
// same level escape arithmetic (cavlc_write_one_level, :429-480), the same
// trailing-ones rule and total_zeros / run_before tables.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define CAVLC_HD __host__ __device__ __forceinline__
#else
#define CAVLC_HD static inline
#endif

namespace b200cavlc {

// ---- tables ------------------------------------------------------------------
// Table 9-5 coeff_token, lengths and codes indexed
// [nC class][TotalCoeff * 4 + TrailingOnes]; classes 0 <= nC < 2, 2 <= nC < 4,
// 4 <= nC < 8, 8 <= nC (a 6-bit fixed-length code), then nC = -1 (chroma DC,
// TotalCoeff <= 4). Entries with TrailingOnes > TotalCoeff are unused (0).
#define B200_CAVLC_COEFF_TOKEN_LEN                                                                              \
  {{1, 0, 0, 0, 6, 2, 0, 0, 8, 6, 3, 0, 9, 8, 7, 5, 10, 9, 8, 6, 11, 10, 9, 7, 13, 11, 10, 8, 13, 13, 11, 9,    \
    13, 13, 13, 10, 14, 14, 13, 11, 14, 14, 14, 13, 15, 15, 14, 14, 15, 15, 15, 14, 16, 15, 15, 15, 16, 16, 16, \
    15, 16, 16, 16, 16, 16, 16, 16, 16},                                                                       \
   {2, 0, 0, 0, 6, 2, 0, 0, 6, 5, 3, 0, 7, 6, 6, 4, 8, 6, 6, 4, 8, 7, 7, 5, 9, 8, 8, 6, 11, 9, 9, 6,            \
    11, 11, 11, 7, 12, 11, 11, 9, 12, 12, 12, 11, 12, 12, 12, 11, 13, 13, 13, 12, 13, 13, 13, 13, 13, 14, 13,   \
    13, 14, 14, 14, 13, 14, 14, 14, 14},                                                                       \
   {4, 0, 0, 0, 6, 4, 0, 0, 6, 5, 4, 0, 6, 5, 5, 4, 7, 5, 5, 4, 7, 5, 5, 4, 7, 6, 6, 4, 7, 6, 6, 4,             \
    8, 7, 7, 5, 8, 8, 7, 6, 9, 8, 8, 7, 9, 9, 8, 8, 9, 9, 9, 8, 10, 9, 9, 9, 10, 10, 10, 10, 10, 10, 10,        \
    10, 10, 10, 10, 10},                                                                                       \
   {6, 0, 0, 0, 6, 6, 0, 0, 6, 6, 6, 0, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6,             \
    6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6}, \
   {2, 0, 0, 0, 6, 1, 0, 0, 6, 6, 3, 0, 6, 7, 7, 6, 6, 8, 8, 7, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,            \
    0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}}
#define B200_CAVLC_COEFF_TOKEN_CODE                                                                             \
  {{1, 0, 0, 0, 5, 1, 0, 0, 7, 4, 1, 0, 7, 6, 5, 3, 7, 6, 5, 3, 7, 6, 5, 4, 15, 6, 5, 4, 11, 14, 5, 4,         \
    8, 10, 13, 4, 15, 14, 9, 4, 11, 10, 13, 12, 15, 14, 9, 12, 11, 10, 13, 8, 15, 1, 9, 12, 11, 14, 13, 8, 7,   \
    10, 9, 12, 4, 6, 5, 8},                                                                                    \
   {3, 0, 0, 0, 11, 2, 0, 0, 7, 7, 3, 0, 7, 10, 9, 5, 7, 6, 5, 4, 4, 6, 5, 6, 7, 6, 5, 8, 15, 6, 5, 4,          \
    11, 14, 13, 4, 15, 10, 9, 4, 11, 14, 13, 12, 8, 10, 9, 8, 15, 14, 13, 12, 11, 10, 9, 12, 7, 11, 6, 8, 9, 8, \
    10, 1, 7, 6, 5, 4},                                                                                        \
   {15, 0, 0, 0, 15, 14, 0, 0, 11, 15, 13, 0, 8, 12, 14, 12, 15, 10, 11, 11, 11, 8, 9, 10, 9, 14, 13, 9,        \
    8, 10, 9, 8, 15, 14, 13, 13, 11, 14, 10, 12, 15, 10, 13, 12, 11, 14, 9, 12, 8, 10, 13, 8, 13, 7, 9, 12, 9,  \
    12, 11, 10, 5, 8, 7, 6, 1, 4, 3, 2},                                                                       \
   {3, 0, 0, 0, 0, 1, 0, 0, 4, 5, 6, 0, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24, 25,  \
    26, 27, 28, 29, 30, 31, 32, 33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43, 44, 45, 46, 47, 48, 49, 50, 51, 52, \
    53, 54, 55, 56, 57, 58, 59, 60, 61, 62, 63},                                                               \
   {1, 0, 0, 0, 7, 1, 0, 0, 4, 6, 1, 0, 3, 3, 2, 5, 2, 3, 2, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,             \
    0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}}

// Tables 9-7 / 9-8 total_zeros for 4x4 blocks ([TotalCoeff - 1][total_zeros])
// and Table 9-9 (a) for chroma DC ([TotalCoeff - 1][total_zeros]).
#define B200_CAVLC_TOTAL_ZEROS_LEN                                                                                \
  {{1, 3, 3, 4, 4, 5, 5, 6, 6, 7, 7, 8, 8, 9, 9, 9}, {3, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 6, 6, 6, 6, 0},          \
   {4, 3, 3, 3, 4, 4, 3, 3, 4, 5, 5, 6, 5, 6, 0, 0}, {5, 3, 4, 4, 3, 3, 3, 4, 3, 4, 5, 5, 5, 0, 0, 0},           \
   {4, 4, 4, 3, 3, 3, 3, 3, 4, 5, 4, 5, 0, 0, 0, 0}, {6, 5, 3, 3, 3, 3, 3, 3, 4, 3, 6, 0, 0, 0, 0, 0},           \
   {6, 5, 3, 3, 3, 2, 3, 4, 3, 6, 0, 0, 0, 0, 0, 0}, {6, 4, 5, 3, 2, 2, 3, 3, 6, 0, 0, 0, 0, 0, 0, 0},           \
   {6, 6, 4, 2, 2, 3, 2, 5, 0, 0, 0, 0, 0, 0, 0, 0}, {5, 5, 3, 2, 2, 2, 4, 0, 0, 0, 0, 0, 0, 0, 0, 0},           \
   {4, 4, 3, 3, 1, 3, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}, {4, 4, 2, 1, 3, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},           \
   {3, 3, 1, 2, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}, {2, 2, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},           \
   {1, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}}
#define B200_CAVLC_TOTAL_ZEROS_CODE                                                                               \
  {{1, 3, 2, 3, 2, 3, 2, 3, 2, 3, 2, 3, 2, 3, 2, 1}, {7, 6, 5, 4, 3, 5, 4, 3, 2, 3, 2, 3, 2, 1, 0, 0},          \
   {5, 7, 6, 5, 4, 3, 4, 3, 2, 3, 2, 1, 1, 0, 0, 0}, {3, 7, 5, 4, 6, 5, 4, 3, 3, 2, 2, 1, 0, 0, 0, 0},           \
   {5, 4, 3, 7, 6, 5, 4, 3, 2, 1, 1, 0, 0, 0, 0, 0}, {1, 1, 7, 6, 5, 4, 3, 2, 1, 1, 0, 0, 0, 0, 0, 0},           \
   {1, 1, 5, 4, 3, 3, 2, 1, 1, 0, 0, 0, 0, 0, 0, 0}, {1, 1, 1, 3, 3, 2, 2, 1, 0, 0, 0, 0, 0, 0, 0, 0},           \
   {1, 0, 1, 3, 2, 1, 1, 1, 0, 0, 0, 0, 0, 0, 0, 0}, {1, 0, 1, 3, 2, 1, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0},           \
   {0, 1, 1, 2, 1, 3, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}, {0, 1, 1, 1, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},           \
   {0, 1, 1, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}, {0, 1, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},           \
   {0, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}}
#define B200_CAVLC_CDC_TOTAL_ZEROS_LEN {{1, 2, 3, 3}, {1, 2, 2, 0}, {1, 1, 0, 0}}
#define B200_CAVLC_CDC_TOTAL_ZEROS_CODE {{1, 1, 1, 0}, {1, 1, 0, 0}, {1, 0, 0, 0}}
// Table 9-10 run_before ([min(zerosLeft, 7) - 1][run_before]).
#define B200_CAVLC_RUN_LEN                                                                                        \
  {{1, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}, {1, 2, 2, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},          \
   {2, 2, 2, 2, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}, {2, 2, 2, 3, 3, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},           \
   {2, 2, 3, 3, 3, 3, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}, {2, 3, 3, 3, 3, 3, 3, 0, 0, 0, 0, 0, 0, 0, 0, 0},           \
   {3, 3, 3, 3, 3, 3, 3, 4, 5, 6, 7, 8, 9, 10, 11, 0}}
#define B200_CAVLC_RUN_CODE                                                                                       \
  {{1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}, {1, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},          \
   {3, 2, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}, {3, 2, 1, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},           \
   {3, 2, 3, 2, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}, {3, 0, 1, 3, 2, 5, 4, 0, 0, 0, 0, 0, 0, 0, 0, 0},           \
   {7, 6, 5, 4, 3, 2, 1, 1, 1, 1, 1, 1, 1, 1, 1, 0}}
// Table 9-4 me(v), inter prediction, chroma 4:2:0: codeNum of coded_block_pattern.
#define B200_CAVLC_INTER_CBP_CODE                                                                                \
  {0,  2,  3,  7,  4,  8,  17, 13, 5,  18, 9,  14, 10, 15, 16, 11, 1,  32, 33, 36, 34, 37, 44, 40,                \
   35, 45, 38, 41, 39, 42, 43, 19, 6,  24, 25, 20, 26, 21, 46, 28, 27, 47, 22, 29, 23, 30, 31, 12}
// Frame zig-zag scan of a 4x4 block (raster positions, Table 8-13).
#define B200_CAVLC_ZIGZAG {0, 1, 4, 8, 5, 2, 3, 6, 9, 12, 13, 10, 7, 11, 14, 15}

// Table storage: __constant__ for the device (cavlc.cu), static const for a
// host build; TAB(x) names the right one.
#if defined(__CUDA_ARCH__)
#define B200_CAVLC_TAB(x) d_##x
#else
#define B200_CAVLC_TAB(x) h_##x
#endif
#define B200_CAVLC_TABLES(Q)                                                     \
  Q uint8_t B200_CAVLC_NAME(ct_len)[5][68] = B200_CAVLC_COEFF_TOKEN_LEN;        \
  Q uint8_t B200_CAVLC_NAME(ct_code)[5][68] = B200_CAVLC_COEFF_TOKEN_CODE;      \
  Q uint8_t B200_CAVLC_NAME(tz_len)[15][16] = B200_CAVLC_TOTAL_ZEROS_LEN;       \
  Q uint8_t B200_CAVLC_NAME(tz_code)[15][16] = B200_CAVLC_TOTAL_ZEROS_CODE;     \
  Q uint8_t B200_CAVLC_NAME(cdtz_len)[3][4] = B200_CAVLC_CDC_TOTAL_ZEROS_LEN;   \
  Q uint8_t B200_CAVLC_NAME(cdtz_code)[3][4] = B200_CAVLC_CDC_TOTAL_ZEROS_CODE; \
  Q uint8_t B200_CAVLC_NAME(run_len)[7][16] = B200_CAVLC_RUN_LEN;               \
  Q uint8_t B200_CAVLC_NAME(run_code)[7][16] = B200_CAVLC_RUN_CODE;             \
  Q uint8_t B200_CAVLC_NAME(cbp_code)[48] = B200_CAVLC_INTER_CBP_CODE;          \
  Q uint8_t B200_CAVLC_NAME(zigzag)[16] = B200_CAVLC_ZIGZAG;

#define B200_CAVLC_NAME(x) h_##x
B200_CAVLC_TABLES(static const)
#undef B200_CAVLC_NAME
#if defined(__CUDACC__)
// global memory (not __constant__): lanes index the tables at different
// positions, which the constant cache would serialise
#define B200_CAVLC_NAME(x) d_##x
B200_CAVLC_TABLES(static __device__)
#undef B200_CAVLC_NAME
#endif

// ---- bit writer ----------------------------------------------------------------
// MSB first into 32-bit words (word k holds stream bits 32k .. 32k+31, the
// first in bit 31). `cur` holds the nf < 32 pending bits, right-aligned.
struct BitW {
  uint32_t* w;
  uint32_t cap_words, nw, cur, pos;
  int nf;
  bool over;
};

CAVLC_HD void bw_init(BitW& b, uint32_t* words, uint32_t cap_words) {
  b.w = words;
  b.cap_words = cap_words;
  b.nw = 0;
  b.cur = 0;
  b.pos = 0;
  b.nf = 0;
  b.over = false;
}

// n <= 32 bits of v (its low n bits).
CAVLC_HD void put(BitW& b, int n, uint32_t v) {
  if (n <= 0) return;
  if (n < 32) v &= (1u << n) - 1u;
  const uint64_t t = ((uint64_t)b.cur << n) | v;
  int nf = b.nf + n;
  if (nf >= 32) {
    nf -= 32;
    if (b.nw < b.cap_words) b.w[b.nw] = (uint32_t)(t >> nf);
    else b.over = true;
    ++b.nw;
    b.cur = nf ? (uint32_t)(t & ((1ull << nf) - 1ull)) : 0u;
  } else {
    b.cur = (uint32_t)t;
  }
  b.nf = nf;
  b.pos += (uint32_t)n;
}

CAVLC_HD void put_zeros(BitW& b, int n) {
  while (n > 32) {
    put(b, 32, 0u);
    n -= 32;
  }
  put(b, n, 0u);
}

// The pending bits as the last (partial) word; call once at the end.
CAVLC_HD void bw_flush(BitW& b) {
  if (b.nf > 0) {
    if (b.nw < b.cap_words) b.w[b.nw] = b.cur << (32 - b.nf);
    else b.over = true;
    ++b.nw;
    b.cur = 0;
    b.nf = 0;
  }
}

CAVLC_HD int ilog2(uint32_t v) {  // floor(log2(v)), v > 0
  int r = 0;
  while (v >>= 1) ++r;
  return r;
}

// Exp-Golomb ue(v) (clause 9.1): floor(log2(v + 1)) zeros, then v + 1.
CAVLC_HD void put_ue(BitW& b, uint32_t v) {
  const uint64_t c = (uint64_t)v + 1u;
  const int l = c >> 32 ? 32 : ilog2((uint32_t)c);
  put_zeros(b, l);
  if (l + 1 > 32) {
    put(b, 1, (uint32_t)(c >> 32));
    put(b, 32, (uint32_t)c);
  } else {
    put(b, l + 1, (uint32_t)c);
  }
}
CAVLC_HD int ue_bits(uint32_t v) { return 2 * ilog2(v + 1u) + 1; }

CAVLC_HD void put_se(BitW& b, int v) { put_ue(b, v > 0 ? (uint32_t)(2 * v - 1) : (uint32_t)(-2 * (int64_t)v)); }

// ---- residual block (clause 9.2) -------------------------------------------------
// One level (level_prefix / level_suffix, 9.2.2.1) with the reference's
// escape arithmetic for level_prefix >= 15 (cavlc.c:429-480); returns the
// next suffixLength.
CAVLC_HD int put_level(BitW& b, int level, bool first, bool t1_lt3, int sl) {
  int code = level > 0 ? 2 * level - 2 : -2 * level - 1;
  if (first && t1_lt3) code -= 2;
  if (sl == 0) {
    if (code < 14) {
      put_zeros(b, code);
      put(b, 1, 1u);
    } else if (code < 30) {
      put_zeros(b, 14);
      put(b, 1, 1u);
      put(b, 4, (uint32_t)(code - 14));
    } else {
      const uint32_t total = (uint32_t)code + 4066u;
      const int ss = ilog2(total);
      put_zeros(b, ss + 3);
      put(b, 1, 1u);
      put(b, ss, total - (1u << ss));
    }
  } else {
    const int prefix = code >> sl;
    if (prefix < 15) {
      put_zeros(b, prefix);
      put(b, 1, 1u);
      put(b, sl, (uint32_t)(code & ((1 << sl) - 1)));
    } else {
      const uint32_t total = (uint32_t)(code - (15 << sl)) + 4096u;
      const int ss = ilog2(total);
      put_zeros(b, ss + 3);
      put(b, 1, 1u);
      put(b, ss, total - (1u << ss));
    }
  }
  const int a = level < 0 ? -level : level;
  if (sl == 0) sl = 1;
  if (a > (3 << (sl - 1)) && sl < 6) ++sl;
  return sl;
}

// A residual block of max_coeff coefficients in scan order: coeff_token,
// trailing-one signs, levels, total_zeros, run_before. vlc: the nC class
// (0..3) or 4 for chroma DC (nC = -1). Returns TotalCoeff.
CAVLC_HD int put_block(BitW& b, const int* sc, int max_coeff, int vlc) {
  uint32_t mask = 0;
  for (int i = 0; i < max_coeff; ++i)
    if (sc[i] != 0) mask |= 1u << i;
  if (!mask) {
    put(b, B200_CAVLC_TAB(ct_len)[vlc][0], B200_CAVLC_TAB(ct_code)[vlc][0]);
    return 0;
  }
  // from the highest frequency down: trailing ones (at most 3, consecutive
  // from the top), the other levels, the zero runs between coefficients
  int tc = 0, t1 = 0, signs = 0, tz = 0, prev = -1;
  int lev[16], run[16];
  for (uint32_t m = mask; m;) {
    const int i = ilog2(m);
    m &= ~(1u << i);
    if (prev >= 0) {
      run[tc - 1] = prev - i - 1;
      tz += prev - i - 1;
    }
    const int v = sc[i];
    if (tc < 3 && (v == 1 || v == -1) && t1 == tc) {
      ++t1;
      signs = (signs << 1) | (v < 0 ? 1 : 0);
    } else {
      lev[tc - t1] = v;
    }
    ++tc;
    prev = i;
  }
  tz += prev;
  const int ti = tc * 4 + t1;
  const int cl = B200_CAVLC_TAB(ct_len)[vlc][ti];
  if (cl > 0) put(b, cl, B200_CAVLC_TAB(ct_code)[vlc][ti]);
  else put_ue(b, (uint32_t)tc);
  if (t1 > 0) put(b, t1, (uint32_t)signs);
  int sl = (tc > 10 && t1 < 3) ? 1 : 0;
  for (int i = 0; i < tc - t1; ++i) sl = put_level(b, lev[i], i == 0, t1 < 3, sl);
  if (tc < max_coeff) {
    if (vlc == 4) {
      if (tz < 4) put(b, B200_CAVLC_TAB(cdtz_len)[tc - 1][tz], B200_CAVLC_TAB(cdtz_code)[tc - 1][tz]);
      else put_ue(b, (uint32_t)tz);
    } else {
      const int l = (tc - 1 < 15 && tz < 16) ? B200_CAVLC_TAB(tz_len)[tc - 1][tz] : 0;
      if (l > 0) put(b, l, B200_CAVLC_TAB(tz_code)[tc - 1][tz]);
      else put_ue(b, (uint32_t)tz);
    }
  }
  int zl = tz;
  for (int i = 1; i < tc && zl > 0; ++i) {
    const int r = run[i - 1];
    const int zi = zl <= 6 ? zl - 1 : 6;
    const int l = r < 16 ? B200_CAVLC_TAB(run_len)[zi][r] : 0;
    if (l > 0) put(b, l, B200_CAVLC_TAB(run_code)[zi][r]);
    else put_ue(b, (uint32_t)r);
    zl -= r;
  }
  return tc;
}

CAVLC_HD int nc_class(int nc) { return nc < 2 ? 0 : (nc < 4 ? 1 : (nc < 8 ? 2 : 3)); }

// A 4x4 block stored in raster positions, zig-zag scanned: all 16
// coefficients (ac = false) or positions 1..15 (ac = true).
CAVLC_HD int put_4x4(BitW& b, const int16_t* blk, bool ac, int nc) {
  int sc[16];
  const int n = ac ? 15 : 16;
  for (int i = 0; i < n; ++i) sc[i] = blk[B200_CAVLC_TAB(zigzag)[i + (ac ? 1 : 0)]];
  return put_block(b, sc, n, nc_class(nc));
}

// Macroblock headers (clause 7.3.5): I16x16 with mb_type 1 + mode +
// 4 * cbp_chroma + 12 * (cbp_luma != 0), intra_chroma_pred_mode and
// mb_qp_delta 0; P_L0_16x16 with its vector difference, the inter
// coded_block_pattern codeNum and mb_qp_delta 0 when cbp != 0.
CAVLC_HD void put_i16_header(BitW& b, int mode, int chroma_mode, int cbp_chroma, int cbp_luma_flag) {
  put_ue(b, (uint32_t)(1 + mode + 4 * cbp_chroma + 12 * cbp_luma_flag));
  put_ue(b, (uint32_t)chroma_mode);
  put_se(b, 0);
}
// t8: the macroblock's luma uses the 8x8 transform (transform_size_8x8_flag,
// present when the luma pattern is nonzero, 7.3.5).
// t8_mode: the picture parameter set has transform_8x8_mode_flag, so every
// macroblock with a coded luma block carries transform_size_8x8_flag (t8,
// 7.3.5: 0 for a macroblock coded with 4x4 transforms).
CAVLC_HD void put_p16_header(BitW& b, int mvd_x, int mvd_y, int cbp, int t8_mode = 0, int t8 = 0) {
  put_ue(b, 0u);
  put_se(b, mvd_x);
  put_se(b, mvd_y);
  put_ue(b, B200_CAVLC_TAB(cbp_code)[cbp]);
  if (t8_mode && (cbp & 15)) put(b, 1, t8 ? 1u : 0u);
  if (cbp > 0) put_se(b, 0);
}

}  // namespace b200cavlc
