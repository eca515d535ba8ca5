// tune.cu - launch parameters chosen by the autotuner.
//
// The kernels' shapes that do not change their results (macroblock rows per
// deblocking CTA, macroblocks per P-chain CTA, the persistent grids of the
// learned form's re-scoring and fallback search, the intra wavefront's CTA
// count, whether the full search stages its windows by TMA or by loads) are
// read at launch from one process-wide table. Zero means the
// built-in default. The table is set through b200enc_tune_set, or loaded
// from a file of "name value" lines (b200enc_tune_load; the environment
// variable B200ENC_TUNE_FILE names one to load before the first launch).
// b200enc/autotune.py times the variants on the device for a frame size and
// writes such a file. No reference counterpart: the reference's shader
// dispatch sizes are fixed in gpu_compute.c.
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "b200enc_internal.h"

namespace {

struct Knob {
  const char* name;
  int lo, hi;
};

// Indexed by the B200ENC_TUNE_* keys of include/b200enc.h.
constexpr Knob kKnobs[B200ENC_TUNE_COUNT] = {
    {"deblock_rows", 1, 6},           // macroblock rows per deblocking CTA
    {"pchain_mbs_per_cta", 1, 4},     // macroblocks per P-chain CTA (1, 2 or 4)
    {"rescore_ctas_per_sm", 1, 16},   // persistent re-scoring grid, CTAs per SM
    {"fallback_ctas_per_sm", 1, 16},  // persistent fallback full-search grid, CTAs per SM
    {"intra_ctas", 1, 1 << 16},       // CTAs of the intra wavefront (rows in flight)
    {"me_stage", 1, 2},               // full-search window staging: 1 word loads, 2 TMA
    {"deblock_tile_w", 1, 16},        // tile deblocking: tile width in macroblocks
    {"deblock_tile_h", 1, 8},         // tile deblocking: tile height in macroblocks
};

std::atomic<int> g_tune[B200ENC_TUNE_COUNT];
std::once_flag g_env_once;

bool valid(int key, int value) {
  if (key < 0 || key >= B200ENC_TUNE_COUNT) return false;
  if (value == 0) return true;
  if (key == B200ENC_TUNE_PCHAIN_MBS_PER_CTA && value != 1 && value != 2 && value != 4) return false;
  return value >= kKnobs[key].lo && value <= kKnobs[key].hi;
}

int load_file(const char* path) {
  FILE* f = fopen(path, "r");
  if (!f) return -1;
  char line[256];
  int n = 0;
  while (fgets(line, sizeof(line), f)) {
    char name[128];
    int value = 0;
    if (line[0] == '#' || sscanf(line, "%127s %d", name, &value) != 2) continue;
    for (int k = 0; k < B200ENC_TUNE_COUNT; ++k)
      if (strcmp(name, kKnobs[k].name) == 0 && valid(k, value)) {
        g_tune[k].store(value);
        ++n;
      }
  }
  fclose(f);
  return n;
}

void load_env() {
  const char* p = getenv("B200ENC_TUNE_FILE");
  if (p && *p && load_file(p) < 0) fprintf(stderr, "[b200enc] B200ENC_TUNE_FILE %s: cannot read\n", p);
}

}  // namespace

// Value of a knob for the launch sites (0 = the built-in default).
int b200enc_tuned(int key) {
  std::call_once(g_env_once, load_env);
  if (key < 0 || key >= B200ENC_TUNE_COUNT) return 0;
  return g_tune[key].load(std::memory_order_relaxed);
}

extern "C" {

int b200enc_tune_set(int key, int value) {
  std::call_once(g_env_once, load_env);
  if (!valid(key, value)) return -1;
  g_tune[key].store(value);
  return 0;
}

int b200enc_tune_get(int key) {
  if (key < 0 || key >= B200ENC_TUNE_COUNT) return -1;
  return b200enc_tuned(key);
}

const char* b200enc_tune_name(int key) {
  return (key >= 0 && key < B200ENC_TUNE_COUNT) ? kKnobs[key].name : nullptr;
}

int b200enc_tune_load(const char* path) {
  std::call_once(g_env_once, load_env);
  return path ? load_file(path) : -1;
}

}  // extern "C"
