// b200enc_internal.h - declarations shared by the library's translation
// units. The public C-ABI is include/b200enc.h (stage entry points) and
// include/gpu_compute.h (the reference's drop-in boundary).
#pragma once
#include <cstddef>
#include <cstdint>

#include "../../include/b200enc.h"

// Value of an autotuned launch parameter (B200ENC_TUNE_*), 0 = the default.
int b200enc_tuned(int key);
