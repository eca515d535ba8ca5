// b200enc_internal.h - declarations shared by the library's translation
// units. The public C-ABI is include/b200enc.h (stage entry points) and
// include/gpu_compute.h (the reference's drop-in boundary).
#pragma once
#include <cstddef>
#include <cstdint>

#include "../../include/b200enc.h"

// Value of an autotuned launch parameter (B200ENC_TUNE_*), 0 = the default.
int b200enc_tuned(int key);

// ---- batched stage launchers (batch.cu drives them) ------------------------
namespace b200enc {
struct BatchTab;
}
#include <cuda_runtime.h>
int b200enc_me_full_search_err(const uint8_t* cur_y, int cur_pitch, const uint8_t* ref_y, int ref_pitch, int W,
                               int H, int RW, int RH, int range, int lambda, int zero_thresh, void* mv_out,
                               const int* mb_list, const int* mb_count, int list_capacity, int flags, uint32_t* err,
                               cudaStream_t st);
int b200enc_me_batch_launch(const b200enc::BatchTab& bt, int range, const int* list, const int* count, int ctas,
                            cudaStream_t st);
int b200enc_p_frame_batch_launch(const b200enc::BatchTab& bt, int n, cudaStream_t st);
int b200enc_i_frame_batch_launch(const b200enc::BatchTab& bt, int ctas, uint32_t max_wait, cudaStream_t st);
int b200enc_deblock_batch_rows(int max_mbw, int max_mbh);
int b200enc_deblock_tiles_launch(int mbw, int mbh, int qp, int is_intra, const uint32_t* nz, const void* mv,
                                 const uint8_t* src_y, const uint8_t* src_uv, uint8_t* dst_y, uint8_t* dst_uv,
                                 int pitch, uint32_t* status, uint32_t max_wait, cudaStream_t stream,
                                 const uint8_t* t8 = nullptr);
int b200enc_deblock_tile_count(int mbw, int mbh, int* tw, int* th);
int b200enc_deblock_tiles_batch_launch(const b200enc::BatchTab& bt, int tiles, uint32_t max_wait, cudaStream_t st);
int b200enc_deblock_batch_launch(const b200enc::BatchTab& bt, int max_mbw, int ctas, uint32_t max_wait,
                                 cudaStream_t st);
int b200enc_proposal_me_batch(void* h, const b200enc::BatchTab& bt, int n, int range, int lambda, int mode,
                              float param, cudaStream_t st);
