// Launchers of the sm_100a decode kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "../device_plan.h"
#include "../ht_tables.h"

namespace sgn {

cudaError_t ht_kernels_init();
// Uploads the HT tables and sets kernel attributes on `device` (current) once.
cudaError_t ensure_device_init(int device);
cudaError_t upload_ht_tables(const HtDecodeTables& host);
size_t ht_magsgn_smem_bytes(uint32_t ms_words, uint32_t max_w);
// HT cleanup: the VLC pass (one lane per block) then the MagSgn pass (one
// warp per block).  ms_words: unstuffed MagSgn capacity per block in 32-bit
// words; max_w: widest code block of the launch.
cudaError_t launch_ht_vlc(const HtJob* jobs, uint32_t njobs, const uint8_t* arena, uint32_t* symbols,
                          cudaStream_t stream);
cudaError_t launch_ht_magsgn(const HtJob* jobs, uint32_t njobs, const uint8_t* arena, const uint32_t* symbols,
                             int32_t* coef, uint32_t* tile_status, uint32_t ms_words, uint32_t max_w,
                             cudaStream_t stream);
cudaError_t launch_ht_cleanup(const HtJob* jobs, uint32_t njobs, const uint8_t* arena, uint32_t* symbols,
                              int32_t* coef, uint32_t* tile_status, uint32_t ms_words, uint32_t max_w,
                              cudaStream_t stream);
cudaError_t launch_ht_refine(const HtJob* jobs, const uint32_t* list, uint32_t n, const uint8_t* arena, int32_t* coef,
                             uint32_t* tile_status, cudaStream_t stream);
// nunits: work units (strip x row segment) of all jobs of the launch.
cudaError_t launch_idwt_level(const IdwtJob* jobs, uint32_t njobs, uint32_t nunits, cudaStream_t stream);
// All jobs of one launch share the pixel format fmt (a PackFormat).
cudaError_t launch_pack(const PackJob* jobs, uint32_t njobs, uint32_t nunits, uint32_t fmt, cudaStream_t stream);

}  // namespace sgn
