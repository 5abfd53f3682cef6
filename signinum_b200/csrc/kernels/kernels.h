// Launchers of the sm_100a decode kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "../device_plan.h"
#include "../ht_tables.h"

namespace sgn {

#ifdef __CUDACC__
// L2 prefetch hint for the 128-byte line holding p (a global address the
// caller may read).  No register waits for it: the bytes a warp will load
// later are requested from HBM early and its loads then hit L2.
__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(__cvta_generic_to_global(p)));
}

// Prefetches every line of the n bytes at p, `step` lines apart starting at
// line `first` (lanes of a warp pass their lane index and 32).  Every
// address passed to the hint lies inside [p, p + n).
__device__ __forceinline__ void prefetch_l2_range(const void* p, size_t n, uint32_t first, uint32_t step) {
  if (n == 0) return;
  const uintptr_t a = (uintptr_t)p, end = a + n, line0 = a & ~(uintptr_t)127;
  for (uintptr_t q = line0 + (uintptr_t)first * 128; q < end; q += (uintptr_t)step * 128)
    prefetch_l2(reinterpret_cast<const void*>(q < a ? a : q));
}
#endif

cudaError_t ht_kernels_init();
// Uploads the HT tables and sets kernel attributes on `device` (current) once.
cudaError_t ensure_device_init(int device);
cudaError_t upload_ht_tables(const HtDecodeTables& host);
size_t ht_magsgn_smem_bytes(uint32_t ms_words, uint32_t max_w, uint32_t warps = 8);
// HT cleanup: the VLC pass (one lane per block, `threads` lanes per CTA) then
// the MagSgn pass (one warp per block, `warps` warps per CTA).  ms_words:
// unstuffed MagSgn capacity per block in 32-bit words; max_w: widest code
// block of the launch.  With `queue` (a zeroed device counter) the MagSgn pass
// runs as a persistent grid of at most persistent_ctas CTAs whose warps take
// `gran` blocks per grab.  Jobs from nsingle on are narrow (at most 32 wide,
// no refinement passes) and decode two per warp, each with half of the
// warp's ms_words (default: none).
// The VLC pass: `threads` per CTA, `lanes` code blocks per warp (a power of
// two, 1..32); `outline`: the bit readers' rare refill paths out of line.
cudaError_t launch_ht_vlc(const HtJob* jobs, uint32_t njobs, const uint8_t* arena, uint32_t* symbols,
                          cudaStream_t stream, uint32_t threads = 128, uint32_t lanes = 32, bool outline = true);
// Both cleanup passes of each block in one CTA (small plans): the VLC chain
// on one lane, MagSgn on a second warp following it row by row.
cudaError_t launch_ht_fused(const HtJob* jobs, uint32_t njobs, const uint8_t* arena, uint32_t* symbols, int32_t* coef,
                           uint32_t* tile_status, uint32_t ms_words, uint32_t max_w, cudaStream_t stream,
                           bool outline);
cudaError_t launch_ht_magsgn(const HtJob* jobs, uint32_t njobs, const uint8_t* arena, const uint32_t* symbols,
                             int32_t* coef, uint32_t* tile_status, uint32_t ms_words, uint32_t max_w,
                             cudaStream_t stream, uint32_t warps = 8, uint32_t* queue = nullptr, uint32_t gran = 0,
                             uint32_t persistent_ctas = 0, uint32_t nsingle = 0xFFFFFFFFu);
cudaError_t ht_magsgn_occupancy(uint32_t ms_words, uint32_t max_w, uint32_t warps, int* ctas_per_sm);
cudaError_t launch_ht_cleanup(const HtJob* jobs, uint32_t njobs, const uint8_t* arena, uint32_t* symbols,
                              int32_t* coef, uint32_t* tile_status, uint32_t ms_words, uint32_t max_w,
                              cudaStream_t stream);
cudaError_t launch_ht_refine(const HtJob* jobs, const uint32_t* list, uint32_t n, const uint8_t* arena, int32_t* coef,
                             uint32_t* tile_status, cudaStream_t stream);
// nunits: work units (strip x row segment) of all jobs of the launch.  With
// `queue` (a zeroed device counter) the kernels run as a persistent grid of
// at most persistent_ctas CTAs whose warps take units from the counter.
// lean: the grid form held to four CTAs per SM (no effect with a queue).
cudaError_t launch_idwt_level(const IdwtJob* jobs, uint32_t njobs, uint32_t nunits, cudaStream_t stream,
                              uint32_t* queue = nullptr, uint32_t persistent_ctas = 0, bool lean = false);
// All jobs of one launch share the pixel format fmt (a PackFormat) and the
// kernel variant (pack_variant of their components and bit depth).
cudaError_t launch_pack(const PackJob* jobs, uint32_t njobs, uint32_t nunits, uint32_t fmt, uint32_t variant,
                        cudaStream_t stream, uint32_t* queue = nullptr, uint32_t persistent_ctas = 0);
cudaError_t idwt_pack_occupancy(uint32_t fmt, int* idwt_ctas_per_sm, int* pack_ctas_per_sm);
// Classic (EBCOT Tier-1) code blocks: a persistent grid of `ctas` CTAs whose
// threads each take blocks from the zeroed counter `queue` and decode them
// with their own slot of `slot_words` 16-bit flag words in `scratch`
// (ctas x classic_threads_per_cta() slots).
cudaError_t launch_classic(const ClassicJob* jobs, const ClassicSeg* segs, uint32_t njobs, const uint8_t* arena,
                           const uint8_t* gather, int32_t* coef, uint16_t* scratch, uint32_t slot_words, uint32_t ctas,
                           uint32_t* queue, cudaStream_t stream);
uint32_t classic_threads_per_cta();
uint32_t classic_ctas_per_sm();  // resident CTAs per SM of the classic kernel
// Irreversible (9/7) forms of the two launches above, same arguments; the
// pack units of launch_pack97 run four warps per CTA.
cudaError_t launch_idwt97_level(const IdwtJob* jobs, uint32_t njobs, uint32_t nunits, cudaStream_t stream,
                                uint32_t* queue = nullptr, uint32_t persistent_ctas = 0);
cudaError_t launch_pack97(const PackJob* jobs, uint32_t njobs, uint32_t nunits, uint32_t fmt, cudaStream_t stream,
                          uint32_t* queue = nullptr, uint32_t persistent_ctas = 0);

}  // namespace sgn
