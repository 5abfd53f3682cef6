// HT code-block decode that allocates nothing.
//
// Some callers of this code cannot allocate device memory: a host
// framework whose own caching allocator owns all of the GPU's memory (a
// cudaMalloc beside it would fail or fragment its pool), a decoder plugin
// that is handed its input and output buffers by its host and may not
// create any of its own, and a real-time loop that must not allocate, nor
// wait on the allocator's implicit synchronisation, once it runs.  They hand
// in device inputs and outputs; the scratch the HT kernels need (one 32-bit
// symbol per quad, written by the VLC pass and read by the MagSgn pass), the
// device copy of the block descriptors and the refinement list live in
// file-scope static device arrays of fixed size, so this entry point calls
// no cudaMalloc, cudaFree or allocating library routine.
//
// The arrays (about 16.4 MiB) are reserved on every device where this
// file's CUDA module is loaded, until the process exits: under CUDA's
// default lazy module loading that is the first call of this entry point on
// the device, under CUDA_MODULE_LOADING=EAGER the library's first use of the
// device.  They are shared by every call on a device and keep the last
// call's contents; calls that overlap on the GPU (different streams, or host
// threads racing) race on them and must be serialised by the caller.
#include <cuda_runtime.h>

#include <cstddef>
#include <cstring>
#include <mutex>

#include "../../../include/signinum_j2k_cuda.h"
#include "../device_plan.h"
#include "../kernels/kernels.h"

using namespace sgn;

// Shared with the rest of the C ABI (sgn_last_error_message).
void sgn_set_last_error_message(const char* msg);

namespace {

constexpr uint32_t kNoAllocMaxBlocks = 4096;
// The quad-symbol table of any code block of at most 4096 samples and at
// most 1024 rows fits in 1024 words (rows padded to an even quad count).
constexpr uint32_t kNoAllocSymbolsPerBlock = 1024;
constexpr int kMaxDevices = 64;

// 16 MiB of quad symbols: the scratch of the HT cleanup pass.
static __device__ __align__(256) uint32_t g_noalloc_symbols[kNoAllocMaxBlocks * kNoAllocSymbolsPerBlock];
static __device__ __align__(256) HtJob g_noalloc_jobs[kNoAllocMaxBlocks];
static __device__ __align__(256) uint32_t g_noalloc_refine[kNoAllocMaxBlocks];
static __device__ __align__(256) uint32_t g_noalloc_refine_count;

static_assert(sizeof(sgn_ht_block) == sizeof(HtJob), "sgn_ht_block must match the device job layout");
static_assert(offsetof(sgn_ht_block, src) == offsetof(HtJob, src), "layout");
static_assert(offsetof(sgn_ht_block, dst) == offsetof(HtJob, dst), "layout");
static_assert(offsetof(sgn_ht_block, reserved) == offsetof(HtJob, sym), "layout");
static_assert(offsetof(sgn_ht_block, lcup) == offsetof(HtJob, lcup), "layout");
static_assert(offsetof(sgn_ht_block, tile) == offsetof(HtJob, tile), "layout");
static_assert(offsetof(sgn_ht_block, stride) == offsetof(HtJob, stride), "layout");
static_assert(offsetof(sgn_ht_block, lref) == offsetof(HtJob, lref), "layout");
static_assert(offsetof(sgn_ht_block, w) == offsetof(HtJob, w), "layout");
static_assert(offsetof(sgn_ht_block, h) == offsetof(HtJob, h), "layout");
static_assert(offsetof(sgn_ht_block, missing_msbs) == offsetof(HtJob, mmsb), "layout");
static_assert(offsetof(sgn_ht_block, passes) == offsetof(HtJob, passes), "layout");
static_assert(offsetof(sgn_ht_block, num_bitplanes) == offsetof(HtJob, nbp), "layout");
static_assert(offsetof(sgn_ht_block, flags) == offsetof(HtJob, flags), "layout");

struct DeviceArrays {
  bool ready = false;
  uint32_t* symbols = nullptr;
  HtJob* jobs = nullptr;
  uint32_t* refine = nullptr;
  uint32_t* refine_count = nullptr;
};

DeviceArrays g_arrays[kMaxDevices];
std::mutex g_setup_mu;

sgn_status fail(sgn_status s, const char* m) {
  sgn_set_last_error_message(m);
  return s;
}

// The coding passes the kernels run for a descriptor, as the codestream
// parser settles them: a refinement pass needs refinement bytes, and with 29
// missing MSBs only the cleanup pass has a bit-plane left.
__host__ __device__ inline uint32_t effective_passes(uint32_t passes, uint32_t lref, uint32_t missing_msbs) {
  if (passes > 1 && (lref == 0 || missing_msbs == 29)) return 1;
  return passes;
}

// Device addresses of the static arrays for the current device: taken once
// per device with cudaGetSymbolAddress (host code must not use the arrays'
// names as device addresses).
sgn_status setup(int device, DeviceArrays** out) {
  if (device < 0 || device >= kMaxDevices) return fail(SGN_ERR_INVALID_ARGUMENT, "device ordinal out of range");
  std::lock_guard<std::mutex> g(g_setup_mu);
  DeviceArrays& a = g_arrays[device];
  if (!a.ready) {
    if (ensure_device_init(device) != cudaSuccess) {
      cudaGetLastError();
      return fail(SGN_ERR_CUDA_RUNTIME, "HT table set-up failed");
    }
    if (cudaGetSymbolAddress((void**)&a.symbols, g_noalloc_symbols) != cudaSuccess ||
        cudaGetSymbolAddress((void**)&a.jobs, g_noalloc_jobs) != cudaSuccess ||
        cudaGetSymbolAddress((void**)&a.refine, g_noalloc_refine) != cudaSuccess ||
        cudaGetSymbolAddress((void**)&a.refine_count, g_noalloc_refine_count) != cudaSuccess) {
      cudaGetLastError();
      return fail(SGN_ERR_CUDA_RUNTIME, "cudaGetSymbolAddress failed for the no-allocation scratch");
    }
    a.ready = true;
  }
  *out = &a;
  return SGN_OK;
}

// Gives every block its slice of the symbol scratch, settles its passes and
// lists the blocks that carry refinement passes.
__global__ void noalloc_prepare_kernel(HtJob* jobs, uint32_t n, uint32_t* refine, uint32_t* refine_count) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  HtJob& job = jobs[j];
  job.sym = (uint64_t)j * kNoAllocSymbolsPerBlock;
  job.passes = (uint8_t)effective_passes(job.passes, job.lref, job.mmsb);
  if (job.passes > 1) refine[atomicAdd(refine_count, 1u)] = j;
}

}  // namespace

extern "C" {

sgn_status sgn_ht_decode_blocks_noalloc(const sgn_ht_block* blocks, uint32_t n, const uint8_t* segments,
                                        size_t segments_len, int32_t* coefficients, size_t coefficients_len,
                                        uint32_t* tile_status, uint32_t n_tiles, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (n > kNoAllocMaxBlocks) return fail(SGN_ERR_INVALID_ARGUMENT, "more than 4096 code blocks in one call");
  if ((n && (!blocks || !segments || !coefficients)) || (n_tiles && !tile_status))
    return fail(SGN_ERR_INVALID_ARGUMENT, "null argument");
  // The kernels store sample pairs with 8-byte stores wherever a block's
  // first sample and row stride are even, which assumes an 8-byte aligned
  // coefficient buffer.
  if (((uintptr_t)coefficients & 7) != 0)
    return fail(SGN_ERR_INVALID_ARGUMENT, "coefficients must be 8-byte aligned");
  if (((uintptr_t)tile_status & 3) != 0) return fail(SGN_ERR_INVALID_ARGUMENT, "tile_status must be 4-byte aligned");
  // Validate the descriptors on the host before any device work: every read
  // stays inside segments[0, segments_len) and every write inside
  // coefficients[0, coefficients_len).
  uint32_t max_w = 1, max_lcup = 0, nref = 0;
  for (uint32_t j = 0; j < n; ++j) {
    const sgn_ht_block& b = blocks[j];
    if (b.w == 0 || b.h == 0 || (uint32_t)b.w * b.h > 4096 ||
        sym_words(b.w, b.h) > kNoAllocSymbolsPerBlock)
      return fail(SGN_ERR_INVALID_ARGUMENT, "code block larger than 4096 samples");
    if (b.passes > 3 || (b.passes && (b.lcup < 2 || b.missing_msbs >= 30)) || b.tile >= n_tiles ||
        b.stride < b.w)
      return fail(SGN_ERR_INVALID_ARGUMENT, "invalid code-block descriptor");
    if (b.dst > coefficients_len || (uint64_t)(b.h - 1) * b.stride + b.w > coefficients_len - b.dst)
      return fail(SGN_ERR_BUFFER, "code block outside the coefficient buffer");
    const uint32_t passes = effective_passes(b.passes, b.lref, b.missing_msbs);
    const uint64_t span = passes == 0 ? 0 : (uint64_t)b.lcup + (passes > 1 ? b.lref : 0);
    if (b.src > segments_len || span > segments_len - b.src)
      return fail(SGN_ERR_BUFFER, "code-block segment outside the segment buffer");
    if (b.w > max_w) max_w = b.w;
    if (passes && b.lcup > max_lcup) max_lcup = b.lcup;
    if (passes > 1) ++nref;
  }
  uint32_t ms_words = (max_lcup + 15) / 4 + 2;
  if (ht_magsgn_smem_bytes(ms_words, max_w) > 227 * 1024)
    return fail(SGN_ERR_UNSUPPORTED, "cleanup segment too long for the MagSgn staging buffer");
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) {
    cudaGetLastError();
    return fail(SGN_ERR_CUDA_UNAVAILABLE, "no current CUDA device");
  }
  DeviceArrays* a = nullptr;
  sgn_status st = setup(device, &a);
  if (st != SGN_OK) return st;
  cudaError_t e = cudaSuccess;
  // What must start at zero: the status words the kernels OR into and the
  // refinement-list counter.  The symbol scratch is written before it is read.
  if (n_tiles) e = cudaMemsetAsync(tile_status, 0, (size_t)n_tiles * sizeof(uint32_t), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(a->refine_count, 0, sizeof(uint32_t), s);
  if (e == cudaSuccess && n) e = cudaMemcpyAsync(a->jobs, blocks, (size_t)n * sizeof(HtJob), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && n) {
    noalloc_prepare_kernel<<<(n + 127) / 128, 128, 0, s>>>(a->jobs, n, a->refine, a->refine_count);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = launch_ht_cleanup(a->jobs, n, segments, a->symbols, coefficients, tile_status, ms_words, max_w, s);
  if (e == cudaSuccess) e = launch_ht_refine(a->jobs, a->refine, nref, segments, coefficients, tile_status, s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(SGN_ERR_CUDA_RUNTIME, cudaGetErrorString(e));
  }
  return SGN_OK;
}

}  // extern "C"
