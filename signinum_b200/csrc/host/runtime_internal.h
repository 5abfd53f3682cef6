// Internals of the CUDA decode runtime shared by the C ABI (runtime.cu) and
// the serving loop (server.cu): the context and plan structures and the plan
// builder.  Not part of the public interface.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "../../../include/signinum_j2k_cuda.h"
#include "../device_plan.h"
#include "codestream.h"

namespace sgn {
namespace rt {

// Minimal fixed pool for host-side parsing of large batches.
class Workers {
 public:
  explicit Workers(unsigned n) {
    for (unsigned i = 0; i < n; ++i) threads_.emplace_back([this] { loop(); });
  }
  ~Workers() {
    {
      std::lock_guard<std::mutex> g(m_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : threads_) t.join();
  }
  // Runs f(i) for i in [0, n) over the pool plus the calling thread.
  // Runs f(i) for i in [0, n) over the pool plus the calling thread and
  // returns once every item is done.  Completion counts items, not helper
  // tasks: a helper that starts late (its thread descheduled) finds no work
  // left and the caller does not wait for it.  Helpers hold the shared state
  // by reference count, never the caller's stack.
  void parallel_for(size_t n, const std::function<void(size_t)>& f) {
    if (n == 0) return;
    if (threads_.empty() || n < 4) {
      for (size_t i = 0; i < n; ++i) f(i);
      return;
    }
    struct Shared {
      std::atomic<size_t> next{0}, done{0};
      size_t n = 0;
      const std::function<void(size_t)>* f = nullptr;
    };
    auto sh = std::make_shared<Shared>();
    sh->n = n;
    sh->f = &f;
    auto body = [this](const std::shared_ptr<Shared>& s) {
      size_t mine = 0;
      for (size_t i; (i = s->next.fetch_add(1)) < s->n;) {
        (*s->f)(i);
        ++mine;
      }
      if (mine && s->done.fetch_add(mine) + mine == s->n) {
        // Under the mutex, so the waiter cannot miss it between its check and its wait.
        std::lock_guard<std::mutex> g(m_);
        cv_done_.notify_all();
      }
    };
    const size_t nw = std::min(threads_.size(), (n + 1) / 2);
    {
      std::lock_guard<std::mutex> g(m_);
      for (size_t k = 0; k < nw; ++k) tasks_.push_back([body, sh] { body(sh); });
    }
    cv_.notify_all();
    body(sh);
    std::unique_lock<std::mutex> lk(m_);
    cv_done_.wait(lk, [&] { return sh->done.load() == n; });
  }

 private:
  void loop() {
    for (;;) {
      std::function<void()> t;
      {
        std::unique_lock<std::mutex> lk(m_);
        cv_.wait(lk, [&] { return stop_ || !tasks_.empty(); });
        if (stop_ && tasks_.empty()) return;
        t = std::move(tasks_.front());
        tasks_.pop_front();
      }
      t();
    }
  }
  std::vector<std::thread> threads_;
  std::deque<std::function<void()>> tasks_;
  std::mutex m_;
  std::condition_variable cv_, cv_done_;
  bool stop_ = false;
};

struct PinnedBuffer {
  uint8_t* p = nullptr;
  size_t cap = 0;
  // Grows geometrically: freeing pinned memory waits for the device, so a
  // buffer reused by calls of slowly growing sizes must not be replaced on
  // every call.
  cudaError_t ensure(size_t n) {
    if (n <= cap) return cudaSuccess;
    const size_t c = std::max<size_t>(n, cap * 2);
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMallocHost((void**)&p, c);
    if (e == cudaSuccess) cap = c;
    return e;
  }
  ~PinnedBuffer() {
    if (p) cudaFreeHost(p);
  }
};

}  // namespace rt
}  // namespace sgn

// Launch shape of a plan's kernels, chosen by the autotuner.
struct LaunchConfig {
  uint32_t vlc_threads = 128;  // threads per CTA of the VLC pass
  uint32_t vlc_lanes = 0;      // code blocks per VLC warp (1..32, a power of two; 0: chosen by block count)
  uint32_t vlc_outline = 1;    // 1: the VLC pass's bit readers refill out of line; 0: inline
  // 1: both cleanup passes in one kernel, a CTA per block (small plans);
  // 0: the VLC and MagSgn kernels; 2: chosen by block count.
  uint32_t ht_fused = 2;
  uint32_t ms_warps = 8;       // warps (code blocks in flight) per CTA of the MagSgn pass
  uint32_t ms_gran = 0;        // 0: one block per warp; > 0: persistent warps take ms_gran blocks per grab
  uint32_t idwt_queue = 0;     // 0: one unit per warp; 1: persistent warps take IDWT units from a queue
  uint32_t idwt_lean = 0;      // grid form: 1, the kernel held to four CTAs per SM
  uint32_t pack_queue = 0;     // the same for the last level + pack
  // DWT tile shape: rows per work unit of the IDWT levels and of the pack,
  // the base rule (idwt_segment_rows) scaled by 2^shift, shift in -4..1.
  int32_t idwt_seg_shift = 0, pack_seg_shift = 0;
  // Persistent grid sizes (SMs x resident CTAs), derived from the above.
  uint32_t ms_ctas = 0, idwt_ctas = 0, pack_ctas = 0;
};

struct sgn_ctx {
  int device = 0;
  int sm_count = 0;
  cudaStream_t stream = nullptr;
  std::atomic<uint64_t> submissions{0};
  std::mutex mu;
  sgn::rt::PinnedBuffer staging;
  sgn::rt::Workers* workers = nullptr;
  // Streams and pinned staging of the pipelined batch call (one per chunk):
  // chunk c's codestream upload overlaps the kernels of chunk c - 1.
  static constexpr int kLanes = 4;
  cudaStream_t lanes[kLanes] = {};
  sgn::rt::PinnedBuffer lane_staging[kLanes];
  // Autotuned launch shapes by workload signature (see plan_signature).
  std::mutex tune_mu;
  std::vector<std::pair<uint64_t, LaunchConfig>> tuned;
};

struct RoundInfo {
  uint32_t job_begin, njobs, ctas;
  uint32_t irreversible;  // 9/7 jobs (launched by the f32 kernel)
};

struct sgn_plan {
  using HtJob = sgn::HtJob;
  using IdwtJob = sgn::IdwtJob;
  using ClassicJob = sgn::ClassicJob;
  using ClassicSeg = sgn::ClassicSeg;
  using PackJob = sgn::PackJob;
  using RoundInfo = ::RoundInfo;
  size_t n = 0;
  uint32_t format = 0;
  std::vector<sgn_status> status;  // host-side (parse/request) status per tile
  std::vector<sgn_surface> surfaces;
  // Device allocations (stream-ordered pool): the input arena, and two
  // arenas the buffers below are parts of: d_work (coefficients, level
  // planes, quad symbols, tile status) and d_tables (job tables, work-queue
  // counters, classic scratch).
  void* d_work = nullptr;
  void* d_tables = nullptr;
  uint8_t* d_input = nullptr;
  bool owns_input = true;  // false: codestreams live in a caller-owned resident arena
  int32_t* d_coef = nullptr;
  int32_t* d_levels = nullptr;
  uint32_t* d_symbols = nullptr;
  HtJob* d_ht = nullptr;
  uint32_t* d_refine = nullptr;
  // Classic (EBCOT) code blocks: jobs, segment table, per-thread flag scratch.
  ClassicJob* d_classic = nullptr;
  ClassicSeg* d_csegs = nullptr;
  uint16_t* d_cscratch = nullptr;
  uint8_t* d_gather = nullptr;  // multi-layer classic blocks' data, gathered per block
  uint32_t nclassic = 0, classic_ctas = 0, classic_slot = 0;
  IdwtJob* d_idwt = nullptr;
  PackJob* d_pack = nullptr;
  uint32_t* d_status = nullptr;
  uint32_t nht = 0, ms_words = 8, max_w = 1, nref = 0, npack = 0, pack_ctas = 0;
  uint32_t nsingle = 0;  // HT jobs before the narrow ones the MagSgn pass decodes two per warp
  // Reversible pack jobs grouped by kernel variant (pack_variant): variant v
  // has npack_v[v] jobs from d_pack + pack_begin[v] covering pack_units_v[v]
  // units; npack and pack_ctas are their totals.  Pack jobs of irreversible
  // tiles follow the npack reversible ones.
  uint32_t pack_begin[sgn::kPackVariants] = {}, npack_v[sgn::kPackVariants] = {},
           pack_units_v[sgn::kPackVariants] = {};
  uint32_t npack97 = 0, pack97_ctas = 0;
  std::vector<RoundInfo> rounds;
  // Host copies of the IDWT and pack job tables (as uploaded), so that the
  // autotuner can change their rows per unit.
  std::vector<IdwtJob> h_idwt;
  std::vector<PackJob> h_pack;
  uint64_t launches = 0;
  uint64_t sig = 0;  // plan_signature on the base tile shapes (the autotuner's cache key)
  uint64_t ht_cleanup_bytes = 0;  // cleanup segment bytes of the HT jobs (profiling rows)
  std::vector<uint32_t> h_status;
  std::vector<uint64_t> tile_coef_off, tile_coef_elems;  // per tile, in d_coef
  // Launch shape and the device work-queue counters (one per queued launch:
  // MagSgn, each IDWT round, each pack variant, 9/7 pack, classic blocks),
  // zeroed at the start of every execution.
  LaunchConfig cfg;
  uint32_t* d_queue = nullptr;
  uint32_t nqueues = 0;
  // The execution captured as a CUDA graph (made on the second execution).
  cudaGraphExec_t graph = nullptr;
  uint64_t executions = 0;
};


namespace sgn {
namespace rt {

sgn_status set_error(sgn_status s, const char* msg);
sgn_status cuda_status(cudaError_t e, const char* where);
int bytes_per_pixel(uint32_t fmt);

// Builds a plan for n codestreams on stream s, using `staging` for the
// uploads (the copies are finished when it returns).  With resident_arena,
// the codestreams already sit in that device buffer at byte offsets
// resident_off[i] (16-byte aligned) and are not copied; datas still give the
// host bytes for parsing.
// layouts (optional, entries may be null) hands in tile layouts parsed
// earlier for the same codestream and resolution (parse_tile with the target
// the request implies); sync_uploads false leaves the copies in flight (the
// caller must not reuse `staging` before the plan has run).
sgn_status build_plan(sgn_ctx* ctx, cudaStream_t s, PinnedBuffer& staging, const uint8_t* const* datas,
                      const size_t* lens, size_t n, uint32_t fmt, const sgn_request* reqs, sgn_plan* plan,
                      const uint8_t* resident_arena = nullptr, const uint64_t* resident_off = nullptr,
                      const TileLayout* const* layouts = nullptr, bool sync_uploads = true);
// Enqueues the plan's kernels on s.
// Launches the plan's kernels on s.  With `ev` (6 events), records ev[0]
// before the HT VLC pass and ev[k] after stage k: VLC, MagSgn, refinement
// and classic blocks, IDWT levels, packs (ev[5] after the last).
sgn_status execute(sgn_plan* p, cudaStream_t s, cudaEvent_t* ev = nullptr);
// Reads the per-tile device status (synchronising s) and merges host statuses.
sgn_status wait_plan(sgn_plan* p, cudaStream_t s, sgn_status* per_tile, size_t* first_failing);
void free_plan_buffers(sgn_plan* p, cudaStream_t s);
// Fills in the persistent grid sizes of cfg for the plan's kernels and
// device, and makes it the plan's launch shape (dropping any captured graph).
sgn_status apply_config(sgn_ctx* ctx, sgn_plan* p, const LaunchConfig& cfg);
// IDWT round k (the 5/3 or the 9/7 kernel) and the pack launches, with the
// plan's work-queue counters when `queued`, on persistent grids of `ctas`.
cudaError_t launch_round(const sgn_plan* p, size_t k, cudaStream_t s, bool queued, uint32_t ctas, bool lean = false);
// The classic (EBCOT) code-block kernel over the plan's classic jobs.
cudaError_t launch_classic_blocks(const sgn_plan* p, cudaStream_t s);
cudaError_t launch_packs(const sgn_plan* p, cudaStream_t s, bool queued, uint32_t ctas);
// Rows per work unit of the plan's IDWT jobs and pack jobs: the base rule of
// each job scaled by 2^ishift / 2^pshift (at least 2 rows, even), with the
// units of every job, round and pack launch recomputed to match.
void set_segments(sgn_plan* p, std::vector<sgn::IdwtJob>& idwt, std::vector<sgn::PackJob>& packs, int ishift,
                  int pshift);
// Workload signature for the autotuner cache: pixel format, job counts and
// block shape classes.
uint64_t plan_signature(const sgn_plan* p);
// Frees the plan's surfaces that are still owned by it, then its buffers.
void release_plan(sgn_plan* p, cudaStream_t s);

}  // namespace rt
}  // namespace sgn
