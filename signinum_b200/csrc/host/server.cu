// Serving loop: continuous batching of tile decode requests.
//
// Registered codestreams stay in one resident device arena (and a host copy
// for packet-header parsing).  Requests wait in a FIFO queue.  The dispatcher
// thread takes as many queued requests as fit in one batch (same pixel
// format, at most max_batch_tiles, estimated device memory within the budget
// left by the batches already in flight), builds a plan over the resident
// arena on a free slot's stream and launches it.  The completer thread waits
// for the in-flight batches in launch order, reads their per-tile statuses
// and publishes one result per request.  With several slots, batches built
// while others decode run concurrently on the device.
#include <cuda_runtime.h>

#include <chrono>
#include <cstring>
#include <deque>
#include <memory>
#include <string>

#include "codestream.h"
#include "runtime_internal.h"

using namespace sgn;
using namespace sgn::rt;

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

struct ResidentTile {
  std::vector<uint8_t> host;  // for header parsing
  uint64_t offset = 0;        // in the device arena (16-byte aligned)
  uint32_t width = 0, height = 0, ncomp = 0;
  bool classic = false;  // classic (EBCOT) code blocks: per-thread scratch instead of quad symbols
  // Packet-header parse per resolution (downscale 1, 2, 4, 8), made by the
  // dispatcher the first time a request needs it and reused afterwards.
  std::unique_ptr<TileLayout> layout[4];
  bool parse_failed[4] = {};
};

int scale_index(const sgn_request& r) {
  if (r.kind != SGN_REQ_SCALED && r.kind != SGN_REQ_REGION_SCALED) return 0;
  switch (r.downscale) {
    case 1: return 0;
    case 2: return 1;
    case 4: return 2;
    case 8: return 3;
    default: return -1;  // rejected by the plan builder
  }
}

struct Request {
  uint64_t ticket;
  uint32_t tile;
  uint32_t format;
  sgn_request req;
  uint64_t bytes;    // admission estimate
  uint64_t samples;  // decoded samples (batch bound)
  Clock::time_point submitted;
};

struct Slot {
  cudaStream_t stream = nullptr;
  cudaEvent_t start = nullptr, done = nullptr;
  PinnedBuffer staging;
  sgn_plan* plan = nullptr;
  std::vector<Request> reqs;
  uint64_t bytes = 0;
  sgn_status launch_status = SGN_OK;
  Clock::time_point launched;
  bool busy = false;
};

// Device bytes one request needs while its batch is in flight: coefficient
// arena, level buffers and quad symbols of the decoded resolution, the output
// surface and the job tables (about 48 bytes per code block).  Classic tiles
// need no quad symbols but per-thread flag scratch (at most (w+2)(h+2) 16-bit
// words per block) and, with several layers, a gathered copy of their data:
// 3 bytes per sample covers both.
uint64_t estimate_bytes(const ResidentTile& t, uint32_t format, const sgn_request& r) {
  const uint64_t d = (r.kind == SGN_REQ_SCALED || r.kind == SGN_REQ_REGION_SCALED) ? std::max(1u, r.downscale) : 1;
  const uint64_t w = (t.width + d - 1) / d, h = (t.height + d - 1) / d;
  const uint64_t samples = w * h * t.ncomp;
  uint64_t out_w = w, out_h = h;
  if (r.kind == SGN_REQ_REGION || r.kind == SGN_REQ_REGION_SCALED) {
    out_w = (r.w + d - 1) / d + 1;
    out_h = (r.h + d - 1) / d + 1;
  }
  const uint64_t coef = samples * 4, levels = samples * 2, symbols = samples * (t.classic ? 3 : 1),
                 jobs = samples / 64 + 4096;
  return coef + levels + symbols + jobs + out_w * out_h * bytes_per_pixel(format) + 4096;
}

uint64_t decoded_samples(const ResidentTile& t, const sgn_request& r) {
  const uint64_t d = (r.kind == SGN_REQ_SCALED || r.kind == SGN_REQ_REGION_SCALED) ? std::max(1u, r.downscale) : 1;
  return ((t.width + d - 1) / d) * ((t.height + d - 1) / d) * t.ncomp;
}

}  // namespace

struct sgn_server {
  sgn_ctx* ctx = nullptr;
  sgn_server_config cfg{};
  uint8_t* arena = nullptr;
  uint64_t arena_used = 0;
  std::vector<std::unique_ptr<ResidentTile>> tiles;
  std::mutex mu;
  std::condition_variable cv_work, cv_done, cv_results;
  std::deque<Request> pending;
  std::vector<Slot> slots;
  std::deque<int> inflight;  // slot indices, launch order
  std::deque<sgn_server_result> results;
  cudaStream_t free_stream = nullptr;
  uint64_t next_ticket = 1;
  bool stopping = false;
  bool dispatch_done = false;
  sgn_server_stats stats{};
  std::thread dispatcher, completer;

  void dispatch_loop();
  void complete_loop();
};

void sgn_server::dispatch_loop() {
  cudaSetDevice(ctx->device);
  for (;;) {
    int si = -1;
    std::vector<Request> batch;
    std::vector<ResidentTile*> batch_tiles;  // stable: tiles are never removed
    uint64_t bytes = 0;
    {
      std::unique_lock<std::mutex> lk(mu);
      for (;;) {
        if (stopping && pending.empty()) {
          dispatch_done = true;
          cv_done.notify_all();
          return;
        }
        si = -1;
        for (size_t k = 0; k < slots.size(); ++k)
          if (!slots[k].busy) {
            si = (int)k;
            break;
          }
        // The head of the queue must fit beside what is in flight; alone on
        // an idle device it is always admitted (submit rejected anything
        // larger than the whole budget).
        if (si >= 0 && !pending.empty() &&
            (inflight.empty() || stats.bytes_in_use + pending.front().bytes <= cfg.device_budget_bytes))
          break;
        cv_work.wait(lk);
      }
      const uint32_t fmt = pending.front().format;
      uint64_t samples = 0;
      while (!pending.empty() && batch.size() < cfg.max_batch_tiles && pending.front().format == fmt &&
             (batch.empty() || ((stats.bytes_in_use + bytes + pending.front().bytes <= cfg.device_budget_bytes) &&
                                (!cfg.max_batch_samples || samples + pending.front().samples <= cfg.max_batch_samples)))) {
        bytes += pending.front().bytes;
        samples += pending.front().samples;
        batch.push_back(pending.front());
        pending.pop_front();
      }
      slots[si].busy = true;
      for (const Request& q : batch) batch_tiles.push_back(tiles[q.tile].get());
      stats.bytes_in_use += bytes;
      stats.peak_bytes_in_use = std::max(stats.peak_bytes_in_use, stats.bytes_in_use);
      stats.max_batch_seen = std::max<uint32_t>(stats.max_batch_seen, (uint32_t)batch.size());
      stats.batches += 1;
    }
    Slot& sl = slots[si];
    const auto t_build = Clock::now();
    const size_t n = batch.size();
    std::vector<const uint8_t*> datas(n);
    std::vector<size_t> lens(n);
    std::vector<uint64_t> offs(n);
    std::vector<sgn_request> reqs(n);
    std::vector<const TileLayout*> layouts(n, nullptr);
    std::vector<std::pair<ResidentTile*, int>> misses;
    for (size_t i = 0; i < n; ++i) {
      ResidentTile& t = *batch_tiles[i];
      datas[i] = t.host.data();
      lens[i] = t.host.size();
      offs[i] = t.offset;
      reqs[i] = batch[i].req;
      const int si_ = scale_index(reqs[i]);
      if (si_ >= 0 && !t.layout[si_] && !t.parse_failed[si_]) {
        t.layout[si_].reset(new TileLayout());
        misses.emplace_back(&t, si_);
      }
    }
    // First use of a tile at a resolution: parse its packet headers once.
    ctx->workers->parallel_for(misses.size(), [&](size_t k) {
      ResidentTile& t = *misses[k].first;
      const int d = 1 << misses[k].second;
      const uint32_t target[2] = {(t.width + d - 1) / d, (t.height + d - 1) / d};
      try {
        parse_tile(t.host.data(), t.host.size(), d == 1 ? nullptr : target, *t.layout[misses[k].second]);
      } catch (const ParseError&) {
        t.parse_failed[misses[k].second] = true;
      }
    });
    for (auto& m : misses)
      if (m.first->parse_failed[m.second]) m.first->layout[m.second].reset();
    for (size_t i = 0; i < n; ++i) {
      const int si_ = scale_index(reqs[i]);
      if (si_ >= 0) layouts[i] = batch_tiles[i]->layout[si_].get();
    }
    sl.plan = new sgn_plan();
    // No upload sync: the slot's staging is reused only after this batch ran.
    sl.launch_status = build_plan(ctx, sl.stream, sl.staging, datas.data(), lens.data(), n, batch[0].format,
                                  reqs.data(), sl.plan, arena, offs.data(), layouts.data(), false);
    cudaEventRecord(sl.start, sl.stream);
    if (sl.launch_status == SGN_OK) sl.launch_status = execute(sl.plan, sl.stream);
    cudaEventRecord(sl.done, sl.stream);
    sl.reqs = std::move(batch);
    sl.bytes = bytes;
    sl.launched = Clock::now();
    {
      std::lock_guard<std::mutex> g(mu);
      stats.build_us_total += (uint64_t)(ms_between(t_build, sl.launched) * 1000.0);
      inflight.push_back(si);
      stats.max_inflight_seen = std::max<uint32_t>(stats.max_inflight_seen, (uint32_t)inflight.size());
    }
    cv_done.notify_all();
  }
}

void sgn_server::complete_loop() {
  cudaSetDevice(ctx->device);
  for (;;) {
    int si;
    {
      std::unique_lock<std::mutex> lk(mu);
      cv_done.wait(lk, [&] { return !inflight.empty() || dispatch_done; });
      if (inflight.empty()) return;
      si = inflight.front();
    }
    Slot& sl = slots[si];
    cudaEventSynchronize(sl.done);
    float gpu_ms = 0.f;
    cudaEventElapsedTime(&gpu_ms, sl.start, sl.done);
    const size_t n = sl.reqs.size();
    std::vector<sgn_status> per(n, sl.launch_status);
    if (sl.launch_status == SGN_OK) wait_plan(sl.plan, sl.stream, per.data(), nullptr);
    const auto now = Clock::now();
    std::vector<sgn_server_result> out(n);
    for (size_t i = 0; i < n; ++i) {
      sgn_server_result& r = out[i];
      std::memset(&r, 0, sizeof(r));
      r.ticket = sl.reqs[i].ticket;
      r.status = per[i];
      r.batch_tiles = (uint32_t)n;
      r.latency_ms = ms_between(sl.reqs[i].submitted, now);
      r.queue_ms = ms_between(sl.reqs[i].submitted, sl.launched);
      if (per[i] == SGN_OK && i < sl.plan->surfaces.size()) {
        r.surface = sl.plan->surfaces[i];
        sl.plan->surfaces[i].device_ptr = 0;  // ownership moves to the caller
      }
    }
    release_plan(sl.plan, sl.stream);
    delete sl.plan;
    sl.plan = nullptr;
    sl.reqs.clear();
    {
      std::lock_guard<std::mutex> g(mu);
      for (auto& r : out) results.push_back(r);
      stats.completed += n;
      stats.gpu_us_total += (uint64_t)(gpu_ms * 1000.0f);
      stats.flight_us_total += (uint64_t)(ms_between(sl.launched, now) * 1000.0);
      stats.bytes_in_use -= sl.bytes;
      sl.busy = false;
      inflight.pop_front();
    }
    cv_work.notify_all();
    cv_results.notify_all();
  }
}

extern "C" {

sgn_status sgn_server_create(sgn_ctx* ctx, const sgn_server_config* config, sgn_server** out) {
  if (!ctx || !out) return set_error(SGN_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  cudaSetDevice(ctx->device);
  auto* sv = new sgn_server();
  sv->ctx = ctx;
  if (config) sv->cfg = *config;
  if (!sv->cfg.device_budget_bytes) sv->cfg.device_budget_bytes = 16ull << 30;
  if (!sv->cfg.resident_capacity_bytes) sv->cfg.resident_capacity_bytes = 1ull << 30;
  if (!sv->cfg.max_batch_tiles) sv->cfg.max_batch_tiles = 512;
  if (!sv->cfg.slots) sv->cfg.slots = 3;
  cudaError_t e = cudaMalloc(&sv->arena, sv->cfg.resident_capacity_bytes);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sv->free_stream, cudaStreamNonBlocking);
  sv->slots.resize(sv->cfg.slots);
  for (auto& sl : sv->slots) {
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&sl.start);
    if (e == cudaSuccess) e = cudaEventCreate(&sl.done);
  }
  // Grow the stream-ordered pool to the admission budget once, so batches
  // never wait on the pool reserving memory (the context keeps what the pool
  // holds: its release threshold is unbounded).
  if (e == cudaSuccess) {
    void* warm = nullptr;
    e = cudaMallocAsync(&warm, sv->cfg.device_budget_bytes, sv->free_stream);
    if (e == cudaSuccess) e = cudaFreeAsync(warm, sv->free_stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(sv->free_stream);
  }
  // Pinned staging for each slot's job tables, sized once for a full batch
  // (about 64 bytes per 1024 decoded samples: an HT job per 32x32 block and
  // the smaller IDWT and pack tables), so that growing it (pinning memory,
  // which waits for the device) does not land between batches.
  if (e == cudaSuccess) {
    const uint64_t samples = sv->cfg.max_batch_samples ? sv->cfg.max_batch_samples : (96ull << 20);
    const size_t bytes = (size_t)std::min<uint64_t>(samples / 1024 * 64 + (1u << 20), 64ull << 20);
    for (auto& sl : sv->slots)
      if (e == cudaSuccess) e = sl.staging.ensure(bytes);
  }
  if (e != cudaSuccess) {
    sgn_status st = cuda_status(e, "server set-up");
    for (auto& sl : sv->slots) {
      if (sl.stream) cudaStreamDestroy(sl.stream);
      if (sl.start) cudaEventDestroy(sl.start);
      if (sl.done) cudaEventDestroy(sl.done);
    }
    if (sv->free_stream) cudaStreamDestroy(sv->free_stream);
    if (sv->arena) cudaFree(sv->arena);
    delete sv;
    return st;
  }
  sv->dispatcher = std::thread([sv] { sv->dispatch_loop(); });
  sv->completer = std::thread([sv] { sv->complete_loop(); });
  *out = sv;
  return SGN_OK;
}

sgn_status sgn_server_register(sgn_server* sv, const uint8_t* data, size_t len, uint32_t* tile_id) {
  if (!sv || !data || !tile_id) return set_error(SGN_ERR_INVALID_ARGUMENT, "null argument");
  auto t = std::make_unique<ResidentTile>();
  try {
    Info info = inspect_codestream(data, len);
    t->width = info.width;
    t->height = info.height;
    t->ncomp = info.components;
    t->classic = !info.ht;
  } catch (const ParseError& pe) {
    return set_error(pe.status, pe.message.c_str());
  }
  // Full-resolution packet headers are parsed here, once; other resolutions
  // on first use.  A codestream that fails to parse is still registered: its
  // requests report the error like the plain call does.
  t->layout[0].reset(new TileLayout());
  try {
    parse_tile(data, len, nullptr, *t->layout[0]);
  } catch (const ParseError&) {
    t->layout[0].reset();
    t->parse_failed[0] = true;
  }
  std::lock_guard<std::mutex> g(sv->mu);
  const uint64_t off = (sv->arena_used + 15) & ~(uint64_t)15;
  if (off + len > sv->cfg.resident_capacity_bytes)
    return set_error(SGN_ERR_OUT_OF_MEMORY, "resident codestream arena is full");
  cudaSetDevice(sv->ctx->device);
  cudaError_t e = cudaMemcpy(sv->arena + off, data, len, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_status(e, "resident upload");
  t->host.assign(data, data + len);
  t->offset = off;
  sv->arena_used = off + len;
  *tile_id = (uint32_t)sv->tiles.size();
  sv->tiles.push_back(std::move(t));
  return SGN_OK;
}

}  // extern "C"

namespace {

// Validates and queues one request; sv->mu is held by the caller.
sgn_status submit_locked(sgn_server* sv, uint32_t tile_id, uint32_t format, const sgn_request* request,
                         uint64_t* ticket) {
  sgn_request r{};
  r.kind = SGN_REQ_FULL;
  r.downscale = 1;
  if (request) r = *request;
  if (format == SGN_FMT_RGBA16) return set_error(SGN_ERR_UNSUPPORTED, "Rgba16 output is not supported");
  if (format > SGN_FMT_RGBA16 || r.kind > SGN_REQ_REGION_SCALED)
    return set_error(SGN_ERR_INVALID_ARGUMENT, "unknown pixel format or request kind");
  Request q;
  {
    if (tile_id >= sv->tiles.size()) return set_error(SGN_ERR_INVALID_ARGUMENT, "unknown tile id");
    const ResidentTile& t = *sv->tiles[tile_id];
    if ((r.kind == SGN_REQ_REGION || r.kind == SGN_REQ_REGION_SCALED) &&
        ((uint64_t)r.x + r.w > t.width || (uint64_t)r.y + r.h > t.height))
      return set_error(SGN_ERR_REGION, "region outside the image");
    q.bytes = estimate_bytes(t, format, r);
    q.samples = decoded_samples(t, r);
    if (q.bytes > sv->cfg.device_budget_bytes) {
      sv->stats.rejected += 1;
      return set_error(SGN_ERR_OUT_OF_MEMORY, "request exceeds the server's device-memory budget");
    }
    q.ticket = sv->next_ticket++;
    q.tile = tile_id;
    q.format = format;
    q.req = r;
    q.submitted = Clock::now();
    sv->pending.push_back(q);
    sv->stats.submitted += 1;
  }
  *ticket = q.ticket;
  return SGN_OK;
}

}  // namespace

extern "C" {

sgn_status sgn_server_submit(sgn_server* sv, uint32_t tile_id, uint32_t format, const sgn_request* request,
                             uint64_t* ticket) {
  if (!sv || !ticket) return set_error(SGN_ERR_INVALID_ARGUMENT, "null argument");
  sgn_status st;
  {
    std::lock_guard<std::mutex> g(sv->mu);
    st = submit_locked(sv, tile_id, format, request, ticket);
  }
  if (st == SGN_OK) sv->cv_work.notify_all();
  return st;
}

sgn_status sgn_server_submit_many(sgn_server* sv, size_t n, const uint32_t* tile_ids, uint32_t format,
                                  const sgn_request* requests, uint64_t* tickets, size_t* submitted) {
  if (!sv || (n && (!tile_ids || !tickets))) return set_error(SGN_ERR_INVALID_ARGUMENT, "null argument");
  sgn_status st = SGN_OK;
  size_t k = 0;
  {
    std::lock_guard<std::mutex> g(sv->mu);
    for (; k < n; ++k) {
      st = submit_locked(sv, tile_ids[k], format, requests ? &requests[k] : nullptr, &tickets[k]);
      if (st != SGN_OK) break;
    }
  }
  if (submitted) *submitted = k;
  if (k) sv->cv_work.notify_all();
  return st;
}

sgn_status sgn_server_poll(sgn_server* sv, sgn_server_result* out, size_t cap, size_t* count, uint32_t timeout_ms) {
  if (!sv || !count || (cap && !out)) return set_error(SGN_ERR_INVALID_ARGUMENT, "null argument");
  std::unique_lock<std::mutex> lk(sv->mu);
  if (sv->results.empty() && timeout_ms)
    sv->cv_results.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return !sv->results.empty(); });
  size_t k = 0;
  while (k < cap && !sv->results.empty()) {
    out[k++] = sv->results.front();
    sv->results.pop_front();
  }
  *count = k;
  return SGN_OK;
}

sgn_status sgn_server_stats_get(sgn_server* sv, sgn_server_stats* out) {
  if (!sv || !out) return set_error(SGN_ERR_INVALID_ARGUMENT, "null argument");
  std::lock_guard<std::mutex> g(sv->mu);
  *out = sv->stats;
  return SGN_OK;
}

void sgn_server_surface_free(sgn_server* sv, sgn_surface* sf) {
  if (!sv || !sf || !sf->device_ptr) return;
  cudaSetDevice(sv->ctx->device);
  // The batch that wrote the surface finished before its result was published.
  cudaFreeAsync((void*)(uintptr_t)sf->device_ptr, sv->free_stream);
  sf->device_ptr = 0;
}

void sgn_server_results_release(sgn_server* sv, sgn_server_result* results, size_t n) {
  if (!sv || !results) return;
  cudaSetDevice(sv->ctx->device);
  for (size_t i = 0; i < n; ++i)
    if (results[i].surface.device_ptr) {
      cudaFreeAsync((void*)(uintptr_t)results[i].surface.device_ptr, sv->free_stream);
      results[i].surface.device_ptr = 0;
    }
}

void sgn_server_destroy(sgn_server* sv) {
  if (!sv) return;
  {
    std::lock_guard<std::mutex> g(sv->mu);
    sv->stopping = true;
  }
  sv->cv_work.notify_all();
  sv->dispatcher.join();  // it sets dispatch_done once the queue is empty
  sv->completer.join();   // it returns once the in-flight batches are published
  cudaSetDevice(sv->ctx->device);
  for (auto& r : sv->results)
    if (r.surface.device_ptr) cudaFreeAsync((void*)(uintptr_t)r.surface.device_ptr, sv->free_stream);
  cudaStreamSynchronize(sv->free_stream);
  for (auto& sl : sv->slots) {
    cudaStreamSynchronize(sl.stream);
    cudaStreamDestroy(sl.stream);
    cudaEventDestroy(sl.start);
    cudaEventDestroy(sl.done);
  }
  cudaStreamDestroy(sv->free_stream);
  cudaFree(sv->arena);
  delete sv;
}

}  // extern "C"
