// Context, device plans and the C ABI of the CUDA decode path.
//
// A plan is the device form of one decode call: the codestreams copied once
// into a device arena, one HtJob per code block (ordered by coded length),
// the IDWT level jobs of every tile grouped into rounds (coarse to fine) and
// one fused last-level/pack job per tile writing straight into the output
// surfaces.  Executing a plan is a fixed sequence of launches on the context
// stream, so a plan can be replayed and captured in a CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <functional>
#include <mutex>
#include <numeric>
#include <thread>
#include <vector>

#include "../../../include/signinum_j2k_cuda.h"
#include "../device_plan.h"
#include "../ebcot.h"
#include "../ht_tables.h"
#include "../kernels/kernels.h"
#include "codestream.h"
#include "profile.h"
#include "roi.h"
#include "runtime_internal.h"

using namespace sgn;

namespace sgn {
namespace rt {

thread_local char g_msg[512];

sgn_status set_error(sgn_status s, const char* msg) {
  std::snprintf(g_msg, sizeof(g_msg), "%s", msg ? msg : "");
  return s;
}

}  // namespace rt
}  // namespace sgn

using namespace sgn::rt;

void sgn_set_last_error_message(const char* msg) { set_error(0, msg); }

namespace sgn {

// Per-device set-up of the decode kernels: the HT lookup tables in device
// memory and the shared-memory opt-in of the MagSgn pass.  Done once per
// device, with that device current.
cudaError_t ensure_device_init(int device) {
  static std::mutex mu;
  static bool done[64] = {};
  static cudaError_t err[64] = {};
  if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> g(mu);
  if (!done[device]) {
    HtDecodeTables t;
    build_decode_tables(t);
    cudaError_t e = upload_ht_tables(t);
    if (e == cudaSuccess) e = ht_kernels_init();
    err[device] = e;
    done[device] = e == cudaSuccess;
    return e;
  }
  return err[device];
}

}  // namespace sgn

namespace sgn {
namespace rt {

sgn_status cuda_status(cudaError_t e, const char* where) {
  if (e == cudaSuccess) return SGN_OK;
  char buf[400];
  std::snprintf(buf, sizeof(buf), "CUDA runtime error in %s: %s", where, cudaGetErrorString(e));
  if (e == cudaErrorMemoryAllocation) return set_error(SGN_ERR_OUT_OF_MEMORY, buf);
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return set_error(SGN_ERR_CUDA_UNAVAILABLE, buf);
  return set_error(SGN_ERR_CUDA_RUNTIME, buf);
}

int bytes_per_pixel(uint32_t fmt) {
  static const int b[] = {1, 3, 4, 2, 6, 8};
  return fmt < 6 ? b[fmt] : 0;
}

namespace {

struct TileWork {
  const TileLayout* L = nullptr;  // the parse below, or a caller's cached one
  TileLayout own;
  sgn_status status = SGN_OK;
  uint32_t crop_x = 0, crop_y = 0, crop_w = 0, crop_h = 0;
  uint32_t region_conv = 0;
};

// Request semantics: DeviceDecodePlan::for_image (device_plan.rs:23-51) for
// the output rectangle, decode_scaled_from_info / decode_region_scaled_from_info
// (crates/signinum-j2k/src/decode.rs:12-71) for the reduced resolution.
void prepare_tile(const uint8_t* data, size_t len, uint32_t fmt, const sgn_request* req, TileWork& tw,
                  const TileLayout* cached) {
  try {
    if (fmt == SGN_FMT_RGBA16) throw ParseError{SGN_ERR_UNSUPPORTED, "Rgba16 output is not supported"};
    if (fmt > SGN_FMT_RGBA16) throw ParseError{SGN_ERR_INVALID_ARGUMENT, "unknown pixel format"};
    Info info = inspect_codestream(data, len);
    uint32_t kind = req ? req->kind : SGN_REQ_FULL;
    uint32_t sx = 0, sy = 0, sw = info.width, sh = info.height, d = 1;
    if (kind == SGN_REQ_REGION || kind == SGN_REQ_REGION_SCALED) {
      sx = req->x;
      sy = req->y;
      sw = req->w;
      sh = req->h;
    }
    if (kind == SGN_REQ_SCALED || kind == SGN_REQ_REGION_SCALED) d = req->downscale;
    if (kind > SGN_REQ_REGION_SCALED) throw ParseError{SGN_ERR_INVALID_ARGUMENT, "unknown request kind"};
    if (d != 1 && d != 2 && d != 4 && d != 8) throw ParseError{SGN_ERR_UNSUPPORTED, "unknown downscale"};
    if ((uint64_t)sx + sw > info.width || (uint64_t)sy + sh > info.height)
      throw ParseError{SGN_ERR_REGION, "region outside the image"};
    uint32_t ox0 = sx / d, oy0 = sy / d;
    uint32_t ox1 = (uint32_t)(((uint64_t)sx + sw + d - 1) / d), oy1 = (uint32_t)(((uint64_t)sy + sh + d - 1) / d);
    uint32_t target[2] = {(info.width + d - 1) / d, (info.height + d - 1) / d};
    if (cached) {
      tw.L = cached;
    } else {
      parse_tile(data, len, d == 1 ? nullptr : target, tw.own);
      tw.L = &tw.own;
    }
    const TileLayout& L = *tw.L;
    bool gray = L.ncomp == 1;
    bool ok_map = (gray && (fmt == SGN_FMT_GRAY8 || fmt == SGN_FMT_GRAY16)) ||
                  (!gray && (fmt == SGN_FMT_RGB8 || fmt == SGN_FMT_RGBA8 || fmt == SGN_FMT_RGB16));
    if (!ok_map) throw ParseError{SGN_ERR_UNSUPPORTED, "backend color space cannot be mapped to requested pixel format"};
    if (kind == SGN_REQ_SCALED) {
      if (L.out_w != ox1 - ox0 || L.out_h != oy1 - oy0)
        throw ParseError{SGN_ERR_BUFFER, "output buffer does not match the reduced image"};
    } else if (kind == SGN_REQ_REGION_SCALED && d > 1) {
      if (ox1 > L.out_w || oy1 > L.out_h) throw ParseError{SGN_ERR_REGION, "scaled region outside the reduced image"};
    }
    tw.crop_x = ox0;
    tw.crop_y = oy0;
    tw.crop_w = ox1 - ox0;
    tw.crop_h = oy1 - oy0;
    tw.region_conv = (kind == SGN_REQ_REGION || kind == SGN_REQ_REGION_SCALED) ? 1 : 0;
    tw.status = SGN_OK;
  } catch (const ParseError& e) {
    tw.status = e.status;
  }
}

template <typename T>
cudaError_t dalloc(T** p, size_t count, cudaStream_t s) {
  *p = nullptr;
  if (count == 0) return cudaSuccess;
  return cudaMallocAsync((void**)p, count * sizeof(T), s);
}

bool is_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// Coded-length bucket of a block: the HT job table is ordered by bucket,
// longest segments first (64-byte steps), which is the order the HT kernels
// take blocks in.  Exact order inside a bucket does not matter.
constexpr uint32_t kLenBuckets = 64;
inline uint32_t len_bucket(uint32_t lcup) { return kLenBuckets - 1 - std::min<uint32_t>(lcup >> 6, kLenBuckets - 1); }
// HT job order: blocks the MagSgn pass decodes one per warp, then the narrow
// ones it decodes two per warp (at most 32 wide, no refinement passes), each
// group by coded length, longest first.
constexpr uint32_t kHtBuckets = 2 * kLenBuckets;
inline bool pairable(const CodeBlock& cb) { return cb.w <= 32 && cb.passes <= 1; }
inline uint32_t ht_bucket(const CodeBlock& cb) { return (pairable(cb) ? kLenBuckets : 0) + len_bucket(cb.lcup); }
// Largest plan (HT blocks) the autotuner tries the fused cleanup kernel on
// (a CTA per block; each waits only on its own chain lane).
constexpr uint32_t kFusedMaxBlocks = 8192;
// Classic blocks by coding passes (0 .. 94), most passes first.
constexpr uint32_t kPassBuckets = 96;
inline uint32_t pass_bucket(uint32_t passes) { return kPassBuckets - 1 - std::min<uint32_t>(passes, kPassBuckets - 1); }

sgn_status build_plan_impl(sgn_ctx* ctx, cudaStream_t s, PinnedBuffer& staging, const uint8_t* const* datas,
                           const size_t* lens, size_t n, uint32_t fmt, const sgn_request* reqs, sgn_plan* plan,
                           const uint8_t* resident_arena, const uint64_t* resident_off,
                           const TileLayout* const* layouts, bool sync_uploads) {
  plan->n = n;
  plan->format = fmt;
  plan->status.assign(n, SGN_OK);
  plan->surfaces.assign(n, sgn_surface{});
  std::vector<TileWork> work(n);
  // Region requests: the code blocks and IDWT windows the region needs
  // (RoiPlan, crates/signinum-j2k-native/src/j2c/roi.rs:18-270).
  std::vector<RoiWindows> rois(n);
  ctx->workers->parallel_for(n, [&](size_t i) {
    if (!datas[i] && lens[i]) {
      work[i].status = SGN_ERR_INVALID_ARGUMENT;
      return;
    }
    prepare_tile(datas[i], lens[i], fmt, reqs ? &reqs[i] : nullptr, work[i], layouts ? layouts[i] : nullptr);
    const TileWork& tw = work[i];
    if (tw.status == SGN_OK && tw.region_conv)
      build_roi_windows(*tw.L, tw.crop_x, tw.crop_y, tw.crop_w, tw.crop_h, rois[i]);
  });
  // Arena layout.
  std::vector<uint64_t> in_off(n, 0), coef_off(n, 0), lvl_off(n, 0), lvl_size(n, 0);
  uint64_t in_total = 0, coef_total = 0, lvl_total = 0;
  uint32_t max_rounds = 0;
  for (size_t i = 0; i < n; ++i) {
    plan->status[i] = work[i].status;
    if (work[i].status != SGN_OK) continue;
    const TileLayout& L = *work[i].L;
    if (resident_arena) {
      in_off[i] = resident_off[i];
    } else {
      in_off[i] = in_total;
      in_total += (lens[i] + 15) & ~(size_t)15;
    }
    coef_off[i] = coef_total;
    coef_total += L.coef_per_comp * L.ncomp;
    uint32_t R = L.levels - L.skipped;  // last decoded resolution
    if (R >= 2) {
      uint32_t d = L.skipped + 1;
      uint64_t w = (L.width + (1ull << d) - 1) >> d, h = (L.height + (1ull << d) - 1) >> d;
      lvl_size[i] = w * h;
      lvl_off[i] = lvl_total;
      lvl_total += 2 * w * h * L.ncomp;
      max_rounds = std::max(max_rounds, R - 1);
    }
  }
  cudaError_t e = cudaSuccess;
  bool direct = true;  // codestreams need no staging copy
  if (resident_arena) {
    plan->d_input = const_cast<uint8_t*>(resident_arena);
    plan->owns_input = false;
  } else {
    if ((e = dalloc(&plan->d_input, in_total, s)) != cudaSuccess) return cuda_status(e, "input arena");
    // When the caller's codestreams are pinned and contiguous in arena order
    // (16-byte padded), they go up in one copy, issued now so that it
    // overlaps the rest of the plan build.
    direct = n > 0 && in_total > 0 && plan->status[0] == SGN_OK;
    for (size_t i = 0; direct && i + 1 < n; ++i)
      direct = plan->status[i + 1] == SGN_OK && datas[i + 1] == datas[i] + ((lens[i] + 15) & ~(size_t)15);
    direct = direct && is_pinned(datas[0]);
    if (direct && (e = cudaMemcpyAsync(plan->d_input, datas[0], in_total, cudaMemcpyHostToDevice, s)) != cudaSuccess)
      return cuda_status(e, "input upload");
  }
  plan->tile_coef_off = coef_off;
  plan->tile_coef_elems.assign(n, 0);
  for (size_t i = 0; i < n; ++i)
    if (plan->status[i] == SGN_OK) plan->tile_coef_elems[i] = work[i].L->coef_per_comp * work[i].L->ncomp;

  // HT job table, pass A (per tile, in parallel): block counts per
  // coded-length bucket, symbol scratch, refinement blocks and the MagSgn
  // staging bound.  Each coded block gets a quad-symbol table of
  // ceil(w/2) x ceil(h/2) words in the symbol scratch.
  struct TileHt {
    uint64_t sym = 0, bytes = 0;
    uint32_t nref = 0, ms_words = 8, ms_half = 0, max_w = 1;
    uint32_t hist[kHtBuckets];
    uint32_t ncls = 0, nseg = 0, slot = 0;  // classic tiles
    uint64_t gather = 0;                    // multi-layer classic tiles
    uint32_t chist[kPassBuckets];           // classic blocks per coding-pass count
  };
  std::vector<TileHt> th(n);
  ctx->workers->parallel_for(n, [&](size_t i) {
    TileHt& t = th[i];
    std::fill(t.hist, t.hist + kHtBuckets, 0u);
    std::fill(t.chist, t.chist + kPassBuckets, 0u);
    if (plan->status[i] != SGN_OK) return;
    if (work[i].L->classic) {
      t.nseg = (uint32_t)work[i].L->segments.size();
      t.gather = work[i].L->gather_bytes;
      for (const CodeBlock& cb : work[i].L->blocks) {
        if (!block_required(rois[i], cb)) continue;
        ++t.ncls;
        ++t.chist[pass_bucket(cb.passes)];
        if (cb.passes) t.slot = std::max<uint32_t>(t.slot, classic_slot_words(cb.w, cb.h));
      }
      return;
    }
    for (const CodeBlock& cb : work[i].L->blocks) {
      if (!block_required(rois[i], cb)) continue;
      ++t.hist[ht_bucket(cb)];
      t.max_w = std::max<uint32_t>(t.max_w, cb.w);
      if (!cb.passes) continue;
      t.sym += sym_words(cb.w, cb.h);
      t.bytes += cb.lcup;
      if (cb.passes > 1) ++t.nref;
      if (cb.ms_words) {  // from the parse (cached layouts carry it)
        t.ms_words = std::max<uint32_t>(t.ms_words, cb.ms_words);
        if (pairable(cb)) t.ms_half = std::max<uint32_t>(t.ms_half, cb.ms_words);
      }
    }
  });
  // Bucket-major, tile-minor start positions; symbol and refinement offsets.
  std::vector<uint64_t> sym_off(n, 0);
  std::vector<uint32_t> ref_off(n, 0), start((size_t)kHtBuckets * n, 0);
  uint64_t sym_total = 0;
  uint32_t nht = 0, nref = 0, ms_words = 8, ms_half = 0, max_w = 1;
  // Classic jobs: bucket-major by coding passes (most first), tile-minor, so
  // that the lanes of a warp take blocks of similar work and the longest
  // blocks start first.
  std::vector<uint32_t> cseg_off(n, 0), cstart((size_t)kPassBuckets * n, 0);
  std::vector<uint64_t> gather_off(n, 0);
  uint32_t ncls = 0, ncseg = 0, cslot = 0;
  uint64_t gather_total = 0;
  for (size_t i = 0; i < n; ++i) {
    gather_off[i] = gather_total;
    gather_total += (th[i].gather + 15) & ~(uint64_t)15;
    cseg_off[i] = ncseg;
    ncseg += th[i].nseg;
    cslot = std::max(cslot, th[i].slot);
  }
  for (uint32_t b = 0; b < kPassBuckets; ++b)
    for (size_t i = 0; i < n; ++i) {
      cstart[(size_t)b * n + i] = ncls;
      ncls += th[i].chist[b];
    }
  for (size_t i = 0; i < n; ++i) {
    sym_off[i] = sym_total;
    sym_total += th[i].sym;
    ref_off[i] = nref;
    nref += th[i].nref;
    ms_words = std::max(ms_words, th[i].ms_words);
    ms_half = std::max(ms_half, th[i].ms_half);
    max_w = std::max(max_w, th[i].max_w);
  }
  for (uint32_t b = 0; b < kHtBuckets; ++b) {
    if (b == kLenBuckets) plan->nsingle = nht;
    for (size_t i = 0; i < n; ++i) {
      start[(size_t)b * n + i] = nht;
      nht += th[i].hist[b];
    }
  }
  plan->nht = nht;
  // Each warp's bit array holds one block, or two narrow ones in its halves.
  plan->ms_words = std::max(ms_words, 2 * ms_half);
  plan->max_w = max_w;
  plan->nref = nref;
  plan->ht_cleanup_bytes = 0;
  for (size_t i = 0; i < n; ++i) plan->ht_cleanup_bytes += th[i].bytes;
  if (ht_magsgn_smem_bytes(plan->ms_words, max_w) > 227 * 1024)
    return set_error(SGN_ERR_UNSUPPORTED, "code-block segment too long for the MagSgn staging buffer");
  {
    // One work arena: coefficients, level planes, quad symbols, tile status
    // (256-byte aligned parts).
    auto up256 = [](size_t v) { return (v + 255) & ~(size_t)255; };
    const size_t at_lvl = up256(coef_total * 4), at_sym = at_lvl + up256(lvl_total * 4);
    const size_t at_st = at_sym + up256(std::max<uint64_t>(sym_total, 1) * 4);
    const size_t bytes = at_st + up256(std::max<size_t>(n, 1) * 4);
    if ((e = cudaMallocAsync(&plan->d_work, bytes, s)) != cudaSuccess) return cuda_status(e, "work arena");
    uint8_t* base = static_cast<uint8_t*>(plan->d_work);
    plan->d_coef = reinterpret_cast<int32_t*>(base);
    plan->d_levels = reinterpret_cast<int32_t*>(base + at_lvl);
    plan->d_symbols = reinterpret_cast<uint32_t*>(base + at_sym);
    plan->d_status = reinterpret_cast<uint32_t*>(base + at_st);
  }

  // IDWT rounds: round r-1 holds resolution r of every tile that has it.
  // Rounds 0 .. max_rounds-1 hold 5/3 levels, the next max_rounds the 9/7
  // levels (each round is one launch of the kernel of its transform).
  std::vector<std::vector<IdwtJob>> rounds(2 * (size_t)max_rounds);
  std::vector<PackJob> packs_v[kPackVariants], packs97;
  auto band_ptr = [&](size_t i, uint32_t c, uint32_t bi) -> int32_t* {
    const TileLayout& L = *work[i].L;
    return plan->d_coef + coef_off[i] + (uint64_t)c * L.coef_per_comp + L.bands[bi].coef_off;
  };
  for (size_t i = 0; i < n; ++i) {
    if (plan->status[i] != SGN_OK) continue;
    const TileLayout& L = *work[i].L;
    const uint32_t R = L.levels - L.skipped;
    auto lvl = [&](uint32_t c, uint32_t r) {
      return plan->d_levels + lvl_off[i] + ((uint64_t)c * 2 + (r & 1)) * lvl_size[i];
    };
    auto res_dim = [&](uint32_t r, bool wdim) {
      uint32_t sh = L.levels - r;
      uint64_t v = wdim ? L.width : L.height;
      return (uint32_t)((v + (1ull << sh) - 1) >> sh);
    };
    for (uint32_t c = 0; c < L.ncomp; ++c) {
      uint32_t b0 = L.comp_band_begin[c];
      for (uint32_t r = 1; r < R; ++r) {
        IdwtJob j;
        j.ll = r == 1 ? band_ptr(i, c, b0) : lvl(c, r - 1);
        j.hl = band_ptr(i, c, b0 + 1 + (r - 1) * 3);
        j.lh = band_ptr(i, c, b0 + 2 + (r - 1) * 3);
        j.hh = band_ptr(i, c, b0 + 3 + (r - 1) * 3);
        j.out = lvl(c, r);
        j.w = res_dim(r, true);
        j.h = res_dim(r, false);
        const uint32_t sw = L.reversible ? kIdwtStripW : kStrip97;
        j.strips = (j.w + sw - 1) / sw;
        j.unit_begin = 0;
        j.seg = idwt_segment_rows(j.h);
        j.ll_band = r == 1 ? 1 : 0;
        j.step[0] = L.bands[b0].step;
        for (uint32_t k = 0; k < 3; ++k) j.step[1 + k] = L.bands[b0 + 1 + (r - 1) * 3 + k].step;
        // 9/7 units re-read seven rows: longer segments, except on levels of
        // 256 rows and more, where doubled units left the last wave mostly
        // idle (1.3 waves for 512^2 tiles).
        if (!L.reversible && j.h < 256) j.seg *= 2;
        if (j.w == 0 || j.h == 0) continue;
        j.x_begin = j.y_begin = j.pad = 0;
        j.y_end = j.h;
        if (rois[i].active) {
          // Only the level's window: whole strips from the one holding its
          // first column, rows from an even one.
          const Window& wnd = rois[i].level[r];
          if (wnd.empty()) continue;
          j.x_begin = wnd.x0 - wnd.x0 % sw;
          j.strips = (wnd.x1 - j.x_begin + sw - 1) / sw;
          j.y_begin = wnd.y0 & ~1u;
          j.y_end = wnd.y1;
        }
        rounds[L.reversible ? r - 1 : max_rounds + r - 1].push_back(j);
      }
    }
    // Output surface.
    const TileWork& tw = work[i];
    sgn_surface& sf = plan->surfaces[i];
    sf.width = tw.crop_w;
    sf.height = tw.crop_h;
    sf.format = fmt;
    sf.backend = SGN_BACKEND_CUDA;
    sf.pitch_bytes = (uint64_t)tw.crop_w * bytes_per_pixel(fmt);
    size_t bytes = std::max<size_t>((size_t)sf.pitch_bytes * sf.height, 1);
    void* outp = nullptr;
    if ((e = cudaMallocAsync(&outp, bytes, s)) != cudaSuccess) return cuda_status(e, "surface");
    sf.device_ptr = (uint64_t)(uintptr_t)outp;
    if (tw.crop_w == 0 || tw.crop_h == 0) continue;
    PackJob pj;
    std::memset(&pj, 0, sizeof(pj));
    for (uint32_t c = 0; c < L.ncomp && c < 3; ++c) {
      uint32_t b0 = L.comp_band_begin[c];
      pj.step[c][0] = L.bands[b0].step;
      if (R > 0)
        for (uint32_t k = 0; k < 3; ++k) pj.step[c][1 + k] = L.bands[b0 + 1 + (R - 1) * 3 + k].step;
      if (R == 0) {
        pj.ll[c] = band_ptr(i, c, b0);
      } else {
        pj.ll[c] = R == 1 ? band_ptr(i, c, b0) : lvl(c, R - 1);
        pj.hl[c] = band_ptr(i, c, b0 + 1 + (R - 1) * 3);
        pj.lh[c] = band_ptr(i, c, b0 + 2 + (R - 1) * 3);
        pj.hh[c] = band_ptr(i, c, b0 + 3 + (R - 1) * 3);
      }
    }
    pj.out = (uint8_t*)outp;
    pj.pitch = sf.pitch_bytes;
    pj.w = L.out_w;
    pj.h = L.out_h;
    pj.cx = tw.crop_x;
    pj.cy = tw.crop_y;
    pj.cw = tw.crop_w;
    pj.ch = tw.crop_h;
    pj.lifting = R > 0 ? 1 : 0;
    pj.ncomp = L.ncomp;
    pj.mct = (L.mct && L.ncomp >= 3) ? 1 : 0;
    pj.bit_depth = L.bit_depth;
    pj.fmt = fmt;
    pj.region_conv = tw.region_conv;
    const uint32_t sw = L.reversible ? kIdwtStripW : kStrip97;
    uint32_t ax = tw.crop_x - tw.crop_x % sw, ay = tw.crop_y & ~1u;
    pj.strips = (tw.crop_x + tw.crop_w - ax + sw - 1) / sw;
    // The 9/7 pack keeps the 5/3 segment length although its units re-read
    // seven rows: 128-row segments left a batch of 512^2 tiles at 1.4 waves
    // of units, 64-row ones fill the last wave far better.
    pj.seg = idwt_segment_rows(tw.crop_h);
    pj.ll_band = R <= 1 ? 1 : 0;
    uint32_t segs = (tw.crop_y + tw.crop_h - ay + pj.seg - 1) / pj.seg;
    const uint32_t v = pack_variant(fmt, L.ncomp, L.bit_depth);
    uint32_t& units = L.reversible ? plan->pack_units_v[v] : plan->pack97_ctas;
    pj.unit_begin = units;
    pj.tile = (uint32_t)i;
    units += pj.strips * segs;
    (L.reversible ? packs_v[v] : packs97).push_back(pj);
  }
  // Flatten the rounds.
  std::vector<IdwtJob> idwt;
  for (size_t k = 0; k < rounds.size(); ++k) {
    auto& rj = rounds[k];
    RoundInfo ri{(uint32_t)idwt.size(), (uint32_t)rj.size(), 0, k >= max_rounds ? 1u : 0u};
    for (IdwtJob& j : rj) {
      j.unit_begin = ri.ctas;
      ri.ctas += j.strips * ((j.y_end - j.y_begin + j.seg - 1) / j.seg);
      idwt.push_back(j);
    }
    if (ri.njobs) plan->rounds.push_back(ri);
  }
  std::vector<PackJob> packs;
  for (uint32_t v = 0; v < kPackVariants; ++v) {
    plan->pack_begin[v] = (uint32_t)packs.size();
    plan->npack_v[v] = (uint32_t)packs_v[v].size();
    plan->pack_ctas += plan->pack_units_v[v];
    packs.insert(packs.end(), packs_v[v].begin(), packs_v[v].end());
  }
  plan->npack = (uint32_t)packs.size();
  plan->npack97 = (uint32_t)packs97.size();
  packs.insert(packs.end(), packs97.begin(), packs97.end());
  // The launch shape: an autotuned one when this context has tuned a plan of
  // the same signature (computed on the base tile shapes); its rows per
  // unit are applied to the job tables before they go up.
  LaunchConfig cfg;
  plan->sig = plan_signature(plan);
  bool found_cfg = false;
  {
    std::lock_guard<std::mutex> g(ctx->tune_mu);
    for (auto& t : ctx->tuned)
      if (t.first == plan->sig) cfg = t.second, found_cfg = true;
  }
  if (!found_cfg) {
    // Untuned plans: a plan whose last level (or largest IDWT round) has
    // fewer units than twice the SMs (one tile, a small batch) takes
    // shorter segments, so that more warps share its rows: down to 4 rows
    // for a 512^2 tile (512 units; 16 rows: 0.165 ms plan latency, 4 rows:
    // 0.146 ms).
    const uint32_t sms = (uint32_t)std::max(1, ctx->sm_count);
    auto shift_for = [&](uint32_t units) {
      return 4 * units < sms ? -4 : 2 * units < sms ? -3 : units < sms ? -2 : units < 2 * sms ? -1 : 0;
    };
    uint32_t round_units = 0;
    for (const RoundInfo& r : plan->rounds) round_units = std::max(round_units, r.ctas);
    if (!plan->rounds.empty()) cfg.idwt_seg_shift = shift_for(round_units);
    if (plan->pack_ctas + plan->pack97_ctas) cfg.pack_seg_shift = shift_for(plan->pack_ctas + plan->pack97_ctas);
  }
  if (cfg.idwt_seg_shift || cfg.pack_seg_shift) set_segments(plan, idwt, packs, cfg.idwt_seg_shift, cfg.pack_seg_shift);
  plan->nclassic = ncls;
  size_t cscratch_bytes = 0;
  if (ncls) {
    plan->classic_slot = std::max<uint32_t>(cslot, 1);
    const uint32_t per = classic_threads_per_cta();
    // As many resident threads as the kernel's occupancy allows (every block
    // a thread of its own where possible: the slowest block sets the time).
    plan->classic_ctas = std::min<uint32_t>((ncls + per - 1) / per, (uint32_t)ctx->sm_count * classic_ctas_per_sm());
    cscratch_bytes = (size_t)plan->classic_ctas * per * plan->classic_slot * sizeof(uint16_t);
  }
  plan->nqueues = (uint32_t)plan->rounds.size() + 3 + kPackVariants;

  // Pinned staging: [codestreams unless direct] [HT jobs] [refine] [IDWT] [pack].
  auto up16 = [](size_t v) { return (v + 15) & ~(size_t)15; };
  const size_t at_ht = direct ? 0 : up16(in_total);
  const size_t at_ref = at_ht + up16((size_t)nht * sizeof(HtJob));
  const size_t at_idwt = at_ref + up16((size_t)nref * 4);
  const size_t at_pack = at_idwt + up16(idwt.size() * sizeof(IdwtJob));
  const size_t at_cls = at_pack + up16(packs.size() * sizeof(PackJob));
  const size_t at_cseg = at_cls + up16((size_t)ncls * sizeof(ClassicJob));
  const size_t at_gather = at_cseg + up16((size_t)ncseg * sizeof(ClassicSeg));
  const size_t stage_bytes = at_gather + up16(gather_total);
  if ((e = staging.ensure(stage_bytes)) != cudaSuccess) return cuda_status(e, "pinned staging");
  {
    // One table arena: the job tables in their staging layout (uploaded by
    // one copy), then the work-queue counters and the classic scratch.
    const size_t tab = stage_bytes - at_ht, at_q = up16(tab), at_cs = at_q + up16((size_t)plan->nqueues * 4);
    if ((e = cudaMallocAsync(&plan->d_tables, at_cs + std::max<size_t>(cscratch_bytes, 16), s)) != cudaSuccess)
      return cuda_status(e, "table arena");
    uint8_t* base = static_cast<uint8_t*>(plan->d_tables);
    plan->d_ht = nht ? reinterpret_cast<HtJob*>(base) : nullptr;
    plan->d_refine = nref ? reinterpret_cast<uint32_t*>(base + (at_ref - at_ht)) : nullptr;
    plan->d_idwt = idwt.empty() ? nullptr : reinterpret_cast<IdwtJob*>(base + (at_idwt - at_ht));
    plan->d_pack = packs.empty() ? nullptr : reinterpret_cast<PackJob*>(base + (at_pack - at_ht));
    plan->d_classic = ncls ? reinterpret_cast<ClassicJob*>(base + (at_cls - at_ht)) : nullptr;
    plan->d_csegs = ncls ? reinterpret_cast<ClassicSeg*>(base + (at_cseg - at_ht)) : nullptr;
    plan->d_gather = gather_total ? base + (at_gather - at_ht) : nullptr;
    plan->d_queue = reinterpret_cast<uint32_t*>(base + at_q);
    plan->d_cscratch = cscratch_bytes ? reinterpret_cast<uint16_t*>(base + at_cs) : nullptr;
  }
  uint8_t* st = staging.p;
  HtJob* ht = reinterpret_cast<HtJob*>(st + at_ht);
  uint32_t* refine = reinterpret_cast<uint32_t*>(st + at_ref);
  // HT job table, pass B (per tile, in parallel): each tile writes its jobs
  // at its cursors in the buckets, and the codestream into staging.
  ctx->workers->parallel_for(n, [&](size_t i) {
    if (plan->status[i] != SGN_OK) return;
    if (!direct) std::memcpy(st + in_off[i], datas[i], lens[i]);
    const TileLayout& L = *work[i].L;
    if (L.classic) {
      // Classic blocks: one job each (all-zero blocks too, so that every
      // block's samples are written), segments after the tile's offset.
      ClassicJob* cjobs = reinterpret_cast<ClassicJob*>(st + at_cls);
      uint32_t ccur[kPassBuckets];
      for (uint32_t b = 0; b < kPassBuckets; ++b) ccur[b] = cstart[(size_t)b * n + i];
      ClassicSeg* cs = reinterpret_cast<ClassicSeg*>(st + at_cseg) + cseg_off[i];
      for (size_t k = 0; k < L.segments.size(); ++k) cs[k] = ClassicSeg{L.segments[k].len, L.segments[k].passes};
      uint8_t* g = st + at_gather + gather_off[i];
      for (const auto& op : L.gather) {
        std::memcpy(g, datas[i] + op.first, op.second);
        g += op.second;
      }
      for (const CodeBlock& cb : L.blocks) {
        if (!block_required(rois[i], cb)) continue;
        const Band& b = L.bands[cb.band];
        ClassicJob& j = cjobs[ccur[pass_bucket(cb.passes)]++];
        std::memset(&j, 0, sizeof(j));
        j.src = L.gathered ? (kClassicGathered | (gather_off[i] + cb.cleanup_off)) : in_off[i] + cb.cleanup_off;
        j.dst = coef_off[i] + (uint64_t)b.comp * L.coef_per_comp + b.coef_off + (uint64_t)cb.y0 * b.w + cb.x0;
        j.seg = cseg_off[i] + cb.seg_begin;
        j.tile = (uint32_t)i;
        j.stride = b.w;
        j.w = cb.w;
        j.h = cb.h;
        j.nseg = cb.nseg;
        j.passes = cb.passes;
        j.bitplanes = (uint8_t)(b.nbp > cb.missing_msbs ? b.nbp - cb.missing_msbs : 0);
        j.band_class = b.type == BAND_HL ? ebcot::kHl : b.type == BAND_HH ? ebcot::kHh : ebcot::kLlLh;
        j.style = L.cbstyle;
      }
      return;
    }
    uint32_t cursor[kHtBuckets];
    for (uint32_t b = 0; b < kHtBuckets; ++b) cursor[b] = start[(size_t)b * n + i];
    uint64_t sym = sym_off[i];
    uint32_t rk = ref_off[i];
    for (const CodeBlock& cb : L.blocks) {
      if (!block_required(rois[i], cb)) continue;
      const Band& b = L.bands[cb.band];
      const uint32_t pos = cursor[ht_bucket(cb)]++;
      HtJob& j = ht[pos];
      std::memset(&j, 0, sizeof(j));
      j.src = in_off[i] + cb.cleanup_off;
      j.dst = coef_off[i] + (uint64_t)b.comp * L.coef_per_comp + b.coef_off + (uint64_t)cb.y0 * b.w + cb.x0;
      j.lcup = cb.lcup;
      j.tile = (uint32_t)i;
      j.stride = b.w;
      j.lref = (uint16_t)cb.lref;
      j.w = cb.w;
      j.h = cb.h;
      j.mmsb = cb.missing_msbs;
      j.passes = cb.passes;
      j.nbp = b.nbp;
      j.flags = L.causal ? 1 : 0;
      if (cb.passes) {
        j.sym = sym;
        sym += sym_words(cb.w, cb.h);
      }
      if (cb.passes > 1) refine[rk++] = pos;
    }
  });
  if (!idwt.empty()) std::memcpy(st + at_idwt, idwt.data(), idwt.size() * sizeof(IdwtJob));
  if (!packs.empty()) std::memcpy(st + at_pack, packs.data(), packs.size() * sizeof(PackJob));
  // Uploads: the codestreams (unless they went up directly) and every job
  // table in one copy.
  if (!direct && in_total && (e = cudaMemcpyAsync(plan->d_input, st, in_total, cudaMemcpyHostToDevice, s)) != cudaSuccess)
    return cuda_status(e, "plan upload");
  if (stage_bytes > at_ht &&
      (e = cudaMemcpyAsync(plan->d_tables, st + at_ht, stage_bytes - at_ht, cudaMemcpyHostToDevice, s)) != cudaSuccess)
    return cuda_status(e, "plan upload");
  // The staging buffer is reused by the next call: finish the copies now
  // (callers that reuse it only after the plan has run pass sync_uploads false).
  if (sync_uploads && (e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_status(e, "plan upload");
  plan->launches = (plan->nht ? 2 : 0) + (plan->nref ? 1 : 0) + (plan->nclassic ? 1 : 0) + plan->rounds.size() +
                   (plan->npack97 ? 1 : 0);
  for (uint32_t v = 0; v < kPackVariants; ++v) plan->launches += plan->npack_v[v] ? 1 : 0;
  for (auto& sf : plan->surfaces) sf.kernel_dispatches = plan->launches;
  // Work-queue counters and the launch shape (an autotuned one when this
  // context has tuned a plan of the same signature).
  plan->h_idwt = std::move(idwt);
  plan->h_pack = std::move(packs);
  return apply_config(ctx, plan, cfg);
}

}  // namespace

uint64_t plan_signature(const sgn_plan* p) {
  auto lg = [](uint64_t v) {
    uint64_t k = 0;
    while (v > 1) {
      v >>= 1;
      ++k;
    }
    return k;
  };
  return (uint64_t)p->format | (lg(p->nht + 1) << 4) | (lg(p->max_w) << 10) | (lg(p->ms_words) << 14) |
         (lg(p->pack_ctas + 1) << 20) | ((uint64_t)p->rounds.size() << 26) | ((uint64_t)(p->nref > 0) << 31) |
         ((uint64_t)lg(p->pack97_ctas + 1) << 32);
}

namespace {

uint32_t scaled_seg(uint32_t base, int shift) {
  uint32_t s = shift > 0 ? base << shift : shift < 0 ? base >> -shift : base;
  return std::max<uint32_t>(2, s & ~1u);
}

}  // namespace

void set_segments(sgn_plan* p, std::vector<IdwtJob>& idwt, std::vector<PackJob>& packs, int ishift, int pshift) {
  for (RoundInfo& r : p->rounds) {
    r.ctas = 0;
    for (uint32_t k = r.job_begin; k < r.job_begin + r.njobs; ++k) {
      IdwtJob& j = idwt[k];
      // The build's rule: 9/7 units re-read seven rows, so levels under 256
      // rows take doubled segments.
      const uint32_t base = idwt_segment_rows(j.h) * (r.irreversible && j.h < 256 ? 2 : 1);
      j.seg = scaled_seg(base, ishift);
      j.unit_begin = r.ctas;
      r.ctas += j.strips * ((j.y_end - j.y_begin + j.seg - 1) / j.seg);
    }
  }
  auto units = [](PackJob& j) { return j.strips * ((j.cy + j.ch - (j.cy & ~1u) + j.seg - 1) / j.seg); };
  p->pack_ctas = 0;
  for (uint32_t v = 0; v < kPackVariants; ++v) {
    p->pack_units_v[v] = 0;
    for (uint32_t k = p->pack_begin[v]; k < p->pack_begin[v] + p->npack_v[v]; ++k) {
      PackJob& j = packs[k];
      j.seg = scaled_seg(idwt_segment_rows(j.ch), pshift);
      j.unit_begin = p->pack_units_v[v];
      p->pack_units_v[v] += units(j);
    }
    p->pack_ctas += p->pack_units_v[v];
  }
  p->pack97_ctas = 0;
  for (uint32_t k = p->npack; k < p->npack + p->npack97; ++k) {
    PackJob& j = packs[k];
    j.seg = scaled_seg(idwt_segment_rows(j.ch), pshift);
    j.unit_begin = p->pack97_ctas;
    p->pack97_ctas += units(j);
  }
}

sgn_status apply_config(sgn_ctx* ctx, sgn_plan* p, const LaunchConfig& in) {
  LaunchConfig c = in;
  int ms = 0, idwt = 0, pack = 0;
  cudaError_t e = ht_magsgn_occupancy(p->ms_words, p->max_w, c.ms_warps ? c.ms_warps : 8, &ms);
  if (e == cudaSuccess) e = idwt_pack_occupancy(p->format < 5 ? p->format : 1, &idwt, &pack);
  if (e != cudaSuccess) return cuda_status(e, "occupancy query");
  if (c.vlc_lanes == 0) {
    // Blocks per VLC warp by default: 32 once the batch has that many blocks
    // for every scheduler (four per SM), fewer for smaller plans, so each
    // block's serial chain runs in a warp with fewer other blocks' paths.
    const uint64_t per_sched = p->nht / (4ull * (uint64_t)std::max(1, ctx->sm_count));
    uint32_t lanes = 1;
    while (lanes < 32 && (uint64_t)lanes * 2 <= per_sched) lanes *= 2;
    c.vlc_lanes = lanes;
  }
  if (c.ht_fused == 2) {
    // Plans of at most six blocks per SM take the fused form: each block's
    // MagSgn follows its own chain instead of the slowest chain of the plan.
    // With more, the MagSgn warps take issue slots from the chains running
    // beside them on the same SMs (one-tile plans, two kernels -> fused:
    // 210 blocks 0.175 -> 0.138 ms, 777 blocks 0.087 -> 0.075 ms, 786
    // 0.217 -> 0.209 ms; 1,027 blocks 0.224 -> 0.253 ms, 3,081 blocks 0.118
    // -> 0.183 ms).
    c.ht_fused = c.vlc_lanes == 1 && p->nht <= 6ull * (uint64_t)std::max(1, ctx->sm_count) &&
                         ht_magsgn_smem_bytes(p->ms_words, p->max_w, 1) <= 200 * 1024
                     ? 1
                     : 0;
  }
  c.ms_ctas = (uint32_t)std::max(1, ms * ctx->sm_count);
  c.idwt_ctas = (uint32_t)std::max(1, idwt * ctx->sm_count);
  c.pack_ctas = (uint32_t)std::max(1, pack * ctx->sm_count);
  p->cfg = c;
  if (p->graph) {
    cudaGraphExecDestroy(p->graph);
    p->graph = nullptr;
  }
  return SGN_OK;
}

cudaError_t launch_classic_blocks(const sgn_plan* p, cudaStream_t s) {
  return launch_classic(p->d_classic, p->d_csegs, p->nclassic, p->d_input, p->d_gather, p->d_coef, p->d_cscratch,
                        p->classic_slot, p->classic_ctas, p->d_queue + p->rounds.size() + 2 + kPackVariants, s);
}

cudaError_t launch_round(const sgn_plan* p, size_t k, cudaStream_t s, bool queued, uint32_t ctas, bool lean) {
  const RoundInfo& r = p->rounds[k];
  uint32_t* q = queued ? p->d_queue + 1 + k : nullptr;
  return r.irreversible ? launch_idwt97_level(p->d_idwt + r.job_begin, r.njobs, r.ctas, s, q, ctas)
                        : launch_idwt_level(p->d_idwt + r.job_begin, r.njobs, r.ctas, s, q, ctas, lean);
}

cudaError_t launch_packs(const sgn_plan* p, cudaStream_t s, bool queued, uint32_t ctas) {
  // Counters: one per reversible variant, then the 9/7 pack.
  uint32_t* q = queued ? p->d_queue + 1 + p->rounds.size() : nullptr;
  cudaError_t e = cudaSuccess;
  for (uint32_t v = 0; v < kPackVariants && e == cudaSuccess; ++v)
    e = launch_pack(p->d_pack + p->pack_begin[v], p->npack_v[v], p->pack_units_v[v], p->format, v, s,
                    q ? q + v : nullptr, ctas);
  if (e == cudaSuccess)
    e = launch_pack97(p->d_pack + p->npack, p->npack97, p->pack97_ctas, p->format, s,
                      q ? q + kPackVariants : nullptr, ctas);
  return e;
}

void free_plan_buffers(sgn_plan* p, cudaStream_t s) {
  if (p->graph) {
    cudaGraphExecDestroy(p->graph);
    p->graph = nullptr;
  }
  void* ptrs[] = {p->owns_input ? p->d_input : nullptr, p->d_work, p->d_tables};
  for (void* q : ptrs)
    if (q) cudaFreeAsync(q, s);
  p->d_input = nullptr;
  p->d_work = p->d_tables = nullptr;
  p->d_coef = p->d_levels = nullptr;
  p->d_symbols = nullptr;
  p->d_status = nullptr;
  p->d_ht = nullptr;
  p->d_refine = nullptr;
  p->d_classic = nullptr;
  p->d_csegs = nullptr;
  p->d_cscratch = nullptr;
  p->d_gather = nullptr;
  p->d_idwt = nullptr;
  p->d_pack = nullptr;
  p->d_queue = nullptr;
}

void release_plan(sgn_plan* p, cudaStream_t s) {
  for (auto& sf : p->surfaces)
    if (sf.device_ptr) cudaFreeAsync((void*)(uintptr_t)sf.device_ptr, s);
  p->surfaces.clear();
  free_plan_buffers(p, s);
}

sgn_status execute(sgn_plan* p, cudaStream_t s, cudaEvent_t* ev) {
  cudaError_t e;
  const LaunchConfig& c = p->cfg;
  auto mark = [&](int k) { return ev ? cudaEventRecord(ev[k], s) : cudaSuccess; };
  if (p->n && (e = cudaMemsetAsync(p->d_status, 0, p->n * sizeof(uint32_t), s)) != cudaSuccess)
    return cuda_status(e, "status reset");
  if (p->d_queue && (e = cudaMemsetAsync(p->d_queue, 0, p->nqueues * sizeof(uint32_t), s)) != cudaSuccess)
    return cuda_status(e, "work queue reset");
  if ((e = mark(0)) != cudaSuccess) return cuda_status(e, "event record");
  if (c.ht_fused == 1) {
    // Both cleanup passes in one launch (its time shows as the VLC stage).
    if ((e = launch_ht_fused(p->d_ht, p->nht, p->d_input, p->d_symbols, p->d_coef, p->d_status, p->ms_words,
                             p->max_w, s, c.vlc_outline != 0)) != cudaSuccess)
      return cuda_status(e, "HT cleanup launch");
    if ((e = mark(1)) != cudaSuccess) return cuda_status(e, "event record");
  } else {
    if ((e = launch_ht_vlc(p->d_ht, p->nht, p->d_input, p->d_symbols, s, c.vlc_threads, c.vlc_lanes,
                           c.vlc_outline != 0)) != cudaSuccess)
      return cuda_status(e, "HT VLC launch");
    if ((e = mark(1)) != cudaSuccess) return cuda_status(e, "event record");
    if ((e = launch_ht_magsgn(p->d_ht, p->nht, p->d_input, p->d_symbols, p->d_coef, p->d_status, p->ms_words,
                              p->max_w, s, c.ms_warps, c.ms_gran ? p->d_queue : nullptr, c.ms_gran, c.ms_ctas,
                              p->nsingle)) != cudaSuccess)
      return cuda_status(e, "HT MagSgn launch");
  }
  if ((e = mark(2)) != cudaSuccess) return cuda_status(e, "event record");
  if ((e = launch_ht_refine(p->d_ht, p->d_refine, p->nref, p->d_input, p->d_coef, p->d_status, s)) != cudaSuccess)
    return cuda_status(e, "HT refinement launch");
  if ((e = launch_classic_blocks(p, s)) != cudaSuccess) return cuda_status(e, "classic block launch");
  if ((e = mark(3)) != cudaSuccess) return cuda_status(e, "event record");
  for (size_t k = 0; k < p->rounds.size(); ++k)
    if ((e = launch_round(p, k, s, c.idwt_queue != 0, c.idwt_ctas, c.idwt_lean != 0)) != cudaSuccess)
      return cuda_status(e, "IDWT launch");
  if ((e = mark(4)) != cudaSuccess) return cuda_status(e, "event record");
  if ((e = launch_packs(p, s, c.pack_queue != 0, c.pack_ctas)) != cudaSuccess) return cuda_status(e, "pack launch");
  if ((e = mark(5)) != cudaSuccess) return cuda_status(e, "event record");
  return SGN_OK;
}

// Re-executions replay the plan as one CUDA graph, captured on the second
// execution (the first one runs eagerly: one-shot plans never pay for a
// capture).
sgn_status execute_graph(sgn_plan* p, cudaStream_t s) {
  ++p->executions;
  if (!p->graph && p->executions >= 2) {
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_status(e, "graph capture");
    sgn_status st = execute(p, s);
    e = cudaStreamEndCapture(s, &g);
    if (st != SGN_OK) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&p->graph, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      p->graph = nullptr;
      return cuda_status(e, "graph instantiate");
    }
  }
  if (p->graph) return cuda_status(cudaGraphLaunch(p->graph, s), "graph launch");
  return execute(p, s);
}

sgn_status wait_plan(sgn_plan* p, cudaStream_t s, sgn_status* per_tile, size_t* first_failing) {
  cudaError_t e;
  p->h_status.assign(p->n, 0);
  if (p->n && (e = cudaMemcpyAsync(p->h_status.data(), p->d_status, p->n * 4, cudaMemcpyDeviceToHost, s)) !=
                  cudaSuccess)
    return cuda_status(e, "status download");
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_status(e, "decode");
  size_t first = SIZE_MAX;
  sgn_status first_status = SGN_OK;
  for (size_t i = 0; i < p->n; ++i) {
    sgn_status st = p->status[i];
    if (st == SGN_OK && p->h_status[i] != 0) st = SGN_ERR_DECODE;
    if (per_tile) per_tile[i] = st;
    if (st != SGN_OK && first == SIZE_MAX) {
      first = i;
      first_status = st;
    }
  }
  if (first_failing) *first_failing = first;
  if (first_status != SGN_OK) set_error(first_status, "tile decode failed");
  return first_status;
}

sgn_status build_plan(sgn_ctx* ctx, cudaStream_t s, PinnedBuffer& staging, const uint8_t* const* datas,
                      const size_t* lens, size_t n, uint32_t fmt, const sgn_request* reqs, sgn_plan* plan,
                      const uint8_t* resident_arena, const uint64_t* resident_off,
                      const TileLayout* const* layouts, bool sync_uploads) {
  return build_plan_impl(ctx, s, staging, datas, lens, n, fmt, reqs, plan, resident_arena, resident_off, layouts,
                         sync_uploads);
}

}  // namespace rt
}  // namespace sgn

extern "C" {

const char* sgn_last_error_message(void) { return g_msg; }

sgn_status sgn_ctx_create(int device, sgn_ctx** out) {
  if (!out) return set_error(SGN_ERR_INVALID_ARGUMENT, "null output");
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    return set_error(SGN_ERR_CUDA_UNAVAILABLE, "CUDA is unavailable on this host");
  }
  if (device < 0 || device >= count) return set_error(SGN_ERR_INVALID_ARGUMENT, "device index out of range");
  if ((e = cudaSetDevice(device)) != cudaSuccess) return cuda_status(e, "cudaSetDevice");
  sgn_ctx* c = new sgn_ctx();
  c->device = device;
  cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
  if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) {
    delete c;
    return cuda_status(e, "cudaStreamCreate");
  }
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  cudaError_t tables_err = sgn::ensure_device_init(device);
  if (tables_err != cudaSuccess) {
    cudaStreamDestroy(c->stream);
    delete c;
    return cuda_status(tables_err, "HT table upload");
  }
  for (auto& l : c->lanes)
    if ((e = cudaStreamCreateWithFlags(&l, cudaStreamNonBlocking)) != cudaSuccess) {
      for (auto& x : c->lanes)
        if (x) cudaStreamDestroy(x);
      cudaStreamDestroy(c->stream);
      delete c;
      return cuda_status(e, "cudaStreamCreate");
    }
  unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  c->workers = new Workers(std::min(hw, 32u) - 1);
  *out = c;
  return SGN_OK;
}

void sgn_ctx_destroy(sgn_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  cudaStreamDestroy(ctx->stream);
  for (auto& l : ctx->lanes) {
    cudaStreamSynchronize(l);
    cudaStreamDestroy(l);
  }
  delete ctx->workers;
  delete ctx;
}

uint64_t sgn_ctx_submissions(const sgn_ctx* ctx) { return ctx ? ctx->submissions.load() : 0; }

void* sgn_ctx_stream(sgn_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

void sgn_ebcot_tables(uint8_t* zc_ll_lh, uint8_t* zc_hl, uint8_t* zc_hh, uint8_t* sc_label, uint8_t* sc_xor,
                      uint8_t* qe_records) {
  using namespace sgn::ebcot;
  for (int n = 0; n < 256; ++n) {
    zc_ll_lh[n] = zc_context((uint8_t)n, kLlLh);
    zc_hl[n] = zc_context((uint8_t)n, kHl);
    zc_hh[n] = zc_context((uint8_t)n, kHh);
    // Patterns with both bits of a neighbour's field set cannot occur; the
    // reference's table holds (0, 0) there.
    bool possible = true;
    for (int sh = 0; sh < 8; sh += 2) possible = possible && ((n >> sh) & 3) != 3;
    sc_label[n] = sc_xor[n] = 0;
    if (possible) sc_context((uint8_t)n, sc_label[n], sc_xor[n]);
  }
  for (int k = 0; k < 47; ++k) {
    qe_records[5 * k] = (uint8_t)(kQe[k] & 0xFF);
    qe_records[5 * k + 1] = (uint8_t)(kQe[k] >> 8);
    qe_records[5 * k + 2] = kNmps[k];
    qe_records[5 * k + 3] = kNlps[k];
    qe_records[5 * k + 4] = kSwitch[k];
  }
}

void sgn_ht_lookup_tables(uint16_t* vlc0, uint16_t* vlc1, uint16_t* uvlc0, uint16_t* uvlc1) {
  HtDecodeTables t;
  build_decode_tables(t);
  if (vlc0) std::memcpy(vlc0, t.vlc[0], sizeof(t.vlc[0]));
  if (vlc1) std::memcpy(vlc1, t.vlc[1], sizeof(t.vlc[1]));
  if (uvlc0) std::memcpy(uvlc0, t.uvlc0, sizeof(t.uvlc0));
  if (uvlc1) std::memcpy(uvlc1, t.uvlc1, sizeof(t.uvlc1));
}

sgn_status sgn_j2k_inspect(const uint8_t* data, size_t len, sgn_info* out) {
  if (!data || !out) return set_error(SGN_ERR_INVALID_ARGUMENT, "null argument");
  try {
    Info i = inspect_codestream(data, len);
    *out = {i.width, i.height, i.components, i.bit_depth, i.levels, i.tiles, i.ht, i.reversible, i.mct};
    return SGN_OK;
  } catch (const ParseError& e) {
    return set_error(e.status, e.message.c_str());
  }
}

// Backend routing of wrap_surface / validate_surface_request
// (crates/signinum-j2k-cuda/src/runtime.rs:19-57): Cuda decodes here; Cpu and
// Auto are the adapter's host-surface branch, which never initialises CUDA
// (session.rs:32-38), so they return before any CUDA call; Metal is an
// unsupported backend.
static sgn_status check_backend(uint32_t backend) {
  if (backend == SGN_BACKEND_CUDA) return SGN_OK;
  if (backend == SGN_BACKEND_CPU || backend == SGN_BACKEND_AUTO)
    return set_error(SGN_ERR_HOST_BACKEND,
                     "Cpu and Auto requests take the adapter's host-surface branch; this library decodes on CUDA only");
  if (backend == SGN_BACKEND_METAL)
    return set_error(SGN_ERR_UNSUPPORTED_BACKEND, "backend request Metal is not supported by signinum-j2k-cuda");
  return set_error(SGN_ERR_INVALID_ARGUMENT, "unknown backend request");
}

sgn_status sgn_plan_create(sgn_ctx* ctx, const uint8_t* const* datas, const size_t* lens, size_t n, uint32_t format,
                           const sgn_request* requests, sgn_plan** out, sgn_status* per_tile) {
  if (!ctx || !out || (n && (!datas || !lens))) return set_error(SGN_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  std::lock_guard<std::mutex> g(ctx->mu);
  cudaSetDevice(ctx->device);
  sgn_plan* p = new sgn_plan();
  sgn_status st;
  try {
    st = build_plan(ctx, ctx->stream, ctx->staging, datas, lens, n, format, requests, p);
  } catch (const std::bad_alloc&) {
    st = set_error(SGN_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
  if (st != SGN_OK) {
    for (auto& sf : p->surfaces)
      if (sf.device_ptr) cudaFreeAsync((void*)(uintptr_t)sf.device_ptr, ctx->stream);
    free_plan_buffers(p, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    delete p;
    return st;
  }
  if (per_tile)
    for (size_t i = 0; i < n; ++i) per_tile[i] = p->status[i];
  *out = p;
  return SGN_OK;
}

sgn_status sgn_plan_execute_async(sgn_ctx* ctx, sgn_plan* plan) {
  if (!ctx || !plan) return set_error(SGN_ERR_INVALID_ARGUMENT, "null argument");
  cudaSetDevice(ctx->device);
  return execute_graph(plan, ctx->stream);
}

sgn_status sgn_plan_execute_timed(sgn_ctx* ctx, sgn_plan* p, float* stage_ms) {
  if (!ctx || !p || !stage_ms) return set_error(SGN_ERR_INVALID_ARGUMENT, "null argument");
  cudaSetDevice(ctx->device);
  cudaEvent_t ev[6];
  for (auto& e : ev) cudaEventCreate(&e);
  sgn_status st = execute(p, ctx->stream, ev);
  cudaError_t e = st == SGN_OK ? cudaEventSynchronize(ev[5]) : cudaSuccess;
  if (st == SGN_OK && e == cudaSuccess) {
    for (int i = 0; i < 5; ++i) cudaEventElapsedTime(&stage_ms[i], ev[i], ev[i + 1]);
    cudaEventElapsedTime(&stage_ms[5], ev[0], ev[5]);
  }
  for (auto& x : ev) cudaEventDestroy(x);
  if (st != SGN_OK) return st;
  return cuda_status(e, "timed execute");
}

}  // extern "C"

namespace {

// Mean device time (ms) of `reps` runs of one stage, CUDA events on s.
template <typename F>
float time_stage(cudaStream_t s, uint32_t reps, F launch, cudaError_t& err) {
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  float ms = 0.f;
  if (err == cudaSuccess) err = launch();  // warm-up
  if (err == cudaSuccess) err = cudaEventRecord(a, s);
  for (uint32_t r = 0; r < reps && err == cudaSuccess; ++r) err = launch();
  if (err == cudaSuccess) err = cudaEventRecord(b, s);
  if (err == cudaSuccess) err = cudaEventSynchronize(b);
  if (err == cudaSuccess) cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return reps ? ms / reps : ms;
}

}  // namespace

extern "C" {

sgn_status sgn_plan_set_launch_shape(sgn_ctx* ctx, sgn_plan* p, uint32_t vlc_threads, uint32_t ms_warps,
                                     uint32_t ms_blocks_per_grab, uint32_t dwt_queue) {
  if (!ctx || !p) return set_error(SGN_ERR_INVALID_ARGUMENT, "null argument");
  if (vlc_threads < 32 || vlc_threads > 128 || vlc_threads % 32 || ms_warps < 1 || ms_warps > 8 || dwt_queue > 3)
    return set_error(SGN_ERR_INVALID_ARGUMENT, "launch shape out of range");
  std::lock_guard<std::mutex> g(ctx->mu);
  cudaSetDevice(ctx->device);
  LaunchConfig c;
  c.vlc_threads = vlc_threads;
  c.ms_warps = ms_warps;
  c.ms_gran = ms_blocks_per_grab;
  c.idwt_queue = dwt_queue & 1;
  c.pack_queue = (dwt_queue >> 1) & 1;
  // The tile shape stays the one the plan's job tables were built with.
  c.idwt_seg_shift = p->cfg.idwt_seg_shift;
  c.pack_seg_shift = p->cfg.pack_seg_shift;
  return apply_config(ctx, p, c);
}

sgn_status sgn_plan_set_cleanup_form(sgn_ctx* ctx, sgn_plan* p, uint32_t fused) {
  if (!ctx || !p) return set_error(SGN_ERR_INVALID_ARGUMENT, "null argument");
  if (fused > 2) return set_error(SGN_ERR_INVALID_ARGUMENT, "cleanup form out of range");
  if (fused == 1 && (p->nht > kFusedMaxBlocks || ht_magsgn_smem_bytes(p->ms_words, p->max_w, 1) > 200 * 1024))
    return set_error(SGN_ERR_UNSUPPORTED, "plan too large for the fused cleanup form");
  std::lock_guard<std::mutex> g(ctx->mu);
  cudaSetDevice(ctx->device);
  LaunchConfig c = p->cfg;
  c.ht_fused = fused;
  return apply_config(ctx, p, c);
}

sgn_status sgn_plan_set_tile_shape(sgn_ctx* ctx, sgn_plan* p, int32_t idwt_seg_shift, int32_t pack_seg_shift) {
  if (!ctx || !p) return set_error(SGN_ERR_INVALID_ARGUMENT, "null argument");
  if (idwt_seg_shift < -4 || idwt_seg_shift > 1 || pack_seg_shift < -4 || pack_seg_shift > 1)
    return set_error(SGN_ERR_INVALID_ARGUMENT, "tile shape shift out of range");
  std::lock_guard<std::mutex> g(ctx->mu);
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  set_segments(p, p->h_idwt, p->h_pack, idwt_seg_shift, pack_seg_shift);
  cudaError_t e = cudaSuccess;
  if (!p->h_idwt.empty())
    e = cudaMemcpyAsync(p->d_idwt, p->h_idwt.data(), p->h_idwt.size() * sizeof(IdwtJob), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && !p->h_pack.empty())
    e = cudaMemcpyAsync(p->d_pack, p->h_pack.data(), p->h_pack.size() * sizeof(PackJob), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e, "tile shape upload");
  LaunchConfig c = p->cfg;
  c.idwt_seg_shift = idwt_seg_shift;
  c.pack_seg_shift = pack_seg_shift;
  return apply_config(ctx, p, c);
}

sgn_status sgn_plan_autotune(sgn_ctx* ctx, sgn_plan* p, uint32_t reps, sgn_tune_report* out) {
  if (!ctx || !p) return set_error(SGN_ERR_INVALID_ARGUMENT, "null argument");
  std::lock_guard<std::mutex> g(ctx->mu);
  cudaSetDevice(ctx->device);
  if (reps == 0) reps = 5;
  cudaStream_t s = ctx->stream;
  cudaError_t e = cudaSuccess;
  // Inputs of every stage in place: one full execution with the current shape.
  sgn_status st = execute(p, s);
  if (st != SGN_OK) return st;
  const LaunchConfig base = p->cfg;
  sgn_tune_report rep;
  std::memset(&rep, 0, sizeof(rep));
  // VLC pass: threads per CTA, code blocks per warp, and the bit readers'
  // refills inline or out of line (inline suits batches of few blocks per
  // lane, out of line the large ones, whose warps diverge more).
  const uint32_t vlc_c[] = {64, 128};
  float best_vlc = 1e30f;
  uint32_t vlc_threads = base.vlc_threads, vlc_lanes = p->cfg.vlc_lanes, vlc_outline = base.vlc_outline;
  for (uint32_t o = 0; o < 2; ++o)
    for (uint32_t t : vlc_c)
      for (uint32_t l = 32; l >= 1; l /= 2) {
        if (l < 32 && (uint64_t)l * 64 > p->nht) continue;  // fewer blocks per warp only pays for small plans
        float ms = time_stage(
            s, reps, [&] { return launch_ht_vlc(p->d_ht, p->nht, p->d_input, p->d_symbols, s, t, l, o != 0); }, e);
        if (t == 128 && l == p->cfg.vlc_lanes && o == base.vlc_outline) rep.vlc_ms_default = ms;
        if (e == cudaSuccess && ms < best_vlc) best_vlc = ms, vlc_threads = t, vlc_lanes = l, vlc_outline = o;
      }
  // MagSgn pass: warps per CTA, grid or queue (blocks per grab).
  struct MsC {
    uint32_t warps, gran;
  } ms_c[] = {{8, 0}, {4, 0}, {8, 1}, {8, 4}, {4, 1}};
  float best_ms = 1e30f;
  LaunchConfig cfg = base;
  uint32_t ms_warps = base.ms_warps, ms_gran = base.ms_gran;
  for (const MsC& m : ms_c) {
    LaunchConfig tc = base;
    tc.ms_warps = m.warps;
    if (apply_config(ctx, p, tc) != SGN_OK) continue;
    const uint32_t ctas = p->cfg.ms_ctas;
    float ms = time_stage(s, reps, [&] {
      cudaError_t x = cudaMemsetAsync(p->d_queue, 0, sizeof(uint32_t), s);
      if (x != cudaSuccess) return x;
      return launch_ht_magsgn(p->d_ht, p->nht, p->d_input, p->d_symbols, p->d_coef, p->d_status, p->ms_words,
                              p->max_w, s, m.warps, m.gran ? p->d_queue : nullptr, m.gran, ctas, p->nsingle);
    }, e);
    if (m.warps == 8 && m.gran == 0) rep.ms_ms_default = ms;
    if (e == cudaSuccess && ms < best_ms) best_ms = ms, ms_warps = m.warps, ms_gran = m.gran;
  }
  // Both cleanup passes fused (a CTA per block) against the best separate
  // pair, on plans small enough for it.
  uint32_t ht_fused = 0, fused_outline = vlc_outline;
  if (p->nht && p->nht <= kFusedMaxBlocks && ht_magsgn_smem_bytes(p->ms_words, p->max_w, 1) <= 200 * 1024) {
    float best_fused = 1e30f;
    for (uint32_t o = 0; o < 2; ++o) {
      float ms = time_stage(s, reps, [&] {
        return launch_ht_fused(p->d_ht, p->nht, p->d_input, p->d_symbols, p->d_coef, p->d_status, p->ms_words,
                               p->max_w, s, o != 0);
      }, e);
      if (e == cudaSuccess && ms < best_fused) best_fused = ms, fused_outline = o;
    }
    if (best_fused < best_vlc + best_ms) ht_fused = 1;
    rep.fused_ms = best_fused;
  }
  // IDWT levels and pack, each: one unit per warp or persistent warps on a
  // queue, and the DWT tile shape (rows per unit: the base rule scaled by
  // 2^shift, shift -4 to 1; the strip is 128 columns, four per lane).
  auto set_shape = [&](int is, int ps) {
    set_segments(p, p->h_idwt, p->h_pack, is, ps);
    cudaError_t x = cudaSuccess;
    if (!p->h_idwt.empty())
      x = cudaMemcpyAsync(p->d_idwt, p->h_idwt.data(), p->h_idwt.size() * sizeof(IdwtJob), cudaMemcpyHostToDevice, s);
    if (x == cudaSuccess && !p->h_pack.empty())
      x = cudaMemcpyAsync(p->d_pack, p->h_pack.data(), p->h_pack.size() * sizeof(PackJob), cudaMemcpyHostToDevice, s);
    if (x == cudaSuccess) x = cudaStreamSynchronize(s);
    return x;
  };
  float best_idwt = 1e30f, best_pack = 1e30f, idwt_default = 0.f, pack_default = 0.f;
  uint32_t idwt_queue = 0, pack_queue = 0, idwt_lean = 0;
  int idwt_shift = 0, pack_shift = 0;
  const uint32_t ictas = p->cfg.idwt_ctas, pctas = p->cfg.pack_ctas;
  for (int sh = -4; sh <= 1 && e == cudaSuccess; ++sh) {
    if ((e = set_shape(sh, sh)) != cudaSuccess) break;
    // IDWT: grid form (at three and at four CTAs per SM) or queue.
    for (uint32_t f = 0; f < 3; ++f) {
      const bool queued = f == 2, lean = f == 1;
      const float ms = time_stage(s, reps, [&] {
        cudaError_t x = cudaMemsetAsync(p->d_queue, 0, p->nqueues * sizeof(uint32_t), s);
        for (size_t k = 0; k < p->rounds.size() && x == cudaSuccess; ++k) x = launch_round(p, k, s, queued, ictas, lean);
        return x;
      }, e);
      if (f == 0 && sh == base.idwt_seg_shift) idwt_default = ms;
      if (e == cudaSuccess && ms < best_idwt) best_idwt = ms, idwt_queue = queued, idwt_lean = lean, idwt_shift = sh;
    }
    for (uint32_t q = 0; q < 2; ++q) {
      float ms = time_stage(s, reps, [&] {
        cudaError_t x = cudaMemsetAsync(p->d_queue, 0, p->nqueues * sizeof(uint32_t), s);
        if (x == cudaSuccess) x = launch_packs(p, s, q != 0, pctas);
        return x;
      }, e);
      if (q == 0 && sh == base.pack_seg_shift) pack_default = ms;
      if (e == cudaSuccess && ms < best_pack) best_pack = ms, pack_queue = q, pack_shift = sh;
    }
  }
  rep.dwt_ms_default = idwt_default + pack_default;
  const float best_dwt = best_idwt + best_pack;
  if (e == cudaSuccess) e = set_shape(idwt_shift, pack_shift);
  if (e != cudaSuccess) {
    set_shape(base.idwt_seg_shift, base.pack_seg_shift);
    apply_config(ctx, p, base);
    return cuda_status(e, "autotune");
  }
  cfg.idwt_seg_shift = idwt_shift;
  cfg.pack_seg_shift = pack_shift;
  cfg.vlc_threads = vlc_threads;
  cfg.vlc_lanes = vlc_lanes;
  cfg.vlc_outline = ht_fused ? fused_outline : vlc_outline;
  cfg.ht_fused = ht_fused;
  cfg.ms_warps = ms_warps;
  cfg.ms_gran = ms_gran;
  cfg.idwt_queue = idwt_queue;
  cfg.idwt_lean = idwt_lean;
  cfg.pack_queue = pack_queue;
  st = apply_config(ctx, p, cfg);
  if (st != SGN_OK) return st;
  // Leave the plan's outputs consistent (the refinement pass is not
  // idempotent when a stage runs alone).
  st = execute(p, s);
  if (st == SGN_OK) st = cuda_status(cudaStreamSynchronize(s), "autotune");
  {
    const uint64_t sig = p->sig;
    std::lock_guard<std::mutex> tg(ctx->tune_mu);
    bool found = false;
    for (auto& t : ctx->tuned)
      if (t.first == sig) t.second = p->cfg, found = true;
    if (!found) ctx->tuned.emplace_back(sig, p->cfg);
  }
  rep.vlc_threads = cfg.vlc_threads;
  rep.vlc_lanes = cfg.vlc_lanes;
  rep.vlc_outline = cfg.vlc_outline;
  rep.ht_fused = cfg.ht_fused;
  rep.idwt_lean = cfg.idwt_lean;
  rep.ms_warps = cfg.ms_warps;
  rep.ms_blocks_per_grab = cfg.ms_gran;
  rep.dwt_queue = cfg.idwt_queue | (cfg.pack_queue << 1);
  rep.idwt_seg_shift = cfg.idwt_seg_shift;
  rep.pack_seg_shift = cfg.pack_seg_shift;
  rep.vlc_ms = best_vlc;
  rep.ms_ms = best_ms;
  rep.dwt_ms = best_dwt;
  if (out) *out = rep;
  return st;
}

sgn_status sgn_plan_wait(sgn_ctx* ctx, sgn_plan* plan, sgn_status* per_tile, size_t* first_failing) {
  if (!ctx || !plan) return set_error(SGN_ERR_INVALID_ARGUMENT, "null argument");
  cudaSetDevice(ctx->device);
  return wait_plan(plan, ctx->stream, per_tile, first_failing);
}

sgn_status sgn_plan_surfaces(const sgn_plan* plan, sgn_surface* outs, size_t n) {
  if (!plan || (n && !outs) || n > plan->n) return set_error(SGN_ERR_INVALID_ARGUMENT, "bad arguments");
  for (size_t i = 0; i < n; ++i) outs[i] = plan->surfaces[i];
  return SGN_OK;
}

uint64_t sgn_plan_kernel_launches(const sgn_plan* plan) { return plan ? plan->launches : 0; }

sgn_status sgn_plan_tile_coefficients(sgn_ctx* ctx, const sgn_plan* plan, size_t tile, int32_t* out, size_t cap,
                                      size_t* count) {
  if (!ctx || !plan || tile >= plan->n || (!out && cap)) return set_error(SGN_ERR_INVALID_ARGUMENT, "bad arguments");
  size_t elems = plan->tile_coef_elems[tile];
  if (count) *count = elems;
  if (elems > cap) return set_error(SGN_ERR_BUFFER, "output buffer too small");
  std::lock_guard<std::mutex> g(ctx->mu);
  cudaSetDevice(ctx->device);
  cudaError_t e = cudaMemcpyAsync(out, plan->d_coef + plan->tile_coef_off[tile], elems * sizeof(int32_t),
                                  cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return cuda_status(e, "coefficient download");
}

sgn_status sgn_j2k_ht_block_table(const uint8_t* data, size_t len, sgn_ht_block* out, size_t cap, size_t* count,
                                  uint64_t* coef_elems) {
  if (!data || (!out && cap)) return set_error(SGN_ERR_INVALID_ARGUMENT, "null argument");
  try {
    TileLayout L;
    parse_tile(data, len, nullptr, L);
    if (count) *count = L.blocks.size();
    if (coef_elems) *coef_elems = L.coef_per_comp * L.ncomp;
    if (L.blocks.size() > cap) return set_error(SGN_ERR_BUFFER, "block table buffer too small");
    for (size_t k = 0; k < L.blocks.size(); ++k) {
      const CodeBlock& cb = L.blocks[k];
      const Band& b = L.bands[cb.band];
      sgn_ht_block& o = out[k];
      std::memset(&o, 0, sizeof(o));
      o.src = cb.cleanup_off;
      o.dst = (uint64_t)b.comp * L.coef_per_comp + b.coef_off + (uint64_t)cb.y0 * b.w + cb.x0;
      o.lcup = cb.lcup;
      o.tile = 0;
      o.stride = b.w;
      o.lref = (uint16_t)cb.lref;
      o.w = cb.w;
      o.h = cb.h;
      o.missing_msbs = cb.missing_msbs;
      o.passes = cb.passes;
      o.num_bitplanes = b.nbp;
      o.flags = L.causal ? 1 : 0;
    }
    return SGN_OK;
  } catch (const ParseError& e) {
    return set_error(e.status, e.message.c_str());
  }
}

sgn_status sgn_j2k_request_blocks(const uint8_t* data, size_t len, uint32_t format, const sgn_request* request,
                                  uint64_t* decoded, uint64_t* total) {
  if (!data || !decoded || !total) return set_error(SGN_ERR_INVALID_ARGUMENT, "null argument");
  TileWork tw;
  prepare_tile(data, len, format, request, tw, nullptr);
  if (tw.status != SGN_OK) return set_error(tw.status, "request rejected");
  RoiWindows roi;
  if (tw.region_conv) build_roi_windows(*tw.L, tw.crop_x, tw.crop_y, tw.crop_w, tw.crop_h, roi);
  uint64_t k = 0;
  for (const CodeBlock& cb : tw.L->blocks) k += block_required(roi, cb) ? 1 : 0;
  *decoded = k;
  *total = tw.L->blocks.size();
  return SGN_OK;
}

void sgn_plan_destroy(sgn_ctx* ctx, sgn_plan* plan) {
  if (!ctx || !plan) return;
  cudaSetDevice(ctx->device);
  for (auto& sf : plan->surfaces)
    if (sf.device_ptr) cudaFreeAsync((void*)(uintptr_t)sf.device_ptr, ctx->stream);
  free_plan_buffers(plan, ctx->stream);
  cudaStreamSynchronize(ctx->stream);
  delete plan;
}

}  // extern "C"

namespace {

// Frees a surface on the context stream; ctx->mu is held by the caller.
void sgn_surface_free_locked(sgn_ctx* ctx, sgn_surface* sf) {
  cudaFreeAsync((void*)(uintptr_t)sf->device_ptr, ctx->stream);
  sf->device_ptr = 0;
}

}  // namespace

extern "C" {

}  // extern "C"

namespace {

const char* backend_name(uint32_t b) {
  static const char* const names[] = {"Auto", "Cpu", "Metal", "Cuda"};
  return b < 4 ? names[b] : "Unknown";
}

const char* format_name(uint32_t f) {
  static const char* const names[] = {"Gray8", "Rgb8", "Rgba8", "Gray16", "Rgb16", "Rgba16"};
  return f < 6 ? names[f] : "Unknown";
}

const char* request_op(const sgn_request* r) {
  static const char* const names[] = {"full", "region", "scaled", "region_scaled"};
  return (r && r->kind < 4) ? names[r->kind] : "full";
}

// A GPU route row (SIGNINUM_GPU_ROUTE_PROFILE) for a call that did not reach
// the device: the adapter's host branch for Cpu / Auto, or an unsupported
// backend.  Dimensions come from a host parse of the header.
void route_not_decoded(const char* op, uint32_t backend, uint32_t format, const uint8_t* data, size_t len,
                       sgn_status st, size_t tiles) {
  if (prof::route_mode() == prof::Mode::Disabled) return;
  prof::Fields f{{"op", op}, {"request", backend_name(backend)}, {"fmt", format_name(format)}};
  if (tiles != 1) {
    f.emplace_back("tiles", std::to_string(tiles));
  } else if (data) {
    try {
      Info i = inspect_codestream(data, len);
      f.emplace_back("width", std::to_string(i.width));
      f.emplace_back("height", std::to_string(i.height));
    } catch (const ParseError&) {
    }
  }
  f.emplace_back("decision", st == SGN_ERR_HOST_BACKEND ? "host_surface" : "unsupported_backend");
  prof::emit_route("j2k", "cuda", f);
}

// Device stage times of a call's plans (SIGNINUM_J2K_PROFILE_STAGES).
struct StageTimes {
  bool on = false;
  uint64_t build_us = 0, blocks = 0, refine_blocks = 0, cleanup_bytes = 0;
  double ms[5] = {0, 0, 0, 0, 0};  // VLC, MagSgn, refinement + classic, IDWT, pack
};

sgn_status decode_tiles_impl(sgn_ctx* ctx, const uint8_t* const* datas, const size_t* lens, size_t n,
                             uint32_t format, const sgn_request* requests, sgn_surface* outs, sgn_status* per_tile,
                             size_t* first_failing, StageTimes& prof_st);

}  // namespace

extern "C" {

sgn_status sgn_j2k_decode_tiles_to_device(sgn_ctx* ctx, const uint8_t* const* datas, const size_t* lens, size_t n,
                                          uint32_t format, const sgn_request* requests, uint32_t backend,
                                          sgn_surface* outs, sgn_status* per_tile, size_t* first_failing) {
  // The backend decides first: Cpu / Auto need no context and touch no CUDA.
  sgn_status bs = check_backend(backend);
  if (bs != SGN_OK) {
    route_not_decoded("tile_batch", backend, format, nullptr, 0, bs, n);
    return bs;
  }
  if (!ctx || (n && (!datas || !lens || !outs))) return set_error(SGN_ERR_INVALID_ARGUMENT, "null argument");
  const auto t0 = std::chrono::steady_clock::now();
  StageTimes pst;
  pst.on = prof::stage_mode() != prof::Mode::Disabled;
  sgn_status st = decode_tiles_impl(ctx, datas, lens, n, format, requests, outs, per_tile, first_failing, pst);
  if (pst.on && n) {
    const uint64_t total_us =
        (uint64_t)std::chrono::duration_cast<std::chrono::microseconds>(std::chrono::steady_clock::now() - t0).count();
    auto us = [](double ms) { return std::to_string((uint64_t)(ms * 1000.0 + 0.5)); };
    prof::emit_stages("j2k", "decode", "cuda",
                      {{"tiles", std::to_string(n)}, {"build_us", std::to_string(pst.build_us)},
                       {"ht_blocks", std::to_string(pst.blocks)}, {"ht_refinement_blocks", std::to_string(pst.refine_blocks)},
                       {"ht_cleanup_bytes", std::to_string(pst.cleanup_bytes)},
                       {"ht_cleanup_us", us(pst.ms[0] + pst.ms[1])}, {"ht_vlc_us", us(pst.ms[0])},
                       {"ht_mag_sgn_us", us(pst.ms[1])}, {"ht_refine_us", us(pst.ms[2])}, {"idwt_us", us(pst.ms[3])},
                       {"pack_us", us(pst.ms[4])}, {"total_us", std::to_string(total_us)}});
  }
  if (n > 1 && prof::route_mode() != prof::Mode::Disabled)
    prof::emit_route("j2k", "cuda",
                     {{"op", "tile_batch"}, {"request", "Cuda"}, {"fmt", format_name(format)},
                      {"tiles", std::to_string(n)}, {"decision", st == SGN_OK ? "cuda_decode" : "cuda_error"}});
  return st;
}

}  // extern "C"

namespace {

sgn_status decode_tiles_impl(sgn_ctx* ctx, const uint8_t* const* datas, const size_t* lens, size_t n,
                             uint32_t format, const sgn_request* requests, sgn_surface* outs, sgn_status* per_tile,
                             size_t* first_failing, StageTimes& pst) {
  if (first_failing) *first_failing = SIZE_MAX;
  for (size_t i = 0; i < n; ++i) outs[i] = sgn_surface{};
  if (n == 0) return SGN_OK;
  std::lock_guard<std::mutex> g(ctx->mu);
  cudaSetDevice(ctx->device);
  ctx->submissions.fetch_add(1);
  // Pipelined: large batches are cut into up to four chunks by coded bytes,
  // each a plan on its own stream with its own staging, built and launched
  // in turn, so the upload of chunk c overlaps the kernels of chunk c - 1 and
  // the host parse of chunk c + 1.  The last chunk carries half the bytes of
  // each of the others: only its kernels run after the last upload.
  uint64_t total = 0;
  for (size_t i = 0; i < n; ++i) total += lens[i];
  const size_t K = std::min<size_t>(total >= (48ull << 20) ? 4 : total >= (12ull << 20) ? 2 : 1, std::max<size_t>(1, n / 2));
  std::vector<size_t> cut(K + 1, n);
  cut[0] = 0;
  {
    // Chunk c < K - 1 ends at 2c / (2K - 1) of the bytes (weights 2, .., 2, 1).
    uint64_t acc = 0;
    size_t c = 1;
    const uint64_t parts = K > 1 ? 2 * K - 1 : 1;
    for (size_t i = 0; i < n && c < K; ++i) {
      acc += lens[i];
      if (acc * parts >= total * 2 * c) cut[c++] = i + 1;
    }
  }
  std::vector<sgn_plan*> plans(K, nullptr);
  std::vector<std::array<cudaEvent_t, 6>> events(K);
  std::vector<sgn_status> statuses(n, SGN_OK);
  sgn_status st = SGN_OK;
  // Pinned codestreams laid out back to back (16-byte padded): every chunk's
  // upload is issued up front, into an arena per chunk, so the host link
  // streams from the start of the call while the chunks are parsed and built
  // (their plans then read the arenas in place).
  auto pad16 = [](size_t v) { return (v + 15) & ~(size_t)15; };
  bool up_front = K > 1 && datas[0] != nullptr;
  for (size_t i = 0; up_front && i + 1 < n; ++i) up_front = datas[i + 1] == datas[i] + pad16(lens[i]);
  up_front = up_front && is_pinned(datas[0]);
  std::vector<uint8_t*> arenas(K, nullptr);
  std::vector<std::vector<uint64_t>> roffs(K);
  if (up_front) {
    for (size_t c = 0; c < K && st == SGN_OK; ++c) {
      const size_t b = cut[c], e = cut[c + 1];
      if (e == b) continue;
      const size_t bytes = (size_t)(datas[e - 1] - datas[b]) + pad16(lens[e - 1]);
      cudaError_t ce = cudaMallocAsync((void**)&arenas[c], bytes, ctx->lanes[c]);
      if (ce == cudaSuccess) ce = cudaMemcpyAsync(arenas[c], datas[b], bytes, cudaMemcpyHostToDevice, ctx->lanes[c]);
      if (ce != cudaSuccess) st = cuda_status(ce, "input upload");
      roffs[c].resize(e - b);
      for (size_t i = b; i < e; ++i) roffs[c][i - b] = (uint64_t)(datas[i] - datas[b]);
    }
  }
  for (size_t c = 0; c < K && st == SGN_OK; ++c) {
    const size_t b = cut[c], m = cut[c + 1] - b;
    if (m == 0) continue;
    plans[c] = new sgn_plan();
    const auto tb = std::chrono::steady_clock::now();
    try {
      st = build_plan(ctx, ctx->lanes[c], ctx->lane_staging[c], datas + b, lens + b, m, format,
                      requests ? requests + b : nullptr, plans[c], arenas[c], up_front ? roffs[c].data() : nullptr,
                      nullptr, false);
    } catch (const std::bad_alloc&) {
      st = set_error(SGN_ERR_OUT_OF_MEMORY, "host allocation failed");
    }
    if (pst.on) {
      pst.build_us += (uint64_t)std::chrono::duration_cast<std::chrono::microseconds>(
                          std::chrono::steady_clock::now() - tb).count();
      for (auto& e : events[c]) cudaEventCreate(&e);
    }
    if (st == SGN_OK) st = execute(plans[c], ctx->lanes[c], pst.on ? events[c].data() : nullptr);
  }
  sgn_status wst = SGN_OK;
  size_t first = SIZE_MAX;
  for (size_t c = 0; c < K; ++c) {
    if (!plans[c]) continue;
    const size_t b = cut[c];
    size_t f = SIZE_MAX;
    if (st == SGN_OK) {
      wait_plan(plans[c], ctx->lanes[c], statuses.data() + b, &f);
      if (pst.on) {
        for (int k = 0; k < 5; ++k) {
          float ms = 0.f;
          if (cudaEventElapsedTime(&ms, events[c][k], events[c][k + 1]) == cudaSuccess) pst.ms[k] += ms;
        }
        cudaGetLastError();
        pst.blocks += plans[c]->nht + plans[c]->nclassic;
        pst.refine_blocks += plans[c]->nref;
        pst.cleanup_bytes += plans[c]->ht_cleanup_bytes;
      }
      if (f != SIZE_MAX && first == SIZE_MAX) {
        first = b + f;
        wst = statuses[b + f];
      }
      for (size_t i = 0; i < plans[c]->n; ++i)
        if (statuses[b + i] == SGN_OK) {
          outs[b + i] = plans[c]->surfaces[i];
          plans[c]->surfaces[i].device_ptr = 0;  // ownership moves to the caller
        }
    } else {
      cudaStreamSynchronize(ctx->lanes[c]);
    }
    release_plan(plans[c], ctx->lanes[c]);
    delete plans[c];
    if (pst.on)
      for (auto& e : events[c]) cudaEventDestroy(e);
  }
  for (size_t c = 0; c < K; ++c)
    if (arenas[c]) {
      if (st != SGN_OK) cudaStreamSynchronize(ctx->lanes[c]);
      cudaFreeAsync(arenas[c], ctx->lanes[c]);
    }
  if (st != SGN_OK) {
    for (size_t i = 0; i < n; ++i) {
      if (outs[i].device_ptr) sgn_surface_free_locked(ctx, &outs[i]);
      if (per_tile) per_tile[i] = st;
    }
    return st;
  }
  if (per_tile)
    for (size_t i = 0; i < n; ++i) per_tile[i] = statuses[i];
  if (first_failing) *first_failing = first;
  if (wst != SGN_OK) set_error(wst, "tile decode failed");
  return wst;
}

}  // namespace

extern "C" {

sgn_status sgn_j2k_decode_to_device(sgn_ctx* ctx, const uint8_t* data, size_t len, uint32_t format,
                                    const sgn_request* request, uint32_t backend, sgn_surface* out) {
  sgn_status bs = check_backend(backend);
  if (bs != SGN_OK) {
    route_not_decoded(request_op(request), backend, format, data, len, bs, 1);
    return bs;
  }
  if (!ctx || !data || !out) return set_error(SGN_ERR_INVALID_ARGUMENT, "null argument");
  sgn_status tile_status = SGN_OK;
  size_t first = 0;
  sgn_status st = sgn_j2k_decode_tiles_to_device(ctx, &data, &len, 1, format, request, backend, out, &tile_status,
                                                 &first);
  if (st == SGN_OK) st = tile_status;
  if (prof::route_mode() != prof::Mode::Disabled) {
    prof::Fields f{{"op", request_op(request)}, {"request", "Cuda"}, {"fmt", format_name(format)}};
    if (st == SGN_OK) {
      f.emplace_back("width", std::to_string(out->width));
      f.emplace_back("height", std::to_string(out->height));
      f.emplace_back("decision", "cuda_decode");
      f.emplace_back("kernel_dispatches", std::to_string(out->kernel_dispatches));
    } else {
      f.emplace_back("decision", "cuda_error");
    }
    prof::emit_route("j2k", "cuda", f);
  }
  return st;
}

sgn_status sgn_surface_download(sgn_ctx* ctx, const sgn_surface* sf, uint8_t* out, size_t out_len, size_t stride) {
  if (!ctx || !sf || (!out && out_len)) return set_error(SGN_ERR_INVALID_ARGUMENT, "null argument");
  size_t row = (size_t)sf->pitch_bytes;
  if (sf->height == 0 || row == 0) return SGN_OK;
  // validate_strided_output_buffer: stride covers a row and the buffer covers
  // (h - 1) strides plus one row.
  if (stride < row || out_len < stride * (sf->height - 1) + row)
    return set_error(SGN_ERR_BUFFER, "output buffer too small for the surface");
  std::lock_guard<std::mutex> g(ctx->mu);
  cudaSetDevice(ctx->device);
  cudaError_t e = cudaMemcpy2DAsync(out, stride, (const void*)(uintptr_t)sf->device_ptr, row, row, sf->height,
                                    cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return cuda_status(e, "surface download");
}

void sgn_surface_free(sgn_ctx* ctx, sgn_surface* sf) {
  if (!ctx || !sf || !sf->device_ptr) return;
  std::lock_guard<std::mutex> g(ctx->mu);
  cudaSetDevice(ctx->device);
  cudaFreeAsync((void*)(uintptr_t)sf->device_ptr, ctx->stream);
  cudaStreamSynchronize(ctx->stream);
  sf->device_ptr = 0;
}

}  // extern "C"
