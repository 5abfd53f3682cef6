// Region-of-interest pruning for region requests: which code blocks a
// decode needs and which part of each IDWT level it must compute.
//
// Restates RoiPlan (crates/signinum-j2k-native/src/j2c/roi.rs:18-270): the
// output window is the requested region at the decoded resolution; walking
// from the finest decoded level down, each level's required output is
// widened by a margin (16 samples for the 5/3 wavelet, 40 for the 9/7,
// idwt_required_output_margin) within the level, and the band samples under
// that window (idwt_input_required_region with idwt_band_index) become the
// windows of the level's HL / LH / HH bands and the required output of the
// level below, down to the LL band.  A code block is required when its
// rectangle meets its band's window (code_block_required).  As there, a
// region that reaches the right or bottom edge of the decoded image, or an
// empty one, gets no plan (the whole tile is decoded).
//
// Tiles here have zero image and tile offsets and no sub-sampling, so every
// rectangle starts at the origin of its band or resolution and the band
// index of output coordinate c is ceil(c / 2) for low-pass bands and
// floor(c / 2) for high-pass ones.
#pragma once

#include <algorithm>
#include <cstdint>
#include <vector>

#include "codestream.h"

namespace sgn {

struct Window {
  uint32_t x0 = 0, y0 = 0, x1 = 0, y1 = 0;
  bool empty() const { return x0 >= x1 || y0 >= y1; }
  bool intersects(uint32_t bx0, uint32_t by0, uint32_t bx1, uint32_t by1) const {
    return x0 < bx1 && bx0 < x1 && y0 < by1 && by0 < y1;
  }
};

struct RoiWindows {
  bool active = false;          // false: decode every block and every level in full
  std::vector<Window> band;     // per band of the layout (empty: no block needed)
  std::vector<Window> level;    // per decoded resolution r (1..R): the level's output to compute
};

namespace roi_detail {

inline void add(Window& slot, const Window& w) {
  if (w.empty()) return;
  if (slot.empty()) {
    slot = w;
    return;
  }
  slot.x0 = std::min(slot.x0, w.x0);
  slot.y0 = std::min(slot.y0, w.y0);
  slot.x1 = std::max(slot.x1, w.x1);
  slot.y1 = std::max(slot.y1, w.y1);
}

// idwt_band_index with origin 0.
inline uint32_t band_index(uint32_t c, bool low) { return low ? (c + 1) / 2 : c / 2; }

// idwt_input_required_region for output window e of a level, into a band of
// bw x bh samples.
inline Window band_region(const Window& e, bool low_x, bool low_y, uint32_t bw, uint32_t bh) {
  if (e.empty()) return Window{};
  Window r;
  r.x0 = std::min(band_index(e.x0, low_x), bw);
  r.x1 = std::min(band_index(e.x1 - 1, low_x) + 1, bw);
  r.y0 = std::min(band_index(e.y0, low_y), bh);
  r.y1 = std::min(band_index(e.y1 - 1, low_y) + 1, bh);
  return r;
}

}  // namespace roi_detail

// Windows of a decode of layout L whose output is the crop (cx, cy, cw, ch)
// of the decoded resolution.
inline void build_roi_windows(const TileLayout& L, uint32_t cx, uint32_t cy, uint32_t cw, uint32_t ch,
                              RoiWindows& out) {
  using namespace roi_detail;
  out = RoiWindows{};
  const uint32_t R = L.levels - L.skipped;
  auto res_dim = [&](uint32_t r, bool wdim) {
    const uint32_t sh = L.levels - r;
    const uint64_t v = wdim ? L.width : L.height;
    return (uint32_t)((v + (1ull << sh) - 1) >> sh);
  };
  const uint32_t wR = res_dim(R, true), hR = res_dim(R, false);
  Window F;
  F.x0 = std::min(cx, wR);
  F.y0 = std::min(cy, hR);
  F.x1 = (uint32_t)std::min<uint64_t>((uint64_t)cx + cw, wR);
  F.y1 = (uint32_t)std::min<uint64_t>((uint64_t)cy + ch, hR);
  if (F.empty() || F.x1 == wR || F.y1 == hR) return;
  out.active = true;
  out.band.assign(L.bands.size(), Window{});
  out.level.assign(R + 1, Window{});
  const uint32_t margin = L.reversible ? 16 : 40;
  for (uint32_t c = 0; c < L.ncomp; ++c) {
    const uint32_t b0 = L.comp_band_begin[c];
    if (R == 0) {
      add(out.band[b0], F);
      continue;
    }
    Window req = F;
    for (uint32_t r = R; r >= 1; --r) {
      const uint32_t w = res_dim(r, true), h = res_dim(r, false);
      Window e;
      e.x0 = req.x0 > margin ? req.x0 - margin : 0;
      e.y0 = req.y0 > margin ? req.y0 - margin : 0;
      e.x1 = std::min(req.x1 + margin, w);
      e.y1 = std::min(req.y1 + margin, h);
      add(out.level[r], e);
      const Band& hl = L.bands[b0 + 1 + (r - 1) * 3];
      const Band& lh = L.bands[b0 + 2 + (r - 1) * 3];
      const Band& hh = L.bands[b0 + 3 + (r - 1) * 3];
      add(out.band[b0 + 1 + (r - 1) * 3], band_region(e, false, true, hl.w, hl.h));
      add(out.band[b0 + 2 + (r - 1) * 3], band_region(e, true, false, lh.w, lh.h));
      add(out.band[b0 + 3 + (r - 1) * 3], band_region(e, false, false, hh.w, hh.h));
      const Window ll = band_region(e, true, true, (w + 1) / 2, (h + 1) / 2);
      if (r == 1) add(out.band[b0], ll);
      else req = ll;
    }
  }
}

// code_block_required: every block without a plan; with one, the blocks
// meeting their band's window.
inline bool block_required(const RoiWindows& roi, const CodeBlock& cb) {
  if (!roi.active) return true;
  const Window& w = roi.band[cb.band];
  return !w.empty() && w.intersects(cb.x0, cb.y0, cb.x0 + cb.w, cb.y0 + cb.h);
}

}  // namespace sgn
