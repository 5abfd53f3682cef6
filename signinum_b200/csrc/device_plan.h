// Device-resident descriptor tables shared by the host plan builder and the
// sm_100a kernels.
//
// One HtJob per code block (the device form of the reference's
// HtOwnedCodeBlockBatchJob, crates/signinum-j2k-native/src/direct_plan.rs:120-149),
// one IdwtJob per (tile, component, decomposition level) (cf. J2kDirectIdwtStep,
// direct_plan.rs:154-177) and one PackJob per tile for the last level fused
// with inverse RCT, DC shift and pixel packing (cf. J2kDirectStoreStep,
// direct_plan.rs:182-205).  Offsets are 64-bit so one arena can hold a
// whole batch.
#pragma once

#include <cstdint>

namespace sgn {

// Work unit of the IDWT kernels: one warp decodes a strip of kIdwtStripW
// columns (four per lane) over `seg` rows of one level (even, chosen per job).
constexpr int kIdwtStripW = 128;
// The 9/7 kernels' strips: 120 output columns (lanes 1..30; lanes 0 and 31
// carry the four columns on either side).
constexpr int kStrip97 = 120;

// Rows per work unit: long segments for big levels (less halo re-reading),
// short ones for small levels, whose few units otherwise each stream many
// rows one after another (more, shorter units finish sooner).
inline uint32_t idwt_segment_rows(uint32_t h) { return h >= 256 ? 64 : h >= 128 ? 16 : h >= 64 ? 8 : 4; }
constexpr int kIdwtWarps = 8;  // warps (units) per CTA

struct HtJob {
  uint64_t src;      // byte offset of the cleanup segment in the input arena
  uint64_t dst;      // element offset of the block's first sample in the coefficient arena
  uint64_t sym;      // element offset of the block's quad-symbol table in the symbol scratch
  uint32_t lcup;     // cleanup segment length (refinement follows it)
  uint32_t tile;     // batch index of the tile (status reporting)
  uint32_t stride;   // band row stride in elements
  uint16_t lref;     // refinement segment length
  uint16_t w, h;
  uint8_t mmsb;      // missing MSBs after placeholder folding (p = 30 - mmsb)
  uint8_t passes;    // 0 = all-zero block, 1 = cleanup, 2 = +SigProp, 3 = +MagRef
  uint8_t nbp;       // magnitude bit-planes of the band (coefficient alignment)
  uint8_t flags;     // bit 0: vertically causal context
  uint8_t pad[2];
};
static_assert(sizeof(HtJob) == 48, "HtJob layout");

// Quad symbol written by the VLC pass: bits 0-15 the CxtVLC entry (rho,
// u_off, e_k, e_1), bits 16-23 u_q (initial row: u_q + 1).  A block whose
// cleanup VLC/MEL decode failed has kSymFailed in its first entry.
constexpr uint32_t kSymFailed = 0xFFFFFFFFu;

// Quad-symbol table of a code block: ceil(h/2) rows of ceil(w/2) symbols,
// each row padded to an even count so a quad pair's two symbols form one
// 8-byte store; tables are padded to a multiple of 4 words, so they start
// 16-byte aligned (rows of a multiple of 4 symbols are written 16 bytes at
// a time).
#ifdef __CUDACC__
__host__ __device__
#endif
inline uint32_t sym_row_stride(uint32_t w) { return (((w + 1) / 2) + 1) & ~1u; }
#ifdef __CUDACC__
__host__ __device__
#endif
inline uint32_t sym_words(uint32_t w, uint32_t h) { return (sym_row_stride(w) * ((h + 1) / 2) + 3) & ~3u; }

// One classic (EBCOT Tier-1) code block: its codeword segments lie back to
// back in the input arena from `src` (classic_block_decode's `data`), the
// segment table entries [seg, seg + nseg) give each segment's bytes and
// coding passes.  passes == 0: an all-zero block.
struct ClassicJob {
  uint64_t src;        // byte offset of the block's first segment in the input arena
  uint64_t dst;        // element offset of the block's first sample in the coefficient arena
  uint32_t seg;        // first segment-table entry
  uint32_t tile;       // batch index of the tile (status reporting)
  uint32_t stride;     // band row stride in elements
  uint16_t w, h;
  uint8_t nseg, passes;
  uint8_t bitplanes;   // the band's bit-planes minus the block's missing ones (> 0 when passes > 0)
  uint8_t band_class;  // zero-coding rule: 0 LL/LH, 1 HL, 2 HH
  uint8_t style;       // code-block style bits
  uint8_t pad[3];
};
static_assert(sizeof(ClassicJob) == 40, "ClassicJob layout");

// ClassicJob::src with this bit set: an offset in the plan's gather area
// (multi-layer blocks, their parts copied back to back) instead of the input.
constexpr uint64_t kClassicGathered = 1ull << 63;

struct ClassicSeg {
  uint32_t len;     // bytes
  uint32_t passes;  // coding passes
};

// 16-bit scratch words a classic block needs: blocks of at most 64 x 64
// keep four 64-bit planes of rows -1 .. h+3 (69 rows); larger ones one flag
// word per sample padded by one on every side.  A multiple of 4, so slots
// stay 8-byte aligned.
#ifdef __CUDACC__
__host__ __device__
#endif
inline uint32_t classic_slot_words(uint32_t w, uint32_t h) {
  return (w <= 64 && h <= 64) ? 4u * 69u * 4u : (((w + 2) * (h + 2) + 3) & ~3u);
}

// Irreversible (9/7) levels use the same tables: band pointers hold int32
// coefficients that the kernel dequantises with `step`, level images (the
// ll input after the first level, and `out`) hold f32 samples.
struct IdwtJob {
  const int32_t* ll;   // ceil(w/2) x ceil(h/2)
  const int32_t* hl;   // floor(w/2) x ceil(h/2)
  const int32_t* lh;   // ceil(w/2) x floor(h/2)
  const int32_t* hh;   // floor(w/2) x floor(h/2)
  int32_t* out;        // w x h, tight
  uint32_t w, h;
  uint32_t strips;      // strips across the level
  uint32_t unit_begin;  // first work unit of this job in its launch
  uint32_t seg;         // output rows per work unit (even)
  uint32_t ll_band;     // 9/7: ll is the LL band (dequantise) rather than a level image
  float step[4];        // 9/7: dequantisation steps of ll, hl, lh, hh
  // Window of the level the units cover: columns from x_begin (a multiple of
  // the strip width) over `strips` strips, rows [y_begin, y_end) with y_begin
  // even.  The whole level (0, 0, h) unless a region request prunes it.
  uint32_t x_begin, y_begin, y_end;
  uint32_t pad;
};
static_assert(sizeof(IdwtJob) == 96, "IdwtJob layout");

enum PackFormat : uint32_t { PACK_GRAY8 = 0, PACK_RGB8 = 1, PACK_RGBA8 = 2, PACK_GRAY16 = 3, PACK_RGB16 = 4 };

// Kernel variant of a reversible tile's pack job: 0 RGB with samples that
// convert by a clamp alone (8-bit samples to 8-bit formats, deeper ones to
// 16-bit formats), 1 RGB rescaled, 2 gray by a clamp, 3 gray rescaled.
constexpr uint32_t kPackVariants = 4;
inline uint32_t pack_variant(uint32_t fmt, uint32_t ncomp, uint32_t bit_depth) {
  const bool u8 = fmt == PACK_GRAY8 || fmt == PACK_RGB8 || fmt == PACK_RGBA8;
  const bool direct = u8 ? bit_depth == 8 : bit_depth > 8;
  return (ncomp >= 3 ? 0u : 2u) + (direct ? 0u : 1u);
}

struct PackJob {
  const int32_t* ll[3];
  const int32_t* hl[3];
  const int32_t* lh[3];
  const int32_t* hh[3];
  uint8_t* out;         // surface (device)
  uint64_t pitch;       // bytes per output row
  uint32_t w, h;        // dimensions of the last decoded level (image at that resolution)
  uint32_t cx, cy, cw, ch;  // crop written to the surface
  uint32_t lifting;     // 1: inputs are the four bands of the last level; 0: ll holds the image
  uint32_t ncomp, mct, bit_depth, fmt, region_conv;
  uint32_t strips;      // strips across the crop (from cx rounded down to kIdwtStripW)
  uint32_t unit_begin;  // first work unit of this job in its launch
  uint32_t seg;         // output rows per work unit (even)
  uint32_t tile;        // batch index (status)
  uint32_t ll_band;     // 9/7: ll[c] are LL bands (dequantise) rather than level images
  float step[3][4];     // 9/7: dequantisation steps of ll, hl, lh, hh per component
};

}  // namespace sgn
