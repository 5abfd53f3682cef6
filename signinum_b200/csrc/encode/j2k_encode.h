// Internal interface of the HTJ2K encoder (lossless, and irreversible 9/7
// for test inputs) and the synthetic generators.
#pragma once

#include <cstdint>
#include <vector>

namespace sgn {
namespace enc {
struct EncodeParams {
  uint32_t width, height, comps, bit_depth, levels, cbw_exp, cbh_exp;
  bool mct;
  int progression;  // 0 LRCP, 1 RLCP, 2 RPCL, 3 PCRL, 4 CPRL
  bool write_tlm;
  bool sop_eph;
  // Irreversible path: ICT (with mct), 9/7, scalar expounded quantisation
  // with relative step rel_step of every band's nominal range.
  bool irreversible = false;
  double rel_step = 1.0 / 256;
  // Classic (EBCOT) Tier-1 instead of HT, with code-block style bits
  // (bypass 0x01, reset 0x02, termall 0x04, vcausal 0x08, segsym 0x20).
  bool classic = false;
  uint8_t cb_style = 0;
  uint32_t layers = 1;  // quality layers (classic only)
  // Precinct exponents (PPx, PPy) of every resolution, 1..15; 0 = one
  // precinct per resolution (no precinct partition signalled).
  uint32_t ppx = 0, ppy = 0;
  // Tile-parts the packets are split into (at packet boundaries), >= 1.
  uint32_t tile_parts = 1;
};
// One classic code block: its codeword segments back to back, each
// segment's length and coding-pass count, and the block's zero bit-planes.
struct ClassicBlockOut {
  std::vector<uint8_t> bytes;
  std::vector<uint32_t> seg_len, seg_passes;
  uint32_t passes = 0, zero_planes = 0;
};
int encode_classic_block(const int32_t* c, size_t stride, uint32_t w, uint32_t h, uint32_t Mb, uint8_t band_class,
                         uint8_t style, ClassicBlockOut& out);
int encode(const uint8_t* pixels, const EncodeParams& P, std::vector<uint8_t>& out);
int encode_ht_block(const int32_t* c, size_t stride, uint32_t w, uint32_t h, uint32_t Mb, std::vector<uint8_t>& out);
}  // namespace enc
namespace synth {
void he_tile(uint64_t seed, uint32_t w, uint32_t h, double sigma, uint8_t* out);
void blank_tile(uint64_t seed, uint32_t w, uint32_t h, uint8_t* out);
void fluor_tile(uint64_t seed, uint32_t w, uint32_t h, uint8_t* out_le16);
}  // namespace synth
}  // namespace sgn
