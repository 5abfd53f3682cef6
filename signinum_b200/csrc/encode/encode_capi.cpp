// C ABI of the HTJ2K encoder (lossless; irreversible for test inputs) and the
// synthetic tile generators.
#include <cstring>
#include <vector>

#include "../../../include/signinum_j2k_encode.h"

#include "j2k_encode.h"

extern "C" {

static int encode_with(const uint8_t* pixels, uint32_t width, uint32_t height, uint32_t components,
                       uint32_t bit_depth, const sgn_encode_options* o, bool irreversible, double rel_step,
                       uint8_t* out, size_t out_cap, size_t* out_len, bool classic = false, uint32_t style = 0,
                       uint32_t layers = 1) {
  sgn::enc::EncodeParams p;
  p.irreversible = irreversible;
  p.rel_step = rel_step;
  p.classic = classic;
  p.cb_style = (uint8_t)(style & 0x2F);
  p.layers = layers;
  if (layers == 0 || layers > 64) return -2;
  p.width = width;
  p.height = height;
  p.comps = components;
  p.bit_depth = bit_depth;
  p.levels = o ? o->max_decomposition_levels : 5;
  p.cbw_exp = o ? o->code_block_width_exp : 4;
  p.cbh_exp = o ? o->code_block_height_exp : 4;
  p.mct = o ? o->use_mct != 0 : true;
  p.progression = o ? (int)o->progression : 0;
  p.write_tlm = o ? o->write_tlm != 0 : false;
  p.sop_eph = o ? o->sop_eph != 0 : false;
  p.ppx = o ? o->precinct_width_exp : 0;
  p.ppy = o ? o->precinct_height_exp : 0;
  p.tile_parts = o && o->tile_parts ? o->tile_parts : 1;
  // Code blocks up to 1024 wide or high with w h <= 4096 (exponents of 4).
  const uint32_t max_exp = 8;
  if (p.cbw_exp > max_exp || p.cbh_exp > max_exp || p.cbw_exp + p.cbh_exp > 8 || p.progression < 0 ||
      p.progression > 4)
    return -2;
  std::vector<uint8_t> cs;
  int rc = sgn::enc::encode(pixels, p, cs);
  if (rc != 0) return rc;
  if (out_len) *out_len = cs.size();
  if (cs.size() > out_cap) return -4;
  std::memcpy(out, cs.data(), cs.size());
  return 0;
}

int sgn_j2k_encode_lossless(const uint8_t* pixels, uint32_t width, uint32_t height, uint32_t components,
                            uint32_t bit_depth, const sgn_encode_options* o, uint8_t* out, size_t out_cap,
                            size_t* out_len) {
  return encode_with(pixels, width, height, components, bit_depth, o, false, 0.0, out, out_cap, out_len);
}

int sgn_j2k_encode_irreversible(const uint8_t* pixels, uint32_t width, uint32_t height, uint32_t components,
                                uint32_t bit_depth, const sgn_encode_options* o, double relative_step,
                                uint8_t* out, size_t out_cap, size_t* out_len) {
  return encode_with(pixels, width, height, components, bit_depth, o, true, relative_step, out, out_cap, out_len);
}

int sgn_j2k_encode_classic(const uint8_t* pixels, uint32_t width, uint32_t height, uint32_t components,
                           uint32_t bit_depth, const sgn_encode_options* o, uint32_t code_block_style,
                           uint32_t irreversible, double relative_step, uint32_t layers, uint8_t* out,
                           size_t out_cap, size_t* out_len) {
  return encode_with(pixels, width, height, components, bit_depth, o, irreversible != 0, relative_step, out, out_cap,
                     out_len, true, code_block_style, layers);
}

void sgn_synth_he_rgb8(uint64_t seed, uint32_t w, uint32_t h, double sigma, uint8_t* out) {
  sgn::synth::he_tile(seed, w, h, sigma, out);
}
void sgn_synth_blank_rgb8(uint64_t seed, uint32_t w, uint32_t h, uint8_t* out) {
  sgn::synth::blank_tile(seed, w, h, out);
}
void sgn_synth_fluor_gray16(uint64_t seed, uint32_t w, uint32_t h, uint8_t* out) {
  sgn::synth::fluor_tile(seed, w, h, out);
}

}  // extern "C"
