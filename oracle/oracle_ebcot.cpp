// Parity oracle (test infrastructure only): classic EBCOT Tier-1 code-block
// decoding, restated from the reference's CPU decoder:
//   crates/signinum-j2k-native/src/j2c/arithmetic_decoder.rs:1-386 (MQ decoder, Annex C),
//   crates/signinum-j2k-native/src/j2c/bitplane.rs:27-1447 (coding passes, Annex D).
// The reference's lookup tables for zero coding and sign coding are computed
// here from the rules of Tables D.1 and D.3; tests compare them with the
// reference's tables by checksum.
#include <cstdint>
#include <cstring>
#include <vector>

#include "oracle_internal.h"

namespace oracle {
namespace {

// QE values and transitions, Table C.2 (arithmetic_decoder.rs:333-386).
struct Qe {
  uint32_t qe;
  uint8_t nmps, nlps, sw;
};
const Qe kQe[47] = {
    {0x5601, 1, 1, 1},   {0x3401, 2, 6, 0},   {0x1801, 3, 9, 0},   {0x0AC1, 4, 12, 0},  {0x0521, 5, 29, 0},
    {0x0221, 38, 33, 0}, {0x5601, 7, 6, 1},   {0x5401, 8, 14, 0},  {0x4801, 9, 14, 0},  {0x3801, 10, 14, 0},
    {0x3001, 11, 17, 0}, {0x2401, 12, 18, 0}, {0x1C01, 13, 20, 0}, {0x1601, 29, 21, 0}, {0x5601, 15, 14, 1},
    {0x5401, 16, 14, 0}, {0x5101, 17, 15, 0}, {0x4801, 18, 16, 0}, {0x3801, 19, 17, 0}, {0x3401, 20, 18, 0},
    {0x3001, 21, 19, 0}, {0x2801, 22, 19, 0}, {0x2401, 23, 20, 0}, {0x2201, 24, 21, 0}, {0x1C01, 25, 22, 0},
    {0x1801, 26, 23, 0}, {0x1601, 27, 24, 0}, {0x1401, 28, 25, 0}, {0x1201, 29, 26, 0}, {0x1101, 30, 27, 0},
    {0x0AC1, 31, 28, 0}, {0x09C1, 32, 29, 0}, {0x08A1, 33, 30, 0}, {0x0521, 34, 31, 0}, {0x0441, 35, 32, 0},
    {0x02A1, 36, 33, 0}, {0x0221, 37, 34, 0}, {0x0141, 38, 35, 0}, {0x0111, 39, 36, 0}, {0x0085, 40, 37, 0},
    {0x0049, 41, 38, 0}, {0x0025, 42, 39, 0}, {0x0015, 43, 40, 0}, {0x0009, 44, 41, 0}, {0x0005, 45, 42, 0},
    {0x0001, 45, 43, 0}, {0x5601, 46, 46, 0},
};

// Context state: index 0..46 and the MPS bit (ArithmeticDecoderContext).
struct Ctx {
  uint8_t index = 0, mps = 0;
};

// MQ decoder with the software conventions of Annex G of T.88
// (arithmetic_decoder.rs:36-270); bytes past the end read as 0xFF.
struct Mq {
  const uint8_t* data;
  size_t len;
  uint32_t c = 0, a = 0, bp = 0, ct = 0;
  uint8_t byte_at(size_t i) const { return i < len ? data[i] : 0xFF; }
  void bytein() {
    if (byte_at(bp) == 0xFF) {
      if (byte_at(bp + 1) > 0x8F) {
        ct = 8;
      } else {
        ++bp;
        c = c + 0xFE00 - ((uint32_t)byte_at(bp) << 9);
        ct = 7;
      }
    } else {
      ++bp;
      c = c + 0xFF00 - ((uint32_t)byte_at(bp) << 8);
      ct = 8;
    }
  }
  Mq(const uint8_t* d, size_t n) : data(d), len(n) {
    c = ((uint32_t)byte_at(0) ^ 0xFF) << 16;
    bytein();
    c <<= 7;
    ct -= 7;
    a = 0x8000;
  }
  void renorm() {
    do {
      if (ct == 0) bytein();
      a <<= 1;
      c <<= 1;
      --ct;
    } while ((a & 0x8000) == 0);
  }
  // DECODE, C.3.2 (the MPS/LPS exchanges of :96-170).
  uint32_t decode(Ctx& cx) {
    const Qe& q = kQe[cx.index];
    a -= q.qe;
    uint32_t d;
    if ((c >> 16) < a) {
      if (a & 0x8000) return cx.mps;
      // MPS_EXCHANGE
      if (a < q.qe) {
        d = 1 - cx.mps;
        if (q.sw) cx.mps ^= 1;
        cx.index = q.nlps;
      } else {
        d = cx.mps;
        cx.index = q.nmps;
      }
    } else {
      c -= a << 16;
      // LPS_EXCHANGE
      if (a < q.qe) {
        a = q.qe;
        d = cx.mps;
        cx.index = q.nmps;
      } else {
        a = q.qe;
        d = 1 - cx.mps;
        if (q.sw) cx.mps ^= 1;
        cx.index = q.nlps;
      }
    }
    renorm();
    return d;
  }
};

// Raw (bypass) bits with the packet-header stuffing rule; past the end, or on
// a bad stuff bit, the reader supplies 1 (BypassDecoder, bitplane.rs:1403-1430,
// non-strict).
struct Raw {
  const uint8_t* data;
  size_t len;
  size_t cur = 0;  // bit position
  bool bit(uint32_t& b) {
    if (cur / 8 >= len) return false;
    b = (data[cur / 8] >> (7 - cur % 8)) & 1;
    ++cur;
    return true;
  }
  uint32_t decode(Ctx&) {
    const bool stuff = cur % 8 == 7 && cur / 8 < len && data[cur / 8] == 0xFF;
    uint32_t b;
    if (!bit(b)) return 1;
    if (stuff) {
      uint32_t s;
      if (!bit(s) || s != 0) return 1;
    }
    return b;
  }
};

// Neighbour significance bits (NeighborSignificances, bitplane.rs:370-420):
// top-left 7, top 6, top-right 5, left 4, bottom-left 3, right 2,
// bottom-right 1, bottom 0.
constexpr uint8_t kSig = 0x80, kRefined = 0x40, kCoded = 0x20;

// Zero-coding context, Table D.1, from the counts of significant horizontal,
// vertical and diagonal neighbours.
uint8_t zc_context(uint8_t n, int band) {
  const int h = ((n >> 4) & 1) + ((n >> 2) & 1);
  const int v = ((n >> 6) & 1) + (n & 1);
  const int d = ((n >> 7) & 1) + ((n >> 5) & 1) + ((n >> 3) & 1) + ((n >> 1) & 1);
  if (band == HH) {
    const int hv = h + v;
    if (d >= 3) return 8;
    if (d == 2) return hv >= 1 ? 7 : 6;
    if (d == 1) return hv >= 2 ? 5 : (hv == 1 ? 4 : 3);
    return hv >= 2 ? 2 : (uint8_t)hv;
  }
  int a = h, b = v;  // LL and LH: horizontal first; HL: swapped
  if (band == HL) {
    a = v;
    b = h;
  }
  if (a == 2) return 8;
  if (a == 1) return b >= 1 ? 7 : (d >= 1 ? 6 : 5);
  if (b == 2) return 4;
  if (b == 1) return 3;
  return d >= 2 ? 2 : (uint8_t)d;
}

// Sign-coding context and XOR bit, Table D.3, from the 2-bit (negative,
// positive) fields of top (bits 6-7), left (4-5), right (2-3) and bottom
// (0-1) neighbours.
void sc_context(uint8_t m, uint8_t& label, uint8_t& xr) {
  auto contrib = [&](int sh) { return (int)((m >> sh) & 1) - (int)((m >> (sh + 1)) & 1); };
  auto clamp1 = [](int x) { return x > 1 ? 1 : (x < -1 ? -1 : x); };
  const int hc = clamp1(contrib(4) + contrib(2)), vc = clamp1(contrib(6) + contrib(0));
  static const uint8_t lab[3][3] = {{13, 12, 11}, {10, 9, 10}, {11, 12, 13}};  // [1-hc][1-vc]
  label = lab[1 - hc][1 - vc];
  xr = (hc < 0 || (hc == 0 && vc < 0)) ? 1 : 0;
}

struct Block {
  uint32_t w, h, pw;
  int band;
  uint8_t style;
  uint8_t bitplanes, max_passes, pos = 0;
  std::vector<uint32_t> coef;  // sign bit 31, magnitude below
  std::vector<uint8_t> state, nb;
  Ctx ctx[19];
  bool vcausal() const { return style & 0x08; }
  void reset_contexts() {
    for (Ctx& c : ctx) c = Ctx();
    ctx[0].index = 4;
    ctx[17].index = 3;
    ctx[18].index = 46;
  }
  size_t at(uint32_t x, uint32_t y) const { return (size_t)(y + 1) * pw + x + 1; }
  uint8_t neighbors(size_t i, uint32_t y) const {
    const bool next_stripe = y + 1 < h && ((y + 1) >> 2) > (y >> 2);
    return (vcausal() && next_stripe) ? (uint8_t)(nb[i] & 0xF4) : nb[i];
  }
  void set_significant(size_t i) {
    if (state[i] & kSig) return;
    state[i] |= kSig;
    nb[i - pw - 1] |= 1 << 1;
    nb[i - pw] |= 1 << 0;
    nb[i - pw + 1] |= 1 << 3;
    nb[i - 1] |= 1 << 2;
    nb[i + 1] |= 1 << 4;
    nb[i + pw - 1] |= 1 << 5;
    nb[i + pw] |= 1 << 6;
    nb[i + pw + 1] |= 1 << 7;
  }
  uint32_t sign(size_t i) const { return coef[i] >> 31; }
  void push_bit(size_t i, uint32_t b) { coef[i] |= b << pos; }
  template <typename D>
  void decode_sign(size_t i, uint32_t y, D& dec, bool raw) {
    const uint8_t s = neighbors(i, y) & 0x55;
    const bool next_stripe = y + 1 < h && ((y + 1) >> 2) > (y >> 2);
    const uint32_t bottom = (vcausal() && next_stripe) ? 0 : sign(i + pw);
    const uint32_t signs = (sign(i - pw) << 6) | (sign(i - 1) << 4) | (sign(i + 1) << 2) | bottom;
    const uint8_t neg = (uint8_t)(s & signs), pos_ = (uint8_t)(s & ~signs);
    uint8_t label, xr;
    sc_context((uint8_t)((neg << 1) | pos_), label, xr);
    uint32_t b = dec.decode(ctx[label]);
    if (!raw) b ^= xr;  // raw sign bits carry no XOR (decode_sign_bit_bypass)
    coef[i] |= b << 31;
  }
  template <typename D>
  void cleanup_coefficient(size_t i, uint32_t y, D& dec, bool raw) {
    if (state[i] & (kSig | kCoded)) return;
    const uint32_t b = dec.decode(ctx[zc_context(neighbors(i, y), band)]);
    push_bit(i, b);
    if (b) {
      decode_sign(i, y, dec, raw);
      set_significant(i);
    }
  }
  // Cleanup pass (cleanup_pass_*, bitplane.rs:773-826, :903-979).
  template <typename D>
  void cleanup(D& dec, bool raw) {
    for (uint32_t by = 0; by < h; by += 4) {
      const uint32_t ye = by + 4 < h ? by + 4 : h;
      for (uint32_t x = 0; x < w; ++x) {
        const size_t top = at(x, by);
        bool run = ye - by == 4;
        for (uint32_t y = by; run && y < by + 4; ++y) {
          const size_t i = top + (size_t)(y - by) * pw;
          run = !(state[i] & (kSig | kCoded)) && neighbors(i, y) == 0;
        }
        if (run) {
          if (dec.decode(ctx[17]) == 0) continue;
          uint32_t f = dec.decode(ctx[18]) << 1;
          f |= dec.decode(ctx[18]);
          const uint32_t sy = by + f;
          const size_t si = top + (size_t)f * pw;
          push_bit(si, 1);
          decode_sign(si, sy, dec, raw);
          set_significant(si);
          for (uint32_t y = sy + 1; y < ye; ++y) cleanup_coefficient(top + (size_t)(y - by) * pw, y, dec, raw);
          continue;
        }
        for (uint32_t y = by; y < ye; ++y) cleanup_coefficient(top + (size_t)(y - by) * pw, y, dec, raw);
      }
    }
  }
  // Significance propagation pass (bitplane.rs:827-865, :981-1027).
  template <typename D>
  void sig_prop(D& dec, bool raw) {
    for (uint32_t by = 0; by < h; by += 4) {
      const uint32_t ye = by + 4 < h ? by + 4 : h;
      for (uint32_t x = 0; x < w; ++x)
        for (uint32_t y = by; y < ye; ++y) {
          const size_t i = at(x, y);
          const uint8_t n = neighbors(i, y);
          if ((state[i] & kSig) || n == 0) continue;
          const uint32_t b = dec.decode(ctx[zc_context(n, band)]);
          push_bit(i, b);
          state[i] |= kCoded;
          if (b) {
            decode_sign(i, y, dec, raw);
            set_significant(i);
          }
        }
    }
  }
  // Magnitude refinement pass (bitplane.rs:867-901, :1029-1062; Table D.4).
  template <typename D>
  void mag_ref(D& dec) {
    for (uint32_t by = 0; by < h; by += 4) {
      const uint32_t ye = by + 4 < h ? by + 4 : h;
      for (uint32_t x = 0; x < w; ++x)
        for (uint32_t y = by; y < ye; ++y) {
          const size_t i = at(x, y);
          if (!(state[i] & kSig) || (state[i] & kCoded)) continue;
          const uint8_t n = neighbors(i, y);
          const uint8_t label = (state[i] & kRefined) ? 16 : (uint8_t)(14 + (n != 0));
          push_bit(i, dec.decode(ctx[label]));
          state[i] |= kRefined;
        }
    }
  }
  // handle_*_coding_passes (bitplane.rs:206-305).
  template <typename D>
  bool passes(uint32_t start, uint32_t end, D& dec, bool raw) {
    for (uint32_t p = start; p < end; ++p) {
      const uint32_t bitplane = (p + 2) / 3;
      pos = (uint8_t)(bitplanes - 1 - bitplane);
      switch (p % 3) {
        case 0:
          cleanup(dec, raw);
          if (style & 0x20) {
            for (int k = 0; k < 4; ++k) dec.decode(ctx[18]);  // segmentation symbol (not checked: non-strict)
          }
          for (uint32_t y = 0; y < h; ++y)
            for (uint32_t x = 0; x < w; ++x) state[at(x, y)] &= (uint8_t)~kCoded;
          break;
        case 1:
          sig_prop(dec, raw);
          break;
        default:
          mag_ref(dec);
          break;
      }
      if (style & 0x02) reset_contexts();
    }
    return true;
  }
};

}  // namespace

void ebcot_qe_records(uint8_t* out) {
  for (int k = 0; k < 47; ++k) {
    out[5 * k] = (uint8_t)(kQe[k].qe & 0xFF);
    out[5 * k + 1] = (uint8_t)(kQe[k].qe >> 8);
    out[5 * k + 2] = kQe[k].nmps;
    out[5 * k + 3] = kQe[k].nlps;
    out[5 * k + 4] = kQe[k].sw;
  }
}

void ebcot_tables(uint8_t* zc_ll_lh, uint8_t* zc_hl, uint8_t* zc_hh, uint8_t* sc_label, uint8_t* sc_xor) {
  for (int n = 0; n < 256; ++n) {
    zc_ll_lh[n] = zc_context((uint8_t)n, LL);
    zc_hl[n] = zc_context((uint8_t)n, HL);
    zc_hh[n] = zc_context((uint8_t)n, HH);
    // Impossible sign combinations (both bits of a field set) are 0 in the
    // reference's table.
    bool possible = true;
    for (int sh = 0; sh < 8; sh += 2) possible = possible && ((n >> sh) & 3) != 3;
    if (possible) {
      sc_context((uint8_t)n, sc_label[n], sc_xor[n]);
    } else {
      sc_label[n] = 0;
      sc_xor[n] = 0;
    }
  }
}

// decode_inner (bitplane.rs:90-185): `data` holds the block's segments back to
// back; segment k covers bytes [seg_start[k], seg_start[k+1]) and coding
// passes [seg_pass[k], seg_pass[k+1]).
bool classic_block_decode(const uint8_t* data, const std::vector<size_t>& seg_start,
                          const std::vector<uint32_t>& seg_pass, uint32_t w, uint32_t h, uint32_t missing,
                          uint32_t num_passes, uint32_t total_bitplanes, int band, uint8_t style, int32_t* out,
                          size_t out_stride) {
  Block b;
  b.w = w;
  b.h = h;
  b.pw = w + 2;
  b.band = band;
  b.style = style;
  const size_t n = (size_t)(w + 2) * (h + 2);
  b.coef.assign(n, 0);
  b.state.assign(n, 0);
  b.nb.assign(n, 0);
  b.reset_contexts();
  // reset_for_job (bitplane.rs:493-548), non-strict.
  b.bitplanes = (uint8_t)(total_bitplanes > missing ? total_bitplanes - missing : 0);
  b.max_passes = (uint8_t)(b.bitplanes == 0 ? 0 : 1 + 3 * (b.bitplanes - 1));
  if (num_passes != 0 && b.bitplanes != 0) {
    const bool normal = !(style & 0x01) && !(style & 0x04);
    if (normal) {
      Mq dec(data, seg_start.back());
      b.passes(0, num_passes < b.max_passes ? num_passes : b.max_passes, dec, false);
    } else {
      for (size_t k = 0; k + 1 < seg_pass.size(); ++k) {
        const uint32_t s = seg_pass[k], e0 = seg_pass[k + 1];
        const uint32_t e = e0 < b.max_passes ? e0 : b.max_passes;
        const uint8_t* d = data + seg_start[k];
        const size_t len = seg_start[k + 1] - seg_start[k];
        const bool arith = !(style & 0x01) || s <= 9 || s % 3 == 0;
        if (arith) {
          Mq dec(d, len);
          b.passes(s, e, dec, false);
        } else {
          Raw dec{d, len};
          b.passes(s, e, dec, true);
        }
      }
    }
  }
  for (uint32_t y = 0; y < h; ++y)
    for (uint32_t x = 0; x < w; ++x) {
      const uint32_t v = b.coef[b.at(x, y)];
      const int32_t m = (int32_t)(v & 0x7FFFFFFFu);
      out[(size_t)y * out_stride + x] = (v >> 31) ? -m : m;
    }
  return true;
}

}  // namespace oracle
