// Classic (EBCOT) Tier-1 code-block encoder: the input side of the classic
// decode path's tests and benchmarks.  Written from ISO/IEC 15444-1 Annex C
// (MQ encoder: INITENC, CODEMPS, CODELPS, RENORME, BYTEOUT, FLUSH) and
// Annex D (significance propagation, magnitude refinement and cleanup passes
// with their contexts), making the same context decisions as the decoder
// (crates/signinum-j2k-native/src/j2c/bitplane.rs), for every code-block
// style: arithmetic-coding bypass, context reset, termination on every pass,
// vertically causal context, segmentation symbols.
#include <algorithm>
#include <cstdint>
#include <vector>

#include "../ebcot.h"
#include "j2k_encode.h"

namespace sgn {
namespace enc {
namespace {

using namespace ebcot;

struct Cx {
  uint8_t index = 0, mps = 0;
};

// MQ encoder (C.2); out[0] is the virtual byte before the codeword.
struct MqEncoder {
  std::vector<uint8_t> buf{0};
  uint32_t a = 0x8000, c = 0;
  int ct = 12;
  void byteout() {
    uint8_t& b = buf.back();
    if (b == 0xFF) {
      buf.push_back((uint8_t)(c >> 20));
      c &= 0xFFFFF;
      ct = 7;
    } else if (c < 0x8000000) {
      buf.push_back((uint8_t)(c >> 19));
      c &= 0x7FFFF;
      ct = 8;
    } else {
      ++b;
      if (b == 0xFF) {
        c &= 0x7FFFFFF;
        buf.push_back((uint8_t)(c >> 20));
        c &= 0xFFFFF;
        ct = 7;
      } else {
        buf.push_back((uint8_t)(c >> 19));
        c &= 0x7FFFF;
        ct = 8;
      }
    }
  }
  void renorm() {
    do {
      a <<= 1;
      c <<= 1;
      if (--ct == 0) byteout();
    } while ((a & 0x8000) == 0);
  }
  void encode(Cx& cx, uint32_t d) {
    const uint32_t qe = kQe[cx.index];
    if (d == cx.mps) {
      a -= qe;
      if ((a & 0x8000) == 0) {
        if (a < qe) a = qe;
        else c += qe;
        cx.index = kNmps[cx.index];
        renorm();
      } else {
        c += qe;
      }
    } else {
      a -= qe;
      if (a < qe) c += qe;
      else a = qe;
      if (kSwitch[cx.index]) cx.mps ^= 1;
      cx.index = kNlps[cx.index];
      renorm();
    }
  }
  // FLUSH (C.2.9): the codeword bytes, a trailing 0xFF dropped (the decoder
  // reads 0xFF past the end).
  std::vector<uint8_t> flush() {
    const uint32_t temp = c + a;
    c |= 0xFFFF;
    if (c >= temp) c -= 0x8000;
    c <<= ct;
    byteout();
    c <<= ct;
    byteout();
    std::vector<uint8_t> out(buf.begin() + 1, buf.end());
    if (!out.empty() && out.back() == 0xFF) out.pop_back();
    return out;
  }
};

// Raw bits for bypassed passes: MSB first, a byte after 0xFF carries 7 bits
// (its MSB a stuffed 0).  A final 0xFF gets a following 0x00 so a decoder
// that reads the stuff bit after it finds one.
struct RawEncoder {
  std::vector<uint8_t> out;
  uint32_t cur = 0;
  int nbits = 0, cap = 8;
  void encode(Cx&, uint32_t d) {
    cur = (cur << 1) | (d & 1);
    if (++nbits == cap) {
      out.push_back((uint8_t)cur);
      cap = cur == 0xFF ? 7 : 8;
      cur = 0;
      nbits = 0;
    }
  }
  std::vector<uint8_t> flush() {
    if (nbits) out.push_back((uint8_t)(cur << (cap - nbits)));
    if (!out.empty() && out.back() == 0xFF) out.push_back(0x00);
    return out;
  }
};

struct BlockCoder {
  uint32_t w, h, pw;
  uint8_t band, style;
  int pos = 0;
  std::vector<uint32_t> mag, sgn;
  std::vector<uint8_t> state, nb;  // state: 0x80 significant, 0x40 refined, 0x20 coded in this bit-plane
  Cx cx[19];
  void reset_contexts() {
    for (int k = 0; k < 19; ++k) cx[k] = Cx{initial_index(k), 0};
  }
  size_t at(uint32_t x, uint32_t y) const { return (size_t)(y + 1) * pw + x + 1; }
  bool next_stripe(uint32_t y) const { return y + 1 < h && ((y + 1) >> 2) > (y >> 2); }
  uint8_t neighbors(size_t i, uint32_t y) const {
    return ((style & kVCausal) && next_stripe(y)) ? (uint8_t)(nb[i] & 0xF4) : nb[i];
  }
  uint32_t bit(size_t i) const { return (mag[i] >> pos) & 1; }
  void set_significant(size_t i) {
    state[i] |= 0x80;
    nb[i - pw - 1] |= 1 << 1;
    nb[i - pw] |= 1 << 0;
    nb[i - pw + 1] |= 1 << 3;
    nb[i - 1] |= 1 << 2;
    nb[i + 1] |= 1 << 4;
    nb[i + pw - 1] |= 1 << 5;
    nb[i + pw] |= 1 << 6;
    nb[i + pw + 1] |= 1 << 7;
  }
  uint32_t sig_sign(size_t j) const { return (state[j] & 0x80) ? sgn[j] : 0; }
  template <typename E>
  void code_sign(size_t i, uint32_t y, E& e, bool raw) {
    const uint8_t s = neighbors(i, y) & 0x55;
    const uint32_t bottom = ((style & kVCausal) && next_stripe(y)) ? 0 : sig_sign(i + pw);
    const uint32_t signs = (sig_sign(i - pw) << 6) | (sig_sign(i - 1) << 4) | (sig_sign(i + 1) << 2) | bottom;
    uint8_t label, xr;
    sc_context((uint8_t)(((s & signs) << 1) | (s & ~signs)), label, xr);
    e.encode(cx[label], raw ? sgn[i] : (sgn[i] ^ xr));
  }
  template <typename E>
  void cleanup_coefficient(size_t i, uint32_t y, E& e, bool raw) {
    if (state[i] & 0xA0) return;
    const uint32_t b = bit(i);
    e.encode(cx[zc_context(neighbors(i, y), band)], b);
    if (b) {
      code_sign(i, y, e, raw);
      set_significant(i);
    }
  }
  template <typename E>
  void cleanup(E& e, bool raw) {
    for (uint32_t by = 0; by < h; by += 4) {
      const uint32_t ye = std::min(by + 4, h);
      for (uint32_t x = 0; x < w; ++x) {
        const size_t top = at(x, by);
        bool run = ye - by == 4;
        for (uint32_t y = by; run && y < ye; ++y) {
          const size_t i = top + (size_t)(y - by) * pw;
          run = !(state[i] & 0xA0) && neighbors(i, y) == 0;
        }
        if (run) {
          uint32_t f = 4;
          for (uint32_t k = 0; k < 4 && f == 4; ++k)
            if (bit(top + (size_t)k * pw)) f = k;
          e.encode(cx[17], f < 4 ? 1 : 0);
          if (f == 4) continue;
          e.encode(cx[18], f >> 1);
          e.encode(cx[18], f & 1);
          const size_t si = top + (size_t)f * pw;
          code_sign(si, by + f, e, raw);
          set_significant(si);
          for (uint32_t y = by + f + 1; y < ye; ++y) cleanup_coefficient(top + (size_t)(y - by) * pw, y, e, raw);
          continue;
        }
        for (uint32_t y = by; y < ye; ++y) cleanup_coefficient(top + (size_t)(y - by) * pw, y, e, raw);
      }
    }
    if (style & kSegSym) {
      e.encode(cx[18], 1);
      e.encode(cx[18], 0);
      e.encode(cx[18], 1);
      e.encode(cx[18], 0);
    }
    for (auto& s : state) s &= (uint8_t)~0x20;
  }
  template <typename E>
  void sig_prop(E& e, bool raw) {
    for (uint32_t by = 0; by < h; by += 4) {
      const uint32_t ye = std::min(by + 4, h);
      for (uint32_t x = 0; x < w; ++x)
        for (uint32_t y = by; y < ye; ++y) {
          const size_t i = at(x, y);
          const uint8_t n = neighbors(i, y);
          if ((state[i] & 0x80) || n == 0) continue;
          const uint32_t b = bit(i);
          e.encode(cx[zc_context(n, band)], b);
          state[i] |= 0x20;
          if (b) {
            code_sign(i, y, e, raw);
            set_significant(i);
          }
        }
    }
  }
  template <typename E>
  void mag_ref(E& e) {
    for (uint32_t by = 0; by < h; by += 4) {
      const uint32_t ye = std::min(by + 4, h);
      for (uint32_t x = 0; x < w; ++x)
        for (uint32_t y = by; y < ye; ++y) {
          const size_t i = at(x, y);
          if (!(state[i] & 0x80) || (state[i] & 0x20)) continue;
          e.encode(cx[mr_context((state[i] & 0x40) != 0, neighbors(i, y))], bit(i));
          state[i] |= 0x40;
        }
    }
  }
};

}  // namespace

int encode_classic_block(const int32_t* c, size_t stride, uint32_t w, uint32_t h, uint32_t Mb, uint8_t band_class,
                         uint8_t style, ClassicBlockOut& out) {
  out = ClassicBlockOut();
  BlockCoder bc;
  bc.w = w;
  bc.h = h;
  bc.pw = w + 2;
  bc.band = band_class;
  bc.style = style;
  const size_t n = (size_t)(w + 2) * (h + 2);
  bc.mag.assign(n, 0);
  bc.sgn.assign(n, 0);
  bc.state.assign(n, 0);
  bc.nb.assign(n, 0);
  uint32_t maxmag = 0;
  for (uint32_t y = 0; y < h; ++y)
    for (uint32_t x = 0; x < w; ++x) {
      const int32_t v = c[(size_t)y * stride + x];
      const uint32_t m = (uint32_t)(v < 0 ? -(int64_t)v : v);
      bc.mag[bc.at(x, y)] = m;
      bc.sgn[bc.at(x, y)] = v < 0 ? 1 : 0;
      maxmag = std::max(maxmag, m);
    }
  uint32_t planes = 0;
  while (planes < 32 && (maxmag >> planes)) ++planes;
  if (planes > Mb) return -3;
  out.zero_planes = Mb - planes;
  if (planes == 0) return 0;  // not included in the packet
  out.passes = 1 + 3 * (planes - 1);
  bc.reset_contexts();
  // Segment boundaries: one for the whole block, one per pass with TERMALL,
  // raw/MQ segments with BYPASS.
  auto seg_of = [&](uint32_t p) -> uint32_t {
    if (style & kTermAll) return p;
    if (style & kBypass) return bypass_segment(p);
    return 0;
  };
  MqEncoder mq;
  RawEncoder raw;
  uint32_t seg_first = 0;
  bool seg_arith = true;
  auto finish = [&](uint32_t end_pass) {
    std::vector<uint8_t> bytes = seg_arith ? mq.flush() : raw.flush();
    out.seg_len.push_back((uint32_t)bytes.size());
    out.seg_passes.push_back(end_pass - seg_first);
    out.bytes.insert(out.bytes.end(), bytes.begin(), bytes.end());
    mq = MqEncoder();
    raw = RawEncoder();
  };
  for (uint32_t p = 0; p < out.passes; ++p) {
    if (p > 0 && seg_of(p) != seg_of(p - 1)) {
      finish(p);
      seg_first = p;
    }
    if (p == seg_first) seg_arith = segment_is_arithmetic(style, p);
    bc.pos = (int)(planes - 1 - (p + 2) / 3);
    switch (p % 3) {
      case 0:
        if (seg_arith) bc.cleanup(mq, false);
        else bc.cleanup(raw, true);
        break;
      case 1:
        if (seg_arith) bc.sig_prop(mq, false);
        else bc.sig_prop(raw, true);
        break;
      default:
        if (seg_arith) bc.mag_ref(mq);
        else bc.mag_ref(raw);
        break;
    }
    if (style & kReset) bc.reset_contexts();
  }
  finish(out.passes);
  return 0;
}

}  // namespace enc
}  // namespace sgn
