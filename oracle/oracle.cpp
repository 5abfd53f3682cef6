// TEST INFRASTRUCTURE ONLY — the parity oracle (see oracle_internal.h).
//
// Codestream parsing, tile geometry, packet parsing (HT and classic), the
// per-sub-band block decode drivers, dequantisation, the inverse 5/3 and 9/7
// DWTs, inverse RCT and ICT, DC shift and the pixel-format conversions,
// restated from crates/signinum-j2k-native and crates/signinum-j2k.  Scope:
// raw J2K codestreams and JP2 files; PPM/PPT and sub-sampled components are
// reported as unsupported here.
#include <algorithm>
#include <array>
#include <cstdio>
#include <string>
#include <tuple>
#include <cmath>
#include <cstring>
#include <memory>
#include <utility>

#include "oracle_internal.h"

namespace oracle {

IntRect IntRect::intersect(const IntRect& o) const {
  IntRect r;
  r.x0 = std::max(x0, o.x0);
  r.y0 = std::max(y0, o.y0);
  r.x1 = std::min(x1, o.x1);
  r.y1 = std::min(y1, o.y1);
  if (r.x1 < r.x0) r.x1 = r.x0;
  if (r.y1 < r.y0) r.y1 = r.y0;
  return r;
}

int bytes_per_pixel(int fmt) {
  switch (fmt) {
    case FMT_GRAY8: return 1;
    case FMT_RGB8: return 3;
    case FMT_RGBA8: return 4;
    case FMT_GRAY16: return 2;
    case FMT_RGB16: return 6;
    case FMT_RGBA16: return 8;
  }
  return 0;
}

[[noreturn]] static void fail(Status s, const char* msg) { throw DecodeError{s, msg}; }

static inline uint32_t div_ceil(uint32_t a, uint32_t b) { return (uint32_t)(((uint64_t)a + b - 1) / b); }
static inline uint64_t div_ceil64(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

// ---------------------------------------------------------------------------
// BitReader, crates/signinum-j2k-native/src/reader.rs:7-187.
struct BitReader {
  const uint8_t* data = nullptr;
  size_t len = 0;
  size_t cur = 0;  // bit position
  BitReader() = default;
  BitReader(const uint8_t* d, size_t n) : data(d), len(n), cur(0) {}
  size_t byte_pos() const { return cur / 8; }
  size_t bit_pos() const { return cur % 8; }
  bool at_end() const { return byte_pos() >= len; }
  void align() {
    size_t b = bit_pos();
    if (b) cur += 8 - b;
  }
  bool peek_bytes(size_t n, const uint8_t** out) const {
    size_t s = byte_pos();
    if (s + n < s || s + n > len) return false;
    *out = data + s;
    return true;
  }
  bool read_bytes(size_t n, const uint8_t** out) {
    if (!peek_bytes(n, out)) return false;
    cur += n * 8;
    return true;
  }
  bool read_byte(uint8_t* v) {
    const uint8_t* p;
    if (!read_bytes(1, &p)) return false;
    *v = *p;
    return true;
  }
  bool skip(size_t n) {
    const uint8_t* p;
    return read_bytes(n, &p);
  }
  bool read_u16(uint16_t* v) {
    const uint8_t* p;
    if (!read_bytes(2, &p)) return false;
    *v = (uint16_t)((p[0] << 8) | p[1]);
    return true;
  }
  bool read_u32(uint32_t* v) {
    const uint8_t* p;
    if (!read_bytes(4, &p)) return false;
    *v = ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3];
    return true;
  }
  bool read_bit(uint32_t* bit) {
    size_t bp = byte_pos();
    if (bp >= len) return false;
    *bit = (data[bp] >> (7 - bit_pos())) & 1;
    ++cur;
    return true;
  }
  bool read_bits_stuffed(uint32_t n, uint32_t* out) {
    uint32_t v = 0;
    for (uint32_t i = 0; i < n; ++i) {
      bool stuff = bit_pos() == 7 && byte_pos() < len && data[byte_pos()] == 0xFF;
      uint32_t b;
      if (!read_bit(&b)) return false;
      v = (v << 1) | b;
      if (stuff) {
        uint32_t sb;
        if (!read_bit(&sb) || sb != 0) return false;
      }
    }
    *out = v;
    return true;
  }
  bool read_marker(uint8_t* m) {
    if (byte_pos() >= len || data[byte_pos()] != 0xFF) return false;
    uint8_t ff;
    read_byte(&ff);
    return read_byte(m);
  }
  bool peek_marker(uint8_t* m) const {
    BitReader c = *this;
    return c.read_marker(m);
  }
};

// ---------------------------------------------------------------------------
// Main header, crates/signinum-j2k-native/src/j2c/codestream.rs.
enum Prog { LRCP = 0, RLCP = 1, RPCL = 2, PCRL = 3, CPRL = 4 };
enum QStyle { QNONE = 0, QDERIVED = 1, QEXPOUNDED = 2 };

struct StepSize { uint16_t mantissa, exponent; };
struct QuantInfo { int style = QNONE; uint8_t guard = 0; std::vector<StepSize> steps; };
struct CodingParams {
  uint8_t ndecomp = 0, nres = 1, cbw = 0, cbh = 0, cbstyle = 0;
  bool reversible = true;
  std::vector<std::pair<uint8_t, uint8_t>> pexp;
};
struct CompSize { uint8_t precision, xr, yr; };
struct CompInfo {
  CompSize size;
  uint8_t flags = 0;  // Scod / Scoc flags
  CodingParams cp;
  QuantInfo q;
  bool ht() const { return (cp.cbstyle & 0x40) != 0; }
  bool causal() const { return (cp.cbstyle & 0x08) != 0; }
  // ComponentInfo::exponent_mantissa, codestream.rs:224-268.
  std::pair<uint16_t, uint16_t> exponent_mantissa(int sb, uint8_t resolution) const {
    int sb_index = sb == HL ? 0 : sb == LH ? 1 : sb == HH ? 2 : 0xFFFF;
    if (q.style == QNONE || q.style == QEXPOUNDED) {
      size_t idx = resolution == 0 ? 0 : 1 + (size_t)(resolution - 1) * 3 + (size_t)sb_index;
      if (idx >= q.steps.size()) fail(ERR_DECODE, "missing step size");
      return {q.steps[idx].exponent, q.steps[idx].mantissa};
    }
    if (q.steps.empty()) fail(ERR_DECODE, "missing step size");
    uint16_t n_ll = cp.ndecomp;
    uint16_t n_b = resolution == 0 ? n_ll : (uint16_t)(n_ll + 1 - resolution);
    int e = (int)q.steps[0].exponent - n_ll;
    if (e < 0) fail(ERR_DECODE, "invalid exponents");
    return {(uint16_t)(e + n_b), q.steps[0].mantissa};
  }
};

struct SizeData {
  uint32_t gw, gh, ox, oy, tw, th, tox, toy;
  std::vector<CompSize> comps;
  uint32_t xsf = 1, ysf = 1, xrsf = 1, yrsf = 1;
  uint32_t ntx() const { return div_ceil(gw - tox, tw); }
  uint32_t nty() const { return div_ceil(gh - toy, th); }
  uint32_t ntiles() const { return ntx() * nty(); }
  uint32_t image_width() const { return div_ceil(gw - ox, xsf * xrsf); }
  uint32_t image_height() const { return div_ceil(gh - oy, ysf * yrsf); }
};

struct Header {
  SizeData siz;
  int prog = LRCP;
  uint8_t num_layers = 1;
  bool mct = false;
  std::vector<CompInfo> comps;
  uint8_t skipped = 0;
  bool strict = false;
};

static bool skip_segment(BitReader& r) {
  uint16_t l;
  if (!r.read_u16(&l) || l < 2) return false;
  return r.skip(l - 2);
}

// coding_style_parameters, codestream.rs:702-747.
static bool coding_params(BitReader& r, uint8_t flags, CodingParams& cp) {
  uint8_t nd, cw, ch, st, tr;
  if (!r.read_byte(&nd) || nd > 32) return false;
  cp.ndecomp = nd;
  cp.nres = (uint8_t)(nd + 1);
  if (!r.read_byte(&cw) || !r.read_byte(&ch) || !r.read_byte(&st) || !r.read_byte(&tr)) return false;
  if (cw > 253 || ch > 253) return false;
  cp.cbw = (uint8_t)(cw + 2);
  cp.cbh = (uint8_t)(ch + 2);
  cp.cbstyle = st;
  if (tr > 1) return false;
  cp.reversible = tr == 1;
  cp.pexp.clear();
  for (int i = 0; i < cp.nres; ++i) {
    if (flags & 1) {
      uint8_t v;
      if (!r.read_byte(&v)) return false;
      cp.pexp.push_back({(uint8_t)(v & 0xF), (uint8_t)(v >> 4)});
    } else {
      cp.pexp.push_back({15, 15});
    }
  }
  return true;
}

struct CodMarker { uint8_t flags; int prog; uint8_t layers; bool mct; CodingParams cp; };

// cod_marker, codestream.rs:794-825.
static bool cod_marker(BitReader& r, CodMarker& c) {
  uint16_t l, layers;
  uint8_t po, m;
  if (!r.read_u16(&l) || !r.read_byte(&c.flags) || !r.read_byte(&po) || po > 4) return false;
  c.prog = po;
  if (!r.read_u16(&layers) || layers == 0 || layers > 32) return false;
  c.layers = (uint8_t)layers;
  if (!r.read_byte(&m)) return false;
  c.mct = m == 1;
  return coding_params(r, c.flags, c.cp);
}

// coc_marker, codestream.rs:828-852.
static bool coc_marker(BitReader& r, uint16_t csiz, uint16_t& idx, uint8_t& flags, CodingParams& cp) {
  uint16_t l;
  if (!r.read_u16(&l)) return false;
  if (csiz < 257) {
    uint8_t b;
    if (!r.read_byte(&b)) return false;
    idx = b;
  } else if (!r.read_u16(&idx)) return false;
  if (!r.read_byte(&flags)) return false;
  return coding_params(r, flags, cp);
}

// quantization_parameters, codestream.rs:897-940.
static bool quant_params(BitReader& r, int style, size_t remaining, QuantInfo& q) {
  q.style = style;
  q.steps.clear();
  if (style == QNONE) {
    for (size_t i = 0; i < remaining; ++i) {
      uint8_t v;
      if (!r.read_byte(&v)) return false;
      q.steps.push_back({0, (uint16_t)(v >> 3)});
    }
  } else if (style == QDERIVED) {
    uint16_t v;
    if (!r.read_u16(&v)) return false;
    q.steps.push_back({(uint16_t)(v & 0x7FF), (uint16_t)(v >> 11)});
  } else {
    for (size_t i = 0; i < remaining / 2; ++i) {
      uint16_t v;
      if (!r.read_u16(&v)) return false;
      q.steps.push_back({(uint16_t)(v & 0x7FF), (uint16_t)(v >> 11)});
    }
  }
  return true;
}

// qcd_marker / qcc_marker, codestream.rs:855-894.
static bool qcd_marker(BitReader& r, QuantInfo& q) {
  uint16_t l;
  uint8_t s;
  if (!r.read_u16(&l) || !r.read_byte(&s) || l < 3) return false;
  int style = s & 0x1F;
  if (style > 2) return false;
  if (!quant_params(r, style, l - 3, q)) return false;
  q.guard = (s >> 5) & 7;
  return true;
}

static bool qcc_marker(BitReader& r, uint16_t csiz, uint16_t& idx, QuantInfo& q) {
  uint16_t l;
  if (!r.read_u16(&l)) return false;
  size_t isz = csiz < 257 ? 1 : 2;
  if (csiz < 257) {
    uint8_t b;
    if (!r.read_byte(&b)) return false;
    idx = b;
  } else if (!r.read_u16(&idx)) return false;
  uint8_t s;
  if (!r.read_byte(&s)) return false;
  int style = s & 0x1F;
  if (style > 2) return false;
  if ((size_t)l < 2 + isz + 1) return false;
  if (!quant_params(r, style, (size_t)l - 2 - isz - 1, q)) return false;
  q.guard = (s >> 5) & 7;
  return true;
}

// size_marker / size_marker_inner, codestream.rs:500-698.
static void size_marker(BitReader& r, SizeData& s) {
  uint16_t l, caps, csiz;
  bool ok = r.read_u16(&l) && r.read_u16(&caps) && r.read_u32(&s.gw) && r.read_u32(&s.gh) && r.read_u32(&s.ox) &&
            r.read_u32(&s.oy) && r.read_u32(&s.tw) && r.read_u32(&s.th) && r.read_u32(&s.tox) &&
            r.read_u32(&s.toy) && r.read_u16(&csiz);
  if (!ok || s.ox >= s.gw || s.oy >= s.gh || csiz == 0) fail(ERR_DECODE, "SIZ parse failure");
  for (uint16_t i = 0; i < csiz; ++i) {
    uint8_t ss, xr, yr;
    if (!r.read_byte(&ss) || !r.read_byte(&xr) || !r.read_byte(&yr)) fail(ERR_DECODE, "SIZ parse failure");
    uint8_t prec = (uint8_t)((ss & 0x7F) + 1);
    if (prec > 32) fail(ERR_DECODE, "SIZ parse failure");
    s.comps.push_back({prec, xr, yr});
  }
  bool same = true;
  for (size_t i = 1; i < s.comps.size(); ++i)
    same = same && s.comps[i].xr == s.comps[0].xr && s.comps[i].yr == s.comps[0].yr;
  if (same) {
    s.xsf = s.comps[0].xr;
    s.ysf = s.comps[0].yr;
  }
  if (s.tw == 0 || s.th == 0 || s.gw == 0 || s.gh == 0) fail(ERR_DECODE, "invalid dimensions");
  if (s.tox >= s.gw || s.toy >= s.gh) fail(ERR_DECODE, "invalid dimensions");
  if (s.tox > s.ox || s.toy > s.oy) fail(ERR_DECODE, "invalid tile offsets");
  if ((uint64_t)s.tox + s.tw <= s.ox || (uint64_t)s.toy + s.th <= s.oy) fail(ERR_DECODE, "invalid tile offsets");
  for (auto& c : s.comps)
    if (c.precision == 0 || c.xr == 0 || c.yr == 0) fail(ERR_DECODE, "invalid component metadata");
  if (s.image_width() > 60000 || s.image_height() > 60000) fail(ERR_DECODE, "image too large");
}

// read_header, codestream.rs:38-187 (with validate, :189-213).
static Header read_header(BitReader& r, const uint32_t* target) {
  uint8_t m;
  if (!r.read_marker(&m) || m != 0x51) fail(ERR_DECODE, "expected SIZ");
  Header h;
  size_marker(r, h.siz);
  uint16_t nc = (uint16_t)h.siz.comps.size();
  bool have_cod = false, have_qcd = false;
  CodMarker cod{};
  QuantInfo qcd;
  std::vector<std::unique_ptr<std::pair<uint8_t, CodingParams>>> coc(nc);
  std::vector<std::unique_ptr<QuantInfo>> qcc(nc);
  for (;;) {
    if (!r.peek_marker(&m)) fail(ERR_DECODE, "invalid marker");
    if (m == 0x90) break;
    r.read_marker(&m);
    switch (m) {
      case 0x50: case 0x59: case 0x5E: case 0x55: case 0x64: case 0x63:  // CAP CPF RGN TLM COM CRG
        if (!skip_segment(r)) fail(ERR_DECODE, "marker parse failure");
        break;
      case 0x52:
        if (!cod_marker(r, cod)) fail(ERR_DECODE, "COD parse failure");
        have_cod = true;
        break;
      case 0x53: {
        uint16_t idx;
        uint8_t flags;
        CodingParams cp;
        if (!coc_marker(r, nc, idx, flags, cp) || idx >= nc) fail(ERR_DECODE, "COC parse failure");
        coc[idx].reset(new std::pair<uint8_t, CodingParams>(flags, cp));
        break;
      }
      case 0x5C:
        if (!qcd_marker(r, qcd)) fail(ERR_DECODE, "QCD parse failure");
        have_qcd = true;
        break;
      case 0x5D: {
        uint16_t idx;
        QuantInfo q;
        if (!qcc_marker(r, nc, idx, q) || idx >= nc) fail(ERR_DECODE, "QCC parse failure");
        qcc[idx].reset(new QuantInfo(q));
        break;
      }
      case 0x60: fail(ERR_UNSUPPORTED, "PPM is outside the oracle's scope");
      default:
        if (m >= 0x30 && m <= 0x3F) break;
        fail(ERR_UNSUPPORTED, "unsupported marker");
    }
  }
  if (!have_cod) fail(ERR_DECODE, "missing COD");
  if (!have_qcd) fail(ERR_DECODE, "missing QCD");
  h.prog = cod.prog;
  h.num_layers = cod.layers;
  h.mct = cod.mct;
  for (uint16_t i = 0; i < nc; ++i) {
    CompInfo ci;
    ci.size = h.siz.comps[i];
    if (coc[i]) {
      ci.flags = (uint8_t)(coc[i]->first | cod.flags);
      ci.cp = coc[i]->second;
    } else {
      ci.flags = cod.flags;
      ci.cp = cod.cp;
    }
    ci.q = qcc[i] ? *qcc[i] : qcd;
    h.comps.push_back(ci);
  }
  uint8_t min_res = 255;
  for (auto& c : h.comps) min_res = std::min(min_res, c.cp.nres);
  uint32_t skipped = 0;
  if (target) {
    uint32_t wr = h.siz.image_width() / target[0], hr = h.siz.image_height() / target[1];
    uint32_t wl = wr ? 31 - (uint32_t)__builtin_clz(wr) : 0;
    uint32_t hl = hr ? 31 - (uint32_t)__builtin_clz(hr) : 0;
    skipped = std::min(wl, hl);
  }
  skipped = std::min<uint32_t>(skipped, (uint32_t)(min_res - 1));
  h.skipped = (uint8_t)skipped;
  h.siz.xrsf *= 1u << skipped;
  h.siz.yrsf *= 1u << skipped;
  for (auto& c : h.comps) {
    size_t max_res = (size_t)c.cp.nres - 1, n = c.q.steps.size();
    if (n == 0) fail(ERR_DECODE, "missing precinct exponents");
    if (c.q.style != QDERIVED && max_res != 0 && 1 + (max_res - 1) * 3 + 2 >= n)
      fail(ERR_DECODE, "insufficient exponents");
  }
  return h;
}

// ---------------------------------------------------------------------------
// Tiles, crates/signinum-j2k-native/src/j2c/tile.rs.
struct Tile {
  uint32_t idx;
  std::vector<BitReader> parts;  // merged tile parts
  std::vector<CompInfo> comps;
  IntRect rect;
  int prog;
  uint8_t num_layers;
  bool mct;
};

static Tile make_tile(uint32_t idx, const Header& h) {
  const SizeData& s = h.siz;
  uint32_t xc = idx % s.ntx(), yc = idx / s.ntx();
  Tile t;
  t.idx = idx;
  t.rect = IntRect::ltrb(std::max(s.tox + xc * s.tw, s.ox), std::max(s.toy + yc * s.th, s.oy),
                         std::min(s.tox + (xc + 1) * s.tw, s.gw), std::min(s.toy + (yc + 1) * s.th, s.gh));
  t.comps = h.comps;
  t.prog = h.prog;
  t.mct = h.mct;
  t.num_layers = h.num_layers;
  return t;
}

// parse_tile_part, tile.rs:162-306.
static void parse_tile_part(BitReader& r, const Header& h, std::vector<Tile>& tiles) {
  uint8_t m;
  if (!r.read_marker(&m) || m != 0x90) fail(ERR_DECODE, "expected SOT");
  uint16_t l, ti;
  uint32_t psot;
  uint8_t tp, ntp;
  if (!r.read_u16(&l) || !r.read_u16(&ti) || !r.read_u32(&psot) || !r.read_byte(&tp) || !r.read_byte(&ntp))
    fail(ERR_DECODE, "SOT parse failure");
  if (ti >= h.siz.ntiles()) fail(ERR_DECODE, "invalid tile index");
  size_t data_len;
  if (psot == 0) {
    data_len = r.len > r.byte_pos() ? r.len - r.byte_pos() : 0;
  } else {
    if (psot < 12) fail(ERR_DECODE, "invalid tile");
    data_len = psot - 12;
  }
  size_t start = r.byte_pos();
  Tile& t = tiles[ti];
  uint16_t nc = (uint16_t)t.comps.size();
  for (;;) {
    if (!r.peek_marker(&m)) {
      if (h.strict) fail(ERR_DECODE, "invalid marker");
      return;
    }
    if (m == 0x93) {
      r.read_marker(&m);
      break;
    }
    if (m == 0xD9) break;
    r.read_marker(&m);
    switch (m) {
      case 0x52: {
        CodMarker cod;
        if (!cod_marker(r, cod)) fail(ERR_DECODE, "COD parse failure");
        t.mct = cod.mct;
        t.num_layers = cod.layers;
        t.prog = cod.prog;
        for (auto& c : t.comps) {
          c.flags |= cod.flags;
          c.cp = cod.cp;
        }
        break;
      }
      case 0x53: {
        uint16_t idx;
        uint8_t flags;
        CodingParams cp;
        if (!coc_marker(r, nc, idx, flags, cp)) fail(ERR_DECODE, "COC parse failure");
        if (idx >= nc) fail(ERR_DECODE, "invalid component metadata");
        t.comps[idx].cp = cp;
        t.comps[idx].flags |= flags;
        break;
      }
      case 0x5C: {
        QuantInfo q;
        if (!qcd_marker(r, q)) fail(ERR_DECODE, "QCD parse failure");
        for (auto& c : t.comps) c.q = q;
        break;
      }
      case 0x5D: {
        uint16_t idx;
        QuantInfo q;
        if (!qcc_marker(r, nc, idx, q)) fail(ERR_DECODE, "QCC parse failure");
        if (idx >= nc) fail(ERR_DECODE, "invalid component metadata");
        t.comps[idx].q = q;
        break;
      }
      case 0x61: fail(ERR_UNSUPPORTED, "PPT is outside the oracle's scope");
      case 0x58: case 0x64:
        if (!skip_segment(r)) fail(ERR_DECODE, "marker parse failure");
        break;
      default:
        if (m >= 0x30 && m <= 0x3F) break;
        fail(ERR_UNSUPPORTED, "unsupported marker");
    }
  }
  size_t used = r.byte_pos() - start;
  if (used > data_len) {
    if (h.strict) fail(ERR_DECODE, "invalid tile");
    return;
  }
  const uint8_t* p;
  if (!r.read_bytes(data_len - used, &p)) fail(ERR_TRUNCATED, "tile-part data truncated");
  t.parts.emplace_back(p, data_len - used);
}

// tile::parse, tile.rs:131-160.
static std::vector<Tile> parse_tiles(BitReader& r, const Header& h) {
  std::vector<Tile> tiles;
  for (uint32_t i = 0; i < h.siz.ntiles(); ++i) tiles.push_back(make_tile(i, h));
  parse_tile_part(r, h, tiles);
  uint8_t m;
  while (r.peek_marker(&m) && m == 0x90) parse_tile_part(r, h, tiles);
  return tiles;
}

// ComponentTile::new (B-12), tile.rs:330-360.
static IntRect comp_rect(const Tile& t, const CompInfo& c) {
  if (c.size.xr == 1 && c.size.yr == 1) return t.rect;
  return IntRect::ltrb(div_ceil(t.rect.x0, c.size.xr), div_ceil(t.rect.y0, c.size.yr), div_ceil(t.rect.x1, c.size.xr),
                       div_ceil(t.rect.y1, c.size.yr));
}

struct ResTile {
  uint8_t res, dlevel;
  IntRect crect;  // component tile rect
  IntRect rect;
  const CompInfo* ci;
  const Tile* tile;
};

// ResolutionTile::new (B-14), tile.rs:380-437.
static ResTile res_tile(const Tile& t, const CompInfo& c, uint8_t r) {
  ResTile rt;
  rt.res = r;
  rt.ci = &c;
  rt.tile = &t;
  rt.crect = comp_rect(t, c);
  uint64_t d = (uint64_t)1 << (c.cp.ndecomp - r);
  rt.rect = IntRect::ltrb((uint32_t)div_ceil64(rt.crect.x0, d), (uint32_t)div_ceil64(rt.crect.y0, d),
                          (uint32_t)div_ceil64(rt.crect.x1, d), (uint32_t)div_ceil64(rt.crect.y1, d));
  rt.dlevel = r == 0 ? c.cp.ndecomp : (uint8_t)(c.cp.ndecomp - (r - 1));
  return rt;
}

// sub_band_rect (B-15), tile.rs:439-485.
static IntRect sub_band_rect(const ResTile& rt, int sb) {
  uint64_t xo = (sb == HL || sb == HH) ? 1 : 0, yo = (sb == LH || sb == HH) ? 1 : 0;
  uint64_t nx = 0, ny = 0;
  if (rt.dlevel > 0) {
    nx = ((uint64_t)1 << (rt.dlevel - 1)) * xo;
    ny = ((uint64_t)1 << (rt.dlevel - 1)) * yo;
  }
  uint64_t den = (uint64_t)1 << rt.dlevel;
  auto f = [&](uint32_t v, uint64_t n) { return (uint32_t)div_ceil64(v > n ? v - n : 0, den); };
  return IntRect::ltrb(f(rt.crect.x0, nx), f(rt.crect.y0, ny), f(rt.crect.x1, nx), f(rt.crect.y1, ny));
}

static uint32_t npx(const ResTile& rt) {
  if (rt.rect.x0 == rt.rect.x1) return 0;
  uint32_t e = rt.ci->cp.pexp[rt.res].first;
  return (uint32_t)(div_ceil64(rt.rect.x1, (uint64_t)1 << e) - (rt.rect.x0 >> e));
}
static uint32_t npy(const ResTile& rt) {
  if (rt.rect.y0 == rt.rect.y1) return 0;
  uint32_t e = rt.ci->cp.pexp[rt.res].second;
  return (uint32_t)(div_ceil64(rt.rect.y1, (uint64_t)1 << e) - (rt.rect.y0 >> e));
}
static uint64_t num_precincts(const ResTile& rt) { return (uint64_t)npx(rt) * npy(rt); }

struct PrecinctData { uint32_t r_x, r_y; IntRect rect; uint64_t idx; };

static uint32_t next_multiple(uint32_t v, uint32_t m) { return v % m == 0 ? v : (v / m + 1) * m; }

// ResolutionTile::precincts, tile.rs:520-629.
static bool precincts(const ResTile& rt, std::vector<PrecinctData>& out) {
  out.clear();
  uint32_t ny = npy(rt), nx = npx(rt);
  uint32_t ppx = rt.ci->cp.pexp[rt.res].first, ppy = rt.ci->cp.pexp[rt.res].second;
  uint32_t ppx0 = ppx, ppy0 = ppy;
  uint32_t ys = (rt.rect.y0 >> ppy) << ppy, xs = (rt.rect.x0 >> ppx) << ppx;
  if (rt.res > 0) {
    if (ppx == 0 || ppy == 0) return false;
    ppx -= 1;
    ppy -= 1;
    xs /= 2;
    ys /= 2;
  }
  uint32_t pw = 1u << ppx, ph = 1u << ppy;
  uint32_t nlr = rt.ci->cp.ndecomp - rt.res;
  if (ppx0 + nlr >= 32 || ppy0 + nlr >= 32) return false;
  uint64_t xstep = (uint64_t)rt.ci->size.xr << (ppx0 + nlr), ystep = (uint64_t)rt.ci->size.yr << (ppy0 + nlr);
  if (xstep > 0xFFFFFFFFull || ystep > 0xFFFFFFFFull) return false;
  uint32_t rx0 = rt.tile->rect.x0, ry = rt.tile->rect.y0;
  if (rx0 % xstep != 0 && ((uint64_t)rt.rect.x0 << nlr) % xstep == 0) rx0 = next_multiple(rx0, (uint32_t)xstep);
  if (ry % ystep != 0 && ((uint64_t)rt.rect.y0 << nlr) % ystep == 0) ry = next_multiple(ry, (uint32_t)ystep);
  for (uint32_t y = 0; y < ny; ++y) {
    uint32_t y0 = y * ph + ys;
    uint32_t rx = rx0;
    for (uint32_t x = 0; x < nx; ++x) {
      uint32_t x0 = x * pw + xs;
      out.push_back({rx, ry, IntRect::ltrb(x0, y0, x0 + pw, y0 + ph), (uint64_t)nx * y + x});
      rx = next_multiple(rx + 1, (uint32_t)xstep);
    }
    ry = next_multiple(ry + 1, (uint32_t)ystep);
  }
  return true;
}

// code_block_width / code_block_height (B-17/B-18), tile.rs:631-667.
static uint32_t cb_w(const ResTile& rt) {
  uint32_t x = rt.ci->cp.cbw, e = rt.ci->cp.pexp[rt.res].first;
  x = rt.res > 0 ? std::min(x, e - 1) : std::min(x, e);
  return 1u << x;
}
static uint32_t cb_h(const ResTile& rt) {
  uint32_t y = rt.ci->cp.cbh, e = rt.ci->cp.pexp[rt.res].second;
  y = rt.res > 0 ? std::min(y, e - 1) : std::min(y, e);
  return 1u << y;
}

// ---------------------------------------------------------------------------
// Tag trees, crates/signinum-j2k-native/src/j2c/tag_tree.rs.
struct TagNode {
  uint32_t w, h, value = 0;
  bool init = false;
  uint16_t level;
  size_t child[4] = {SIZE_MAX, SIZE_MAX, SIZE_MAX, SIZE_MAX};
  uint32_t tlw() const { return std::min(1u << (level - 1), w); }
  uint32_t tlh() const { return std::min(1u << (level - 1), h); }
};

static size_t build_tag(uint32_t w, uint32_t h, uint16_t level, std::vector<TagNode>& nodes, TagNode& out) {
  out = TagNode();
  out.w = w;
  out.h = h;
  out.level = level;
  if (level == 0) return 0;
  uint32_t tw = out.tlw(), th = out.tlh();
  uint32_t dims[4][2] = {{tw, th}, {w - tw, th}, {tw, h - th}, {w - tw, h - th}};
  for (int i = 0; i < 4; ++i) {
    TagNode n;
    build_tag(dims[i][0], dims[i][1], (uint16_t)(level - 1), nodes, n);
    if (n.w > 0 && n.h > 0) {
      out.child[i] = nodes.size();
      nodes.push_back(n);
    }
  }
  return 0;
}

static size_t new_tag_tree(uint32_t w, uint32_t h, std::vector<TagNode>& nodes) {
  auto lg = [](uint32_t v) {
    uint32_t p = 1, l = 0;
    while (p < v) { p <<= 1; ++l; }
    return l;
  };
  uint32_t level = std::max(lg(w), lg(h));
  TagNode root;
  build_tag(w, h, (uint16_t)level, nodes, root);
  nodes.push_back(root);
  return nodes.size() - 1;
}

static bool read_tag(size_t ni, uint32_t x, uint32_t y, BitReader& r, uint32_t parent, uint32_t max_val,
                     std::vector<TagNode>& nodes, uint32_t& out) {
  TagNode& n = nodes[ni];
  if (!n.init) {
    uint32_t v = std::max(parent, n.value);
    for (;;) {
      if (v >= max_val) break;
      uint32_t b;
      if (!r.read_bits_stuffed(1, &b)) return false;
      if (b == 0) ++v;
      else {
        n.init = true;
        break;
      }
    }
    n.value = v;
  }
  if (n.value >= max_val || n.level == 0) {
    out = n.value;
    return true;
  }
  uint32_t tw = n.tlw(), th = n.tlh();
  bool left = x < tw, top = y < th;
  size_t c = n.child[(left ? 0 : 1) + (top ? 0 : 2)];
  uint32_t nx = left ? x : x - tw, ny = top ? y : y - th;
  uint32_t pv = n.value;
  return read_tag(c, nx, ny, r, pv, max_val, nodes, out);
}

// ---------------------------------------------------------------------------
// Build, crates/signinum-j2k-native/src/j2c/build.rs.
struct Segment { uint8_t idx; uint32_t len; const uint8_t* data; uint8_t passes = 0; };
struct CodeBlock {
  IntRect rect;
  uint32_t xi, yi;
  bool included = false;
  uint8_t missing = 0, passes = 0, nonempty = 0;
  uint32_t lblock = 3;
  std::vector<std::vector<Segment>> layers;  // per layer; empty vector = None
  std::vector<bool> has_layer;
};
struct Precinct { std::vector<size_t> cbs; size_t incl_tree, zbp_tree; };
struct SubBand { int type; IntRect rect; std::vector<size_t> precincts; std::vector<float> coef; };
struct CompBands {
  size_t ll;
  std::vector<std::array<size_t, 3>> decomp;  // per resolution >= 1
  std::vector<IntRect> decomp_rect;
};

struct Storage {
  std::vector<SubBand> bands;
  std::vector<Precinct> precs;
  std::vector<CodeBlock> cbs;
  std::vector<TagNode> nodes;
  std::vector<CompBands> comps;
};

static void build_precincts(const ResTile& rt, size_t band_idx, const Tile& t, Storage& st) {
  std::vector<PrecinctData> pd;
  if (!precincts(rt, pd)) fail(ERR_DECODE, "invalid precinct");
  IntRect sb = st.bands[band_idx].rect;
  uint32_t cw = cb_w(rt), ch = cb_h(rt);
  for (auto& p : pd) {
    uint32_t x0 = (std::max(p.rect.x0, sb.x0) / cw) * cw;
    uint32_t y0 = (std::max(p.rect.y0, sb.y0) / ch) * ch;
    uint32_t x1 = div_ceil(std::min(p.rect.x1, sb.x1), cw) * cw;
    uint32_t y1 = div_ceil(std::min(p.rect.y1, sb.y1), ch) * ch;
    IntRect area = IntRect::ltrb(x0, y0, x1, y1);
    uint32_t ncx = sb.width() == 0 ? 0 : area.width() / cw;
    uint32_t ncy = sb.height() == 0 ? 0 : area.height() / ch;
    Precinct pr;
    for (uint32_t yi = 0; yi < ncy; ++yi)
      for (uint32_t xi = 0; xi < ncx; ++xi) {
        CodeBlock cb;
        cb.xi = xi;
        cb.yi = yi;
        cb.rect = IntRect::ltrb(area.x0 + xi * cw, area.y0 + yi * ch, area.x0 + xi * cw + cw, area.y0 + yi * ch + ch)
                      .intersect(sb);
        cb.layers.resize(t.num_layers);
        cb.has_layer.assign(t.num_layers, false);
        pr.cbs.push_back(st.cbs.size());
        st.cbs.push_back(std::move(cb));
      }
    pr.incl_tree = new_tag_tree(ncx, ncy, st.nodes);
    pr.zbp_tree = new_tag_tree(ncx, ncy, st.nodes);
    st.bands[band_idx].precincts.push_back(st.precs.size());
    st.precs.push_back(std::move(pr));
  }
}

// build_decompositions, build.rs:18-111.
static void build(const Tile& t, Storage& st) {
  for (const CompInfo& c : t.comps) {
    CompBands cb;
    auto add_band = [&](int type, const ResTile& rt) {
      SubBand b;
      b.type = type;
      b.rect = sub_band_rect(rt, type);
      b.coef.assign((size_t)b.rect.width() * b.rect.height(), 0.0f);
      st.bands.push_back(std::move(b));
      size_t idx = st.bands.size() - 1;
      build_precincts(rt, idx, t, st);
      return idx;
    };
    ResTile r0 = res_tile(t, c, 0);
    cb.ll = add_band(LL, r0);
    for (uint8_t r = 1; r < c.cp.nres; ++r) {
      ResTile rt = res_tile(t, c, r);
      std::array<size_t, 3> d;
      d[0] = add_band(HL, rt);
      d[1] = add_band(LH, rt);
      d[2] = add_band(HH, rt);
      cb.decomp.push_back(d);
      cb.decomp_rect.push_back(rt.rect);
    }
    st.comps.push_back(std::move(cb));
  }
}

// ---------------------------------------------------------------------------
// Progression, crates/signinum-j2k-native/src/j2c/progression.rs.
struct Prg { uint8_t layer, res, comp; uint64_t prec; };

static std::vector<Prg> progression(const Tile& t) {
  std::vector<Prg> out;
  uint8_t max_res = 0;
  for (auto& c : t.comps) max_res = std::max(max_res, c.cp.nres);
  uint8_t nl = t.num_layers, nc = (uint8_t)t.comps.size();
  auto comp_max_res = [&](uint8_t c) { return std::min(max_res, t.comps[c].cp.nres); };
  if (t.prog == LRCP) {
    // layer_resolution_component_position_progression, progression.rs:114-170.
    // The resolution bound is taken from component 0 (max_resolution(min_comp)).
    uint8_t rmax = comp_max_res(0);
    for (uint8_t l = 0; l < nl; ++l)
      for (uint8_t r = 0; r < rmax; ++r)
        for (uint8_t c = 0; c < nc; ++c) {
          if (r >= t.comps[c].cp.nres) fail(ERR_DECODE, "resolution missing in a component");
          ResTile rt = res_tile(t, t.comps[c], r);
          uint64_t n = num_precincts(rt);
          for (uint64_t p = 0; p < n; ++p) out.push_back({l, r, c, p});
        }
    return out;
  }
  if (t.prog == RLCP) {
    // resolution_layer_component_position_progression, progression.rs:173-228.
    for (uint8_t r = 0; r < max_res; ++r)
      for (uint8_t l = 0; l < nl; ++l)
        for (uint8_t c = 0; c < nc; ++c) {
          if (r >= comp_max_res(c)) continue;
          ResTile rt = res_tile(t, t.comps[c], r);
          uint64_t n = num_precincts(rt);
          for (uint64_t p = 0; p < n; ++p) out.push_back({l, r, c, p});
        }
    return out;
  }
  // position_progression_common, progression.rs:245-290.
  struct Ps { uint8_t res; uint32_t py, px; uint8_t comp; uint64_t idx; };
  std::vector<Ps> el;
  for (uint8_t c = 0; c < nc; ++c)
    for (uint8_t r = 0; r < t.comps[c].cp.nres && r < max_res; ++r) {
      ResTile rt = res_tile(t, t.comps[c], r);
      std::vector<PrecinctData> pd;
      if (!precincts(rt, pd)) fail(ERR_DECODE, "invalid progression iterator");
      for (auto& p : pd) el.push_back({r, p.r_y, p.r_x, c, p.idx});
    }
  auto key = [&](const Ps& a) {
    if (t.prog == RPCL) return std::make_tuple((uint64_t)a.res, (uint64_t)a.py, (uint64_t)a.px, (uint64_t)a.comp, a.idx);
    if (t.prog == PCRL) return std::make_tuple((uint64_t)a.py, (uint64_t)a.px, (uint64_t)a.comp, (uint64_t)a.res, a.idx);
    return std::make_tuple((uint64_t)a.comp, (uint64_t)a.py, (uint64_t)a.px, (uint64_t)a.res, a.idx);
  };
  std::stable_sort(el.begin(), el.end(), [&](const Ps& a, const Ps& b) { return key(a) < key(b); });
  for (auto& e : el)
    for (uint8_t l = 0; l < nl; ++l) out.push_back({l, e.res, e.comp, e.idx});
  return out;
}

// ---------------------------------------------------------------------------
// Packets, crates/signinum-j2k-native/src/j2c/segment.rs.
static std::vector<size_t> bands_of(const Storage& st, uint8_t comp, uint8_t res) {
  const CompBands& cb = st.comps[comp];
  if (res == 0) return {cb.ll};
  const auto& d = cb.decomp[res - 1];
  return {d[0], d[1], d[2]};
}

// resolve_ht_segments + parse_ht_segment_lengths, segment.rs:304-394, :542-581.
static bool resolve_ht(size_t band, const Prg& pg, BitReader& r, Storage& st) {
  const SubBand& sb = st.bands[band];
  if (pg.prec >= sb.precincts.size()) return false;
  Precinct& pr = st.precs[sb.precincts[pg.prec]];
  for (size_t cbi : pr.cbs) {
    CodeBlock& cb = st.cbs[cbi];
    // resolve_code_block_inclusion, segment.rs:409-479.
    bool first = !cb.included;
    bool inc;
    if (cb.included) {
      uint32_t b;
      if (!r.read_bits_stuffed(1, &b)) return false;
      inc = b == 1;
    } else {
      uint32_t v;
      if (!read_tag(pr.incl_tree, cb.xi, cb.yi, r, 0, (uint32_t)pg.layer + 1, st.nodes, v)) return false;
      inc = v <= pg.layer;
    }
    if (!inc) continue;
    if (first) {
      uint32_t v;
      if (!read_tag(pr.zbp_tree, cb.xi, cb.yi, r, 0, UINT32_MAX, st.nodes, v)) return false;
      cb.missing = (uint8_t)v;
    }
    cb.included = true;
    if (!first || cb.passes != 0 || cb.nonempty != 0) return false;
    if (cb.has_layer[pg.layer]) return false;
    // decode_num_ht_coding_passes, segment.rs:508-530.
    uint32_t np = 1, b;
    if (!r.read_bits_stuffed(1, &b)) return false;
    if (b == 1) {
      np = 2;
      if (!r.read_bits_stuffed(1, &b)) return false;
      if (b == 1) {
        uint32_t e;
        if (!r.read_bits_stuffed(2, &e)) return false;
        np = 3 + e;
        if (e == 3) {
          if (!r.read_bits_stuffed(5, &e)) return false;
          np = 6 + e;
          if (e == 31) {
            if (!r.read_bits_stuffed(7, &e)) return false;
            np = 37 + e;
          }
        }
      }
    }
    if (np > 255 || np > 1 + 3 * 31) return false;
    uint32_t groups = (np > 1 ? np - 1 : 0) / 3;
    uint32_t missing = (uint32_t)cb.missing + groups;
    if (missing > 255) return false;
    uint32_t ph = groups * 3;
    uint32_t actual = np - ph;
    uint32_t inc_l = 0;
    for (;;) {
      if (!r.read_bits_stuffed(1, &b)) return false;
      if (b == 0) break;
      ++inc_l;
    }
    cb.lblock += inc_l;
    uint32_t lg = 31 - (uint32_t)__builtin_clz(ph + 1);
    uint32_t bits = cb.lblock + lg;
    if (bits > 255) return false;
    uint32_t lcup;
    if (!r.read_bits_stuffed(bits, &lcup)) return false;
    if (lcup < 2 || lcup >= 65535) return false;
    uint32_t lref = 0;
    if (actual > 1) {
      uint32_t rb = cb.lblock + (actual > 2 ? 1 : 0);
      if (rb > 255 || !r.read_bits_stuffed(rb, &lref)) return false;
      if (lref >= 2047) return false;
    }
    cb.missing = (uint8_t)missing;
    std::vector<Segment>& segs = cb.layers[pg.layer];
    segs.push_back({0, lcup, nullptr});
    if (actual > 1) segs.push_back({1, lref, nullptr});
    cb.has_layer[pg.layer] = true;
    cb.passes = (uint8_t)actual;
    cb.nonempty = (uint8_t)(cb.nonempty + 1);
  }
  return true;
}

// decode_num_classic_coding_passes (Table B.4), segment.rs:482-506: prefix
// codes are matched by peeking, longest first.
static bool classic_num_passes(BitReader& r, uint32_t& np) {
  auto peek = [&](uint32_t n, uint32_t want) {
    BitReader c = r;
    uint32_t v;
    return c.read_bits_stuffed(n, &v) && v == want;
  };
  uint32_t v;
  if (peek(9, 0x1FF)) {
    r.read_bits_stuffed(9, &v);
    if (!r.read_bits_stuffed(7, &v)) return false;
    np = v + 37;
  } else if (peek(4, 0xF)) {
    r.read_bits_stuffed(4, &v);
    if (!r.read_bits_stuffed(5, &v)) return false;
    np = v + 6;
  } else if (peek(4, 0xE)) {
    r.read_bits_stuffed(4, &v);
    np = 5;
  } else if (peek(4, 0xD)) {
    r.read_bits_stuffed(4, &v);
    np = 4;
  } else if (peek(4, 0xC)) {
    r.read_bits_stuffed(4, &v);
    np = 3;
  } else if (peek(2, 0x2)) {
    r.read_bits_stuffed(2, &v);
    np = 2;
  } else if (peek(1, 0)) {
    r.read_bits_stuffed(1, &v);
    np = 1;
  } else {
    return false;
  }
  return true;
}

// segment_idx_for_bypass, segment.rs:585-591.
static uint32_t bypass_segment(uint32_t p) { return p < 10 ? 0 : 1 + 2 * ((p - 10) / 3) + ((p - 10) % 3 == 2 ? 1 : 0); }

// resolve_classic_segments, segment.rs:168-302.
static bool resolve_classic(size_t band, const Prg& pg, BitReader& r, Storage& st, uint8_t style) {
  const SubBand& sb = st.bands[band];
  if (pg.prec >= sb.precincts.size()) return false;
  Precinct& pr = st.precs[sb.precincts[pg.prec]];
  for (size_t cbi : pr.cbs) {
    CodeBlock& cb = st.cbs[cbi];
    bool first = !cb.included;
    bool inc;
    if (cb.included) {
      uint32_t b;
      if (!r.read_bits_stuffed(1, &b)) return false;
      inc = b == 1;
    } else {
      uint32_t v;
      if (!read_tag(pr.incl_tree, cb.xi, cb.yi, r, 0, (uint32_t)pg.layer + 1, st.nodes, v)) return false;
      inc = v <= pg.layer;
    }
    if (!inc) continue;
    if (first) {
      uint32_t v;
      if (!read_tag(pr.zbp_tree, cb.xi, cb.yi, r, 0, UINT32_MAX, st.nodes, v)) return false;
      cb.missing = (uint8_t)v;
    }
    cb.included = true;
    uint32_t added;
    if (!classic_num_passes(r, added)) return false;
    uint32_t inc_l = 0, b;
    for (;;) {
      if (!r.read_bits_stuffed(1, &b)) return false;
      if (b == 0) break;
      ++inc_l;
    }
    cb.lblock += inc_l;
    const uint32_t prev = cb.passes, cum = prev + added;
    if (cum > 1 + 3 * 31) return false;
    auto seg_idx = [&](uint32_t p) -> uint32_t {
      if (style & 0x04) return p;
      if (style & 0x01) return bypass_segment(p);
      return cb.nonempty;
    };
    std::vector<Segment>& segs = cb.layers[pg.layer];
    auto push = [&](uint32_t idx, uint32_t count) {
      uint32_t bits = cb.lblock + (31 - (uint32_t)__builtin_clz(count)), len;
      if (bits > 32 || !r.read_bits_stuffed(bits, &len)) return false;
      segs.push_back({(uint8_t)idx, len, nullptr, (uint8_t)count});
      return true;
    };
    uint32_t last = seg_idx(prev), count = 0;
    for (uint32_t p = prev; p < cum; ++p) {
      const uint32_t s = seg_idx(p);
      if (s != last) {
        if (!push(last, count)) return false;
        last = s;
        count = 1;
      } else {
        ++count;
      }
    }
    if (count > 0 && !push(last, count)) return false;
    cb.has_layer[pg.layer] = true;
    cb.passes = (uint8_t)cum;
    cb.nonempty = (uint8_t)(cb.nonempty + 1);
  }
  return true;
}

// parse_inner, segment.rs:53-148 (merged tile parts only).
static bool parse_part(BitReader& r, const std::vector<Prg>& prog, size_t& pi, const Tile& t, Storage& st) {
  while (!r.at_end()) {
    if (pi >= prog.size()) return false;
    const Prg pg = prog[pi++];
    const CompInfo& ci = t.comps[pg.comp];
    std::vector<size_t> bands = bands_of(st, pg.comp, pg.res);
    uint8_t m;
    if ((ci.flags & 2) && r.peek_marker(&m) && m == 0x91) {
      r.read_marker(&m);
      if (!r.skip(4)) return false;
    }
    uint32_t b;
    if (!r.read_bits_stuffed(1, &b)) return false;
    bool zero = b == 0;
    if (!zero)
      for (size_t bi : bands)
        if (!(ci.ht() ? resolve_ht(bi, pg, r, st) : resolve_classic(bi, pg, r, st, ci.cp.cbstyle))) return false;
    r.align();
    if (ci.flags & 4) {
      if (!r.read_marker(&m) || m != 0x92) return false;
    }
    if (!zero) {
      for (size_t bi : bands) {
        SubBand& sb = st.bands[bi];
        if (pg.prec >= sb.precincts.size()) return false;
        Precinct& pr = st.precs[sb.precincts[pg.prec]];
        for (size_t cbi : pr.cbs) {
          CodeBlock& cb = st.cbs[cbi];
          if (!cb.has_layer[pg.layer]) continue;
          for (Segment& s : cb.layers[pg.layer]) {
            const uint8_t* p;
            if (!r.read_bytes(s.len, &p)) return false;
            s.data = p;
          }
        }
      }
    }
  }
  return true;
}

// ---------------------------------------------------------------------------
// Inverse 5/3, crates/signinum-j2k-native/src/j2c/idwt.rs.
static inline size_t pse_left(size_t i, size_t off) { return i > off ? i - off : off - i; }
static inline size_t pse_right(size_t i, size_t off, size_t n) {
  size_t ni = i + off;
  if (ni >= n) return n - 2 - (ni - n);
  return ni;
}

// reversible_filter_53r / filter_step_horizontal, idwt.rs:741-765, :836-862.
static void filter_row(float* s, size_t w, size_t x0) {
  if (w == 1) {
    if (x0 % 2) s[0] *= 0.5f;
    return;
  }
  size_t fe = x0 % 2, fo = 1 - fe;
  auto step = [&](size_t first, bool update) {
    auto f = [&](float v, float l, float r) {
      return update ? v - std::floor((l + r) * 0.25f + 0.5f) : v + std::floor((l + r) * 0.5f);
    };
    if (first == 0) s[0] = f(s[0], s[pse_left(0, 1)], s[pse_right(0, 1, w)]);
    size_t ms = first == 0 ? 2 : 1;
    for (size_t i = ms; i + 1 < w; i += 2) s[i] = f(s[i], s[i - 1], s[i + 1]);
    if (w > 1 && (w - 1) % 2 == first) {
      size_t i = w - 1;
      s[i] = f(s[i], s[pse_left(i, 1)], s[pse_right(i, 1, w)]);
    }
  };
  step(fe, true);
  step(fo, false);
}

// filter_vertical_impl / reversible_filter_53r_simd, idwt.rs:927-1014.
static void filter_cols(float* s, size_t w, size_t h, size_t y0) {
  if (h == 1) {
    if (y0 % 2)
      for (size_t c = 0; c < w; ++c) s[c] *= 0.5f;
    return;
  }
  size_t fe = y0 % 2, fo = 1 - fe;
  for (int pass = 0; pass < 2; ++pass) {
    size_t first = pass == 0 ? fe : fo;
    for (size_t row = first; row < h; row += 2) {
      size_t ra = pse_left(row, 1), rb = pse_right(row, 1, h);
      for (size_t c = 0; c < w; ++c) {
        float v = s[row * w + c], a = s[ra * w + c], b = s[rb * w + c];
        s[row * w + c] = pass == 0 ? v - std::floor((a + b) * 0.25f + 0.5f) : v + std::floor((a + b) * 0.5f);
      }
    }
  }
}

// Irreversible 9/7: irreversible_filter_97i / irreversible_filter_97i_simd,
// idwt.rs:767-836, :1016-1140 (Table F.4 constants; math::mul_add is fused on
// an FMA host, as the B200 host is).
static const float kNegAlpha = 1.5861343f, kNegBeta = 0.052980117f, kNegGamma = -0.8829111f,
                   kNegDelta = -0.44350687f, kKappa = 1.2301741f;

static void filter_row97(float* s, size_t w, size_t x0) {
  if (w == 1) {
    if (x0 % 2) s[0] *= 0.5f;
    return;
  }
  size_t fe = x0 % 2, fo = 1 - fe;
  const float inv_k = 1.0f / kKappa;
  const float k0 = fe == 0 ? kKappa : inv_k, k1 = fe == 0 ? inv_k : kKappa;
  for (size_t i = 0; i + 1 < w; i += 2) {
    s[i] *= k0;
    s[i + 1] *= k1;
  }
  if (w % 2 == 1) s[w - 1] *= k0;
  auto step = [&](size_t first, float c) {
    auto f = [&](float v, float l, float r) { return std::fma(l + r, c, v); };
    if (first == 0) s[0] = f(s[0], s[pse_left(0, 1)], s[pse_right(0, 1, w)]);
    size_t ms = first == 0 ? 2 : 1;
    for (size_t i = ms; i + 1 < w; i += 2) s[i] = f(s[i], s[i - 1], s[i + 1]);
    if ((w - 1) % 2 == first) {
      size_t i = w - 1;
      s[i] = f(s[i], s[pse_left(i, 1)], s[pse_right(i, 1, w)]);
    }
  };
  step(fe, kNegDelta);
  step(fo, kNegGamma);
  step(fe, kNegBeta);
  step(fo, kNegAlpha);
}

static void filter_cols97(float* s, size_t w, size_t h, size_t y0) {
  if (h == 1) {
    if (y0 % 2)
      for (size_t c = 0; c < w; ++c) s[c] *= 0.5f;
    return;
  }
  size_t fe = y0 % 2, fo = 1 - fe;
  const float inv_k = 1.0f / kKappa;
  const float k0 = fe == 0 ? kKappa : inv_k, k1 = fe == 0 ? inv_k : kKappa;
  for (size_t row = 0; row + 1 < h; row += 2)
    for (size_t c = 0; c < w; ++c) {
      s[row * w + c] *= k0;
      s[(row + 1) * w + c] *= k1;
    }
  if (h % 2 == 1)
    for (size_t c = 0; c < w; ++c) s[(h - 1) * w + c] *= k0;
  const size_t firsts[4] = {fe, fo, fe, fo};
  const float cs[4] = {kNegDelta, kNegGamma, kNegBeta, kNegAlpha};
  for (int k = 0; k < 4; ++k)
    for (size_t row = firsts[k]; row < h; row += 2) {
      size_t ra = pse_left(row, 1), rb = pse_right(row, 1, h);
      for (size_t c = 0; c < w; ++c)
        s[row * w + c] = std::fma(s[ra * w + c] + s[rb * w + c], cs[k], s[row * w + c]);
    }
}

// filter_2d with interleave_samples, idwt.rs:535-712.
static void idwt_level(const std::vector<float>& ll, const SubBand& hl, const SubBand& lh, const SubBand& hh,
                       const IntRect& rect, std::vector<float>& out, bool reversible) {
  size_t w = rect.width(), h = rect.height();
  out.assign(w * h, 0.0f);
  uint32_t u0 = rect.x0, u1 = rect.x1, v0 = rect.y0, v1 = rect.y1;
  size_t nul = div_ceil(u1, 2) - div_ceil(u0, 2), nuh = u1 / 2 - u0 / 2;
  size_t nvl = div_ceil(v1, 2) - div_ceil(v0, 2), nvh = v1 / 2 - v0 / 2;
  size_t fw = u0 % 2 == 0 ? nul : nuh, sw = u0 % 2 == 0 ? nuh : nul;
  size_t er = v0 % 2 == 0 ? 0 : 1, orr = v0 % 2 == 0 ? 1 : 0;
  auto rows = [&](const float* fb, const float* sb, size_t start, size_t n) {
    for (size_t v = 0; v < n; ++v) {
      size_t orow = start + v * 2;
      if (orow >= h) break;
      const float* f = fb + v * fw;
      const float* s2 = sb + v * sw;
      float* o = out.data() + orow * w;
      size_t np = std::min(fw, sw);
      for (size_t i = 0; i < np; ++i) {
        o[i * 2] = f[i];
        o[i * 2 + 1] = s2[i];
      }
      if (fw > np) o[np * 2] = f[np];
    }
  };
  const float* llp = ll.data();
  if (u0 % 2 == 0) rows(llp, hl.coef.data(), er, nvl);
  else rows(hl.coef.data(), llp, er, nvl);
  if (u0 % 2 == 0) rows(lh.coef.data(), hh.coef.data(), orr, nvh);
  else rows(hh.coef.data(), lh.coef.data(), orr, nvh);
  if (w > 0 && h > 0) {
    if (reversible) {
      for (size_t y = 0; y < h; ++y) filter_row(out.data() + y * w, w, rect.x0);
      filter_cols(out.data(), w, h, rect.y0);
    } else {
      for (size_t y = 0; y < h; ++y) filter_row97(out.data() + y * w, w, rect.x0);
      filter_cols97(out.data(), w, h, rect.y0);
    }
  }
}

// ---------------------------------------------------------------------------
// Decode driver, crates/signinum-j2k-native/src/j2c/decode.rs:42-126, :796-871.
struct Planes {
  uint32_t w = 0, h = 0;
  std::vector<std::vector<float>> data;
  std::vector<uint8_t> depth;
};

static int32_t coefficient_to_i32(uint32_t v, uint8_t kmax) {
  uint32_t shift = kmax >= 31 ? 0 : 31u - kmax;
  int32_t m = (int32_t)((v & 0x7FFFFFFFu) >> shift);
  return (v & 0x80000000u) ? -m : m;
}

// decode_sub_band_bitplanes + decode_sub_band_ht_blocks (non-backend path),
// decode.rs:1117-1171, :1682-1716; ht_block_decode::decode_with_stats :236-300.
static void decode_band(Storage& st, size_t bi, uint8_t res, const CompInfo& ci, const Header& h) {
  SubBand& sb = st.bands[bi];
  auto em = ci.exponent_mantissa(sb.type, res);
  // Dequantisation step (decode.rs:1130-1151): 2^(R_b - exponent) * (1 + mantissa / 2048),
  // R_b = precision + log2 gain of the band (LL 0, HL/LH 1, HH 2); pow2i, math.rs:550-556.
  float step = 1.0f;
  if (ci.q.style != QNONE) {
    int gain = sb.type == LL ? 0 : sb.type == HH ? 2 : 1;
    int e = (int)ci.size.precision + gain - (int)em.first;
    float p2 = e >= 0 ? (float)(1u << e) : 1.0f / (float)(1u << -e);
    step = p2 * (1.0f + (float)em.second / 2048.0f);
  }
  int nb = (int)ci.q.guard + (int)em.first - 1;
  if (nb < 0) fail(ERR_DECODE, "invalid bitplane count");
  if (nb > 32) fail(ERR_DECODE, "too many bitplanes");
  uint8_t num_bitplanes = (uint8_t)nb;
  if (!ci.ht()) {
    // Classic code blocks (decode_sub_band_bitplanes, decode.rs:1290-1345):
    // the layers' segments are combined as in decode_inner (bitplane.rs:90-128).
    std::vector<int32_t> blk;
    for (size_t pi : sb.precincts)
      for (size_t cbi : st.precs[pi].cbs) {
        CodeBlock& cb = st.cbs[cbi];
        uint32_t w = cb.rect.width(), hh = cb.rect.height();
        std::vector<uint8_t> data;
        std::vector<size_t> seg_start{0};
        std::vector<uint32_t> seg_pass{0};
        uint32_t last = 0, passes = 0;
        for (size_t l = 0; l < cb.layers.size(); ++l) {
          if (!cb.has_layer[l]) continue;
          for (const Segment& s : cb.layers[l]) {
            if (s.idx != last) {
              seg_start.push_back(data.size());
              seg_pass.push_back(passes);
              last = s.idx;
            }
            if (s.len) data.insert(data.end(), s.data, s.data + s.len);
            passes += s.passes;
          }
        }
        seg_start.push_back(data.size());
        seg_pass.push_back(passes);
        blk.assign((size_t)w * hh, 0);
        classic_block_decode(data.data(), seg_start, seg_pass, w, hh, cb.missing, cb.passes, num_bitplanes, sb.type,
                             ci.cp.cbstyle, blk.data(), w);
        uint32_t xo = cb.rect.x0 - sb.rect.x0, yo = cb.rect.y0 - sb.rect.y0;
        for (uint32_t y = 0; y < hh; ++y)
          for (uint32_t x = 0; x < w; ++x)
            sb.coef[(size_t)(yo + y) * sb.rect.width() + xo + x] = (float)blk[(size_t)y * w + x] * step;
      }
    return;
  }
  std::vector<uint32_t> buf;
  for (size_t pi : sb.precincts) {
    for (size_t cbi : st.precs[pi].cbs) {
      CodeBlock& cb = st.cbs[cbi];
      uint32_t w = cb.rect.width(), hh = cb.rect.height();
      buf.assign((size_t)w * hh, 0);
      if (num_bitplanes != 0) {
        if (num_bitplanes > 31) fail(ERR_DECODE, "too many bitplanes");
        uint32_t actual = num_bitplanes > cb.missing ? num_bitplanes - cb.missing : 0;
        if (cb.passes != 0 && actual != 0) {
          const uint8_t *cu = nullptr, *rf = nullptr;
          uint32_t lc = 0, lr = 0;
          bool have_c = false, have_r = false;
          for (size_t l = 0; l < cb.layers.size(); ++l) {
            if (!cb.has_layer[l]) continue;
            for (const Segment& s : cb.layers[l]) {
              if (s.idx == 0 && !have_c) { cu = s.data; lc = s.data ? s.len : 0; have_c = true; }
              else if (s.idx == 1 && !have_r) { rf = s.data; lr = s.data ? s.len : 0; have_r = true; }
              else fail(ERR_UNSUPPORTED, "unexpected HTJ2K segment layout");
            }
          }
          if (!have_c) fail(ERR_DECODE, "code-block decode failure");
          static const uint8_t empty = 0;
          if (!ht_block_decode(cu ? cu : &empty, lc, rf ? rf : &empty, lr, cb.missing, cb.passes, w, hh, w,
                               ci.causal(), buf.data()))
            fail(ERR_DECODE, "code-block decode failure");
        }
      }
      uint32_t xo = cb.rect.x0 - sb.rect.x0, yo = cb.rect.y0 - sb.rect.y0;
      for (uint32_t y = 0; y < hh; ++y)
        for (uint32_t x = 0; x < w; ++x)
          sb.coef[(size_t)(yo + y) * sb.rect.width() + xo + x] =
              (float)coefficient_to_i32(buf[(size_t)y * w + x], num_bitplanes) * step;
    }
  }
}

static void decode_codestream(const uint8_t* data, size_t len, const uint32_t* target, Planes& planes,
                              Header* hdr_out = nullptr, Storage* st_out = nullptr, uint32_t st_comp = 0) {
  BitReader r(data, len);
  uint8_t m;
  if (len < 4 || data[0] != 0xFF || data[1] != 0x4F || data[2] != 0xFF || data[3] != 0x51)
    fail(ERR_DECODE, "invalid signature");
  r.read_marker(&m);
  Header h = read_header(r, target);
  if (hdr_out) *hdr_out = h;
  for (auto& c : h.comps) {
    if (c.size.xr != 1 || c.size.yr != 1) fail(ERR_UNSUPPORTED, "sub-sampled components are outside the oracle's scope");
  }
  BitReader body(data + r.byte_pos(), len - r.byte_pos());
  std::vector<Tile> tiles = parse_tiles(body, h);
  if (tiles.empty()) fail(ERR_DECODE, "invalid tile");
  planes.w = h.siz.image_width();
  planes.h = h.siz.image_height();
  planes.data.assign(tiles[0].comps.size(), std::vector<float>((size_t)planes.w * planes.h, 0.0f));
  planes.depth.clear();
  for (auto& c : tiles[0].comps) planes.depth.push_back(c.size.precision);
  for (const Tile& t : tiles) {
    Storage st;
    build(t, st);
    // segment::parse, segment.rs:17-51.
    bool ht = false;
    for (auto& c : t.comps) ht = ht || c.ht();
    if (t.num_layers > 1 && ht) fail(ERR_UNSUPPORTED, "multi-layer HTJ2K packet assembly");
    std::vector<Prg> prog = progression(t);
    size_t pi = 0;
    for (const BitReader& part : t.parts) {
      BitReader pr = part;
      if (!parse_part(pr, prog, pi, t, st) && h.strict) fail(ERR_DECODE, "invalid tile");
    }
    for (size_t ci = 0; ci < t.comps.size(); ++ci) {
      const CompInfo& c = t.comps[ci];
      for (uint8_t res = 0; res < c.cp.nres - h.skipped; ++res)
        for (size_t bi : bands_of(st, (uint8_t)ci, res)) decode_band(st, bi, res, c, h);
    }
    if (st_out && t.idx == 0) {
      (void)st_comp;
      *st_out = std::move(st);
      return;
    }
    for (size_t ci = 0; ci < h.comps.size(); ++ci) {
      const CompInfo& c = t.comps[ci];
      const CompBands& cb = st.comps[ci];
      size_t nd = cb.decomp.size() - std::min<size_t>(cb.decomp.size(), h.skipped);
      std::vector<float> cur = st.bands[cb.ll].coef, nxt;
      IntRect rect = st.bands[cb.ll].rect;
      for (size_t d = 0; d < nd; ++d) {
        const auto& ids = cb.decomp[d];
        idwt_level(cur, st.bands[ids[0]], st.bands[ids[1]], st.bands[ids[2]], cb.decomp_rect[d], nxt, c.cp.reversible);
        std::swap(cur, nxt);
        rect = cb.decomp_rect[d];
      }
      // store, decode.rs:1731-1820 (scale 1, no output region).
      ResTile rt = res_tile(t, c, (uint8_t)(c.cp.nres - 1 - h.skipped));
      float shift = t.mct ? 0.0f : (float)(1u << (c.size.precision - 1));
      uint32_t sx = h.siz.ox > rect.x0 ? h.siz.ox - rect.x0 : 0;
      uint32_t sy = h.siz.oy > rect.y0 ? h.siz.oy - rect.y0 : 0;
      if (shift != 0.0f)
        for (float& v : cur) v += shift;
      uint32_t ox = rt.rect.x0 > h.siz.ox ? rt.rect.x0 - h.siz.ox : 0;
      uint32_t oy = rt.rect.y0 > h.siz.oy ? rt.rect.y0 - h.siz.oy : 0;
      uint32_t rw = rect.width();
      for (uint32_t y = sy; y < rect.height(); ++y) {
        uint32_t orow = oy + (y - sy);
        if (orow >= planes.h) break;
        uint32_t n = rw - sx;
        if (ox + n > planes.w) fail(ERR_DECODE, "store out of range");
        std::memcpy(&planes.data[ci][(size_t)orow * planes.w + ox], &cur[(size_t)y * rw + sx], n * sizeof(float));
      }
    }
  }
  if (tiles[0].mct) {
    // mct::apply_inverse (reversible branch) + apply_sign_shift, mct.rs:11-64, :117-150; decode.rs:1720-1729.
    if (planes.data.size() >= 3) {
      auto& c = tiles[0].comps;
      if (c[0].cp.reversible != c[1].cp.reversible || c[1].cp.reversible != c[2].cp.reversible)
        fail(ERR_DECODE, "mct");
      float *y0 = planes.data[0].data(), *y1 = planes.data[1].data(), *y2 = planes.data[2].data();
      if (c[0].cp.reversible) {
        for (size_t i = 0; i < planes.data[0].size(); ++i) {
          float a = y0[i], b = y1[i], cc = y2[i];
          float i1 = a - std::floor((cc + b) * 0.25f);
          y0[i] = cc + i1;
          y1[i] = i1;
          y2[i] = b + i1;
        }
      } else {
        // Irreversible ICT (mct.rs:80-115), fused multiply-adds as on the SIMD path.
        for (size_t i = 0; i < planes.data[0].size(); ++i) {
          float a = y0[i], b = y1[i], cc = y2[i];
          y0[i] = std::fma(cc, 1.402f, a);
          y1[i] = std::fma(cc, -0.71414f, std::fma(b, -0.34413f, a));
          y2[i] = std::fma(b, 1.772f, a);
        }
      }
    }
    for (size_t ci = 0; ci < planes.data.size(); ++ci) {
      float add = (float)(1u << (planes.depth[ci] - 1));
      for (float& v : planes.data[ci]) v += add;
    }
  }
}

// ---------------------------------------------------------------------------
// Pixel conversion, crates/signinum-j2k-native/src/lib.rs:1772-1840, :2202-2294;
// crates/signinum-j2k/src/decode.rs:235-356, :430-545.
static inline float rnd(float v) { return std::round(v); }
static inline uint8_t sat_u8(float v) {
  if (!(v > 0.0f)) return 0;  // `as u8` saturates (NaN -> 0)
  if (v >= 255.0f) return 255;
  return (uint8_t)v;
}

// interleave_and_convert: the full-image u8 path.
static uint8_t full_u8(float v, uint8_t depth, bool all8) {
  if (all8) return sat_u8(rnd(v));
  float mul = 255.0f;
  return sat_u8(rnd((v / (float)((1u << depth) - 1)) * mul));
}

// sample_as_u8: the region u8 path.
static uint8_t region_u8(float v, uint8_t depth) {
  float r = rnd(v);
  if (depth == 8) return (uint8_t)std::min(std::max(r, 0.0f), 255.0f);
  float maxv = depth >= 16 ? 65535.0f : (float)std::max<uint32_t>((1u << depth) - 1, 1);
  float c = std::min(std::max(r, 0.0f), maxv);
  return sat_u8(rnd((c / maxv) * 255.0f));
}

// decode_native: clamp to [0, 2^bd-1] at native depth, then u16 widening
// (convert_or_copy_u16) for depths <= 8.
static uint16_t native_u16(float v, uint8_t depth) {
  float maxv = (float)((1u << depth) - 1);
  float r = rnd(v);
  float c = r < 0.0f ? 0.0f : (r > maxv ? maxv : r);
  if (depth <= 8) {
    uint32_t s = (uint32_t)(uint8_t)c;
    uint32_t mx = std::max<uint32_t>((1u << std::min<uint32_t>(depth, 16)) - 1, 1);
    return (uint16_t)((s * 65535u + mx / 2) / mx);
  }
  return (uint16_t)c;
}

static void convert(const Planes& p, int fmt, bool region, uint32_t rx, uint32_t ry, uint32_t rw, uint32_t rh,
                    std::vector<uint8_t>& out) {
  size_t nc = p.data.size();
  bool rgb = nc >= 3;
  if (nc != 1 && nc != 3) fail(ERR_UNSUPPORTED, "only gray and RGB codestreams are in the oracle's scope");
  bool all8 = true;
  for (auto d : p.depth) all8 = all8 && d == 8;
  int bpp = bytes_per_pixel(fmt);
  out.assign((size_t)rw * rh * bpp, 0);
  bool ok_map = (fmt == FMT_GRAY8 && !rgb) || (fmt == FMT_RGB8 && rgb) || (fmt == FMT_RGBA8 && rgb) ||
                (fmt == FMT_GRAY16 && !rgb) || (fmt == FMT_RGB16 && rgb);
  if (!ok_map) fail(ERR_UNSUPPORTED, "backend color space cannot be mapped to requested pixel format");
  for (uint32_t y = 0; y < rh; ++y)
    for (uint32_t x = 0; x < rw; ++x) {
      size_t si = (size_t)(ry + y) * p.w + rx + x;
      uint8_t* o = out.data() + ((size_t)y * rw + x) * bpp;
      if (fmt == FMT_GRAY16 || fmt == FMT_RGB16) {
        for (size_t c = 0; c < nc; ++c) {
          uint16_t v = native_u16(p.data[c][si], p.depth[0]);
          o[2 * c] = (uint8_t)(v & 0xFF);
          o[2 * c + 1] = (uint8_t)(v >> 8);
        }
      } else {
        for (size_t c = 0; c < nc; ++c)
          o[c] = region ? region_u8(p.data[c][si], p.depth[c]) : full_u8(p.data[c][si], p.depth[c], all8);
        if (fmt == FMT_RGBA8) o[3] = 255;
      }
    }
}

// JP2 container: parse_image_info / parse_jp2 / parse_jp2h / parse_colr /
// read_box_header (crates/signinum-j2k/src/parse/mod.rs:17-31,
// parse/boxes.rs:10-245).  Returns the codestream range; raw codestreams
// are passed through.
struct Jp2 {
  size_t off = 0, len = 0;
  bool jp2 = false;
  int colr = -1;         // enumerated colour space; -2 ICC / other method
  bool channels = false; // pclr / cmap / cdef in jp2h
};

static uint32_t rd_be32(const uint8_t* p) {
  return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | (uint32_t)p[3];
}

static void read_box(const uint8_t* d, size_t n, size_t at, char type[5], size_t& body, size_t& end) {
  if (at + 8 > n) fail(ERR_TRUNCATED, "box header truncated");
  uint32_t l = rd_be32(d + at);
  std::memcpy(type, d + at + 4, 4);
  type[4] = 0;
  body = at + 8;
  if (l == 0) {
    end = n;
  } else if (l == 1) {
    if (at + 16 > n) fail(ERR_TRUNCATED, "extended box header truncated");
    uint64_t x = ((uint64_t)rd_be32(d + at + 8) << 32) | rd_be32(d + at + 12);
    if (x < 16) fail(ERR_DECODE, "extended box length smaller than header");
    body = at + 16;
    end = at + (size_t)x;
  } else if (l < 8) {
    fail(ERR_DECODE, "box length smaller than header");
  } else {
    end = at + l;
  }
}

static Jp2 container(const uint8_t* d, size_t n) {
  static const uint8_t sig[12] = {0, 0, 0, 12, 'j', 'P', ' ', ' ', 0x0D, 0x0A, 0x87, 0x0A};
  Jp2 j;
  if (n >= 8 && std::memcmp(d, sig, 8) == 0) {
    if (n < 12) fail(ERR_TRUNCATED, "too short for the JP2 signature");
    bool have_sig = false, have_ftyp = false, have_jp2h = false, have_ihdr = false, have_jp2c = false;
    size_t at = 0;
    while (at < n) {
      char t[5];
      size_t body, end;
      read_box(d, n, at, t, body, end);
      if (end > n) fail(ERR_TRUNCATED, "box payload truncated");
      const std::string type(t);
      if (type == "jP  ") {
        if (have_sig || at != 0) fail(ERR_DECODE, "signature box must appear exactly once at the start");
        if (end - body != 4 || std::memcmp(d + body, sig + 8, 4) != 0) fail(ERR_DECODE, "invalid JP2 signature");
        have_sig = true;
      } else if (type == "ftyp") {
        if (!have_sig || have_ftyp || have_jp2h || have_jp2c) fail(ERR_DECODE, "misplaced ftyp");
        if (end - body < 8) fail(ERR_DECODE, "ftyp payload shorter than 8 bytes");
        have_ftyp = true;
      } else if (type == "jp2h") {
        if (!have_ftyp || have_jp2h || have_jp2c) fail(ERR_DECODE, "misplaced jp2h");
        const uint8_t* h = d + body;
        const size_t hn = end - body;
        size_t ia = 0;
        while (ia < hn) {
          char it[5];
          size_t ib, ie;
          read_box(h, hn, ia, it, ib, ie);
          if (ie > hn) ie = hn;
          const std::string itype(it);
          const size_t len = ie > ib ? ie - ib : 0;
          if (itype == "ihdr") {
            if (len < 14) fail(ERR_DECODE, "ihdr payload shorter than 14 bytes");
            have_ihdr = true;
          } else if (itype == "colr" && len >= 3) {
            if (h[ib] == 1 && len >= 7) j.colr = (int)rd_be32(h + ib + 3);
            else if (h[ib] == 2) j.colr = -2;
          } else if (itype == "pclr" || itype == "cmap" || itype == "cdef") {
            j.channels = true;
          }
          ia = ie;
        }
        have_jp2h = true;
      } else if (type == "jp2c") {
        if (!have_jp2h || have_jp2c) fail(ERR_DECODE, "misplaced jp2c");
        j.off = body;
        j.len = end - body;
        have_jp2c = true;
      }
      at = end;
    }
    if (!have_ftyp || !have_jp2h || !have_ihdr || !have_jp2c) fail(ERR_DECODE, "missing required JP2 box");
    j.jp2 = true;
    return j;
  }
  if (n >= 4 && d[0] == 0xFF && d[1] == 0x4F && d[2] == 0xFF && d[3] == 0x51) {
    j.len = n;
    return j;
  }
  fail(ERR_UNSUPPORTED, "input is not a JP2 container or raw JPEG 2000 codestream");
  return j;
}

static Info inspect_raw(const uint8_t* data, size_t len);

Info inspect(const uint8_t* data, size_t len) {
  const Jp2 j = container(data, len);
  return inspect_raw(data + j.off, j.len);
}

static Info inspect_raw(const uint8_t* data, size_t len) {
  BitReader r(data, len);
  uint8_t m;
  if (len < 4 || data[0] != 0xFF || data[1] != 0x4F || data[2] != 0xFF || data[3] != 0x51)
    fail(ERR_DECODE, "invalid signature");
  r.read_marker(&m);
  Header h = read_header(r, nullptr);
  Info i;
  i.width = h.siz.image_width();
  i.height = h.siz.image_height();
  i.components = (uint32_t)h.comps.size();
  i.bit_depth = h.comps[0].size.precision;
  i.levels = h.comps[0].cp.ndecomp;
  i.tiles = h.siz.ntiles();
  i.ht = 1;
  for (auto& c : h.comps) i.ht = i.ht && c.ht();
  i.reversible = h.comps[0].cp.reversible;
  i.mct = h.mct;
  return i;
}

void decode(const uint8_t* data, size_t len, int fmt, const Request& req, std::vector<uint8_t>& out,
            uint32_t& out_w, uint32_t& out_h) {
  if (fmt == FMT_RGBA16) fail(ERR_UNSUPPORTED, "Rgba16 output is not supported");
  if (fmt < 0 || fmt > FMT_RGBA16) fail(ERR_UNSUPPORTED, "unknown pixel format");
  const Jp2 j = container(data, len);
  data += j.off;
  len = j.len;
  Info info = inspect_raw(data, len);
  uint32_t W = info.width, H = info.height;
  // DeviceDecodePlan::for_image, crates/signinum-j2k/src/adapter/device_plan.rs:23-51.
  uint32_t sx = 0, sy = 0, sw = W, sh = H, d = 1;
  if (req.kind == REQ_REGION || req.kind == REQ_REGION_SCALED) {
    sx = req.x; sy = req.y; sw = req.w; sh = req.h;
  }
  if (req.kind == REQ_SCALED || req.kind == REQ_REGION_SCALED) d = req.denom;
  if (d != 1 && d != 2 && d != 4 && d != 8) fail(ERR_UNSUPPORTED, "unknown downscale");
  if ((uint64_t)sx + sw > W || (uint64_t)sy + sh > H) fail(ERR_REGION, "region outside the image");
  // Rect::scaled_covering, crates/signinum-core/src/types.rs:69-83.
  uint32_t ox0 = sx / d, oy0 = sy / d, ox1 = div_ceil(sx + sw, d), oy1 = div_ceil(sy + sh, d);
  out_w = ox1 - ox0;
  out_h = oy1 - oy0;
  // write_components_u8_output / write_u16_output (crates/signinum-j2k/src/
  // decode.rs:235-273, :430-470): the decoded colour space must map onto the
  // format; from a JP2 colr box only sRGB (3 components) and greyscale (1)
  // map here.
  if (j.jp2 && (j.channels || (j.colr != -1 && !((j.colr == 16 && info.components == 3) ||
                                                  (j.colr == 17 && info.components == 1)))))
    fail(ERR_UNSUPPORTED, "backend color space cannot be mapped to the requested pixel format");
  Planes p;
  if (d == 1) {
    decode_codestream(data, len, nullptr, p);
    bool region = req.kind != REQ_FULL;
    convert(p, fmt, region, sx, sy, sw, sh, out);
    return;
  }
  // decode_scaled_from_info / decode_region_scaled_from_info, crates/signinum-j2k/src/decode.rs:12-71.
  uint32_t target[2] = {div_ceil(W, d), div_ceil(H, d)};
  decode_codestream(data, len, target, p);
  if (req.kind == REQ_SCALED) {
    if (p.w != out_w || p.h != out_h) fail(ERR_BUFFER, "output buffer does not match reduced image");
    convert(p, fmt, false, 0, 0, p.w, p.h, out);
    return;
  }
  if (ox1 > p.w || oy1 > p.h) fail(ERR_REGION, "scaled region outside the reduced image");
  convert(p, fmt, true, ox0, oy0, out_w, out_h, out);
}

void subband_coefficients(const uint8_t* data, size_t len, uint32_t comp, std::vector<int32_t>& out) {
  Planes p;
  Header h;
  Storage st;
  decode_codestream(data, len, nullptr, p, &h, &st, comp);
  out.clear();
  if (comp >= st.comps.size()) fail(ERR_DECODE, "component out of range");
  const CompBands& cb = st.comps[comp];
  auto add = [&](size_t bi) {
    for (float v : st.bands[bi].coef) out.push_back((int32_t)v);
  };
  add(cb.ll);
  for (auto& d : cb.decomp)
    for (size_t bi : d) add(bi);
}

}  // namespace oracle
