// Host-side codestream parsing for the CUDA decode path (see codestream.h).
#include "codestream.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <tuple>

namespace sgn {
namespace {

[[noreturn]] void fail(int32_t s, const char* m) { throw ParseError{s, m}; }

inline uint32_t cdiv(uint64_t a, uint64_t b) { return (uint32_t)((a + b - 1) / b); }

// Byte/bit reader with the packet-header bit-stuffing rule (B.10.1: after a
// 0xFF byte the next byte carries an extra zero bit in its MSB).
struct Reader {
  const uint8_t* d;
  size_t n, bit = 0;  // bit position
  Reader(const uint8_t* p, size_t len) : d(p), n(len) {}
  size_t pos() const { return bit >> 3; }
  bool end() const { return pos() >= n; }
  bool u8(uint8_t& v) {
    if (pos() + 1 > n) return false;
    v = d[pos()];
    bit += 8;
    return true;
  }
  bool u16(uint16_t& v) {
    if (pos() + 2 > n) return false;
    v = (uint16_t)((d[pos()] << 8) | d[pos() + 1]);
    bit += 16;
    return true;
  }
  bool u32(uint32_t& v) {
    if (pos() + 4 > n) return false;
    const uint8_t* p = d + pos();
    v = ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3];
    bit += 32;
    return true;
  }
  bool skip(size_t k) {
    if (pos() + k < pos() || pos() + k > n) return false;
    bit += k * 8;
    return true;
  }
  bool marker(uint8_t& m) {
    if (pos() + 2 > n || d[pos()] != 0xFF) return false;
    m = d[pos() + 1];
    bit += 16;
    return true;
  }
  bool peek_marker(uint8_t& m) const {
    if (pos() + 2 > n || d[pos()] != 0xFF) return false;
    m = d[pos() + 1];
    return true;
  }
  void align() { bit = (bit + 7) & ~(size_t)7; }
  // read_bits_with_stuffing (reader.rs:129-160): cnt bits, most significant
  // first; after the last bit of an 0xFF byte the next byte's top bit is a
  // stuffed zero (a one there is an error) and is skipped.  Takes the bits
  // of one byte per step.
  bool bits(uint32_t cnt, uint32_t& out) {
    uint32_t v = 0;
    while (cnt) {
      const size_t p = bit >> 3;
      if (p >= n) return false;
      const uint32_t avail = 8 - (uint32_t)(bit & 7), take = cnt < avail ? cnt : avail;
      const uint32_t byte = d[p];
      v = (v << take) | ((byte >> (avail - take)) & ((1u << take) - 1));
      bit += take;
      cnt -= take;
      if (take == avail && byte == 0xFF) {
        if ((bit >> 3) >= n) return false;
        if ((d[bit >> 3] >> 7) & 1) return false;
        ++bit;
      }
    }
    out = v;
    return true;
  }
};

struct CodingStyle {
  uint8_t flags = 0, ndecomp = 0, cbw = 0, cbh = 0, cbstyle = 0, transform = 1;
  uint8_t pexp_x[33], pexp_y[33];
};

struct Quant {
  uint8_t style = 0, guard = 0;
  std::vector<uint16_t> exps;   // exponent per band entry
  std::vector<uint16_t> mants;  // mantissa per band entry (0 without quantisation)
};

struct Comp {
  uint8_t precision, xr, yr;
  CodingStyle cs;
  Quant q;
};

bool read_coding_style(Reader& r, uint8_t flags, CodingStyle& cs) {
  uint8_t cw, ch;
  if (!r.u8(cs.ndecomp) || cs.ndecomp > 32) return false;
  if (!r.u8(cw) || !r.u8(ch) || !r.u8(cs.cbstyle) || !r.u8(cs.transform)) return false;
  if (cw > 8 || ch > 8 || cw + ch > 8 || cs.transform > 1) return false;
  cs.cbw = (uint8_t)(cw + 2);
  cs.cbh = (uint8_t)(ch + 2);
  cs.flags = flags;
  for (int i = 0; i <= cs.ndecomp; ++i) {
    if (flags & 1) {
      uint8_t v;
      if (!r.u8(v)) return false;
      cs.pexp_x[i] = v & 0xF;
      cs.pexp_y[i] = v >> 4;
    } else {
      cs.pexp_x[i] = 15;
      cs.pexp_y[i] = 15;
    }
  }
  return true;
}

bool read_quant(Reader& r, size_t body, Quant& q) {
  uint8_t s;
  if (body < 1 || !r.u8(s)) return false;
  q.style = s & 0x1F;
  q.guard = s >> 5;
  q.exps.clear();
  q.mants.clear();
  if (q.style == 0) {
    for (size_t i = 0; i + 1 < body; ++i) {
      uint8_t v;
      if (!r.u8(v)) return false;
      q.exps.push_back((uint16_t)(v >> 3));
      q.mants.push_back(0);
    }
  } else if (q.style == 1 || q.style == 2) {
    for (size_t i = 0; i + 2 < body + 1; i += 2) {
      uint16_t v;
      if (!r.u16(v)) return false;
      q.exps.push_back((uint16_t)(v >> 11));
      q.mants.push_back((uint16_t)(v & 0x7FF));
    }
  } else {
    return false;
  }
  return true;
}

struct MainHeader {
  uint32_t gw, gh, ox, oy, tw, th, tox, toy;
  std::vector<Comp> comps;
  uint8_t prog = 0;
  uint16_t layers = 1;
  bool mct = false;
  size_t end;  // offset of the first SOT
};

// Main header: codestream.rs:38-187.
MainHeader read_main_header(const uint8_t* data, size_t len) {
  if (len < 4 || data[0] != 0xFF || data[1] != 0x4F || data[2] != 0xFF || data[3] != 0x51)
    fail(ST_DECODE, "invalid codestream signature");
  Reader r(data, len);
  r.skip(4);
  MainHeader h;
  uint16_t lsiz, rsiz, csiz;
  if (!r.u16(lsiz) || !r.u16(rsiz) || !r.u32(h.gw) || !r.u32(h.gh) || !r.u32(h.ox) || !r.u32(h.oy) ||
      !r.u32(h.tw) || !r.u32(h.th) || !r.u32(h.tox) || !r.u32(h.toy) || !r.u16(csiz))
    fail(ST_TRUNCATED, "SIZ truncated");
  if (h.ox >= h.gw || h.oy >= h.gh || csiz == 0 || h.tw == 0 || h.th == 0) fail(ST_DECODE, "invalid SIZ");
  if (h.tox >= h.gw || h.toy >= h.gh || h.tox > h.ox || h.toy > h.oy) fail(ST_DECODE, "invalid tile offsets");
  if ((uint64_t)h.tox + h.tw <= h.ox || (uint64_t)h.toy + h.th <= h.oy) fail(ST_DECODE, "invalid tile offsets");
  for (uint16_t i = 0; i < csiz; ++i) {
    uint8_t ss, xr, yr;
    if (!r.u8(ss) || !r.u8(xr) || !r.u8(yr)) fail(ST_TRUNCATED, "SIZ truncated");
    Comp c;
    c.precision = (uint8_t)((ss & 0x7F) + 1);
    c.xr = xr;
    c.yr = yr;
    if (c.precision > 32 || xr == 0 || yr == 0) fail(ST_DECODE, "invalid component metadata");
    h.comps.push_back(c);
  }
  bool have_cod = false, have_qcd = false;
  CodingStyle cod;
  Quant qcd;
  std::vector<int> coc_set(csiz, 0), qcc_set(csiz, 0);
  std::vector<CodingStyle> coc(csiz);
  std::vector<Quant> qcc(csiz);
  for (;;) {
    uint8_t m;
    if (!r.peek_marker(m)) fail(ST_DECODE, "invalid marker in main header");
    if (m == 0x90) break;
    r.marker(m);
    uint16_t L;
    if (m >= 0x30 && m <= 0x3F) continue;
    if (!r.u16(L) || L < 2) fail(ST_TRUNCATED, "marker segment truncated");
    size_t seg_end = r.pos() + L - 2;
    if (seg_end > len) fail(ST_TRUNCATED, "marker segment truncated");
    switch (m) {
      case 0x52: {  // COD
        uint8_t flags, prog, mct;
        uint16_t layers;
        if (!r.u8(flags) || !r.u8(prog) || !r.u16(layers) || !r.u8(mct) || !read_coding_style(r, flags, cod))
          fail(ST_DECODE, "COD parse failure");
        if (prog > 4 || layers == 0 || layers > 32) fail(ST_DECODE, "COD parse failure");
        h.prog = prog;
        h.layers = layers;
        h.mct = mct == 1;
        have_cod = true;
        break;
      }
      case 0x53: {  // COC
        uint16_t idx;
        uint8_t b, flags;
        if (csiz < 257) {
          if (!r.u8(b)) fail(ST_DECODE, "COC parse failure");
          idx = b;
        } else if (!r.u16(idx)) fail(ST_DECODE, "COC parse failure");
        if (idx >= csiz || !r.u8(flags) || !read_coding_style(r, flags, coc[idx])) fail(ST_DECODE, "COC parse failure");
        coc_set[idx] = 1;
        break;
      }
      case 0x5C:  // QCD
        if (!read_quant(r, L - 2, qcd)) fail(ST_DECODE, "QCD parse failure");
        have_qcd = true;
        break;
      case 0x5D: {  // QCC
        uint16_t idx;
        uint8_t b;
        size_t isz = csiz < 257 ? 1 : 2;
        if (csiz < 257) {
          if (!r.u8(b)) fail(ST_DECODE, "QCC parse failure");
          idx = b;
        } else if (!r.u16(idx)) fail(ST_DECODE, "QCC parse failure");
        if (idx >= csiz || L < 2 + isz + 1 || !read_quant(r, L - 2 - isz, qcc[idx])) fail(ST_DECODE, "QCC parse failure");
        qcc_set[idx] = 1;
        break;
      }
      case 0x60:
        fail(ST_UNSUPPORTED, "PPM packed packet headers are not supported by the CUDA path");
      case 0x50: case 0x59: case 0x5E: case 0x55: case 0x64: case 0x63:  // CAP CPF RGN TLM COM CRG
        break;
      default:
        fail(ST_UNSUPPORTED, "unsupported marker in main header");
    }
    r.bit = seg_end * 8;
  }
  if (!have_cod) fail(ST_DECODE, "missing COD");
  if (!have_qcd) fail(ST_DECODE, "missing QCD");
  for (uint16_t i = 0; i < csiz; ++i) {
    Comp& c = h.comps[i];
    c.cs = coc_set[i] ? coc[i] : cod;
    if (coc_set[i]) c.cs.flags |= cod.flags;
    c.q = qcc_set[i] ? qcc[i] : qcd;
  }
  h.end = r.pos();
  return h;
}

// Node values of every tag tree of a tile, in one pool (a node's known flag
// in bit 31 of its value), so that a precinct band's trees cost no
// allocation of their own.
struct TagPool {
  std::vector<uint32_t> nodes;
};

struct TagTree {
  uint32_t levels = 0;
  uint32_t lw[17];
  size_t base[17];  // first node of each level in the pool
  void init(uint32_t w, uint32_t h, TagPool& pool) {
    levels = 0;
    size_t total = pool.nodes.size();
    for (;;) {
      lw[levels] = w;
      base[levels] = total;
      total += (size_t)w * h;
      ++levels;
      if (w <= 1 && h <= 1) break;
      w = (w + 1) / 2;
      h = (h + 1) / 2;
    }
    pool.nodes.resize(total, 0);
  }
  // read_tag_node, tag_tree.rs:118-190, unrolled over levels.
  bool read(uint32_t x, uint32_t y, uint32_t threshold, Reader& r, uint32_t& out, TagPool& pool) {
    constexpr uint32_t kKnown = 1u << 31;
    uint32_t parent = 0;
    for (uint32_t l = levels; l-- > 0;) {
      uint32_t& node = pool.nodes[base[l] + (size_t)(y >> l) * lw[l] + (x >> l)];
      if (!(node & kKnown)) {
        uint32_t v = std::max(parent, node);
        bool known = false;
        while (v < threshold) {
          uint32_t b;
          if (!r.bits(1, b)) return false;
          if (b == 0) ++v;
          else {
            known = true;
            break;
          }
        }
        node = v | (known ? kKnown : 0u);
      }
      const uint32_t val = node & ~kKnown;
      if (val >= threshold || l == 0) {
        out = val;
        return true;
      }
      parent = val;
    }
    out = parent;
    return true;
  }
};

struct PrecinctBand {  // one (precinct, sub-band) pair
  uint32_t band;
  uint32_t cb_x0, cb_y0, ncx, ncy, cbw, cbh;
  uint32_t first_block;  // index into the flat block-state array
  TagTree incl, zbp;
};

struct BlockState {
  uint32_t band, x0, y0, w, h;
  bool included = false;
  uint8_t missing = 0, passes = 0;
  uint32_t lblock = 3;
  uint32_t lcup = 0, lref = 0;
  int64_t cleanup_off = -1, ref_off = -1;
  uint16_t ms_words = 0;  // HT: CodeBlock::ms_words, from the segment's last two bytes
  // Classic: the codeword-segment parts of every layer in stream order
  // (segment index, bytes, passes, offset in the codestream).
  struct Part {
    uint32_t idx, len, passes;
    int64_t off;
  };
  std::vector<Part> parts;
  uint32_t nonempty = 0;  // layers that contributed to the block
};

// Number of coding passes of a classic block (Table B.4,
// decode_num_classic_coding_passes, segment.rs:482-506): prefixes matched by
// peeking, longest first.
bool classic_passes(Reader& r, uint32_t& np) {
  auto peek = [&](uint32_t n, uint32_t want) {
    Reader c = r;
    uint32_t v;
    return c.bits(n, v) && v == want;
  };
  uint32_t v;
  if (peek(9, 0x1FF)) {
    r.bits(9, v);
    if (!r.bits(7, v)) return false;
    np = v + 37;
  } else if (peek(4, 0xF)) {
    r.bits(4, v);
    if (!r.bits(5, v)) return false;
    np = v + 6;
  } else if (peek(4, 0xE) || peek(4, 0xD) || peek(4, 0xC)) {
    r.bits(4, v);
    np = v - 0xC + 3;
  } else if (peek(2, 0x2)) {
    r.bits(2, v);
    np = 2;
  } else if (peek(1, 0)) {
    r.bits(1, v);
    np = 1;
  } else {
    return false;
  }
  return true;
}

struct Packet {  // one (layer, component, resolution, precinct)
  uint8_t comp, res;
  uint16_t layer;
  uint32_t precinct;
  uint32_t pb_begin, pb_count;
  uint64_t sort_py, sort_px;
};

}  // namespace

namespace {

Info inspect_raw(const uint8_t* data, size_t len);
void parse_tile_raw(const uint8_t* data, size_t len, const uint32_t* target, TileLayout& T);

// ---------------------------------------------------------------------------
// JP2 container (crates/signinum-j2k/src/parse/boxes.rs:10-245,
// parse/mod.rs:17-31): the box order rules, and what of the colour
// specification the decode path can honour.

struct Container {
  size_t off = 0, len = 0;  // the codestream inside the input
  bool jp2 = false;
  int colr = -1;            // enumerated colour space of the colr box, -1 none, -2 ICC / other method
  bool channel_boxes = false;  // pclr / cmap / cdef present in jp2h
};

struct BoxHeader {
  uint32_t type;
  size_t payload, end;
};

uint32_t be32(const uint8_t* p) { return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3]; }
constexpr uint32_t fourcc(char a, char b, char c, char d) {
  return ((uint32_t)(uint8_t)a << 24) | ((uint32_t)(uint8_t)b << 16) | ((uint32_t)(uint8_t)c << 8) | (uint8_t)d;
}

BoxHeader box_header(const uint8_t* d, size_t len, size_t off) {
  if (off + 8 > len) fail(ST_TRUNCATED, "box header truncated");
  const uint32_t lbox = be32(d + off);
  BoxHeader h{be32(d + off + 4), off + 8, 0};
  if (lbox == 0) {
    h.end = len;
  } else if (lbox == 1) {
    if (off + 16 > len) fail(ST_TRUNCATED, "extended box header truncated");
    const uint64_t xl = ((uint64_t)be32(d + off + 8) << 32) | be32(d + off + 12);
    if (xl < 16) fail(ST_DECODE, "extended box length smaller than header");
    if (xl > (uint64_t)SIZE_MAX - off) fail(ST_DECODE, "extended box length overflow");
    h.payload = off + 16;
    h.end = off + (size_t)xl;
  } else if (lbox < 8) {
    fail(ST_DECODE, "box length smaller than header");
  } else {
    h.end = off + lbox;
  }
  return h;
}

Container locate(const uint8_t* d, size_t len) {
  static const uint8_t kSig[12] = {0, 0, 0, 12, 'j', 'P', ' ', ' ', 0x0D, 0x0A, 0x87, 0x0A};
  Container c;
  if (len >= 8 && std::memcmp(d, kSig, 8) == 0) {
    if (len < 12) fail(ST_TRUNCATED, "input shorter than the JP2 signature");
    bool sig = false, ftyp = false, jp2h = false, ihdr = false, jp2c = false;
    for (size_t off = 0; off < len;) {
      const BoxHeader b = box_header(d, len, off);
      if (b.end > len) fail(ST_TRUNCATED, "box payload truncated");
      const uint8_t* pl = d + b.payload;
      const size_t pn = b.end - b.payload;
      if (b.type == fourcc('j', 'P', ' ', ' ')) {
        if (sig || off != 0) fail(ST_DECODE, "signature box must appear exactly once at the start of the file");
        if (pn != 4 || std::memcmp(pl, kSig + 8, 4) != 0) fail(ST_DECODE, "invalid JP2 signature payload");
        sig = true;
      } else if (b.type == fourcc('f', 't', 'y', 'p')) {
        if (!sig || ftyp || jp2h || jp2c) fail(ST_DECODE, "file type box must appear exactly once before jp2h and jp2c");
        if (pn < 8) fail(ST_DECODE, "ftyp payload shorter than 8 bytes");
        ftyp = true;
      } else if (b.type == fourcc('j', 'p', '2', 'h')) {
        if (!ftyp || jp2h || jp2c) fail(ST_DECODE, "jp2h must appear exactly once after ftyp and before jp2c");
        for (size_t o = 0; o < pn;) {
          const BoxHeader ib = box_header(pl, pn, o);
          const size_t iend = std::min(ib.end, pn);  // inner boxes are bounded by jp2h
          const uint8_t* ip = pl + ib.payload;
          const size_t in = iend > ib.payload ? iend - ib.payload : 0;
          if (ib.type == fourcc('i', 'h', 'd', 'r')) {
            if (in < 14) fail(ST_DECODE, "ihdr payload shorter than 14 bytes");
            ihdr = true;
          } else if (ib.type == fourcc('c', 'o', 'l', 'r')) {
            if (in >= 3) {
              if (ip[0] == 1 && in >= 7) c.colr = (int)be32(ip + 3);
              else if (ip[0] == 2) c.colr = -2;
            }
          } else if (ib.type == fourcc('p', 'c', 'l', 'r') || ib.type == fourcc('c', 'm', 'a', 'p') ||
                     ib.type == fourcc('c', 'd', 'e', 'f')) {
            c.channel_boxes = true;
          }
          o = ib.end;
        }
        jp2h = true;
      } else if (b.type == fourcc('j', 'p', '2', 'c')) {
        if (!jp2h || jp2c) fail(ST_DECODE, "jp2c must appear exactly once after jp2h");
        c.off = b.payload;
        c.len = pn;
        jp2c = true;
      }
      off = b.end;
    }
    if (!ftyp) fail(ST_DECODE, "missing required box ftyp");
    if (!jp2h) fail(ST_DECODE, "missing required box jp2h");
    if (!ihdr) fail(ST_DECODE, "missing required box ihdr");
    if (!jp2c) fail(ST_DECODE, "missing required box jp2c");
    c.jp2 = true;
    return c;
  }
  if (len >= 4 && d[0] == 0xFF && d[1] == 0x4F && d[2] == 0xFF && d[3] == 0x51) {
    c.len = len;
    return c;
  }
  fail(ST_UNSUPPORTED, "input is not a JP2 container or raw JPEG 2000 codestream");
  return c;
}

}  // namespace

Info inspect_codestream(const uint8_t* data, size_t len) {
  const Container c = locate(data, len);
  return inspect_raw(data + c.off, c.len);
}

void parse_tile(const uint8_t* data, size_t len, const uint32_t* target, TileLayout& T) {
  const Container c = locate(data, len);
  parse_tile_raw(data + c.off, c.len, target, T);
  // The pixel formats map the decoded components as the reference's output
  // writers do (crates/signinum-j2k/src/decode.rs:235-273, :430-470): an
  // enumerated sRGB / greyscale colour specification must agree with the
  // component count; palettes, channel definitions, sYCC and ICC profiles
  // are not mapped by this path.
  if (c.jp2) {
    if (c.channel_boxes) fail(ST_UNSUPPORTED, "JP2 palette / channel definition boxes are not supported by the CUDA path");
    if (c.colr != -1 && !((c.colr == 16 && T.ncomp == 3) || (c.colr == 17 && T.ncomp == 1)))
      fail(ST_UNSUPPORTED, "backend color space cannot be mapped to the requested pixel format");
  }
  // Offsets into the file rather than the codestream (gathered classic
  // blocks address their gather area instead).
  if (T.gathered) {
    for (auto& op : T.gather) op.first += (uint32_t)c.off;
  } else {
    for (CodeBlock& cb : T.blocks) {
      cb.cleanup_off += (uint32_t)c.off;
      if (cb.passes > 1 && !T.classic) cb.ref_off += (uint32_t)c.off;
    }
  }
}

namespace {

Info inspect_raw(const uint8_t* data, size_t len) {
  MainHeader h = read_main_header(data, len);
  Info i;
  uint32_t xsf = 1, ysf = 1;
  bool same = true;
  for (auto& c : h.comps) same = same && c.xr == h.comps[0].xr && c.yr == h.comps[0].yr;
  if (same) { xsf = h.comps[0].xr; ysf = h.comps[0].yr; }
  i.width = cdiv(h.gw - h.ox, xsf);
  i.height = cdiv(h.gh - h.oy, ysf);
  if (i.width > 60000 || i.height > 60000) fail(ST_DECODE, "image too large");
  i.components = (uint32_t)h.comps.size();
  i.bit_depth = h.comps[0].precision;
  i.levels = h.comps[0].cs.ndecomp;
  i.tiles = cdiv(h.gw - h.tox, h.tw) * cdiv(h.gh - h.toy, h.th);
  i.ht = 1;
  for (auto& c : h.comps) i.ht = i.ht && ((c.cs.cbstyle & 0x40) != 0);
  i.reversible = h.comps[0].cs.transform == 1;
  i.mct = h.mct;
  return i;
}

void parse_tile_raw(const uint8_t* data, size_t len, const uint32_t* target, TileLayout& T) {
  MainHeader h = read_main_header(data, len);
  const uint32_t nc = (uint32_t)h.comps.size();
  if (h.ox || h.oy || h.tox || h.toy) fail(ST_UNSUPPORTED, "image/tile offsets are not supported by the CUDA path");
  if (cdiv(h.gw, h.tw) * cdiv(h.gh, h.th) != 1) fail(ST_UNSUPPORTED, "multi-tile codestreams are not supported by the CUDA path");
  if (nc != 1 && nc != 3) fail(ST_UNSUPPORTED, "only gray and RGB codestreams are supported by the CUDA path");
  if (h.gw > 60000 || h.gh > 60000) fail(ST_DECODE, "image too large");
  // Tile-parts (tile.rs:162-306); per-tile COD/COC/QCD/QCC update the components.
  Reader r(data, len);
  r.bit = h.end * 8;
  std::vector<std::pair<size_t, size_t>> parts;
  bool first_part = true;
  uint8_t m;
  while (r.peek_marker(m) && m == 0x90) {
    r.marker(m);
    uint16_t lsot, isot;
    uint32_t psot;
    uint8_t tp, ntp;
    if (!r.u16(lsot) || !r.u16(isot) || !r.u32(psot) || !r.u8(tp) || !r.u8(ntp)) fail(ST_TRUNCATED, "SOT truncated");
    if (isot != 0) fail(ST_DECODE, "invalid tile index");
    size_t start = r.pos();
    size_t data_len;
    if (psot == 0) data_len = len > start ? len - start : 0;
    else {
      if (psot < 12) fail(ST_DECODE, "invalid tile-part length");
      data_len = psot - 12;
    }
    bool sod = false;
    for (;;) {
      if (!r.peek_marker(m)) break;  // non-strict: a broken tile-part header ends parsing
      r.marker(m);
      if (m == 0x93) { sod = true; break; }
      if (m == 0xD9) break;
      if (m >= 0x30 && m <= 0x3F) continue;
      uint16_t L;
      if (!r.u16(L) || L < 2 || r.pos() + L - 2 > len) fail(ST_TRUNCATED, "marker segment truncated");
      size_t seg_end = r.pos() + L - 2;
      if (m == 0x52) {
        uint8_t flags, prog, mct;
        uint16_t layers;
        CodingStyle cs;
        if (!r.u8(flags) || !r.u8(prog) || !r.u16(layers) || !r.u8(mct) || !read_coding_style(r, flags, cs) ||
            prog > 4 || layers == 0 || layers > 32)
          fail(ST_DECODE, "COD parse failure");
        h.prog = prog;
        h.layers = layers;
        h.mct = mct == 1;
        for (auto& c : h.comps) {
          uint8_t f = (uint8_t)(c.cs.flags | cs.flags);
          c.cs = cs;
          c.cs.flags = f;
        }
      } else if (m == 0x53) {
        uint16_t idx;
        uint8_t b, flags;
        CodingStyle cs;
        if (nc < 257) {
          if (!r.u8(b)) fail(ST_DECODE, "COC parse failure");
          idx = b;
        } else if (!r.u16(idx)) fail(ST_DECODE, "COC parse failure");
        if (idx >= nc || !r.u8(flags) || !read_coding_style(r, flags, cs)) fail(ST_DECODE, "COC parse failure");
        uint8_t f = (uint8_t)(h.comps[idx].cs.flags | flags);
        h.comps[idx].cs = cs;
        h.comps[idx].cs.flags = f;
      } else if (m == 0x5C) {
        Quant q;
        if (!read_quant(r, L - 2, q)) fail(ST_DECODE, "QCD parse failure");
        for (auto& c : h.comps) c.q = q;
      } else if (m == 0x5D) {
        uint16_t idx;
        uint8_t b;
        size_t isz = nc < 257 ? 1 : 2;
        Quant q;
        if (nc < 257) {
          if (!r.u8(b)) fail(ST_DECODE, "QCC parse failure");
          idx = b;
        } else if (!r.u16(idx)) fail(ST_DECODE, "QCC parse failure");
        if (idx >= nc || L < 2 + isz + 1 || !read_quant(r, L - 2 - isz, q)) fail(ST_DECODE, "QCC parse failure");
        h.comps[idx].q = q;
      } else if (m == 0x61) {
        fail(ST_UNSUPPORTED, "PPT packed packet headers are not supported by the CUDA path");
      } else if (m != 0x58 && m != 0x64) {
        fail(ST_UNSUPPORTED, "unsupported marker in tile-part header");
      }
      r.bit = seg_end * 8;
    }
    (void)first_part;
    first_part = false;
    if (!sod) break;
    size_t used = r.pos() - start;
    if (used > data_len) break;
    size_t body = data_len - used;
    if (r.pos() + body > len) fail(ST_TRUNCATED, "tile-part data truncated");
    parts.push_back({r.pos(), body});
    r.skip(body);
  }
  if (parts.empty()) fail(ST_DECODE, "no tile-part data");
  // Component checks for this path.
  const Comp& c0 = h.comps[0];
  for (auto& c : h.comps) {
    if (c.xr != 1 || c.yr != 1) fail(ST_UNSUPPORTED, "sub-sampled components are not supported by the CUDA path");
    if (c.cs.cbstyle != c0.cs.cbstyle) fail(ST_UNSUPPORTED, "components with different code-block styles");
    if (c.cs.transform != c0.cs.transform) fail(ST_UNSUPPORTED, "components with different wavelet transforms");
    // The reversible path is integer arithmetic: a quantised 5/3 codestream
    // (non-integer dequantised samples) is outside it.
    if (c.cs.transform == 1 && c.q.style != 0) fail(ST_UNSUPPORTED, "quantized reversible coding is not supported by the CUDA path");
    if (c.cs.ndecomp != c0.cs.ndecomp) fail(ST_UNSUPPORTED, "components with different level counts");
    if (c.precision != c0.precision || c.precision > 16) fail(ST_UNSUPPORTED, "component precision not supported by the CUDA path");
    if ((c.cs.cbstyle & 0x08) != (c0.cs.cbstyle & 0x08)) fail(ST_UNSUPPORTED, "mixed code-block styles");
    size_t max_res = c.cs.ndecomp, n = c.q.exps.size();
    if (n == 0) fail(ST_DECODE, "missing step sizes");
    if (c.q.style != 1 && max_res != 0 && 1 + (max_res - 1) * 3 + 2 >= n) fail(ST_DECODE, "insufficient exponents");
  }
  const bool classic = !(c0.cs.cbstyle & 0x40);
  if (h.layers > 1 && !classic) fail(ST_UNSUPPORTED, "multi-layer HTJ2K packet assembly");
  const uint32_t nlayers = h.layers;
  const uint32_t W = h.gw, H = h.gh, L = c0.cs.ndecomp;
  T = TileLayout();
  T.width = W;
  T.height = H;
  T.ncomp = nc;
  T.bit_depth = c0.precision;
  T.levels = L;
  T.mct = h.mct;
  T.reversible = c0.cs.transform == 1;
  T.causal = (c0.cs.cbstyle & 0x08) != 0;
  T.classic = classic;
  T.cbstyle = c0.cs.cbstyle;
  T.gathered = classic && nlayers > 1;
  uint32_t skipped = 0;
  if (target) {
    uint32_t wr = W / target[0], hr = H / target[1];
    uint32_t wl = wr ? 31 - (uint32_t)__builtin_clz(wr) : 0, hl = hr ? 31 - (uint32_t)__builtin_clz(hr) : 0;
    skipped = std::min(std::min(wl, hl), L);
  }
  T.skipped = skipped;
  T.out_w = cdiv(W, 1ull << skipped);
  T.out_h = cdiv(H, 1ull << skipped);
  const uint32_t nres_dec = L + 1 - skipped;
  // Bands: LL (resolution 0), then HL, LH, HH per resolution (build.rs:18-111).
  std::vector<Packet> packets;
  std::vector<PrecinctBand> pbs;
  std::vector<BlockState> blocks;
  TagPool tags;
  {
    // Room for every block of every band (and its tag-tree nodes) up front.
    const uint64_t cbs = (1ull << (h.comps[0].cs.cbw + h.comps[0].cs.cbh));
    const uint64_t est = (uint64_t)nc * ((uint64_t)W * H / std::max<uint64_t>(cbs, 1) + 8ull * (L + 1)) * 4 / 3 + 16;
    if (est < (1u << 22)) {
      blocks.reserve(est);
      tags.nodes.reserve(est * 3);
    }
  }
  T.comp_band_begin.resize(nc);
  for (uint32_t c = 0; c < nc; ++c) {
    const CodingStyle& cs = h.comps[c].cs;
    T.comp_band_begin[c] = (uint32_t)T.bands.size();
    uint64_t off = 0;
    for (uint32_t res = 0; res <= L; ++res) {
      uint32_t d = res == 0 ? L : L - res + 1;  // decomposition level
      uint64_t den = 1ull << d, half = d ? 1ull << (d - 1) : 0;
      auto span = [&](uint32_t full, bool high) -> uint32_t {
        uint64_t n = high ? (full > half ? full - half : 0) : full;
        return (uint32_t)((n + den - 1) / den);
      };
      uint8_t types[3] = {BAND_HL, BAND_LH, BAND_HH};
      uint32_t nb = res == 0 ? 1 : 3;
      uint32_t band_first = (uint32_t)T.bands.size();
      for (uint32_t k = 0; k < nb; ++k) {
        Band b;
        b.comp = (uint8_t)c;
        b.res = (uint8_t)res;
        b.type = res == 0 ? BAND_LL : types[k];
        bool hx = b.type == BAND_HL || b.type == BAND_HH, hy = b.type == BAND_LH || b.type == BAND_HH;
        b.w = span(W, hx);
        b.h = span(H, hy);
        // ComponentInfo::exponent_mantissa (codestream.rs:224-268): one entry
        // per band, or, derived, the LL entry with the exponent moved by the
        // band's level.
        const Quant& q = h.comps[c].q;
        int expo, mant;
        if (q.style == 1) {
          int e = (int)q.exps[0] - (int)L;
          if (e < 0) fail(ST_DECODE, "invalid exponents");
          expo = e + (int)(res == 0 ? L : L + 1 - res);
          mant = q.mants[0];
        } else {
          size_t ei = res == 0 ? 0 : 1 + (size_t)(res - 1) * 3 + (b.type - 1);
          if (ei >= q.exps.size()) fail(ST_DECODE, "missing step size");
          expo = q.exps[ei];
          mant = q.mants[ei];
        }
        // Dequantisation step (decode.rs:1130-1151): 2^(R_b - exponent) *
        // (1 + mantissa / 2048), R_b = precision + log2 gain (LL 0, HL/LH 1,
        // HH 2); exact in float.
        b.step = 1.0f;
        if (q.style != 0) {
          const int gain = b.type == BAND_LL ? 0 : b.type == BAND_HH ? 2 : 1;
          b.step = std::ldexp(1.0f + (float)mant / 2048.0f, (int)h.comps[c].precision + gain - expo);
        }
        int nbp = (int)q.guard + expo - 1;
        if (nbp < 0) fail(ST_DECODE, "invalid bitplane count");
        if (nbp > 32 && res < nres_dec) fail(ST_DECODE, "too many bitplanes");
        b.nbp = (uint8_t)std::min(nbp, 255);
        b.coef_off = off;
        if (res < nres_dec) off += (uint64_t)b.w * b.h;
        T.bands.push_back(b);
      }
      // Precincts of this resolution (tile.rs:487-629): the resolution rect
      // is [0, ceil(W/2^(L-res))) x [0, ceil(H/2^(L-res))).
      uint32_t rw = cdiv(W, 1ull << (L - res)), rh = cdiv(H, 1ull << (L - res));
      uint32_t ppx = cs.pexp_x[res], ppy = cs.pexp_y[res];
      if (res > 0 && (ppx == 0 || ppy == 0)) fail(ST_DECODE, "invalid precinct");
      uint32_t npx = rw == 0 ? 0 : cdiv(rw, 1ull << ppx), npy = rh == 0 ? 0 : cdiv(rh, 1ull << ppy);
      uint32_t sx = res > 0 ? ppx - 1 : ppx, sy = res > 0 ? ppy - 1 : ppy;  // precinct size in band coordinates
      uint32_t xcb = std::min<uint32_t>(cs.cbw, sx), ycb = std::min<uint32_t>(cs.cbh, sy);
      uint32_t cbw = 1u << xcb, cbh = 1u << ycb;
      uint64_t xstep = 1ull << std::min<uint32_t>(ppx + (L - res), 63), ystep = 1ull << std::min<uint32_t>(ppy + (L - res), 63);
      for (uint32_t py = 0; py < npy; ++py)
        for (uint32_t px = 0; px < npx; ++px) {
          Packet pk;
          pk.comp = (uint8_t)c;
          pk.res = (uint8_t)res;
          pk.layer = 0;
          pk.precinct = py * npx + px;
          pk.pb_begin = (uint32_t)pbs.size();
          pk.pb_count = nb;
          pk.sort_px = px * xstep;
          pk.sort_py = py * ystep;
          for (uint32_t k = 0; k < nb; ++k) {
            const Band& b = T.bands[band_first + k];
            PrecinctBand pbd;
            pbd.band = band_first + k;
            uint64_t prx0 = (uint64_t)px << sx, pry0 = (uint64_t)py << sy;
            uint64_t prx1 = prx0 + (1ull << sx), pry1 = pry0 + (1ull << sy);
            uint64_t ax0 = (prx0 / cbw) * cbw, ay0 = (pry0 / cbh) * cbh;
            uint64_t ax1 = ((std::min<uint64_t>(prx1, b.w) + cbw - 1) / cbw) * cbw;
            uint64_t ay1 = ((std::min<uint64_t>(pry1, b.h) + cbh - 1) / cbh) * cbh;
            pbd.cb_x0 = (uint32_t)ax0;
            pbd.cb_y0 = (uint32_t)ay0;
            pbd.ncx = (b.w == 0 || ax1 <= ax0) ? 0 : (uint32_t)((ax1 - ax0) / cbw);
            pbd.ncy = (b.h == 0 || ay1 <= ay0) ? 0 : (uint32_t)((ay1 - ay0) / cbh);
            pbd.cbw = cbw;
            pbd.cbh = cbh;
            pbd.first_block = (uint32_t)blocks.size();
            if ((uint64_t)pbd.ncx * pbd.ncy > (1u << 24)) fail(ST_DECODE, "too many code blocks");
            for (uint32_t yi = 0; yi < pbd.ncy; ++yi)
              for (uint32_t xi = 0; xi < pbd.ncx; ++xi) {
                BlockState bs;
                bs.band = pbd.band;
                bs.x0 = pbd.cb_x0 + xi * cbw;
                bs.y0 = pbd.cb_y0 + yi * cbh;
                bs.w = std::min<uint32_t>(bs.x0 + cbw, b.w) - bs.x0;
                bs.h = std::min<uint32_t>(bs.y0 + cbh, b.h) - bs.y0;
                blocks.push_back(bs);
              }
            pbd.incl.init(std::max<uint32_t>(pbd.ncx, 1), std::max<uint32_t>(pbd.ncy, 1), tags);
            pbd.zbp.init(std::max<uint32_t>(pbd.ncx, 1), std::max<uint32_t>(pbd.ncy, 1), tags);
            pbs.push_back(std::move(pbd));
          }
          packets.push_back(pk);
        }
    }
    T.coef_per_comp = off;
  }
  // Packet order (progression.rs:114-338): every (component, resolution,
  // precinct) once per layer; LRCP and RLCP place the layer first and second,
  // the position orders innermost.
  if (nlayers > 1) {
    const size_t n1 = packets.size();
    for (uint32_t l = 1; l < nlayers; ++l)
      for (size_t i = 0; i < n1; ++i) {
        Packet pk = packets[i];
        pk.layer = (uint16_t)l;
        packets.push_back(pk);
      }
  }
  std::vector<uint32_t> order(packets.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = (uint32_t)i;
  auto key = [&](const Packet& p) {
    const uint64_t l = p.layer;
    switch (h.prog) {
      case 0:  // LRCP: layer, resolution, component, precinct
        return std::make_tuple(l, (uint64_t)p.res, (uint64_t)p.comp, (uint64_t)0, (uint64_t)p.precinct, (uint64_t)0);
      case 1:  // RLCP: resolution, layer, component, precinct
        return std::make_tuple((uint64_t)p.res, l, (uint64_t)p.comp, (uint64_t)0, (uint64_t)p.precinct, (uint64_t)0);
      case 2:  // RPCL
        return std::make_tuple((uint64_t)p.res, p.sort_py, p.sort_px, (uint64_t)p.comp, (uint64_t)p.precinct, l);
      case 3:  // PCRL
        return std::make_tuple(p.sort_py, p.sort_px, (uint64_t)p.comp, (uint64_t)p.res, (uint64_t)p.precinct, l);
      default:  // CPRL
        return std::make_tuple((uint64_t)p.comp, p.sort_py, p.sort_px, (uint64_t)p.res, (uint64_t)p.precinct, l);
    }
  };
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return key(packets[a]) < key(packets[b]); });
  // Packet headers and bodies (segment.rs:53-148, :304-394, :409-479, :508-581).
  size_t next_packet = 0;
  for (auto& part : parts) {
    Reader pr(data + part.first, part.second);
    bool ok = true;
    while (ok && !pr.end()) {
      if (next_packet >= order.size()) { ok = false; break; }
      const Packet& pk = packets[order[next_packet++]];
      // Classic blocks with parts in this packet: (block, first new part).
      std::vector<std::pair<BlockState*, size_t>> fresh;
      const CodingStyle& cs = h.comps[pk.comp].cs;
      uint8_t mk;
      if ((cs.flags & 2) && pr.peek_marker(mk) && mk == 0x91) {
        pr.marker(mk);
        if (!pr.skip(4)) { ok = false; break; }
      }
      uint32_t nz;
      if (!pr.bits(1, nz)) { ok = false; break; }
      for (uint32_t k = 0; nz && ok && k < pk.pb_count; ++k) {
        PrecinctBand& pb = pbs[pk.pb_begin + k];
        for (uint32_t yi = 0; ok && yi < pb.ncy; ++yi)
          for (uint32_t xi = 0; ok && xi < pb.ncx; ++xi) {
            BlockState& bs = blocks[pb.first_block + yi * pb.ncx + xi];
            bool first = !bs.included;
            uint32_t v;
            bool inc;
            if (bs.included) {
              if (!pr.bits(1, v)) { ok = false; break; }
              inc = v == 1;
            } else {
              // Included in this layer when its first layer is at most pk.layer.
              if (!pb.incl.read(xi, yi, (uint32_t)pk.layer + 1, pr, v, tags)) { ok = false; break; }
              inc = v <= pk.layer;
            }
            if (!inc) continue;
            if (first) {
              if (!pb.zbp.read(xi, yi, UINT32_MAX, pr, v, tags)) { ok = false; break; }
              bs.missing = (uint8_t)v;
            }
            bs.included = true;
            if (classic) {
              // resolve_classic_segments (segment.rs:168-302): this layer's
              // passes continue the block's; a new part starts where the
              // segment index changes (every pass with termination on each
              // pass, the bypass rule, else one per contributing layer).
              uint32_t np, b, incr = 0;
              if (!classic_passes(pr, np)) { ok = false; break; }
              for (;;) {
                if (!pr.bits(1, b)) { ok = false; break; }
                if (!b) break;
                ++incr;
              }
              if (!ok) break;
              bs.lblock += incr;
              const uint32_t prev = bs.passes, cum = prev + np;
              if (cum > 1 + 3 * 31) { ok = false; break; }
              const uint8_t st = cs.cbstyle;
              auto seg_of = [&](uint32_t p) -> uint32_t {
                return (st & 0x04) ? p
                       : (st & 0x01) ? (p < 10 ? 0 : 1 + 2 * ((p - 10) / 3) + ((p - 10) % 3 == 2))
                                     : bs.nonempty;
              };
              fresh.push_back({&bs, bs.parts.size()});
              uint32_t last = seg_of(prev), count = 0;
              for (uint32_t p = prev; ok && p <= cum; ++p) {
                if (p == cum || seg_of(p) != last) {
                  if (count) {
                    uint32_t len, nbits = bs.lblock + (31 - (uint32_t)__builtin_clz(count));
                    if (nbits > 32 || !pr.bits(nbits, len) || len > 0x7FFFFFFF) { ok = false; break; }
                    bs.parts.push_back({last, len, count, -1});
                  }
                  if (p == cum) break;
                  last = seg_of(p);
                  count = 0;
                }
                ++count;
              }
              if (!ok) break;
              bs.passes = (uint8_t)cum;
              ++bs.nonempty;
              continue;
            }
            if (!first || bs.passes != 0) { ok = false; break; }
            uint32_t np = 1, b;
            if (!pr.bits(1, b)) { ok = false; break; }
            if (b) {
              np = 2;
              if (!pr.bits(1, b)) { ok = false; break; }
              if (b) {
                uint32_t e;
                if (!pr.bits(2, e)) { ok = false; break; }
                np = 3 + e;
                if (e == 3) {
                  if (!pr.bits(5, e)) { ok = false; break; }
                  np = 6 + e;
                  if (e == 31) {
                    if (!pr.bits(7, e)) { ok = false; break; }
                    np = 37 + e;
                  }
                }
              }
            }
            if (np > 94) { ok = false; break; }
            uint32_t groups = (np - 1) / 3;
            if ((uint32_t)bs.missing + groups > 255) { ok = false; break; }
            uint32_t ph = groups * 3, actual = np - ph;
            uint32_t incr = 0;
            for (;;) {
              if (!pr.bits(1, b)) { ok = false; break; }
              if (!b) break;
              ++incr;
            }
            if (!ok) break;
            bs.lblock += incr;
            uint32_t nbits = bs.lblock + (31 - (uint32_t)__builtin_clz(ph + 1));
            uint32_t lcup;
            if (nbits > 255 || !pr.bits(nbits, lcup) || lcup < 2 || lcup >= 65535) { ok = false; break; }
            uint32_t lref = 0;
            if (actual > 1) {
              uint32_t rb = bs.lblock + (actual > 2 ? 1 : 0);
              if (rb > 255 || !pr.bits(rb, lref) || lref >= 2047) { ok = false; break; }
            }
            bs.missing = (uint8_t)(bs.missing + groups);
            bs.passes = (uint8_t)actual;
            bs.lcup = lcup;
            bs.lref = lref;
          }
      }
      if (!ok) break;
      pr.align();
      if (cs.flags & 4) {
        if (!pr.marker(mk) || mk != 0x92) { ok = false; break; }
      }
      for (auto& f : fresh)
        for (size_t k = f.second; ok && k < f.first->parts.size(); ++k) {
          auto& part_k = f.first->parts[k];
          part_k.off = (int64_t)(part.first + pr.pos());
          if (!pr.skip(part_k.len)) ok = false;
        }
      for (uint32_t k = 0; nz && ok && !classic && k < pk.pb_count; ++k) {
        PrecinctBand& pb = pbs[pk.pb_begin + k];
        for (uint32_t i = 0; ok && i < pb.ncx * pb.ncy; ++i) {
          BlockState& bs = blocks[pb.first_block + i];
          if (bs.passes == 0 || bs.cleanup_off >= 0) continue;
          size_t at = part.first + pr.pos();
          if (!pr.skip(bs.lcup)) { ok = false; break; }
          bs.cleanup_off = (int64_t)at;
          if (bs.lcup >= 2) {
            // Scup from the segment's last two bytes, read here while the
            // walk is at the segment (the bodies are visited in stream order).
            const uint8_t* seg = data + at;
            const uint32_t scup = ((uint32_t)seg[bs.lcup - 1] << 4) + (seg[bs.lcup - 2] & 0x0F);
            if (scup <= bs.lcup) bs.ms_words = (uint16_t)std::min<uint32_t>((bs.lcup - scup + 15) / 4 + 2, 0xFFFFu);
          }
          if (bs.passes > 1 && !classic) {
            size_t at2 = part.first + pr.pos();
            if (!pr.skip(bs.lref)) { ok = false; break; }
            bs.ref_off = (int64_t)at2;
          }
        }
      }
    }
  }
  // Segment table for the decoded resolutions (decode.rs:1554-1718 checks).
  T.blocks.reserve(blocks.size());
  for (const BlockState& bs : blocks) {
    const Band& b = T.bands[bs.band];
    if (b.res >= nres_dec || bs.w == 0 || bs.h == 0) continue;
    CodeBlock cb;
    cb.band = bs.band;
    cb.x0 = bs.x0;
    cb.y0 = bs.y0;
    cb.w = (uint16_t)bs.w;
    cb.h = (uint16_t)bs.h;
    cb.missing_msbs = bs.missing;
    cb.passes = bs.passes;
    cb.cleanup_off = 0;
    cb.lcup = 0;
    cb.ref_off = 0;
    cb.lref = 0;
    uint32_t nbp = b.nbp;
    uint32_t actual = nbp > bs.missing ? nbp - bs.missing : 0;
    if (nbp > 31) fail(ST_DECODE, "too many bitplanes");
    if (classic) {
      // Classic blocks keep every pass; the kernel decodes the first
      // 1 + 3 (bitplanes - 1) of them (reset_for_job, bitplane.rs:493-548).
      // Parts of one segment index form one codeword segment (decode_inner,
      // bitplane.rs:90-128).  With one layer a block's parts lie back to back
      // in its packet; with several they are gathered into one run.
      if (nbp == 0 || bs.passes == 0 || actual == 0) {
        cb.passes = 0;
      } else {
        cb.seg_begin = (uint32_t)T.segments.size();
        uint64_t total = 0;
        for (size_t k = 0; k < bs.parts.size(); ++k) {
          const auto& pt = bs.parts[k];
          if (pt.off < 0) fail(ST_DECODE, "code-block decode failure: missing segment data");
          if (k > 0 && pt.idx == bs.parts[k - 1].idx) {
            T.segments.back().len += pt.len;
            T.segments.back().passes = (uint8_t)(T.segments.back().passes + pt.passes);
          } else {
            T.segments.push_back({pt.len, (uint8_t)pt.passes});
          }
          total += pt.len;
        }
        if (T.segments.size() - cb.seg_begin > 255) fail(ST_DECODE, "too many codeword segments");
        if (total > 0x7FFFFFFF) fail(ST_DECODE, "code-block data too long");
        cb.nseg = (uint8_t)(T.segments.size() - cb.seg_begin);
        cb.lcup = (uint32_t)total;
        if (!T.gathered) {
          cb.cleanup_off = bs.parts.empty() ? 0 : (uint32_t)bs.parts[0].off;
        } else {
          cb.cleanup_off = (uint32_t)T.gather_bytes;
          for (const auto& pt : bs.parts) {
            T.gather.push_back({(uint32_t)pt.off, pt.len});
            T.gather_bytes += pt.len;
          }
        }
      }
      T.blocks.push_back(cb);
      continue;
    }
    if (nbp == 0 || bs.passes == 0 || actual == 0) {
      cb.passes = 0;  // all-zero block
    } else {
      uint32_t passes = bs.passes;
      if (passes > 1 && (bs.ref_off < 0 || bs.lref == 0)) passes = 1;
      if (bs.cleanup_off < 0) fail(ST_DECODE, "code-block decode failure: missing cleanup segment data");
      if (passes > 3 || bs.missing >= 30 || bs.lcup < 2) fail(ST_DECODE, "code-block decode failure");
      if (bs.missing == 29 && passes > 1) passes = 1;
      cb.passes = (uint8_t)passes;
      cb.cleanup_off = (uint32_t)bs.cleanup_off;
      cb.lcup = bs.lcup;
      cb.ms_words = bs.ms_words;
      if (passes > 1) {
        cb.ref_off = (uint32_t)bs.ref_off;
        cb.lref = bs.lref;
      }
    }
    T.blocks.push_back(cb);
  }
}

}  // namespace

}  // namespace sgn
