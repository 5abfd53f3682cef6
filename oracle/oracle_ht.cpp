// TEST INFRASTRUCTURE ONLY — the parity oracle (see oracle_internal.h).
//
// HT code-block decoding: a restatement of
// crates/signinum-j2k-native/src/j2c/ht_block_decode.rs (MEL, forward/reverse
// bit readers, cleanup symbols, magnitude/sign, sigma, SigProp, MagRef).
#include <cstring>
#include <vector>

#include "oracle_internal.h"

namespace oracle {
namespace {

#include "../signinum_b200/csrc/tables/cxtvlc_rows.inc"

struct Tables {
  uint16_t vlc[2][1024];
  uint16_t uvlc0[320];
  uint16_t uvlc1[256];
  Tables();
};

// Prefix of one UVLC code word read LSB-first (T.814 Annex C: "1" -> 1,
// "01" -> 2, "001" -> 3 with a 1-bit suffix, "000" -> 5 with a 5-bit suffix).
static void uvlc_prefix(uint32_t bits, uint32_t& pfx, uint32_t& plen, uint32_t& slen) {
  if (bits & 1) { pfx = 1; plen = 1; slen = 0; }
  else if (bits & 2) { pfx = 2; plen = 2; slen = 0; }
  else if (bits & 4) { pfx = 3; plen = 3; slen = 1; }
  else { pfx = 5; plen = 3; slen = 5; }
}

// The packed layout matches ht_tables.rs:181/211 as consumed by
// decode_cleanup_symbols (ht_block_decode.rs:1115-1125): bits 0-2 prefix bits,
// 3-6 suffix bits, 7-9 first suffix bits, 10-12 first prefix, 13-15 second prefix.
static uint16_t uvlc_entry(uint32_t mode, uint32_t bits, bool initial) {
  uint32_t p0 = 0, l0 = 0, s0 = 0, p1 = 0, l1 = 0, s1 = 0;
  switch (mode) {
    case 0: return 0;
    case 1: uvlc_prefix(bits, p0, l0, s0); break;
    case 2: uvlc_prefix(bits, p1, l1, s1); break;
    case 3:
      uvlc_prefix(bits, p0, l0, s0);
      if (initial && p0 > 2) { p1 = 1 + ((bits >> l0) & 1); l1 = 1; s1 = 0; }
      else uvlc_prefix(bits >> l0, p1, l1, s1);
      break;
    case 4:
      uvlc_prefix(bits, p0, l0, s0);
      uvlc_prefix(bits >> l0, p1, l1, s1);
      p0 += 2; p1 += 2;
      break;
  }
  return (uint16_t)((l0 + l1) | ((s0 + s1) << 3) | (s0 << 7) | (p0 << 10) | (p1 << 13));
}

Tables::Tables() {
  std::memset(this, 0, sizeof(*this));
  const unsigned char (*rows[2])[7] = {CXTVLC_ROWS_INITIAL, CXTVLC_ROWS_NONINITIAL};
  const int counts[2] = {CXTVLC_ROWS_INITIAL_COUNT, CXTVLC_ROWS_NONINITIAL_COUNT};
  for (int t = 0; t < 2; ++t) {
    for (int i = 0; i < counts[t]; ++i) {
      const unsigned char* r = rows[t][i];
      uint32_t cq = r[0], cwd = r[1], len = r[2];
      uint16_t e = (uint16_t)((r[5] << 12) | (r[6] << 8) | (r[3] << 4) | (r[4] << 3) | len);
      for (uint32_t b = 0; b < 128; ++b)
        if ((b & ((1u << len) - 1)) == cwd) vlc[t][(cq << 7) | b] = e;
    }
  }
  for (uint32_t m = 0; m < 5; ++m)
    for (uint32_t b = 0; b < 64; ++b) uvlc0[m * 64 + b] = uvlc_entry(m, b, true);
  for (uint32_t m = 0; m < 4; ++m)
    for (uint32_t b = 0; b < 64; ++b) uvlc1[m * 64 + b] = uvlc_entry(m, b, false);
}

const Tables& tables() {
  static const Tables t;
  return t;
}

// MelDecoder, ht_block_decode.rs:782-880.
struct Mel {
  const uint8_t* data;
  size_t pos, remaining;
  bool unstuff = false;
  uint8_t cur = 0, bits_left = 0;
  int k = 0, num_runs = 0;
  uint64_t runs = 0;
  Mel(const uint8_t* d, size_t lcup, size_t scup) : data(d), pos(lcup - scup), remaining(scup - 1) {}
  uint32_t read_bit() {
    if (bits_left == 0) {
      uint8_t byte;
      if (remaining > 0) { byte = data[pos++]; --remaining; }
      else byte = 0xFF;
      if (remaining == 0) byte |= 0x0F;
      cur = byte;
      bits_left = 8 - (unstuff ? 1 : 0);
      unstuff = byte == 0xFF;
    }
    --bits_left;
    return (cur >> bits_left) & 1;
  }
  uint32_t read_bits(int n) {
    uint32_t v = 0;
    for (int i = 0; i < n; ++i) v = (v << 1) | read_bit();
    return v;
  }
  void more() {
    static const int EXP[13] = {0, 0, 0, 1, 1, 1, 2, 2, 2, 3, 3, 4, 5};
    while (num_runs < 8) {
      int e = EXP[k];
      uint32_t first = read_bit();
      uint64_t run;
      if (first == 1) {
        k = k + 1 < 12 ? k + 1 : 12;
        run = (((uint64_t)1 << e) - 1) << 1;
      } else {
        k = k > 0 ? k - 1 : 0;
        run = ((uint64_t)read_bits(e) << 1) | 1;
      }
      runs |= run << (num_runs * 7);
      ++num_runs;
      if (e == 5 && first == 0 && num_runs >= 8) break;
    }
  }
  int get_run() {
    if (num_runs == 0) more();
    int r = (int)(runs & 0x7F);
    runs >>= 7;
    --num_runs;
    return r;
  }
};

// ForwardBitReader, ht_block_decode.rs:888-930.
template <uint8_t PAD>
struct Fwd {
  const uint8_t* data;
  size_t len, pos = 0;
  uint64_t tmp = 0;
  uint32_t bits = 0;
  bool unstuff = false;
  Fwd(const uint8_t* d, size_t n) : data(d), len(n) {}
  void fill() {
    while (bits <= 32) {
      uint8_t b = pos < len ? data[pos++] : PAD;
      tmp |= (uint64_t)b << bits;
      bits += 8 - (unstuff ? 1 : 0);
      unstuff = b == 0xFF;
    }
  }
  uint32_t fetch() {
    if (bits < 32) fill();
    return (uint32_t)tmp;
  }
  void advance(uint32_t n) { tmp >>= n; bits -= n; }
};

// ReverseBitReader, ht_block_decode.rs:932-1000.
struct Rev {
  const uint8_t* data;
  long pos;
  size_t remaining;
  uint64_t tmp;
  uint32_t bits;
  bool unstuff;
  static Rev vlc(const uint8_t* d, size_t lcup, size_t scup) {
    Rev r;
    r.data = d;
    uint8_t b = d[lcup - 2];
    r.tmp = b >> 4;
    r.bits = 4 - (((r.tmp & 7) == 7) ? 1 : 0);
    r.pos = (long)lcup - 3;
    r.remaining = scup - 2;
    r.unstuff = (b | 0x0F) > 0x8F;
    return r;
  }
  static Rev mrp(const uint8_t* d, size_t n) {
    Rev r;
    r.data = d; r.pos = (long)n - 1; r.remaining = n; r.tmp = 0; r.bits = 0; r.unstuff = true;
    return r;
  }
  void fill() {
    while (bits <= 32) {
      uint8_t b = 0;
      if (remaining > 0) { b = data[pos]; --pos; --remaining; }
      uint32_t db = 8 - ((unstuff && (b & 0x7F) == 0x7F) ? 1 : 0);
      tmp |= (uint64_t)b << bits;
      bits += db;
      unstuff = b > 0x8F;
    }
  }
  uint32_t fetch() {
    if (bits < 32) fill();
    return (uint32_t)tmp;
  }
  uint32_t advance(uint32_t n) { tmp >>= n; bits -= n; return (uint32_t)tmp; }
};

static inline uint32_t clz32(uint32_t v) { return v ? (uint32_t)__builtin_clz(v) : 32; }
static inline uint32_t ctz32(uint32_t v) { return (uint32_t)__builtin_ctz(v); }
static inline uint32_t popc32(uint32_t v) { return (uint32_t)__builtin_popcount(v); }

// decode_mag_sgn_sample_with_vn, ht_block_decode.rs:1010-1032.
static inline uint32_t magsgn_sample(Fwd<0xFF>& ms, uint32_t inf, uint32_t bit, uint32_t uq, uint32_t p,
                                     uint32_t& v_out) {
  if ((inf & (1u << (4 + bit))) == 0) { v_out = 0; return 0; }
  uint32_t ms_val = ms.fetch();
  uint32_t m_n = uq - ((inf >> (12 + bit)) & 1);
  ms.advance(m_n);
  uint32_t value = ms_val << 31;
  uint32_t mask = m_n == 0 ? 0 : ((1u << m_n) - 1);
  uint32_t v_n = ms_val & mask;
  v_n |= ((inf >> (8 + bit)) & 1) << m_n;
  v_n |= 1;
  value |= (v_n + 2) << (p - 1);
  v_out = v_n;
  return value;
}

static size_t sstride(uint32_t w) { return (size_t)((w + 2 + 7) & ~7u); }
static size_t mstride(uint32_t w) { return (size_t)((((w + 3) / 4) + 2 + 7) & ~7u); }

// cleanup_segment_suffix_length, ht_block_decode.rs:1042-1054.
static bool scup_of(const uint8_t* d, size_t len, size_t lcup, size_t& scup) {
  if (lcup < 2 || len < lcup) return false;
  scup = ((size_t)d[lcup - 1] << 4) + (d[lcup - 2] & 0x0F);
  if (scup < 2 || scup > lcup || scup > 4079) return false;
  return true;
}

// decode_cleanup_symbols, ht_block_decode.rs:1056-1205.
static bool cleanup_symbols(const uint8_t* d, size_t lcup, size_t scup, uint32_t width, uint32_t height,
                            size_t sstr, uint16_t* s) {
  const Tables& T = tables();
  Mel mel(d, lcup, scup);
  Rev vlc = Rev::vlc(d, lcup, scup);
  int run = mel.get_run();
  uint32_t c_q = 0;
  size_t ro = 0;
  uint32_t x = 0;
  while (x < width) {
    uint32_t v = vlc.fetch();
    uint32_t t0 = T.vlc[0][c_q + (v & 0x7F)];
    if (c_q == 0) {
      run -= 2;
      t0 = run == -1 ? t0 : 0;
      if (run < 0) run = mel.get_run();
    }
    s[ro] = (uint16_t)t0;
    x += 2;
    c_q = ((t0 & 0x10) << 3) | ((t0 & 0xE0) << 2);
    v = vlc.advance(t0 & 7);
    uint32_t t1 = T.vlc[0][c_q + (v & 0x7F)];
    if (c_q == 0 && x < width) {
      run -= 2;
      t1 = run == -1 ? t1 : 0;
      if (run < 0) run = mel.get_run();
    }
    if (x >= width) t1 = 0;
    s[ro + 2] = (uint16_t)t1;
    x += 2;
    c_q = ((t1 & 0x10) << 3) | ((t1 & 0xE0) << 2);
    v = vlc.advance(t1 & 7);
    uint32_t mode = ((t0 & 8) << 3) | ((t1 & 8) << 4);
    if (mode == 0xC0) {
      run -= 2;
      if (run == -1) mode += 0x40;
      if (run < 0) run = mel.get_run();
    }
    uint32_t ue = T.uvlc0[mode + (v & 0x3F)];
    v = vlc.advance(ue & 7);
    ue >>= 3;
    uint32_t len = ue & 0xF;
    uint32_t tmp = v & ((1u << len) - 1);
    v = vlc.advance(len);
    ue >>= 4;
    len = ue & 7;
    ue >>= 3;
    s[ro + 1] = (uint16_t)(1 + (ue & 7) + (tmp & ~(0xFFu << len)));
    s[ro + 3] = (uint16_t)(1 + (ue >> 3) + (tmp >> len));
    ro += 4;
  }
  s[ro] = 0;
  s[ro + 1] = 0;
  for (uint32_t y = 2; y < height; y += 2) {
    size_t rb = (size_t)(y >> 1) * sstr, pb = rb - sstr;
    uint32_t xx = 0;
    c_q = 0;
    size_t r = rb;
    while (xx < width) {
      size_t o = r - rb;
      c_q |= ((uint32_t)s[pb + o] & 0xA0) << 2;
      c_q |= ((uint32_t)s[pb + o + 2] & 0x20) << 4;
      uint32_t v = vlc.fetch();
      uint32_t t0 = T.vlc[1][c_q + (v & 0x7F)];
      if (c_q == 0) {
        run -= 2;
        t0 = run == -1 ? t0 : 0;
        if (run < 0) run = mel.get_run();
      }
      s[r] = (uint16_t)t0;
      xx += 2;
      c_q = ((t0 & 0x40) << 2) | ((t0 & 0x80) << 1);
      c_q |= (uint32_t)s[pb + o] & 0x80;
      c_q |= ((uint32_t)s[pb + o + 2] & 0xA0) << 2;
      c_q |= ((uint32_t)s[pb + o + 4] & 0x20) << 4;
      v = vlc.advance(t0 & 7);
      uint32_t t1 = T.vlc[1][c_q + (v & 0x7F)];
      if (c_q == 0 && xx < width) {
        run -= 2;
        t1 = run == -1 ? t1 : 0;
        if (run < 0) run = mel.get_run();
      }
      if (xx >= width) t1 = 0;
      s[r + 2] = (uint16_t)t1;
      xx += 2;
      c_q = ((t1 & 0x40) << 2) | ((t1 & 0x80) << 1);
      c_q |= (uint32_t)s[pb + o + 2] & 0x80;
      v = vlc.advance(t1 & 7);
      uint32_t mode = ((t0 & 8) << 3) | ((t1 & 8) << 4);
      uint32_t ue = T.uvlc1[mode + (v & 0x3F)];
      v = vlc.advance(ue & 7);
      ue >>= 3;
      uint32_t len = ue & 0xF;
      uint32_t tmp = v & ((1u << len) - 1);
      v = vlc.advance(len);
      ue >>= 4;
      len = ue & 7;
      ue >>= 3;
      s[r + 1] = (uint16_t)((ue & 7) + (tmp & ~(0xFFu << len)));
      s[r + 3] = (uint16_t)((ue >> 3) + (tmp >> len));
      r += 4;
    }
    s[r] = 0;
    s[r + 1] = 0;
  }
  return true;
}

// build_sigma_from_cleanup_phase, ht_block_decode.rs:1207-1252.
static void build_sigma(const uint16_t* c, uint16_t* sg, uint32_t width, uint32_t height, size_t sstr,
                        size_t mstr) {
  for (uint32_t y = 0; y < height; y += 4) {
    size_t sp = (size_t)(y >> 1) * sstr, dp = (size_t)(y >> 2) * mstr;
    for (uint32_t x = 0; x < width; x += 4, sp += 4, ++dp) {
      uint32_t t0 = ((c[sp] & 0x30u) >> 4) | ((c[sp] & 0xC0u) >> 2);
      t0 |= ((c[sp + 2] & 0x30u) << 4) | ((c[sp + 2] & 0xC0u) << 6);
      uint32_t t1 = ((c[sp + sstr] & 0x30u) >> 2) | (c[sp + sstr] & 0xC0u);
      t1 |= ((c[sp + sstr + 2] & 0x30u) << 6) | ((c[sp + sstr + 2] & 0xC0u) << 8);
      sg[dp] = (uint16_t)(t0 | t1);
    }
    sg[dp] = 0;
  }
  size_t db = (size_t)((height + 3) / 4) * mstr;
  for (size_t x = 0; x <= (width + 3) / 4; ++x) sg[db + x] = 0;
}

static const uint32_t SPREAD[16] = {0x33,   0x76,   0xEC,   0xC8,   0x330,   0x760,   0xEC0,   0xC80,
                                    0x3300, 0x7600, 0xEC00, 0xC800, 0x33000, 0x76000, 0xEC000, 0xC8000};

static inline uint32_t pair16(const uint16_t* v, size_t i) { return (uint32_t)v[i] | ((uint32_t)v[i + 1] << 16); }

// apply_significance_propagation_phase, ht_block_decode.rs:1254-1375.
static void sigprop(const uint8_t* ref, size_t lref, const uint16_t* sigma, uint32_t* out, uint32_t width,
                    uint32_t height, uint32_t stride, size_t mstr, bool causal, uint32_t p, uint16_t* prev_row) {
  size_t prl = (width + 3) / 4 + 8;
  std::memset(prev_row, 0, prl * sizeof(uint16_t));
  Fwd<0> sp(ref, lref);
  for (uint32_t y = 0; y < height; y += 4) {
    uint32_t pattern = 0xFFFF;
    if (height - y < 4) {
      pattern = 0x7777;
      if (height - y < 3) {
        pattern = 0x3333;
        if (height - y < 2) pattern = 0x1111;
      }
    }
    uint32_t prev = 0;
    size_t cur_row = (size_t)(y >> 2) * mstr, next_row = cur_row + mstr;
    size_t dpp = (size_t)y * stride;
    for (uint32_t x = 0; x < width; x += 4) {
      uint32_t col_pattern = pattern;
      int s = (int)x + 4 - (int)width;
      if (s < 0) s = 0;
      col_pattern >>= (uint32_t)(s * 4);
      size_t idx = x >> 2;
      uint32_t ps = (uint32_t)prev_row[idx] | ((uint32_t)prev_row[idx + 1] << 16);
      uint32_t ns = pair16(sigma, next_row + idx);
      uint32_t u = (ps & 0x88888888u) >> 3;
      if (!causal) u |= (ns & 0x11111111u) << 3;
      uint32_t cs = pair16(sigma, cur_row + idx);
      uint32_t mbr = cs;
      mbr |= (cs & 0x77777777u) << 1;
      mbr |= (cs & 0xEEEEEEEEu) >> 1;
      mbr |= u;
      uint32_t t = mbr;
      mbr |= t << 4;
      mbr |= t >> 4;
      mbr |= prev >> 12;
      mbr &= col_pattern;
      mbr &= ~cs;
      uint32_t new_sig = 0;
      if (mbr != 0) {
        uint32_t cwd = sp.fetch();
        uint32_t cnt = 0;
        uint32_t inv_sig = ~cs & col_pattern;
        uint32_t cand = mbr, processed = 0;
        while (cand != 0) {
          uint32_t bit = ctz32(cand);
          uint32_t m = 1u << bit;
          cand &= ~m;
          processed |= m;
          if (cwd & 1) {
            new_sig |= m;
            cand |= SPREAD[bit] & inv_sig & ~processed;
          }
          cwd >>= 1;
          ++cnt;
        }
        if (new_sig != 0) {
          uint32_t value = 3u << (p - 2);
          size_t base = dpp + x;
          uint32_t sb = new_sig;
          while (sb != 0) {
            uint32_t bit = ctz32(sb);
            sb &= ~(1u << bit);
            size_t off = (size_t)(bit >> 2) + (size_t)(bit & 3) * stride;
            out[base + off] = ((cwd & 1) << 31) | value;
            cwd >>= 1;
            ++cnt;
          }
        }
        sp.advance(cnt);
      }
      uint32_t comb = new_sig | cs;
      prev_row[idx] = (uint16_t)comb;
      if (idx + 1 < prl) prev_row[idx + 1] = (uint16_t)(comb >> 16);
      uint32_t np = comb;
      np |= (comb & 0x7777u) << 1;
      np |= (comb & 0xEEEEu) >> 1;
      prev = (np | u) & 0xF000;
    }
  }
}

// apply_magnitude_refinement_phase, ht_block_decode.rs:1377-1433.
static bool magref(const uint8_t* ref, size_t lref, const uint16_t* sigma, uint32_t* out, uint32_t width,
                   uint32_t height, uint32_t stride, size_t mstr, uint32_t p) {
  if (p < 2) return false;
  Rev mr = Rev::mrp(ref, lref);
  uint32_t half = 1u << (p - 2);
  for (uint32_t y = 0; y < height; y += 4) {
    size_t csi = (size_t)(y >> 2) * mstr;
    size_t dpp = (size_t)y * stride;
    for (uint32_t i = 0; i < width; i += 8) {
      uint32_t cwd = mr.fetch();
      uint32_t sig = pair16(sigma, csi);
      csi += 2;
      uint32_t col_mask = 0xF;
      if (sig != 0) {
        for (uint32_t j = 0; j < 8; ++j) {
          if (sig & col_mask) {
            size_t dp = dpp + i + j;
            uint32_t sm = 0x11111111u & col_mask;
            for (int k = 0; k < 4; ++k) {
              if (sig & sm) {
                uint32_t sym = cwd & 1;
                sym = (1 - sym) << (p - 1);
                sym |= half;
                out[dp] ^= sym;
                cwd >>= 1;
              }
              sm <<= 1;
              dp += stride;
            }
          }
          col_mask <<= 4;
        }
      }
      mr.advance(popc32(sig));
    }
  }
  return true;
}

// decode_magnitude_sign_phase, ht_block_decode.rs:1435-1561.
static bool magsgn(const uint8_t* d, size_t lcup, size_t scup, const uint16_t* s, uint32_t* out, uint32_t mmsb,
                   uint32_t width, uint32_t height, uint32_t stride, size_t sstr, uint32_t* vn) {
  size_t vw = (width + 1) / 2 + 2;
  std::memset(vn, 0, vw * sizeof(uint32_t));
  uint32_t p = 30 - mmsb, mmsbp2 = mmsb + 2;
  Fwd<0xFF> ms(d, lcup - scup);
  uint32_t prev = 0, x = 0;
  size_t sp = 0, vp = 0, dp = 0;
  bool second = height > 1;
  uint32_t vt;
  while (x < width) {
    uint32_t inf = s[sp], uq = s[sp + 1];
    if (uq > mmsbp2) return false;
    out[dp] = magsgn_sample(ms, inf, 0, uq, p, vt);
    uint32_t v1;
    uint32_t val1 = magsgn_sample(ms, inf, 1, uq, p, v1);
    if (second) out[dp + stride] = val1;
    vn[vp] = prev | v1;
    prev = 0;
    ++dp; ++x;
    if (x >= width) { ++vp; break; }
    out[dp] = magsgn_sample(ms, inf, 2, uq, p, vt);
    uint32_t v3;
    uint32_t val3 = magsgn_sample(ms, inf, 3, uq, p, v3);
    if (second) out[dp + stride] = val3;
    prev = v3;
    ++dp; ++x; sp += 2; ++vp;
  }
  vn[vp] = prev;
  for (uint32_t y = 2; y < height; y += 2) {
    size_t spp = (size_t)(y >> 1) * sstr;
    size_t vpp = 0;
    size_t dpp = (size_t)y * stride;
    uint32_t pv = 0, xx = 0;
    bool sec = y + 1 < height;
    while (xx < width) {
      uint32_t inf = s[spp], u_q = s[spp + 1];
      uint32_t gamma = inf & 0xF0;
      gamma &= gamma - 0x10;
      uint32_t emax = vn[vpp] | vn[vpp + 1];
      emax = 31 - clz32(emax | 2);
      uint32_t kappa = gamma != 0 ? emax : 1;
      uint32_t uq = u_q + kappa;
      if (uq > mmsbp2) return false;
      out[dpp] = magsgn_sample(ms, inf, 0, uq, p, vt);
      uint32_t v1;
      uint32_t val1 = magsgn_sample(ms, inf, 1, uq, p, v1);
      if (sec) out[dpp + stride] = val1;
      vn[vpp] = pv | v1;
      pv = 0;
      ++dpp; ++xx;
      if (xx >= width) { ++vpp; break; }
      out[dpp] = magsgn_sample(ms, inf, 2, uq, p, vt);
      uint32_t v3;
      uint32_t val3 = magsgn_sample(ms, inf, 3, uq, p, v3);
      if (sec) out[dpp + stride] = val3;
      pv = v3;
      ++dpp; ++xx; spp += 2; ++vpp;
    }
    vn[vpp] = pv;
  }
  return true;
}

}  // namespace

const uint16_t* vlc_table(int which) { return tables().vlc[which & 1]; }
const uint16_t* uvlc_table(int which) { return which ? tables().uvlc1 : tables().uvlc0; }

// decode_impl, ht_block_decode.rs:1563-1683 (PHASE_LIMIT_MAGREF).
bool ht_block_decode(const uint8_t* cleanup, size_t lcup, const uint8_t* refinement, size_t lref,
                     uint32_t missing_msbs, uint32_t num_passes, uint32_t width, uint32_t height,
                     uint32_t stride, bool stripe_causal, uint32_t* out) {
  if (num_passes > 1 && lref == 0) num_passes = 1;
  if (num_passes > 3 || missing_msbs > 30) return false;
  if (missing_msbs == 30) return false;
  if (missing_msbs == 29 && num_passes > 1) num_passes = 1;
  uint32_t p = 30 - missing_msbs;
  if (lcup < 2) return false;
  size_t scup;
  if (!scup_of(cleanup, lcup, lcup, scup)) return false;
  size_t quad_rows = (height + 1) / 2;
  size_t sstr = sstride(width);
  std::vector<uint16_t> scratch(sstr * (quad_rows + 1), 0);
  if (!cleanup_symbols(cleanup, lcup, scup, width, height, sstr, scratch.data())) return false;
  std::vector<uint32_t> vn((width + 1) / 2 + 2, 0);
  if (!magsgn(cleanup, lcup, scup, scratch.data(), out, missing_msbs, width, height, stride, sstr, vn.data()))
    return false;
  if (num_passes > 1) {
    size_t sigma_rows = (height + 3) / 4 + 1;
    size_t mstr = mstride(width);
    std::vector<uint16_t> sigma(sigma_rows * mstr, 0);
    build_sigma(scratch.data(), sigma.data(), width, height, sstr, mstr);
    std::vector<uint16_t> prev_row((width + 3) / 4 + 8, 0);
    sigprop(refinement, lref, sigma.data(), out, width, height, stride, mstr, stripe_causal, p, prev_row.data());
    if (num_passes > 2) {
      if (!magref(refinement, lref, sigma.data(), out, width, height, stride, mstr, p)) return false;
    }
  }
  return true;
}

}  // namespace oracle
