// Lossless HTJ2K encoder (host C++): the input side of the decode path.
//
// Produces raw J2K codestreams the way the reference's lossless facade does
// (crates/signinum-j2k/src/encode.rs:166-372 over
// crates/signinum-j2k-native/src/j2c/encode.rs:265-480): DC level shift,
// reversible colour transform, forward 5/3 with vertical then horizontal
// lifting per level, no quantisation (exponents bit_depth + band gain, guard
// bits raised to 2 with RCT), HT cleanup-only code blocks, one layer, one
// precinct per resolution unless precinct exponents are given (then the
// resolutions are cut into precincts, code blocks clipped to them, packets
// per precinct in the progression's order), SIZ/CAP/COD/QCD/[TLM]/SOT/SOD/EOC
// markers.
//
// The irreversible mode produces lossy inputs for the 9/7 decode path (it
// has no counterpart in the reference, which encodes losslessly only): DC
// shift, ICT, forward 9/7 lifting (Table F.4 factors) with vertical then
// horizontal passes, and scalar expounded quantisation with one relative
// step for every band, q = sign(y) floor(|y| / step_b),
// step_b = 2^(bit_depth + gain_b - eps) (1 + mu / 2048).
//
// The HT block coder is written here from the HTJ2K cleanup-pass definition
// (T.814): MEL run coding of quad significance in zero contexts, CxtVLC
// codewords with UVLC exponent offsets in a backward-growing VLC stream, and
// magnitude/sign bits in a forward stream, ending in the Scup trailer.  Every
// context and exponent predictor mirrors what the decoder recomputes.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

#include "../ebcot.h"
#include "../ht_tables.h"
#include "j2k_encode.h"

namespace sgn {
namespace enc {

static const HtEncodeTables& enc_tables() {
  static HtEncodeTables* t = [] {
    auto* p = new HtEncodeTables;
    build_encode_tables(*p);
    return p;
  }();
  return *t;
}

// Forward byte stream, bits LSB-first; a byte after 0xFF carries 7 bits.
struct MagSgnWriter {
  std::vector<uint8_t> buf;
  uint64_t tmp = 0;
  uint32_t used = 0, cap = 8;
  void put(uint32_t v, uint32_t n) {
    if (n == 0) return;
    tmp |= (uint64_t)(v & (n >= 32 ? 0xFFFFFFFFu : ((1u << n) - 1))) << used;
    used += n;
    while (used >= cap) {
      uint8_t b = (uint8_t)(tmp & ((1u << cap) - 1));
      buf.push_back(b);
      tmp >>= cap;
      used -= cap;
      cap = b == 0xFF ? 7 : 8;
    }
  }
  void terminate() {
    if (used > 0) {
      uint8_t b = (uint8_t)((tmp | (0xFFu << used)) & ((1u << cap) - 1));
      if (cap == 7) b &= 0x7F;
      if (b != 0xFF) buf.push_back(b);
    } else if (!buf.empty() && buf.back() == 0xFF) {
      buf.pop_back();  // the decoder pads the stream with 0xFF anyway
    }
    used = 0;
    tmp = 0;
  }
};

// MEL: adaptive run-length coder of binary events, bits MSB-first.
struct MelWriter {
  std::vector<uint8_t> buf;
  uint32_t tmp = 0, remaining = 8;
  int k = 0;
  uint32_t run = 0;
  static int exp_of(int k) {
    static const int E[13] = {0, 0, 0, 1, 1, 1, 2, 2, 2, 3, 3, 4, 5};
    return E[k];
  }
  void emit(uint32_t bit) {
    tmp = (tmp << 1) | (bit & 1);
    if (--remaining == 0) {
      buf.push_back((uint8_t)tmp);
      remaining = tmp == 0xFF ? 7 : 8;
      tmp = 0;
    }
  }
  void event(bool one) {
    if (!one) {
      if (++run >= (1u << exp_of(k))) {
        emit(1);
        run = 0;
        k = std::min(k + 1, 12);
      }
    } else {
      emit(0);
      for (int t = exp_of(k) - 1; t >= 0; --t) emit((run >> t) & 1);
      run = 0;
      k = std::max(k - 1, 0);
    }
  }
};

// VLC: grows backward from the end of the segment; bits LSB-first within a
// byte; a byte following (in reading order) one above 0x8F whose low seven
// bits would all be ones keeps its top bit clear.
struct VlcWriter {
  std::vector<uint8_t> rev;  // rev[0] is the last byte of the segment
  uint32_t tmp, used;
  bool last_gt_8f;
  VlcWriter() {
    rev.push_back(0xFF);  // placeholder for Scup >> 4
    tmp = 0xF;            // placeholder for Scup & 0xF
    used = 4;
    last_gt_8f = true;
  }
  void put(uint32_t v, uint32_t n) {
    while (n > 0) {
      uint32_t avail = 8 - (last_gt_8f ? 1 : 0) - used;
      uint32_t t = std::min(avail, n);
      tmp |= (v & ((1u << t) - 1)) << used;
      used += t;
      avail -= t;
      n -= t;
      v >>= t;
      if (avail == 0) {
        if (last_gt_8f && tmp != 0x7F) {
          last_gt_8f = false;
          continue;
        }
        rev.push_back((uint8_t)tmp);
        last_gt_8f = tmp > 0x8F;
        tmp = 0;
        used = 0;
      }
    }
  }
};

static inline uint32_t bitlen(uint32_t v) { return v ? 32 - (uint32_t)__builtin_clz(v) : 0; }

// UVLC code for u >= 1 (no extension bits: u <= 32).
static void uvlc_code(uint32_t u, uint32_t& pre, uint32_t& plen, uint32_t& suf, uint32_t& slen) {
  if (u == 1) { pre = 1; plen = 1; suf = 0; slen = 0; }
  else if (u == 2) { pre = 2; plen = 2; suf = 0; slen = 0; }
  else if (u <= 4) { pre = 4; plen = 3; suf = u - 3; slen = 1; }
  else { pre = 0; plen = 3; suf = u - 5; slen = 5; }
}

struct Quad {
  uint32_t rho = 0;
  uint32_t E[4] = {0, 0, 0, 0};
  uint32_t v[4] = {0, 0, 0, 0};
  uint32_t emax = 0;
  uint32_t U = 0, uq = 0, uoff = 0, ek = 0;
};

// Encodes one code block's cleanup pass with its lowest bit-plane at 0.
// Returns 0 on success (out empty when every coefficient is zero), or -1 when
// a magnitude needs more than Mb bits or an exponent needs UVLC extension bits.
int encode_ht_block(const int32_t* c, size_t stride, uint32_t w, uint32_t h, uint32_t Mb, std::vector<uint8_t>& out) {
  out.clear();
  bool any = false;
  for (uint32_t y = 0; y < h && !any; ++y)
    for (uint32_t x = 0; x < w; ++x)
      if (c[y * stride + x] != 0) { any = true; break; }
  if (!any) return 0;
  const HtEncodeTables& T = enc_tables();
  const uint32_t nq = (w + 1) / 2, nqr = (h + 1) / 2;
  std::vector<Quad> prev(nq + 3), cur(nq + 3);
  MagSgnWriter ms;
  MelWriter mel;
  VlcWriter vlc;
  auto load = [&](uint32_t qx, uint32_t qy, Quad& q) -> int {
    q = Quad();
    for (int i = 0; i < 4; ++i) {
      uint32_t x = 2 * qx + (i >> 1), y = 2 * qy + (i & 1);
      if (x >= w || y >= h) continue;
      int32_t val = c[(size_t)y * stride + x];
      if (val == 0) continue;
      uint32_t mu = (uint32_t)(val < 0 ? -(int64_t)val : val);
      if (Mb < 31 && mu >= (1u << Mb)) return -1;
      uint32_t s = val < 0 ? 1 : 0;
      q.rho |= 1u << i;
      q.v[i] = 2 * (mu - 1) + s;
      q.E[i] = bitlen(2 * mu - 1);
      q.emax = std::max(q.emax, q.E[i]);
    }
    return 0;
  };
  auto emb_of = [](const Quad& q) {
    uint32_t e = 0;
    for (int i = 0; i < 4; ++i)
      if ((q.rho >> i & 1) && q.E[i] == q.U) e |= 1u << i;
    return e;
  };
  auto codeword = [&](int tb, uint32_t ctx, Quad& q) -> int {
    uint32_t emb = q.uoff ? emb_of(q) : 0;
    const HtEncodeEntry& e = T.e[tb][ctx][q.rho][q.uoff][emb];
    if (!e.valid) return -1;
    vlc.put(e.cwd, e.len);
    q.ek = e.e_k;
    return 0;
  };
  auto magsgn = [&](const Quad& q) {
    for (int i = 0; i < 4; ++i) {
      if (!(q.rho >> i & 1)) continue;
      uint32_t m = q.U - ((q.ek >> i) & 1);
      ms.put(q.v[i], m);
    }
  };
  for (uint32_t qy = 0; qy < nqr; ++qy) {
    const bool initial = qy == 0;
    for (uint32_t qx = 0; qx < nq; ++qx)
      if (load(qx, qy, cur[qx]) != 0) return -1;
    for (uint32_t qx = nq; qx < nq + 3; ++qx) cur[qx] = Quad();
    // Exponent offsets: kappa is 1 in the initial row; elsewhere it follows
    // the largest exponent among the four samples above when the quad has
    // two or more significant samples.
    for (uint32_t qx = 0; qx < nq; ++qx) {
      Quad& q = cur[qx];
      uint32_t kappa = 1;
      if (!initial && __builtin_popcount(q.rho) >= 2) {
        uint32_t e = 0;
        if (qx > 0) e = std::max(e, prev[qx - 1].E[3]);
        e = std::max(e, prev[qx].E[1]);
        e = std::max(e, prev[qx].E[3]);
        e = std::max(e, prev[qx + 1].E[1]);
        kappa = std::max<uint32_t>(e, 2) - 1;
      }
      q.U = std::max(q.emax, kappa);
      q.uq = q.U - kappa;
      q.uoff = q.uq > 0 ? 1 : 0;
      if (q.uq > 32) return -1;
    }
    uint32_t c_q = 0;
    for (uint32_t a = 0; a < nq; a += 2) {
      Quad& A = cur[a];
      Quad& B = cur[a + 1];
      const bool hasB = a + 1 < nq;
      if (initial) {
        if (c_q == 0) mel.event(A.rho != 0);
        if (c_q != 0 || A.rho != 0)
          if (codeword(0, c_q, A) != 0) return -1;
        uint32_t tA = A.rho << 4;
        c_q = ((tA & 0x10) << 3 | (tA & 0xE0) << 2) >> 7;
        if (hasB) {
          if (c_q == 0) mel.event(B.rho != 0);
          if (c_q != 0 || B.rho != 0)
            if (codeword(0, c_q, B) != 0) return -1;
          uint32_t tB = B.rho << 4;
          c_q = ((tB & 0x10) << 3 | (tB & 0xE0) << 2) >> 7;
        } else {
          c_q = 0;
        }
        uint32_t p0, l0, s0, n0, p1, l1, s1, n1;
        if (A.uoff && B.uoff) {
          bool both = A.uq > 2 && B.uq > 2;
          mel.event(both);
          if (both) {
            uvlc_code(A.uq - 2, p0, l0, s0, n0);
            uvlc_code(B.uq - 2, p1, l1, s1, n1);
            vlc.put(p0, l0); vlc.put(p1, l1); vlc.put(s0, n0); vlc.put(s1, n1);
          } else if (A.uq > 2) {
            uvlc_code(A.uq, p0, l0, s0, n0);
            vlc.put(p0, l0);
            vlc.put(B.uq - 1, 1);
            vlc.put(s0, n0);
          } else {
            uvlc_code(A.uq, p0, l0, s0, n0);
            uvlc_code(B.uq, p1, l1, s1, n1);
            vlc.put(p0, l0); vlc.put(p1, l1); vlc.put(s0, n0); vlc.put(s1, n1);
          }
        } else if (A.uoff) {
          uvlc_code(A.uq, p0, l0, s0, n0);
          vlc.put(p0, l0); vlc.put(s0, n0);
        } else if (B.uoff) {
          uvlc_code(B.uq, p1, l1, s1, n1);
          vlc.put(p1, l1); vlc.put(s1, n1);
        }
      } else {
        // Context from the row above (rho of quads a, a+1, a+2) and from the
        // quad to the left, as the decoder rebuilds it.
        auto t = [&](uint32_t i) { return prev[i].rho << 4; };
        uint32_t cq = (c_q << 7);
        cq |= (t(a) & 0xA0) << 2;
        cq |= (t(a + 1) & 0x20) << 4;
        uint32_t ctxA = cq >> 7;
        if (ctxA == 0) mel.event(A.rho != 0);
        if (ctxA != 0 || A.rho != 0)
          if (codeword(1, ctxA, A) != 0) return -1;
        uint32_t tA = A.rho << 4;
        cq = ((tA & 0x40) << 2) | ((tA & 0x80) << 1);
        cq |= t(a) & 0x80;
        cq |= (t(a + 1) & 0xA0) << 2;
        cq |= (t(a + 2) & 0x20) << 4;
        uint32_t ctxB = cq >> 7;
        uint32_t tB = 0;
        if (hasB) {
          if (ctxB == 0) mel.event(B.rho != 0);
          if (ctxB != 0 || B.rho != 0)
            if (codeword(1, ctxB, B) != 0) return -1;
          tB = B.rho << 4;
        }
        cq = ((tB & 0x40) << 2) | ((tB & 0x80) << 1);
        cq |= t(a + 1) & 0x80;
        c_q = cq >> 7;
        uint32_t p0 = 0, l0 = 0, s0 = 0, n0 = 0, p1 = 0, l1 = 0, s1 = 0, n1 = 0;
        if (A.uoff) uvlc_code(A.uq, p0, l0, s0, n0);
        if (hasB && B.uoff) uvlc_code(B.uq, p1, l1, s1, n1);
        vlc.put(p0, l0); vlc.put(p1, l1); vlc.put(s0, n0); vlc.put(s1, n1);
      }
      magsgn(A);
      if (hasB) magsgn(B);
    }
    std::swap(prev, cur);
  }
  // Terminate MEL and VLC, fusing their meeting bytes when the bits allow.
  if (mel.run > 0) mel.emit(1);
  uint32_t mel_tmp = (mel.tmp << mel.remaining) & 0xFF;
  uint32_t mel_mask = (0xFFu << mel.remaining) & 0xFF;
  uint32_t vlc_mask = (1u << vlc.used) - 1;
  if ((mel_mask | vlc_mask) != 0) {
    uint32_t fuse = mel_tmp | vlc.tmp;
    if (((((fuse ^ mel_tmp) & mel_mask) | ((fuse ^ vlc.tmp) & vlc_mask)) == 0) && fuse != 0xFF && vlc.rev.size() > 1) {
      mel.buf.push_back((uint8_t)fuse);
    } else {
      mel.buf.push_back((uint8_t)mel_tmp);
      vlc.rev.push_back((uint8_t)vlc.tmp);
    }
  }
  ms.terminate();
  size_t scup = mel.buf.size() + vlc.rev.size();
  if (scup < 2 || scup > 4079) return -1;
  out = ms.buf;
  out.insert(out.end(), mel.buf.begin(), mel.buf.end());
  for (size_t i = vlc.rev.size(); i-- > 0;) out.push_back(vlc.rev[i]);
  size_t L = out.size();
  out[L - 1] = (uint8_t)(scup >> 4);
  out[L - 2] = (uint8_t)((out[L - 2] & 0xF0) | (scup & 0xF));
  return 0;
}

// ---------------------------------------------------------------------------
// Packet headers: MSB-first bits; after a 0xFF byte the next byte carries 7.
struct HeaderWriter {
  std::vector<uint8_t> buf;
  uint32_t tmp = 0, n = 0, cap = 8;
  void bit(uint32_t b) {
    tmp = (tmp << 1) | (b & 1);
    if (++n == cap) {
      buf.push_back((uint8_t)tmp);
      cap = tmp == 0xFF ? 7 : 8;
      tmp = 0;
      n = 0;
    }
  }
  void bits(uint32_t v, uint32_t cnt) {
    for (uint32_t i = cnt; i-- > 0;) bit((v >> i) & 1);
  }
  void flush() {
    if (n > 0) {
      buf.push_back((uint8_t)(tmp << (cap - n)));
      n = 0;
      tmp = 0;
    }
    if (!buf.empty() && buf.back() == 0xFF) buf.push_back(0x00);
  }
};

// Tag tree over a w x h grid of leaves (standard quad-tree, levels aligned to
// the origin).
struct TagTree {
  std::vector<std::vector<uint32_t>> value, low;
  std::vector<std::vector<uint8_t>> known;
  std::vector<uint32_t> lw, lh;
  TagTree(uint32_t w, uint32_t h, const std::vector<uint32_t>& leaves) {
    uint32_t cw = w, ch = h;
    for (;;) {
      lw.push_back(cw);
      lh.push_back(ch);
      value.emplace_back((size_t)cw * ch, UINT32_MAX);
      low.emplace_back((size_t)cw * ch, 0);
      known.emplace_back((size_t)cw * ch, 0);
      if (cw <= 1 && ch <= 1) break;
      cw = (cw + 1) / 2;
      ch = (ch + 1) / 2;
    }
    value[0] = leaves;
    for (size_t l = 1; l < value.size(); ++l)
      for (uint32_t y = 0; y < lh[l - 1]; ++y)
        for (uint32_t x = 0; x < lw[l - 1]; ++x) {
          uint32_t& p = value[l][(y / 2) * lw[l] + x / 2];
          p = std::min(p, value[l - 1][(size_t)y * lw[l - 1] + x]);
        }
  }
  void encode(uint32_t x, uint32_t y, uint32_t threshold, HeaderWriter& hw) {
    size_t L = value.size();
    uint32_t lowv = 0;
    for (size_t l = L; l-- > 0;) {
      size_t i = (size_t)(y >> l) * lw[l] + (x >> l);
      if (low[l][i] < lowv) low[l][i] = lowv;
      else lowv = low[l][i];
      while (lowv < threshold) {
        if (lowv >= value[l][i]) {
          if (!known[l][i]) {
            hw.bit(1);
            known[l][i] = 1;
          }
          break;
        }
        hw.bit(0);
        ++lowv;
      }
      low[l][i] = lowv;
    }
  }
};

struct CodeBlockOut {
  std::vector<uint8_t> bytes;
  ClassicBlockOut classic;  // classic Tier-1 segments (bytes unused then)
  bool empty() const { return bytes.empty() && classic.passes == 0; }
};

struct Band {
  uint32_t w = 0, h = 0, cbw = 0, cbh = 0, ncx = 0, ncy = 0, mb = 0;
  std::vector<CodeBlockOut> blocks;
};

static inline int32_t floor_div(int32_t a, int sh) { return a >> sh; }

// Whole-sample symmetric extension of a line of n samples with stride s.
template <typename T>
static T& ext(T* x, long i, size_t n, size_t s) {
  if (i < 0) i = -i;
  if (i >= (long)n) i = 2 * ((long)n - 1) - i;
  return x[(size_t)i * s];
}

// Forward 5/3 lifting of one line (n samples, stride s), origin even.
static void fwd53(int32_t* x, size_t n, size_t s) {
  if (n < 2) return;
  auto at = [&](long i) -> int32_t& { return ext(x, i, n, s); };
  for (long i = 1; i < (long)n; i += 2) at(i) -= floor_div(at(i - 1) + at(i + 1), 1);
  for (long i = 0; i < (long)n; i += 2) at(i) += floor_div(at(i - 1) + at(i + 1) + 2, 2);
}

// Forward 9/7 lifting of one line, origin even: predict/update steps with
// alpha, beta, gamma, delta, then low samples scaled by 1/K, high by K.
static void fwd97(double* x, size_t n, size_t s) {
  if (n < 2) return;
  auto at = [&](long i) -> double& { return ext(x, i, n, s); };
  const double a = -1.586134342059924, b = -0.052980118572961, g = 0.882911075530934, d = 0.443506852043971;
  const double k = 1.230174104914001;
  for (long i = 1; i < (long)n; i += 2) at(i) += a * (at(i - 1) + at(i + 1));
  for (long i = 0; i < (long)n; i += 2) at(i) += b * (at(i - 1) + at(i + 1));
  for (long i = 1; i < (long)n; i += 2) at(i) += g * (at(i - 1) + at(i + 1));
  for (long i = 0; i < (long)n; i += 2) at(i) += d * (at(i - 1) + at(i + 1));
  for (long i = 0; i < (long)n; ++i) at(i) *= (i % 2 == 0) ? 1.0 / k : k;
}

// L levels of a separable decomposition of a w x h plane: vertical then
// horizontal lifting of the current LL, then de-interleaving.  hl/lh/hh[d]
// hold level d (1 = finest); lw/lh_[d] the LL size after level d.
template <typename T, typename Lift>
static void decompose(std::vector<T> cur, uint32_t W, uint32_t H, uint32_t L, Lift lift, std::vector<T>& ll_out,
                      std::vector<std::vector<T>>& hl, std::vector<std::vector<T>>& lh,
                      std::vector<std::vector<T>>& hh, std::vector<uint32_t>& lw, std::vector<uint32_t>& lhh) {
  uint32_t cw = W, ch = H;
  hl.assign(L + 1, {});
  lh.assign(L + 1, {});
  hh.assign(L + 1, {});
  lw.assign(L + 2, 0);
  lhh.assign(L + 2, 0);
  lw[0] = W;
  lhh[0] = H;
  for (uint32_t d = 1; d <= L; ++d) {
    for (uint32_t x = 0; x < cw; ++x) lift(&cur[x], ch, cw);
    for (uint32_t y = 0; y < ch; ++y) lift(&cur[(size_t)y * cw], cw, 1);
    uint32_t lwd = (cw + 1) / 2, hwd = cw / 2, lhd = (ch + 1) / 2, hhd = ch / 2;
    std::vector<T> ll((size_t)lwd * lhd);
    hl[d].assign((size_t)hwd * lhd, 0);
    lh[d].assign((size_t)lwd * hhd, 0);
    hh[d].assign((size_t)hwd * hhd, 0);
    for (uint32_t y = 0; y < ch; ++y)
      for (uint32_t x = 0; x < cw; ++x) {
        T v = cur[(size_t)y * cw + x];
        if (y % 2 == 0 && x % 2 == 0) ll[(size_t)(y / 2) * lwd + x / 2] = v;
        else if (y % 2 == 0) hl[d][(size_t)(y / 2) * hwd + x / 2] = v;
        else if (x % 2 == 0) lh[d][(size_t)(y / 2) * lwd + x / 2] = v;
        else hh[d][(size_t)(y / 2) * hwd + x / 2] = v;
      }
    cur.swap(ll);
    cw = lwd;
    ch = lhd;
    lw[d] = cw;
    lhh[d] = ch;
  }
  ll_out.swap(cur);
}

// Scalar quantisation of a band: sign(y) floor(|y| / step), magnitudes
// clamped to the band's mb bit-planes.
static std::vector<int32_t> quantize(const std::vector<double>& y, double step, uint32_t mb) {
  std::vector<int32_t> q(y.size());
  const double maxq = (double)((1u << std::min<uint32_t>(mb, 30)) - 1);
  for (size_t i = 0; i < y.size(); ++i) {
    double m = std::min(std::floor(std::fabs(y[i]) / step), maxq);
    q[i] = y[i] < 0 ? -(int32_t)m : (int32_t)m;
  }
  return q;
}

static void put16(std::vector<uint8_t>& o, uint32_t v) { o.push_back((uint8_t)(v >> 8)); o.push_back((uint8_t)v); }
static void put32(std::vector<uint8_t>& o, uint32_t v) { put16(o, v >> 16); put16(o, v & 0xFFFF); }

int encode(const uint8_t* pixels, const EncodeParams& P, std::vector<uint8_t>& out) {
  const uint32_t W = P.width, H = P.height, C = P.comps, bd = P.bit_depth;
  if (W == 0 || H == 0 || C == 0 || C > 4 || bd == 0 || bd > 16) return -2;
  uint32_t maxl = 0;
  {
    uint32_t m = std::min(W, H);
    while ((2u << maxl) <= m) ++maxl;
    if (m <= 1) maxl = 0;
  }
  const uint32_t L = std::min(P.levels, maxl);
  const bool mct = P.mct && C >= 3;
  const bool irr = P.irreversible;
  const uint32_t guard = (mct || irr) ? 2 : 1;
  // Relative step of the irreversible path as 2^-eps (1 + mu / 2048).
  uint32_t q_eps = 0, q_mu = 0;
  if (irr) {
    if (!(P.rel_step > 0.0) || P.rel_step >= 1.0) return -2;
    while (q_eps < 24 && std::ldexp(1.0, -(int)q_eps) > P.rel_step) ++q_eps;
    double m = std::round((P.rel_step * std::ldexp(1.0, (int)q_eps) - 1.0) * 2048.0);
    q_mu = (uint32_t)std::min(std::max(m, 0.0), 2047.0);
    if (q_eps < 1) return -2;
  }
  const size_t N = (size_t)W * H;
  const int32_t shift = 1 << (bd - 1);
  auto sample = [&](size_t i, uint32_t c) -> int32_t {
    int32_t v = bd <= 8 ? pixels[i * C + c] : (int32_t)(pixels[(i * C + c) * 2] | (pixels[(i * C + c) * 2 + 1] << 8));
    return (v & ((1 << bd) - 1)) - shift;
  };
  std::vector<std::vector<int32_t>> comp(irr ? 0 : C, std::vector<int32_t>(N));
  std::vector<std::vector<double>> compf(irr ? C : 0, std::vector<double>(N));
  if (!irr) {
    for (size_t i = 0; i < N; ++i)
      for (uint32_t c = 0; c < C; ++c) comp[c][i] = sample(i, c);
    if (mct) {
      for (size_t i = 0; i < N; ++i) {
        int32_t r = comp[0][i], g = comp[1][i], b = comp[2][i];
        comp[0][i] = floor_div(r + 2 * g + b, 2);
        comp[1][i] = b - g;
        comp[2][i] = r - g;
      }
    }
  } else {
    for (size_t i = 0; i < N; ++i)
      for (uint32_t c = 0; c < C; ++c) compf[c][i] = sample(i, c);
    if (mct) {
      for (size_t i = 0; i < N; ++i) {
        double r = compf[0][i], g = compf[1][i], b = compf[2][i];
        compf[0][i] = 0.299 * r + 0.587 * g + 0.114 * b;
        compf[1][i] = -0.168736 * r - 0.331264 * g + 0.5 * b;
        compf[2][i] = 0.5 * r - 0.418688 * g - 0.081312 * b;
      }
    }
  }
  // Per component: bands[0] = LL, then HL, LH, HH per resolution 1..L.
  std::vector<std::vector<Band>> bands(C);
  // Precincts (B.6): resolution r is cut into 2^PPx x 2^PPy precincts; in
  // its sub-bands that is 2^(PPx-1) x 2^(PPy-1) samples (2^PPx x 2^PPy in
  // the LL band of resolution 0), and code blocks are clipped to that size
  // (B.7: xcb' = min(xcb, PPx - 1), or PPx at resolution 0).
  const bool precincts = P.ppx || P.ppy;
  if (precincts && (P.ppx < 1 || P.ppy < 1 || P.ppx > 15 || P.ppy > 15)) return -2;
  auto band_pp = [&](uint32_t pp, uint32_t r) { return r == 0 ? pp : pp - 1; };
  auto cb_w = [&](uint32_t r) {
    return 1u << (precincts ? std::min(P.cbw_exp + 2, band_pp(P.ppx, r)) : P.cbw_exp + 2);
  };
  auto cb_h = [&](uint32_t r) {
    return 1u << (precincts ? std::min(P.cbh_exp + 2, band_pp(P.ppy, r)) : P.cbh_exp + 2);
  };
  std::vector<uint32_t> res_w(L + 1), res_h(L + 1);  // resolution sizes
  auto band_mb = [&](uint32_t gain) { return irr ? guard + q_eps - 1 : guard + bd + gain - 1; };
  for (uint32_t c = 0; c < C; ++c) {
    std::vector<int32_t> cur;
    std::vector<std::vector<int32_t>> hl, lh, hh;
    std::vector<uint32_t> lw, lhh;
    if (!irr) {
      decompose(std::move(comp[c]), W, H, L, fwd53, cur, hl, lh, hh, lw, lhh);
    } else {
      std::vector<double> llf;
      std::vector<std::vector<double>> hlf, lhf, hhf;
      decompose(std::move(compf[c]), W, H, L, fwd97, llf, hlf, lhf, hhf, lw, lhh);
      auto step = [&](uint32_t gain) { return std::ldexp(1.0 + q_mu / 2048.0, (int)(bd + gain) - (int)q_eps); };
      cur = quantize(llf, step(0), band_mb(0));
      hl.assign(L + 1, {});
      lh.assign(L + 1, {});
      hh.assign(L + 1, {});
      for (uint32_t d = 1; d <= L; ++d) {
        hl[d] = quantize(hlf[d], step(1), band_mb(1));
        lh[d] = quantize(lhf[d], step(1), band_mb(1));
        hh[d] = quantize(hhf[d], step(2), band_mb(2));
      }
    }
    const uint32_t cw = lw[L], ch = lhh[L];
    auto make_band = [&](const std::vector<int32_t>& data, uint32_t w, uint32_t h, uint32_t gain,
                         uint8_t band_class, uint32_t cbw, uint32_t cbh) -> int {
      Band b;
      b.w = w;
      b.h = h;
      b.cbw = cbw;
      b.cbh = cbh;
      b.mb = band_mb(gain);
      b.ncx = w ? (w + cbw - 1) / cbw : 0;
      b.ncy = h ? (h + cbh - 1) / cbh : 0;
      for (uint32_t by = 0; by < b.ncy; ++by)
        for (uint32_t bx = 0; bx < b.ncx; ++bx) {
          uint32_t x0 = bx * cbw, y0 = by * cbh, bw = std::min(cbw, w - x0), bh = std::min(cbh, h - y0);
          CodeBlockOut cb;
          if (P.classic) {
            if (encode_classic_block(&data[(size_t)y0 * w + x0], w, bw, bh, b.mb, band_class, P.cb_style,
                                     cb.classic) != 0)
              return -3;
          } else if (encode_ht_block(&data[(size_t)y0 * w + x0], w, bw, bh, b.mb, cb.bytes) != 0) {
            return -3;
          }
          b.blocks.push_back(std::move(cb));
        }
      bands[c].push_back(std::move(b));
      return 0;
    };
    if (c == 0)
      for (uint32_t r = 0; r <= L; ++r) {
        res_w[r] = lw[L - r];
        res_h[r] = lhh[L - r];
      }
    if (make_band(cur, cw, ch, 0, ebcot::kLlLh, cb_w(0), cb_h(0)) != 0) return -3;
    for (uint32_t r = 1; r <= L; ++r) {
      uint32_t d = L + 1 - r;  // decomposition level of resolution r
      uint32_t pw = lw[d - 1], ph = lhh[d - 1];
      uint32_t lwd = (pw + 1) / 2, hwd = pw / 2, lhd = (ph + 1) / 2, hhd = ph / 2;
      if (make_band(hl[d], hwd, lhd, 1, ebcot::kHl, cb_w(r), cb_h(r)) != 0) return -3;
      if (make_band(lh[d], lwd, hhd, 1, ebcot::kLlLh, cb_w(r), cb_h(r)) != 0) return -3;
      if (make_band(hh[d], hwd, hhd, 2, ebcot::kHh, cb_w(r), cb_h(r)) != 0) return -3;
    }
  }
  // Packets: one layer, one precinct per resolution.
  std::vector<uint8_t> tile;
  uint32_t sop_seq = 0;
  // Quality layers (classic only): block passes are split evenly over the
  // layers, the bytes of a codeword segment in proportion to its passes
  // (a decoder joins a segment's parts from all layers back together).
  const uint32_t NL = P.classic ? std::max<uint32_t>(P.layers, 1) : 1;
  auto layer_first = [&](uint32_t np, uint32_t l) { return (uint32_t)((uint64_t)np * l / NL); };
  struct Part {
    uint32_t off, len, passes;
  };
  auto layer_parts = [&](const ClassicBlockOut& k, uint32_t l) {
    std::vector<Part> parts;
    const uint32_t a = layer_first(k.passes, l), z = layer_first(k.passes, l + 1);
    uint32_t s0 = 0, o0 = 0;
    for (size_t i = 0; i < k.seg_len.size(); ++i) {
      const uint32_t s1 = s0 + k.seg_passes[i], len = k.seg_len[i];
      const uint32_t pa = std::max(a, s0), pz = std::min(z, s1);
      if (pa < pz) {
        auto at = [&](uint32_t t) { return o0 + (uint32_t)((uint64_t)len * (t - s0) / (s1 - s0)); };
        parts.push_back({at(pa), at(pz) - at(pa), pz - pa});
      }
      s0 = s1;
      o0 += len;
    }
    return parts;
  };
  // Precinct grid of resolution r: npx x npy precincts of 2^PPx x 2^PPy.
  auto n_prec = [&](uint32_t r, bool x) -> uint32_t {
    const uint32_t n = x ? res_w[r] : res_h[r], pp = x ? P.ppx : P.ppy;
    return !precincts ? 1u : (n + (1u << pp) - 1) >> pp;
  };
  auto res_of = [](size_t bi) -> uint32_t { return bi == 0 ? 0u : (uint32_t)((bi - 1) / 3 + 1); };
  // The code blocks of precinct p of a band: block columns [x0, x1) and
  // rows [y0, y1) of the band's block grid.
  struct Range {
    uint32_t x0, x1, y0, y1;
  };
  auto prec_blocks = [&](const Band& b, size_t bi, uint32_t p) -> Range {
    if (!precincts) return {0, b.ncx, 0, b.ncy};
    const uint32_t r = res_of(bi), npx = n_prec(r, true);
    const uint32_t px = p % npx, py = p / npx;
    const uint32_t bpw = 1u << band_pp(P.ppx, r), bph = 1u << band_pp(P.ppy, r);  // band precinct size
    const uint32_t kx = bpw / b.cbw, ky = bph / b.cbh;                              // blocks per precinct side
    return {std::min(px * kx, b.ncx), std::min((px + 1) * kx, b.ncx), std::min(py * ky, b.ncy),
            std::min((py + 1) * ky, b.ncy)};
  };
  // Packet state that lasts over the layers: per (band, precinct) the
  // inclusion (leaf: first layer with passes) and zero-bit-plane tag trees;
  // per block whether it was included and its Lblock.
  struct PrecState {
    std::unique_ptr<TagTree> ti, tz;
  };
  struct BandState {
    std::vector<PrecState> prec;
    std::vector<uint8_t> included;
    std::vector<uint32_t> lblock;
  };
  std::vector<std::vector<BandState>> bstate(C);
  for (uint32_t c = 0; c < C; ++c)
    for (size_t bi = 0; bi < bands[c].size(); ++bi) {
      Band& b = bands[c][bi];
      BandState st;
      const uint32_t r = res_of(bi), np = n_prec(r, true) * n_prec(r, false);
      st.prec.resize(np);
      for (uint32_t p = 0; p < np; ++p) {
        const Range R = prec_blocks(b, bi, p);
        if (R.x1 <= R.x0 || R.y1 <= R.y0) continue;
        std::vector<uint32_t> incl, zbp;
        for (uint32_t y = R.y0; y < R.y1; ++y)
          for (uint32_t x = R.x0; x < R.x1; ++x) {
            const CodeBlockOut& cb = b.blocks[(size_t)y * b.ncx + x];
            uint32_t first = 0xFFFFu;  // never included
            if (!cb.empty()) {
              first = 0;
              if (P.classic)
                while (layer_first(cb.classic.passes, first + 1) == layer_first(cb.classic.passes, first)) ++first;
            }
            incl.push_back(first);
            // Empty leaves are never coded.
            zbp.push_back(cb.empty() ? 0xFFFFu : (P.classic ? cb.classic.zero_planes : b.mb - 1));
          }
        st.prec[p].ti.reset(new TagTree(R.x1 - R.x0, R.y1 - R.y0, incl));
        st.prec[p].tz.reset(new TagTree(R.x1 - R.x0, R.y1 - R.y0, zbp));
      }
      st.included.assign(b.blocks.size(), 0);
      st.lblock.assign(b.blocks.size(), 3);
      bstate[c].push_back(std::move(st));
    }
  auto passes_in = [&](const CodeBlockOut& cb, uint32_t l) -> uint32_t {
    if (cb.empty()) return 0;
    if (!P.classic) return l == 0 ? 1 : 0;
    return layer_first(cb.classic.passes, l + 1) - layer_first(cb.classic.passes, l);
  };
  auto packet = [&](uint32_t c, uint32_t r, uint32_t l, uint32_t p) {
    size_t b0 = r == 0 ? 0 : 1 + (size_t)(r - 1) * 3, nb = r == 0 ? 1 : 3;
    bool any = false;
    for (size_t bi = b0; bi < b0 + nb; ++bi) {
      const Band& b = bands[c][bi];
      const Range R = prec_blocks(b, bi, p);
      for (uint32_t y = R.y0; y < R.y1; ++y)
        for (uint32_t x = R.x0; x < R.x1; ++x) any = any || passes_in(b.blocks[(size_t)y * b.ncx + x], l) > 0;
    }
    if (P.sop_eph) {
      tile.push_back(0xFF); tile.push_back(0x91);
      put16(tile, 4);
      put16(tile, sop_seq++ & 0xFFFF);
    }
    HeaderWriter hw;
    std::vector<std::pair<const uint8_t*, uint32_t>> body;
    if (!any) {
      hw.bit(0);
    } else {
      hw.bit(1);
      for (size_t bi = b0; bi < b0 + nb; ++bi) {
        Band& b = bands[c][bi];
        BandState& st = bstate[c][bi];
        const Range R = prec_blocks(b, bi, p);
        if (R.x1 <= R.x0 || R.y1 <= R.y0) continue;
        PrecState& ps = st.prec[p];
        for (uint32_t y = R.y0; y < R.y1; ++y)
          for (uint32_t x = R.x0; x < R.x1; ++x) {
            const size_t i = (size_t)y * b.ncx + x;
            const auto& cb = b.blocks[i];
            const uint32_t np = passes_in(cb, l);
            if (!st.included[i]) {
              ps.ti->encode(x - R.x0, y - R.y0, l + 1, hw);
              if (np == 0) continue;
              ps.tz->encode(x - R.x0, y - R.y0, UINT32_MAX, hw);
              st.included[i] = 1;
            } else {
              hw.bit(np > 0 ? 1 : 0);
              if (np == 0) continue;
            }
            if (P.classic) {
              // Number of coding passes (Table B.4), Lblock increment, then
              // one length per codeword segment part of Lblock +
              // floor(log2(passes)) bits (B.10.6-B.10.7).
              if (np == 1) hw.bit(0);
              else if (np == 2) hw.bits(0x2, 2);
              else if (np <= 5) hw.bits(0xC | (np - 3), 4);
              else if (np <= 36) { hw.bits(0xF, 4); hw.bits(np - 6, 5); }
              else { hw.bits(0x1FF, 9); hw.bits(np - 37, 7); }
              const std::vector<Part> parts = layer_parts(cb.classic, l);
              uint32_t inc = 0;
              for (const Part& pt : parts) {
                const uint32_t lg = bitlen(pt.passes) - 1, need = bitlen(pt.len);
                if (need > st.lblock[i] + lg) inc = std::max(inc, need - st.lblock[i] - lg);
              }
              for (uint32_t k = 0; k < inc; ++k) hw.bit(1);
              hw.bit(0);
              st.lblock[i] += inc;
              for (const Part& pt : parts) {
                hw.bits(pt.len, st.lblock[i] + bitlen(pt.passes) - 1);
                body.push_back({cb.classic.bytes.data() + pt.off, pt.len});
              }
              continue;
            }
            hw.bit(0);  // one coding pass
            uint32_t len = (uint32_t)cb.bytes.size();
            uint32_t need = bitlen(len);
            uint32_t k = need > 3 ? need - 3 : 0;
            for (uint32_t n = 0; n < k; ++n) hw.bit(1);
            hw.bit(0);
            hw.bits(len, 3 + k);
            body.push_back({cb.bytes.data(), len});
          }
      }
    }
    hw.flush();
    tile.insert(tile.end(), hw.buf.begin(), hw.buf.end());
    if (P.sop_eph) { tile.push_back(0xFF); tile.push_back(0x92); }
    for (auto& part : body) tile.insert(tile.end(), part.first, part.first + part.second);
  };
  // Packet order (B.12.1).  LRCP and RLCP nest layer, resolution,
  // component and precinct (raster order) as named.  The position-driven
  // orders walk the tile's sample grid (y outer, x inner) and take, at each
  // position, the precincts whose top-left corner lies there: with zero
  // image and tile origins and no sub-sampling, precinct (px, py) of
  // resolution r starts at (px, py) * 2^(PP + levels - r) on that grid.
  // RPCL: r, then position, then component; PCRL: position, component, r;
  // CPRL: component, position, r; the layers innermost.
  struct Pk {
    std::array<uint64_t, 5> key;
    uint32_t c, r, l, p;
  };
  std::vector<Pk> order;
  for (uint32_t c = 0; c < C; ++c)
    for (uint32_t r = 0; r <= L; ++r) {
      const uint32_t npx = n_prec(r, true), npy = n_prec(r, false);
      for (uint32_t p = 0; p < npx * npy; ++p) {
        const uint64_t ty = precincts ? (uint64_t)(p / npx) << (P.ppy + L - r) : 0;
        const uint64_t tx = precincts ? (uint64_t)(p % npx) << (P.ppx + L - r) : 0;
        for (uint32_t l = 0; l < NL; ++l) {
          std::array<uint64_t, 5> k{};
          switch (P.progression) {
            case 0: k = {l, r, c, p, 0}; break;
            case 1: k = {r, l, c, p, 0}; break;
            case 2: k = {r, ty, tx, c, l}; break;
            case 3: k = {ty, tx, c, r, l}; break;
            default: k = {c, ty, tx, r, l}; break;
          }
          order.push_back({k, c, r, l, p});
        }
      }
    }
  std::sort(order.begin(), order.end(), [](const Pk& a, const Pk& b) { return a.key < b.key; });
  std::vector<size_t> pkt_end;  // end offset in `tile` of each packet
  for (const Pk& k : order) {
    packet(k.c, k.r, k.l, k.p);
    pkt_end.push_back(tile.size());
  }
  // Tile-parts: the packets in order, cut into nearly equal runs.
  const uint32_t NT = std::max<uint32_t>(1, std::min<uint32_t>(P.tile_parts, (uint32_t)std::max<size_t>(1, order.size())));
  if (NT > 255) return -2;
  std::vector<size_t> part_end(NT);
  for (uint32_t t = 0; t < NT; ++t) {
    const size_t k = (size_t)((uint64_t)order.size() * (t + 1) / NT);
    part_end[t] = k == 0 ? 0 : pkt_end[k - 1];
  }
  part_end[NT - 1] = tile.size();
  // Codestream.
  out.clear();
  out.push_back(0xFF); out.push_back(0x4F);  // SOC
  out.push_back(0xFF); out.push_back(0x51);  // SIZ
  put16(out, 38 + 3 * C);
  put16(out, P.classic ? 0 : 0x4000);  // Rsiz: HTJ2K unless classic
  put32(out, W); put32(out, H); put32(out, 0); put32(out, 0);
  put32(out, W); put32(out, H); put32(out, 0); put32(out, 0);
  put16(out, C);
  for (uint32_t c = 0; c < C; ++c) { out.push_back((uint8_t)(bd - 1)); out.push_back(1); out.push_back(1); }
  if (!P.classic) {
    out.push_back(0xFF); out.push_back(0x50);  // CAP
    put16(out, 8);
    put32(out, 0x00020000);
    uint32_t mbits = bd - 1;
    uint32_t bp = mbits <= 8 ? 0 : (mbits < 28 ? mbits - 8 : 13 + (mbits >> 2));
    put16(out, bp);
  }
  out.push_back(0xFF); out.push_back(0x52);  // COD
  put16(out, 12 + (precincts ? L + 1 : 0));
  out.push_back((P.sop_eph ? 0x06 : 0x00) | (precincts ? 0x01 : 0x00));
  out.push_back((uint8_t)P.progression);
  put16(out, NL);
  out.push_back(mct ? 1 : 0);
  out.push_back((uint8_t)L);
  out.push_back((uint8_t)P.cbw_exp);
  out.push_back((uint8_t)P.cbh_exp);
  out.push_back(P.classic ? (uint8_t)(P.cb_style & 0x3F) : 0x40);  // code-block style
  out.push_back(irr ? 0 : 1);  // wavelet: 0 = 9/7 irreversible, 1 = 5/3 reversible
  if (precincts)
    for (uint32_t r = 0; r <= L; ++r) out.push_back((uint8_t)((P.ppy << 4) | P.ppx));
  out.push_back(0xFF); out.push_back(0x5C);  // QCD
  if (irr) {
    put16(out, 3 + 2 * (1 + 3 * L));
    out.push_back((uint8_t)((guard << 5) | 2));  // scalar expounded
    for (uint32_t k = 0; k < 1 + 3 * L; ++k) put16(out, (q_eps << 11) | q_mu);
  } else {
    put16(out, 3 + 1 + 3 * L);
    out.push_back((uint8_t)(guard << 5));
    out.push_back((uint8_t)(bd << 3));
    for (uint32_t l = 0; l < L; ++l) {
      out.push_back((uint8_t)((bd + 1) << 3));
      out.push_back((uint8_t)((bd + 1) << 3));
      out.push_back((uint8_t)((bd + 2) << 3));
    }
  }
  auto psot = [&](uint32_t t) {
    const size_t b = t == 0 ? 0 : part_end[t - 1];
    return (uint32_t)(12 + 2 + (part_end[t] - b));
  };
  if (P.write_tlm) {
    // One entry per tile-part: Stlm 0x60 = 16-bit Ttlm, 32-bit Ptlm.
    out.push_back(0xFF); out.push_back(0x55);
    put16(out, 4 + 6 * NT);
    out.push_back(0);
    out.push_back(0x60);
    for (uint32_t t = 0; t < NT; ++t) {
      put16(out, 0);
      put32(out, psot(t));
    }
  }
  for (uint32_t t = 0; t < NT; ++t) {
    out.push_back(0xFF); out.push_back(0x90);  // SOT
    put16(out, 10);
    put16(out, 0);
    put32(out, psot(t));
    out.push_back((uint8_t)t);   // TPsot
    out.push_back((uint8_t)NT);  // TNsot
    out.push_back(0xFF); out.push_back(0x93);  // SOD
    const size_t b = t == 0 ? 0 : part_end[t - 1];
    out.insert(out.end(), tile.begin() + (long)b, tile.begin() + (long)part_end[t]);
  }
  out.push_back(0xFF); out.push_back(0xD9);  // EOC
  return 0;
}

}  // namespace enc
}  // namespace sgn
