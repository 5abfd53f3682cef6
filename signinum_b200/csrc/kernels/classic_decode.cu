// Classic JPEG 2000 Tier-1 (EBCOT) code-block decoding on sm_100a.
//
// The arithmetic follows the reference's CPU decoder exactly
// (crates/signinum-j2k-native/src/j2c/arithmetic_decoder.rs: the MQ decoder
// of Annex C with 0xFF past the end of a segment; bitplane.rs: the cleanup,
// significance propagation and magnitude refinement passes of Annex D with
// run-length and uniform contexts, vertically causal contexts, context reset,
// segmentation symbols, termination on every pass and arithmetic-coding
// bypass with raw sign bits).  Coefficients come out as int32 values
// (sign x magnitude, bit 0 the least significant decoded bit-plane), the
// layout the HT kernels write, so the IDWT and pack kernels run unchanged.
//
// Mapping: the MQ decoder is one serial chain per code block, so a thread
// decodes a block.  A persistent grid of threads takes blocks from a device
// counter.  Each thread owns a slot of 16-bit flag words in global scratch,
// one per sample of the block padded by one on every side (low byte: the
// significance of the eight neighbours, as the reference keeps it; high
// byte: significant, refined, coded in this bit-plane, sign); the magnitude
// bits accumulate in place in the coefficient arena.  The probability table,
// the context-label tables and each thread's 19 context states live in
// shared memory.
#include <algorithm>
#include <cstdint>

#include "../device_plan.h"
#include "../ebcot.h"
#include "kernels.h"

namespace sgn {
namespace {

using namespace ebcot;

constexpr int kClassicThreads = 128;
constexpr uint16_t kSigF = 0x8000, kRefF = 0x4000, kCodF = 0x2000, kSgnF = 0x1000;

struct Tables {
  uint32_t qe[47];  // qe | nmps << 16 | nlps << 23 | switch << 30
  uint8_t zc[3][256];
  uint8_t sc[256];  // label | xor << 7
  uint8_t cx[19][kClassicThreads];  // per thread: index | mps << 7
};

struct MqDec {
  const uint8_t* d;
  uint32_t len, bp, c, a, ct;
  __device__ __forceinline__ uint32_t byte_at(uint32_t i) const { return i < len ? (uint32_t)__ldg(d + i) : 0xFFu; }
  __device__ __forceinline__ void bytein() {
    if (byte_at(bp) == 0xFF) {
      if (byte_at(bp + 1) > 0x8F) {
        ct = 8;
      } else {
        ++bp;
        c = c + 0xFE00u - (byte_at(bp) << 9);
        ct = 7;
      }
    } else {
      ++bp;
      c = c + 0xFF00u - (byte_at(bp) << 8);
      ct = 8;
    }
  }
  __device__ __forceinline__ void init(const uint8_t* data, uint32_t n) {
    d = data;
    len = n;
    bp = 0;
    c = (byte_at(0) ^ 0xFFu) << 16;
    bytein();
    c <<= 7;
    ct -= 7;
    a = 0x8000;
  }
  __device__ __forceinline__ uint32_t decode(uint8_t& cx, const uint32_t* qe) {
    const uint32_t e = qe[cx & 0x7F];
    const uint32_t q = e & 0xFFFF, mps = cx >> 7;
    a -= q;
    uint32_t dbit;
    if ((c >> 16) < a) {
      if (a & 0x8000) return mps;
      if (a < q) {  // MPS exchange
        dbit = 1 - mps;
        cx = (uint8_t)((((e >> 23) & 0x7F)) | ((mps ^ ((e >> 30) & 1)) << 7));
      } else {
        dbit = mps;
        cx = (uint8_t)(((e >> 16) & 0x7F) | (mps << 7));
      }
    } else {
      c -= a << 16;
      if (a < q) {  // LPS exchange
        a = q;
        dbit = mps;
        cx = (uint8_t)(((e >> 16) & 0x7F) | (mps << 7));
      } else {
        a = q;
        dbit = 1 - mps;
        cx = (uint8_t)(((e >> 23) & 0x7F) | ((mps ^ ((e >> 30) & 1)) << 7));
      }
    }
    // RENORMD (C.3.3), shifting as many bits at once as A needs and the
    // byte buffer holds (as the reference's renormalize does).
    while ((a & 0x8000) == 0) {
      if (ct == 0) bytein();
      const uint32_t sh = min((uint32_t)__clz(a) - 16, ct);
      a <<= sh;
      c <<= sh;
      ct -= sh;
    }
    return dbit;
  }
};

// Raw bits of a bypassed segment: packet-header stuffing; 1 past the end or on
// a bad stuff bit (the reference's non-strict BypassDecoder).
struct RawDec {
  const uint8_t* d;
  uint32_t len, cur;
  __device__ __forceinline__ bool bit(uint32_t& b) {
    if ((cur >> 3) >= len) return false;
    b = (__ldg(d + (cur >> 3)) >> (7 - (cur & 7))) & 1;
    ++cur;
    return true;
  }
  __device__ __forceinline__ uint32_t decode(uint8_t&, const uint32_t*) {
    const bool stuff = (cur & 7) == 7 && (cur >> 3) < len && __ldg(d + (cur >> 3)) == 0xFF;
    uint32_t b;
    if (!bit(b)) return 1;
    if (stuff) {
      uint32_t s;
      if (!bit(s) || s != 0) return 1;
    }
    return b;
  }
};

struct Block {
  uint16_t* f;    // flag words, (w + 2) x (h + 2)
  uint32_t* out;  // coefficients, row stride `stride`
  uint32_t w, h, pw, stride, pos;
  uint8_t band, style;
  Tables* t;
  int tid;
  __device__ __forceinline__ uint8_t& cx(int label) { return t->cx[label][tid]; }
  __device__ __forceinline__ uint32_t fi(uint32_t x, uint32_t y) const { return (y + 1) * pw + x + 1; }
  __device__ __forceinline__ uint32_t& co(uint32_t x, uint32_t y) { return out[(size_t)y * stride + x]; }
  __device__ __forceinline__ bool next_stripe(uint32_t y) const { return y + 1 < h && ((y + 1) >> 2) > (y >> 2); }
  __device__ __forceinline__ uint8_t nbr(uint32_t i, uint32_t y) const {
    const uint8_t n = (uint8_t)f[i];
    return ((style & kVCausal) && next_stripe(y)) ? (uint8_t)(n & 0xF4) : n;
  }
  __device__ __forceinline__ void set_significant(uint32_t i) {
    f[i] |= kSigF;
    f[i - pw - 1] |= 1 << 1;
    f[i - pw] |= 1 << 0;
    f[i - pw + 1] |= 1 << 3;
    f[i - 1] |= 1 << 2;
    f[i + 1] |= 1 << 4;
    f[i + pw - 1] |= 1 << 5;
    f[i + pw] |= 1 << 6;
    f[i + pw + 1] |= 1 << 7;
  }
  __device__ __forceinline__ uint32_t sgn(uint32_t i) const { return (f[i] >> 12) & 1; }
  template <typename D>
  __device__ __forceinline__ void decode_sign(uint32_t i, uint32_t x, uint32_t y, D& dec, bool raw) {
    const uint8_t s = nbr(i, y) & 0x55;
    const uint32_t bottom = ((style & kVCausal) && next_stripe(y)) ? 0 : sgn(i + pw);
    const uint32_t signs = (sgn(i - pw) << 6) | (sgn(i - 1) << 4) | (sgn(i + 1) << 2) | bottom;
    const uint8_t e = t->sc[(uint8_t)(((s & signs) << 1) | (s & ~signs))];
    uint32_t b = dec.decode(cx(e & 0x7F), t->qe);
    if (!raw) b ^= e >> 7;
    if (b) {
      f[i] |= kSgnF;
      co(x, y) |= 0x80000000u;
    }
  }
  template <typename D>
  __device__ __forceinline__ void cleanup_one(uint32_t x, uint32_t y, D& dec, bool raw) {
    const uint32_t i = fi(x, y);
    if (f[i] & (kSigF | kCodF)) return;
    const uint32_t b = dec.decode(cx(t->zc[band][nbr(i, y)]), t->qe);
    if (b) {
      co(x, y) |= 1u << pos;
      decode_sign(i, x, y, dec, raw);
      set_significant(i);
    }
  }
  template <typename D>
  __device__ void cleanup(D& dec, bool raw) {
    for (uint32_t by = 0; by < h; by += 4) {
      const uint32_t ye = min(by + 4, h);
      for (uint32_t x = 0; x < w; ++x) {
        bool run = ye - by == 4;
        for (uint32_t y = by; run && y < ye; ++y) {
          const uint32_t i = fi(x, y);
          run = !(f[i] & (kSigF | kCodF)) && nbr(i, y) == 0;
        }
        if (run) {
          if (dec.decode(cx(17), t->qe) == 0) continue;
          uint32_t k = dec.decode(cx(18), t->qe) << 1;
          k |= dec.decode(cx(18), t->qe);
          const uint32_t sy = by + k, i = fi(x, sy);
          co(x, sy) |= 1u << pos;
          decode_sign(i, x, sy, dec, raw);
          set_significant(i);
          for (uint32_t y = sy + 1; y < ye; ++y) cleanup_one(x, y, dec, raw);
          continue;
        }
        for (uint32_t y = by; y < ye; ++y) cleanup_one(x, y, dec, raw);
      }
    }
  }
  template <typename D>
  __device__ void sig_prop(D& dec, bool raw) {
    for (uint32_t by = 0; by < h; by += 4) {
      const uint32_t ye = min(by + 4, h);
      for (uint32_t x = 0; x < w; ++x)
        for (uint32_t y = by; y < ye; ++y) {
          const uint32_t i = fi(x, y);
          const uint8_t n = nbr(i, y);
          if ((f[i] & kSigF) || n == 0) continue;
          const uint32_t b = dec.decode(cx(t->zc[band][n]), t->qe);
          f[i] |= kCodF;
          if (b) {
            co(x, y) |= 1u << pos;
            decode_sign(i, x, y, dec, raw);
            set_significant(i);
          }
        }
    }
  }
  template <typename D>
  __device__ void mag_ref(D& dec) {
    for (uint32_t by = 0; by < h; by += 4) {
      const uint32_t ye = min(by + 4, h);
      for (uint32_t x = 0; x < w; ++x)
        for (uint32_t y = by; y < ye; ++y) {
          const uint32_t i = fi(x, y);
          const uint16_t fl = f[i];
          if (!(fl & kSigF) || (fl & kCodF)) continue;
          const uint32_t b = dec.decode(cx(mr_context((fl & kRefF) != 0, nbr(i, y))), t->qe);
          co(x, y) |= b << pos;
          f[i] |= kRefF;
        }
    }
  }
  __device__ void reset_contexts() {
    for (int k = 0; k < 19; ++k) cx(k) = initial_index(k);
  }
  template <typename D>
  __device__ void passes(uint32_t start, uint32_t end, uint32_t bitplanes, D& dec, bool raw) {
    for (uint32_t p = start; p < end; ++p) {
      pos = bitplanes - 1 - (p + 2) / 3;
      const uint32_t kind = p % 3;
      if (kind == 0) {
        cleanup(dec, raw);
        if (style & kSegSym)
          for (int k = 0; k < 4; ++k) dec.decode(cx(18), t->qe);
        for (uint32_t y = 0; y < h; ++y)
          for (uint32_t x = 0; x < w; ++x) f[fi(x, y)] &= (uint16_t)~kCodF;
      } else if (kind == 1) {
        sig_prop(dec, raw);
      } else {
        mag_ref(dec);
      }
      if (style & kReset) reset_contexts();
    }
  }
};

// Blocks of at most 64 x 64 samples: per row four 64-bit planes (bit x =
// column x) in the thread's scratch slot, rows -1 .. h+3 with zero padding:
// significant, sign, refined, coded in this bit-plane.  A pass walks the
// stripes; the six rows around a stripe live in registers while its columns
// are scanned (the neighbour-significance byte of a sample is assembled from
// three-bit windows of the rows above, at and below it), and the four rows
// of the stripe go back at its end.  Magnitude and sign bits are OR-ed into
// the coefficient words with reductions that nothing waits on.
constexpr uint32_t kSmallRows = 64 + 5;
static_assert(4 * kSmallRows * 4 == 1104, "small-block slot of classic_slot_words");

struct Small {
  uint64_t* P;  // sig, sgn, ref, cod planes of kSmallRows rows; row y at y + 1
  uint32_t* out;
  uint32_t w, h, stride, pos;
  uint8_t band, style;
  Tables* t;
  int tid;
  __device__ __forceinline__ uint8_t& cx(int label) { return t->cx[label][tid]; }
  __device__ __forceinline__ uint64_t* plane(int k) { return P + k * kSmallRows; }
  // Bits x-1, x, x+1 of a row (columns outside the block read 0).
  __device__ static __forceinline__ uint32_t w3(uint64_t r, uint32_t x) {
    return (uint32_t)(x ? (r >> (x - 1)) : (r << 1)) & 7u;
  }
  __device__ static __forceinline__ uint32_t bit_at(uint64_t r, uint32_t x) { return (uint32_t)(r >> x) & 1u; }
  __device__ __forceinline__ void reset_contexts() {
    for (int k = 0; k < 19; ++k) cx(k) = initial_index(k);
  }

  template <int KIND, typename D>
  __device__ void pass(D& dec, bool raw) {
    uint64_t* S = plane(0);
    uint64_t* G = plane(1);
    uint64_t* R = plane(2);
    uint64_t* C = plane(3);
    const bool vcausal = style & kVCausal;
    for (uint32_t y0 = 0; y0 < h; y0 += 4) {
      const uint32_t nr = min(4u, h - y0);
      uint64_t s[6], g[6], c[4], r[4];
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        s[k] = S[y0 + k];
        g[k] = G[y0 + k];
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        c[k] = C[y0 + 1 + k];
        r[k] = R[y0 + 1 + k];
      }
      // Vertically causal: the stripe's last row ignores the row below it.
      const bool cut = vcausal && y0 + 4 < h;
      for (uint32_t x = 0; x < w; ++x) {
        const uint64_t bx = 1ull << x;
        auto nbr = [&](int k) -> uint32_t {
          const uint32_t u = w3(s[k], x), m = w3(s[k + 1], x), d = (cut && k == 3) ? 0u : w3(s[k + 2], x);
          return ((u & 1) << 7) | ((u & 2) << 5) | ((u & 4) << 3) | ((m & 1) << 4) | ((d & 1) << 3) | (m & 4) |
                 ((d & 4) >> 1) | ((d & 2) >> 1);
        };
        auto sign = [&](int k, uint32_t n) {
          const uint32_t sg = n & 0x55;
          const uint32_t top = bit_at(g[k], x), left = x ? bit_at(g[k + 1], x - 1) : 0u;
          const uint32_t right = x < 63 ? bit_at(g[k + 1], x + 1) : 0u;
          const uint32_t bottom = (cut && k == 3) ? 0u : bit_at(g[k + 2], x);
          const uint32_t signs = (top << 6) | (left << 4) | (right << 2) | bottom;
          const uint8_t e = t->sc[(uint8_t)(((sg & signs) << 1) | (sg & ~signs))];
          uint32_t b = dec.decode(cx(e & 0x7F), t->qe);
          if (!raw) b ^= e >> 7;
          return b;
        };
        uint32_t* col = out + (size_t)y0 * stride + x;
        // A sample turning significant: its magnitude bit, sign, and state.
        auto significant = [&](int k, uint32_t n) {
          const uint32_t sb = sign(k, n);
          atomicOr(col + (size_t)k * stride, (1u << pos) | (sb << 31));
          s[k + 1] |= bx;
          if (sb) g[k + 1] |= bx;
        };
        if (KIND == 0) {
          int first = 0;
          if (nr == 4) {
            bool run = true;
#pragma unroll
            for (int k = 0; k < 4; ++k) run = run && !((s[k + 1] | c[k]) & bx) && nbr(k) == 0;
            if (run) {
              if (dec.decode(cx(17), t->qe) == 0) continue;
              uint32_t f = dec.decode(cx(18), t->qe) << 1;
              f |= dec.decode(cx(18), t->qe);
#pragma unroll
              for (int k = 0; k < 4; ++k)
                if ((uint32_t)k == f) significant(k, nbr(k));
              first = (int)f + 1;
            }
          }
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            if (k < first || (uint32_t)k >= nr || ((s[k + 1] | c[k]) & bx)) continue;
            const uint32_t n = nbr(k);
            if (dec.decode(cx(t->zc[band][n]), t->qe)) significant(k, n);
          }
        } else if (KIND == 1) {
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            if ((uint32_t)k >= nr || (s[k + 1] & bx)) continue;
            const uint32_t n = nbr(k);
            if (n == 0) continue;
            c[k] |= bx;
            if (dec.decode(cx(t->zc[band][n]), t->qe)) significant(k, n);
          }
        } else {
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            if ((uint32_t)k >= nr || !(s[k + 1] & bx) || (c[k] & bx)) continue;
            const uint32_t b = dec.decode(cx(mr_context((r[k] & bx) != 0, nbr(k))), t->qe);
            if (b) atomicOr(col + (size_t)k * stride, 1u << pos);
            r[k] |= bx;
          }
        }
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if ((uint32_t)k >= nr) continue;
        S[y0 + 1 + k] = s[k + 1];
        G[y0 + 1 + k] = g[k + 1];
        R[y0 + 1 + k] = r[k];
        C[y0 + 1 + k] = KIND == 0 ? 0ull : c[k];  // the cleanup pass ends the bit-plane
      }
    }
  }

  template <typename D>
  __device__ void passes(uint32_t start, uint32_t end, uint32_t bitplanes, D& dec, bool raw) {
    for (uint32_t p = start; p < end; ++p) {
      pos = bitplanes - 1 - (p + 2) / 3;
      const uint32_t kind = p % 3;
      if (kind == 0) {
        pass<0>(dec, raw);
        if (style & kSegSym)
          for (int k = 0; k < 4; ++k) dec.decode(cx(18), t->qe);
      } else if (kind == 1) {
        pass<1>(dec, raw);
      } else {
        pass<2>(dec, raw);
      }
      if (style & kReset) reset_contexts();
    }
  }
};

__device__ void decode_general(const ClassicJob& job, const ClassicSeg* __restrict__ segs, const uint8_t* data,
                               uint32_t* out, uint16_t* slot, Tables* t);

template <typename B>
__device__ __forceinline__ void run_passes(B& b, const ClassicJob& job, const ClassicSeg* __restrict__ segs,
                                           const uint8_t* data) {
  const uint32_t max_passes = 1 + 3 * ((uint32_t)job.bitplanes - 1);
  if (!(job.style & (kBypass | kTermAll))) {
    uint32_t total = 0;
    for (uint32_t k = 0; k < job.nseg; ++k) total += segs[job.seg + k].len;
    MqDec dec;
    dec.init(data, total);
    b.passes(0, min((uint32_t)job.passes, max_passes), job.bitplanes, dec, false);
    return;
  }
  uint32_t start = 0, off = 0;
  for (uint32_t k = 0; k < job.nseg; ++k) {
    const ClassicSeg s = segs[job.seg + k];
    const uint32_t end = min(start + s.passes, max_passes);
    if (segment_is_arithmetic(job.style, start)) {
      MqDec dec;
      dec.init(data + off, s.len);
      b.passes(start, end, job.bitplanes, dec, false);
    } else {
      RawDec dec{data + off, s.len, 0};
      b.passes(start, end, job.bitplanes, dec, true);
    }
    start += s.passes;
    off += s.len;
  }
}

__device__ void decode_block(const ClassicJob& job, const ClassicSeg* __restrict__ segs,
                             const uint8_t* __restrict__ input, const uint8_t* __restrict__ gather,
                             int32_t* __restrict__ coef, uint16_t* slot, Tables* t) {
  const uint32_t w = job.w, h = job.h, stride = job.stride;
  // The block's segments, in the input or (multi-layer) in the gather area.
  const uint8_t* data =
      (job.src & kClassicGathered) ? gather + (job.src & ~kClassicGathered) : input + job.src;
  uint32_t* out = reinterpret_cast<uint32_t*>(coef + job.dst);
  for (uint32_t y = 0; y < h; ++y)
    for (uint32_t x = 0; x < w; ++x) out[(size_t)y * stride + x] = 0;
  if (job.passes == 0 || job.bitplanes == 0) return;
  if (w <= 64 && h <= 64) {
    Small b;
    b.P = reinterpret_cast<uint64_t*>(slot);
    b.out = out;
    b.w = w;
    b.h = h;
    b.stride = stride;
    b.pos = 0;
    b.band = job.band_class;
    b.style = job.style;
    b.t = t;
    b.tid = threadIdx.x;
    for (uint32_t i = 0; i < 4 * kSmallRows; ++i) b.P[i] = 0;
    b.reset_contexts();
    run_passes(b, job, segs, data);
  } else {
    decode_general(job, segs, data, out, slot, t);
  }
  // The magnitude and sign bits arrived by reductions in L2: read them there.
  for (uint32_t y = 0; y < h; ++y)
    for (uint32_t x = 0; x < w; ++x) {
      const uint32_t v = __ldcg(out + (size_t)y * stride + x);
      const int32_t m = (int32_t)(v & 0x7FFFFFFFu);
      out[(size_t)y * stride + x] = (uint32_t)((v >> 31) ? -m : m);
    }
}

// Blocks wider or taller than 64: one 16-bit flag word per padded sample.
__device__ void decode_general(const ClassicJob& job, const ClassicSeg* __restrict__ segs, const uint8_t* data,
                               uint32_t* out, uint16_t* slot, Tables* t) {
  const uint32_t w = job.w, h = job.h, stride = job.stride;
  Block b;
  b.f = slot;
  b.out = out;
  b.w = w;
  b.h = h;
  b.pw = w + 2;
  b.stride = stride;
  b.pos = 0;
  b.band = job.band_class;
  b.style = job.style;
  b.t = t;
  b.tid = threadIdx.x;
  for (uint32_t i = 0; i < (w + 2) * (h + 2); ++i) slot[i] = 0;
  b.reset_contexts();
  run_passes(b, job, segs, data);
}

}  // namespace

// Table C.2 packed per index: qe | nmps << 16 | nlps << 23 | switch << 30
// (built on the host from ebcot.h and passed by value).
struct QeTable {
  uint32_t e[47];
};

__global__ void __launch_bounds__(kClassicThreads) classic_kernel(const ClassicJob* __restrict__ jobs,
                                                                  const ClassicSeg* __restrict__ segs, uint32_t njobs,
                                                                  const uint8_t* __restrict__ arena,
                                                                  const uint8_t* __restrict__ gather,
                                                                  int32_t* __restrict__ coef, uint16_t* scratch,
                                                                  uint32_t slot_words, uint32_t* queue, QeTable qt) {
  __shared__ Tables t;
  for (int i = threadIdx.x; i < 47; i += blockDim.x) t.qe[i] = qt.e[i];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) {
    t.zc[0][i] = zc_context((uint8_t)i, kLlLh);
    t.zc[1][i] = zc_context((uint8_t)i, kHl);
    t.zc[2][i] = zc_context((uint8_t)i, kHh);
    uint8_t label, xr;
    sc_context((uint8_t)i, label, xr);
    t.sc[i] = (uint8_t)(label | (xr << 7));
  }
  __syncthreads();
  uint16_t* slot = scratch + ((size_t)blockIdx.x * blockDim.x + threadIdx.x) * slot_words;
  for (;;) {
    const uint32_t j = atomicAdd(queue, 1u);
    if (j >= njobs) break;
    decode_block(jobs[j], segs, arena, gather, coef, slot, &t);
  }
}

cudaError_t launch_classic(const ClassicJob* jobs, const ClassicSeg* segs, uint32_t njobs, const uint8_t* arena,
                           const uint8_t* gather, int32_t* coef, uint16_t* scratch, uint32_t slot_words, uint32_t ctas,
                           uint32_t* queue, cudaStream_t stream) {
  if (njobs == 0) return cudaSuccess;
  if (!scratch || !queue || ctas == 0) return cudaErrorInvalidValue;
  QeTable qt;
  for (int i = 0; i < 47; ++i)
    qt.e[i] = kQe[i] | ((uint32_t)kNmps[i] << 16) | ((uint32_t)kNlps[i] << 23) | ((uint32_t)kSwitch[i] << 30);
  classic_kernel<<<ctas, kClassicThreads, 0, stream>>>(jobs, segs, njobs, arena, gather, coef, scratch, slot_words,
                                                       queue, qt);
  return cudaGetLastError();
}

uint32_t classic_threads_per_cta() { return kClassicThreads; }

uint32_t classic_ctas_per_sm() {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, classic_kernel, kClassicThreads, 0) != cudaSuccess || n < 1)
    n = 1;
  return (uint32_t)n;
}

}  // namespace sgn
