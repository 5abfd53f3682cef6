// HT code-block decoding on sm_100a.
//
// Decodes HTJ2K code blocks (T.814) into sign-magnitude coefficients and
// writes them as int32 sub-band samples, bit-exact with the reference's
// decode_impl (crates/signinum-j2k-native/src/j2c/ht_block_decode.rs:1563-1683)
// followed by coefficient_to_i32 (:225-234).
//
// Work mapping, in two passes over the blocks of a launch (ordered by coded
// length on the host, so neighbouring blocks carry similar work):
//  1. ht_vlc_kernel: one lane per code block runs the MEL / CxtVLC / UVLC
//     chain, the only inherently serial part of the cleanup pass, and writes
//     one 32-bit symbol per quad to a scratch table;
//  2. ht_magsgn_kernel: one warp per code block decodes magnitudes and signs,
//     a quad per lane, with a warp prefix scan of per-quad bit counts over the
//     block's unstuffed MagSgn stream staged in shared memory, and writes
//     whole rows with coalesced stores; blocks at most 32 wide without
//     refinement passes go two per warp, one per half-warp.
// Plans of few blocks run both passes in ht_cleanup_fused_kernel instead: a
// CTA per block, whose MagSgn warp follows the block's VLC chain row by row.
// Refinement passes (SigProp/MagRef) run in ht_refine_kernel for the few
// blocks that carry them.
#include <algorithm>
#include <cstdint>

#include "../device_plan.h"
#include "../ht_tables.h"
#include "kernels.h"

namespace sgn {

__device__ HtDecodeTables g_ht_tables;

namespace {

constexpr int kHtThreads = 128;
constexpr uint32_t kStatusDecode = 1u;

struct SmemTables {
  uint16_t vlc0[1024];
  uint16_t vlc1[1024];
  uint16_t uvlc0[320];
  uint16_t uvlc1[256];
};

__device__ __forceinline__ uint8_t ld8(const uint8_t* p) { return __ldg(p); }

// MEL bit-buffer refill, out of line (it runs once every several runs, and
// inlined its byte loop would sit in every step of the VLC chain): appends
// bytes until more than 56 bits are buffered.  After a 0xFF byte the next
// byte carries 7 bits; the last byte is ORed with 0x0F and the stream
// continues with 0xFF bytes.  State passed and returned by value, so it
// stays in registers.
struct MelFill {
  uint64_t buf;
  uint32_t pos, remaining, unstuff;
  int bits;
};
// The out-of-line refill loop.  While 32 bits or fewer are buffered, four
// bytes that are not the segment's last, after a byte that is not 0xFF and
// with no 0xFF among their first three (each then carries 8 bits) go in as
// one word from four independent loads; other bytes one at a time.  (The
// inline form keeps the byte loop alone: the word step measured slower
// inlined in the chain.)
__device__ __forceinline__ void mel_fill(const uint8_t* data, MelFill& f) {
  while (f.bits <= 56) {
    if (f.bits <= 32 && f.remaining >= 5 && !f.unstuff) {
      const uint8_t* p = data + f.pos;
      const uint32_t b0 = __ldg(p), b1 = __ldg(p + 1), b2 = __ldg(p + 2), b3 = __ldg(p + 3);
      if (b0 != 0xFF && b1 != 0xFF && b2 != 0xFF) {
        f.buf |= (uint64_t)((b0 << 24) | (b1 << 16) | (b2 << 8) | b3) << (32 - f.bits);
        f.bits += 32;
        f.pos += 4;
        f.remaining -= 4;
        f.unstuff = b3 == 0xFF;
        continue;
      }
    }
    uint32_t b;
    if (f.remaining > 0) {
      b = __ldg(data + f.pos);
      ++f.pos;
      --f.remaining;
    } else {
      b = 0xFF;
    }
    if (f.remaining == 0) b |= 0x0F;
    const int nb = 8 - (int)f.unstuff;
    f.buf |= (uint64_t)(b & ((1u << nb) - 1)) << (64 - f.bits - nb);
    f.bits += nb;
    f.unstuff = b == 0xFF;
  }
}
__device__ __noinline__ MelFill mel_refill(const uint8_t* data, MelFill f) {
  mel_fill(data, f);
  return f;
}

// MEL run decoder (ht_block_decode.rs:782-880).  The reference decodes runs
// into a small queue; here each run is decoded when it is needed, from a
// 64-bit buffer of unstuffed MEL bits (most significant bit first), with no
// inner loop: lanes of a warp decode different blocks, so a short fixed
// sequence per run diverges far less than a queue refill.
template <bool OUTLINE>
struct MelT {
  const uint8_t* data;
  uint32_t pos, remaining, unstuff;
  uint64_t buf;  // unread bits, left-aligned
  int bits, k;
  __device__ void init(const uint8_t* d, uint32_t lcup, uint32_t scup) {
    data = d;
    pos = lcup - scup;
    remaining = scup - 1;
    unstuff = 0;
    buf = 0;
    bits = 0;
    k = 0;
  }
  // OUTLINE: the refill is the out-of-line mel_refill; otherwise its loop
  // is inlined (which is faster depends on the batch: the autotuner picks).
  __device__ __forceinline__ void refill() {
    if constexpr (OUTLINE) {
      const MelFill f = mel_refill(data, MelFill{buf, pos, remaining, unstuff, bits});
      buf = f.buf;
      pos = f.pos;
      remaining = f.remaining;
      unstuff = f.unstuff;
      bits = f.bits;
    } else {
      while (bits <= 56) {
        uint32_t b;
        if (remaining > 0) {
          b = ld8(data + pos);
          ++pos;
          --remaining;
        } else {
          b = 0xFF;
        }
        if (remaining == 0) b |= 0x0F;
        const int nb = 8 - (int)unstuff;
        buf |= (uint64_t)(b & ((1u << nb) - 1)) << (64 - bits - nb);
        bits += nb;
        unstuff = b == 0xFF;
      }
    }
  }
  __device__ __forceinline__ int get_run() {
    if (bits < 6) refill();
    // MEL exponent table {0,0,0,1,1,1,2,2,2,3,3,4,5}, 3 bits per state.
    constexpr uint64_t kExp = (0ull << 0) | (0ull << 3) | (0ull << 6) | (1ull << 9) | (1ull << 12) | (1ull << 15) |
                              (2ull << 18) | (2ull << 21) | (2ull << 24) | (3ull << 27) | (3ull << 30) |
                              (4ull << 33) | (5ull << 36);
    const int e = (int)((kExp >> (3 * k)) & 7);
    const bool first = (buf >> 63) != 0;
    const uint32_t v = e ? (uint32_t)((buf << 1) >> (64 - e)) : 0u;
    const int used = first ? 1 : 1 + e;
    k = first ? min(k + 1, 12) : max(k - 1, 0);
    buf <<= used;
    bits -= used;
    return first ? ((1 << e) - 1) << 1 : (int)((v << 1) | 1);
  }
};

// Four bytes (highest address first) into the backward VLC reader's bit
// buffer one at a time, for words with a byte whose low 7 bits are all ones
// (after a byte above 0x8F such a byte loses its top bit to stuffing).  Out
// of line: it is the rare case of a refill.
struct VlcPush {
  uint64_t tmp;
  uint32_t bits, unstuff;
};
__device__ __noinline__ VlcPush vlc_push4(uint32_t wv, uint64_t tmp, uint32_t bits, uint32_t unstuff) {
#pragma unroll
  for (int k = 3; k >= 0; --k) {
    const uint32_t b = (wv >> (8 * k)) & 0xFF;
    const uint32_t db = 8 - ((unstuff && (b & 0x7F) == 0x7F) ? 1 : 0);
    tmp |= (uint64_t)b << bits;
    bits += db;
    unstuff = b > 0x8F;
  }
  return VlcPush{tmp, bits, unstuff};
}

// Backward VLC reader (ht_block_decode.rs:932-1000, new_vlc).
template <bool OUTLINE>
struct VlcT {
  const uint8_t* data;
  int pos;
  uint32_t remaining;
  uint64_t tmp;
  uint32_t bits, unstuff;
  // Word refills walk down 4 bytes at a time, so their two aligned words
  // are the previous refill's low word and the word below it: that one is
  // loaded a refill ahead (w_lo) and the refill itself never waits on memory.
  const uint32_t* wp;  // aligned word of the next refill's low half
  uint32_t w_lo, w_hi, sh8;
  __device__ void init(const uint8_t* d, uint32_t lcup, uint32_t scup) {
    data = d;
    uint32_t b = ld8(d + lcup - 2);
    tmp = b >> 4;
    bits = 4 - (((tmp & 7) == 7) ? 1 : 0);
    pos = (int)lcup - 3;
    remaining = scup - 2;
    unstuff = (b | 0x0F) > 0x8F;
    init_words();
  }
  // The MagRef reader (new_mrp, ht_block_decode.rs:1377-1433): the whole
  // refinement segment of n bytes from its last byte down, stuffing from the
  // start.
  __device__ void init_mrp(const uint8_t* d, uint32_t n) {
    data = d;
    tmp = 0;
    bits = 0;
    pos = (int)n - 1;
    remaining = n;
    unstuff = 1;
    init_words();
  }
  // Word-refill state for bytes pos - 3 .. pos; every initialiser calls it.
  __device__ __forceinline__ void init_words() {
    w_lo = w_hi = 0;
    wp = nullptr;
    sh8 = 0;
    if (remaining >= 4) {
      // Both words hold bytes of the segment (pos - 3 .. pos).
      const uintptr_t addr = (uintptr_t)(data + pos - 3);
      wp = reinterpret_cast<const uint32_t*>(addr & ~(uintptr_t)3);
      sh8 = (uint32_t)(addr & 3) * 8;
      w_lo = __ldg(wp);
      w_hi = sh8 ? __ldg(wp + 1) : 0u;
    }
  }
  __device__ __forceinline__ void push(uint32_t b) {
    const uint32_t db = 8 - ((unstuff && (b & 0x7F) == 0x7F) ? 1 : 0);
    tmp |= (uint64_t)b << bits;
    bits += db;
    unstuff = b > 0x8F;
  }
  // Appends bytes (walking backwards) until more than 32 bits are buffered;
  // past the segment the reader supplies zero bytes.  Four bytes at a time
  // come from one unaligned 32-bit read (two aligned loads inside the
  // segment), so the byte steps do not wait on one load each.
  __device__ __forceinline__ void fill() {
    while (bits <= 32) {
      if (remaining >= 4) {
        const uint32_t wv = __funnelshift_r(w_lo, w_hi, sh8);
        w_hi = w_lo;
        --wp;
        // The next word refill (when 4 more bytes remain) reads bytes down to
        // pos - 7, all inside the segment, so its low word is one of them.
        w_lo = remaining >= 8 ? __ldg(wp) : 0u;
        pos -= 4;
        remaining -= 4;
        if (__vcmpeq4(wv | 0x80808080u, 0xFFFFFFFFu) == 0) {
          // No byte has its low 7 bits all ones, so none loses a bit to
          // stuffing: the four bytes (highest address first) go in whole.
          tmp |= (uint64_t)__byte_perm(wv, 0, 0x0123) << bits;
          bits += 32;
          unstuff = (wv & 0xFF) > 0x8F;
        } else if constexpr (OUTLINE) {
          const VlcPush r = vlc_push4(wv, tmp, bits, unstuff);
          tmp = r.tmp;
          bits = r.bits;
          unstuff = r.unstuff;
        } else {
          push(wv >> 24);
          push((wv >> 16) & 0xFF);
          push((wv >> 8) & 0xFF);
          push(wv & 0xFF);
        }
      } else {
        uint32_t b = 0;
        if (remaining > 0) {
          b = ld8(data + pos);
          --pos;
          --remaining;
        }
        push(b);
      }
    }
  }
  __device__ __forceinline__ uint32_t fetch() {
    if (bits < 32) fill();
    return (uint32_t)tmp;
  }
  __device__ __forceinline__ uint32_t advance(uint32_t n) {
    tmp >>= n;
    bits -= n;
    return (uint32_t)tmp;
  }
};

// The refinement passes use the out-of-line forms.
using Mel = MelT<true>;
using Vlc = VlcT<true>;

// Forward reader with 0xFF stuffing (ht_block_decode.rs:888-930).
template <uint32_t PAD>
struct Fwd {
  const uint8_t* data;
  uint32_t len, pos;
  uint64_t tmp;
  uint32_t bits, unstuff;
  __device__ void init(const uint8_t* d, uint32_t n) {
    data = d;
    len = n;
    pos = 0;
    tmp = 0;
    bits = 0;
    unstuff = 0;
  }
  __device__ __forceinline__ void fill() {
    while (bits <= 32) {
      uint32_t b = pos < len ? (uint32_t)ld8(data + pos) : PAD;
      ++pos;
      tmp |= (uint64_t)b << bits;
      bits += 8 - unstuff;
      unstuff = b == 0xFF;
    }
  }
  __device__ __forceinline__ uint32_t fetch() {
    if (bits < 32) fill();
    return (uint32_t)tmp;
  }
  __device__ __forceinline__ void advance(uint32_t n) {
    tmp >>= n;
    bits -= n;
  }
};

__device__ __forceinline__ int32_t to_i32(uint32_t v, uint32_t nbp) {
  uint32_t shift = nbp >= 31 ? 0 : 31 - nbp;
  int32_t m = (int32_t)((v & 0x7FFFFFFFu) >> shift);
  return (v & 0x80000000u) ? -m : m;
}

// Row-above context of blocks at most 64 wide (REG): the significance of
// the two bottom samples of each quad (entry bits 5 and 7, the only part of
// a quad the row below takes its context from) in one 64-bit mask S, four
// bits per quad pair k at bits 4k .. 4k+3: {first quad's bit 5, second
// quad's bit 5, first quad's bit 7, second quad's bit 7}.  In that order a
// quad's two context bits from above (entry bits 7 and 9 of c_q: the left
// quad's bit 7 or its own bit 5; its own bit 7 or the right quad's bit 5)
// are ORs of adjacent bits of S: with Q = S | S >> 1, quad 2k takes
// Q[4k-1] and Q[4k+1], quad 2k+1 Q[4k+1] and Q[4k+3].
__device__ __forceinline__ uint32_t pair_nibble(uint32_t t0, uint32_t t1) {
  return (t0 & 0xA0u) | ((t1 & 0xA0u) << 1);  // the pair's four bits at bits 5 .. 8
}
// Appends a pair's nibble to the row mask under construction (pairs enter
// at the top and move down four bits per pair; the row's end aligns them).
__device__ __forceinline__ uint64_t push_nibble(uint64_t S, uint32_t nib) {
  return (S >> 4) | ((uint64_t)nib << 55);
}
// Context bit 8 of a quad from its left neighbour t in the same row (not
// the initial row): either of the neighbour's right-column samples.
__device__ __forceinline__ uint32_t left_ctx(uint32_t t) { return ((t & 0xC0u) + 0xC0u) & 0x100u; }

// CxtVLC / MEL / UVLC pass of one block (decode_cleanup_symbols,
// ht_block_decode.rs:1056-1205): the serial chain of the cleanup pass.  Writes
// one 32-bit symbol per quad (entry | u << 16) into the block's symbol table,
// quad rows of nq entries.  The row above gives the context: with REG (blocks
// at most 64 wide, nq <= 32) its two context bits per quad live in a 64-bit
// register, otherwise they are read back from the symbol table.
// After each quad row is in the symbol table, row_done(rows written so far)
// (the fused small-plan kernel publishes progress with it).  The row's pairs
// are staged at stage[pair * stage_stride + stage_slot].
struct NoRowHook {
  static constexpr bool kUnroll2 = false;  // the pair loop left to the compiler
  __device__ void operator()(uint32_t) const {}
};
template <bool REG, bool OUTLINE, typename RowHook = NoRowHook>
__device__ bool decode_vlc(const HtJob& job, const uint8_t* src, uint32_t* __restrict__ sym, const SmemTables& T,
                           uint2* __restrict__ stage, uint32_t stage_stride, uint32_t stage_slot,
                           RowHook row_done = RowHook()) {
  const uint32_t lcup = job.lcup, w = job.w, h = job.h;
  if (lcup < 2) return false;
  uint32_t scup = ((uint32_t)ld8(src + lcup - 1) << 4) + (ld8(src + lcup - 2) & 0x0F);
  if (scup < 2 || scup > lcup || scup > 4079) return false;
  MelT<OUTLINE> mel;
  mel.init(src, lcup, scup);
  VlcT<OUTLINE> vlc;
  vlc.init(src, lcup, scup);
  int run = mel.get_run();
  const uint32_t nq = (w + 1) / 2, qs = sym_row_stride(w);
  uint32_t* row = sym;
  // REG blocks whose rows hold a multiple of 4 symbols stage each row's
  // pairs in the lane's shared-memory column and write the row with 16-byte
  // stores (far fewer scattered store requests than one per pair).
  const bool staged = REG && (qs & 3) == 0;
  const uint32_t lanes = stage_stride, tid = stage_slot;
  auto put = [&](uint32_t q, uint32_t a, uint32_t b) {
    if (staged) stage[(q >> 1) * lanes + tid] = make_uint2(a, b);
    else *reinterpret_cast<uint2*>(row + q) = make_uint2(a, b);  // q even, rows padded to even
  };
  auto flush = [&]() {
    if constexpr (REG) {
      if (!staged) return;
      for (uint32_t k = 0; 2 * k < nq; k += 2) {
        const uint2 a = stage[k * lanes + tid];
        const uint2 b = 2 * (k + 1) < nq ? stage[(k + 1) * lanes + tid] : make_uint2(0, 0);
        *reinterpret_cast<uint4*>(row + 2 * k) = make_uint4(a.x, a.y, b.x, b.y);
      }
    }
  };
  // REG: the finished row's context mask S (pair_nibble); pairs enter it at
  // the top, so the row's end shifts it down by 4 bits per absent pair.
  uint64_t S = 0;
  const uint32_t row_align = 64 - 4 * ((nq + 1) / 2);
  // Initial quad row.
  {
    uint32_t c_q = 0;
    for (uint32_t q = 0; q < nq; q += 2) {
      uint32_t v = vlc.fetch();
      uint32_t t0 = T.vlc0[c_q + (v & 0x7F)];
      if (c_q == 0) {
        run -= 2;
        t0 = run == -1 ? t0 : 0;
        if (run < 0) run = mel.get_run();
      }
      c_q = ((t0 & 0x10) << 3) | ((t0 & 0xE0) << 2);
      // The pair's bits (at most 30) are read from the 32-bit window v with
      // 32-bit shifts; the reader advances once, by their sum, at the end.
      const uint32_t l0 = t0 & 7;
      v >>= l0;
      const bool hasB = q + 1 < nq;
      uint32_t t1 = T.vlc0[c_q + (v & 0x7F)];
      if (c_q == 0 && hasB) {
        run -= 2;
        t1 = run == -1 ? t1 : 0;
        if (run < 0) run = mel.get_run();
      }
      if (!hasB) t1 = 0;
      c_q = ((t1 & 0x10) << 3) | ((t1 & 0xE0) << 2);
      const uint32_t l1 = t1 & 7;
      v >>= l1;
      uint32_t mode = ((t0 & 8) << 3) | ((t1 & 8) << 4);
      if (mode == 0xC0) {
        run -= 2;
        if (run == -1) mode += 0x40;
        if (run < 0) run = mel.get_run();
      }
      uint32_t ue = T.uvlc0[mode + (v & 0x3F)];
      const uint32_t lp = ue & 7;
      v >>= lp;
      ue >>= 3;
      uint32_t len = ue & 0xF;
      uint32_t tmp = v & ((1u << len) - 1);
      vlc.advance(l0 + l1 + lp + len);
      ue >>= 4;
      len = ue & 7;
      ue >>= 3;
      put(q, t0 | ((1 + (ue & 7) + (tmp & ~(0xFFu << len))) << 16), t1 | ((1 + (ue >> 3) + (tmp >> len)) << 16));
      if (REG) S = push_nibble(S, pair_nibble(t0, t1));
    }
    if (REG) S >>= row_align;
    flush();
    row_done(1u);
  }
  // Other quad rows: context from the row above (quads q, q+1, q+2).
  for (uint32_t y = 2; y < h; y += 2) {
    const uint32_t* prev = row;
    row += qs;
    uint32_t c_q = 0;
    // REG: Qc = (S | S >> 1) >> (4k + 1) for pair k (bits 0 and 2: Q[4k+1],
    // Q[4k+3]); up7 = Q[4k-1] at bit 7 (Q[-1] = S[0]).
    uint64_t Qc = 0;
    uint32_t up7 = 0;
    uint32_t pq0 = 0, pq1 = 0;
    if (REG) {
      Qc = (S | (S >> 1)) >> 1;
      up7 = ((uint32_t)S & 1u) << 7;
      S = 0;
    } else {
      pq0 = prev[0] & 0xFFFF;
      pq1 = nq > 1 ? prev[1] & 0xFFFF : 0;
    }
    // One quad pair of the row (a lambda so that the loop can be unrolled
    // for one caller only).
    auto pair_step = [&](uint32_t q) {
      uint32_t pq2 = 0, pq3 = 0, a1 = 0;
      if (REG) {
        const uint32_t qc = (uint32_t)Qc;
        c_q |= up7 | ((qc & 1u) << 9);  // quad q
        a1 = (qc & 5u) << 7;             // quad q + 1
        up7 = (qc & 4u) << 5;
        Qc >>= 4;
      } else {
        pq2 = q + 2 < nq ? prev[q + 2] & 0xFFFF : 0;
        pq3 = q + 3 < nq ? prev[q + 3] & 0xFFFF : 0;
        c_q |= (pq0 & 0xA0) << 2;
        c_q |= (pq1 & 0x20) << 4;
      }
      uint32_t v = vlc.fetch();
      uint32_t t0 = T.vlc1[c_q + (v & 0x7F)];
      if (c_q == 0) {
        run -= 2;
        t0 = run == -1 ? t0 : 0;
        if (run < 0) run = mel.get_run();
      }
      c_q = left_ctx(t0);
      if (REG) c_q |= a1;
      else c_q |= (pq0 & 0x80) | ((pq1 & 0xA0) << 2) | ((pq2 & 0x20) << 4);
      const uint32_t l0 = t0 & 7;
      v >>= l0;
      const bool hasB = q + 1 < nq;
      uint32_t t1 = T.vlc1[c_q + (v & 0x7F)];
      if (c_q == 0 && hasB) {
        run -= 2;
        t1 = run == -1 ? t1 : 0;
        if (run < 0) run = mel.get_run();
      }
      if (!hasB) t1 = 0;
      c_q = left_ctx(t1);
      if (!REG) c_q |= pq1 & 0x80;
      const uint32_t l1 = t1 & 7;
      v >>= l1;
      uint32_t mode = ((t0 & 8) << 3) | ((t1 & 8) << 4);
      uint32_t ue = T.uvlc1[mode + (v & 0x3F)];
      const uint32_t lp = ue & 7;
      v >>= lp;
      ue >>= 3;
      uint32_t len = ue & 0xF;
      uint32_t tmp = v & ((1u << len) - 1);
      vlc.advance(l0 + l1 + lp + len);
      ue >>= 4;
      len = ue & 7;
      ue >>= 3;
      put(q, t0 | (((ue & 7) + (tmp & ~(0xFFu << len))) << 16), t1 | (((ue >> 3) + (tmp >> len)) << 16));
      if (REG) {
        S = push_nibble(S, pair_nibble(t0, t1));
      } else {
        pq0 = pq2;
        pq1 = pq3;
      }
    };
    if constexpr (RowHook::kUnroll2) {
#pragma unroll 2
      for (uint32_t q = 0; q < nq; q += 2) pair_step(q);
    } else {
      for (uint32_t q = 0; q < nq; q += 2) pair_step(q);
    }
    if (REG) S >>= row_align;
    flush();
    row_done(y / 2 + 1);
  }
  return true;
}

}  // namespace

// Pass 1: one lane per code block runs the VLC chain, `lanes` (a power of
// two up to 32) code blocks per warp: warp k takes blocks k * lanes ..
// k * lanes + lanes - 1 on its first lanes.  The lanes of a warp follow
// different blocks' branches, and a warp pays for every path any of its
// lanes takes at each step; fewer blocks per warp make each chain step
// shorter, which a plan with few blocks (one tile) wants, while a large
// batch fills the SMs with 32 blocks per warp.  OUTLINE: the bit readers'
// rare refill paths as out-of-line calls (MelT, VlcT).
template <bool OUTLINE>
__global__ void __launch_bounds__(kHtThreads) ht_vlc_kernel(const HtJob* __restrict__ jobs, uint32_t njobs,
                                                            const uint8_t* __restrict__ arena,
                                                            uint32_t* __restrict__ symbols, uint32_t lanes) {
  __shared__ SmemTables T;
  __shared__ uint2 stage[16 * kHtThreads];  // per lane: the pairs of one row of a 64-wide block
  {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(&g_ht_tables);
    uint32_t* d = reinterpret_cast<uint32_t*>(&T);
    for (uint32_t i = threadIdx.x; i < sizeof(SmemTables) / 4; i += blockDim.x) d[i] = src[i];
  }
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31;
  if (lane >= lanes) return;
  const uint32_t j = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * lanes + lane;
  if (j >= njobs) return;
  const HtJob job = jobs[j];
  if (job.passes == 0) return;
  uint32_t* sym = symbols + job.sym;
  const bool ok = job.w <= 64 ? decode_vlc<true, OUTLINE>(job, arena + job.src, sym, T, stage, blockDim.x, threadIdx.x)
                              : decode_vlc<false, OUTLINE>(job, arena + job.src, sym, T, stage, blockDim.x, threadIdx.x);
  if (!ok) sym[0] = kSymFailed;
}

namespace {

constexpr int kMsWarps = 8;  // warps (code blocks in flight) per CTA of the MagSgn pass

// The lane's four stream bytes x (byte j at 8 j; zero past the segment) as
// one bit string from the position of its first byte: byte j sits at
// r_j = 8 j minus the 0xFF bytes among the lane's bytes before byte j - 1
// and the byte before the lane (pf).  Bytes that follow an 0xFF carry 7 bits
// (their top bit, a stuffed zero, overlaps the next byte and is ORed in as
// the reference's reader does).  At most 32 bits: r_3 <= 24.
__device__ __forceinline__ uint32_t lane_bits(uint32_t x, uint32_t pf, uint32_t f0, uint32_t f1) {
  const uint32_t r1 = 8 - pf, r2 = r1 + 8 - f0, r3 = r2 + 8 - f1;
  return (x & 0xFFu) | (((x >> 8) & 0xFFu) << r1) | (((x >> 16) & 0xFFu) << r2) | ((x >> 24) << r3);
}

// ORs a lane's bit string v into the bit array W at bit position pos (two
// words at most).
__device__ __forceinline__ void or_bits(uint32_t* W, uint32_t pos, uint32_t v) {
  const uint32_t wi = pos >> 5, sh = pos & 31;
  atomicOr(&W[wi], v << sh);
  if (sh && (v >> (32 - sh))) atomicOr(&W[wi + 1], v >> (32 - sh));
}

// Unstuffs the forward MagSgn byte stream [0, len) into a bit array W
// (bit k of the stream = bit k%32 of W[k/32]): each byte contributes 8 bits,
// or 7 after a 0xFF byte, ORed in at its offset exactly as the reference's
// ForwardBitReader accumulates it (ht_block_decode.rs:888-930).  Bits past
// the end read as ones (the reader pads with 0xFF).  Returns the number of
// real bits.
//
// The warp takes 128 bytes per step, four per lane.  A step with no 0xFF
// byte (and none just before it) is a plain bit shift of the input: each
// lane stores one whole output word built from its word and its right
// neighbour's.  Other steps place every byte at its own offset.
__device__ uint32_t unstuff_magsgn(const uint8_t* src, uint32_t len, uint32_t* W, uint32_t nwords) {
  const uint32_t lane = threadIdx.x & 31;
  for (uint32_t i = lane; i < nwords; i += 32) W[i] = 0;
  __syncwarp();
  uint32_t ff_total = 0;  // 0xFF bytes among bytes [0, base)
  uint32_t prev_ff = 0;   // byte base - 1 is 0xFF
  for (uint32_t base = 0; base < len; base += 128) {
    const uint32_t i0 = base + 4 * lane;
    // Bytes i0 .. i0+3 (zero past len), little-endian.  Both aligned words
    // hold a byte of the segment, so they lie inside its allocation.
    uint32_t x = 0;
    if (i0 < len) {
      const uintptr_t addr = (uintptr_t)(src + i0);
      const uint32_t* wp = reinterpret_cast<const uint32_t*>(addr & ~(uintptr_t)3);
      const uint32_t sh = (uint32_t)(addr & 3);
      const uint32_t nvalid = min(4u, len - i0);
      const uint32_t lo = __ldg(wp);
      const uint32_t hi = sh + nvalid > 4 ? __ldg(wp + 1) : 0u;
      x = __funnelshift_r(lo, hi, 8 * sh);
      if (nvalid < 4) x &= 0xFFFFFFFFu >> (8 * (4 - nvalid));
    }
    const uint32_t fm = i0 < len ? __vcmpeq4(x, 0xFFFFFFFFu) : 0u;  // 0xFF per 0xFF byte
    // Padding bytes beyond len are zero, never 0xFF.
    const bool full = base + 128 <= len;
    if (full && !prev_ff && !__any_sync(0xFFFFFFFFu, fm != 0)) {
      // Stream bit of byte base: 8 * base minus one per 0xFF before it.
      const uint32_t P = 8 * base - ff_total;
      const uint32_t s = P & 31, wb = P >> 5;
      const uint32_t xn = __shfl_down_sync(0xFFFFFFFFu, x, 1);
      if (lane < 31) W[wb + lane + 1] = __funnelshift_l(x, xn, s);
      if (lane == 0) atomicOr(&W[wb], x << s);
      if (lane == 31 && s) atomicOr(&W[wb + 32], x >> (32 - s));
      continue;
    }
    const uint32_t f0 = fm & 1, f1 = (fm >> 8) & 1, f2 = (fm >> 16) & 1, f3 = (fm >> 24) & 1;
    const uint32_t b0 = __ballot_sync(0xFFFFFFFFu, f0), b1 = __ballot_sync(0xFFFFFFFFu, f1);
    const uint32_t b2 = __ballot_sync(0xFFFFFFFFu, f2), b3 = __ballot_sync(0xFFFFFFFFu, f3);
    const uint32_t lt = (1u << lane) - 1;
    // 0xFF bytes among [0, i0) and whether byte i0 - 1 is one.
    const uint32_t F = ff_total + __popc(b0 & lt) + __popc(b1 & lt) + __popc(b2 & lt) + __popc(b3 & lt);
    uint32_t pf = __shfl_up_sync(0xFFFFFFFFu, f3, 1);
    if (lane == 0) pf = prev_ff;
    // Byte i0 is shortened by the 0xFF bytes among [0, i0 - 1); the lane's
    // other bytes follow it (lane_bits).
    if (x) or_bits(W, 8 * i0 - (F - pf), lane_bits(x, pf, f0, f1));
    ff_total += __popc(b0) + __popc(b1) + __popc(b2) + __popc(b3);
    const uint32_t last = min(base + 128, len) - 1 - base;  // last byte of the step
    const uint32_t lb = last >> 2, lj = last & 3;
    const uint32_t lf = lj == 0 ? b0 : lj == 1 ? b1 : lj == 2 ? b2 : b3;
    prev_ff = (lf >> lb) & 1;
  }
  // Real bits: 8 per byte minus one per byte that follows a 0xFF.
  const uint32_t end_bits = len ? 8 * len - (ff_total - prev_ff) : 0;
  __syncwarp();
  // Padding: every bit from end_bits on is one.
  for (uint32_t wi = lane; wi < nwords; wi += 32) {
    uint32_t lo = wi * 32;
    if (lo >= end_bits) W[wi] = 0xFFFFFFFFu;
    else if (lo + 32 > end_bits) W[wi] |= 0xFFFFFFFFu << (end_bits - lo);
  }
  __syncwarp();
  return end_bits;
}

__device__ __forceinline__ uint32_t bits_at(const uint32_t* W, uint32_t nwords, uint32_t off) {
  uint32_t wi = off >> 5, sh = off & 31;
  uint32_t lo = wi < nwords ? W[wi] : 0xFFFFFFFFu;
  uint32_t hi = wi + 1 < nwords ? W[wi + 1] : 0xFFFFFFFFu;
  return __funnelshift_r(lo, hi, sh);
}

// Per-quad magnitude/sign arithmetic of the row loops below, with the quad's
// four samples as the four bytes of one word (byte i = sample i, the order
// of the quad's bits in the stream: (0,0), (0,1), (1,0), (1,1) by column
// pairs).  A bit count m_n is at most 31 and a quad's total at most 124, so
// bytewise sums never carry and a multiply by 0x01010101 forms every
// sample's inclusive prefix inside the quad at once.

// Byte i = bit i of the nibble x.
__device__ __forceinline__ uint32_t spread4(uint32_t x) { return (x * 0x00204081u) & 0x01010101u; }

struct QuadBits {
  uint32_t m;    // m_n per sample: U - e_k when significant, else 0
  uint32_t cs;   // per sample, the bits of the samples before it in the quad
  uint32_t tot;  // the quad's bits
};

// U is the quad's u_q (plus the exponent bound kappa after the first row);
// U > mmsb + 2 marks an invalid stream, which the caller flags and whose
// block comes out as zeros, so clamping U to 31 here (the bytes then cannot
// carry) changes no valid result.
__device__ __forceinline__ QuadBits quad_bits(uint32_t inf, uint32_t U) {
  const uint32_t sig = spread4((inf >> 4) & 0xFu), k = spread4(inf >> 12);
  const uint32_t m = (min(U, 31u) * 0x01010101u - k) & (sig * 0xFFu);
  const uint32_t incl = m * 0x01010101u;
  return QuadBits{m, incl - m, incl >> 24};
}

// The 32 stream bits from bit c (< 64) of the 64-bit window hi:lo.
__device__ __forceinline__ uint32_t window_bits(uint32_t lo, uint32_t hi, uint32_t c) {
  return (uint32_t)((((uint64_t)hi << 32) | lo) >> c);
}

// Sample i's coefficient from its bits msv (sign first, then the magnitude
// bits below the implied ones), bit count m, known-1 bit e1 and
// significance: decode_mag_sgn_sample_with_vn's v_n (ht_block_decode.rs:1010-1032)
// gives the sign-magnitude word sign << 31 | (v + 2) << (p - 1) in 32-bit
// arithmetic (whose top bit, in the largest valid magnitudes, the shift can
// set as well); RAW returns that word, otherwise coefficient_to_i32
// (:225-234) of it: (word & 0x7FFFFFFF) >> (31 - nbp), negated when the top
// bit is set, computed as (word << 1) >> rs with rs = 32 - nbp (1 when
// nbp >= 31; the shift clamps at 32).  E receives the bit length of v (0
// when insignificant), the exponent the row below needs.
template <bool RAW>
__device__ __forceinline__ int32_t sample_value(uint32_t msv, uint32_t m, uint32_t e1, bool sig, uint32_t p,
                                                uint32_t rs, uint32_t& E) {
  const uint32_t mask = __funnelshift_lc(0xFFFFFFFFu, 0u, m);
  const uint32_t v = (msv & mask) | (e1 << m) | 1u;
  E = sig ? 32 - __clz(v) : 0u;
  const uint32_t word = (msv << 31) | ((v + 2) << (p - 1));
  if (RAW) return sig ? (int32_t)word : 0;
  const int32_t mag = (int32_t)__funnelshift_rc(word << 1, 0u, rs);
  return sig ? ((int32_t)word < 0 ? -mag : mag) : 0;
}

// The four samples of a quad whose stream bits start at `off`: one clamped
// three-word window read serves all four when the quad holds fewer than 64
// bits; otherwise each sample reads its own 32 bits.
template <bool RAW>
__device__ __forceinline__ void quad_samples(const uint32_t* W, uint32_t ms_words, uint32_t lim, uint32_t off,
                                             uint32_t inf, const QuadBits& qb, uint32_t p, uint32_t rs,
                                             int32_t val[4], uint32_t E[4]) {
  uint32_t lo, hi;
  {
    const uint32_t o = min(off, lim), wi = o >> 5, sh = o & 31;
    const uint32_t a0 = W[wi], a1 = W[wi + 1], a2 = W[wi + 2];
    lo = __funnelshift_r(a0, a1, sh);
    hi = __funnelshift_r(a1, a2, sh);
  }
  uint32_t msv[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) msv[i] = window_bits(lo, hi, (qb.cs >> (8 * i)) & 0xFFu);
  if (qb.tot >= 64) {
#pragma unroll
    for (int i = 0; i < 4; ++i) msv[i] = bits_at(W, ms_words, off + ((qb.cs >> (8 * i)) & 0xFFu));
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
    val[i] = sample_value<RAW>(msv[i], (qb.m >> (8 * i)) & 0xFFu, (inf >> (8 + i)) & 1u, (inf >> (4 + i)) & 1u, p,
                               rs, E[i]);
}


// The magnitude/sign rows of one block (decode_magnitude_sign_phase,
// ht_block_decode.rs:1435-1561) for the calling warp.  Per quad row the lanes
// take one quad each; a warp prefix scan of the per-quad bit counts gives each
// lane its bit offset in the unstuffed stream W, and the lane reads its bits
// through one 64-bit window.  The exponent bound kappa needs the bit lengths
// of v_n of the four samples above the quad: with NARROW (blocks at most 64
// wide, one quad per lane per row) they stay in registers and come from the
// neighbouring lanes by shuffles, otherwise they are kept per column in
// shared memory (Ebase, two rows of `cols` bytes).  Returns true (on every
// lane) when the stream is invalid.
// Rows are taken as they are: the two-pass form decodes symbols a kernel
// earlier.
struct NoRowWait {
  static constexpr bool kLive = false;
  __device__ bool operator()(uint32_t) const { return true; }
};
template <bool NARROW, bool RAW, typename RowWait = NoRowWait>
__device__ bool magsgn_rows(const HtJob& job, const uint32_t* W, uint32_t ms_words, uint8_t* Ebase, uint32_t cols,
                            const uint32_t* __restrict__ sym, int32_t* __restrict__ dst,
                            RowWait row_ready = RowWait()) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t w = job.w, h = job.h, stride = job.stride;
  const uint32_t mmsb = job.mmsb, p = 30 - mmsb, mmsbp2 = mmsb + 2, nbp = job.nbp;
  const uint32_t rs = nbp >= 31 ? 1u : 32u - nbp;
  // Window reads start at most at bit `lim`, so that words wi .. wi + 2 lie
  // in the array (it holds at least 5 words).  The array ends with at least
  // 64 bits of ones past the stream (its padding), and `lim` lies beyond
  // those bits' start, so a clamped read returns the ones an unclamped one
  // would have seen past the end of the stream.
  const uint32_t lim = 32 * (ms_words - 3);
  const bool pairs = ((job.dst | stride) & 1) == 0;  // 8-byte aligned sample pairs
  const uint32_t nq = (w + 1) / 2, qs = sym_row_stride(w);
  uint8_t* Eprev = Ebase;  // wide blocks: bit lengths of v_n per column + 1, row above
  uint8_t* Ecur = Ebase + cols;
  if (!NARROW) {
    for (uint32_t c = lane; c < cols; c += 32) Eprev[c] = 0;
    __syncwarp();
  }
  uint32_t e_left = 0, e_right = 0;  // NARROW: bottom-row bit lengths of this lane's quad
  uint32_t rowbase = 0;
  bool bad = false;
  // Running pointers: sample row y of the block and quad row r of its symbols.
  int32_t* row0 = dst;
  const uint32_t* srow = sym;
  for (uint32_t y = 0; y < h; y += 2, row0 += 2 * (size_t)stride, srow += qs) {
    // The fused form waits for the quad row's symbols (warp-uniform result;
    // false: the chain failed or the wait ran out, and the block is invalid).
    if (!row_ready(y >> 1)) {
      bad = true;
      break;
    }
    const bool initial = y == 0, second = y + 1 < h;
    // NARROW rows have at most 32 quads: one pass, known at compile time.
    const uint32_t c0_end = NARROW ? 1u : nq;
    for (uint32_t c0 = 0; c0 < c0_end; c0 += 32) {
      const uint32_t q = c0 + lane;
      const bool active = q < nq;
      // Symbols written by the same CTA's chain lane are read past L1.
      const uint32_t s = active ? (RowWait::kLive ? __ldcg(srow + q) : srow[q]) : 0;
      const uint32_t inf = s & 0xFFFF;
      uint32_t U = s >> 16;
      if (!initial) {
        uint32_t e;
        if (NARROW) {
          // Columns 2q-1 and 2q+2 belong to the neighbouring lanes' quads;
          // outside the block they are zero (lanes past nq hold zeros).
          uint32_t l = __shfl_up_sync(0xFFFFFFFFu, e_right, 1);
          uint32_t rr = __shfl_down_sync(0xFFFFFFFFu, e_left, 1);
          if (lane == 0) l = 0;
          if (lane == 31) rr = 0;
          e = max(max(l, e_left), max(e_right, rr));
        } else {
          // Columns 2q-1 .. 2q+2 of the row above live at Eprev[col + 1]
          // (index <= 2*nq + 1 <= w + 2 < max_w + 4 for an active lane).
          e = active ? max(max((uint32_t)Eprev[2 * q], (uint32_t)Eprev[2 * q + 1]),
                           max((uint32_t)Eprev[2 * q + 2], (uint32_t)Eprev[2 * q + 3]))
                     : 0;
        }
        uint32_t gamma = inf & 0xF0;
        gamma &= gamma - 0x10;
        if (active) U += gamma != 0 ? max(e, 2u) - 1 : 1;
      }
      bad |= active && U > mmsbp2;
      const QuadBits qb = quad_bits(inf, U);
      // Warp inclusive scan of the bit counts.
      uint32_t inc = qb.tot;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        uint32_t v = __shfl_up_sync(0xFFFFFFFFu, inc, d);
        if (lane >= (uint32_t)d) inc += v;
      }
      const uint32_t chunk_bits = __shfl_sync(0xFFFFFFFFu, inc, 31);
      const uint32_t off = rowbase + inc - qb.tot;
      rowbase += chunk_bits;
      int32_t val[4];
      uint32_t E[4];
      quad_samples<RAW>(W, ms_words, lim, off, inf, qb, p, rs, val, E);
      if (active) {
        const uint32_t x = 2 * q;
        int32_t* p0 = row0 + x;
        if (pairs && x + 1 < w) {
          *reinterpret_cast<int2*>(p0) = make_int2(val[0], val[2]);
          if (second) *reinterpret_cast<int2*>(p0 + stride) = make_int2(val[1], val[3]);
        } else {
          p0[0] = val[0];
          if (second) p0[stride] = val[1];
          if (x + 1 < w) {
            p0[1] = val[2];
            if (second) p0[stride + 1] = val[3];
          }
        }
        if (!NARROW) {
          // Bottom-row exponents of this quad for the next quad row.
          Ecur[x + 1] = (uint8_t)E[1];
          Ecur[x + 2] = x + 1 < w ? (uint8_t)E[3] : 0;
        }
      }
      if (NARROW) {
        e_left = active ? E[1] : 0;
        e_right = active && 2 * q + 1 < w ? E[3] : 0;
      }
    }
    if (!NARROW) {
      __syncwarp();
      // Columns outside [0, w) stay zero in both buffers.
      if (lane == 0) {
        Ecur[0] = 0;
        Ecur[w + 1] = 0;
        Ecur[w + 2] = 0;
      }
      __syncwarp();
      uint8_t* t = Eprev;
      Eprev = Ecur;
      Ecur = t;
    }
  }
  return __any_sync(0xFFFFFFFFu, bad);
}
}  // namespace

// Narrow blocks (at most 32 wide: 16 quads a row) would leave half of a
// warp idle, so a warp takes two of them, one per half-warp (lanes 0-15 and
// 16-31).  The functions below are unstuff_magsgn and magsgn_rows for that
// case: every shuffle, ballot and scan runs on all 32 lanes with the
// half-warp as its segment, and both halves run the longer block's loop
// trip counts (a half past its own work idles), so no warp-synchronous
// operation sits in a branch that one half skips.

// unstuff_magsgn for the calling half-warp's stream: 64 bytes per step.
__device__ uint32_t unstuff_half(const uint8_t* src, uint32_t len, uint32_t* W, uint32_t nwords) {
  const uint32_t lane = threadIdx.x & 31, gl = lane & 15, gsh = lane & 16;
  for (uint32_t i = gl; i < nwords; i += 16) W[i] = 0;
  __syncwarp();
  const uint32_t steps = (len + 63) / 64;
  const uint32_t nsteps = max(steps, __shfl_xor_sync(0xFFFFFFFFu, steps, 16));
  uint32_t ff_total = 0;  // 0xFF bytes among bytes [0, base)
  uint32_t prev_ff = 0;   // byte base - 1 is 0xFF
  for (uint32_t k = 0; k < nsteps; ++k) {
    const uint32_t base = 64 * k, i0 = base + 4 * gl;
    uint32_t x = 0;
    if (i0 < len) {
      const uintptr_t addr = (uintptr_t)(src + i0);
      const uint32_t* wp = reinterpret_cast<const uint32_t*>(addr & ~(uintptr_t)3);
      const uint32_t sh = (uint32_t)(addr & 3);
      const uint32_t nvalid = min(4u, len - i0);
      const uint32_t lo = __ldg(wp);
      const uint32_t hi = sh + nvalid > 4 ? __ldg(wp + 1) : 0u;
      x = __funnelshift_r(lo, hi, 8 * sh);
      if (nvalid < 4) x &= 0xFFFFFFFFu >> (8 * (4 - nvalid));
    }
    const uint32_t fm = i0 < len ? __vcmpeq4(x, 0xFFFFFFFFu) : 0u;
    // One vote first: a step in which neither half has an 0xFF byte (and no
    // 0xFF byte just before it) is a plain shift of the input in both, and
    // needs neither the per-byte votes nor the 0xFF counts.
    const uint32_t any_ff = (__ballot_sync(0xFFFFFFFFu, fm != 0) >> gsh) & 0xFFFFu;  // every lane votes
    const bool plain = base >= len || (base + 64 <= len && !prev_ff && any_ff == 0);
    if (__all_sync(0xFFFFFFFFu, plain)) {
      const uint32_t xn = __shfl_down_sync(0xFFFFFFFFu, x, 1, 16);
      if (base < len) {
        const uint32_t P = 8 * base - ff_total;
        const uint32_t s = P & 31, wb = P >> 5;
        if (gl < 15) W[wb + gl + 1] = __funnelshift_l(x, xn, s);
        if (gl == 0) atomicOr(&W[wb], x << s);
        if (gl == 15 && s) atomicOr(&W[wb + 16], x >> (32 - s));
      }
      continue;
    }
    const uint32_t f0 = fm & 1, f1 = (fm >> 8) & 1, f2 = (fm >> 16) & 1, f3 = (fm >> 24) & 1;
    const uint32_t b0 = (__ballot_sync(0xFFFFFFFFu, f0) >> gsh) & 0xFFFFu;
    const uint32_t b1 = (__ballot_sync(0xFFFFFFFFu, f1) >> gsh) & 0xFFFFu;
    const uint32_t b2 = (__ballot_sync(0xFFFFFFFFu, f2) >> gsh) & 0xFFFFu;
    const uint32_t b3 = (__ballot_sync(0xFFFFFFFFu, f3) >> gsh) & 0xFFFFu;
    const uint32_t xn = __shfl_down_sync(0xFFFFFFFFu, x, 1, 16);
    uint32_t pf = __shfl_up_sync(0xFFFFFFFFu, f3, 1, 16);
    if (base < len) {
      if (base + 64 <= len && !prev_ff && (b0 | b1 | b2 | b3) == 0) {
        const uint32_t P = 8 * base - ff_total;
        const uint32_t s = P & 31, wb = P >> 5;
        if (gl < 15) W[wb + gl + 1] = __funnelshift_l(x, xn, s);
        if (gl == 0) atomicOr(&W[wb], x << s);
        if (gl == 15 && s) atomicOr(&W[wb + 16], x >> (32 - s));
      } else {
        const uint32_t lt = (1u << gl) - 1;
        const uint32_t F = ff_total + __popc(b0 & lt) + __popc(b1 & lt) + __popc(b2 & lt) + __popc(b3 & lt);
        if (gl == 0) pf = prev_ff;
        if (x) or_bits(W, 8 * i0 - (F - pf), lane_bits(x, pf, f0, f1));
      }
      ff_total += __popc(b0) + __popc(b1) + __popc(b2) + __popc(b3);
      const uint32_t last = min(base + 64, len) - 1 - base;  // last byte of the step
      const uint32_t lb = last >> 2, lj = last & 3;
      const uint32_t lf = lj == 0 ? b0 : lj == 1 ? b1 : lj == 2 ? b2 : b3;
      prev_ff = (lf >> lb) & 1;
    }
  }
  const uint32_t end_bits = len ? 8 * len - (ff_total - prev_ff) : 0;
  __syncwarp();
  for (uint32_t wi = gl; wi < nwords; wi += 16) {
    uint32_t lo = wi * 32;
    if (lo >= end_bits) W[wi] = 0xFFFFFFFFu;
    else if (lo + 32 > end_bits) W[wi] |= 0xFFFFFFFFu << (end_bits - lo);
  }
  __syncwarp();
  return end_bits;
}

// magsgn_rows<true, false> for the calling half-warp's block (live) over
// hmax rows, the taller of the two blocks' heights.  Returns true on the
// half's lanes when its stream is invalid.
__device__ bool magsgn_rows_half(const HtJob& job, bool live, const uint32_t* W, uint32_t ms_words, uint32_t hmax,
                                 const uint32_t* __restrict__ sym, int32_t* __restrict__ dst) {
  const uint32_t lane = threadIdx.x & 31, gl = lane & 15, gsh = lane & 16;
  const uint32_t w = live ? job.w : 0, h = live ? job.h : 0, stride = job.stride;
  const uint32_t mmsb = job.mmsb, p = 30 - mmsb, mmsbp2 = mmsb + 2, nbp = job.nbp;
  const uint32_t rs = nbp >= 31 ? 1u : 32u - nbp;
  // As in magsgn_rows: clamped window reads stay in the half's words.
  const uint32_t lim = live ? 32 * (ms_words - 3) : 0;
  const bool pairs = ((job.dst | stride) & 1) == 0;
  const uint32_t nq = (w + 1) / 2, qs = sym_row_stride(w);
  uint32_t e_left = 0, e_right = 0, rowbase = 0;
  bool bad = false;
  // Per lane, invariant over the rows: its quad column, whether it holds a
  // quad, whether the quad has a right column and whether the pair goes out
  // in one 8-byte store; running pointers to its samples and its symbols.
  const uint32_t q = gl;
  const bool lane_q = q < nq, has_right = 2 * q + 1 < w, pair_store = pairs && has_right;
  int32_t* lp = dst + 2 * q;
  const uint32_t* sp = sym + q;
  for (uint32_t y = 0; y < hmax; y += 2, lp += 2 * (size_t)stride, sp += qs) {
    const bool initial = y == 0, second = y + 1 < h;
    const bool active = y < h && lane_q;
    const uint32_t s = active ? *sp : 0;
    const uint32_t inf = s & 0xFFFF;
    uint32_t U = s >> 16;
    if (!initial) {
      uint32_t l = __shfl_up_sync(0xFFFFFFFFu, e_right, 1, 16);
      uint32_t rr = __shfl_down_sync(0xFFFFFFFFu, e_left, 1, 16);
      if (gl == 0) l = 0;
      if (gl == 15) rr = 0;
      const uint32_t e = max(max(l, e_left), max(e_right, rr));
      uint32_t gamma = inf & 0xF0;
      gamma &= gamma - 0x10;
      if (active) U += gamma != 0 ? max(e, 2u) - 1 : 1;
    }
    bad |= active && U > mmsbp2;
    const QuadBits qb = quad_bits(inf, U);
    uint32_t inc = qb.tot;
#pragma unroll
    for (int d = 1; d < 16; d <<= 1) {
      uint32_t v = __shfl_up_sync(0xFFFFFFFFu, inc, d, 16);
      if (gl >= (uint32_t)d) inc += v;
    }
    const uint32_t chunk_bits = __shfl_sync(0xFFFFFFFFu, inc, 15, 16);
    const uint32_t off = rowbase + inc - qb.tot;
    rowbase += chunk_bits;
    int32_t val[4];
    uint32_t E[4];
    quad_samples<false>(W, ms_words, lim, off, inf, qb, p, rs, val, E);
    if (active) {
      if (pair_store) {
        *reinterpret_cast<int2*>(lp) = make_int2(val[0], val[2]);
        if (second) *reinterpret_cast<int2*>(lp + stride) = make_int2(val[1], val[3]);
      } else {
        lp[0] = val[0];
        if (second) lp[stride] = val[1];
        if (has_right) {
          lp[1] = val[2];
          if (second) lp[stride + 1] = val[3];
        }
      }
    }
    e_left = active ? E[1] : 0;
    e_right = active && has_right ? E[3] : 0;
  }
  return ((__ballot_sync(0xFFFFFFFFu, bad) >> gsh) & 0xFFFFu) != 0;
}

// Pass 2: one warp per code block decodes magnitudes and signs
// (decode_magnitude_sign_phase, ht_block_decode.rs:1435-1561).  Per quad row
// the lanes take one quad each: the exponent bound kappa comes from the four
// samples above (bit lengths of the previous row's v_n, kept per column in
// shared memory), each lane sums its samples' m_n, a warp prefix scan turns
// the sums into bit offsets inside the unstuffed MagSgn stream, and the row
// is written with coalesced stores.
namespace {

// Magnitudes and signs of one code block by the calling warp; W and Ebase
// are the warp's shared-memory bit array and exponent rows.
template <typename RowWait = NoRowWait>
__device__ void magsgn_block(const HtJob& job, const uint8_t* __restrict__ arena,
                             const uint32_t* __restrict__ symbols, int32_t* __restrict__ coef,
                             uint32_t* __restrict__ tile_status, uint32_t ms_words, uint32_t cols, uint32_t* W,
                             uint8_t* Ebase, RowWait row_ready = RowWait()) {
  const uint32_t lane = threadIdx.x & 31;
  int32_t* dst = coef + job.dst;
  const uint32_t w = job.w, h = job.h, stride = job.stride;
  if (job.passes == 0) {
    for (uint32_t y = 0; y < h; ++y)
      for (uint32_t x = lane; x < w; x += 32) dst[(size_t)y * stride + x] = 0;
    return;
  }
  const uint32_t* sym = symbols + job.sym;
  const uint8_t* src = arena + job.src;
  // The block's cleanup bytes and quad symbols are requested from HBM before
  // the first of them is loaded: the unstuffing steps and the quad rows then
  // read them from L2.
  prefetch_l2_range(src, job.lcup, lane, 32);
  uint32_t lcup = job.lcup, scup = 0;
  bool ok;
  if constexpr (RowWait::kLive) {
    // The chain is still running: its failure arrives through row_ready, and
    // the segment checks it starts with are repeated here.
    ok = lcup >= 2;
    if (ok) {
      scup = ((uint32_t)ld8(src + lcup - 1) << 4) + (ld8(src + lcup - 2) & 0x0F);
      ok = scup >= 2 && scup <= lcup && scup <= 4079;
    }
  } else {
    prefetch_l2_range(sym, (size_t)sym_row_stride(w) * ((h + 1) / 2) * 4, lane, 32);
    ok = sym[0] != kSymFailed;
    if (ok) scup = ((uint32_t)ld8(src + lcup - 1) << 4) + (ld8(src + lcup - 2) & 0x0F);
  }
  if (ok) ok = (lcup - scup + 15) / 4 + 2 <= ms_words;
  if (ok) {
    const uint32_t ms_len = lcup - scup;
    // The block's own words of the bit array (at most ms_words, checked
    // above): they are zeroed, filled and padded with ones past the stream,
    // and reads beyond them return ones, so bits past the end still read as
    // the reference's 0xFF padding.
    const uint32_t words = (ms_len + 15) / 4 + 2;
    unstuff_magsgn(src, ms_len, W, words);
    // Blocks with refinement passes keep the sign-magnitude words for them.
    const bool raw = job.passes > 1;
    const bool bad =
        job.w <= 64 ? (raw ? magsgn_rows<true, true>(job, W, words, Ebase, cols, sym, dst, row_ready)
                           : magsgn_rows<true, false>(job, W, words, Ebase, cols, sym, dst, row_ready))
                    : (raw ? magsgn_rows<false, true>(job, W, words, Ebase, cols, sym, dst, row_ready)
                           : magsgn_rows<false, false>(job, W, words, Ebase, cols, sym, dst, row_ready));
    ok = !bad;
  }
  if (!ok) {
    __syncwarp();
    for (uint32_t y = 0; y < h; ++y)
      for (uint32_t x = lane; x < w; x += 32) dst[(size_t)y * stride + x] = 0;
    if (lane == 0) atomicOr(&tile_status[job.tile], kStatusDecode);
  }
  __syncwarp();  // the warp's shared buffers are reused by its next block
}

// Two narrow blocks, jobs[a] on lanes 0-15 and jobs[b] on lanes 16-31 (b ==
// UINT32_MAX: none), each with half of the warp's bit array (half_words
// words); both at most 32 wide with no refinement passes (the host orders
// such blocks after the others).  Same results as magsgn_block on each.
__device__ void magsgn_pair(const HtJob* __restrict__ jobs, uint32_t a, uint32_t b, const uint8_t* __restrict__ arena,
                            const uint32_t* __restrict__ symbols, int32_t* __restrict__ coef,
                            uint32_t* __restrict__ tile_status, uint32_t half_words, uint32_t* W) {
  const uint32_t lane = threadIdx.x & 31, g = lane >> 4, gl = lane & 15;
  const bool present = g == 0 || b != 0xFFFFFFFFu;
  const HtJob job = jobs[present ? (g ? b : a) : a];
  uint32_t* Wg = W + g * half_words;
  int32_t* dst = coef + job.dst;
  const uint32_t* sym = symbols + job.sym;
  const uint8_t* src = arena + job.src;
  const bool coded = present && job.passes != 0;
  bool ok = coded;
  if (ok) {
    prefetch_l2_range(src, job.lcup, gl, 16);
    prefetch_l2_range(sym, (size_t)sym_row_stride(job.w) * ((job.h + 1) / 2) * 4, gl, 16);
    ok = sym[0] != kSymFailed;
  }
  uint32_t ms_len = 0, words = 0;
  if (ok) {
    const uint32_t lcup = job.lcup;
    const uint32_t scup = ((uint32_t)ld8(src + lcup - 1) << 4) + (ld8(src + lcup - 2) & 0x0F);
    ok = (lcup - scup + 15) / 4 + 2 <= half_words;
    if (ok) {
      ms_len = lcup - scup;
      words = (ms_len + 15) / 4 + 2;
    }
  }
  unstuff_half(src, ms_len, Wg, words);
  const uint32_t hh = ok ? job.h : 0;
  const uint32_t hmax = max(hh, __shfl_xor_sync(0xFFFFFFFFu, hh, 16));
  const bool bad = magsgn_rows_half(job, ok, Wg, words, hmax, sym, dst);
  if (present && (!ok || bad)) {
    // No coded passes: zeros; an invalid stream: zeros and the tile's status.
    for (uint32_t y = 0; y < job.h; ++y)
      for (uint32_t x = gl; x < job.w; x += 16) dst[(size_t)y * job.stride + x] = 0;
    if (coded && gl == 0) atomicOr(&tile_status[job.tile], kStatusDecode);
  }
  __syncwarp();  // the warp's shared buffers are reused by its next work item
}

}  // namespace

// Pass 2: one warp per code block decodes magnitudes and signs
// (decode_magnitude_sign_phase, ht_block_decode.rs:1435-1561).  Grid form
// (queue == nullptr): warp k of CTA c takes block c * warps + k.  Queue form:
// a persistent grid whose warps take `gran` consecutive blocks at a time
// from the device work queue (an atomic counter over the job table, which is
// ordered by coded length, longest first).
//
// Work items: jobs [0, nsingle) one per warp; the narrow jobs after them
// (at most 32 wide, no refinement passes) two per warp, item nsingle + k
// taking jobs nsingle + 2k and nsingle + 2k + 1.
template <bool QUEUE>
__global__ void __launch_bounds__(kMsWarps * 32) ht_magsgn_kernel(const HtJob* __restrict__ jobs, uint32_t njobs,
                                                                  const uint8_t* __restrict__ arena,
                                                                  const uint32_t* __restrict__ symbols,
                                                                  int32_t* __restrict__ coef,
                                                                  uint32_t* __restrict__ tile_status,
                                                                  uint32_t ms_words, uint32_t max_w, uint32_t* queue,
                                                                  uint32_t gran, uint32_t nsingle) {
  extern __shared__ __align__(16) uint8_t smem[];
  const uint32_t nw = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t cols = max_w + 4;
  uint32_t* W = reinterpret_cast<uint32_t*>(smem) + (size_t)warp * ms_words;
  uint8_t* Ebase = smem + (size_t)nw * ms_words * 4 + (size_t)warp * 2 * cols;
  const uint32_t nitems = nsingle + (njobs - nsingle + 1) / 2;
  auto item = [&](uint32_t it) {
    if (it < nsingle) {
      magsgn_block(jobs[it], arena, symbols, coef, tile_status, ms_words, cols, W, Ebase);
    } else {
      const uint32_t a = nsingle + 2 * (it - nsingle);
      magsgn_pair(jobs, a, a + 1 < njobs ? a + 1 : 0xFFFFFFFFu, arena, symbols, coef, tile_status, ms_words / 2, W);
    }
  };
  if constexpr (!QUEUE) {
    const uint32_t it = blockIdx.x * nw + warp;
    if (it < nitems) item(it);
  } else {
    for (;;) {
      uint32_t base = 0;
      if (lane == 0) base = atomicAdd(queue, gran);
      base = __shfl_sync(0xFFFFFFFFu, base, 0);
      if (base >= nitems) break;
      const uint32_t end = min(base + gran, nitems);
      for (uint32_t it = base; it < end; ++it) item(it);
    }
  }
}

// Small plans: one CTA of two warps per code block runs both cleanup passes
// at once.  Lane 0 of warp 0 runs the block's VLC chain (decode_vlc) and
// publishes each finished quad row in shared memory; warp 1 unstuffs the
// MagSgn stream meanwhile and decodes each quad row's magnitudes and signs as
// soon as its symbols are out, so the block's MagSgn work hides behind its
// own chain instead of waiting for the slowest chain of the plan (a plan of
// one tile is as long as its longest block's chain).  Waits are bounded: a
// row that does not arrive within kFusedSpinLimit polls (tens of
// milliseconds, far beyond any chain) fails the block like an invalid
// stream.
namespace {

constexpr uint32_t kFusedThreads = 64;
constexpr uint32_t kRowsFailed = 0xFFFFFFFFu;
constexpr uint32_t kFusedSpinLimit = 1u << 20;

// The chain lane's row hook: the row's symbols, then its flag.  Its pair
// loop is unrolled twice (a fused plan runs few chains per SM, each on a
// warp of its own: 0.146 -> 0.139 ms for a 512^2 tile; the two-pass VLC
// kernel, 32 chains per warp, is slower unrolled).
struct FusedPublish {
  static constexpr bool kUnroll2 = true;
  volatile uint32_t* progress;
  __device__ void operator()(uint32_t rows) const {
    __threadfence_block();
    *progress = rows;
  }
};

struct FusedRowWait {
  static constexpr bool kLive = true;
  const volatile uint32_t* progress;  // quad rows published, or kRowsFailed
  __device__ bool operator()(uint32_t row) const {
    uint32_t ready = 1;
    if ((threadIdx.x & 31) == 0) {
      uint32_t p = *progress;
      for (uint32_t it = 0; p != kRowsFailed && p <= row && it < kFusedSpinLimit; ++it) {
        __nanosleep(32);
        p = *progress;
      }
      ready = p != kRowsFailed && p > row;
    }
    ready = __shfl_sync(0xFFFFFFFFu, ready, 0);
    __threadfence_block();  // the row's symbols are read after its flag
    return ready != 0;
  }
};

}  // namespace

template <bool OUTLINE>
__global__ void __launch_bounds__(kFusedThreads) ht_cleanup_fused_kernel(
    const HtJob* __restrict__ jobs, uint32_t njobs, const uint8_t* __restrict__ arena, uint32_t* __restrict__ symbols,
    int32_t* __restrict__ coef, uint32_t* __restrict__ tile_status, uint32_t ms_words, uint32_t max_w) {
  __shared__ SmemTables T;
  __shared__ uint2 stage[16];  // the chain lane's pairs of one row of a 64-wide block
  __shared__ uint32_t rows_done;
  extern __shared__ __align__(16) uint8_t smem[];
  {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(&g_ht_tables);
    uint32_t* d = reinterpret_cast<uint32_t*>(&T);
    for (uint32_t i = threadIdx.x; i < sizeof(SmemTables) / 4; i += blockDim.x) d[i] = src[i];
  }
  if (threadIdx.x == 0) rows_done = 0;
  __syncthreads();
  if (blockIdx.x >= njobs) return;
  const HtJob job = jobs[blockIdx.x];
  volatile uint32_t* progress = &rows_done;
  if (threadIdx.x < 32) {
    if (threadIdx.x != 0 || job.passes == 0) return;
    uint32_t* sym = symbols + job.sym;
    const FusedPublish publish{progress};
    const bool ok = job.w <= 64 ? decode_vlc<true, OUTLINE>(job, arena + job.src, sym, T, stage, 1, 0, publish)
                                : decode_vlc<false, OUTLINE>(job, arena + job.src, sym, T, stage, 1, 0, publish);
    if (!ok) {
      __threadfence_block();
      *progress = kRowsFailed;
    }
    return;
  }
  const uint32_t cols = max_w + 4;
  magsgn_block(job, arena, symbols, coef, tile_status, ms_words, cols, reinterpret_cast<uint32_t*>(smem),
               smem + (size_t)ms_words * 4, FusedRowWait{progress});
}

// ---------------------------------------------------------------------------
// Refinement passes for blocks with more than one coding pass.

namespace {

__device__ __forceinline__ uint32_t pair16(const uint16_t* v, uint32_t i) {
  return (uint32_t)v[i] | ((uint32_t)v[i + 1] << 16);
}

__device__ const uint32_t kSpread[16] = {0x33,   0x76,   0xEC,   0xC8,   0x330,   0x760,   0xEC0,   0xC80,
                                         0x3300, 0x7600, 0xEC00, 0xC800, 0x33000, 0x76000, 0xEC000, 0xC8000};

}  // namespace

// One thread per refinement block.  The block's cleanup result (raw
// sign-magnitude words written by ht_magsgn_kernel) gives the significance
// map; SigProp (ht_block_decode.rs:1254-1375) and MagRef (:1377-1433) then
// update the words in place, and the block is converted to int32.
__global__ void ht_refine_kernel(const HtJob* __restrict__ jobs, const uint32_t* __restrict__ list, uint32_t n,
                                 const uint8_t* __restrict__ arena, int32_t* __restrict__ coef,
                                 uint32_t* __restrict__ tile_status) {
  // sigma for blocks up to 4096 samples: rows (h/4 + 1) x stride ((w/4) + 2 + 7) & ~7.
  constexpr uint32_t kSigmaCap = 2560;
  uint16_t sigma[kSigmaCap];
  uint16_t prev_row[272];
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const HtJob job = jobs[list[k]];
    uint32_t* out = reinterpret_cast<uint32_t*>(coef + job.dst);
    const uint32_t w = job.w, h = job.h, stride = job.stride;
    const uint32_t mstr = (((w + 3) / 4) + 2 + 7) & ~7u;
    const uint32_t srows = (h + 3) / 4 + 1;
    bool ok = srows * mstr <= kSigmaCap && (w + 3) / 4 + 8 <= 272;
    const uint32_t p = 30 - job.mmsb;
    if (ok) {
      // Significance of the cleanup pass, 4-row stripes x 4-column groups
      // (build_sigma_from_cleanup_phase layout, :1207-1252).
      for (uint32_t i = 0; i < srows * mstr; ++i) sigma[i] = 0;
      for (uint32_t y = 0; y < h; ++y)
        for (uint32_t x = 0; x < w; ++x)
          if (out[(size_t)y * stride + x] != 0) {
            uint32_t idx = (y >> 2) * mstr + (x >> 2);
            sigma[idx] |= (uint16_t)(1u << (((x & 3) << 2) | (y & 3)));
          }
      const uint8_t* ref = arena + job.src + job.lcup;
      const uint32_t lref = job.lref;
      // SigProp.
      {
        uint32_t prl = (w + 3) / 4 + 8;
        for (uint32_t i = 0; i < prl; ++i) prev_row[i] = 0;
        Fwd<0> sp;
        sp.init(ref, lref);
        const bool causal = job.flags & 1;
        for (uint32_t y = 0; y < h; y += 4) {
          uint32_t pattern = 0xFFFF;
          if (h - y < 4) {
            pattern = 0x7777;
            if (h - y < 3) {
              pattern = 0x3333;
              if (h - y < 2) pattern = 0x1111;
            }
          }
          uint32_t prev = 0;
          uint32_t cur_row = (y >> 2) * mstr, next_row = cur_row + mstr;
          size_t dpp = (size_t)y * stride;
          for (uint32_t x = 0; x < w; x += 4) {
            uint32_t colp = pattern;
            int s = (int)x + 4 - (int)w;
            if (s < 0) s = 0;
            colp >>= (uint32_t)(s * 4);
            uint32_t idx = x >> 2;
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
            mbr &= colp;
            mbr &= ~cs;
            uint32_t new_sig = 0;
            if (mbr != 0) {
              uint32_t cwd = sp.fetch();
              uint32_t cnt = 0;
              uint32_t inv_sig = ~cs & colp;
              uint32_t cand = mbr, processed = 0;
              while (cand != 0) {
                uint32_t bit = __ffs(cand) - 1;
                uint32_t m = 1u << bit;
                cand &= ~m;
                processed |= m;
                if (cwd & 1) {
                  new_sig |= m;
                  cand |= kSpread[bit] & inv_sig & ~processed;
                }
                cwd >>= 1;
                ++cnt;
              }
              if (new_sig != 0) {
                uint32_t value = 3u << (p - 2);
                size_t bb = dpp + x;
                uint32_t sb = new_sig;
                while (sb != 0) {
                  uint32_t bit = __ffs(sb) - 1;
                  sb &= ~(1u << bit);
                  size_t off = (size_t)(bit >> 2) + (size_t)(bit & 3) * stride;
                  out[bb + off] = ((cwd & 1) << 31) | value;
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
      // MagRef.
      if (job.passes > 2) {
        if (p < 2) {
          ok = false;
        } else {
          // Backward reader over the refinement segment (new_mrp).
          Vlc mr;
          mr.init_mrp(ref, lref);
          uint32_t half = 1u << (p - 2);
          for (uint32_t y = 0; y < h; y += 4) {
            uint32_t csi = (y >> 2) * mstr;
            size_t dpp = (size_t)y * stride;
            for (uint32_t i = 0; i < w; i += 8) {
              uint32_t cwd = mr.fetch();
              uint32_t sig = pair16(sigma, csi);
              csi += 2;
              uint32_t col_mask = 0xF;
              if (sig != 0) {
                for (uint32_t j = 0; j < 8; ++j) {
                  if (sig & col_mask) {
                    size_t dp = dpp + i + j;
                    uint32_t sm = 0x11111111u & col_mask;
                    for (int kk = 0; kk < 4; ++kk) {
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
              mr.advance(__popc(sig));
            }
          }
        }
      }
    }
    // Convert to int32 coefficients (or zero the block on failure).
    for (uint32_t y = 0; y < h; ++y)
      for (uint32_t x = 0; x < w; ++x) {
        uint32_t& v = out[(size_t)y * stride + x];
        v = ok ? (uint32_t)to_i32(v, job.nbp) : 0u;
      }
    if (!ok) atomicOr(&tile_status[job.tile], kStatusDecode);
  }
}

size_t ht_magsgn_smem_bytes(uint32_t ms_words, uint32_t max_w, uint32_t warps) {
  return (size_t)warps * ms_words * 4 + (size_t)warps * 2 * (max_w + 4);
}

cudaError_t ht_kernels_init() {
  // The VLC pass's lanes read their blocks' bytes a few at a time over the
  // whole chain, so its L1 hit rate matters more than a ninth resident CTA:
  // left to itself the driver sizes shared memory for the CTAs that the
  // registers allow (228 KB, 28 KB of L1); 72 % (164 KB, 7 CTAs of 21.6 KB)
  // leaves 92 KB of L1 (C2 VLC pass 0.96 -> 0.88 ms).
  for (const void* k : {(const void*)ht_vlc_kernel<true>, (const void*)ht_vlc_kernel<false>}) {
    const cudaError_t c = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 72);
    if (c != cudaSuccess) return c;
  }
  for (const void* k : {(const void*)ht_cleanup_fused_kernel<true>, (const void*)ht_cleanup_fused_kernel<false>}) {
    const cudaError_t c = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (c != cudaSuccess) return c;
  }
  cudaError_t e = cudaFuncSetAttribute(ht_magsgn_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(ht_magsgn_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
}

cudaError_t launch_ht_vlc(const HtJob* jobs, uint32_t njobs, const uint8_t* arena, uint32_t* symbols,
                          cudaStream_t stream, uint32_t threads, uint32_t lanes, bool outline) {
  if (njobs == 0) return cudaSuccess;
  if (threads == 0 || threads > kHtThreads || threads % 32) threads = kHtThreads;
  if (lanes == 0 || lanes > 32 || (lanes & (lanes - 1))) lanes = 32;
  const uint32_t warps = (njobs + lanes - 1) / lanes, per_cta = threads / 32;
  const uint32_t grid = (warps + per_cta - 1) / per_cta;
  if (outline) ht_vlc_kernel<true><<<grid, threads, 0, stream>>>(jobs, njobs, arena, symbols, lanes);
  else ht_vlc_kernel<false><<<grid, threads, 0, stream>>>(jobs, njobs, arena, symbols, lanes);
  return cudaGetLastError();
}

cudaError_t launch_ht_fused(const HtJob* jobs, uint32_t njobs, const uint8_t* arena, uint32_t* symbols, int32_t* coef,
                           uint32_t* tile_status, uint32_t ms_words, uint32_t max_w, cudaStream_t stream,
                           bool outline) {
  if (njobs == 0) return cudaSuccess;
  const size_t smem = ht_magsgn_smem_bytes(ms_words, max_w, 1);
  if (smem > 200 * 1024) return cudaErrorInvalidValue;
  if (outline)
    ht_cleanup_fused_kernel<true><<<njobs, kFusedThreads, smem, stream>>>(jobs, njobs, arena, symbols, coef,
                                                                          tile_status, ms_words, max_w);
  else
    ht_cleanup_fused_kernel<false><<<njobs, kFusedThreads, smem, stream>>>(jobs, njobs, arena, symbols, coef,
                                                                           tile_status, ms_words, max_w);
  return cudaGetLastError();
}

cudaError_t launch_ht_magsgn(const HtJob* jobs, uint32_t njobs, const uint8_t* arena, const uint32_t* symbols,
                             int32_t* coef, uint32_t* tile_status, uint32_t ms_words, uint32_t max_w,
                             cudaStream_t stream, uint32_t warps, uint32_t* queue, uint32_t gran,
                             uint32_t persistent_ctas, uint32_t nsingle) {
  if (njobs == 0) return cudaSuccess;
  if (warps == 0 || warps > kMsWarps) warps = kMsWarps;
  nsingle = std::min(nsingle, njobs);
  size_t smem = ht_magsgn_smem_bytes(ms_words, max_w, warps);
  if (smem > 227 * 1024) return cudaErrorInvalidValue;
  const uint32_t nitems = nsingle + (njobs - nsingle + 1) / 2;
  uint32_t ctas = (nitems + warps - 1) / warps;
  if (queue) {
    if (gran == 0) gran = 1;
    ctas = std::max(1u, std::min(ctas, persistent_ctas));
  }
  if (queue)
    ht_magsgn_kernel<true><<<ctas, warps * 32, smem, stream>>>(jobs, njobs, arena, symbols, coef, tile_status,
                                                               ms_words, max_w, queue, gran, nsingle);
  else
    ht_magsgn_kernel<false><<<ctas, warps * 32, smem, stream>>>(jobs, njobs, arena, symbols, coef, tile_status,
                                                                ms_words, max_w, nullptr, 0, nsingle);
  return cudaGetLastError();
}

cudaError_t ht_magsgn_occupancy(uint32_t ms_words, uint32_t max_w, uint32_t warps, int* ctas_per_sm) {
  if (warps == 0 || warps > kMsWarps) warps = kMsWarps;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, ht_magsgn_kernel<true>, warps * 32,
                                                       ht_magsgn_smem_bytes(ms_words, max_w, warps));
}

cudaError_t launch_ht_cleanup(const HtJob* jobs, uint32_t njobs, const uint8_t* arena, uint32_t* symbols,
                              int32_t* coef, uint32_t* tile_status, uint32_t ms_words, uint32_t max_w,
                              cudaStream_t stream) {
  cudaError_t e = launch_ht_vlc(jobs, njobs, arena, symbols, stream, kHtThreads);
  if (e != cudaSuccess) return e;
  return launch_ht_magsgn(jobs, njobs, arena, symbols, coef, tile_status, ms_words, max_w, stream, kMsWarps, nullptr,
                          0, 0, njobs);
}

cudaError_t launch_ht_refine(const HtJob* jobs, const uint32_t* list, uint32_t n, const uint8_t* arena, int32_t* coef,
                             uint32_t* tile_status, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  uint32_t threads = 64, blocks = (n + threads - 1) / threads;
  ht_refine_kernel<<<blocks, threads, 0, stream>>>(jobs, list, n, arena, coef, tile_status);
  return cudaGetLastError();
}

cudaError_t upload_ht_tables(const HtDecodeTables& host) {
  return cudaMemcpyToSymbol(g_ht_tables, &host, sizeof(HtDecodeTables));
}

}  // namespace sgn
