// HT code-block decoding on sm_100a.
//
// Decodes HTJ2K code blocks (T.814) into sign-magnitude coefficients and
// writes them as int32 sub-band samples, bit-exact with the reference's
// decode_impl (crates/signinum-j2k-native/src/j2c/ht_block_decode.rs:1563-1683)
// followed by coefficient_to_i32 (:225-234).
//
// Work mapping: one thread decodes one code block; the blocks of a launch are
// ordered by coded length on the host so the 32 blocks of a warp carry
// similar work.  The cleanup pass is fused row by row: for each quad row the
// thread runs the MEL/VLC/UVLC chain (the serial part) and immediately the
// magnitude/sign pass of that row, so the only per-block state is one row of
// quad symbols and exponents, kept in shared memory (no global scratch).
// Refinement passes (SigProp/MagRef) run in ht_refine_kernel for the few
// blocks that carry them.
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

// MEL run decoder (ht_block_decode.rs:782-880).
struct Mel {
  const uint8_t* data;
  uint32_t pos, remaining;
  uint32_t unstuff, cur, bits_left;
  int k, num_runs;
  uint64_t runs;
  __device__ void init(const uint8_t* d, uint32_t lcup, uint32_t scup) {
    data = d;
    pos = lcup - scup;
    remaining = scup - 1;
    unstuff = 0;
    cur = 0;
    bits_left = 0;
    k = 0;
    num_runs = 0;
    runs = 0;
  }
  __device__ __forceinline__ uint32_t bit() {
    if (bits_left == 0) {
      uint32_t b;
      if (remaining > 0) {
        b = ld8(data + pos);
        ++pos;
        --remaining;
      } else {
        b = 0xFF;
      }
      if (remaining == 0) b |= 0x0F;
      cur = b;
      bits_left = 8 - unstuff;
      unstuff = b == 0xFF;
    }
    --bits_left;
    return (cur >> bits_left) & 1;
  }
  __device__ void more() {
    while (num_runs < 8) {
      // MEL exponent table {0,0,0,1,1,1,2,2,2,3,3,4,5}.
      int e = (k < 3) ? 0 : (k < 6) ? 1 : (k < 9) ? 2 : (k < 11) ? 3 : (k == 11) ? 4 : 5;
      uint32_t first = bit();
      uint64_t run;
      if (first) {
        k = k + 1 < 12 ? k + 1 : 12;
        run = ((1ull << e) - 1) << 1;
      } else {
        k = k > 0 ? k - 1 : 0;
        uint32_t v = 0;
        for (int i = 0; i < e; ++i) v = (v << 1) | bit();
        run = ((uint64_t)v << 1) | 1;
      }
      runs |= run << (num_runs * 7);
      ++num_runs;
      if (e == 5 && first == 0 && num_runs >= 8) break;
    }
  }
  __device__ __forceinline__ int get_run() {
    if (num_runs == 0) more();
    int r = (int)(runs & 0x7F);
    runs >>= 7;
    --num_runs;
    return r;
  }
};

// Backward VLC reader (ht_block_decode.rs:932-1000, new_vlc).
struct Vlc {
  const uint8_t* data;
  int pos;
  uint32_t remaining;
  uint64_t tmp;
  uint32_t bits, unstuff;
  __device__ void init(const uint8_t* d, uint32_t lcup, uint32_t scup) {
    data = d;
    uint32_t b = ld8(d + lcup - 2);
    tmp = b >> 4;
    bits = 4 - (((tmp & 7) == 7) ? 1 : 0);
    pos = (int)lcup - 3;
    remaining = scup - 2;
    unstuff = (b | 0x0F) > 0x8F;
  }
  __device__ __forceinline__ void fill() {
    while (bits <= 32) {
      uint32_t b = 0;
      if (remaining > 0) {
        b = ld8(data + pos);
        --pos;
        --remaining;
      }
      uint32_t db = 8 - ((unstuff && (b & 0x7F) == 0x7F) ? 1 : 0);
      tmp |= (uint64_t)b << bits;
      bits += db;
      unstuff = b > 0x8F;
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

__device__ __forceinline__ uint32_t bitlen(uint32_t v) { return 32 - __clz(v); }

__device__ __forceinline__ int32_t to_i32(uint32_t v, uint32_t nbp) {
  uint32_t shift = nbp >= 31 ? 0 : 31 - nbp;
  int32_t m = (int32_t)((v & 0x7FFFFFFFu) >> shift);
  return (v & 0x80000000u) ? -m : m;
}

// decode_mag_sgn_sample_with_vn (ht_block_decode.rs:1010-1032).
__device__ __forceinline__ uint32_t magsgn_sample(Fwd<0xFF>& ms, uint32_t inf, uint32_t bit, uint32_t uq, uint32_t p,
                                                  uint32_t& vn) {
  if ((inf & (1u << (4 + bit))) == 0) {
    vn = 0;
    return 0;
  }
  uint32_t msv = ms.fetch();
  uint32_t m_n = uq - ((inf >> (12 + bit)) & 1);
  ms.advance(m_n);
  uint32_t value = msv << 31;
  uint32_t mask = m_n == 0 ? 0 : (m_n >= 32 ? 0xFFFFFFFFu : ((1u << m_n) - 1));
  uint32_t v = msv & mask;
  v |= ((inf >> (8 + bit)) & 1) << m_n;
  v |= 1;
  value |= (v + 2) << (p - 1);
  vn = v;
  return value;
}

// Per-thread row state in shared memory, interleaved by thread so that the
// threads of a warp hit distinct banks.
struct RowState {
  uint16_t* prevT;  // quad symbols of the previous quad row
  uint16_t* curT;   // quad symbols of this row
  uint8_t* curU;    // u_q of this row (initial row: u_q + 1)
  uint8_t* vE;      // exponent bound from the row above, per quad boundary
  uint32_t step;    // element stride between consecutive entries of one thread
  __device__ __forceinline__ uint16_t& pt(uint32_t i) { return prevT[i * step]; }
  __device__ __forceinline__ uint16_t& ct(uint32_t i) { return curT[i * step]; }
  __device__ __forceinline__ uint8_t& cu(uint32_t i) { return curU[i * step]; }
  __device__ __forceinline__ uint8_t& ve(uint32_t i) { return vE[i * step]; }
};

__device__ void zero_block(int32_t* dst, uint32_t stride, uint32_t w, uint32_t h) {
  for (uint32_t y = 0; y < h; ++y)
    for (uint32_t x = 0; x < w; ++x) dst[(size_t)y * stride + x] = 0;
}

// Cleanup + magnitude/sign decode of one block (decode_cleanup_symbols,
// ht_block_decode.rs:1056-1205, and decode_magnitude_sign_phase, :1435-1561,
// fused per quad row).  Returns false where the reference returns None.
__device__ bool decode_cleanup(const HtJob& job, const uint8_t* src, int32_t* dst, RowState& st,
                               const SmemTables& T) {
  const uint32_t lcup = job.lcup, w = job.w, h = job.h, stride = job.stride;
  if (lcup < 2) return false;
  uint32_t scup = ((uint32_t)ld8(src + lcup - 1) << 4) + (ld8(src + lcup - 2) & 0x0F);
  if (scup < 2 || scup > lcup || scup > 4079) return false;
  const uint32_t mmsb = job.mmsb, p = 30 - mmsb, mmsbp2 = mmsb + 2;
  const bool raw = job.passes > 1;  // keep sign-magnitude words for the refinement kernel
  const uint32_t nbp = job.nbp;
  Mel mel;
  mel.init(src, lcup, scup);
  Vlc vlc;
  vlc.init(src, lcup, scup);
  Fwd<0xFF> ms;
  ms.init(src, lcup - scup);
  int run = mel.get_run();
  const uint32_t nq = (w + 1) / 2;
  for (uint32_t i = 0; i < nq + 3; ++i) st.pt(i) = 0;
  for (uint32_t i = 0; i < nq + 2; ++i) st.ve(i) = 0;
  for (uint32_t y = 0; y < h; y += 2) {
    const bool initial = y == 0;
    // ---- CxtVLC / MEL / UVLC for this quad row.
    uint32_t c_q = 0;
    uint32_t q = 0;
    for (uint32_t x = 0; x < w; q += 2) {
      uint32_t t0, t1, ue;
      uint32_t v = vlc.fetch();
      if (initial) {
        t0 = T.vlc0[c_q + (v & 0x7F)];
        if (c_q == 0) {
          run -= 2;
          t0 = run == -1 ? t0 : 0;
          if (run < 0) run = mel.get_run();
        }
        st.ct(q) = (uint16_t)t0;
        x += 2;
        c_q = ((t0 & 0x10) << 3) | ((t0 & 0xE0) << 2);
        v = vlc.advance(t0 & 7);
        t1 = T.vlc0[c_q + (v & 0x7F)];
        if (c_q == 0 && x < w) {
          run -= 2;
          t1 = run == -1 ? t1 : 0;
          if (run < 0) run = mel.get_run();
        }
        if (x >= w) t1 = 0;
        st.ct(q + 1) = (uint16_t)t1;
        x += 2;
        c_q = ((t1 & 0x10) << 3) | ((t1 & 0xE0) << 2);
        v = vlc.advance(t1 & 7);
        uint32_t mode = ((t0 & 8) << 3) | ((t1 & 8) << 4);
        if (mode == 0xC0) {
          run -= 2;
          if (run == -1) mode += 0x40;
          if (run < 0) run = mel.get_run();
        }
        ue = T.uvlc0[mode + (v & 0x3F)];
      } else {
        uint32_t pq0 = st.pt(q), pq1 = st.pt(q + 1), pq2 = st.pt(q + 2);
        c_q |= (pq0 & 0xA0) << 2;
        c_q |= (pq1 & 0x20) << 4;
        t0 = T.vlc1[c_q + (v & 0x7F)];
        if (c_q == 0) {
          run -= 2;
          t0 = run == -1 ? t0 : 0;
          if (run < 0) run = mel.get_run();
        }
        st.ct(q) = (uint16_t)t0;
        x += 2;
        c_q = ((t0 & 0x40) << 2) | ((t0 & 0x80) << 1);
        c_q |= pq0 & 0x80;
        c_q |= (pq1 & 0xA0) << 2;
        c_q |= (pq2 & 0x20) << 4;
        v = vlc.advance(t0 & 7);
        t1 = T.vlc1[c_q + (v & 0x7F)];
        if (c_q == 0 && x < w) {
          run -= 2;
          t1 = run == -1 ? t1 : 0;
          if (run < 0) run = mel.get_run();
        }
        if (x >= w) t1 = 0;
        st.ct(q + 1) = (uint16_t)t1;
        x += 2;
        c_q = ((t1 & 0x40) << 2) | ((t1 & 0x80) << 1);
        c_q |= pq1 & 0x80;
        v = vlc.advance(t1 & 7);
        uint32_t mode = ((t0 & 8) << 3) | ((t1 & 8) << 4);
        ue = T.uvlc1[mode + (v & 0x3F)];
      }
      v = vlc.advance(ue & 7);
      ue >>= 3;
      uint32_t len = ue & 0xF;
      uint32_t tmp = v & ((1u << len) - 1);
      vlc.advance(len);
      ue >>= 4;
      len = ue & 7;
      ue >>= 3;
      uint32_t add = initial ? 1 : 0;
      st.cu(q) = (uint8_t)(add + (ue & 7) + (tmp & ~(0xFFu << len)));
      st.cu(q + 1) = (uint8_t)(add + (ue >> 3) + (tmp >> len));
    }
    st.ct(q) = 0;
    st.ct(q + 1) = 0;
    st.ct(q + 2) = 0;
    // ---- Magnitude/sign for this quad row.
    const bool second = y + 1 < h;
    int32_t* row0 = dst + (size_t)y * stride;
    int32_t* row1 = row0 + stride;
    uint32_t prev_v3 = 0;
    uint32_t x = 0;
    for (uint32_t qi = 0; x < w; ++qi) {
      uint32_t inf = st.ct(qi);
      uint32_t uq = st.cu(qi);
      if (!initial) {
        uint32_t gamma = inf & 0xF0;
        gamma &= gamma - 0x10;
        uint32_t e = max((uint32_t)st.ve(qi), (uint32_t)st.ve(qi + 1));
        uint32_t emax = max(e, 2u) - 1;
        uq += gamma != 0 ? emax : 1;
      }
      if (uq > mmsbp2) return false;
      uint32_t v0, v1, v2, v3;
      uint32_t a0 = magsgn_sample(ms, inf, 0, uq, p, v0);
      uint32_t a1 = magsgn_sample(ms, inf, 1, uq, p, v1);
      if (raw) {
        row0[x] = (int32_t)a0;
        if (second) row1[x] = (int32_t)a1;
      } else {
        row0[x] = to_i32(a0, nbp);
        if (second) row1[x] = to_i32(a1, nbp);
      }
      st.ve(qi) = (uint8_t)bitlen(prev_v3 | v1);
      prev_v3 = 0;
      ++x;
      if (x >= w) {
        st.ve(qi + 1) = 0;
        break;
      }
      uint32_t a2 = magsgn_sample(ms, inf, 2, uq, p, v2);
      uint32_t a3 = magsgn_sample(ms, inf, 3, uq, p, v3);
      if (raw) {
        row0[x] = (int32_t)a2;
        if (second) row1[x] = (int32_t)a3;
      } else {
        row0[x] = to_i32(a2, nbp);
        if (second) row1[x] = to_i32(a3, nbp);
      }
      prev_v3 = v3;
      ++x;
      if (x >= w) st.ve(qi + 1) = (uint8_t)bitlen(prev_v3);
    }
    // This row's symbols become the context of the next row.
    for (uint32_t i = 0; i < nq + 3; ++i) st.pt(i) = st.ct(i);
  }
  return true;
}

}  // namespace

__global__ void __launch_bounds__(kHtThreads) ht_cleanup_kernel(const HtJob* __restrict__ jobs, uint32_t njobs,
                                                                 const uint8_t* __restrict__ arena,
                                                                 int32_t* __restrict__ coef,
                                                                 uint32_t* __restrict__ tile_status, uint32_t max_nq) {
  extern __shared__ __align__(16) uint8_t smem[];
  SmemTables& T = *reinterpret_cast<SmemTables*>(smem);
  {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(&g_ht_tables);
    uint32_t* dstw = reinterpret_cast<uint32_t*>(smem);
    for (uint32_t i = threadIdx.x; i < sizeof(SmemTables) / 4; i += blockDim.x) dstw[i] = src[i];
  }
  __syncthreads();
  const uint32_t rows = max_nq + 4;
  uint8_t* base = smem + sizeof(SmemTables);
  RowState st;
  st.step = blockDim.x;
  st.prevT = reinterpret_cast<uint16_t*>(base) + threadIdx.x;
  st.curT = reinterpret_cast<uint16_t*>(base) + (size_t)rows * blockDim.x + threadIdx.x;
  uint8_t* b8 = base + (size_t)rows * blockDim.x * 4;
  st.curU = b8 + threadIdx.x;
  st.vE = b8 + (size_t)rows * blockDim.x + threadIdx.x;
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < njobs; j += gridDim.x * blockDim.x) {
    const HtJob job = jobs[j];
    int32_t* dst = coef + job.dst;
    if (job.passes == 0) {
      zero_block(dst, job.stride, job.w, job.h);
      continue;
    }
    if ((uint32_t)((job.w + 1) / 2) > max_nq || !decode_cleanup(job, arena + job.src, dst, st, T)) {
      zero_block(dst, job.stride, job.w, job.h);
      atomicOr(&tile_status[job.tile], kStatusDecode);
    }
  }
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
// sign-magnitude words written by ht_cleanup_kernel) gives the significance
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
          mr.data = ref;
          mr.pos = (int)lref - 1;
          mr.remaining = lref;
          mr.tmp = 0;
          mr.bits = 0;
          mr.unstuff = 1;
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

size_t ht_cleanup_smem_bytes(uint32_t max_nq, uint32_t threads) {
  size_t rows = max_nq + 4;
  return sizeof(SmemTables) + rows * threads * 6;
}

cudaError_t ht_kernels_init() {
  cudaError_t e = cudaFuncSetAttribute(ht_cleanup_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
  return e;
}

cudaError_t launch_ht_cleanup(const HtJob* jobs, uint32_t njobs, const uint8_t* arena, int32_t* coef,
                              uint32_t* tile_status, uint32_t max_nq, cudaStream_t stream) {
  if (njobs == 0) return cudaSuccess;
  // Wide code blocks need more row state per thread: shrink the CTA so the
  // row state stays within the shared-memory budget.
  uint32_t threads = kHtThreads;
  while (threads > 32 && ht_cleanup_smem_bytes(max_nq, threads) > 200 * 1024) threads /= 2;
  size_t smem = ht_cleanup_smem_bytes(max_nq, threads);
  uint32_t blocks = (njobs + threads - 1) / threads;
  ht_cleanup_kernel<<<blocks, threads, smem, stream>>>(jobs, njobs, arena, coef, tile_status, max_nq);
  return cudaGetLastError();
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
