// Classic JPEG 2000 Tier-1 (EBCOT) data shared by the device decoder and the
// host encoder of test inputs: the MQ coder's probability estimation table
// (ISO/IEC 15444-1 Table C.2, as in the reference's
// crates/signinum-j2k-native/src/j2c/arithmetic_decoder.rs:333-386), the
// initial context states (Table D.7) and the context rules of Tables D.1,
// D.3 and D.4 over the neighbour-significance byte the reference keeps per
// coefficient (bitplane.rs:370-420): top-left 7, top 6, top-right 5, left 4,
// bottom-left 3, right 2, bottom-right 1, bottom 0.
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define SGN_HD __host__ __device__
#else
#define SGN_HD
#endif

namespace sgn {
namespace ebcot {

// Code-block style bits (COD/COC SPcod "code-block style").
constexpr uint8_t kBypass = 0x01, kReset = 0x02, kTermAll = 0x04, kVCausal = 0x08, kSegSym = 0x20;

// Table C.2: Qe, NMPS, NLPS, SWITCH for indices 0..46.
constexpr uint16_t kQe[47] = {0x5601, 0x3401, 0x1801, 0x0AC1, 0x0521, 0x0221, 0x5601, 0x5401, 0x4801, 0x3801,
                              0x3001, 0x2401, 0x1C01, 0x1601, 0x5601, 0x5401, 0x5101, 0x4801, 0x3801, 0x3401,
                              0x3001, 0x2801, 0x2401, 0x2201, 0x1C01, 0x1801, 0x1601, 0x1401, 0x1201, 0x1101,
                              0x0AC1, 0x09C1, 0x08A1, 0x0521, 0x0441, 0x02A1, 0x0221, 0x0141, 0x0111, 0x0085,
                              0x0049, 0x0025, 0x0015, 0x0009, 0x0005, 0x0001, 0x5601};
constexpr uint8_t kNmps[47] = {1,  2,  3,  4,  5,  38, 7,  8,  9,  10, 11, 12, 13, 29, 15, 16,
                               17, 18, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 32,
                               33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43, 44, 45, 45, 46};
constexpr uint8_t kNlps[47] = {1,  6,  9,  12, 29, 33, 6,  14, 14, 14, 17, 18, 20, 21, 14, 14,
                               15, 16, 17, 18, 19, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29,
                               30, 31, 32, 33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43, 46};
constexpr uint8_t kSwitch[47] = {1, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0,
                                 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};

// Context labels: 0..8 zero coding, 9..13 sign, 14..16 refinement,
// 17 run length, 18 uniform.  Initial indices (Table D.7): 4 for label 0,
// 3 for run length, 46 for uniform, 0 for the rest; MPS 0.
SGN_HD inline uint8_t initial_index(int label) { return label == 0 ? 4 : label == 17 ? 3 : label == 18 ? 46 : 0; }

// Band classes of Table D.1: LL and LH share one rule, HL swaps the roles of
// horizontal and vertical neighbours, HH counts diagonals first.
enum BandClass : uint8_t { kLlLh = 0, kHl = 1, kHh = 2 };

// Table D.1: zero-coding context from the neighbour-significance byte.
SGN_HD inline uint8_t zc_context(uint8_t n, uint8_t band) {
  const int h = ((n >> 4) & 1) + ((n >> 2) & 1);
  const int v = ((n >> 6) & 1) + (n & 1);
  const int d = ((n >> 7) & 1) + ((n >> 5) & 1) + ((n >> 3) & 1) + ((n >> 1) & 1);
  if (band == kHh) {
    const int hv = h + v;
    if (d >= 3) return 8;
    if (d == 2) return hv >= 1 ? 7 : 6;
    if (d == 1) return hv >= 2 ? 5 : (hv == 1 ? 4 : 3);
    return (uint8_t)(hv >= 2 ? 2 : hv);
  }
  const int a = band == kHl ? v : h, b = band == kHl ? h : v;
  if (a == 2) return 8;
  if (a == 1) return b >= 1 ? 7 : (d >= 1 ? 6 : 5);
  if (b == 2) return 4;
  if (b == 1) return 3;
  return (uint8_t)(d >= 2 ? 2 : d);
}

// Table D.3: sign-coding context label and XOR bit from 2-bit (negative,
// positive) fields of the top (bits 6-7), left (4-5), right (2-3) and bottom
// (0-1) neighbours.
SGN_HD inline void sc_context(uint8_t m, uint8_t& label, uint8_t& xr) {
  const int left = (int)((m >> 4) & 1) - (int)((m >> 5) & 1), right = (int)((m >> 2) & 1) - (int)((m >> 3) & 1);
  const int top = (int)((m >> 6) & 1) - (int)((m >> 7) & 1), bottom = (int)(m & 1) - (int)((m >> 1) & 1);
  int hc = left + right, vc = top + bottom;
  hc = hc > 1 ? 1 : (hc < -1 ? -1 : hc);
  vc = vc > 1 ? 1 : (vc < -1 ? -1 : vc);
  if (hc == 0) {
    label = (uint8_t)(vc == 0 ? 9 : 10);
    xr = vc < 0 ? 1 : 0;
  } else {
    label = (uint8_t)(vc == 0 ? 12 : (vc == hc ? 13 : 11));
    xr = hc < 0 ? 1 : 0;
  }
}

// Table D.4: magnitude-refinement context.
SGN_HD inline uint8_t mr_context(bool refined, uint8_t n) { return refined ? 16 : (uint8_t)(n ? 15 : 14); }

// Coding-pass segments (segment_idx_for_bypass, segment.rs:585-591): with
// arithmetic-coding bypass, passes 0..9 form segment 0, then each bit-plane
// has a raw segment (significance propagation + refinement) and an MQ one
// (cleanup).
SGN_HD inline uint32_t bypass_segment(uint32_t pass) {
  return pass < 10 ? 0 : 1 + 2 * ((pass - 10) / 3) + ((pass - 10) % 3 == 2 ? 1 : 0);
}

// Whether the segment starting at `pass` is MQ coded (bitplane.rs:154-166).
SGN_HD inline bool segment_is_arithmetic(uint8_t style, uint32_t pass) {
  return !(style & kBypass) || pass <= 9 || pass % 3 == 0;
}

}  // namespace ebcot
}  // namespace sgn

#undef SGN_HD
