// HTJ2K lookup tables built from the CxtVLC codeword rows (T.814 Annex C).
//
// Decoder form: a 7-bit lookup per VLC context, packed as
//   bits 0-2 codeword length, bit 3 u_off, bits 4-7 rho, bits 8-11 e_1,
//   bits 12-15 e_k
// (the layout consumed by the reference's cleanup decoder,
// crates/signinum-j2k-native/src/j2c/ht_tables.rs:3,92), and the UVLC prefix
// lookups (ht_tables.rs:181,211) generated from the UVLC code definition.
// Encoder form: for each (table, context, rho, u_off, emb) the cheapest
// codeword whose e_1 equals emb & e_k.
#pragma once

#include <cstdint>
#include <cstring>

namespace sgn {

#include "tables/cxtvlc_rows.inc"

struct HtDecodeTables {
  uint16_t vlc[2][1024];  // [initial row?0:1][(c_q << 7) | next 7 bits]
  uint16_t uvlc0[320];    // initial row: modes 0x00..0x100
  uint16_t uvlc1[256];    // other rows: modes 0x00..0xC0
};

struct HtEncodeEntry {
  uint8_t cwd, len, e_k, valid;
};

struct HtEncodeTables {
  // [table][c_q][rho][u_off][emb]
  HtEncodeEntry e[2][8][16][2][16];
};

// UVLC prefix read LSB-first: "1" -> 1, "01" -> 2, "001" -> 3 (+1 suffix bit),
// "000" -> 5 (+5 suffix bits).
inline void uvlc_prefix(uint32_t bits, uint32_t& pfx, uint32_t& plen, uint32_t& slen) {
  if (bits & 1) { pfx = 1; plen = 1; slen = 0; }
  else if (bits & 2) { pfx = 2; plen = 2; slen = 0; }
  else if (bits & 4) { pfx = 3; plen = 3; slen = 1; }
  else { pfx = 5; plen = 3; slen = 5; }
}

// mode: 0 none, 1 first quad only, 2 second only, 3 both, 4 both after a MEL
// "both above two" event (initial row only, each prefix value raised by 2).
inline uint16_t uvlc_lookup_entry(uint32_t mode, uint32_t bits, bool initial_row) {
  uint32_t p0 = 0, l0 = 0, s0 = 0, p1 = 0, l1 = 0, s1 = 0;
  if (mode == 0) return 0;
  if (mode == 1) {
    uvlc_prefix(bits, p0, l0, s0);
  } else if (mode == 2) {
    uvlc_prefix(bits, p1, l1, s1);
  } else if (mode == 3) {
    uvlc_prefix(bits, p0, l0, s0);
    if (initial_row && p0 > 2) {
      // Initial-row pair whose first u_q exceeds 2: the second u_q (1 or 2)
      // is sent as one raw bit.
      p1 = 1 + ((bits >> l0) & 1);
      l1 = 1;
      s1 = 0;
    } else {
      uvlc_prefix(bits >> l0, p1, l1, s1);
    }
  } else {
    uvlc_prefix(bits, p0, l0, s0);
    uvlc_prefix(bits >> l0, p1, l1, s1);
    p0 += 2;
    p1 += 2;
  }
  return (uint16_t)((l0 + l1) | ((s0 + s1) << 3) | (s0 << 7) | (p0 << 10) | (p1 << 13));
}

inline void build_decode_tables(HtDecodeTables& t) {
  std::memset(&t, 0, sizeof(t));
  const unsigned char(*rows[2])[7] = {CXTVLC_ROWS_INITIAL, CXTVLC_ROWS_NONINITIAL};
  const int counts[2] = {CXTVLC_ROWS_INITIAL_COUNT, CXTVLC_ROWS_NONINITIAL_COUNT};
  for (int tb = 0; tb < 2; ++tb)
    for (int i = 0; i < counts[tb]; ++i) {
      const unsigned char* r = rows[tb][i];
      uint32_t len = r[2];
      uint16_t e = (uint16_t)((r[5] << 12) | (r[6] << 8) | (r[3] << 4) | (r[4] << 3) | len);
      for (uint32_t b = 0; b < 128; ++b)
        if ((b & ((1u << len) - 1)) == r[1]) t.vlc[tb][((uint32_t)r[0] << 7) | b] = e;
    }
  for (uint32_t m = 0; m < 5; ++m)
    for (uint32_t b = 0; b < 64; ++b) t.uvlc0[m * 64 + b] = uvlc_lookup_entry(m, b, true);
  for (uint32_t m = 0; m < 4; ++m)
    for (uint32_t b = 0; b < 64; ++b) t.uvlc1[m * 64 + b] = uvlc_lookup_entry(m, b, false);
}

inline void build_encode_tables(HtEncodeTables& t) {
  std::memset(&t, 0, sizeof(t));
  const unsigned char(*rows[2])[7] = {CXTVLC_ROWS_INITIAL, CXTVLC_ROWS_NONINITIAL};
  const int counts[2] = {CXTVLC_ROWS_INITIAL_COUNT, CXTVLC_ROWS_NONINITIAL_COUNT};
  for (int tb = 0; tb < 2; ++tb)
    for (int i = 0; i < counts[tb]; ++i) {
      const unsigned char* r = rows[tb][i];
      uint32_t cq = r[0], cwd = r[1], len = r[2], rho = r[3], uoff = r[4], ek = r[5], e1 = r[6];
      for (uint32_t emb = 0; emb < 16; ++emb) {
        if (uoff == 0 && emb != 0) continue;
        if (uoff == 1 && ((emb & ek) != e1)) continue;
        HtEncodeEntry& d = t.e[tb][cq][rho][uoff][emb];
        int pc = __builtin_popcount(ek), dpc = __builtin_popcount(d.e_k);
        if (!d.valid || pc > dpc || (pc == dpc && len < d.len)) {
          d.cwd = (uint8_t)cwd;
          d.len = (uint8_t)len;
          d.e_k = (uint8_t)ek;
          d.valid = 1;
        }
      }
    }
}

}  // namespace sgn
