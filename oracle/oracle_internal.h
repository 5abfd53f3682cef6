// TEST INFRASTRUCTURE ONLY — the parity oracle.
//
// A CPU restatement of the reference's pure-Rust HTJ2K decoder
// (frames-sg/signinum 0.4.2, crates/signinum-j2k-native and the codec layer in
// crates/signinum-j2k).  Only the tests, the smoke check and the benchmark's
// CPU-baseline leg may load this code; the product library never links it.
//
// Every function below names the reference file:line it restates.  Sample
// arithmetic is kept in f32 exactly as the reference does (all reversible
// values are integers below 2^24, so the floors are exact).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace oracle {

// Error classes mirror the reference's error predicates
// (crates/signinum-j2k-cuda/src/error.rs:7-41).
enum Status : int {
  OK = 0,
  ERR_UNSUPPORTED = 1,  // is_unsupported / is_not_implemented
  ERR_BUFFER = 2,       // is_buffer_error
  ERR_TRUNCATED = 3,    // is_truncated
  ERR_DECODE = 4,       // any other decode error
  ERR_REGION = 5,       // J2kError::InvalidRegion
};

struct DecodeError {
  Status status;
  std::string message;
};

struct IntRect {
  uint32_t x0 = 0, y0 = 0, x1 = 0, y1 = 0;
  static IntRect ltrb(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    IntRect r;
    r.x0 = a; r.y0 = b; r.x1 = c; r.y1 = d;
    return r;
  }
  uint32_t width() const { return x1 > x0 ? x1 - x0 : 0; }
  uint32_t height() const { return y1 > y0 ? y1 - y0 : 0; }
  IntRect intersect(const IntRect& o) const;
};

// Pixel formats of signinum-core (PixelFormat) used on this path.
enum PixelFormat : int { FMT_GRAY8 = 0, FMT_RGB8 = 1, FMT_RGBA8 = 2, FMT_GRAY16 = 3, FMT_RGB16 = 4, FMT_RGBA16 = 5 };
int bytes_per_pixel(int fmt);

// Sub-band types (SubBandType).
enum SbType { LL = 0, HL = 1, LH = 2, HH = 3 };

enum RequestKind : int { REQ_FULL = 0, REQ_REGION = 1, REQ_SCALED = 2, REQ_REGION_SCALED = 3 };

struct Request {
  int kind = REQ_FULL;
  uint32_t x = 0, y = 0, w = 0, h = 0;  // region
  uint32_t denom = 1;                   // Downscale denominator: 1, 2, 4, 8
};

struct Info {
  uint32_t width = 0, height = 0;
  uint32_t components = 0;
  uint32_t bit_depth = 0;
  uint32_t levels = 0;       // decomposition levels of component 0
  uint32_t tiles = 0;
  uint32_t ht = 0;           // 1 when every component uses HT block coding
  uint32_t reversible = 0;
  uint32_t mct = 0;
};

Info inspect(const uint8_t* data, size_t len);

// Decodes one codestream with the request semantics of
// crates/signinum-j2k-cuda/src/decoder.rs:31-140 (output dims from
// DeviceDecodePlan) into a tight buffer of out_w*out_h*bpp bytes.
void decode(const uint8_t* data, size_t len, int fmt, const Request& req,
            std::vector<uint8_t>& out, uint32_t& out_w, uint32_t& out_h);

// HT code-block decode on its own (the reference's decode_impl,
// crates/signinum-j2k-native/src/j2c/ht_block_decode.rs:1563-1683).  Writes
// the raw sign-magnitude u32 words; returns false where decode_impl returns None.
bool ht_block_decode(const uint8_t* cleanup, size_t lcup, const uint8_t* refinement, size_t lref,
                     uint32_t missing_msbs, uint32_t num_passes, uint32_t width, uint32_t height,
                     uint32_t stride, bool stripe_causal, uint32_t* out);

// Classic (EBCOT) Tier-1 decode of one code block (oracle_ebcot.cpp;
// bitplane.rs:90-185 and the passes it calls).  `data` holds the block's
// codeword segments back to back: segment k covers bytes [seg_start[k],
// seg_start[k+1]) and coding passes [seg_pass[k], seg_pass[k+1]).  `band`
// is the sub-band type (LL 0, HL 1, LH 2, HH 3), `style` the code-block style
// byte of COD/COC.  Writes w x h int32 coefficients (stride out_stride).
bool classic_block_decode(const uint8_t* data, const std::vector<size_t>& seg_start,
                          const std::vector<uint32_t>& seg_pass, uint32_t w, uint32_t h, uint32_t missing,
                          uint32_t num_passes, uint32_t total_bitplanes, int band, uint8_t style, int32_t* out,
                          size_t out_stride);

// The zero-coding (Table D.1, per band class) and sign-coding (Table D.3)
// context tables over all 256 neighbour-significance patterns.
void ebcot_tables(uint8_t* zc_ll_lh, uint8_t* zc_hl, uint8_t* zc_hh, uint8_t* sc_label, uint8_t* sc_xor);
// The MQ probability table (Table C.2) as 47 (u16 qe LE, nmps, nlps, switch) records.
void ebcot_qe_records(uint8_t* out);

// Sub-band coefficients of component `comp` (after HT decode, before IDWT),
// concatenated in the reference's sub-band order (LL, then HL, LH, HH for each
// resolution), as int32 values.
void subband_coefficients(const uint8_t* data, size_t len, uint32_t comp, std::vector<int32_t>& out);

// The packed HT lookup tables the oracle decodes with (VLC0, VLC1, UVLC0, UVLC1).
const uint16_t* vlc_table(int which);
const uint16_t* uvlc_table(int which);

}  // namespace oracle
