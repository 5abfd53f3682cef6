/* Lossless HTJ2K encode and seeded synthetic tiles (host only).
 *
 * The input side of the decode path: it produces the codestreams the
 * benchmarks and parity tests decode.  sgn_j2k_encode_lossless stands where
 * the reference's lossless facade stands
 * (encode_j2k_lossless, crates/signinum-j2k/src/encode.rs:166-188, with
 * J2kLosslessEncodeOptions :70-96 and the native EncodeOptions of
 * crates/signinum-j2k-native/src/j2c/encode.rs:35-80); the synthetic
 * generators have no counterpart in the reference (they describe the
 * benchmark workloads).
 */
#ifndef SIGNINUM_J2K_ENCODE_H
#define SIGNINUM_J2K_ENCODE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum sgn_progression {
  SGN_PROG_LRCP = 0,
  SGN_PROG_RLCP = 1,
  SGN_PROG_RPCL = 2,
  SGN_PROG_PCRL = 3,
  SGN_PROG_CPRL = 4
} sgn_progression;

typedef struct sgn_encode_options {
  uint32_t max_decomposition_levels; /* clamped to floor(log2(min(w, h))) */
  uint32_t code_block_width_exp;     /* code-block width = 2^(exp + 2); 4 -> 64 */
  uint32_t code_block_height_exp;
  uint32_t use_mct;                  /* reversible colour transform for >= 3 components */
  uint32_t progression;              /* sgn_progression */
  uint32_t write_tlm;
  uint32_t sop_eph;                  /* emit SOP/EPH packet markers */
  uint32_t precinct_width_exp;       /* PPx of every resolution, 1..15; 0 (with height 0): no precincts */
  uint32_t precinct_height_exp;      /* PPy */
  uint32_t tile_parts;               /* tile-parts the packets are split into (0 or 1: one) */
} sgn_encode_options;

/* pixels: interleaved samples, 1 byte each for bit_depth <= 8, else u16 LE.
 * Writes at most out_cap bytes; *out_len receives the codestream length (also
 * when out_cap is too small, in which case the return is -4).
 * Returns 0, -2 (invalid geometry), -3 (a coefficient exceeds the coder's
 * range) or -4 (buffer too small). */
int sgn_j2k_encode_lossless(const uint8_t* pixels, uint32_t width, uint32_t height, uint32_t components,
                            uint32_t bit_depth, const sgn_encode_options* options, uint8_t* out, size_t out_cap,
                            size_t* out_len);

/* Irreversible HTJ2K encode, the lossy input of the 9/7 decode path: DC
 * shift, ICT when options->use_mct and components >= 3, forward 9/7 and
 * scalar expounded quantisation with the same relative step for every band
 * (step_b = relative_step * 2^(bit_depth + gain_b), rounded to the
 * 5-bit exponent / 11-bit mantissa form).  This mode has no counterpart in
 * the reference (its encoder is lossless only); it exists to produce
 * irreversible codestreams of any size for the decode path's parity tests.
 * Returns as sgn_j2k_encode_lossless; -2 also for relative_step outside (0, 1). */
int sgn_j2k_encode_irreversible(const uint8_t* pixels, uint32_t width, uint32_t height, uint32_t components,
                                uint32_t bit_depth, const sgn_encode_options* options, double relative_step,
                                uint8_t* out, size_t out_cap, size_t* out_len);

/* Classic (EBCOT Tier-1, non-HT) encode, for the classic decode path's
 * tests and benchmarks: code_block_style holds the COD style bits
 * (0x01 arithmetic-coding bypass, 0x02 context reset, 0x04 termination on
 * every pass, 0x08 vertically causal context, 0x20 segmentation symbols);
 * irreversible selects the lossy mode of sgn_j2k_encode_irreversible with
 * relative_step, else the transform is lossless 5/3; layers (>= 1) quality
 * layers split every block's coding passes evenly.  Like the irreversible
 * mode it has no counterpart in the reference's public encoder.  Returns as
 * sgn_j2k_encode_lossless. */
int sgn_j2k_encode_classic(const uint8_t* pixels, uint32_t width, uint32_t height, uint32_t components,
                           uint32_t bit_depth, const sgn_encode_options* options, uint32_t code_block_style,
                           uint32_t irreversible, double relative_step, uint32_t layers, uint8_t* out,
                           size_t out_cap, size_t* out_len);

/* Seeded synthetic tiles (tight, interleaved). */
void sgn_synth_he_rgb8(uint64_t seed, uint32_t width, uint32_t height, double noise_sigma, uint8_t* out);
void sgn_synth_blank_rgb8(uint64_t seed, uint32_t width, uint32_t height, uint8_t* out);
void sgn_synth_fluor_gray16(uint64_t seed, uint32_t width, uint32_t height, uint8_t* out_le16);

#ifdef __cplusplus
}
#endif

#endif
