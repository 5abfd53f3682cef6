// Host-side codestream parsing for the CUDA decode path.
//
// Parses the main header, the tile-part headers and every packet header of a
// single-tile HTJ2K codestream and produces the per-code-block segment table
// that the device kernels consume.  The semantics follow the reference's
// parser (crates/signinum-j2k-native/src/j2c/codestream.rs:38-187,
// tile.rs:131-306, build.rs:14-240, progression.rs:114-338,
// segment.rs:17-581, tag_tree.rs:118-238); the data layout is this library's
// own: flat arrays of bands and code blocks with offsets into the original
// codestream bytes, so the device reads segments in place.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace sgn {

// Status values equal the C ABI's sgn_status codes (include/signinum_j2k_cuda.h).
enum Status : int32_t {
  ST_OK = 0,
  ST_UNSUPPORTED = 1,
  ST_BUFFER = 2,
  ST_TRUNCATED = 3,
  ST_DECODE = 4,
  ST_REGION = 5,
};

struct ParseError {
  int32_t status;
  std::string message;
};

enum BandType : uint8_t { BAND_LL = 0, BAND_HL = 1, BAND_LH = 2, BAND_HH = 3 };

struct Band {
  uint8_t comp, res, type, nbp;  // nbp: number of magnitude bit-planes (E-2)
  uint32_t w, h;                 // sub-band dimensions (origin 0)
  float step;                    // dequantisation step (1 without quantisation)
  uint64_t coef_off;             // element offset within the tile's coefficient block
};

struct CodeBlock {
  uint32_t band;        // index into TileLayout::bands
  uint32_t x0, y0;      // position inside the band
  uint16_t w, h;
  uint32_t cleanup_off; // byte offset of the cleanup segment in the codestream (classic: of the first segment)
  uint32_t lcup;        // classic: the bytes of all segments, back to back
  uint32_t ref_off;     // byte offset of the refinement segment (when lref > 0)
  uint32_t lref;
  uint8_t missing_msbs, passes;
  // HT: 32-bit words of the unstuffed MagSgn stream the decode stages
  // ((Lcup - Scup + 15) / 4 + 2, Scup from the segment's last two bytes);
  // 0 when Scup exceeds Lcup or the block has no coded passes.
  uint16_t ms_words = 0;
  uint32_t seg_begin = 0;  // classic: first entry in TileLayout::segments
  uint8_t nseg = 0;        // classic: codeword segments of the block
};

// A classic code block's codeword segment: its bytes and coding passes.
struct ClassicSegment {
  uint32_t len;
  uint8_t passes;
};

struct TileLayout {
  uint32_t width = 0, height = 0;  // full image (= tile) dimensions
  uint32_t ncomp = 0;
  uint32_t bit_depth = 0;          // component 0 precision (all components equal)
  uint32_t levels = 0;             // decomposition levels
  bool mct = false;
  bool reversible = true;          // 5/3 (integer path); false: 9/7 with dequantisation
  bool causal = false;             // vertically causal context (code-block style bit 3)
  bool classic = false;            // classic (EBCOT) Tier-1 code blocks instead of HT
  uint8_t cbstyle = 0;             // code-block style byte of COD/COC
  std::vector<ClassicSegment> segments;  // classic: per block, in block order
  // Multi-layer classic: the blocks' parts (codestream offset, bytes) to copy
  // back to back into a gather area; CodeBlock::cleanup_off is then an offset
  // in that area (gather_bytes long) instead of the codestream.
  bool gathered = false;
  std::vector<std::pair<uint32_t, uint32_t>> gather;
  uint64_t gather_bytes = 0;
  uint32_t skipped = 0;            // resolution levels dropped for a reduced decode
  uint32_t out_w = 0, out_h = 0;   // dimensions of the decoded (possibly reduced) image
  std::vector<Band> bands;         // per component: LL, then HL/LH/HH per resolution
  std::vector<uint32_t> comp_band_begin;  // first band of each component
  std::vector<CodeBlock> blocks;   // only blocks of resolutions that are decoded
  uint64_t coef_per_comp = 0;      // elements of the decoded bands of one component
};

struct Info {
  uint32_t width, height, components, bit_depth, levels, tiles, ht, reversible, mct;
};

// Throws ParseError.
Info inspect_codestream(const uint8_t* data, size_t len);

// Parses a codestream for decoding.  `target` (two entries) requests a reduced
// resolution the way DecodeSettings::target_resolution does
// (codestream.rs:149-167); nullptr decodes at full resolution.
void parse_tile(const uint8_t* data, size_t len, const uint32_t* target, TileLayout& out);

}  // namespace sgn
