// JPEG 2000 frames of a DICOM file with encapsulated Pixel Data: the step
// before the decode path on whole-slide DICOM files.  Follows the
// reference's extract_dicom_encapsulated_frames_with_limit
// (crates/signinum-j2k-metal/src/dicom.rs:22-95): find the Pixel Data
// element (7FE0,0010) of undefined length, read its Basic Offset Table item,
// read the fragment items up to the sequence delimiter, and group fragments
// into frames by the Basic Offset Table, else by the Extended Offset Table
// (7FE0,0001) with its Lengths (7FE0,0002) trimming padded frames, else one
// frame per fragment.  Frames are written back to back into the caller's
// buffer, each starting 16-byte aligned, so the buffer can go straight to the
// batch decode call.
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../../include/signinum_j2k_cuda.h"

void sgn_set_last_error_message(const char* msg);

namespace {

struct DicomError {
  sgn_status status;
  const char* what;
};

[[noreturn]] void truncated(const char* what) { throw DicomError{SGN_ERR_TRUNCATED, what}; }
[[noreturn]] void malformed(const char* what) { throw DicomError{SGN_ERR_DECODE, what}; }

constexpr uint8_t kPixelData[4] = {0xE0, 0x7F, 0x10, 0x00};
constexpr uint8_t kExtOffsets[4] = {0xE0, 0x7F, 0x01, 0x00};
constexpr uint8_t kExtLengths[4] = {0xE0, 0x7F, 0x02, 0x00};
constexpr uint8_t kItem[4] = {0xFE, 0xFF, 0x00, 0xE0};
constexpr uint8_t kSeqEnd[4] = {0xFE, 0xFF, 0xDD, 0xE0};
constexpr uint32_t kUndefined = 0xFFFFFFFFu;

struct Input {
  const uint8_t* d;
  size_t n;
  uint32_t u16(size_t at, const char* what) const {
    if (at + 2 > n || at + 2 < at) truncated(what);
    return (uint32_t)d[at] | ((uint32_t)d[at + 1] << 8);
  }
  uint32_t u32(size_t at, const char* what) const {
    if (at + 4 > n || at + 4 < at) truncated(what);
    return (uint32_t)d[at] | ((uint32_t)d[at + 1] << 8) | ((uint32_t)d[at + 2] << 16) | ((uint32_t)d[at + 3] << 24);
  }
  // First occurrence of a 4-byte tag in [0, end).
  size_t find(const uint8_t tag[4], size_t end) const {
    for (size_t i = 0; i + 4 <= end; ++i)
      if (std::memcmp(d + i, tag, 4) == 0) return i;
    return SIZE_MAX;
  }
};

bool explicit_vr(const uint8_t* vr) { return vr[0] >= 'A' && vr[0] <= 'Z' && vr[1] >= 'A' && vr[1] <= 'Z'; }

bool long_vr(const uint8_t* vr) {
  static const char* kLong[] = {"OB", "OD", "OF", "OL", "OV", "OW", "SQ", "UC", "UR", "UT", "UN"};
  for (const char* v : kLong)
    if (vr[0] == v[0] && vr[1] == v[1]) return true;
  return false;
}

// Value offset and length of the element whose tag starts at `tag`.
void element_header(const Input& in, size_t tag, const char* what, size_t& value, uint32_t& length) {
  const size_t after = tag + 4;
  if (after + 2 > in.n) truncated(what);
  const uint8_t* vr = in.d + after;
  if (explicit_vr(vr)) {
    if (long_vr(vr)) {
      value = after + 8;
      length = in.u32(after + 4, what);
    } else {
      value = after + 4;
      length = in.u16(after + 2, what);
    }
  } else {
    value = after + 4;
    length = in.u32(after, what);
  }
}

// An 8-byte little-endian table (7FE0,0001 / 7FE0,0002) before the Pixel Data.
bool u64_table_before(const Input& in, const uint8_t tag[4], size_t before, const char* what,
                      std::vector<uint64_t>& out) {
  const size_t at = in.find(tag, before);
  if (at == SIZE_MAX) return false;
  size_t value;
  uint32_t length;
  element_header(in, at, what, value, length);
  if (length == kUndefined) malformed("Extended Offset Table element has undefined length");
  if (value + length > in.n || value + length < value) truncated(what);
  if (length % 8) malformed(what);
  out.resize(length / 8);
  for (size_t k = 0; k < out.size(); ++k) {
    uint64_t v = 0;
    for (int b = 7; b >= 0; --b) v = (v << 8) | in.d[value + 8 * k + b];
    out[k] = v;
  }
  return true;
}

struct Fragment {
  uint64_t item_offset;  // from the first fragment's item tag
  size_t off, len;       // payload in the input
};

// Frames as (input ranges) lists, in frame order.
std::vector<std::vector<std::pair<size_t, size_t>>> extract(const Input& in, size_t limit) {
  std::vector<std::vector<std::pair<size_t, size_t>>> frames;
  if (limit == 0) return frames;
  // Pixel Data: encapsulated means undefined length (dicom.rs:97-159).
  const size_t tag = in.find(kPixelData, in.n);
  if (tag == SIZE_MAX) throw DicomError{SGN_ERR_DECODE, "Pixel Data element not found"};
  if (tag + 8 > in.n) truncated("Pixel Data header");
  size_t value;
  uint32_t length;
  element_header(in, tag, "Pixel Data length", value, length);
  if (length != kUndefined) throw DicomError{SGN_ERR_UNSUPPORTED, "Pixel Data is not encapsulated"};
  if (value > in.n) truncated("Pixel Data value");
  std::vector<uint64_t> ext_off, ext_len;
  const bool have_off = u64_table_before(in, kExtOffsets, tag, "Extended Offset Table", ext_off);
  const bool have_len = u64_table_before(in, kExtLengths, tag, "Extended Offset Table Lengths", ext_len);
  if (have_off && have_len && ext_off.size() != ext_len.size())
    malformed("Extended Offset Table and Lengths have different entry counts");
  // Basic Offset Table item (dicom.rs:161-193).
  if (value + 4 > in.n) truncated("Basic Offset Table item tag");
  if (std::memcmp(in.d + value, kItem, 4) != 0)
    malformed("encapsulated Pixel Data does not start with a Basic Offset Table item");
  const uint32_t bot_len = in.u32(value + 4, "Basic Offset Table length");
  const size_t bot = value + 8;
  if (bot + bot_len > in.n || bot + bot_len < bot) truncated("Basic Offset Table payload");
  if (bot_len % 4) malformed("Basic Offset Table length is not a multiple of four");
  std::vector<uint64_t> offsets(bot_len / 4);
  for (size_t k = 0; k < offsets.size(); ++k) offsets[k] = in.u32(bot + 4 * k, "Basic Offset Table");
  const std::vector<uint64_t>& table = offsets.empty() ? ext_off : offsets;
  const bool by_table = !table.empty();
  const bool trim = offsets.empty() && !ext_off.empty() && have_len;
  // Fragments (dicom.rs:195-264): stop at the first item of frame `limit`
  // when a table is given, after `limit` fragments otherwise.
  const uint64_t stop = by_table && limit < table.size() ? table[limit] : UINT64_MAX;
  std::vector<Fragment> frags;
  size_t cur = bot + bot_len;
  size_t first = SIZE_MAX;
  for (;;) {
    if (cur + 4 > in.n) truncated("Pixel Data item tag");
    const uint8_t* t = in.d + cur;
    const uint32_t len = in.u32(cur + 4, "Pixel Data item length");
    const size_t item = cur;
    cur += 8;
    if (std::memcmp(t, kSeqEnd, 4) == 0) {
      if (len != 0) malformed("non-zero sequence delimitation length");
      break;
    }
    if (std::memcmp(t, kItem, 4) != 0) malformed("expected item tag in encapsulated Pixel Data");
    if (len == kUndefined) malformed("undefined-length Pixel Data item");
    if (cur + len > in.n || cur + len < cur) truncated("Pixel Data item payload");
    if (first == SIZE_MAX) first = item;
    const uint64_t item_offset = item - first;
    if (item_offset >= stop) break;
    frags.push_back({item_offset, cur, len});
    if (!by_table && frags.size() >= limit) break;
    cur += len;
  }
  if (frags.empty()) return frames;
  if (!by_table) {
    for (const Fragment& f : frags) frames.push_back({{f.off, f.len}});
    return frames;
  }
  // Frames from the offset table (dicom.rs:389-428).
  const size_t count = std::min(table.size(), limit);
  for (size_t i = 0; i < count; ++i) {
    const uint64_t start = table[i], end = i + 1 < table.size() ? table[i + 1] : UINT64_MAX;
    if (end <= start) malformed("offset table offsets are not strictly increasing");
    std::vector<std::pair<size_t, size_t>> fr;
    uint64_t have = 0;
    const uint64_t cap = trim ? ext_len[i] : UINT64_MAX;
    for (const Fragment& f : frags) {
      if (f.item_offset < start || f.item_offset >= end) continue;
      if (trim) {
        const uint64_t take = std::min<uint64_t>(f.len, cap > have ? cap - have : 0);
        fr.push_back({f.off, (size_t)take});
        have += take;
        if (have >= cap) break;
      } else {
        fr.push_back({f.off, f.len});
        have += f.len;
      }
    }
    if (have == 0) malformed("offset table frame has no fragments");
    frames.push_back(std::move(fr));
  }
  return frames;
}

}  // namespace

extern "C" {

sgn_status sgn_dicom_frames(const uint8_t* data, size_t len, size_t limit, uint8_t* out, size_t out_cap,
                            uint64_t* frame_offsets, uint64_t* frame_lens, size_t frames_cap, size_t* nframes,
                            size_t* out_bytes) {
  if (!data || !nframes || !out_bytes) {
    sgn_set_last_error_message("null argument");
    return SGN_ERR_INVALID_ARGUMENT;
  }
  try {
    const auto frames = extract(Input{data, len}, limit);
    size_t total = 0;
    for (const auto& fr : frames) {
      size_t n = 0;
      for (const auto& part : fr) n += part.second;
      total = ((total + 15) & ~(size_t)15) + n;
    }
    *nframes = frames.size();
    *out_bytes = total;
    if (!out) return SGN_OK;  // size query
    if (out_cap < total || frames_cap < frames.size() || !frame_offsets || !frame_lens) {
      sgn_set_last_error_message("output buffers too small for the frames");
      return SGN_ERR_BUFFER;
    }
    size_t at = 0;
    for (size_t i = 0; i < frames.size(); ++i) {
      at = (at + 15) & ~(size_t)15;
      frame_offsets[i] = at;
      size_t n = 0;
      for (const auto& part : frames[i]) {
        std::memcpy(out + at + n, data + part.first, part.second);
        n += part.second;
      }
      frame_lens[i] = n;
      at += n;
    }
    return SGN_OK;
  } catch (const DicomError& e) {
    sgn_set_last_error_message(e.what);
    return e.status;
  }
}

}  // extern "C"
