// TEST INFRASTRUCTURE ONLY — C ABI of the parity oracle for the Python tests
// and the benchmark's CPU-baseline leg.
//
// oracle_decode_batch restates the reference CPU tile batch
// (decode_tiles_into, crates/signinum-j2k/src/batch.rs:110-147 with
// tile_batch_worker_count, crates/signinum-core/src/batch.rs:20-30): W worker
// threads over contiguous chunks of ceil(n/W) tiles, serial decode per tile,
// lowest failing index reported.
#include <algorithm>
#include <cstdio>
#include <atomic>
#include <cstring>
#include <thread>
#include <vector>

#include "oracle_internal.h"

using namespace oracle;

extern "C" {

struct oracle_info {
  uint32_t width, height, components, bit_depth, levels, tiles, ht, reversible, mct;
};

static thread_local char g_err[256];

const char* oracle_last_error() { return g_err; }

static int set_err(const DecodeError& e) {
  std::snprintf(g_err, sizeof(g_err), "%s", e.message.c_str());
  return e.status;
}

int oracle_inspect(const uint8_t* data, size_t len, oracle_info* out) {
  try {
    Info i = inspect(data, len);
    *out = {i.width, i.height, i.components, i.bit_depth, i.levels, i.tiles, i.ht, i.reversible, i.mct};
    return 0;
  } catch (const DecodeError& e) {
    return set_err(e);
  }
}

// Output dims are returned in out_w/out_h; the pixels are written tight
// (out_w * bpp bytes per row) when out_cap is large enough, else ERR_BUFFER.
int oracle_decode(const uint8_t* data, size_t len, int fmt, int kind, uint32_t rx, uint32_t ry, uint32_t rw,
                  uint32_t rh, uint32_t denom, uint8_t* out, size_t out_cap, uint32_t* out_w, uint32_t* out_h) {
  try {
    Request q;
    q.kind = kind;
    q.x = rx; q.y = ry; q.w = rw; q.h = rh;
    q.denom = denom;
    std::vector<uint8_t> buf;
    uint32_t w, h;
    decode(data, len, fmt, q, buf, w, h);
    *out_w = w;
    *out_h = h;
    if (buf.size() > out_cap) {
      std::snprintf(g_err, sizeof(g_err), "output buffer too small");
      return ERR_BUFFER;
    }
    if (!buf.empty()) std::memcpy(out, buf.data(), buf.size());
    return 0;
  } catch (const DecodeError& e) {
    return set_err(e);
  }
}

int oracle_ht_block_decode(const uint8_t* cleanup, size_t lcup, const uint8_t* ref, size_t lref, uint32_t mmsb,
                           uint32_t passes, uint32_t w, uint32_t h, int causal, uint32_t* out) {
  return ht_block_decode(cleanup, lcup, ref, lref, mmsb, passes, w, h, w, causal != 0, out) ? 0 : ERR_DECODE;
}

// Number of int32 sub-band coefficients written for component `comp`; the
// caller passes cap and gets -1 on error or when cap is too small.
long oracle_subband_coefficients(const uint8_t* data, size_t len, uint32_t comp, int32_t* out, size_t cap) {
  try {
    std::vector<int32_t> v;
    subband_coefficients(data, len, comp, v);
    if (v.size() > cap) return -1;
    std::memcpy(out, v.data(), v.size() * sizeof(int32_t));
    return (long)v.size();
  } catch (const DecodeError& e) {
    set_err(e);
    return -1;
  }
}

void oracle_ebcot_tables(uint8_t* zc_ll_lh, uint8_t* zc_hl, uint8_t* zc_hh, uint8_t* sc_label, uint8_t* sc_xor,
                         uint8_t* qe_records) {
  ebcot_tables(zc_ll_lh, zc_hl, zc_hh, sc_label, sc_xor);
  ebcot_qe_records(qe_records);
}

void oracle_tables(uint16_t* vlc0, uint16_t* vlc1, uint16_t* uvlc0, uint16_t* uvlc1) {
  std::memcpy(vlc0, vlc_table(0), 1024 * 2);
  std::memcpy(vlc1, vlc_table(1), 1024 * 2);
  std::memcpy(uvlc0, uvlc_table(0), 320 * 2);
  std::memcpy(uvlc1, uvlc_table(1), 256 * 2);
}

// Full-request tile batch into caller-owned tight buffers (outs[i] holds
// out_caps[i] bytes).  Returns -1 on success, else the lowest failing index;
// per_tile[i] receives each tile's status.
long oracle_decode_batch(const uint8_t* const* datas, const size_t* lens, size_t n, int fmt, uint8_t* const* outs,
                         const size_t* out_caps, int workers, int* per_tile) {
  if (n == 0) return -1;
  size_t w = workers > 0 ? (size_t)workers : std::max<size_t>(1, std::thread::hardware_concurrency());
  w = std::min(w, n);
  size_t chunk = (n + w - 1) / w;
  std::vector<std::thread> threads;
  for (size_t t = 0; t < w; ++t) {
    size_t b = t * chunk, e = std::min(n, b + chunk);
    if (b >= e) break;
    threads.emplace_back([=]() {
      for (size_t i = b; i < e; ++i) {
        uint32_t ow, oh;
        per_tile[i] = oracle_decode(datas[i], lens[i], fmt, REQ_FULL, 0, 0, 0, 0, 1, outs[i], out_caps[i], &ow, &oh);
      }
    });
  }
  for (auto& th : threads) th.join();
  for (size_t i = 0; i < n; ++i)
    if (per_tile[i] != 0) return (long)i;
  return -1;
}

}  // extern "C"
