// Inverse reversible 5/3 DWT and the fused last level + inverse RCT + DC
// shift + pixel pack, on sm_100a.
//
// Arithmetic follows the reference exactly: per level, interleave the four
// sub-bands, then the horizontal lifting pass (update even samples with
// floor((l + r) / 4 + 1/2), then predict odd samples with floor((l + r) / 2)),
// then the vertical pass (crates/signinum-j2k-native/src/j2c/idwt.rs:535-555,
// :741-765, :972-1014), with periodic symmetric extension at the edges
// (:908-925).  All values are integers, so int32 with arithmetic shifts gives
// the reference's f32 floors bit for bit.
//
// Memory mapping: each CTA produces a 64x32 tile of one level.  It stages the
// tile plus a 2-sample halo from the four bands into shared memory (mirrored
// loads at the image edges; symmetric extension commutes with the lifting
// steps), runs both lifting passes there and writes the tile once, so every
// level reads its inputs and writes its output exactly once from HBM.  The
// last level keeps all components of the tile in shared memory and finishes
// the pixels in the same kernel: inverse RCT (mct.rs:117-150), +2^(bd-1)
// (decode.rs:1720-1729, :1748-1752) and the conversion to the requested
// pixel format (crates/signinum-j2k-native/src/lib.rs:1772-1840, :2202-2294;
// crates/signinum-j2k/src/decode.rs:345-356, :517-545).
#include <cstdint>

#include "../device_plan.h"
#include "kernels.h"

namespace sgn {
namespace {

constexpr int TW = kIdwtTileW, TH = kIdwtTileH, HALO = kIdwtHalo;
constexpr int SW = TW + 2 * HALO, SH = TH + 2 * HALO;

// Periodic symmetric extension of index i into [0, n): reflect about the
// first and last samples until inside (the staged halo overshoots by at most
// two samples, so one or two reflections suffice).
__device__ __forceinline__ int fold(int i, int n) {
  if (n == 1) return 0;
#pragma unroll 1
  for (int k = 0; k < 8 && (i < 0 || i >= n); ++k) i = i < 0 ? -i : 2 * (n - 1) - i;
  return i;
}

// Sample (gx, gy) of the interleaved level image (origin 0: even columns come
// from the low bands, even rows from LL/HL).
__device__ __forceinline__ int32_t interleaved(const int32_t* ll, const int32_t* hl, const int32_t* lh,
                                               const int32_t* hh, int gx, int gy, int w, int h) {
  gx = fold(gx, w);
  gy = fold(gy, h);
  const int lw = (w + 1) >> 1, hw = w >> 1;
  const int32_t* b;
  int s;
  if ((gy & 1) == 0) {
    if ((gx & 1) == 0) { b = ll; s = lw; } else { b = hl; s = hw; }
  } else {
    if ((gx & 1) == 0) { b = lh; s = lw; } else { b = hh; s = hw; }
  }
  return __ldg(b + (size_t)(gy >> 1) * s + (gx >> 1));
}

// Stages the tile at (x0, y0) plus its halo into S.  Interior tiles (halo
// inside the image) load each band as a block of rows, coalesced along the
// band row; edge tiles fold every index.
__device__ __forceinline__ void stage_tile(int32_t (*S)[SW], const int32_t* ll, const int32_t* hl, const int32_t* lh,
                                           const int32_t* hh, int x0, int y0, int w, int h) {
  const int tid = threadIdx.x, nt = blockDim.x;
  if (x0 >= HALO && y0 >= HALO && x0 + TW + HALO <= w && y0 + TH + HALO <= h) {
    constexpr int BW = SW / 2, BH = SH / 2;  // band samples per staged tile
    const int lw = (w + 1) >> 1, hw = w >> 1;
    const int bx0 = (x0 - HALO) >> 1, by0 = (y0 - HALO) >> 1;
    for (int i = tid; i < 4 * BH * BW; i += nt) {
      const int band = i / (BH * BW), r = i - band * (BH * BW);
      const int by = r / BW, bx = r - by * BW;
      const int32_t* b = band == 0 ? ll : band == 1 ? hl : band == 2 ? lh : hh;
      const int s = (band & 1) ? hw : lw;
      S[2 * by + (band >> 1)][2 * bx + (band & 1)] = __ldg(b + (size_t)(by0 + by) * s + bx0 + bx);
    }
  } else {
    for (int i = tid; i < SH * SW; i += nt) {
      const int ly = i / SW, lx = i - ly * SW;
      S[ly][lx] = interleaved(ll, hl, lh, hh, x0 - HALO + lx, y0 - HALO + ly, w, h);
    }
  }
}

// Both lifting passes on one staged tile.  The tile origin is even, so the
// parity of a shared-memory column equals the parity of its image column.
__device__ __forceinline__ void lift_tile(int32_t (*S)[SW], int w, int h) {
  const int tid = threadIdx.x, nt = blockDim.x;
  if (w > 1) {
    for (int i = tid; i < SH * (SW / 2 - 1); i += nt) {
      int ly = i / (SW / 2 - 1), lx = 2 + 2 * (i % (SW / 2 - 1));  // even columns 2..SW-2
      S[ly][lx] -= (S[ly][lx - 1] + S[ly][lx + 1] + 2) >> 2;
    }
    __syncthreads();
    for (int i = tid; i < SH * (SW / 2 - 1); i += nt) {
      int ly = i / (SW / 2 - 1), lx = 1 + 2 * (i % (SW / 2 - 1));  // odd columns 1..SW-3
      S[ly][lx] += (S[ly][lx - 1] + S[ly][lx + 1]) >> 1;
    }
    __syncthreads();
  }
  if (h > 1) {
    for (int i = tid; i < (SH / 2 - 1) * SW; i += nt) {
      int ly = 2 + 2 * (i / SW), lx = i % SW;  // even rows 2..SH-2
      S[ly][lx] -= (S[ly - 1][lx] + S[ly + 1][lx] + 2) >> 2;
    }
    __syncthreads();
    for (int i = tid; i < (SH / 2 - 1) * SW; i += nt) {
      int ly = 1 + 2 * (i / SW), lx = i % SW;  // odd rows 1..SH-3
      S[ly][lx] += (S[ly - 1][lx] + S[ly + 1][lx]) >> 1;
    }
    __syncthreads();
  }
}

template <typename Job>
__device__ __forceinline__ const Job& find_job(const Job* jobs, uint32_t njobs) {
  uint32_t lo = 0, hi = njobs - 1;
  while (lo < hi) {
    uint32_t mid = (lo + hi + 1) >> 1;
    if (jobs[mid].cta_begin <= blockIdx.x) lo = mid;
    else hi = mid - 1;
  }
  return jobs[lo];
}

}  // namespace

__global__ void __launch_bounds__(kIdwtThreads) idwt_level_kernel(const IdwtJob* __restrict__ jobs, uint32_t njobs) {
  __shared__ int32_t S[SH][SW];
  const IdwtJob& job = find_job(jobs, njobs);
  const uint32_t local = blockIdx.x - job.cta_begin;
  const int x0 = (int)(local % job.tiles_x) * TW, y0 = (int)(local / job.tiles_x) * TH;
  const int w = (int)job.w, h = (int)job.h;
  stage_tile(S, job.ll, job.hl, job.lh, job.hh, x0, y0, w, h);
  __syncthreads();
  lift_tile(S, w, h);
  for (int i = threadIdx.x; i < TH * TW; i += blockDim.x) {
    int ly = i / TW, lx = i % TW;
    int gx = x0 + lx, gy = y0 + ly;
    if (gx < w && gy < h) job.out[(size_t)gy * w + gx] = S[ly + HALO][lx + HALO];
  }
}

namespace {

__device__ __forceinline__ uint8_t sat_u8f(float r) { return (uint8_t)fminf(fmaxf(r, 0.0f), 255.0f); }

__device__ __forceinline__ uint8_t to_u8(int32_t v, uint32_t bd, uint32_t region) {
  if (bd == 8) return (uint8_t)min(max(v, 0), 255);
  if (region) {
    // sample_as_u8: round, clamp to the depth's maximum, rescale to 8 bits.
    float maxv = bd >= 16 ? 65535.0f : (float)max((1 << bd) - 1, 1);
    float c = fminf(fmaxf((float)v, 0.0f), maxv);
    return sat_u8f(roundf(__fmul_rn(__fdiv_rn(c, maxv), 255.0f)));
  }
  // interleave_and_convert slow path: round(v / (2^bd - 1) * 255) as u8.
  float d = (float)((1u << bd) - 1);
  return sat_u8f(roundf(__fmul_rn(__fdiv_rn((float)v, d), 255.0f)));
}

__device__ __forceinline__ uint16_t to_u16(int32_t v, uint32_t bd) {
  int32_t maxv = (int32_t)((1u << bd) - 1);
  int32_t c = min(max(v, 0), maxv);
  if (bd <= 8) {
    uint32_t mx = max((1u << bd) - 1, 1u);
    return (uint16_t)(((uint32_t)c * 65535u + mx / 2) / mx);
  }
  return (uint16_t)c;
}

}  // namespace

__global__ void __launch_bounds__(kIdwtThreads) pack_kernel(const PackJob* __restrict__ jobs, uint32_t njobs) {
  __shared__ int32_t S[3][SH][SW];
  __shared__ __align__(16) uint8_t O[TH][TW * 8 + 16];
  const PackJob& job = find_job(jobs, njobs);
  const uint32_t local = blockIdx.x - job.cta_begin;
  const int ax = (int)(job.cx & ~1u);
  const int x0 = ax + (int)(local % job.tiles_x) * TW, y0 = (int)(job.cy & ~1u) + (int)(local / job.tiles_x) * TH;
  const int w = (int)job.w, h = (int)job.h;
  const int nc = (int)job.ncomp;
  for (int c = 0; c < nc; ++c) {
    if (job.lifting) {
      stage_tile(S[c], job.ll[c], job.hl[c], job.lh[c], job.hh[c], x0, y0, w, h);
    } else {
      for (int i = threadIdx.x; i < TH * TW; i += blockDim.x) {
        int ly = i / TW, lx = i % TW;
        int gx = x0 + lx, gy = y0 + ly;
        S[c][ly + HALO][lx + HALO] = (gx < w && gy < h) ? __ldg(job.ll[c] + (size_t)gy * w + gx) : 0;
      }
    }
  }
  __syncthreads();
  if (job.lifting)
    for (int c = 0; c < nc; ++c) lift_tile(S[c], w, h);
  const int cx0 = (int)job.cx, cy0 = (int)job.cy, cx1 = cx0 + (int)job.cw, cy1 = cy0 + (int)job.ch;
  const int32_t shift = 1 << (job.bit_depth - 1);
  const uint32_t fmt = job.fmt, bd = job.bit_depth, reg = job.region_conv;
  const int bpp = fmt == PACK_GRAY8 ? 1 : fmt == PACK_RGB8 ? 3 : fmt == PACK_RGBA8 ? 4 : fmt == PACK_GRAY16 ? 2 : 6;
  // Packed pixels of each tile row, staged at the same offset modulo 16 as
  // their destination so the copy-out can use 16-byte stores.
  const int xs = max(x0, cx0), xe = min(x0 + TW, cx1);
  const int npix = xe - xs;
  for (int i = threadIdx.x; i < TH * TW; i += blockDim.x) {
    int ly = i / TW, lx = i % TW;
    int gx = x0 + lx, gy = y0 + ly;
    if (gx < cx0 || gx >= cx1 || gy < cy0 || gy >= cy1) continue;
    int32_t v0 = S[0][ly + HALO][lx + HALO], v1 = 0, v2 = 0;
    if (nc >= 3) {
      v1 = S[1][ly + HALO][lx + HALO];
      v2 = S[2][ly + HALO][lx + HALO];
      if (job.mct) {
        int32_t g = v0 - ((v2 + v1) >> 2);
        int32_t r = v2 + g, b = v1 + g;
        v0 = r;
        v1 = g;
        v2 = b;
      }
      v1 += shift;
      v2 += shift;
    }
    v0 += shift;
    const uint64_t gbase = (uint64_t)(gy - cy0) * job.pitch + (uint64_t)(xs - cx0) * bpp;
    uint8_t* o = &O[ly][(gbase & 15) + (size_t)(gx - xs) * bpp];
    switch (fmt) {
      case PACK_GRAY8: o[0] = to_u8(v0, bd, reg); break;
      case PACK_RGB8:
        o[0] = to_u8(v0, bd, reg);
        o[1] = to_u8(v1, bd, reg);
        o[2] = to_u8(v2, bd, reg);
        break;
      case PACK_RGBA8:
        o[0] = to_u8(v0, bd, reg);
        o[1] = to_u8(v1, bd, reg);
        o[2] = to_u8(v2, bd, reg);
        o[3] = 255;
        break;
      case PACK_GRAY16: {
        uint16_t a = to_u16(v0, bd);
        o[0] = (uint8_t)a;
        o[1] = (uint8_t)(a >> 8);
        break;
      }
      case PACK_RGB16: {
        uint16_t a = to_u16(v0, bd), g = to_u16(v1, bd), c = to_u16(v2, bd);
        o[0] = (uint8_t)a;
        o[1] = (uint8_t)(a >> 8);
        o[2] = (uint8_t)g;
        o[3] = (uint8_t)(g >> 8);
        o[4] = (uint8_t)c;
        o[5] = (uint8_t)(c >> 8);
        break;
      }
    }
  }
  __syncthreads();
  if (npix <= 0) return;
  // Copy-out: one warp per row; bytes up to the first 16-byte boundary, then
  // 16-byte vectors, then the tail.
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const int nbytes = npix * bpp;
  for (int ly = warp; ly < TH; ly += nwarps) {
    const int gy = y0 + ly;
    if (gy < cy0 || gy >= cy1) continue;
    const uint64_t gbase = (uint64_t)(gy - cy0) * job.pitch + (uint64_t)(xs - cx0) * bpp;
    uint8_t* g = job.out + gbase;
    const uint8_t* src = &O[ly][gbase & 15];
    int head = (int)((16 - ((uintptr_t)g & 15)) & 15);
    if (head > nbytes) head = nbytes;
    if (lane < head) g[lane] = src[lane];
    const int nvec = (nbytes - head) >> 4;
    const uint4* sv = reinterpret_cast<const uint4*>(src + head);
    uint4* gv = reinterpret_cast<uint4*>(g + head);
    for (int k = lane; k < nvec; k += 32) gv[k] = sv[k];
    const int done = head + (nvec << 4);
    if (lane < nbytes - done) g[done + lane] = src[done + lane];
  }
}

cudaError_t launch_idwt_level(const IdwtJob* jobs, uint32_t njobs, uint32_t total_ctas, cudaStream_t stream) {
  if (njobs == 0 || total_ctas == 0) return cudaSuccess;
  idwt_level_kernel<<<total_ctas, kIdwtThreads, 0, stream>>>(jobs, njobs);
  return cudaGetLastError();
}

cudaError_t launch_pack(const PackJob* jobs, uint32_t njobs, uint32_t total_ctas, cudaStream_t stream) {
  if (njobs == 0 || total_ctas == 0) return cudaSuccess;
  pack_kernel<<<total_ctas, kIdwtThreads, 0, stream>>>(jobs, njobs);
  return cudaGetLastError();
}

}  // namespace sgn
