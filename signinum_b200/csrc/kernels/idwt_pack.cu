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

// Periodic symmetric extension of index i into [0, n).
__device__ __forceinline__ int fold(int i, int n) {
  if (n == 1) return 0;
  int p = 2 * (n - 1);
  int m = i % p;
  if (m < 0) m += p;
  return m >= n ? p - m : m;
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
  for (int i = threadIdx.x; i < SH * SW; i += blockDim.x) {
    int ly = i / SW, lx = i % SW;
    S[ly][lx] = interleaved(job.ll, job.hl, job.lh, job.hh, x0 - HALO + lx, y0 - HALO + ly, w, h);
  }
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
  const PackJob& job = find_job(jobs, njobs);
  const uint32_t local = blockIdx.x - job.cta_begin;
  const int ax = (int)(job.cx & ~1u);
  const int x0 = ax + (int)(local % job.tiles_x) * TW, y0 = (int)(job.cy & ~1u) + (int)(local / job.tiles_x) * TH;
  const int w = (int)job.w, h = (int)job.h;
  const int nc = (int)job.ncomp;
  for (int c = 0; c < nc; ++c) {
    if (job.lifting) {
      for (int i = threadIdx.x; i < SH * SW; i += blockDim.x) {
        int ly = i / SW, lx = i % SW;
        S[c][ly][lx] = interleaved(job.ll[c], job.hl[c], job.lh[c], job.hh[c], x0 - HALO + lx, y0 - HALO + ly, w, h);
      }
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
    uint8_t* o = job.out + (size_t)(gy - cy0) * job.pitch;
    const int ox = gx - cx0;
    switch (fmt) {
      case PACK_GRAY8: o[ox] = to_u8(v0, bd, reg); break;
      case PACK_RGB8:
        o[3 * ox] = to_u8(v0, bd, reg);
        o[3 * ox + 1] = to_u8(v1, bd, reg);
        o[3 * ox + 2] = to_u8(v2, bd, reg);
        break;
      case PACK_RGBA8:
        o[4 * ox] = to_u8(v0, bd, reg);
        o[4 * ox + 1] = to_u8(v1, bd, reg);
        o[4 * ox + 2] = to_u8(v2, bd, reg);
        o[4 * ox + 3] = 255;
        break;
      case PACK_GRAY16: reinterpret_cast<uint16_t*>(o)[ox] = to_u16(v0, bd); break;
      case PACK_RGB16: {
        uint16_t* p = reinterpret_cast<uint16_t*>(o) + 3 * ox;
        p[0] = to_u16(v0, bd);
        p[1] = to_u16(v1, bd);
        p[2] = to_u16(v2, bd);
        break;
      }
    }
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
