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
// Mapping: one warp per unit = a strip of 64 columns x `seg` rows of a level.
// Lane k owns image columns (2k, 2k+1) of the strip, i.e. band column k of
// the low and high bands, so every band load and every row store is
// coalesced.  Horizontal lifting of a row needs the odd neighbour on the left
// and the updated even neighbour on the right: both come from warp shuffles
// (the strip's edge lanes load the one extra band sample they need).  The
// vertical pass streams down the rows keeping the previous odd row and the
// previous updated even row in registers.  Symmetric extension is done by
// reflecting row/column indices (it commutes with the lifting steps), so the
// edges need no special arithmetic.  No shared memory, no barriers.
//
// The last level keeps the streams of all components of a pixel in the same
// lane and finishes the pixels there: inverse RCT (mct.rs:117-150),
// +2^(bd-1) (decode.rs:1720-1729, :1748-1752) and the conversion to the
// requested pixel format (crates/signinum-j2k-native/src/lib.rs:1772-1840,
// :2202-2294; crates/signinum-j2k/src/decode.rs:345-356, :517-545); packed
// rows are staged per warp in shared memory and written with 16-byte stores.
#include <cstdint>

#include "../device_plan.h"
#include "kernels.h"

namespace sgn {
namespace {

constexpr int kLanes = 32;

// Periodic symmetric extension of index i into [0, n) (reflections about the
// first and last samples; the streams overshoot by at most a few samples).
__device__ __forceinline__ int fold(int i, int n) {
  if ((unsigned)i < (unsigned)n) return i;
  if (n == 1) return 0;
#pragma unroll 1
  for (int k = 0; k < 8 && (i < 0 || i >= n); ++k) i = i < 0 ? -i : 2 * (n - 1) - i;
  return i;
}

struct Bands {
  const int32_t* ll;
  const int32_t* hl;
  const int32_t* lh;
  const int32_t* hh;
  int w, h;
};

// Band samples of one interleaved row at this lane's columns (col, col + 1),
// col = 2b, plus the extra samples the strip's edge lanes need.  Loads only:
// the lifting happens in lift_row, so a caller can keep the next rows' loads
// in flight while it lifts the current ones.
struct RawRow {
  int lo, hi;     // low band (column col), high band (column col + 1)
  int hi_left;    // lane 0: high band at column col - 1
  int lo_r, hi_r; // lane 31: low / high band at columns col + 2, col + 3
};

__device__ __forceinline__ RawRow load_row(const Bands& B, int y, int b, int lane) {
  y = fold(y, B.h);
  const int r = y >> 1;
  const int lw = (B.w + 1) >> 1, hw = B.w >> 1;
  const int32_t* Lr = ((y & 1) ? B.lh : B.ll) + (size_t)r * lw;
  const int32_t* Hr = ((y & 1) ? B.hh : B.hl) + (size_t)r * hw;
  const int col = 2 * b;
  RawRow R;
  R.lo = col < B.w ? __ldg(Lr + b) : 0;
  R.hi = col + 1 < B.w ? __ldg(Hr + b) : 0;
  R.hi_left = (lane == 0 && b > 0) ? __ldg(Hr + b - 1) : 0;
  R.lo_r = (lane == kLanes - 1 && col + 2 < B.w) ? __ldg(Lr + b + 1) : 0;
  R.hi_r = (lane == kLanes - 1 && col + 3 < B.w) ? __ldg(Hr + b + 1) : 0;
  return R;
}

// Horizontal lifting of a loaded row: (even, odd) samples of this lane.
// Lanes past the right edge return garbage.
__device__ __forceinline__ int2 lift_row(const RawRow& R, int w, int b, int lane) {
  if (w == 1) return make_int2(R.lo, 0);
  const int col = 2 * b;
  int hi = R.hi;
  int hiL = __shfl_up_sync(0xFFFFFFFFu, hi, 1);
  if (lane == 0) hiL = b == 0 ? hi : R.hi_left;  // column -1 mirrors column 1
  if (col + 1 >= w) hi = hiL;                     // column w mirrors column w - 2
  const int E = R.lo - ((hiL + hi + 2) >> 2);
  int ER = __shfl_down_sync(0xFFFFFFFFu, E, 1);
  if (lane == kLanes - 1 && col + 2 < w) {
    const int hi2 = col + 3 < w ? R.hi_r : hi;
    ER = R.lo_r - ((hi + hi2 + 2) >> 2);
  }
  if (col + 2 >= w) ER = E;  // column w mirrors column w - 2
  return make_int2(E, hi + ((E + ER) >> 1));
}

__device__ __forceinline__ int2 hrow(const Bands& B, int y, int b, int lane) {
  return lift_row(load_row(B, y, b, lane), B.w, b, lane);
}

// Vertical 5/3 stream over output rows [ys, ye) (ys even) of NC level
// images at once; emit(y, v[NC]) receives each finished row.  With PREFETCH
// the loads of row pair m + 1 are issued before row pair m is lifted (more
// registers; used where a warp streams one component).
template <int NC, bool PREFETCH, typename Emit>
__device__ __forceinline__ void stream_rows(const Bands* B, int b, int lane, int ys, int ye, Emit emit) {
  const int h = B[0].h, w = B[0].w;
  int2 v[NC];
  if (h == 1) {
#pragma unroll
    for (int c = 0; c < NC; ++c) v[c] = hrow(B[c], 0, b, lane);
    emit(0, v);
    return;
  }
  int2 xo_prev[NC], ev_prev[NC];
  RawRow re[NC], ro[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    re[c] = load_row(B[c], ys, b, lane);
    ro[c] = load_row(B[c], ys + 1, b, lane);
    xo_prev[c] = hrow(B[c], ys - 1, b, lane);
    ev_prev[c] = make_int2(0, 0);
  }
  for (int m = ys >> 1;; ++m) {
    const int ye_row = 2 * m, yo_row = 2 * m + 1;
    const bool more = yo_row < ye;
    if (!PREFETCH && m != (ys >> 1)) {
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        re[c] = load_row(B[c], ye_row, b, lane);
        ro[c] = load_row(B[c], yo_row, b, lane);
      }
    }
    RawRow ne[NC], no[NC];
    int2 ev[NC], xo[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      if (PREFETCH && more) {
        ne[c] = load_row(B[c], ye_row + 2, b, lane);
        no[c] = load_row(B[c], yo_row + 2, b, lane);
      }
      const int2 xe = lift_row(re[c], w, b, lane);
      xo[c] = lift_row(ro[c], w, b, lane);
      ev[c].x = xe.x - ((xo_prev[c].x + xo[c].x + 2) >> 2);
      ev[c].y = xe.y - ((xo_prev[c].y + xo[c].y + 2) >> 2);
    }
    if (ye_row - 1 >= ys && ye_row - 1 < ye) {
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        v[c].x = xo_prev[c].x + ((ev_prev[c].x + ev[c].x) >> 1);
        v[c].y = xo_prev[c].y + ((ev_prev[c].y + ev[c].y) >> 1);
      }
      emit(ye_row - 1, v);
    }
    if (ye_row < ye) emit(ye_row, ev);
    if (!more) break;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      xo_prev[c] = xo[c];
      ev_prev[c] = ev[c];
      if (PREFETCH) {
        re[c] = ne[c];
        ro[c] = no[c];
      }
    }
  }
}

template <typename Job>
__device__ __forceinline__ const Job& find_job(const Job* jobs, uint32_t njobs, uint32_t unit) {
  uint32_t lo = 0, hi = njobs - 1;
  while (lo < hi) {
    uint32_t mid = (lo + hi + 1) >> 1;
    if (jobs[mid].unit_begin <= unit) lo = mid;
    else hi = mid - 1;
  }
  return jobs[lo];
}

}  // namespace

__global__ void __launch_bounds__(kIdwtWarps * 32) idwt_level_kernel(const IdwtJob* __restrict__ jobs,
                                                                     uint32_t njobs, uint32_t nunits) {
  const uint32_t unit = blockIdx.x * kIdwtWarps + (threadIdx.x >> 5);
  if (unit >= nunits) return;
  const int lane = threadIdx.x & 31;
  const IdwtJob& job = find_job(jobs, njobs, unit);
  const uint32_t local = unit - job.unit_begin;
  const int x0 = (int)(local % job.strips) * kIdwtStripW;
  const int ys = (int)(local / job.strips) * (int)job.seg;
  const int w = (int)job.w, h = (int)job.h;
  const int ye = min(ys + (int)job.seg, h);
  Bands B{job.ll, job.hl, job.lh, job.hh, w, h};
  const int b = (x0 >> 1) + lane, col = 2 * b;
  int32_t* out = job.out;
  stream_rows<1, true>(&B, b, lane, ys, ye, [&](int y, const int2* v) {
    int32_t* row = out + (size_t)y * w;
    if (col < w) row[col] = v[0].x;
    if (col + 1 < w) row[col + 1] = v[0].y;
  });
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

constexpr int kRowBytes = kIdwtStripW * 8 + 16;

// Packs one pixel (components v0..v2 after the inverse RCT) into o.
template <int FMT>
__device__ __forceinline__ void put_pixel(uint8_t* o, int32_t v0, int32_t v1, int32_t v2, uint32_t bd, uint32_t reg) {
  switch (FMT) {
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
    default: {
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

template <int FMT>
__host__ __device__ constexpr int pack_bpp() {
  return FMT == PACK_GRAY8 ? 1 : FMT == PACK_RGB8 ? 3 : FMT == PACK_RGBA8 ? 4 : FMT == PACK_GRAY16 ? 2 : 6;
}

template <int NC, int FMT>
__device__ __forceinline__ void pack_unit(const PackJob& job, int x0, int ys, int ye, int lane, uint8_t* rowbuf) {
  const int w = (int)job.w;
  const int cx0 = (int)job.cx, cy0 = (int)job.cy, cx1 = cx0 + (int)job.cw;
  const uint32_t bd = job.bit_depth, reg = job.region_conv;
  constexpr int bpp = pack_bpp<FMT>();
  const int32_t shift = 1 << (bd - 1);
  const bool mct = NC == 3 && job.mct;
  const int b = (x0 >> 1) + lane, col = 2 * b;
  const int xs = max(x0, cx0), xe = min(x0 + kIdwtStripW, cx1);
  const int nbytes = (xe - xs) * bpp;
  auto emit = [&](int y, const int2* v) {
    if (y < cy0 || y >= cy0 + (int)job.ch) return;  // warp-uniform
    const uint64_t gbase = (uint64_t)(y - cy0) * job.pitch + (uint64_t)(xs - cx0) * bpp;
    const int off = (int)(gbase & 15);
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int px = col + k;
      if (px < xs || px >= xe) continue;
      int32_t c0 = k ? v[0].y : v[0].x, c1 = 0, c2 = 0;
      if (NC == 3) {
        c1 = k ? v[1].y : v[1].x;
        c2 = k ? v[2].y : v[2].x;
        if (mct) {
          const int32_t g = c0 - ((c2 + c1) >> 2);
          const int32_t r = c2 + g, bl = c1 + g;
          c0 = r;
          c1 = g;
          c2 = bl;
        }
        c1 += shift;
        c2 += shift;
      }
      c0 += shift;
      put_pixel<FMT>(rowbuf + off + (px - xs) * bpp, c0, c1, c2, bd, reg);
    }
    __syncwarp();
    // Copy-out: bytes up to the first 16-byte boundary, 16-byte vectors, tail.
    uint8_t* g = job.out + gbase;
    const uint8_t* src = rowbuf + off;
    int head = (int)((16 - ((uintptr_t)g & 15)) & 15);
    if (head > nbytes) head = nbytes;
    if (lane < head) g[lane] = src[lane];
    const int nvec = (nbytes - head) >> 4;
    const uint4* sv = reinterpret_cast<const uint4*>(src + head);
    uint4* gv = reinterpret_cast<uint4*>(g + head);
    for (int k = lane; k < nvec; k += 32) gv[k] = sv[k];
    const int done = head + (nvec << 4);
    if (lane < nbytes - done) g[done + lane] = src[done + lane];
    __syncwarp();
  };
  if (job.lifting) {
    Bands B[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) B[c] = Bands{job.ll[c], job.hl[c], job.lh[c], job.hh[c], w, (int)job.h};
    stream_rows<NC, NC == 1>(B, b, lane, ys, ye, emit);
  } else {
    // Nothing left to lift: the image is the LL band itself.
    for (int y = ys; y < ye; ++y) {
      int2 v[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const int32_t* row = job.ll[c] + (size_t)y * w;
        v[c].x = col < w ? __ldg(row + col) : 0;
        v[c].y = col + 1 < w ? __ldg(row + col + 1) : 0;
      }
      emit(y, v);
    }
  }
}

}  // namespace

template <int FMT>
__global__ void __launch_bounds__(kIdwtWarps * 32) pack_kernel(const PackJob* __restrict__ jobs, uint32_t njobs,
                                                               uint32_t nunits) {
  __shared__ __align__(16) uint8_t rowbufs[kIdwtWarps][kRowBytes];
  const uint32_t warp = threadIdx.x >> 5;
  const uint32_t unit = blockIdx.x * kIdwtWarps + warp;
  if (unit >= nunits) return;
  const int lane = threadIdx.x & 31;
  const PackJob& job = find_job(jobs, njobs, unit);
  const uint32_t local = unit - job.unit_begin;
  const int x0 = (int)(job.cx & ~(uint32_t)(kIdwtStripW - 1)) + (int)(local % job.strips) * kIdwtStripW;
  const int ys = (int)(job.cy & ~1u) + (int)(local / job.strips) * (int)job.seg;
  const int ye = min(ys + (int)job.seg, (int)(job.cy + job.ch));
  if (job.ncomp >= 3) pack_unit<3, FMT>(job, x0, ys, ye, lane, rowbufs[warp]);
  else pack_unit<1, FMT>(job, x0, ys, ye, lane, rowbufs[warp]);
}

cudaError_t launch_idwt_level(const IdwtJob* jobs, uint32_t njobs, uint32_t nunits, cudaStream_t stream) {
  if (njobs == 0 || nunits == 0) return cudaSuccess;
  idwt_level_kernel<<<(nunits + kIdwtWarps - 1) / kIdwtWarps, kIdwtWarps * 32, 0, stream>>>(jobs, njobs, nunits);
  return cudaGetLastError();
}

cudaError_t launch_pack(const PackJob* jobs, uint32_t njobs, uint32_t nunits, uint32_t fmt, cudaStream_t stream) {
  if (njobs == 0 || nunits == 0) return cudaSuccess;
  const dim3 grid((nunits + kIdwtWarps - 1) / kIdwtWarps), block(kIdwtWarps * 32);
  switch (fmt) {
    case PACK_GRAY8: pack_kernel<PACK_GRAY8><<<grid, block, 0, stream>>>(jobs, njobs, nunits); break;
    case PACK_RGB8: pack_kernel<PACK_RGB8><<<grid, block, 0, stream>>>(jobs, njobs, nunits); break;
    case PACK_RGBA8: pack_kernel<PACK_RGBA8><<<grid, block, 0, stream>>>(jobs, njobs, nunits); break;
    case PACK_GRAY16: pack_kernel<PACK_GRAY16><<<grid, block, 0, stream>>>(jobs, njobs, nunits); break;
    case PACK_RGB16: pack_kernel<PACK_RGB16><<<grid, block, 0, stream>>>(jobs, njobs, nunits); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace sgn
