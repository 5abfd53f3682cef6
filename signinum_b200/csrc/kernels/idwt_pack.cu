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
// Mapping: one warp per unit = a strip of 128 columns x `seg` rows of a level.
// Lane k owns image columns 4k .. 4k+3 of the strip, i.e. band columns 2k and
// 2k+1 of the low and high bands, read as 8-byte pairs, so every band load
// and every row store is coalesced.  Horizontal lifting of a row needs the
// odd neighbour on the left and the updated even neighbour on the right: both
// come from warp shuffles (the strip's edge lanes load the extra band samples
// they need).  The vertical pass streams down the rows keeping the previous
// odd row and the previous updated even row in registers.  Symmetric
// extension is done by reflecting row/column indices (it commutes with the
// lifting steps), so the edges need no special arithmetic.  No barriers.
//
// The last level keeps the streams of all components of a pixel in the same
// lane and finishes the pixels there: inverse RCT (mct.rs:117-150),
// +2^(bd-1) (decode.rs:1720-1729, :1748-1752) and the conversion to the
// requested pixel format (crates/signinum-j2k-native/src/lib.rs:1772-1840,
// :2202-2294; crates/signinum-j2k/src/decode.rs:345-356, :517-545); each lane
// packs its four pixels into 32-bit words, the words of a row are staged per
// warp in shared memory and the row is written with 16-byte stores.
#include <algorithm>
#include <cstdint>

#include "../device_plan.h"
#include "kernels.h"

namespace sgn {
namespace {

constexpr int kLanes = 32;
static_assert(kIdwtStripW == 4 * kLanes, "one strip is four columns per lane");

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
  bool vec;  // w % 4 == 0 and 8-byte aligned bases: every band row starts 8-byte aligned
};

__device__ __forceinline__ Bands make_bands(const int32_t* ll, const int32_t* hl, const int32_t* lh,
                                            const int32_t* hh, int w, int h) {
  const uintptr_t a = (uintptr_t)ll | (uintptr_t)hl | (uintptr_t)lh | (uintptr_t)hh;
  return Bands{ll, hl, lh, hh, w, h, (w & 3) == 0 && (a & 7) == 0};
}

// Band samples of one interleaved row at this lane's band columns b, b + 1
// (image columns 2b .. 2b+3), plus the extra samples the strip's edge lanes
// need.  Loads only: lifting happens in lift_row, so a caller can keep the
// next rows' loads in flight while it lifts the current ones.
struct RawRow {
  int lo0, lo1, hi0, hi1;  // low / high band at columns b, b + 1
  int x1;                  // lane 0: high band at column b - 1; lane 31: low band at column b + 2
  int x2;                  // lane 31: high band at column b + 2
};

// INTERIOR: the strip starts at column 128 or later and ends at least two
// columns before the level's right edge (interior_strip), so every lane's
// columns and the edge lanes' extra samples lie inside the level and no
// column needs a bounds test or a mirror.
__device__ __forceinline__ bool interior_strip(int x0, int w) {
  return x0 >= (int)kIdwtStripW && x0 + (int)kIdwtStripW + 2 <= w;
}

template <bool INTERIOR = false>
__device__ __forceinline__ RawRow load_row(const Bands& B, int y, int b, int lane) {
  y = fold(y, B.h);
  const int r = y >> 1;
  const int lw = (B.w + 1) >> 1, hw = B.w >> 1;
  const int32_t* Lr = ((y & 1) ? B.lh : B.ll) + (size_t)r * lw;
  const int32_t* Hr = ((y & 1) ? B.hh : B.hl) + (size_t)r * hw;
  RawRow R;
  if (INTERIOR) {
    if (B.vec) {
      const int2 l = __ldg(reinterpret_cast<const int2*>(Lr + b));
      const int2 h = __ldg(reinterpret_cast<const int2*>(Hr + b));
      R.lo0 = l.x;
      R.lo1 = l.y;
      R.hi0 = h.x;
      R.hi1 = h.y;
    } else {
      R.lo0 = __ldg(Lr + b);
      R.lo1 = __ldg(Lr + b + 1);
      R.hi0 = __ldg(Hr + b);
      R.hi1 = __ldg(Hr + b + 1);
    }
    R.x1 = lane == 0 ? __ldg(Hr + b - 1) : lane == kLanes - 1 ? __ldg(Lr + b + 2) : 0;
    R.x2 = lane == kLanes - 1 ? __ldg(Hr + b + 2) : 0;
    return R;
  }
  if (B.vec && b + 1 < hw) {
    // b is even and both band widths are even: one 8-byte load per band.
    const int2 l = __ldg(reinterpret_cast<const int2*>(Lr + b));
    const int2 h = __ldg(reinterpret_cast<const int2*>(Hr + b));
    R.lo0 = l.x;
    R.lo1 = l.y;
    R.hi0 = h.x;
    R.hi1 = h.y;
  } else {
    R.lo0 = b < lw ? __ldg(Lr + b) : 0;
    R.lo1 = b + 1 < lw ? __ldg(Lr + b + 1) : 0;
    R.hi0 = b < hw ? __ldg(Hr + b) : 0;
    R.hi1 = b + 1 < hw ? __ldg(Hr + b + 1) : 0;
  }
  R.x1 = (lane == 0 && b > 0) ? __ldg(Hr + b - 1) : (lane == kLanes - 1 && b + 2 < lw) ? __ldg(Lr + b + 2) : 0;
  R.x2 = (lane == kLanes - 1 && b + 2 < hw) ? __ldg(Hr + b + 2) : 0;
  return R;
}

// Horizontal lifting of a loaded row: samples of image columns 2b .. 2b+3
// (x: 2b, y: 2b+1, z: 2b+2, w: 2b+3).  Columns past the right edge return
// garbage.  X[-1] mirrors X[1] and X[w] mirrors X[w-2].
template <bool INTERIOR = false>
__device__ __forceinline__ int4 lift_row(const RawRow& R, int w, int b, int lane) {
  if (INTERIOR) {
    int hm1 = __shfl_up_sync(0xFFFFFFFFu, R.hi1, 1);  // X[c-1]
    if (lane == 0) hm1 = R.x1;
    const int h0 = R.hi0, h1 = R.hi1;                  // X[c+1], X[c+3]
    const int e0 = R.lo0 - ((hm1 + h0 + 2) >> 2);      // X[c]
    const int e1 = R.lo1 - ((h0 + h1 + 2) >> 2);       // X[c+2]
    int e2 = __shfl_down_sync(0xFFFFFFFFu, e0, 1);     // X[c+4]
    if (lane == kLanes - 1) e2 = R.x1 - ((h1 + R.x2 + 2) >> 2);
    return make_int4(e0, h0 + ((e0 + e1) >> 1), e1, h1 + ((e1 + e2) >> 1));
  }
  if (w == 1) return make_int4(R.lo0, 0, 0, 0);
  const int c = 2 * b;
  int hm1 = __shfl_up_sync(0xFFFFFFFFu, R.hi1, 1);  // X[c-1]
  if (lane == 0) hm1 = b == 0 ? R.hi0 : R.x1;
  const int h0 = c + 1 < w ? R.hi0 : hm1;              // X[c+1]
  const int h1 = c + 3 < w ? R.hi1 : h0;               // X[c+3]
  const int e0 = R.lo0 - ((hm1 + h0 + 2) >> 2);        // X[c]
  int e1 = R.lo1 - ((h0 + h1 + 2) >> 2);               // X[c+2]
  int e2 = __shfl_down_sync(0xFFFFFFFFu, e0, 1);       // X[c+4]
  if (lane == kLanes - 1 && c + 4 < w) {
    const int h2 = c + 5 < w ? R.x2 : h1;
    e2 = R.x1 - ((h1 + h2 + 2) >> 2);
  }
  if (c + 2 >= w) e1 = e0;  // column w mirrors column w - 2
  if (c + 4 >= w) e2 = e1;
  return make_int4(e0, h0 + ((e0 + e1) >> 1), e1, h1 + ((e1 + e2) >> 1));
}

template <bool INTERIOR = false>
__device__ __forceinline__ int4 hrow(const Bands& B, int y, int b, int lane) {
  return lift_row<INTERIOR>(load_row<INTERIOR>(B, y, b, lane), B.w, b, lane);
}

__device__ __forceinline__ int4 vupdate(int4 xe, int4 a, int4 c) {
  return make_int4(xe.x - ((a.x + c.x + 2) >> 2), xe.y - ((a.y + c.y + 2) >> 2), xe.z - ((a.z + c.z + 2) >> 2),
                   xe.w - ((a.w + c.w + 2) >> 2));
}
__device__ __forceinline__ int4 vpredict(int4 xo, int4 a, int4 c) {
  return make_int4(xo.x + ((a.x + c.x) >> 1), xo.y + ((a.y + c.y) >> 1), xo.z + ((a.z + c.z) >> 1),
                   xo.w + ((a.w + c.w) >> 1));
}

// Vertical 5/3 stream over output rows [ys, ye) (ys even) of NC level images
// at once; emit(y, v[NC]) receives each finished row (four columns per lane).
// With PREFETCH the loads of row pair m + 1 are issued before row pair m is
// lifted (more registers; used where a warp streams one component).
template <int NC, bool PREFETCH, bool INTERIOR, typename Emit>
__device__ __forceinline__ void stream_rows(const Bands* B, int b, int lane, int ys, int ye, Emit emit) {
  const int h = B[0].h, w = B[0].w;
  int4 v[NC];
  if (h == 1) {
#pragma unroll
    for (int c = 0; c < NC; ++c) v[c] = hrow<INTERIOR>(B[c], 0, b, lane);
    emit(0, v);
    return;
  }
  int4 xo_prev[NC], ev_prev[NC];
  RawRow re[NC], ro[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    re[c] = load_row<INTERIOR>(B[c], ys, b, lane);
    ro[c] = load_row<INTERIOR>(B[c], ys + 1, b, lane);
    xo_prev[c] = hrow<INTERIOR>(B[c], ys - 1, b, lane);
    ev_prev[c] = make_int4(0, 0, 0, 0);
  }
  for (int m = ys >> 1;; ++m) {
    const int ye_row = 2 * m, yo_row = 2 * m + 1;
    const bool more = yo_row < ye;
    const bool first = m == (ys >> 1);
    RawRow ne[NC], no[NC];
    int4 ev[NC], xo[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      // Without PREFETCH one component's rows are loaded at a time.
      if (!PREFETCH && !first) {
        re[c] = load_row<INTERIOR>(B[c], ye_row, b, lane);
        ro[c] = load_row<INTERIOR>(B[c], yo_row, b, lane);
      }
      if (PREFETCH && more) {
        ne[c] = load_row<INTERIOR>(B[c], ye_row + 2, b, lane);
        no[c] = load_row<INTERIOR>(B[c], yo_row + 2, b, lane);
      }
      const int4 xe = lift_row<INTERIOR>(re[c], w, b, lane);
      xo[c] = lift_row<INTERIOR>(ro[c], w, b, lane);
      ev[c] = vupdate(xe, xo_prev[c], xo[c]);
    }
    if (ye_row - 1 >= ys && ye_row - 1 < ye) {
#pragma unroll
      for (int c = 0; c < NC; ++c) v[c] = vpredict(xo_prev[c], ev_prev[c], ev[c]);
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

// Per-lane shared-memory slots (int4 each) of the three-component stream:
// 0..2 previous odd row (horizontally lifted), 3..5 previous updated even
// row (also the finished row 2m), 6..8 the finished row 2m - 1.
constexpr int kStreamSlots = 9;

// Vertical 5/3 stream over rows [ys, ye) of three level images, one
// component at a time: the lifting state lives in the lane's own
// shared-memory slots `st` (slot k at st[k * 32 + lane]) and the components'
// band descriptors in the warp's shared table `tab`, so only one
// component's rows are in registers at once.  emit(y, v[3]) as stream_rows.
template <bool INTERIOR, typename Emit>
__device__ __forceinline__ void stream_rows3(const Bands* tab, int b, int lane, int ys, int ye, int4* st,
                                             Emit emit) {
  const int w = tab[0].w, h = tab[0].h;
  auto bands = [&](int c) -> const Bands& { return tab[c]; };
  auto slot = [&](int k) -> int4& { return st[k * kLanes + lane]; };
  int4 v[3];
  if (h == 1) {
#pragma unroll
    for (int c = 0; c < 3; ++c) v[c] = hrow<INTERIOR>(bands(c), 0, b, lane);
    emit(0, v);
    return;
  }
#pragma unroll 1
  for (int c = 0; c < 3; ++c) {
    slot(c) = hrow<INTERIOR>(bands(c), ys - 1, b, lane);
    slot(3 + c) = make_int4(0, 0, 0, 0);
  }
  // The rows of the next component (or of the next row pair's first
  // component) are loaded while the current one is lifted.
  RawRow re = load_row<INTERIOR>(bands(0), ys, b, lane), ro = load_row<INTERIOR>(bands(0), ys + 1, b, lane);
  for (int m = ys >> 1;; ++m) {
    const int ye_row = 2 * m, yo_row = 2 * m + 1;
    const bool more = yo_row < ye;
#pragma unroll 1
    for (int c = 0; c < 3; ++c) {
      RawRow ne = re, no = ro;
      if (c < 2) {
        const Bands& N = bands(c + 1);
        ne = load_row<INTERIOR>(N, ye_row, b, lane);
        no = load_row<INTERIOR>(N, yo_row, b, lane);
      } else if (more) {
        const Bands& N = bands(0);
        ne = load_row<INTERIOR>(N, ye_row + 2, b, lane);
        no = load_row<INTERIOR>(N, yo_row + 2, b, lane);
      }
      const int4 xe = lift_row<INTERIOR>(re, w, b, lane);
      const int4 xo = lift_row<INTERIOR>(ro, w, b, lane);
      re = ne;
      ro = no;
      const int4 xo_prev = slot(c), ev_prev = slot(3 + c);
      const int4 ev = vupdate(xe, xo_prev, xo);
      slot(6 + c) = vpredict(xo_prev, ev_prev, ev);
      slot(c) = xo;
      slot(3 + c) = ev;
    }
    if (ye_row - 1 >= ys && ye_row - 1 < ye) {
#pragma unroll
      for (int c = 0; c < 3; ++c) v[c] = slot(6 + c);
      emit(ye_row - 1, v);
    }
    if (ye_row < ye) {
#pragma unroll
      for (int c = 0; c < 3; ++c) v[c] = slot(3 + c);
      emit(ye_row, v);
    }
    if (yo_row >= ye) break;
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

namespace {

// Next work unit of the calling warp: the grid form takes one unit per warp;
// the queue form (persistent grid) takes units from a device counter until
// they run out.  Returns false when the warp is done.
__device__ __forceinline__ bool next_unit(uint32_t* queue, uint32_t nunits, bool& first, uint32_t& unit) {
  if (!queue) {
    unit = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const bool go = first && unit < nunits;
    first = false;
    return go;
  }
  uint32_t u = 0;
  if ((threadIdx.x & 31) == 0) u = atomicAdd(queue, 1u);
  unit = __shfl_sync(0xFFFFFFFFu, u, 0);
  return unit < nunits;
}

__device__ __forceinline__ void idwt_unit(const IdwtJob* __restrict__ jobs, uint32_t njobs, uint32_t unit) {
  const int lane = threadIdx.x & 31;
  const IdwtJob& job = find_job(jobs, njobs, unit);
  const uint32_t local = unit - job.unit_begin;
  const int x0 = (int)job.x_begin + (int)(local % job.strips) * kIdwtStripW;
  const int ys = (int)job.y_begin + (int)(local / job.strips) * (int)job.seg;
  const int w = (int)job.w, h = (int)job.h;
  const int ye = min(ys + (int)job.seg, (int)job.y_end);
  const Bands B = make_bands(job.ll, job.hl, job.lh, job.hh, w, h);
  const int b = (x0 >> 1) + 2 * lane, col = 2 * b;
  int32_t* out = job.out;
  // Rows of w int32 from a 16-byte aligned base: 16-byte stores when w % 4 == 0.
  const bool vec_out = (w & 3) == 0 && (((uintptr_t)out) & 15) == 0;
  auto emit = [&](int y, const int4* v) {
    int32_t* row = out + (size_t)y * w;
    if (vec_out && col + 3 < w) {
      *reinterpret_cast<int4*>(row + col) = v[0];
    } else {
      if (col < w) row[col] = v[0].x;
      if (col + 1 < w) row[col + 1] = v[0].y;
      if (col + 2 < w) row[col + 2] = v[0].z;
      if (col + 3 < w) row[col + 3] = v[0].w;
    }
  };
  if (interior_strip(x0, w)) stream_rows<1, true, true>(&B, b, lane, ys, ye, emit);
  else stream_rows<1, true, false>(&B, b, lane, ys, ye, emit);
}

}  // namespace

// QUEUE: persistent grid taking units from the device counter `queue`;
// otherwise one unit per warp.
// The grid form held to four CTAs per SM (64 registers, a few bytes of
// spills): more units in flight, which the large levels of uneven batches
// want (C2 levels 0.728 -> 0.680 ms) and the uniform 512^2 batch does not
// (0.158 -> 0.163 ms); the autotuner picks.
__global__ void __launch_bounds__(kIdwtWarps * 32, 4) idwt_level_lean_kernel(const IdwtJob* __restrict__ jobs,
                                                                            uint32_t njobs, uint32_t nunits) {
  const uint32_t unit = blockIdx.x * kIdwtWarps + (threadIdx.x >> 5);
  if (unit < nunits) idwt_unit(jobs, njobs, unit);
}

template <bool QUEUE>
__global__ void __launch_bounds__(kIdwtWarps * 32) idwt_level_kernel(const IdwtJob* __restrict__ jobs,
                                                                     uint32_t njobs, uint32_t nunits,
                                                                     uint32_t* queue) {
  if (!QUEUE) {
    const uint32_t unit = blockIdx.x * kIdwtWarps + (threadIdx.x >> 5);
    if (unit < nunits) idwt_unit(jobs, njobs, unit);
    return;
  }
  bool first = true;
  for (uint32_t unit; next_unit(queue, nunits, first, unit);) idwt_unit(jobs, njobs, unit);
}

namespace {

__device__ __forceinline__ uint32_t sat_u8f(float r) { return (uint32_t)fminf(fmaxf(r, 0.0f), 255.0f); }

// DIRECT: the sample needs only a clamp (8-bit samples to u8, or samples of
// more than 8 bits to u16); chosen per unit so the hot loop holds no float or
// division path.
template <bool DIRECT>
__device__ __forceinline__ uint32_t to_u8(int32_t v, uint32_t bd, uint32_t region) {
  if (DIRECT || bd == 8) return (uint32_t)min(max(v, 0), 255);
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

template <bool DIRECT>
__device__ __forceinline__ uint32_t to_u16(int32_t v, uint32_t bd) {
  int32_t maxv = (int32_t)((1u << bd) - 1);
  int32_t c = min(max(v, 0), maxv);
  if (!DIRECT && bd <= 8) {
    uint32_t mx = max((1u << bd) - 1, 1u);
    return ((uint32_t)c * 65535u + mx / 2) / mx;
  }
  return (uint32_t)c;
}

template <int FMT>
__host__ __device__ constexpr int pack_bpp() {
  return FMT == PACK_GRAY8 ? 1 : FMT == PACK_RGB8 ? 3 : FMT == PACK_RGBA8 ? 4 : FMT == PACK_GRAY16 ? 2 : 6;
}

// Byte q (a compile-time constant after unrolling) of a lane's packed words.
__device__ __forceinline__ void put_byte(uint32_t* wds, int q, uint32_t byte) { wds[q >> 2] |= byte << (8 * (q & 3)); }

// Packs pixel p (components c0..c2 after the inverse RCT and DC shift) at
// byte p * bpp of the lane's four-pixel group.
template <int FMT, bool DIRECT>
__device__ __forceinline__ void put_pixel(uint32_t* wds, int p, int32_t c0, int32_t c1, int32_t c2, uint32_t bd,
                                          uint32_t reg) {
  constexpr int B = pack_bpp<FMT>();
  const int q = p * B;
  if (FMT == PACK_GRAY8) {
    put_byte(wds, q, to_u8<DIRECT>(c0, bd, reg));
  } else if (FMT == PACK_RGB8 || FMT == PACK_RGBA8) {
    put_byte(wds, q, to_u8<DIRECT>(c0, bd, reg));
    put_byte(wds, q + 1, to_u8<DIRECT>(c1, bd, reg));
    put_byte(wds, q + 2, to_u8<DIRECT>(c2, bd, reg));
    if (FMT == PACK_RGBA8) put_byte(wds, q + 3, 255u);
  } else if (FMT == PACK_GRAY16) {
    const uint32_t a = to_u16<DIRECT>(c0, bd);
    put_byte(wds, q, a & 0xFF);
    put_byte(wds, q + 1, a >> 8);
  } else {
    const uint32_t a = to_u16<DIRECT>(c0, bd), g = to_u16<DIRECT>(c1, bd), c = to_u16<DIRECT>(c2, bd);
    put_byte(wds, q, a & 0xFF);
    put_byte(wds, q + 1, a >> 8);
    put_byte(wds, q + 2, g & 0xFF);
    put_byte(wds, q + 3, g >> 8);
    put_byte(wds, q + 4, c & 0xFF);
    put_byte(wds, q + 5, c >> 8);
  }
}

__device__ __forceinline__ int lane_comp(const int4& v, int p) { return p == 0 ? v.x : p == 1 ? v.y : p == 2 ? v.z : v.w; }

// Row buffer per warp: up to 15 bytes of alignment shift + 128 pixels x 6 bytes.
constexpr int kRowWords = (16 + kIdwtStripW * 6) / 4;

// Writes one output row of a warp's strip: each lane's packed words (four
// pixels of BPP bytes) are staged in the warp's row buffer so that the copied
// range has the destination's alignment mod 16, then columns [xs, xe) go out
// as the bytes up to the first 16-byte boundary, 16-byte vectors and a tail.
// g: the destination of column xs in the row; lane k's words hold columns
// x0 + 4k .. x0 + 4k + 3.  When the destination is 4-byte aligned and the
// columns [xs, xs + nbytes / BPP) start and end on lane boundaries (whole
// strips of a tile, the common case), every lane inside writes its BPP words
// itself: four pixels of BPP bytes are BPP 32-bit words at a 4-byte aligned
// place.  Otherwise the row goes through the warp's buffer as below.
template <int BPP>
__device__ __forceinline__ void store_row(uint8_t* g, int x0, int xs, int nbytes, int lane, uint32_t* rowbuf,
                                          const uint32_t* wds) {
  const int xe = xs + nbytes / BPP;
  if ((((uintptr_t)g & 3) | ((xs - x0) & 3) | ((xe - x0) & 3)) == 0) {  // warp-uniform
    const int c = x0 + 4 * lane;
    if (c >= xs && c < xe) {
      uint32_t* d = reinterpret_cast<uint32_t*>(g + (size_t)(c - xs) * BPP);
#pragma unroll
      for (int k = 0; k < BPP; ++k) d[k] = wds[k];
    }
    return;
  }
  uint8_t* rowbytes = reinterpret_cast<uint8_t*>(rowbuf);
  const int sh = (int)(((uintptr_t)g - (uintptr_t)((xs - x0) * BPP)) & 15);
  if ((sh & 3) == 0) {
    uint32_t* dst = rowbuf + (sh >> 2) + lane * BPP;
#pragma unroll
    for (int k = 0; k < BPP; ++k) dst[k] = wds[k];
  } else {
    uint8_t* dst = rowbytes + sh + lane * 4 * BPP;
#pragma unroll
    for (int q = 0; q < 4 * BPP; ++q) dst[q] = (uint8_t)(wds[q >> 2] >> (8 * (q & 3)));
  }
  __syncwarp();
  const uint8_t* src = rowbytes + sh + (xs - x0) * BPP;
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
}

template <int NC, int FMT, bool DIRECT>
__device__ __forceinline__ void pack_unit(const PackJob& job, int x0, int ys, int ye, int lane, uint32_t* rowbuf,
                                          int4* st, Bands* tab) {
  constexpr int BPP = pack_bpp<FMT>();
  const int w = (int)job.w;
  const int cx0 = (int)job.cx, cy0 = (int)job.cy, cx1 = cx0 + (int)job.cw, cy1 = cy0 + (int)job.ch;
  const uint32_t bd = job.bit_depth, reg = job.region_conv;
  const int32_t shift = 1 << (bd - 1);
  const bool mct = NC == 3 && job.mct;
  const int b = (x0 >> 1) + 2 * lane, col = 2 * b;
  const int xs = max(x0, cx0), xe = min(x0 + kIdwtStripW, cx1);
  const int nbytes = (xe - xs) * BPP;
  auto emit = [&](int y, const int4* v) {
    if (y < cy0 || y >= cy1) return;  // warp-uniform
    uint32_t wds[BPP];
#pragma unroll
    for (int k = 0; k < BPP; ++k) wds[k] = 0;
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      int32_t c0 = lane_comp(v[0], p), c1 = 0, c2 = 0;
      if (NC == 3) {
        c1 = lane_comp(v[1], p);
        c2 = lane_comp(v[2], p);
        if (mct) {
          const int32_t gg = c0 - ((c2 + c1) >> 2);
          const int32_t r = c2 + gg, bl = c1 + gg;
          c0 = r;
          c1 = gg;
          c2 = bl;
        }
        c1 += shift;
        c2 += shift;
      }
      c0 += shift;
      put_pixel<FMT, DIRECT>(wds, p, c0, c1, c2, bd, reg);
    }
    store_row<BPP>(job.out + (uint64_t)(y - cy0) * job.pitch + (uint64_t)(xs - cx0) * BPP, x0, xs, nbytes, lane,
                   rowbuf, wds);
  };
  if (job.lifting) {
    if (NC == 3) {
      // The components' band descriptors, read from the job once per unit.
      if (lane < 3) tab[lane] = make_bands(job.ll[lane], job.hl[lane], job.lh[lane], job.hh[lane], w, (int)job.h);
      __syncwarp();
      if (interior_strip(x0, w)) stream_rows3<true>(tab, b, lane, ys, ye, st, emit);
      else stream_rows3<false>(tab, b, lane, ys, ye, st, emit);
      __syncwarp();  // the table is rewritten by the warp's next unit
    } else {
      const Bands B = make_bands(job.ll[0], job.hl[0], job.lh[0], job.hh[0], w, (int)job.h);
      if (interior_strip(x0, w)) stream_rows<1, true, true>(&B, b, lane, ys, ye, emit);
      else stream_rows<1, true, false>(&B, b, lane, ys, ye, emit);
    }
  } else {
    // Nothing left to lift: the image is the LL band itself.
    for (int y = ys; y < ye; ++y) {
      int4 v[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const int32_t* row = job.ll[c] + (size_t)y * w;
        v[c].x = col < w ? __ldg(row + col) : 0;
        v[c].y = col + 1 < w ? __ldg(row + col + 1) : 0;
        v[c].z = col + 2 < w ? __ldg(row + col + 2) : 0;
        v[c].w = col + 3 < w ? __ldg(row + col + 3) : 0;
      }
      emit(y, v);
    }
  }
}

}  // namespace

template <int FMT, int NC, bool DIRECT>
__device__ __forceinline__ void pack_one(const PackJob* __restrict__ jobs, uint32_t njobs, uint32_t unit,
                                         uint32_t* rowbuf, int4* st, Bands* tab) {
  const int lane = threadIdx.x & 31;
  const PackJob& job = find_job(jobs, njobs, unit);
  const uint32_t local = unit - job.unit_begin;
  const int x0 = (int)(job.cx & ~(uint32_t)(kIdwtStripW - 1)) + (int)(local % job.strips) * kIdwtStripW;
  const int ys = (int)(job.cy & ~1u) + (int)(local / job.strips) * (int)job.seg;
  const int ye = min(ys + (int)job.seg, (int)(job.cy + job.ch));
  pack_unit<NC, FMT, DIRECT>(job, x0, ys, ye, lane, rowbuf, st, tab);
}

// One kernel per (pixel format, components, conversion) variant, with the
// jobs of a launch all of that variant (pack_variant): each variant gets the
// registers it needs and none of the others' code.  NC 3: RGB tiles, 1: gray;
// DIRECT: samples convert with a clamp alone.  The gray stream keeps its
// lifting state in registers (the RGB one in shared memory), so it runs
// three CTAs per SM with room for it instead of four.
template <int FMT, int NC, bool DIRECT, bool QUEUE>
__global__ void __launch_bounds__(kIdwtWarps * 32, NC == 3 ? 4 : 3) pack_kernel(const PackJob* __restrict__ jobs, uint32_t njobs,
                                                               uint32_t nunits, uint32_t* queue) {
  __shared__ __align__(16) uint32_t rowbufs[kIdwtWarps][kRowWords];
  __shared__ int4 states[kIdwtWarps][kStreamSlots * kLanes];
  __shared__ Bands tabs[kIdwtWarps][3];
  uint32_t* rowbuf = rowbufs[threadIdx.x >> 5];
  int4* st = states[threadIdx.x >> 5];
  Bands* tab = tabs[threadIdx.x >> 5];
  if (!QUEUE) {
    const uint32_t unit = blockIdx.x * kIdwtWarps + (threadIdx.x >> 5);
    if (unit < nunits) pack_one<FMT, NC, DIRECT>(jobs, njobs, unit, rowbuf, st, tab);
    return;
  }
  bool first = true;
  for (uint32_t unit; next_unit(queue, nunits, first, unit);)
    pack_one<FMT, NC, DIRECT>(jobs, njobs, unit, rowbuf, st, tab);
}

// ---------------------------------------------------------------------------
// Irreversible 9/7 levels and the fused last level + inverse ICT + DC shift +
// pack (crates/signinum-j2k-native/src/j2c/idwt.rs:767-836, :1016-1140;
// mct.rs:80-115; decode.rs:1130-1151 for the dequantisation).
//
// Every sample goes through the reference's own sequence of f32 roundings:
// band coefficient x step, then per level the horizontal pass (even columns
// x K, odd x 1/K, then the four lifting steps delta, gamma, beta, alpha as
// fma(left + right, c, x)), then the same vertical pass.  Only __fmul_rn /
// __fadd_rn / fmaf are used, so no multiply is contracted into a
// neighbouring add and the results match the reference's f32 arithmetic bit
// for bit.  Symmetric extension is done by reflecting indices, which
// commutes with the lifting steps (reflected positions compute the same sums
// in the other order, and f32 addition is commutative).
//
// Mapping: a warp per strip of kStrip97 = 120 output columns x `seg` rows.
// Lane k holds the four columns x0 - 4 + 4k .. x0 - 1 + 4k, so lanes 0 and
// 31 hold the four columns on either side of the strip: a sample after the
// four lifting steps depends on the samples within four columns of it, so
// lanes 1..30 finish exact values while every lane runs the same code (each
// step takes one neighbour from the adjacent lane by a shuffle; the edge
// lanes' own results are not used).  Vertically a four-stage pipeline runs
// down the rows, loading rows 2m+2 and 2m+3 per step and finishing rows 2m
// (after beta) and 2m-1 (after alpha); a unit starting at row ys primes from
// row ys-3.  The next rows' raw samples are loaded one step (or, for three
// components, one component) ahead.

constexpr float kNegAlpha97 = 1.5861343f, kNegBeta97 = 0.052980117f, kNegGamma97 = -0.8829111f,
                kNegDelta97 = -0.44350687f, kKappa97 = 1.2301741f;
constexpr int kWarps97 = 4;  // warps per CTA of the 9/7 pack kernel (its shared state is larger)
static_assert(kStrip97 == 4 * (kLanes - 2), "lanes 1..30 hold a strip's output columns");

namespace {

// Whole-sample symmetric extension into [0, n) of an index at most four
// samples outside it (every sample an exact output depends on).  Indices
// further out (columns of lanes whose results are unused) end at the nearest
// in-range index of the same parity, so the band they select (low for even,
// high for odd) and the row inside it stay in bounds.
__device__ __forceinline__ int fold97(int i, int n) {
  if ((unsigned)i < (unsigned)n) return i;
  if (n == 1) return 0;
#pragma unroll 1
  for (int k = 0; k < 4 && (unsigned)i >= (unsigned)n; ++k) i = i < 0 ? -i : 2 * (n - 1) - i;
  if (i < 0) return i & 1;
  if (i >= n) return (n - 1) - (((n - 1) ^ i) & 1);
  return i;
}

struct Src97 {
  const int32_t* ll;
  const int32_t* hl;
  const int32_t* lh;
  const int32_t* hh;
  float q[4];    // dequantisation steps of ll, hl, lh, hh
  int w, h;
  bool ll_band;  // ll is the LL band; otherwise the previous level's f32 image
  bool fast;     // the strip's 128 columns lie inside the level and rows are 8-byte aligned
};

__device__ __forceinline__ Src97 make_src97(const int32_t* ll, const int32_t* hl, const int32_t* lh,
                                            const int32_t* hh, const float* q, bool ll_band, int w, int h, int c0) {
  const uintptr_t a = (uintptr_t)ll | (uintptr_t)hl | (uintptr_t)lh | (uintptr_t)hh;
  const bool fast = (w & 3) == 0 && (a & 7) == 0 && c0 >= 0 && c0 + 4 * kLanes <= w;
  return Src97{ll, hl, lh, hh, {q[0], q[1], q[2], q[3]}, w, h, ll_band, fast};
}

// The raw words of a lane's four columns of one interleaved row (low band at
// the even columns, high band at the odd ones), loaded ahead of their use.
struct Raw97 {
  int32_t e0, o0, e1, o1;
};

__device__ __forceinline__ void row_bands(const Src97& S, int y, const int32_t*& lo, const int32_t*& hi) {
  y = fold97(y, S.h);
  const int r = y >> 1;
  lo = ((y & 1) ? S.lh : S.ll) + (size_t)r * ((S.w + 1) >> 1);
  hi = ((y & 1) ? S.hh : S.hl) + (size_t)r * (S.w >> 1);
}

// c: the lane's first column (even).
__device__ __forceinline__ Raw97 load97(const Src97& S, int y, int c) {
  const int32_t *lo, *hi;
  row_bands(S, y, lo, hi);
  if (S.fast) {
    const int2 l = __ldg(reinterpret_cast<const int2*>(lo + (c >> 1)));
    const int2 h = __ldg(reinterpret_cast<const int2*>(hi + (c >> 1)));
    return Raw97{l.x, h.x, l.y, h.y};
  }
  // Reflection keeps a column's parity, so even columns stay in the low band.
  const int w = S.w;
  return Raw97{__ldg(lo + (fold97(c, w) >> 1)), __ldg(hi + (fold97(c + 1, w) >> 1)), __ldg(lo + (fold97(c + 2, w) >> 1)),
               __ldg(hi + (fold97(c + 3, w) >> 1))};
}

__device__ __forceinline__ float lstep(float l, float r, float c, float x) { return fmaf(__fadd_rn(l, r), c, x); }

// Dequantises (or reinterprets) a loaded row and runs the horizontal 9/7
// synthesis: the lane's four columns (exact on lanes 1..30).
__device__ __forceinline__ float4 lift97(const Src97& S, int y, const Raw97& R, float K, float IK) {
  const bool odd = fold97(y, S.h) & 1;
  const float ql = odd ? S.q[2] : S.q[0], qh = odd ? S.q[3] : S.q[1];
  float e0, e1;
  if (!odd && !S.ll_band) {
    e0 = __int_as_float(R.e0);
    e1 = __int_as_float(R.e1);
  } else {
    e0 = __fmul_rn(__int2float_rn(R.e0), ql);
    e1 = __fmul_rn(__int2float_rn(R.e1), ql);
  }
  float o0 = __fmul_rn(__int2float_rn(R.o0), qh), o1 = __fmul_rn(__int2float_rn(R.o1), qh);
  if (S.w == 1) return make_float4(e0, 0.0f, 0.0f, 0.0f);
  e0 = __fmul_rn(e0, K);
  e1 = __fmul_rn(e1, K);
  o0 = __fmul_rn(o0, IK);
  o1 = __fmul_rn(o1, IK);
  // delta: even columns; gamma: odd; beta: even; alpha: odd.
  const float om1 = __shfl_up_sync(0xFFFFFFFFu, o1, 1);
  const float e0a = lstep(om1, o0, kNegDelta97, e0), e1a = lstep(o0, o1, kNegDelta97, e1);
  const float ep4a = __shfl_down_sync(0xFFFFFFFFu, e0a, 1);
  const float o0b = lstep(e0a, e1a, kNegGamma97, o0), o1b = lstep(e1a, ep4a, kNegGamma97, o1);
  const float om1b = __shfl_up_sync(0xFFFFFFFFu, o1b, 1);
  const float e0c = lstep(om1b, o0b, kNegBeta97, e0a), e1c = lstep(o0b, o1b, kNegBeta97, e1a);
  const float ep4c = __shfl_down_sync(0xFFFFFFFFu, e0c, 1);
  return make_float4(e0c, lstep(e0c, e1c, kNegAlpha97, o0b), e1c, lstep(e1c, ep4c, kNegAlpha97, o1b));
}

__device__ __forceinline__ float4 scale4(float4 v, float k) {
  return make_float4(__fmul_rn(v.x, k), __fmul_rn(v.y, k), __fmul_rn(v.z, k), __fmul_rn(v.w, k));
}
__device__ __forceinline__ float4 lstep4(float4 a, float4 b, float c, float4 x) {
  return make_float4(lstep(a.x, b.x, c, x.x), lstep(a.y, b.y, c, x.y), lstep(a.z, b.z, c, x.z),
                     lstep(a.w, b.w, c, x.w));
}

// Vertical 9/7 stream over rows [ys, ye) (ys even) of NC level images.
// col is the lane's first column; src(c) gives component c's bands;
// st(c, k) is its lifting state (k 0: the
// last odd input row, 1..3: the last rows after delta, gamma, beta, the
// beta row being the step's finished even row; 4: its finished odd row);
// emit(y, v[NC]) receives each
// finished row.  Components are lifted one at a time while the next
// component's (or the next step's) rows load.
template <int NC, typename SrcOf, typename State, typename Emit>
__device__ __forceinline__ void stream97(SrcOf src, int h, int col, int ys, int ye, float K, float IK, State st,
                                         Emit emit) {
  float4 v[NC];
  if (h == 1) {
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const Src97& S = src(c);
      v[c] = lift97(S, 0, load97(S, 0, col), K, IK);
    }
    emit(0, v);
    return;
  }
  const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll 1
  for (int c = 0; c < NC; ++c) {
    const Src97& S = src(c);
    st(c, 0) = scale4(lift97(S, ys - 3, load97(S, ys - 3, col), K, IK), IK);
    st(c, 1) = zero;
    st(c, 2) = zero;
    st(c, 3) = zero;
  }
  const int m0 = (ys >> 1) - 2, m1 = ye >> 1;
  Raw97 re, ro;
  {
    const Src97& S = src(0);
    re = load97(S, 2 * m0 + 2, col);
    ro = load97(S, 2 * m0 + 3, col);
  }
  for (int m = m0; m <= m1; ++m) {
#pragma unroll 1
    for (int c = 0; c < NC; ++c) {
      // Loads of the next component's rows, or of the next step's first one.
      Raw97 ne = re, no = ro;
      if (c + 1 < NC) {
        const Src97& N = src(c + 1);
        ne = load97(N, 2 * m + 2, col);
        no = load97(N, 2 * m + 3, col);
      } else if (m < m1) {
        const Src97& N = src(0);
        ne = load97(N, 2 * m + 4, col);
        no = load97(N, 2 * m + 5, col);
      }
      const Src97& S = src(c);
      const float4 xe = scale4(lift97(S, 2 * m + 2, re, K, IK), K);
      const float4 xo = scale4(lift97(S, 2 * m + 3, ro, K, IK), IK);
      re = ne;
      ro = no;
      const float4 xp = st(c, 0), s1p = st(c, 1), s2p = st(c, 2), s3p = st(c, 3);
      const float4 s1 = lstep4(xp, xo, kNegDelta97, xe);   // row 2m+2
      const float4 s2 = lstep4(s1p, s1, kNegGamma97, xp);  // row 2m+1
      const float4 s3 = lstep4(s2p, s2, kNegBeta97, s1p);  // row 2m, final
      st(c, 4) = lstep4(s3p, s3, kNegAlpha97, s2p);        // row 2m-1, final
      st(c, 0) = xo;
      st(c, 1) = s1;
      st(c, 2) = s2;
      st(c, 3) = s3;
    }
    // The step's finished odd row 2m - 1, then its even row 2m, through one
    // call site of emit (its pixel conversions are long: one copy of them
    // in the loop keeps the code small).
#pragma unroll 1
    for (int k = 0; k < 2; ++k) {
      const int y = 2 * m - 1 + k;
      if (y >= ys && y < ye) {
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          const float4 odd = st(c, 4), even = st(c, 3);
          v[c] = k ? even : odd;
        }
        emit(y, v);
      }
    }
  }
}

__device__ __forceinline__ void idwt97_unit(const IdwtJob* __restrict__ jobs, uint32_t njobs, uint32_t unit, float IK) {
  const int lane = threadIdx.x & 31;
  const IdwtJob& job = find_job(jobs, njobs, unit);
  const uint32_t local = unit - job.unit_begin;
  const int x0 = (int)job.x_begin + (int)(local % job.strips) * kStrip97;
  const int ys = (int)job.y_begin + (int)(local / job.strips) * (int)job.seg;
  const int w = (int)job.w, h = (int)job.h;
  const int ye = min(ys + (int)job.seg, (int)job.y_end);
  const int col = x0 - 4 + 4 * lane;
  const Src97 S = make_src97(job.ll, job.hl, job.lh, job.hh, job.step, job.ll_band != 0, w, h, x0 - 4);
  float* out = reinterpret_cast<float*>(job.out);
  const bool mine = lane >= 1 && lane <= kLanes - 2;
  const bool vec_out = (w & 3) == 0 && (((uintptr_t)out) & 15) == 0;
  float4 state[5];
  const Src97* sp = &S;
  stream97<1>([sp](int) -> const Src97& { return *sp; }, h, col, ys, ye, kKappa97, IK,
              [&](int, int k) -> float4& { return state[k]; },
              [&](int y, const float4* v) {
                if (!mine) return;
                float* rowp = out + (size_t)y * w;
                if (vec_out && col + 3 < w) {
                  *reinterpret_cast<float4*>(rowp + col) = v[0];
                } else {
                  if (col < w) rowp[col] = v[0].x;
                  if (col + 1 < w) rowp[col + 1] = v[0].y;
                  if (col + 2 < w) rowp[col + 2] = v[0].z;
                  if (col + 3 < w) rowp[col + 3] = v[0].w;
                }
              });
}

}  // namespace

template <bool QUEUE>
__global__ void __launch_bounds__(kIdwtWarps * 32) idwt97_level_kernel(const IdwtJob* __restrict__ jobs,
                                                                       uint32_t njobs, uint32_t nunits,
                                                                       uint32_t* queue) {
  const float IK = __fdiv_rn(1.0f, kKappa97);
  if (!QUEUE) {
    const uint32_t unit = blockIdx.x * kIdwtWarps + (threadIdx.x >> 5);
    if (unit < nunits) idwt97_unit(jobs, njobs, unit, IK);
    return;
  }
  bool first = true;
  for (uint32_t unit; next_unit(queue, nunits, first, unit);) idwt97_unit(jobs, njobs, unit, IK);
}

namespace {

__device__ __forceinline__ float lane_compf(const float4& v, int p) {
  return p == 0 ? v.x : p == 1 ? v.y : p == 2 ? v.z : v.w;
}

// `as u8` of a rounded f32: NaN and negatives 0, saturating at 255.
__device__ __forceinline__ uint32_t sat_u8_round(float r) {
  if (!(r > 0.0f)) return 0u;
  if (r >= 255.0f) return 255u;
  return (uint32_t)r;
}

// Sample conversions of the f32 path (crates/signinum-j2k-native/src/lib.rs:1772-1840,
// :2202-2294; crates/signinum-j2k/src/decode.rs:345-356, :517-545).
__device__ __forceinline__ uint32_t f_to_u8(float v, uint32_t bd, uint32_t region) {
  const float r = roundf(v);
  if (region) {
    // sample_as_u8: round, clamp to the depth's maximum, rescale to 8 bits.
    if (bd == 8) return (uint32_t)fminf(fmaxf(r, 0.0f), 255.0f);
    const float maxv = bd >= 16 ? 65535.0f : (float)max((1 << bd) - 1, 1);
    const float c = fminf(fmaxf(r, 0.0f), maxv);
    return sat_u8_round(roundf(__fmul_rn(__fdiv_rn(c, maxv), 255.0f)));
  }
  // interleave_and_convert: rounded as u8 at 8 bits, else rescaled.
  if (bd == 8) return sat_u8_round(r);
  return sat_u8_round(roundf(__fmul_rn(__fdiv_rn(v, (float)((1u << bd) - 1)), 255.0f)));
}

// decode_native: round, clamp to [0, 2^bd - 1], widen depths <= 8 to 16 bits.
__device__ __forceinline__ uint32_t f_to_u16(float v, uint32_t bd) {
  const float maxv = (float)((1u << bd) - 1);
  const float r = roundf(v);
  const float c = r < 0.0f ? 0.0f : (r > maxv ? maxv : r);
  if (bd <= 8) {
    const uint32_t s = (uint32_t)(uint8_t)c, mx = max((1u << bd) - 1, 1u);
    return (s * 65535u + mx / 2) / mx;
  }
  return (uint32_t)c;
}

template <int FMT>
__device__ __forceinline__ void put_pixel97(uint32_t* wds, int p, float c0, float c1, float c2, uint32_t bd,
                                            uint32_t reg) {
  constexpr int B = pack_bpp<FMT>();
  const int q = p * B;
  if (FMT == PACK_GRAY8) {
    put_byte(wds, q, f_to_u8(c0, bd, reg));
  } else if (FMT == PACK_RGB8 || FMT == PACK_RGBA8) {
    put_byte(wds, q, f_to_u8(c0, bd, reg));
    put_byte(wds, q + 1, f_to_u8(c1, bd, reg));
    put_byte(wds, q + 2, f_to_u8(c2, bd, reg));
    if (FMT == PACK_RGBA8) put_byte(wds, q + 3, 255u);
  } else if (FMT == PACK_GRAY16) {
    const uint32_t a = f_to_u16(c0, bd);
    put_byte(wds, q, a & 0xFF);
    put_byte(wds, q + 1, a >> 8);
  } else {
    const uint32_t a = f_to_u16(c0, bd), g = f_to_u16(c1, bd), c = f_to_u16(c2, bd);
    put_byte(wds, q, a & 0xFF);
    put_byte(wds, q + 1, a >> 8);
    put_byte(wds, q + 2, g & 0xFF);
    put_byte(wds, q + 3, g >> 8);
    put_byte(wds, q + 4, c & 0xFF);
    put_byte(wds, q + 5, c >> 8);
  }
}

// Shared-memory slots of a lane's three-component 9/7 stream: 5 per component
// (the stream's st(c, 0..4)).
constexpr int kSlots97 = 5 * 3;

template <int NC, int FMT>
__device__ __forceinline__ void pack97_unit(const PackJob& job, int x0, int ys, int ye, int lane, uint32_t* rowbuf,
                                            float4* st, Src97* tab, float IK) {
  constexpr int BPP = pack_bpp<FMT>();
  const int w = (int)job.w, h = (int)job.h;
  const int cx0 = (int)job.cx, cy0 = (int)job.cy, cx1 = cx0 + (int)job.cw, cy1 = cy0 + (int)job.ch;
  const uint32_t bd = job.bit_depth, reg = job.region_conv;
  const float shift = (float)(1u << (bd - 1));
  const bool ict = NC == 3 && job.mct;
  const int col = x0 - 4 + 4 * lane;
  const int xs = max(x0, cx0), xe = min(x0 + kStrip97, cx1);
  const int nbytes = (xe - xs) * BPP;
  auto emit = [&](int y, const float4* v) {
    if (y < cy0 || y >= cy1) return;  // warp-uniform
    uint32_t wds[BPP];
#pragma unroll
    for (int k = 0; k < BPP; ++k) wds[k] = 0;
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      float c0 = lane_compf(v[0], p), c1 = 0.0f, c2 = 0.0f;
      if (NC == 3) {
        c1 = lane_compf(v[1], p);
        c2 = lane_compf(v[2], p);
        if (ict) {
          // mct.rs:80-115 with fused multiply-adds.
          const float r = fmaf(c2, 1.402f, c0);
          const float g = fmaf(c2, -0.71414f, fmaf(c1, -0.34413f, c0));
          const float bl = fmaf(c1, 1.772f, c0);
          c0 = r;
          c1 = g;
          c2 = bl;
        }
        c1 = __fadd_rn(c1, shift);
        c2 = __fadd_rn(c2, shift);
      }
      c0 = __fadd_rn(c0, shift);
      put_pixel97<FMT>(wds, p, c0, c1, c2, bd, reg);
    }
    // Lane k's words are columns x0 - 4 + 4k ..: the row starts at x0 - 4.
    store_row<BPP>(job.out + (uint64_t)(y - cy0) * job.pitch + (uint64_t)(xs - cx0) * BPP, x0 - 4, xs, nbytes,
                   lane, rowbuf, wds);
  };
  if (job.lifting) {
    if (NC == 3) {
      // The components' band descriptors, read from the job once per unit.
      if (lane < 3)
        tab[lane] = make_src97(job.ll[lane], job.hl[lane], job.lh[lane], job.hh[lane], job.step[lane],
                               job.ll_band != 0, w, h, x0 - 4);
      __syncwarp();
      stream97<3>([&](int c) -> const Src97& { return tab[c]; }, h, col, ys, ye, kKappa97, IK,
                  [&](int c, int k) -> float4& { return st[(c * 5 + k) * kLanes + lane]; }, emit);
      __syncwarp();
    } else {
      const Src97 S = make_src97(job.ll[0], job.hl[0], job.lh[0], job.hh[0], job.step[0], job.ll_band != 0, w, h,
                                 x0 - 4);
      float4 state[5];
      const Src97* sp = &S;
      stream97<1>([sp](int) -> const Src97& { return *sp; }, h, col, ys, ye, kKappa97, IK,
                  [&](int, int k) -> float4& { return state[k]; }, emit);
    }
  } else {
    // Nothing to lift: the image is the LL band itself (dequantised).
    for (int y = ys; y < ye; ++y) {
      float4 v[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const int32_t* rowp = job.ll[c] + (size_t)y * w;
        const float q = job.step[c][0];
        auto at = [&](int k) {
          const int x = col + k;
          return x >= 0 && x < w ? __fmul_rn(__int2float_rn(__ldg(rowp + x)), q) : 0.0f;
        };
        v[c] = make_float4(at(0), at(1), at(2), at(3));
      }
      emit(y, v);
    }
  }
}

}  // namespace

template <int FMT, bool QUEUE>
__global__ void __launch_bounds__(kWarps97 * 32) pack97_kernel(const PackJob* __restrict__ jobs, uint32_t njobs,
                                                               uint32_t nunits, uint32_t* queue) {
  __shared__ __align__(16) uint32_t rowbufs[kWarps97][kRowWords];
  __shared__ float4 states[kWarps97][kSlots97 * kLanes];
  __shared__ Src97 tabs[kWarps97][3];
  const float IK = __fdiv_rn(1.0f, kKappa97);
  uint32_t* rowbuf = rowbufs[threadIdx.x >> 5];
  float4* st = states[threadIdx.x >> 5];
  Src97* tab = tabs[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  auto one = [&](uint32_t unit) {
    const PackJob& job = find_job(jobs, njobs, unit);
    const uint32_t local = unit - job.unit_begin;
    const int x0 = (int)(job.cx - job.cx % kStrip97) + (int)(local % job.strips) * kStrip97;
    const int ys = (int)(job.cy & ~1u) + (int)(local / job.strips) * (int)job.seg;
    const int ye = min(ys + (int)job.seg, (int)(job.cy + job.ch));
    // RGB formats take RGB tiles, gray formats gray ones (the host maps them
    // so), so the format fixes the component count.
    constexpr int NC = (FMT == PACK_GRAY8 || FMT == PACK_GRAY16) ? 1 : 3;
    pack97_unit<NC, FMT>(job, x0, ys, ye, lane, rowbuf, st, tab, IK);
  };
  if (!QUEUE) {
    const uint32_t unit = blockIdx.x * kWarps97 + (threadIdx.x >> 5);
    if (unit < nunits) one(unit);
    return;
  }
  bool first = true;
  for (uint32_t unit; next_unit(queue, nunits, first, unit);) one(unit);
}

cudaError_t launch_idwt97_level(const IdwtJob* jobs, uint32_t njobs, uint32_t nunits, cudaStream_t stream,
                                uint32_t* queue, uint32_t persistent_ctas) {
  if (njobs == 0 || nunits == 0) return cudaSuccess;
  uint32_t ctas = (nunits + kIdwtWarps - 1) / kIdwtWarps;
  if (queue) ctas = std::max(1u, std::min(ctas, persistent_ctas));
  if (queue) idwt97_level_kernel<true><<<ctas, kIdwtWarps * 32, 0, stream>>>(jobs, njobs, nunits, queue);
  else idwt97_level_kernel<false><<<ctas, kIdwtWarps * 32, 0, stream>>>(jobs, njobs, nunits, nullptr);
  return cudaGetLastError();
}

cudaError_t launch_pack97(const PackJob* jobs, uint32_t njobs, uint32_t nunits, uint32_t fmt, cudaStream_t stream,
                          uint32_t* queue, uint32_t persistent_ctas) {
  if (njobs == 0 || nunits == 0) return cudaSuccess;
  uint32_t ctas = (nunits + kWarps97 - 1) / kWarps97;
  if (queue) ctas = std::max(1u, std::min(ctas, persistent_ctas));
  const dim3 grid(ctas), block(kWarps97 * 32);
#define SGN_PACK97_LAUNCH(F)                                                                   \
  case F:                                                                                       \
    if (queue) pack97_kernel<F, true><<<grid, block, 0, stream>>>(jobs, njobs, nunits, queue); \
    else pack97_kernel<F, false><<<grid, block, 0, stream>>>(jobs, njobs, nunits, nullptr);    \
    break;
  switch (fmt) {
    SGN_PACK97_LAUNCH(PACK_GRAY8)
    SGN_PACK97_LAUNCH(PACK_RGB8)
    SGN_PACK97_LAUNCH(PACK_RGBA8)
    SGN_PACK97_LAUNCH(PACK_GRAY16)
    SGN_PACK97_LAUNCH(PACK_RGB16)
    default: return cudaErrorInvalidValue;
  }
#undef SGN_PACK97_LAUNCH
  return cudaGetLastError();
}

cudaError_t launch_idwt_level(const IdwtJob* jobs, uint32_t njobs, uint32_t nunits, cudaStream_t stream,
                              uint32_t* queue, uint32_t persistent_ctas, bool lean) {
  if (njobs == 0 || nunits == 0) return cudaSuccess;
  uint32_t ctas = (nunits + kIdwtWarps - 1) / kIdwtWarps;
  if (queue) ctas = std::max(1u, std::min(ctas, persistent_ctas));
  if (queue) idwt_level_kernel<true><<<ctas, kIdwtWarps * 32, 0, stream>>>(jobs, njobs, nunits, queue);
  else if (lean) idwt_level_lean_kernel<<<ctas, kIdwtWarps * 32, 0, stream>>>(jobs, njobs, nunits);
  else idwt_level_kernel<false><<<ctas, kIdwtWarps * 32, 0, stream>>>(jobs, njobs, nunits, nullptr);
  return cudaGetLastError();
}

namespace {

template <int F, int NC, bool D>
cudaError_t launch_pack_variant(const PackJob* jobs, uint32_t njobs, uint32_t nunits, dim3 grid, cudaStream_t stream,
                                uint32_t* queue) {
  if (queue) pack_kernel<F, NC, D, true><<<grid, kIdwtWarps * 32, 0, stream>>>(jobs, njobs, nunits, queue);
  else pack_kernel<F, NC, D, false><<<grid, kIdwtWarps * 32, 0, stream>>>(jobs, njobs, nunits, nullptr);
  return cudaGetLastError();
}

// RGB formats take RGB tiles (variants 0, 1), gray formats gray ones (2, 3).
template <int F>
cudaError_t launch_pack_format(uint32_t variant, const PackJob* jobs, uint32_t njobs, uint32_t nunits, dim3 grid,
                               cudaStream_t stream, uint32_t* queue) {
  if constexpr (F == PACK_GRAY8 || F == PACK_GRAY16) {
    if (variant == 2) return launch_pack_variant<F, 1, true>(jobs, njobs, nunits, grid, stream, queue);
    if (variant == 3) return launch_pack_variant<F, 1, false>(jobs, njobs, nunits, grid, stream, queue);
  } else {
    if (variant == 0) return launch_pack_variant<F, 3, true>(jobs, njobs, nunits, grid, stream, queue);
    if (variant == 1) return launch_pack_variant<F, 3, false>(jobs, njobs, nunits, grid, stream, queue);
  }
  return cudaErrorInvalidValue;
}

}  // namespace

cudaError_t launch_pack(const PackJob* jobs, uint32_t njobs, uint32_t nunits, uint32_t fmt, uint32_t variant,
                        cudaStream_t stream, uint32_t* queue, uint32_t persistent_ctas) {
  if (njobs == 0 || nunits == 0) return cudaSuccess;
  uint32_t ctas = (nunits + kIdwtWarps - 1) / kIdwtWarps;
  if (queue) ctas = std::max(1u, std::min(ctas, persistent_ctas));
  const dim3 grid(ctas);
  switch (fmt) {
    case PACK_GRAY8: return launch_pack_format<PACK_GRAY8>(variant, jobs, njobs, nunits, grid, stream, queue);
    case PACK_RGB8: return launch_pack_format<PACK_RGB8>(variant, jobs, njobs, nunits, grid, stream, queue);
    case PACK_RGBA8: return launch_pack_format<PACK_RGBA8>(variant, jobs, njobs, nunits, grid, stream, queue);
    case PACK_GRAY16: return launch_pack_format<PACK_GRAY16>(variant, jobs, njobs, nunits, grid, stream, queue);
    case PACK_RGB16: return launch_pack_format<PACK_RGB16>(variant, jobs, njobs, nunits, grid, stream, queue);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t idwt_pack_occupancy(uint32_t fmt, int* idwt_ctas_per_sm, int* pack_ctas_per_sm) {
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(idwt_ctas_per_sm, idwt_level_kernel<true>,
                                                                kIdwtWarps * 32, 0);
  if (e != cudaSuccess) return e;
  // Every variant has the same launch bounds and shared memory; the direct
  // one of the format stands for them.
  switch (fmt) {
#define SGN_PACK_OCC(F)                                                                                    \
    case F:                                                                                                 \
      return cudaOccupancyMaxActiveBlocksPerMultiprocessor(                                                 \
          pack_ctas_per_sm, pack_kernel<F, (F == PACK_GRAY8 || F == PACK_GRAY16) ? 1 : 3, true, true>,     \
          kIdwtWarps * 32, 0);
    SGN_PACK_OCC(PACK_GRAY8)
    SGN_PACK_OCC(PACK_RGB8)
    SGN_PACK_OCC(PACK_RGBA8)
    SGN_PACK_OCC(PACK_GRAY16)
    SGN_PACK_OCC(PACK_RGB16)
#undef SGN_PACK_OCC
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace sgn
