// Host emulation of the CUDA features the decode kernels use, so that their
// source compiles as C++ and runs on CPU threads under AddressSanitizer
// (test infrastructure only).  A CTA is blockDim std::threads; the lanes of a
// warp meet at a barrier in every shuffle, vote and __syncwarp, the CTA at
// every __syncthreads.  Every lane of a warp must reach each warp operation,
// which holds for the kernels (they only use them in warp-uniform control
// flow).  Floating-point intrinsics map to plain IEEE operations; the file is
// compiled with -ffp-contract=off so none is fused.
#pragma once
#include <algorithm>
#include <atomic>
#include <thread>
#include <barrier>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <cstdio>
#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __noinline__ __attribute__((noinline))
#define __launch_bounds__(...)
#define __restrict__
#define __shared__ static
#define __align__(n) __attribute__((aligned(n)))
typedef int cudaError_t;
typedef void* cudaStream_t;
struct dim3e { unsigned x = 0, y = 0, z = 0; };
extern thread_local dim3e threadIdx, blockIdx;
extern dim3e blockDim, gridDim;
struct int2 { int x, y; };
struct int4 { int x, y, z, w; };
struct uint4 { unsigned x, y, z, w; };
struct float4 { float x, y, z, w; };
struct uint2 { unsigned x, y; };
inline uint2 make_uint2(unsigned a, unsigned b) { return {a, b}; }
inline uint4 make_uint4(unsigned a, unsigned b, unsigned c, unsigned d) { return {a, b, c, d}; }
inline int2 make_int2(int a, int b) { return {a, b}; }
// Per-byte equality: 0xFF in each byte where a and b agree.
inline unsigned __vcmpeq4(unsigned a, unsigned b) {
  unsigned r = 0;
  for (int i = 0; i < 4; ++i)
    if (((a >> (8 * i)) & 0xFF) == ((b >> (8 * i)) & 0xFF)) r |= 0xFFu << (8 * i);
  return r;
}
inline int4 make_int4(int a, int b, int c, int d) { return {a, b, c, d}; }
inline float4 make_float4(float a, float b, float c, float d) { return {a, b, c, d}; }
template <class T> inline T __ldg(const T* p) { return *p; }
// L2 prefetch hints have no effect on the host; the range form still checks
// that every hinted address lies inside the range it was given.
inline void prefetch_l2(const void*) {}
inline void prefetch_l2_range(const void* p, size_t n, uint32_t first, uint32_t step) {
  if (n == 0) return;
  const uintptr_t a = (uintptr_t)p, end = a + n, line0 = a & ~(uintptr_t)127;
  for (uintptr_t q = line0 + (uintptr_t)first * 128; q < end; q += (uintptr_t)step * 128) {
    const uintptr_t h = q < a ? a : q;
    if (h < a || h >= end) std::abort();
    (void)*reinterpret_cast<const volatile uint8_t*>(h);  // under ASan: the byte must be addressable
  }
}
template <class T> inline T __ldcg(const T* p) { return *p; }
inline float __fmul_rn(float a, float b) { return a * b; }
inline float __fadd_rn(float a, float b) { return a + b; }
inline float __fdiv_rn(float a, float b) { return a / b; }
inline float __int2float_rn(int v) { return (float)v; }
inline float __int_as_float(int v) { float f; std::memcpy(&f, &v, 4); return f; }
inline int __popc(unsigned v) { return __builtin_popcount(v); }
using std::max;
using std::min;
struct WarpEmu {
  std::barrier<> bar{32};
  uint64_t slot[32];
};
extern thread_local WarpEmu* g_warp;
extern thread_local std::barrier<>* g_block;
inline void __syncthreads() { g_block->arrive_and_wait(); }
inline unsigned vote(bool p, int mode) {
  const int lane = threadIdx.x & 31;
  g_warp->slot[lane] = p ? 1 : 0;
  g_warp->bar.arrive_and_wait();
  unsigned m = 0;
  for (int i = 0; i < 32; ++i) m |= (unsigned)(g_warp->slot[i] & 1) << i;
  g_warp->bar.arrive_and_wait();
  return mode == 0 ? m : (m != 0);
}
inline unsigned __ballot_sync(unsigned, bool p) { return vote(p, 0); }
inline int __any_sync(unsigned, bool p) { return (int)vote(p, 1); }
inline int __all_sync(unsigned, bool p) { return vote(p, 0) == 0xFFFFFFFFu; }
inline unsigned __funnelshift_r(unsigned lo, unsigned hi, unsigned sh) {
  uint64_t v = ((uint64_t)hi << 32) | lo;
  return (unsigned)(v >> (sh & 31));
}
inline unsigned __funnelshift_l(unsigned lo, unsigned hi, unsigned sh) {
  uint64_t v = ((uint64_t)hi << 32) | lo;
  return (unsigned)((v << (sh & 31)) >> 32);
}
inline unsigned __funnelshift_lc(unsigned lo, unsigned hi, unsigned sh) {
  uint64_t v = ((uint64_t)hi << 32) | lo;
  sh = sh > 32 ? 32 : sh;
  return (unsigned)((v << sh) >> 32);
}
// The clamping right funnel shift: the low word of (hi:lo) >> min(sh, 32).
inline unsigned __funnelshift_rc(unsigned lo, unsigned hi, unsigned sh) {
  uint64_t v = ((uint64_t)hi << 32) | lo;
  sh = sh > 32 ? 32 : sh;
  return (unsigned)(v >> sh);
}
inline int __clz(unsigned v) { return v ? __builtin_clz(v) : 32; }
inline int __ffs(unsigned v) { return v ? __builtin_ctz(v) + 1 : 0; }
inline int __ffsll(long long v) { return v ? __builtin_ctzll((unsigned long long)v) + 1 : 0; }
inline unsigned __byte_perm(unsigned x, unsigned y, unsigned s) {
  uint8_t b[8];
  for (int i = 0; i < 4; ++i) { b[i] = (uint8_t)(x >> (8 * i)); b[4 + i] = (uint8_t)(y >> (8 * i)); }
  unsigned r = 0;
  for (int i = 0; i < 4; ++i) r |= (unsigned)b[(s >> (4 * i)) & 7] << (8 * i);
  return r;
}
inline unsigned atomicOr(unsigned* p, unsigned v) { return __atomic_fetch_or(p, v, __ATOMIC_SEQ_CST); }
extern uint8_t g_dyn_smem[];
template <class T> inline T shfl_from(T v, int src_of_lane_fn_lane, bool ok) {
  const int lane = threadIdx.x & 31;
  uint64_t bits = 0;
  std::memcpy(&bits, &v, sizeof(T));
  g_warp->slot[lane] = bits;
  g_warp->bar.arrive_and_wait();
  T r = v;
  if (ok) std::memcpy(&r, &g_warp->slot[src_of_lane_fn_lane], sizeof(T));
  g_warp->bar.arrive_and_wait();
  return r;
}
// Shuffles over segments of `width` lanes (a power of two, 32 by default):
// a source outside the caller's segment leaves the caller's own value.
template <class T> inline T __shfl_up_sync(unsigned, T v, int d, int width = 32) {
  const int lane = threadIdx.x & 31;
  return shfl_from(v, lane - d, (lane & (width - 1)) - d >= 0);
}
template <class T> inline T __shfl_down_sync(unsigned, T v, int d, int width = 32) {
  const int lane = threadIdx.x & 31;
  return shfl_from(v, lane + d, (lane & (width - 1)) + d < width);
}
template <class T> inline T __shfl_sync(unsigned, T v, int src, int width = 32) {
  const int lane = threadIdx.x & 31;
  return shfl_from(v, (lane & ~(width - 1)) + (src & (width - 1)), true);
}
template <class T> inline T __shfl_xor_sync(unsigned, T v, int m, int width = 32) {
  const int lane = threadIdx.x & 31, src = lane ^ m;
  return shfl_from(v, src & 31, (src & ~(width - 1)) == (lane & ~(width - 1)));
}
inline void __syncwarp() { g_warp->bar.arrive_and_wait(); }
// The fused kernel's producer and consumer warps meet through shared memory:
// fences order the host threads' accesses, a sleep yields the thread.
inline void __threadfence_block() { std::atomic_thread_fence(std::memory_order_seq_cst); }
inline void __nanosleep(unsigned) { std::this_thread::yield(); }
inline unsigned atomicAdd(unsigned* p, unsigned v) {
  unsigned o = __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST);
  return o;
}
