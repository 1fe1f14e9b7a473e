// Device helpers shared by the sweep kernels: Philox4x32-10 (Salmon, Moraes,
// Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11), the
// counter layout of the engine's random stream, and the exactly-rounded fp32
// arithmetic the O(3) update is specified in.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "engine.h"

namespace gpumc {

// Bounds-checked builds (compiled with -DGPUMC_DEBUG_BOUNDS; the stand-in for
// a memory sanitizer): GPUMC_IN(i, n) is true when 0 <= i < n; otherwise it
// counts the violation in this module's counters, keeps the first failing
// source line, and is false, so the guarded load or store is skipped instead
// of touching memory outside its buffer.  In release builds it is the
// constant true and compiles away.  Each compiled module has its own
// counters; bounds_read_<module>() (GPUMC_BOUNDS_MODULE) reads and clears them.
#ifdef GPUMC_DEBUG_BOUNDS
static __device__ unsigned long long g_bounds_hits;
static __device__ unsigned int g_bounds_line;
static __device__ __noinline__ bool bounds_fail(unsigned int line) {
  if (atomicAdd(&g_bounds_hits, 1ull) == 0ull) g_bounds_line = line;
  return false;
}
#define GPUMC_IN(i, n) \
  (((unsigned long long)(long long)(i) < (unsigned long long)(long long)(n)) || ::gpumc::bounds_fail(__LINE__))
#define GPUMC_BOUNDS_MODULE(name)                                                                   \
  int bounds_read_##name(unsigned long long* hits, unsigned int* line) {                           \
    const unsigned long long zero = 0;                                                              \
    if (cudaMemcpyFromSymbol(hits, g_bounds_hits, sizeof(*hits)) != cudaSuccess) return -1;         \
    if (cudaMemcpyFromSymbol(line, g_bounds_line, sizeof(*line)) != cudaSuccess) return -1;         \
    return cudaMemcpyToSymbol(g_bounds_hits, &zero, sizeof(zero)) == cudaSuccess ? 0 : -1;          \
  }
#else
#define GPUMC_IN(i, n) true
#define GPUMC_BOUNDS_MODULE(name)                                       \
  int bounds_read_##name(unsigned long long* hits, unsigned int* line) { \
    *hits = 0;                                                         \
    *line = 0;                                                         \
    return 1;                                                          \
  }
#endif

// Loads and stores of element i of a buffer of n elements, checked in
// bounds-checked builds (an out-of-range load returns zero).
template <typename T>
__device__ __forceinline__ T ld_chk(const T* p, long long i, long long n) {
  return GPUMC_IN(i, n) ? p[i] : T{};
}
template <typename T>
__device__ __forceinline__ void st_chk(T* p, long long i, long long n, T v) {
  if (GPUMC_IN(i, n)) p[i] = v;
}

__device__ __forceinline__ uint4 philox10(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
    const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
    c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
  }
  return c;
}

// Counter: word0 = index (chunk id or site id), word1 = colour | tag << 1 |
// plane_pair << 8 | (index >> 32) << 16, words 2/3 = sweep.
__device__ __forceinline__ uint4 draw(uint64_t key, uint64_t index, uint32_t colour, uint32_t tag,
                                      uint32_t plane_pair, uint64_t sweep) {
  uint4 c = make_uint4((uint32_t)index,
                       colour | (tag << 1) | (plane_pair << 8) | ((uint32_t)(index >> 32) << 16),
                       (uint32_t)sweep, (uint32_t)(sweep >> 32));
  return philox10(c, (uint32_t)key, (uint32_t)(key >> 32));
}

// Philox4x32-10 of counter (index, ctrl, sweep) with the sweep-uniform part
// of round 1 precomputed and the round keys bumped on the fly: five
// registers, for kernels where resident warps matter more than two adds per
// round.  ctrl0 (given once) and ctrl (per call) are XORed into word 1, so a
// call equals draw() with word 1 = ctrl0 ^ ctrl.  Each round multiply is a
// separate high and low product.
struct RunPhilox {
  uint32_t a, b, c, k0, k1;
};
__device__ __forceinline__ RunPhilox make_run_philox(uint64_t key, uint64_t sweep, uint32_t ctrl0) {
  RunPhilox P;
  P.k0 = (uint32_t)key;
  P.k1 = (uint32_t)(key >> 32);
  const uint32_t c2 = (uint32_t)sweep, c3 = (uint32_t)(sweep >> 32);
  P.a = __umulhi(0xCD9E8D57u, c2) ^ P.k0 ^ ctrl0;
  P.b = 0xCD9E8D57u * c2;
  P.c = c3 ^ P.k1;
  return P;
}
__device__ __forceinline__ uint4 run_philox(const RunPhilox& P, uint32_t index, uint32_t ctrl) {
  const uint64_t p00 = (uint64_t)0xD2511F53u * index;
  uint4 c = make_uint4(P.a ^ ctrl, P.b, (uint32_t)(p00 >> 32) ^ P.c, (uint32_t)p00);
  uint32_t k0 = P.k0, k1 = P.k1;
#pragma unroll
  for (int r = 1; r < 10; ++r) {
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
    // separate high and low products (the multi-spin kernel measured 10 %
    // faster than with one 32x32->64 wide product per multiply)
    const uint32_t h0 = __umulhi(0xD2511F53u, c.x), l0 = 0xD2511F53u * c.x;
    const uint32_t h1 = __umulhi(0xCD9E8D57u, c.z), l1 = 0xCD9E8D57u * c.z;
    c = make_uint4(h1 ^ c.y ^ k0, l1, h0 ^ c.w ^ k1, l0);
  }
  return c;
}

// v wrapped into [0, n) for v in [-n, 2n) (halo coordinates): no division
__device__ __forceinline__ int wrap1(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

__device__ __forceinline__ int wrapi(int v, int n) {
  v %= n;
  return v < 0 ? v + n : v;
}

// Exact decision u < T for the 80-bit threshold T = head:tail, given the
// 16-bit head draw u16 that already tied with head.
static __device__ __noinline__ bool refine_accept(uint64_t key, uint64_t site, uint32_t colour,
                                           uint64_t sweep, unsigned long long tail) {
  uint4 o = draw(key, site, colour, TAG_ACC_REFINE, 0, sweep);
  unsigned long long r = (unsigned long long)o.x | ((unsigned long long)o.y << 32);
  return r < tail;
}

// Potts proposal: uniform r in [0, n) from a 16-bit draw with Lemire's
// multiply-shift and exact rejection; rejected draws retry with 32-bit values
// from a per-site refine batch.
static __device__ __noinline__ uint32_t potts_refine(uint64_t key, uint64_t site, uint32_t colour,
                                              uint64_t sweep, uint32_t n) {
  uint4 o = draw(key, site, colour, TAG_PROP_REFINE, 0, sweep);
  const uint32_t rej = (uint32_t)(0x100000000ull % n);
  uint32_t v[4] = {o.x, o.y, o.z, o.w};
  unsigned long long m = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    m = (unsigned long long)v[i] * n;
    if ((uint32_t)m >= rej) return (uint32_t)(m >> 32);
  }
  return (uint32_t)(m >> 32);
}

// ---- exactly rounded fp32 building blocks (no contraction into FMA) ------
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float fsqrt(float a) { return __fsqrt_rn(a); }

// exp(x) for x <= 0: Cody-Waite split into 2^n * e^t with |t| <= ln2/2 and
// the degree-7 Taylor polynomial of e^t (truncation error < 5e-9 relative).
__device__ __forceinline__ float exp_neg(float x) {
  if (!(x <= 0.0f)) return 1.0f;
  if (x < -87.0f) return 0.0f;
  const float y = fmul(x, 0x1.715476p+0f);
  const float n = floorf(fadd(y, 0.5f));
  const float f = fsub(y, n);
  const float t = fmul(f, 0x1.62e430p-1f);
  // Horner steps as fused multiply-adds (one rounding each)
  float p = 0x1.a01a02p-13f;
  p = __fmaf_rn(p, t, 0x1.6c16c2p-10f);
  p = __fmaf_rn(p, t, 0x1.111112p-7f);
  p = __fmaf_rn(p, t, 0x1.555556p-5f);
  p = __fmaf_rn(p, t, 0x1.555556p-3f);
  p = __fmaf_rn(p, t, 0.5f);
  p = __fmaf_rn(p, t, 1.0f);
  p = __fmaf_rn(p, t, 1.0f);
  const int ni = (int)n;
  const float scale = __int_as_float((ni + 127) << 23);
  return fmul(p, scale);
}

// (cos, sin) of 2*pi*u/2^32: octant from the top 3 bits, the angle inside the
// octant from the next 24 bits, Taylor polynomials on [0, pi/4] evaluated
// with fused multiply-adds; the octant swaps and negates the pair.
__device__ __forceinline__ void sincos_turn(uint32_t u, float& c, float& s) {
  const uint32_t octant = u >> 29;
  float t = fmul((float)((u >> 5) & 0xFFFFFFu), 0x1p-24f);
  if (octant & 1u) t = fsub(1.0f, t);
  const float th = fmul(t, 0x1.921fb6p-1f);
  const float t2 = fmul(th, th);
  float sp = 0x1.71de3ap-19f;
  sp = __fmaf_rn(sp, t2, -0x1.a01a02p-13f);
  sp = __fmaf_rn(sp, t2, 0x1.111112p-7f);
  sp = __fmaf_rn(sp, t2, -0x1.555556p-3f);
  sp = __fmaf_rn(sp, t2, 1.0f);
  const float sn = fmul(th, sp);
  float cp = -0x1.27e4fcp-22f;
  cp = __fmaf_rn(cp, t2, 0x1.a01a02p-16f);
  cp = __fmaf_rn(cp, t2, -0x1.6c16c2p-10f);
  cp = __fmaf_rn(cp, t2, 0x1.555556p-5f);
  cp = __fmaf_rn(cp, t2, -0.5f);
  const float cs = __fmaf_rn(cp, t2, 1.0f);
  // octants 1, 2, 5, 6 swap; cos < 0 in octants 2..5, sin < 0 in 4..7
  const bool sw = ((octant + 1u) & 2u) != 0u;
  const float a = sw ? sn : cs, b = sw ? cs : sn;
  c = ((octant + 2u) & 4u) ? -a : a;
  s = (octant & 4u) ? -b : b;
}

// 1 - exp(-x) for x >= 0: the Taylor series x (1 - x/2 + x^2/6 - ... +
// x^8/9!) in Horner form with fused multiply-adds below x = 1/2 (truncation
// < 1e-9 relative), else 1 - exp_neg(-x) (no cancellation there).
__device__ __forceinline__ float one_minus_exp_neg(float x) {
  if (x < 0.5f) {
    float p = 0x1.71de3ap-19f;
    p = __fmaf_rn(p, x, -0x1.a01a02p-16f);
    p = __fmaf_rn(p, x, 0x1.a01a02p-13f);
    p = __fmaf_rn(p, x, -0x1.6c16c2p-10f);
    p = __fmaf_rn(p, x, 0x1.111112p-7f);
    p = __fmaf_rn(p, x, -0x1.555556p-5f);
    p = __fmaf_rn(p, x, 0x1.555556p-3f);
    p = __fmaf_rn(p, x, -0.5f);
    p = __fmaf_rn(p, x, 1.0f);
    return fmul(x, p);
  }
  return fsub(1.0f, exp_neg(-x));
}

// 2 atanh(s) = ln((1 + s) / (1 - s)) for |s| <= 0.1716: 2 s (1 + s^2/3 + ... +
// s^10/11), Horner in s^2 with fused multiply-adds (truncation < 1e-10).
__device__ __forceinline__ float two_atanh_small(float s) {
  const float s2 = fmul(s, s);
  float q = 0x1.745d18p-4f;
  q = __fmaf_rn(q, s2, 0x1.c71c72p-4f);
  q = __fmaf_rn(q, s2, 0x1.24924ap-3f);
  q = __fmaf_rn(q, s2, 0x1.99999ap-3f);
  q = __fmaf_rn(q, s2, 0x1.555556p-2f);
  q = __fmaf_rn(q, s2, 1.0f);
  return fmul(fmul(2.0f, s), q);
}

// ln(1 - y) for 0 <= y < 1 - 2^-25.  Below y = 1/4 from y directly
// (s = -y / (2 - y), no rounding of 1 - y); above, from z = 1 - y (exact for
// y >= 1/2) split as m 2^e with m in [sqrt(1/2), sqrt(2)]:
// ln z = e ln 2 + 2 atanh((m - 1) / (m + 1)).
__device__ __forceinline__ float log_one_minus(float y) {
  if (y < 0.25f) return two_atanh_small(fdiv(-y, fsub(2.0f, y)));
  const float z = fsub(1.0f, y);
  const int bits = __float_as_int(z);
  int e = (bits >> 23) - 127;
  float m = __int_as_float((bits & 0x7FFFFF) | 0x3F800000);
  if (m > 0x1.6a09e6p+0f) {
    m = fmul(m, 0.5f);
    e += 1;
  }
  const float sm = fdiv(fsub(m, 1.0f), fadd(m, 1.0f));
  return fadd(fmul((float)e, 0x1.62e430p-1f), two_atanh_small(sm));
}

// log-space Metropolis decision of Carlo.rs/src/acceptance.rs:11-22 with u
// built from the top 53 bits of a 64-bit draw.
__device__ __forceinline__ bool accept_log(double logA, unsigned long long u64) {
  if (isnan(logA)) return false;
  if (logA >= 0.0) return true;
  if (isinf(logA)) return false;
  double u = (double)(u64 >> 11) * 0x1p-53;
  if (u < 2.2250738585072014e-308) u = 2.2250738585072014e-308;
  return log(u) < logA;
}

__device__ __forceinline__ void atomic_add_i64(unsigned long long* p, long long v) {
  atomicAdd(p, (unsigned long long)v);
}

// CTA-wide sums of N per-thread values (long long or double): a shuffle tree
// per warp, then thread 0 adds the other warps' totals in warp order and
// returns with the CTA's totals in v.  Every thread of the CTA must call it.
// The caller then issues one atomic per accumulator per CTA instead of one
// per warp: same-address atomics serialise in L2, which launches of many
// small tiles would otherwise wait on.
template <typename T, int N>
__device__ __forceinline__ void cta_sum(T (&v)[N]) {
  __shared__ T part[kThreads / 32][N];
  const unsigned full = 0xFFFFFFFFu;
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_xor_sync(full, v[i], o);
  __syncthreads();  // a previous call's reads of `part` are over
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int i = 0; i < N; ++i) part[threadIdx.x >> 5][i] = v[i];
  __syncthreads();
  if (threadIdx.x == 0)
    for (int w = 1; w < kThreads / 32; ++w)
#pragma unroll
      for (int i = 0; i < N; ++i) v[i] += part[w][i];
}

}  // namespace gpumc
