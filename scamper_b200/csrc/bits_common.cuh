// Helpers shared by the bit-sliced sweep kernels (Ising: 1 bit plane per
// parity; Potts q <= 4: 2 bit planes per parity): Philox with the
// sweep-uniform part of round 1 and the round keys hoisted out of the site
// loop, and the tile geometry (64-site row segments, rows with or without a
// two-row halo, whole rows or x-split column ranges).
#pragma once
#include "device_common.cuh"

namespace gpumc {

struct BitsPhilox {
  uint32_t a, b, c;
  uint32_t k0[10], k1[10];
};

__device__ __forceinline__ BitsPhilox make_bits_philox(uint64_t key, uint64_t sweep) {
  BitsPhilox P;
  const uint32_t k0 = (uint32_t)key, k1 = (uint32_t)(key >> 32);
  const uint32_t c2 = (uint32_t)sweep, c3 = (uint32_t)(sweep >> 32);
  P.a = __umulhi(0xCD9E8D57u, c2) ^ k0;
  P.b = 0xCD9E8D57u * c2;
  P.c = c3 ^ k1;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    P.k0[r] = k0 + (uint32_t)r * 0x9E3779B9u;
    P.k1[r] = k1 + (uint32_t)r * 0xBB67AE85u;
  }
  return P;
}

// Philox4x32-10 of counter (index, ctrl, sweep_lo, sweep_hi) with the
// sweep-uniform part of round 1 precomputed.  Each round multiply is a
// separate high and low product (measured 0.7 % faster in the resident Ising
// kernel than one 32x32->64 wide product, after the kernel's other changes;
// an earlier version of the kernel had it the other way round by 1 %).
__device__ __forceinline__ uint4 bits_philox(const BitsPhilox& P, uint32_t index, uint32_t ctrl) {
  const uint64_t p00 = (uint64_t)0xD2511F53u * index;
  uint4 c = make_uint4(P.a ^ ctrl, P.b, (uint32_t)(p00 >> 32) ^ P.c, (uint32_t)p00);
#pragma unroll
  for (int r = 1; r < 10; ++r) {
    const uint32_t h0 = __umulhi(0xD2511F53u, c.x), l0 = 0xD2511F53u * c.x;
    const uint32_t h1 = __umulhi(0xCD9E8D57u, c.z), l1 = 0xCD9E8D57u * c.z;
    c = make_uint4(h1 ^ c.y ^ P.k0[r], l1, h0 ^ c.w ^ P.k1[r], l0);
  }
  return c;
}

// Tile geometry: shared plane of R rows x NC columns of packed segments;
// column cc holds segment s0 + cc - xh (wrapped).
struct BitsGeom {
  int lx, ly, pitch, nseg;      // nseg = segments per row (pitch = 64 nseg)
  int s0, ns, xh, NC;           // first segment, owned segments, halo columns
  int y0, hv, R;                // rows y0-yo .. y0+hv+yo-1
  int yo;                       // halo rows above the tile (2), or 0 for a
  bool yw;                      // whole-plane 3D tile: rows wrap inside the tile
  int hlast;                    // valid site pairs of the last segment of a row
  int col, row0, rstep, iters_load, iters_black, iters_white;
  long long gbytes;             // bytes of one int8 buffer of the lattice (bounds checks)
  int pw;                       // words of one shared plane (R x NC)
};

__device__ __forceinline__ int wrap_i(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

__device__ __forceinline__ BitsGeom make_bits_geom(const TileItem& t, const LatDesc* L) {
  BitsGeom g;
  g.lx = L->lx;
  g.ly = L->ly;
  g.pitch = L->pitch;
  g.nseg = L->pitch >> 6;
  g.s0 = t.x0 >> 6;
  g.ns = min(t.cx, g.nseg - g.s0);
  g.xh = g.ns < g.nseg ? 1 : 0;
  g.NC = g.ns + 2 * g.xh;
  g.y0 = t.y0;
  g.hv = min(t.ty, g.ly - t.y0);
  // a 3D tile that spans whole planes needs no y halo: its rows wrap
  g.yw = L->dims == 3 && t.y0 == 0 && t.ty >= g.ly && g.xh == 0;
  g.yo = g.yw ? 0 : 2;
  g.R = g.yw ? g.hv : g.hv + 4;
  g.hlast = (g.lx - 64 * (g.nseg - 1)) >> 1;
  g.rstep = kThreads / g.NC;
  g.col = threadIdx.x % g.NC;
  g.row0 = threadIdx.x / g.NC;
  g.iters_load = (g.R + g.rstep - 1) / g.rstep;
  g.iters_black = (g.R - 2 + 2 * (g.yo == 0) + g.rstep - 1) / g.rstep;
  g.iters_white = (g.hv + g.rstep - 1) / g.rstep;
  g.gbytes = (long long)L->pitch * L->ly * (L->dims == 3 ? L->lz : 1);
  g.pw = g.R * g.NC;
  return g;
}

}  // namespace gpumc
