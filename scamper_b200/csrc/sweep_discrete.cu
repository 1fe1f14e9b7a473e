// Fused two-colour checkerboard sweep for int8 Ising and q-state Potts spins
// on periodic square (2D) and cubic (3D) lattices.
//
// Method (one kernel launch = one full sweep of every lattice in the launch):
//   * each CTA owns a tile of one lattice: tile_cx 16-site chunks x tile_y
//     rows (x tile_z planes in 3D, marched plane by plane through a 4-slot
//     shared-memory ring);
//   * it stages the tile plus a 2-site halo from the read buffer into shared
//     memory, updates colour 0 on the tile and a 1-site halo ring (halo sites
//     are recomputed redundantly: the counter-based RNG makes them identical to
//     the owner's result), then colour 1 on the tile, and writes the tile to
//     the other ping-pong buffer.  HBM traffic is one read and one write of
//     every byte per sweep.
//   * spins are handled 16 at a time (one uint4): neighbour counts come from
//     SWAR byte arithmetic on 32-bit words, one Philox4x32-10 call supplies the
//     eight 16-bit acceptance draws of a chunk's eight same-colour sites, and a
//     draw that ties the 16-bit threshold head is refined with 64 more bits
//     (acceptance exact to 2^-80 against the f64 exp(-beta dE)).
//
// Reference semantics restated: Ising dE (CMC.rs/src/lattice/interaction.rs:
// 73-84, :149-181), Potts proposal uniform over the other q-1 states
// (CMC.rs/src/lattice/models.rs:212-218), acceptance min(1, exp(-beta dE))
// (Carlo.rs/src/acceptance.rs:11-22), cached energy += dE
// (CMC.rs/src/lattice/state.rs:127-136), observables Energy and |M|
// (CMC.rs/src/observables/*.rs).  The visit order is the checkerboard, not the
// reference's random permutation (CMC.rs/src/core/visit.rs:50-56); both
// sample the same Boltzmann distribution.
#include "device_common.cuh"
#include "epilogue.cuh"

namespace gpumc {

constexpr int kMaxItems = 6;  // chunk items per thread in one colour pass
constexpr uint32_t kM2 = 0x02020202u;

struct SiteTab {
  uint32_t head[kMaxClasses];
  unsigned long long tail[kMaxClasses];
};

// Per-chunk update of the sites of one colour.  `bp` = byte parity of the
// colour's sites, `owned` = bitmask of bytes owned by this tile (for the
// energy accounting), `site0` = linear site index of byte 0.
template <int MODEL, int DIM>
__device__ __forceinline__ uint4 update_chunk(const uint4 own, const uint4 up, const uint4 dn,
                                              const uint4 zm, const uint4 zp, uint32_t wprev,
                                              uint32_t wnext, int bp, const uint4 rnd,
                                              const uint4 rprop, const SiteTab& tab, int q,
                                              uint64_t key, uint64_t site0, uint32_t colour,
                                              uint64_t sweep, uint32_t owned, int& dE, int& nacc) {
  constexpr int zc = 2 * DIM;
  const uint32_t o[4] = {own.x, own.y, own.z, own.w};
  const uint32_t u[4] = {up.x, up.y, up.z, up.w};
  const uint32_t d[4] = {dn.x, dn.y, dn.z, dn.w};
  const uint32_t a[4] = {zm.x, zm.y, zm.z, zm.w};
  const uint32_t b[4] = {zp.x, zp.y, zp.z, zp.w};
  const uint32_t rr[4] = {rnd.x, rnd.y, rnd.z, rnd.w};
  const uint32_t rp[4] = {rprop.x, rprop.y, rprop.z, rprop.w};
  uint32_t res[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint32_t lw = __funnelshift_l(i == 0 ? wprev : o[i - 1], o[i], 8);
    const uint32_t rw = __funnelshift_r(o[i], i == 3 ? wnext : o[i + 1], 8);
    uint32_t out = o[i];
    if (MODEL == ISING) {
      uint32_t k2 = ((o[i] ^ lw) & kM2) + ((o[i] ^ rw) & kM2) + ((o[i] ^ u[i]) & kM2) +
                    ((o[i] ^ d[i]) & kM2);
      if (DIM == 3) k2 += ((o[i] ^ a[i]) & kM2) + ((o[i] ^ b[i]) & kM2);
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int sb = bp + 2 * j;
        const int sh = 8 * sb;
        const int k = (k2 >> (sh + 1)) & 7;
        const uint32_t uu = j ? (rr[i] >> 16) : (rr[i] & 0xFFFFu);
        const uint32_t th = tab.head[k];
        bool acc = uu < th;
        if (uu == th)
          acc = refine_accept(key, site0 + 4 * i + sb, colour, sweep, tab.tail[k]);
        if (acc) {
          out ^= 0xFEu << sh;
          if ((owned >> (4 * i + sb)) & 1u) {
            dE += 2 * (zc - 2 * k);
            ++nacc;
          }
        }
      }
    } else {
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int sb = bp + 2 * j;
        const int sh = 8 * sb;
        const uint32_t s = (o[i] >> sh) & 0xFFu;
        const uint32_t pu = j ? (rp[i] >> 16) : (rp[i] & 0xFFFFu);
        const uint32_t n = (uint32_t)(q - 1);
        const uint32_t m = pu * n;
        uint32_t r = m >> 16;
        if ((m & 0xFFFFu) < (65536u % n)) r = potts_refine(key, site0 + 4 * i + sb, colour, sweep, n);
        const uint32_t t = r < s ? r : r + 1;
        const uint32_t nb0 = (lw >> sh) & 0xFFu, nb1 = (rw >> sh) & 0xFFu;
        const uint32_t nb2 = (u[i] >> sh) & 0xFFu, nb3 = (d[i] >> sh) & 0xFFu;
        int nold = (nb0 == s) + (nb1 == s) + (nb2 == s) + (nb3 == s);
        int nnew = (nb0 == t) + (nb1 == t) + (nb2 == t) + (nb3 == t);
        if (DIM == 3) {
          const uint32_t nb4 = (a[i] >> sh) & 0xFFu, nb5 = (b[i] >> sh) & 0xFFu;
          nold += (nb4 == s) + (nb5 == s);
          nnew += (nb4 == t) + (nb5 == t);
        }
        const int dd = nnew - nold;
        const int cls = dd + zc;
        const uint32_t uu = j ? (rr[i] >> 16) : (rr[i] & 0xFFFFu);
        const uint32_t th = tab.head[cls];
        bool acc = uu < th;
        if (uu == th)
          acc = refine_accept(key, site0 + 4 * i + sb, colour, sweep, tab.tail[cls]);
        if (acc) {
          out = (out & ~(0xFFu << sh)) | (t << sh);
          if ((owned >> (4 * i + sb)) & 1u) {
            dE -= dd;
            ++nacc;
          }
        }
      }
    }
    res[i] = out;
  }
  return make_uint4(res[0], res[1], res[2], res[3]);
}

// Scalar update of one halo site held in shared memory at `p` (row stride S,
// plane pointers zmp/zpp for 3D).  The site's draws come from its own chunk.
template <int MODEL, int DIM>
__device__ __forceinline__ int8_t update_site(const int8_t* p, int S, const int8_t* zmp,
                                              const int8_t* zpp, int xr, int y, int z, int ly,
                                              int lx, int pc, const SiteTab& tab, int q,
                                              uint64_t key, uint32_t colour, uint64_t sweep) {
  constexpr int zc = 2 * DIM;
  const int8_t s = p[0];
  int8_t nb[6] = {p[-1], p[1], p[-S], p[S], 0, 0};
  if (DIM == 3) {
    nb[4] = zmp[0];
    nb[5] = zpp[0];
  }
  const uint64_t rho = (uint64_t)y + (uint64_t)ly * (uint64_t)z;
  const uint64_t chunk = rho * (uint64_t)pc + (uint64_t)(xr >> 4);
  const uint64_t site = rho * (uint64_t)lx + (uint64_t)xr;
  const int slot = (xr & 15) >> 1;
  const uint4 rv = draw(key, chunk, colour, TAG_ACC, 0, sweep);
  const uint32_t w = (slot >> 1) == 0 ? rv.x : (slot >> 1) == 1 ? rv.y : (slot >> 1) == 2 ? rv.z : rv.w;
  const uint32_t uu = (slot & 1) ? (w >> 16) : (w & 0xFFFFu);
  if (MODEL == ISING) {
    int k = 0;
#pragma unroll
    for (int i = 0; i < zc; ++i) k += nb[i] != s;
    const uint32_t th = tab.head[k];
    bool acc = uu < th;
    if (uu == th) acc = refine_accept(key, site, colour, sweep, tab.tail[k]);
    return acc ? (int8_t)-s : s;
  } else {
    const uint4 pv = draw(key, chunk, colour, TAG_PROP, 0, sweep);
    const uint32_t pw = (slot >> 1) == 0 ? pv.x : (slot >> 1) == 1 ? pv.y : (slot >> 1) == 2 ? pv.z : pv.w;
    const uint32_t pu = (slot & 1) ? (pw >> 16) : (pw & 0xFFFFu);
    const uint32_t n = (uint32_t)(q - 1);
    const uint32_t m = pu * n;
    uint32_t r = m >> 16;
    if ((m & 0xFFFFu) < (65536u % n)) r = potts_refine(key, site, colour, sweep, n);
    const int t = (int)r < s ? (int)r : (int)r + 1;
    int nold = 0, nnew = 0;
#pragma unroll
    for (int i = 0; i < zc; ++i) {
      nold += nb[i] == s;
      nnew += nb[i] == t;
    }
    const int cls = nnew - nold + zc;
    const uint32_t th = tab.head[cls];
    bool acc = uu < th;
    if (uu == th) acc = refine_accept(key, site, colour, sweep, tab.tail[cls]);
    return acc ? (int8_t)t : s;
  }
}

__device__ __forceinline__ uint32_t owned_bytes(int remaining) {
  // bit b set for bytes b < remaining (remaining = valid bytes in this chunk)
  if (remaining >= 16) return 0xFFFFu;
  if (remaining <= 0) return 0u;
  return (1u << remaining) - 1u;
}

struct PlaneGeom {
  int x0, W, S, Wv, ncv, R;  // R = rows held per plane = Hv + 4
};

// Stage rows y0-2 .. y0+Hv+1 of plane z into a shared-memory plane buffer.
__device__ __forceinline__ void load_plane(uint8_t* plane, const int8_t* src, int pitch, int lx,
                                           int ly, int y0, int z, const PlaneGeom& g) {
  const int tid = threadIdx.x;
  for (int i = tid; i < g.R * g.ncv; i += kThreads) {
    const int r = i / g.ncv, c = i - r * g.ncv;
    const int y = wrapi(y0 - 2 + r, ly);
    const size_t off = ((size_t)z * ly + y) * (size_t)pitch + g.x0 + 16 * c;
    *(uint4*)(plane + r * g.S + 16 + 16 * c) = __ldg((const uint4*)(src + off));
  }
}
// Write the wrapped x-halo bytes (x0-2, x0-1, x0+Wv, x0+Wv+1) of every row.
__device__ __forceinline__ void load_plane_halo(uint8_t* plane, const int8_t* src, int pitch,
                                                int lx, int ly, int y0, int z,
                                                const PlaneGeom& g) {
  const int tid = threadIdx.x;
  for (int i = tid; i < g.R * 4; i += kThreads) {
    const int r = i >> 2, j = i & 3;
    const int pos = j < 2 ? g.x0 - 2 + j : g.x0 + g.Wv + (j - 2);
    const int y = wrapi(y0 - 2 + r, ly);
    const int xr = wrapi(pos, lx);
    plane[r * g.S + 16 + (pos - g.x0)] = src[((size_t)z * ly + y) * (size_t)pitch + xr];
  }
}

// Colour-0 pass on rows [1, R-1) of `plane` (tile + 1-row halo), results held
// in registers, then written back after a barrier; halo columns x0-1 and
// x0+Wv are recomputed with the scalar path.
template <int MODEL, int DIM>
__device__ __forceinline__ void black_pass(uint8_t* plane, const uint8_t* pzm, const uint8_t* pzp,
                                           const PlaneGeom& g, int y0, int z, int ly, int lx,
                                           int pc, int hv, const SiteTab& tab, int q, uint64_t key,
                                           uint64_t sweep, bool owned_plane, int& dE, int& nacc) {
  const int tid = threadIdx.x;
  const int rows = g.R - 2;
  const int nitems = rows * g.ncv;
  uint4 res[kMaxItems];
  const uint4 zero4 = make_uint4(0, 0, 0, 0);
#pragma unroll
  for (int it = 0; it < kMaxItems; ++it) {
    const int i = tid + it * kThreads;
    if (i < nitems) {
      const int r = 1 + i / g.ncv, c = i - (r - 1) * g.ncv;
      const uint8_t* p = plane + r * g.S + 16 + 16 * c;
      const int y = wrapi(y0 - 2 + r, ly);
      const int x = g.x0 + 16 * c;
      const uint4 own = *(const uint4*)p;
      const uint4 up = *(const uint4*)(p - g.S);
      const uint4 dn = *(const uint4*)(p + g.S);
      uint4 zmv = zero4, zpv = zero4;
      if (DIM == 3) {
        zmv = *(const uint4*)(pzm + (p - plane));
        zpv = *(const uint4*)(pzp + (p - plane));
      }
      const uint32_t wprev = *(const uint32_t*)(p - 4);
      const uint32_t wnext = *(const uint32_t*)(p + 16);
      const int bp = (y + z) & 1;
      const uint64_t rho = (uint64_t)y + (uint64_t)ly * (uint64_t)z;
      const uint64_t chunk = rho * (uint64_t)pc + (uint64_t)(x >> 4);
      const uint4 rnd = draw(key, chunk, 0, TAG_ACC, 0, sweep);
      const uint4 rpr = MODEL == POTTS ? draw(key, chunk, 0, TAG_PROP, 0, sweep) : zero4;
      const bool row_owned = owned_plane && r >= 2 && r < 2 + hv;
      const uint32_t owned = row_owned ? owned_bytes(g.Wv - 16 * c) : 0u;
      res[it] = update_chunk<MODEL, DIM>(own, up, dn, zmv, zpv, wprev, wnext, bp, rnd, rpr, tab, q,
                                         key, rho * (uint64_t)lx + (uint64_t)x, 0u, sweep, owned,
                                         dE, nacc);
    }
  }
  // scalar halo sites: two per row
  int8_t hval = 0;
  int hoff = -1;
  if (tid < rows * 2) {
    const int r = 1 + (tid >> 1);
    const int pos = (tid & 1) ? g.x0 + g.Wv : g.x0 - 1;
    const int y = wrapi(y0 - 2 + r, ly);
    const int xr = wrapi(pos, lx);
    const int off = r * g.S + 16 + (pos - g.x0);
    if (((xr + y + z) & 1) == 0) {
      hoff = off;
      hval = update_site<MODEL, DIM>((const int8_t*)plane + off, g.S, (const int8_t*)pzm + off,
                                     (const int8_t*)pzp + off, xr, y, z, ly, lx, pc, tab, q, key,
                                     0u, sweep);
    }
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < kMaxItems; ++it) {
    const int i = tid + it * kThreads;
    if (i < nitems) {
      const int r = 1 + i / g.ncv, c = i - (r - 1) * g.ncv;
      *(uint4*)(plane + r * g.S + 16 + 16 * c) = res[it];
    }
  }
  __syncthreads();
  if (hoff >= 0) plane[hoff] = (uint8_t)hval;
  __syncthreads();
}

// Colour-1 pass on the tile rows, writing the finished chunks to HBM and
// accumulating the magnetisation / Potts histogram of owned sites.
template <int MODEL, int DIM>
__device__ __forceinline__ void white_pass(const uint8_t* plane, const uint8_t* pzm,
                                           const uint8_t* pzp, const PlaneGeom& g, int y0, int z,
                                           int ly, int lx, int pc, int pitch, int hv,
                                           const SiteTab& tab, int q, uint64_t key, uint64_t sweep,
                                           int8_t* dst, int& dE, int& nacc, int& mag,
                                           int* cnt) {
  const int tid = threadIdx.x;
  const int nitems = hv * g.ncv;
  const uint4 zero4 = make_uint4(0, 0, 0, 0);
  for (int i = tid; i < nitems; i += kThreads) {
    const int r = 2 + i / g.ncv, c = i - (r - 2) * g.ncv;
    const uint8_t* p = plane + r * g.S + 16 + 16 * c;
    const int y = wrapi(y0 - 2 + r, ly);
    const int x = g.x0 + 16 * c;
    const uint4 own = *(const uint4*)p;
    const uint4 up = *(const uint4*)(p - g.S);
    const uint4 dn = *(const uint4*)(p + g.S);
    uint4 zmv = zero4, zpv = zero4;
    if (DIM == 3) {
      zmv = *(const uint4*)(pzm + (p - plane));
      zpv = *(const uint4*)(pzp + (p - plane));
    }
    const uint32_t wprev = *(const uint32_t*)(p - 4);
    const uint32_t wnext = *(const uint32_t*)(p + 16);
    const int bp = (1 + y + z) & 1;
    const uint64_t rho = (uint64_t)y + (uint64_t)ly * (uint64_t)z;
    const uint64_t chunk = rho * (uint64_t)pc + (uint64_t)(x >> 4);
    const uint4 rnd = draw(key, chunk, 1, TAG_ACC, 0, sweep);
    const uint4 rpr = MODEL == POTTS ? draw(key, chunk, 1, TAG_PROP, 0, sweep) : zero4;
    const uint32_t owned = owned_bytes(g.Wv - 16 * c);
    const uint4 res = update_chunk<MODEL, DIM>(own, up, dn, zmv, zpv, wprev, wnext, bp, rnd, rpr,
                                               tab, q, key, rho * (uint64_t)lx + (uint64_t)x, 1u,
                                               sweep, owned, dE, nacc);
    *(uint4*)(dst + rho * (uint64_t)pitch + x) = res;
    const uint32_t w[4] = {res.x, res.y, res.z, res.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const uint32_t nib = (owned >> (4 * k)) & 0xFu;
      const uint32_t bm = (nib & 1u ? 0xFFu : 0u) | (nib & 2u ? 0xFF00u : 0u) |
                          (nib & 4u ? 0xFF0000u : 0u) | (nib & 8u ? 0xFF000000u : 0u);
      if (MODEL == ISING) {
        mag = __dp4a((int)(w[k] & bm), 0x01010101, mag);
      } else {
#pragma unroll
        for (int s = 0; s < kMaxPottsCounts; ++s) {
          if (s < q) {
            const uint32_t x8 = w[k] ^ (0x01010101u * (uint32_t)s);
            // bytes equal to s -> 0x80 flag
            const uint32_t t8 = ((x8 & 0x7F7F7F7Fu) + 0x7F7F7F7Fu);
            const uint32_t z8 = ~(t8 | x8 | 0x7F7F7F7Fu) & bm;
            cnt[s] += __popc(z8);
          }
        }
      }
    }
  }
}

template <int MODEL>
__device__ __forceinline__ void flush_accumulators(LatDesc* L, int dE, int nacc, int mag,
                                                   const int* cnt, int q) {
  // warp reduction, then one atomic per warp
  const unsigned full = 0xFFFFFFFFu;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    dE += __shfl_xor_sync(full, dE, o);
    nacc += __shfl_xor_sync(full, nacc, o);
    mag += __shfl_xor_sync(full, mag, o);
  }
  int c[kMaxPottsCounts];
#pragma unroll
  for (int s = 0; s < kMaxPottsCounts; ++s) {
    c[s] = cnt[s];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c[s] += __shfl_xor_sync(full, c[s], o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (dE) atomic_add_i64(&L->acc.dE, dE);
    if (nacc) atomic_add_i64(&L->acc.accepted, nacc);
    if (MODEL == ISING) {
      if (mag) atomic_add_i64(&L->acc.mag, mag);
    } else {
      for (int s = 0; s < kMaxPottsCounts && s < q; ++s)
        if (c[s]) atomic_add_i64(&L->acc.counts[s], c[s]);
    }
  }
}

__device__ __forceinline__ void load_table(SiteTab& tab, const LatDesc* L, const GroupDesc* G) {
  const int label = G->label[L->replica];
  for (int i = threadIdx.x; i < G->n_cls; i += kThreads) {
    tab.head[i] = G->head[label * G->n_cls + i];
    tab.tail[i] = G->tail[label * G->n_cls + i];
  }
}

template <int MODEL>
__global__ void __launch_bounds__(kThreads)
    k_sweep_discrete_2d(const TileItem* __restrict__ tiles, LatDesc* __restrict__ lats,
                        GroupDesc* __restrict__ groups, LaunchCtl* __restrict__ ctl) {
  extern __shared__ __align__(16) uint8_t smem[];
  __shared__ SiteTab tab;
  const TileItem t = tiles[blockIdx.x];
  LatDesc* L = &lats[t.lat];
  const GroupDesc* G = &groups[L->group];
  const int lx = L->lx, ly = L->ly, pitch = L->pitch, q = L->q;
  const uint64_t sweep = L->sweep, key = L->key;
  if (sweep >= L->target) {  // finished lattice: nothing to do this launch
    launch_epilogue(lats, groups, ctl);
    return;
  }
  const int8_t* cur = (const int8_t*)L->buf[sweep & 1];
  int8_t* nxt = (int8_t*)L->buf[(sweep & 1) ^ 1];
  load_table(tab, L, G);
  PlaneGeom g;
  g.x0 = t.x0;
  g.W = L->tile_cx * 16;
  g.S = g.W + 32;
  g.Wv = min(g.W, lx - t.x0);
  g.ncv = (g.Wv + 15) >> 4;
  const int hv = min(L->tile_y, ly - t.y0);
  g.R = hv + 4;
  const int pc = pitch >> 4;
  load_plane(smem, cur, pitch, lx, ly, t.y0, 0, g);
  __syncthreads();
  load_plane_halo(smem, cur, pitch, lx, ly, t.y0, 0, g);
  __syncthreads();
  int dE = 0, nacc = 0, mag = 0;
  int cnt[kMaxPottsCounts] = {0, 0, 0, 0, 0, 0, 0, 0};
  black_pass<MODEL, 2>(smem, smem, smem, g, t.y0, 0, ly, lx, pc, hv, tab, q, key, sweep, true, dE,
                       nacc);
  white_pass<MODEL, 2>(smem, smem, smem, g, t.y0, 0, ly, lx, pc, pitch, hv, tab, q, key, sweep,
                       nxt, dE, nacc, mag, cnt);
  flush_accumulators<MODEL>(L, dE, nacc, mag, cnt, q);
  launch_epilogue(lats, groups, ctl);
}

// 3D: the tile is tile_cx chunks x tile_y rows in the xy plane, marched over
// tile_z planes.  Step s loads plane z0-2+s, updates colour 0 on plane
// z0-3+s (its z neighbours are the still-old colour-1 planes around it) and
// colour 1 on plane z0-4+s (whose z neighbours have finished colour 0).
template <int MODEL>
__global__ void __launch_bounds__(kThreads)
    k_sweep_discrete_3d(const TileItem* __restrict__ tiles, LatDesc* __restrict__ lats,
                        GroupDesc* __restrict__ groups, LaunchCtl* __restrict__ ctl) {
  extern __shared__ __align__(16) uint8_t smem[];
  __shared__ SiteTab tab;
  const TileItem t = tiles[blockIdx.x];
  LatDesc* L = &lats[t.lat];
  const GroupDesc* G = &groups[L->group];
  const int lx = L->lx, ly = L->ly, lz = L->lz, pitch = L->pitch, q = L->q;
  const uint64_t sweep = L->sweep, key = L->key;
  if (sweep >= L->target) {
    launch_epilogue(lats, groups, ctl);
    return;
  }
  const int8_t* cur = (const int8_t*)L->buf[sweep & 1];
  int8_t* nxt = (int8_t*)L->buf[(sweep & 1) ^ 1];
  load_table(tab, L, G);
  PlaneGeom g;
  g.x0 = t.x0;
  g.W = L->tile_cx * 16;
  g.S = g.W + 32;
  g.Wv = min(g.W, lx - t.x0);
  g.ncv = (g.Wv + 15) >> 4;
  const int hv = min(L->tile_y, ly - t.y0);
  const int dv = min(L->tile_z, lz - t.z0);
  g.R = hv + 4;
  const int plane_bytes = g.R * g.S;
  const int pc = pitch >> 4;
  int dE = 0, nacc = 0, mag = 0;
  int cnt[kMaxPottsCounts] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int s = 0; s < dv + 4; ++s) {
    const int zl = t.z0 - 2 + s;
    uint8_t* pl = smem + (s & 3) * plane_bytes;
    load_plane(pl, cur, pitch, lx, ly, t.y0, wrapi(zl, lz), g);
    __syncthreads();
    load_plane_halo(pl, cur, pitch, lx, ly, t.y0, wrapi(zl, lz), g);
    __syncthreads();
    if (s >= 2) {
      const int zb = zl - 1;
      uint8_t* pb = smem + ((s - 1) & 3) * plane_bytes;
      const uint8_t* pm = smem + ((s - 2) & 3) * plane_bytes;
      const uint8_t* pp = pl;
      const bool owned_plane = zb >= t.z0 && zb < t.z0 + dv;
      black_pass<MODEL, 3>(pb, pm, pp, g, t.y0, wrapi(zb, lz), ly, lx, pc, hv, tab, q, key, sweep,
                           owned_plane, dE, nacc);
    }
    if (s >= 4) {
      const int zw = zl - 2;
      const uint8_t* pw = smem + ((s - 2) & 3) * plane_bytes;
      const uint8_t* pm = smem + ((s - 3) & 3) * plane_bytes;
      const uint8_t* pp = smem + ((s - 1) & 3) * plane_bytes;
      white_pass<MODEL, 3>(pw, pm, pp, g, t.y0, wrapi(zw, lz), ly, lx, pc, pitch, hv, tab, q, key,
                           sweep, nxt, dE, nacc, mag, cnt);
    }
    __syncthreads();  // the next load overwrites the slot read by this white pass
  }
  flush_accumulators<MODEL>(L, dE, nacc, mag, cnt, q);
  launch_epilogue(lats, groups, ctl);
}

template __global__ void k_sweep_discrete_2d<ISING>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template __global__ void k_sweep_discrete_2d<POTTS>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template __global__ void k_sweep_discrete_3d<ISING>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template __global__ void k_sweep_discrete_3d<POTTS>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);

}  // namespace gpumc
