// Cluster updates for int8 Ising and q-state Potts spins on periodic square
// and cubic lattices: Swendsen-Wang (SWCore, CMC.rs/src/algorithms/
// swendsen_wang.rs:73-138) and Wolff (WolffCore, CMC.rs/src/algorithms/
// wolff.rs:73-135), with the models' bond rules (ClusterModel for IsingModel /
// PottsModel, CMC.rs/src/lattice/models.rs:112-155, :294-338): a bond between
// equal neighbours is active with p = 1 - exp(-2 beta J) (Ising) or
// 1 - exp(-beta J) (Potts), J >= 0.
//
// One sweep is four launches over tiles of 16x16 (2D) or 8x8x4 (3D) sites,
// one thread per site:
//   1. k_cluster_local: each site draws its +x, +y (, +z) bonds and the bonds
//      inside the tile are merged by union-find in shared memory; every site
//      stores the global index of its tile-local root in the lattice's label
//      array;
//   2. k_cluster_global: the bonds that leave the tile (recomputed from the
//      same draws) are merged by lock-free union-find on the label array
//      (atomicCAS hooks of roots; path halving);
//   3. k_cluster_flip: each site finds its root (storing it: full path
//      compression) and writes the cluster's new value to the other
//      ping-pong buffer;
//   4. k_cluster_account: from the old and new buffers, the exact energy
//      change of each site's + bonds, the magnetisation (Ising) or state
//      histogram (Potts) and the changed-site count, then the launch epilogue.
// Every union hooks the larger root under the smaller (locally the local
// index order is the global site order), so the minimum site index of a
// component is never hooked: the final root of every cluster is its minimum
// site, independent of thread timing.  The cluster's decision is a function
// of that root, and the oracle (sequential union-find, minimum root)
// reproduces the device trajectory bit for bit.
//
// Random streams (restated by the oracle), counter word 1 = tag << 1 |
// plane << 8 | (index >> 32) << 16:
//   bonds   Philox(site, TAG_SW, plane 0): words 0-1 = +x uniform, 2-3 = +y;
//           plane 1 (3D): words 0-1 = +z; active iff u64 < T = floor(p 2^64);
//   SW      Philox(root, TAG_SWFLIP): Ising: +1 iff bit 31 of word 0; Potts:
//           state = word * q >> 32 over words 0..3 with exact rejection
//           (word * q mod 2^32 < 2^32 mod q), else 0;
//   Wolff   Philox(0, TAG_WOLFF, plane 0): seed = u64 * N >> 64 over words
//           0-1, then 2-3, with exact rejection, else 0; Potts target: the
//           other state word * (q-1) >> 32 over Philox(0, TAG_WOLFF, plane 1)
//           with rejection, skipping the seed's state; Ising target: -s_seed.
// The reference draws one f64 per edge and one decision per root in site
// order; the checkerboard-free cluster sweep here is distributionally the
// same update.  "Accepted" counts the sites whose spin changed.
//
// O(3) (ClusterModel for ONModel, CMC.rs/src/lattice/models.rs:516-579): the
// embedded Ising variables sigma = s . r along a random unit vector r drawn
// per sweep (Philox(0, TAG_O3CL): z = 1 - 2 u, phi from word 1, as the hot
// start draws a unit vector); a bond is active with p = 1 - exp(-2 beta J
// sigma_i sigma_j) when sigma_i sigma_j > 0 (fp32, the engine's own 1 - e^-x;
// active iff the 64-bit uniform is below p 2^64, exact for an fp32 p); a
// flipped cluster is reflected, s - 2 sigma r, renormalised by one Newton
// step.  Swendsen-Wang reflects a cluster iff bit 31 of word 0 of
// Philox(root, TAG_SWFLIP) is set; Wolff reflects the seed's cluster.  The
// spins are three fp32 planes in two ping-pong buffers; the energy change is
// the exact fp64 change of the fp32 configuration.
#include "device_common.cuh"
#include "epilogue.cuh"

namespace gpumc {

template <int DIM>
struct ClusterTile {
  static constexpr int TX = DIM == 2 ? 16 : 8, TY = DIM == 2 ? 16 : 8, TZ = DIM == 2 ? 1 : 4;
};

struct ClusterSite {
  int x, y, z;
  bool in;
  uint32_t site;  // compact index x + lx (y + ly z)
  size_t addr;    // byte offset in the int8 buffer
};

template <int DIM>
__device__ __forceinline__ ClusterSite cluster_site(const TileItem& t, const LatDesc* L) {
  using T = ClusterTile<DIM>;
  ClusterSite c;
  const int tx = threadIdx.x % T::TX, ty = (threadIdx.x / T::TX) % T::TY, tz = threadIdx.x / (T::TX * T::TY);
  c.x = t.x0 + tx;
  c.y = t.y0 + ty;
  c.z = t.z0 + tz;
  const int lz = DIM == 3 ? L->lz : 1;
  c.in = c.x < L->lx && c.y < L->ly && c.z < lz;
  c.site = (uint32_t)c.x + (uint32_t)L->lx * ((uint32_t)c.y + (uint32_t)L->ly * (uint32_t)c.z);
  c.addr = ((size_t)c.z * L->ly + c.y) * (size_t)L->pitch + c.x;
  return c;
}

// + neighbour d (0: x, 1: y, 2: z) of a site: compact index and byte offset
template <int DIM>
__device__ __forceinline__ void cluster_neighbour(const LatDesc* L, const ClusterSite& c, int d, uint32_t& site,
                                                  size_t& addr) {
  int x = c.x, y = c.y, z = c.z;
  if (d == 0) x = x + 1 < L->lx ? x + 1 : 0;
  if (d == 1) y = y + 1 < L->ly ? y + 1 : 0;
  if (d == 2) z = z + 1 < L->lz ? z + 1 : 0;
  site = (uint32_t)x + (uint32_t)L->lx * ((uint32_t)y + (uint32_t)L->ly * (uint32_t)z);
  addr = ((size_t)z * L->ly + y) * (size_t)L->pitch + x;
}

// Elements of one spin buffer of a lattice (bounds checks).
__device__ __forceinline__ long long cl_elems(const LatDesc* L) {
  return (long long)L->pitch * L->ly * (L->dims == 3 ? L->lz : 1);
}

// Active + bonds of a site (bit d), from the old configuration.
template <int DIM>
__device__ __forceinline__ uint32_t cluster_bonds(const LatDesc* L, const ClusterSite& c, const int8_t* cur,
                                                  unsigned long long thr, uint64_t sweep) {
  const long long ne = cl_elems(L);
  const int8_t s = ld_chk(cur, (long long)c.addr, ne);
  const uint4 o = draw(L->key, c.site, 0u, TAG_SW, 0u, sweep);
  uint32_t b = 0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    uint32_t ns;
    size_t na;
    cluster_neighbour<DIM>(L, c, d, ns, na);
    unsigned long long u;
    if (d == 0) u = (unsigned long long)o.x | ((unsigned long long)o.y << 32);
    else if (d == 1) u = (unsigned long long)o.z | ((unsigned long long)o.w << 32);
    else {
      const uint4 o2 = draw(L->key, c.site, 0u, TAG_SW, 1u, sweep);
      u = (unsigned long long)o2.x | ((unsigned long long)o2.y << 32);
    }
    if (ld_chk(cur, (long long)na, ne) == s && u < thr) b |= 1u << d;
  }
  return b;
}

__device__ __forceinline__ int local_find(const volatile int* par, int a) {
  int p = par[a];
  while (p != a) {
    a = p;
    p = par[a];
  }
  return a;
}

// Lock-free union in shared memory: the larger root is hooked under the
// smaller; a failed CAS means the root was hooked meanwhile, so retry.
__device__ __forceinline__ void local_union(int* par, int a, int b) {
  a = local_find(par, a);
  b = local_find(par, b);
  while (a != b) {
    if (a < b) {
      const int t = a;
      a = b;
      b = t;
    }
    const int old = atomicCAS(&par[a], a, b);
    if (old == a) return;
    a = local_find(par, old);
    b = local_find(par, b);
  }
}

// Root of a site in the global label array (labels only ever point to smaller
// indices); path halving stores only into non-root entries, which no CAS can
// target, so they are benign.
__device__ __forceinline__ uint32_t global_find(uint32_t* lab, uint32_t a) {
  uint32_t cur = __ldcg(lab + a);
  if (cur == a) return a;
  uint32_t prev = a;
  uint32_t next = __ldcg(lab + cur);
  while (cur > next) {
    __stcg(lab + prev, next);
    prev = cur;
    cur = next;
    next = __ldcg(lab + cur);
  }
  return cur;
}

__device__ __forceinline__ void global_union(uint32_t* lab, uint32_t a, uint32_t b) {
  a = global_find(lab, a);
  b = global_find(lab, b);
  while (a != b) {
    if (a < b) {
      const uint32_t t = a;
      a = b;
      b = t;
    }
    const uint32_t old = atomicCAS(lab + a, a, b);
    if (old == a) return;
    a = global_find(lab, old);
    b = global_find(lab, b);
  }
}

__device__ __forceinline__ unsigned long long cluster_threshold(const LatDesc* L, const GroupDesc* G) {
  const int label = __ldcg(&G->label[L->replica]);
  return G->tail[label * G->n_cls];
}

template <int DIM, int MODEL, int WOLFF>
__global__ void __launch_bounds__(kThreads)
    k_cluster_local(const TileItem* __restrict__ tiles, LatDesc* __restrict__ lats, GroupDesc* __restrict__ groups,
                    LaunchCtl* __restrict__ ctl) {
  using T = ClusterTile<DIM>;
  __shared__ int par[kThreads];
  const TileItem t = tiles[blockIdx.x];
  const LatDesc* L = &lats[t.lat];
  const uint64_t sweep = L->sweep;
  if (sweep >= L->target) return;
  const GroupDesc* G = &groups[L->group];
  const int8_t* cur = (const int8_t*)L->buf[sweep & 1];
  uint32_t* lab = (uint32_t*)L->aux;
  const ClusterSite c = cluster_site<DIM>(t, L);
  par[threadIdx.x] = threadIdx.x;
  const uint32_t b = c.in ? cluster_bonds<DIM>(L, c, cur, cluster_threshold(L, G), sweep) : 0u;
  __syncthreads();
  const int tx = threadIdx.x % T::TX, ty = (threadIdx.x / T::TX) % T::TY, tz = threadIdx.x / (T::TX * T::TY);
  // bonds to a + neighbour inside the tile (no wrap) merge locally
  if ((b & 1u) && tx + 1 < T::TX && c.x + 1 < L->lx) local_union(par, threadIdx.x, threadIdx.x + 1);
  if ((b & 2u) && ty + 1 < T::TY && c.y + 1 < L->ly) local_union(par, threadIdx.x, threadIdx.x + T::TX);
  if (DIM == 3 && (b & 4u) && tz + 1 < T::TZ && c.z + 1 < L->lz)
    local_union(par, threadIdx.x, threadIdx.x + T::TX * T::TY);
  __syncthreads();
  if (c.in) {
    const int r = local_find(par, threadIdx.x);
    const int rx = t.x0 + r % T::TX, ry = t.y0 + (r / T::TX) % T::TY, rz = t.z0 + r / (T::TX * T::TY);
    lab[c.site] = (uint32_t)rx + (uint32_t)L->lx * ((uint32_t)ry + (uint32_t)L->ly * (uint32_t)rz);
  }
}

template <int DIM, int MODEL, int WOLFF>
__global__ void __launch_bounds__(kThreads)
    k_cluster_global(const TileItem* __restrict__ tiles, LatDesc* __restrict__ lats, GroupDesc* __restrict__ groups,
                     LaunchCtl* __restrict__ ctl) {
  using T = ClusterTile<DIM>;
  const TileItem t = tiles[blockIdx.x];
  const LatDesc* L = &lats[t.lat];
  const uint64_t sweep = L->sweep;
  if (sweep >= L->target) return;
  const GroupDesc* G = &groups[L->group];
  const ClusterSite c = cluster_site<DIM>(t, L);
  if (!c.in) return;
  const int tx = threadIdx.x % T::TX, ty = (threadIdx.x / T::TX) % T::TY, tz = threadIdx.x / (T::TX * T::TY);
  const bool edge_x = tx + 1 == T::TX || c.x + 1 == L->lx;
  const bool edge_y = ty + 1 == T::TY || c.y + 1 == L->ly;
  const bool edge_z = DIM == 3 && (tz + 1 == T::TZ || c.z + 1 == L->lz);
  if (!(edge_x || edge_y || edge_z)) return;
  const int8_t* cur = (const int8_t*)L->buf[sweep & 1];
  uint32_t* lab = (uint32_t*)L->aux;
  const uint32_t b = cluster_bonds<DIM>(L, c, cur, cluster_threshold(L, G), sweep);
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    const bool edge = d == 0 ? edge_x : (d == 1 ? edge_y : edge_z);
    if (edge && (b >> d & 1u)) {
      uint32_t ns;
      size_t na;
      cluster_neighbour<DIM>(L, c, d, ns, na);
      global_union(lab, c.site, ns);
    }
  }
}

// Uniform integer in [0, n) from the four words of a Philox block by
// multiply-shift with exact rejection; 0 if every word is rejected.
__device__ __forceinline__ uint32_t uniform_below(const uint4 o, uint32_t n) {
  const uint32_t rej = (uint32_t)(0x100000000ull % n);
  const uint32_t w[4] = {o.x, o.y, o.z, o.w};
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const unsigned long long m = (unsigned long long)w[i] * n;
    if ((uint32_t)m >= rej) return (uint32_t)(m >> 32);
  }
  return 0u;
}

// Wolff seed site in [0, n) from a 64-bit multiply-shift with exact rejection.
__device__ __forceinline__ uint32_t wolff_seed(const uint4 o, uint64_t n) {
  const unsigned long long u[2] = {(unsigned long long)o.x | ((unsigned long long)o.y << 32),
                                   (unsigned long long)o.z | ((unsigned long long)o.w << 32)};
  const unsigned long long rej = (0ull - (unsigned long long)n) % (unsigned long long)n;  // 2^64 mod n
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    if (u[i] * (unsigned long long)n >= rej) return (uint32_t)__umul64hi(u[i], (unsigned long long)n);
  }
  return 0u;
}

template <int MODEL, int WOLFF>
struct ClusterRule {
  uint64_t key, sweep;
  int q;
  uint32_t seed_root;  // Wolff
  int8_t target;       // Wolff
  __device__ __forceinline__ int8_t apply(uint32_t root, int8_t s) const {
    if (WOLFF) return root == seed_root ? target : s;
    const uint4 o = draw(key, root, 0u, TAG_SWFLIP, 0u, sweep);
    if (MODEL == ISING) return (o.x >> 31) ? (int8_t)1 : (int8_t)-1;
    return (int8_t)uniform_below(o, (uint32_t)q);
  }
};

template <int MODEL>
__device__ __forceinline__ int bond_energy(int8_t a, int8_t b) {
  return MODEL == ISING ? -(int)a * (int)b : -(int)(a == b);
}

template <int DIM, int MODEL, int WOLFF>
__global__ void __launch_bounds__(kThreads)
    k_cluster_flip(const TileItem* __restrict__ tiles, LatDesc* __restrict__ lats, GroupDesc* __restrict__ groups,
                   LaunchCtl* __restrict__ ctl) {
  const TileItem t = tiles[blockIdx.x];
  const LatDesc* L = &lats[t.lat];
  const uint64_t sweep = L->sweep;
  if (sweep >= L->target) return;
  const int8_t* cur = (const int8_t*)L->buf[sweep & 1];
  int8_t* nxt = (int8_t*)L->buf[(sweep & 1) ^ 1];
  uint32_t* lab = (uint32_t*)L->aux;
  ClusterRule<MODEL, WOLFF> rule;
  rule.key = L->key;
  rule.sweep = sweep;
  rule.q = L->q;
  rule.seed_root = 0;
  rule.target = 0;
  if (WOLFF) {
    const uint32_t seed = wolff_seed(draw(L->key, 0ull, 0u, TAG_WOLFF, 0u, sweep), (uint64_t)L->n_sites);
    const int lx = L->lx, ly = L->ly;
    const int sx = (int)(seed % (uint32_t)lx), sy = (int)((seed / (uint32_t)lx) % (uint32_t)ly);
    const int sz = (int)(seed / ((uint32_t)lx * (uint32_t)ly));
    const int8_t ss = ld_chk(cur, (long long)(((size_t)sz * ly + sy) * (size_t)L->pitch + sx), cl_elems(L));
    if (MODEL == ISING) {
      rule.target = (int8_t)-ss;
    } else {
      const uint32_t r = uniform_below(draw(L->key, 0ull, 0u, TAG_WOLFF, 1u, sweep), (uint32_t)(L->q - 1));
      rule.target = (int8_t)((int)r < ss ? (int)r : (int)r + 1);
    }
    rule.seed_root = global_find(lab, seed);
  }
  const ClusterSite c = cluster_site<DIM>(t, L);
  if (!c.in) return;
  const uint32_t r = global_find(lab, c.site);
  if (GPUMC_IN(c.site, L->n_sites)) __stcg(lab + c.site, r);
  st_chk(nxt, (long long)c.addr, cl_elems(L), rule.apply(r, ld_chk(cur, (long long)c.addr, cl_elems(L))));
}

// Accounting of a lattice's sums: one block reduction, then one atomic per
// counter (called by every thread of the CTA).
template <int MODEL>
__device__ __forceinline__ void flush_cluster(LatDesc* L, long long dE, long long mag, long long nch,
                                              int* s_cnt, long long (*s_red)[3]) {
  const unsigned full = 0xFFFFFFFFu;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    dE += __shfl_xor_sync(full, dE, o);
    mag += __shfl_xor_sync(full, mag, o);
    nch += __shfl_xor_sync(full, nch, o);
  }
  if ((threadIdx.x & 31) == 0) {
    s_red[threadIdx.x >> 5][0] = dE;
    s_red[threadIdx.x >> 5][1] = mag;
    s_red[threadIdx.x >> 5][2] = nch;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    long long v = 0;
    for (int w = 0; w < kThreads / 32; ++w) v += s_red[w][threadIdx.x];
    if (v) {
      if (threadIdx.x == 0) atomic_add_i64(&L->acc.dE, v);
      if (threadIdx.x == 1 && MODEL == ISING) atomic_add_i64(&L->acc.mag, v);
      if (threadIdx.x == 2) atomic_add_i64(&L->acc.accepted, v);
    }
  }
  if (MODEL == POTTS && threadIdx.x < kMaxPottsCounts) {
    if (s_cnt[threadIdx.x]) atomic_add_i64(&L->acc.counts[threadIdx.x], s_cnt[threadIdx.x]);
    s_cnt[threadIdx.x] = 0;
  }
  __syncthreads();
}

// Energy change, magnetisation / state histogram and changed count of the
// sweep, from the old and new buffers.  A CTA strides over the launch's tiles
// (ctl->n_tiles) and flushes its sums when the lattice changes, so the
// per-lattice accumulators see a few atomics per CTA rather than per warp.
template <int DIM, int MODEL, int WOLFF>
__global__ void __launch_bounds__(kThreads)
    k_cluster_account(const TileItem* __restrict__ tiles, LatDesc* __restrict__ lats, GroupDesc* __restrict__ groups,
                      LaunchCtl* __restrict__ ctl) {
  __shared__ int s_cnt[kMaxPottsCounts];
  __shared__ long long s_red[kThreads / 32][3];
  if (threadIdx.x < kMaxPottsCounts) s_cnt[threadIdx.x] = 0;
  __syncthreads();
  const int n_tiles = ctl->n_tiles;
  int cur_lat = -1;
  long long dE = 0, mag = 0, nch = 0;
  for (int ti = blockIdx.x; ti < n_tiles; ti += gridDim.x) {
    const TileItem t = tiles[ti];
    if (t.lat != cur_lat) {
      if (cur_lat >= 0) flush_cluster<MODEL>(&lats[cur_lat], dE, mag, nch, s_cnt, s_red);
      dE = mag = nch = 0;
      cur_lat = t.lat;
    }
    const LatDesc* L = &lats[t.lat];
    const uint64_t sweep = L->sweep;
    if (sweep >= L->target) continue;
    const int8_t* cur = (const int8_t*)L->buf[sweep & 1];
    const int8_t* nxt = (const int8_t*)L->buf[(sweep & 1) ^ 1];
    const ClusterSite c = cluster_site<DIM>(t, L);
    if (c.in) {
      const long long ne = cl_elems(L);
      const int8_t s = ld_chk(cur, (long long)c.addr, ne), sn = ld_chk(nxt, (long long)c.addr, ne);
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        uint32_t ns;
        size_t na;
        cluster_neighbour<DIM>(L, c, d, ns, na);
        dE += bond_energy<MODEL>(sn, ld_chk(nxt, (long long)na, ne)) - bond_energy<MODEL>(s, ld_chk(cur, (long long)na, ne));
      }
      nch += sn != s;
      if (MODEL == ISING) mag += sn;
      else atomicAdd(&s_cnt[sn], 1);
    }
  }
  if (cur_lat >= 0) flush_cluster<MODEL>(&lats[cur_lat], dE, mag, nch, s_cnt, s_red);
  launch_epilogue(lats, groups, ctl);
}

// ---------------------------------------------------------------------------
// O(3)
// ---------------------------------------------------------------------------
struct O3Axis {
  float rx, ry, rz, c2bj;  // reflection axis, 2 beta J
};

__device__ __forceinline__ O3Axis o3_axis(const LatDesc* L, const GroupDesc* G, uint64_t sweep) {
  const uint4 o = draw(L->key, 0ull, 0u, TAG_O3CL, 0u, sweep);
  O3Axis a;
  const float t = fmul((float)(o.x >> 8), 0x1p-24f);
  a.rz = fsub(1.0f, fmul(2.0f, t));
  const float rho = fsqrt(fmul(fsub(1.0f, a.rz), fadd(1.0f, a.rz)));
  float c, sn;
  sincos_turn(o.y, c, sn);
  a.rx = fmul(rho, c);
  a.ry = fmul(rho, sn);
  const int label = __ldcg(&G->label[L->replica]);
  a.c2bj = fmul(fmul(2.0f, G->betas_f[label]), G->Jf);
  return a;
}

struct O3Spin {
  float x, y, z;
};

__device__ __forceinline__ O3Spin o3_get(const float* S, size_t cs, size_t i) {
  return O3Spin{ld_chk(S, (long long)i, (long long)cs), ld_chk(S + cs, (long long)i, (long long)cs),
                ld_chk(S + 2 * cs, (long long)i, (long long)cs)};
}

__device__ __forceinline__ float o3_sigma(const O3Spin& v, const O3Axis& a) {
  return fadd(fadd(fmul(v.x, a.rx), fmul(v.y, a.ry)), fmul(v.z, a.rz));
}

__device__ __forceinline__ O3Spin o3_reflect(const O3Spin& v, const O3Axis& a) {
  const float k = fmul(2.0f, o3_sigma(v, a));
  float px = fsub(v.x, fmul(k, a.rx)), py = fsub(v.y, fmul(k, a.ry)), pz = fsub(v.z, fmul(k, a.rz));
  const float n2 = fadd(fadd(fmul(px, px), fmul(py, py)), fmul(pz, pz));
  const float f = fsub(1.5f, fmul(0.5f, n2));
  return O3Spin{fmul(px, f), fmul(py, f), fmul(pz, f)};
}

struct O3Site {
  int x, y, z;
  bool in;
  uint32_t site;
  size_t idx;  // float index in a component plane
};

template <int DIM>
__device__ __forceinline__ O3Site o3_site(const TileItem& t, const LatDesc* L) {
  const ClusterSite c = cluster_site<DIM>(t, L);
  O3Site o;
  o.x = c.x;
  o.y = c.y;
  o.z = c.z;
  o.in = c.in;
  o.site = c.site;
  o.idx = ((size_t)c.z * L->ly + c.y) * (size_t)L->pitch + c.x;
  return o;
}

template <int DIM>
__device__ __forceinline__ size_t o3_neighbour(const LatDesc* L, const O3Site& c, int d, uint32_t& site) {
  int x = c.x, y = c.y, z = c.z;
  if (d == 0) x = x + 1 < L->lx ? x + 1 : 0;
  if (d == 1) y = y + 1 < L->ly ? y + 1 : 0;
  if (d == 2) z = z + 1 < L->lz ? z + 1 : 0;
  site = (uint32_t)x + (uint32_t)L->lx * ((uint32_t)y + (uint32_t)L->ly * (uint32_t)z);
  return ((size_t)z * L->ly + y) * (size_t)L->pitch + x;
}

template <int DIM>
__device__ __forceinline__ uint32_t o3_bonds(const LatDesc* L, const O3Site& c, const float* S, size_t cs,
                                             const O3Axis& a, uint64_t sweep) {
  const float si = o3_sigma(o3_get(S, cs, c.idx), a);
  const uint4 o = draw(L->key, c.site, 0u, TAG_SW, 0u, sweep);
  uint32_t b = 0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    uint32_t ns;
    const size_t ni = o3_neighbour<DIM>(L, c, d, ns);
    const float prod = fmul(si, o3_sigma(o3_get(S, cs, ni), a));
    if (!(prod > 0.0f)) continue;
    const float p = one_minus_exp_neg(fmul(a.c2bj, prod));
    const unsigned long long thr =
        p >= 1.0f ? ~0ull : (unsigned long long)__dmul_rn((double)p, 18446744073709551616.0);
    unsigned long long u;
    if (d == 0) u = (unsigned long long)o.x | ((unsigned long long)o.y << 32);
    else if (d == 1) u = (unsigned long long)o.z | ((unsigned long long)o.w << 32);
    else {
      const uint4 o2 = draw(L->key, c.site, 0u, TAG_SW, 1u, sweep);
      u = (unsigned long long)o2.x | ((unsigned long long)o2.y << 32);
    }
    if (u < thr) b |= 1u << d;
  }
  return b;
}

template <int DIM, int WOLFF>
__global__ void __launch_bounds__(kThreads)
    k_cluster_o3_local(const TileItem* __restrict__ tiles, LatDesc* __restrict__ lats, GroupDesc* __restrict__ groups,
                       LaunchCtl* __restrict__ ctl) {
  using T = ClusterTile<DIM>;
  __shared__ int par[kThreads];
  const TileItem t = tiles[blockIdx.x];
  const LatDesc* L = &lats[t.lat];
  const uint64_t sweep = L->sweep;
  if (sweep >= L->target) return;
  const GroupDesc* G = &groups[L->group];
  const float* S = (const float*)L->buf[sweep & 1];
  const size_t cs = (size_t)L->pitch * L->ly * L->lz;
  uint32_t* lab = (uint32_t*)L->aux;
  const O3Site c = o3_site<DIM>(t, L);
  par[threadIdx.x] = threadIdx.x;
  const O3Axis a = o3_axis(L, G, sweep);
  const uint32_t b = c.in ? o3_bonds<DIM>(L, c, S, cs, a, sweep) : 0u;
  __syncthreads();
  const int tx = threadIdx.x % T::TX, ty = (threadIdx.x / T::TX) % T::TY, tz = threadIdx.x / (T::TX * T::TY);
  if ((b & 1u) && tx + 1 < T::TX && c.x + 1 < L->lx) local_union(par, threadIdx.x, threadIdx.x + 1);
  if ((b & 2u) && ty + 1 < T::TY && c.y + 1 < L->ly) local_union(par, threadIdx.x, threadIdx.x + T::TX);
  if (DIM == 3 && (b & 4u) && tz + 1 < T::TZ && c.z + 1 < L->lz)
    local_union(par, threadIdx.x, threadIdx.x + T::TX * T::TY);
  __syncthreads();
  if (c.in) {
    const int r = local_find(par, threadIdx.x);
    const int rx = t.x0 + r % T::TX, ry = t.y0 + (r / T::TX) % T::TY, rz = t.z0 + r / (T::TX * T::TY);
    lab[c.site] = (uint32_t)rx + (uint32_t)L->lx * ((uint32_t)ry + (uint32_t)L->ly * (uint32_t)rz);
  }
}

template <int DIM, int WOLFF>
__global__ void __launch_bounds__(kThreads)
    k_cluster_o3_global(const TileItem* __restrict__ tiles, LatDesc* __restrict__ lats, GroupDesc* __restrict__ groups,
                        LaunchCtl* __restrict__ ctl) {
  using T = ClusterTile<DIM>;
  const TileItem t = tiles[blockIdx.x];
  const LatDesc* L = &lats[t.lat];
  const uint64_t sweep = L->sweep;
  if (sweep >= L->target) return;
  const GroupDesc* G = &groups[L->group];
  const O3Site c = o3_site<DIM>(t, L);
  if (!c.in) return;
  const int tx = threadIdx.x % T::TX, ty = (threadIdx.x / T::TX) % T::TY, tz = threadIdx.x / (T::TX * T::TY);
  const bool edge_x = tx + 1 == T::TX || c.x + 1 == L->lx;
  const bool edge_y = ty + 1 == T::TY || c.y + 1 == L->ly;
  const bool edge_z = DIM == 3 && (tz + 1 == T::TZ || c.z + 1 == L->lz);
  if (!(edge_x || edge_y || edge_z)) return;
  const float* S = (const float*)L->buf[sweep & 1];
  const size_t cs = (size_t)L->pitch * L->ly * L->lz;
  uint32_t* lab = (uint32_t*)L->aux;
  const uint32_t b = o3_bonds<DIM>(L, c, S, cs, o3_axis(L, G, sweep), sweep);
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    const bool edge = d == 0 ? edge_x : (d == 1 ? edge_y : edge_z);
    if (edge && (b >> d & 1u)) {
      uint32_t ns;
      o3_neighbour<DIM>(L, c, d, ns);
      global_union(lab, c.site, ns);
    }
  }
}

template <int DIM, int WOLFF>
__global__ void __launch_bounds__(kThreads)
    k_cluster_o3_flip(const TileItem* __restrict__ tiles, LatDesc* __restrict__ lats, GroupDesc* __restrict__ groups,
                      LaunchCtl* __restrict__ ctl) {
  const TileItem t = tiles[blockIdx.x];
  const LatDesc* L = &lats[t.lat];
  const uint64_t sweep = L->sweep;
  if (sweep >= L->target) return;
  const GroupDesc* G = &groups[L->group];
  const float* S = (const float*)L->buf[sweep & 1];
  float* N = (float*)L->buf[(sweep & 1) ^ 1];
  const size_t cs = (size_t)L->pitch * L->ly * L->lz;
  uint32_t* lab = (uint32_t*)L->aux;
  uint32_t seed_root = 0;
  if (WOLFF) seed_root = global_find(lab, wolff_seed(draw(L->key, 0ull, 0u, TAG_WOLFF, 0u, sweep), (uint64_t)L->n_sites));
  const O3Site c = o3_site<DIM>(t, L);
  if (!c.in) return;
  const uint32_t r = global_find(lab, c.site);
  __stcg(lab + c.site, r);
  const O3Spin v = o3_get(S, cs, c.idx);
  const bool refl = WOLFF ? r == seed_root : (draw(L->key, r, 0u, TAG_SWFLIP, 0u, sweep).x >> 31) != 0u;
  const O3Spin w = refl ? o3_reflect(v, o3_axis(L, G, sweep)) : v;
  N[c.idx] = w.x;
  N[cs + c.idx] = w.y;
  N[2 * cs + c.idx] = w.z;
}

template <int DIM, int WOLFF>
__global__ void __launch_bounds__(kThreads)
    k_cluster_o3_account(const TileItem* __restrict__ tiles, LatDesc* __restrict__ lats, GroupDesc* __restrict__ groups,
                         LaunchCtl* __restrict__ ctl) {
  __shared__ double s_red[kThreads / 32][4];
  __shared__ long long s_nch[kThreads / 32];
  const int n_tiles = ctl->n_tiles;
  int cur_lat = -1;
  double dE = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
  long long nch = 0;
  auto flush = [&](LatDesc* L) {
    const double mJ = -groups[L->group].J;
    const unsigned full = 0xFFFFFFFFu;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      dE += __shfl_xor_sync(full, dE, o);
      mx += __shfl_xor_sync(full, mx, o);
      my += __shfl_xor_sync(full, my, o);
      mz += __shfl_xor_sync(full, mz, o);
      nch += __shfl_xor_sync(full, nch, o);
    }
    if ((threadIdx.x & 31) == 0) {
      s_red[threadIdx.x >> 5][0] = dE;
      s_red[threadIdx.x >> 5][1] = mx;
      s_red[threadIdx.x >> 5][2] = my;
      s_red[threadIdx.x >> 5][3] = mz;
      s_nch[threadIdx.x >> 5] = nch;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
      double v = 0.0;
      for (int w = 0; w < kThreads / 32; ++w) v += s_red[w][threadIdx.x];
      double* dst = threadIdx.x == 0 ? &L->acc.dEf : threadIdx.x == 1 ? &L->acc.mx : threadIdx.x == 2 ? &L->acc.my : &L->acc.mz;
      atomicAdd(dst, threadIdx.x == 0 ? mJ * v : v);
    } else if (threadIdx.x == 4) {
      long long v = 0;
      for (int w = 0; w < kThreads / 32; ++w) v += s_nch[w];
      if (v) atomic_add_i64(&L->acc.accepted, v);
    }
    __syncthreads();
    dE = mx = my = mz = 0.0;
    nch = 0;
  };
  for (int ti = blockIdx.x; ti < n_tiles; ti += gridDim.x) {
    const TileItem t = tiles[ti];
    if (t.lat != cur_lat) {
      if (cur_lat >= 0) flush(&lats[cur_lat]);
      cur_lat = t.lat;
    }
    const LatDesc* L = &lats[t.lat];
    const uint64_t sweep = L->sweep;
    if (sweep >= L->target) continue;
    const float* S = (const float*)L->buf[sweep & 1];
    const float* N = (const float*)L->buf[(sweep & 1) ^ 1];
    const size_t cs = (size_t)L->pitch * L->ly * L->lz;
    const O3Site c = o3_site<DIM>(t, L);
    if (c.in) {
      const O3Spin v = o3_get(S, cs, c.idx), w = o3_get(N, cs, c.idx);
      double e = 0.0;
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        uint32_t ns;
        const size_t ni = o3_neighbour<DIM>(L, c, d, ns);
        const O3Spin vo = o3_get(S, cs, ni), wo = o3_get(N, cs, ni);
        e += ((double)w.x * wo.x + (double)w.y * wo.y + (double)w.z * wo.z) -
             ((double)v.x * vo.x + (double)v.y * vo.y + (double)v.z * vo.z);
      }
      dE += e;  // change of the + bond products; -J applied at the flush
      mx += (double)w.x;
      my += (double)w.y;
      mz += (double)w.z;
      nch += (w.x != v.x) | (w.y != v.y) | (w.z != v.z);
    }
  }
  if (cur_lat >= 0) flush(&lats[cur_lat]);
  launch_epilogue(lats, groups, ctl);
}

#define CLUSTER_O3_INSTANTIATE(DIM, WOLFF)                                                                       \
  template __global__ void k_cluster_o3_local<DIM, WOLFF>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);    \
  template __global__ void k_cluster_o3_global<DIM, WOLFF>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);   \
  template __global__ void k_cluster_o3_flip<DIM, WOLFF>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);     \
  template __global__ void k_cluster_o3_account<DIM, WOLFF>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
CLUSTER_O3_INSTANTIATE(2, 0)
CLUSTER_O3_INSTANTIATE(3, 0)
CLUSTER_O3_INSTANTIATE(2, 1)
CLUSTER_O3_INSTANTIATE(3, 1)

#define CLUSTER_INSTANTIATE(DIM, MODEL, WOLFF)                                                                 \
  template __global__ void k_cluster_local<DIM, MODEL, WOLFF>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*); \
  template __global__ void k_cluster_global<DIM, MODEL, WOLFF>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*); \
  template __global__ void k_cluster_flip<DIM, MODEL, WOLFF>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*); \
  template __global__ void k_cluster_account<DIM, MODEL, WOLFF>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
CLUSTER_INSTANTIATE(2, ISING, 0)
CLUSTER_INSTANTIATE(3, ISING, 0)
CLUSTER_INSTANTIATE(2, POTTS, 0)
CLUSTER_INSTANTIATE(3, POTTS, 0)
CLUSTER_INSTANTIATE(2, ISING, 1)
CLUSTER_INSTANTIATE(3, ISING, 1)
CLUSTER_INSTANTIATE(2, POTTS, 1)
CLUSTER_INSTANTIATE(3, POTTS, 1)

GPUMC_BOUNDS_MODULE(cluster)

}  // namespace gpumc
