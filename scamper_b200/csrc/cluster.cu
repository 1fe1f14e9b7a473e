// Cluster updates for int8 Ising and q-state Potts spins on periodic square
// and cubic lattices: Swendsen-Wang (SWCore, CMC.rs/src/algorithms/
// swendsen_wang.rs:73-138) and Wolff (WolffCore, CMC.rs/src/algorithms/
// wolff.rs:73-135), with the models' bond rules (ClusterModel for IsingModel /
// PottsModel, CMC.rs/src/lattice/models.rs:112-155, :294-338): a bond between
// equal neighbours is active with p = 1 - exp(-2 beta J) (Ising) or
// 1 - exp(-beta J) (Potts), J >= 0.
//
// One sweep is three launches over tiles of 16x16 (2D) or 8x8x4 (3D) sites,
// one thread per site:
//   1. k_cluster_local: each site draws its +x, +y (, +z) bonds and the bonds
//      inside the tile are merged by union-find in shared memory; every site
//      stores the global index of its tile-local root in the lattice's label
//      array;
//   2. k_cluster_global: the bonds that leave the tile (recomputed from the
//      same draws) are merged by lock-free union-find on the label array
//      (atomicCAS hooks of roots; path halving);
//   3. k_cluster_flip: each site finds its root and takes the cluster's new
//      value, writes it to the other ping-pong buffer and accumulates the
//      exact energy change of its + bonds (the neighbour's new value is
//      derived from the neighbour's root, so no site reads a value being
//      written), then the launch epilogue runs.
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

// Active + bonds of a site (bit d), from the old configuration.
template <int DIM>
__device__ __forceinline__ uint32_t cluster_bonds(const LatDesc* L, const ClusterSite& c, const int8_t* cur,
                                                  unsigned long long thr, uint64_t sweep) {
  const int8_t s = cur[c.addr];
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
    if (cur[na] == s && u < thr) b |= 1u << d;
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
  __shared__ int s_cnt[kMaxPottsCounts];
  const TileItem t = tiles[blockIdx.x];
  LatDesc* L = &lats[t.lat];
  const uint64_t sweep = L->sweep;
  if (sweep >= L->target) {
    launch_epilogue(lats, groups, ctl);
    return;
  }
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
    const int8_t ss = cur[((size_t)sz * ly + sy) * (size_t)L->pitch + sx];
    if (MODEL == ISING) {
      rule.target = (int8_t)-ss;
    } else {
      const uint32_t r = uniform_below(draw(L->key, 0ull, 0u, TAG_WOLFF, 1u, sweep), (uint32_t)(L->q - 1));
      rule.target = (int8_t)((int)r < ss ? (int)r : (int)r + 1);
    }
    rule.seed_root = global_find(lab, seed);
  }
  if (threadIdx.x < kMaxPottsCounts) s_cnt[threadIdx.x] = 0;
  __syncthreads();
  const ClusterSite c = cluster_site<DIM>(t, L);
  long long dE = 0, mag = 0, nch = 0;
  if (c.in) {
    const int8_t s = cur[c.addr];
    const int8_t sn = rule.apply(global_find(lab, c.site), s);
    nxt[c.addr] = sn;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      uint32_t ns;
      size_t na;
      cluster_neighbour<DIM>(L, c, d, ns, na);
      const int8_t o = cur[na];
      const int8_t on = rule.apply(global_find(lab, ns), o);
      dE += bond_energy<MODEL>(sn, on) - bond_energy<MODEL>(s, o);
    }
    nch = sn != s;
    if (MODEL == ISING) mag = sn;
    else atomicAdd(&s_cnt[sn], 1);
  }
  const unsigned full = 0xFFFFFFFFu;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    dE += __shfl_xor_sync(full, dE, o);
    mag += __shfl_xor_sync(full, mag, o);
    nch += __shfl_xor_sync(full, nch, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (dE) atomic_add_i64(&L->acc.dE, dE);
    if (nch) atomic_add_i64(&L->acc.accepted, nch);
    if (MODEL == ISING && mag) atomic_add_i64(&L->acc.mag, mag);
  }
  __syncthreads();
  if (MODEL == POTTS && threadIdx.x < kMaxPottsCounts && s_cnt[threadIdx.x])
    atomic_add_i64(&L->acc.counts[threadIdx.x], s_cnt[threadIdx.x]);
  launch_epilogue(lats, groups, ctl);
}

#define CLUSTER_INSTANTIATE(DIM, MODEL, WOLFF)                                                                 \
  template __global__ void k_cluster_local<DIM, MODEL, WOLFF>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*); \
  template __global__ void k_cluster_global<DIM, MODEL, WOLFF>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*); \
  template __global__ void k_cluster_flip<DIM, MODEL, WOLFF>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
CLUSTER_INSTANTIATE(2, ISING, 0)
CLUSTER_INSTANTIATE(3, ISING, 0)
CLUSTER_INSTANTIATE(2, POTTS, 0)
CLUSTER_INSTANTIATE(3, POTTS, 0)
CLUSTER_INSTANTIATE(2, ISING, 1)
CLUSTER_INSTANTIATE(3, ISING, 1)
CLUSTER_INSTANTIATE(2, POTTS, 1)
CLUSTER_INSTANTIATE(3, POTTS, 1)

}  // namespace gpumc
