// Multi-spin-coded Ising: 64 replicas of one lattice packed one bit per
// replica in a uint64 per site (bit r = replica r, 1 = spin up), as in the
// reference's MultiSpinIsing (CMC.rs/src/multi_spin.rs:28-151).
//
// Per site the anti-aligned neighbour count of every replica is formed with a
// bit-sliced adder tree over the XORs with the z neighbour words.  The 64
// Bernoulli decisions u_r < T[k_r] (T = 80-bit fixed-point threshold of
// exp(-beta dE), k_r = replica r's class) are made at once by a bit-serial
// comparator over random bit planes (plane j = bit j of every replica's
// uniform u_r, most significant first), stopping as soon as every replica's
// comparison is decided: ~log2(64)+2 planes on average instead of 64 draws.
// Each replica's decisions depend only on its own bit of each plane.
//
// The joint energy of all 64 replicas (the quantity the reference's PT weight
// uses, MultiSpinIsing::packed_total_energy, multi_spin.rs:180-197) is tracked
// exactly from the flip masks; per-replica energies and magnetisations come
// from the measurement kernel k_msc_measure.
#include "device_common.cuh"
#include "epilogue.cuh"

namespace gpumc {

constexpr int kMscMaxItems = 4;

// Acceptance table of a sweep in the comparator's form.  Classes with p < 1
// ("pending") are those with dE > 0: at most z/2 of them for the Ising table
// (k < z/2 anti-aligned neighbours for J > 0, k > z/2 for J < 0); every other
// class is accepted outright.  pneg[i][b] = ~0 where bit b of pending class
// i is 0; tw[j] bit i = bit j (most significant first) of the 80-bit
// threshold of pending class i.
struct MscTab {
  int npend;
  uint32_t pneg[3][3];
  unsigned char tw[80];
};

__device__ __forceinline__ void load_msc_table(MscTab& tab, const LatDesc* L, const GroupDesc* G) {
  if (threadIdx.x != 0) return;
  const int label = G->label[L->replica];
  const int n = min(G->n_cls, 7);
  const uint32_t* head = G->head + label * G->n_cls;
  const unsigned long long* tail = G->tail + label * G->n_cls;
  int pc[3] = {0, 0, 0}, np = 0;
  for (int k = 0; k < n; ++k)
    if (head[k] < 65536u && np < 3) pc[np++] = k;
  tab.npend = np;
  for (int i = 0; i < 3; ++i)
    for (int b = 0; b < 3; ++b) tab.pneg[i][b] = (i < np && ((pc[i] >> b) & 1)) ? 0u : 0xFFFFFFFFu;
  for (int j = 0; j < 80; ++j) {
    unsigned int v = 0;
    for (int i = 0; i < np; ++i) {
      const uint32_t h = head[pc[i]];
      const unsigned long long t = tail[pc[i]];
      const unsigned int bit = j < 16 ? (h >> (15 - j)) & 1u : (unsigned int)((t >> (79 - j)) & 1ull);
      v |= bit << i;
    }
    tab.tw[j] = (unsigned char)v;
  }
}

__device__ __forceinline__ unsigned long long rep64(uint32_t v) {
  return (unsigned long long)v | ((unsigned long long)v << 32);
}

template <int DIM>
__device__ __forceinline__ unsigned long long msc_site(unsigned long long w,
                                                       const unsigned long long* nb,
                                                       const MscTab& tab, const RunPhilox& P,
                                                       uint64_t site, uint32_t colour, long long& dE) {
  constexpr int zc = 2 * DIM;
  constexpr int kPend = DIM;  // z / 2
  unsigned long long x[6];
#pragma unroll
  for (int i = 0; i < zc; ++i) x[i] = w ^ nb[i];
  unsigned long long b0, b1, b2;
  if (DIM == 2) {
    const unsigned long long s0 = x[0] ^ x[1] ^ x[2];
    const unsigned long long c0 = (x[0] & x[1]) | (x[2] & (x[0] ^ x[1]));
    b0 = s0 ^ x[3];
    const unsigned long long c1 = s0 & x[3];
    b1 = c0 ^ c1;
    b2 = c0 & c1;
  } else {
    const unsigned long long s0 = x[0] ^ x[1] ^ x[2];
    const unsigned long long c0 = (x[0] & x[1]) | (x[2] & (x[0] ^ x[1]));
    const unsigned long long s1 = x[3] ^ x[4] ^ x[5];
    const unsigned long long c1 = (x[3] & x[4]) | (x[5] & (x[3] ^ x[4]));
    b0 = s0 ^ s1;
    const unsigned long long c2 = s0 & s1;
    b1 = c0 ^ c1 ^ c2;
    b2 = (c0 & c1) | (c2 & (c0 ^ c1));
  }
  // replicas of each pending class (class k = b2 b1 b0 in bits)
  unsigned long long m[kPend], pending = 0;
#pragma unroll
  for (int i = 0; i < kPend; ++i) {
    m[i] = 0;
    if (i < tab.npend) {
      m[i] = (b0 ^ rep64(tab.pneg[i][0])) & (b1 ^ rep64(tab.pneg[i][1])) & (b2 ^ rep64(tab.pneg[i][2]));
      pending |= m[i];
    }
  }
  // bit-serial comparison of the 64 uniforms, two planes per draw
  const uint32_t ctrl = (uint32_t)(site >> 32) << 16;
  unsigned long long lt = 0, eq = pending;
  for (int pair = 0; pair < 40 && eq; ++pair) {
    const uint4 o = run_philox(P, (uint32_t)site, ctrl | ((uint32_t)pair << 8));
    const unsigned long long u0 = (unsigned long long)o.x | ((unsigned long long)o.y << 32);
    const unsigned long long u1 = (unsigned long long)o.z | ((unsigned long long)o.w << 32);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const unsigned long long u = h ? u1 : u0;
      const unsigned int tb = tab.tw[2 * pair + h];
      unsigned long long tj = 0;
#pragma unroll
      for (int i = 0; i < kPend; ++i)
        if ((tb >> i) & 1u) tj |= m[i];
      lt |= eq & tj & ~u;
      eq &= ~(tj ^ u);
    }
  }
  const unsigned long long flip = ~pending | lt;
  // dE = sum over flipped replicas of 2 (z - 2 k)
  dE += 2LL * zc * __popcll(flip) -
        4LL * (__popcll(flip & b0) + 2LL * __popcll(flip & b1) + 4LL * __popcll(flip & b2));
  return w ^ flip;
}

// four CTAs per SM in 2D (64 registers, a few spilled words) measured 3 %
// faster than three at 80 registers
template <int DIM>
__global__ void __launch_bounds__(kThreads, DIM == 2 ? 4 : 3)
    k_sweep_msc(const TileItem* __restrict__ tiles, LatDesc* __restrict__ lats,
                GroupDesc* __restrict__ groups, LaunchCtl* __restrict__ ctl) {
  extern __shared__ __align__(16) unsigned long long wsm[];
  __shared__ MscTab tab;
  const TileItem t = tiles[blockIdx.x];
  LatDesc* L = &lats[t.lat];
  const GroupDesc* G = &groups[L->group];
  const uint64_t sweep = L->sweep;
  if (sweep >= L->target) {
    group_epilogue(t.pad, lats, groups, ctl);
    return;
  }
  const int lx = L->lx, ly = L->ly, lz = DIM == 3 ? L->lz : 1, pitch = L->pitch;
  const uint64_t key = L->key;
  const unsigned long long* cur = (const unsigned long long*)L->buf[sweep & 1];
  unsigned long long* nxt = (unsigned long long*)L->buf[(sweep & 1) ^ 1];
  load_msc_table(tab, L, G);
  const int Wv = min(t.cx * 2, lx - t.x0);
  const int hv = min(t.ty, ly - t.y0);
  const int S = Wv + 4, R = hv + 4;
  const int plane = R * S;
  const long long gwords = (long long)pitch * ly * lz;  // words of one buffer (bounds checks)
  long long dE = 0;
  // words k, k + kThreads, ... of the R x S staged rows, walked by a
  // division-free (row, column) cursor
  const int lc0 = threadIdx.x % S, lr0 = threadIdx.x / S;
  const int lstep_c = kThreads % S, lstep_r = kThreads / S;
  auto load = [&](unsigned long long* pl, int z) {
    int r = lr0, c = lc0;
    while (r < R) {
      const int y = wrap1(t.y0 - 2 + r, ly);
      const int x = wrap1(t.x0 - 2 + c, lx);
      st_chk(pl, r * S + c, plane, ld_chk(cur, (long long)(((size_t)z * ly + y) * (size_t)pitch + x), gwords));
      c += lstep_c;
      r += lstep_r;
      if (c >= S) {
        c -= S;
        ++r;
      }
    }
  };
  auto pass = [&](unsigned long long* pl, const unsigned long long* pm,
                  const unsigned long long* pp, int colour, int z, bool owned_plane) {
    const int rlo = colour == 0 ? 1 : 2;
    const int nrows = colour == 0 ? hv + 2 : hv;
    const int xlo = colour == 0 ? t.x0 - 1 : t.x0;
    const int half = colour == 0 ? (Wv + 2) / 2 : Wv / 2;
    const int nitems = nrows * half;
    unsigned long long res[kMscMaxItems];
    int roff[kMscMaxItems];
    const RunPhilox P = make_run_philox(key, sweep, (uint32_t)colour | (TAG_MSC << 1));
    // items threadIdx.x, + kThreads, ... as (row, column) cursors
    const int dr = kThreads / half, dk = kThreads - dr * half;
    int ir = threadIdx.x / half, ik = threadIdx.x - ir * half;
#pragma unroll
    for (int it = 0; it < kMscMaxItems; ++it) {
      roff[it] = -1;
      const int i = threadIdx.x + it * kThreads;
      const int r = rlo + ir, k = ik;
      ik += dk;
      ir += dr;
      if (ik >= half) {
        ik -= half;
        ++ir;
      }
      if (i < nitems) {
        const int y = wrap1(t.y0 - 2 + r, ly);
        const int pos = xlo + 2 * k + ((xlo + y + z + colour) & 1);
        const int off = r * S + (pos - t.x0 + 2);
        unsigned long long nb[6] = {ld_chk(pl, off - 1, plane), ld_chk(pl, off + 1, plane),
                                    ld_chk(pl, off - S, plane), ld_chk(pl, off + S, plane), 0, 0};
        if (DIM == 3) {
          nb[4] = ld_chk(pm, off, plane);
          nb[5] = ld_chk(pp, off, plane);
        }
        const int xr = wrap1(pos, lx);
        const uint64_t site = ((uint64_t)z * ly + y) * (uint64_t)lx + (uint64_t)xr;
        const bool owned = owned_plane && r >= 2 && r < 2 + hv && pos >= t.x0 && pos < t.x0 + Wv;
        long long de = 0;
        const unsigned long long nw = msc_site<DIM>(ld_chk(pl, off, plane), nb, tab, P, site, (uint32_t)colour, de);
        res[it] = nw;
        roff[it] = off;
        if (owned) {
          dE += de;
          st_chk(nxt, (long long)(((size_t)z * ly + y) * (size_t)pitch + xr), gwords, nw);
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < kMscMaxItems; ++it)
      if (roff[it] >= 0) st_chk(pl, roff[it], plane, res[it]);
    __syncthreads();
  };
  if (DIM == 2) {
    load(wsm, 0);
    __syncthreads();
    pass(wsm, wsm, wsm, 0, 0, true);
    pass(wsm, wsm, wsm, 1, 0, true);
  } else {
    const int dv = min(t.tz, lz - t.z0);
    for (int s = 0; s < dv + 4; ++s) {
      const int zl = t.z0 - 2 + s;
      unsigned long long* pl = wsm + (s & 3) * plane;
      load(pl, wrapi(zl, lz));
      __syncthreads();
      if (s >= 2) {
        const int zb = zl - 1;
        pass(wsm + ((s - 1) & 3) * plane, wsm + ((s - 2) & 3) * plane, pl, 0, wrapi(zb, lz),
             zb >= t.z0 && zb < t.z0 + dv);
      }
      if (s >= 4) {
        const int zw = zl - 2;
        pass(wsm + ((s - 2) & 3) * plane, wsm + ((s - 3) & 3) * plane,
             wsm + ((s - 1) & 3) * plane, 1, wrapi(zw, lz), true);
      }
      __syncthreads();
    }
  }
  long long v[1] = {dE};
  cta_sum(v);
  if (threadIdx.x == 0 && v[0]) atomic_add_i64(&L->acc.dE, v[0]);
  group_epilogue(t.pad, lats, groups, ctl);
}

// Per-replica magnetisation and energy of a multi-spin lattice: positional
// popcounts of the site words and of the +x/+y/+z bond XORs, via 16-plane
// bit-sliced (vertical) counters per thread flushed into shared counters.
// counters[r] = up spins of replica r, counters[64 + r] = anti-aligned bonds.
// The lattice's current buffer is read through its descriptor, so the launch
// can be captured in a graph independently of the ping-pong parity.
template <int DIM>
__global__ void __launch_bounds__(kThreads)
    k_msc_measure(const LatDesc* __restrict__ lats, int lat, unsigned long long* counters) {
  __shared__ unsigned long long s_up[64], s_anti[64];
  const LatDesc* L = &lats[lat];
  const int lx = L->lx, ly = L->ly, lz = DIM == 3 ? L->lz : 1, pitch = L->pitch;
  const unsigned long long* words = (const unsigned long long*)L->buf[L->sweep & 1];
  if (threadIdx.x < 64) {
    s_up[threadIdx.x] = 0;
    s_anti[threadIdx.x] = 0;
  }
  __syncthreads();
  const long long n = (long long)lx * ly * lz;
  unsigned long long cu[16], ca[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) cu[i] = ca[i] = 0;
  auto vadd = [](unsigned long long* c, unsigned long long v) {
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const unsigned long long t = c[i] & v;
      c[i] ^= v;
      v = t;
    }
  };
  auto flush = [&](unsigned long long* c, unsigned long long* dst) {
    for (int r = 0; r < 64; ++r) {
      unsigned long long v = 0;
#pragma unroll
      for (int i = 0; i < 16; ++i) v |= ((c[i] >> r) & 1ull) << i;
      if (v) atomicAdd(&dst[r], v);
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) c[i] = 0;
  };
  int filled = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n; s += stride) {
    const int x = (int)(s % lx);
    const long long rho = s / lx;
    const int y = (int)(rho % ly);
    const int z = (int)(rho / ly);
    const unsigned long long w = words[rho * pitch + x];
    vadd(cu, w);
    const int xp = x + 1 < lx ? x + 1 : 0;
    const int yp = y + 1 < ly ? y + 1 : 0;
    vadd(ca, w ^ words[rho * pitch + xp]);
    vadd(ca, w ^ words[((long long)z * ly + yp) * pitch + x]);
    if (DIM == 3) {
      const int zp = z + 1 < lz ? z + 1 : 0;
      vadd(ca, w ^ words[((long long)zp * ly + y) * pitch + x]);
    }
    if (++filled == 16000) {
      flush(cu, s_up);
      flush(ca, s_anti);
      filled = 0;
    }
  }
  flush(cu, s_up);
  flush(ca, s_anti);
  __syncthreads();
  if (threadIdx.x < 64) {
    atomicAdd(&counters[threadIdx.x], s_up[threadIdx.x]);
    atomicAdd(&counters[64 + threadIdx.x], s_anti[threadIdx.x]);
  }
}

// Converts the measurement counters of every word lattice of a multi-spin
// group into 64 records per word lattice (energy -J (bonds - 2 anti_r),
// magnetisation sum 2 up_r - N) and clears the counters.
__global__ void k_msc_record(LatDesc* lats, GroupDesc* groups, int group,
                             unsigned long long* counters) {
  GroupDesc* G = &groups[group];
  const int n_rep = G->n_rep;
  const uint64_t done = lats[G->first_lat].sweep;
  if (done == 0 || done - 1 < G->measure_from || done == G->msc_recorded) {
    // still thermalizing, or no new sweep since the last record: discard
    for (int i = threadIdx.x; i < 128 * n_rep; i += blockDim.x) counters[i] = 0;
    return;
  }
  const bool ok = G->rec_count < G->rec_cap;
  for (int i = threadIdx.x; i < 64 * n_rep; i += blockDim.x) {
    const int w = i >> 6, r = i & 63;
    const LatDesc* L = &lats[G->first_lat + w];
    const long long n = L->n_sites;
    const long long bonds = (long long)L->dims * n;
    unsigned long long* c = counters + (size_t)w * 128;
    const long long up = (long long)c[r];
    const long long anti = (long long)c[64 + r];
    if (ok) {
      Record R;
      R.energy = -G->J * (double)(bonds - 2 * anti);
      R.m[0] = (double)(2 * up - n);
      R.m[1] = R.m[2] = 0.0;
      R.accepted = 0.0;
      R.label = G->label[w];
      R.pad = 0;
      R.sweep = L->sweep - 1;
      G->records[(size_t)G->rec_count * 64 * n_rep + i] = R;
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 128 * n_rep; i += blockDim.x) counters[i] = 0;
  if (threadIdx.x == 0) {
    if (ok) G->rec_count += 1;
    else G->overflow = 1;
    G->msc_recorded = done;
  }
}

template __global__ void k_sweep_msc<2>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template __global__ void k_sweep_msc<3>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template __global__ void k_msc_measure<2>(const LatDesc*, int, unsigned long long*);
template __global__ void k_msc_measure<3>(const LatDesc*, int, unsigned long long*);

GPUMC_BOUNDS_MODULE(sweep_msc)

}  // namespace gpumc
