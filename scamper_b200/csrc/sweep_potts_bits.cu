// Bit-sliced fused checkerboard sweep for int8 q-state Potts spins, q <= 4,
// on periodic square (2D) and cubic (3D) lattices.
//
// Same skeleton as the Ising kernel (sweep_ising_bits.cu): the int8 lattice
// is read and written once per sweep, and each 64-site row segment is packed
// into two parity halves (even x / odd x), here with two bit planes each
// (state = 2 b1 + b0), so a colour pass updates 32 sites at once:
//   * proposal: new = v < s ? v : v + 1 with v uniform in [0, q-1) (the
//     reference's "uniform over the other q-1 states", CMC.rs/src/lattice/
//     models.rs:212-218); q = 2: v = 0; q = 3: v = one random bit; q = 4:
//     v = two random bits, v = 3 rejected and redrawn from the next pair of
//     planes (at most kPottsPropRounds rounds, then v = 0: probability
//     4^-32 per site);
//   * the equality masks of each neighbour with the old and the new state
//     feed one bit-sliced counter: cls = #(neighbours equal to the new state)
//     + #(neighbours different from the old state) = d + z, the acceptance
//     class of dE = -J d (d = n_new - n_old);
//   * acceptance u < T[cls] (80-bit thresholds of exp(-beta dE)) by the
//     bit-serial comparator over Philox bit planes, most significant first;
//     classes with p = 1 are accepted outright.
// A colour pass reads only the other colour and writes only its own, so both
// passes update the shared tile in place.
//
// Random stream (also restated by the oracle), segment g = rho * ceil(Lx/64)
// + x/64, colour c, bit i of a plane = colour site (x & 63) >> 1:
//   proposal round r: words 2(r & 1) (low bit) and 2(r & 1) + 1 (high bit)
//     of Philox4x32-10(key, (g, c | TAG_PBITS << 1 | (r >> 1) << 8, sweep));
//   acceptance plane j: word j & 3 of Philox(key, (g, c | TAG_PACC << 1 |
//     (j >> 2) << 8, sweep)).
//
// Reference semantics: Potts energy -J sum delta(s_i, s_j) and its change
// (CMC.rs/src/lattice/models.rs:191-380), acceptance min(1, exp(-beta dE))
// (Carlo.rs/src/acceptance.rs:11-22), energy cache += dE
// (CMC.rs/src/lattice/state.rs:127-136), order parameter from the state
// histogram (models.rs:276-291).
#include "bits_common.cuh"
#include "epilogue.cuh"

namespace gpumc {

constexpr int kPottsPropRounds = 32;
constexpr int kPottsMaxPend = 6;  // pending classes: at most z (dE > 0)

// Acceptance table of the pass: pending classes (p < 1) as 4-bit patterns
// and their 80-bit thresholds as 0/1 values, four planes per 16-byte word.
struct PottsTab {
  int npend;
  uint32_t pend_neg[kPottsMaxPend][4];  // ~0 where bit b of the class is 0
  uint4 tq[20][kPottsMaxPend];
};

__device__ __forceinline__ void load_potts_table(PottsTab& tab, const LatDesc* L, const GroupDesc* G) {
  const int label = __ldcg(&G->label[L->replica]);
  const int n = G->n_cls;
  const uint32_t* head = G->head + label * n;
  const unsigned long long* tail = G->tail + label * n;
  int pc[kPottsMaxPend] = {0, 0, 0, 0, 0, 0}, np = 0;
  for (int k = 0; k < n; ++k)
    if (head[k] < 65536u && np < kPottsMaxPend) pc[np++] = k;
  if (threadIdx.x == 0) {
    tab.npend = np;
    for (int i = 0; i < kPottsMaxPend; ++i)
      for (int b = 0; b < 4; ++b)
        tab.pend_neg[i][b] = (i < np && ((pc[i] >> b) & 1)) ? 0u : 0xFFFFFFFFu;
  }
  for (int e = threadIdx.x; e < 80 * kPottsMaxPend; e += kThreads) {
    const int j = e / kPottsMaxPend, i = e - kPottsMaxPend * j;
    uint32_t v = 0;
    if (i < np) {
      const uint32_t h = head[pc[i]];
      const unsigned long long t = tail[pc[i]];
      v = j < 16 ? (h >> (15 - j)) & 1u : (uint32_t)((t >> (79 - j)) & 1ull);
    }
    reinterpret_cast<uint32_t*>(&tab.tq[j >> 2][i])[j & 3] = v;
  }
}

// Bits 0 and 1 of 64 int8 states (x order) -> {E0, E1, O0, O1} (E even x,
// O odd x): the chosen bit of each byte is moved to the byte's top and four
// such bits are gathered into a nibble by one multiply.
__device__ __forceinline__ uint4 pack_potts(const uint4 v0, const uint4 v1, const uint4 v2, const uint4 v3) {
  const uint32_t w[16] = {v0.x, v0.y, v0.z, v0.w, v1.x, v1.y, v1.z, v1.w,
                          v2.x, v2.y, v2.z, v2.w, v3.x, v3.y, v3.z, v3.w};
  uint32_t E0 = 0, E1 = 0, O0 = 0, O1 = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint32_t ev = __byte_perm(w[2 * k], w[2 * k + 1], 0x6420);
    const uint32_t od = __byte_perm(w[2 * k], w[2 * k + 1], 0x7531);
    const uint32_t m = 0xFu << (4 * k);
    E0 |= ((((ev << 7) & 0x80808080u) * 0x00204081u) >> (28 - 4 * k)) & m;
    E1 |= ((((ev << 6) & 0x80808080u) * 0x00204081u) >> (28 - 4 * k)) & m;
    O0 |= ((((od << 7) & 0x80808080u) * 0x00204081u) >> (28 - 4 * k)) & m;
    O1 |= ((((od << 6) & 0x80808080u) * 0x00204081u) >> (28 - 4 * k)) & m;
  }
  return make_uint4(E0, E1, O0, O1);
}

// {E0, E1, O0, O1} -> 64 int8 states (2 b1 + b0).
__device__ __forceinline__ void unpack_potts(const uint4 p, uint4& v0, uint4& v1, uint4& v2, uint4& v3) {
  uint32_t w[16];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint32_t e0 = (p.x >> (4 * k)) & 0xFu, e1 = (p.y >> (4 * k)) & 0xFu;
    const uint32_t o0 = (p.z >> (4 * k)) & 0xFu, o1 = (p.w >> (4 * k)) & 0xFu;
    const uint32_t es = ((e0 * 0x00204081u) & 0x01010101u) + 2u * ((e1 * 0x00204081u) & 0x01010101u);
    const uint32_t os = ((o0 * 0x00204081u) & 0x01010101u) + 2u * ((o1 * 0x00204081u) & 0x01010101u);
    w[2 * k] = __byte_perm(es, os, 0x5140);
    w[2 * k + 1] = __byte_perm(es, os, 0x7362);
  }
  v0 = make_uint4(w[0], w[1], w[2], w[3]);
  v1 = make_uint4(w[4], w[5], w[6], w[7]);
  v2 = make_uint4(w[8], w[9], w[10], w[11]);
  v3 = make_uint4(w[12], w[13], w[14], w[15]);
}

// Stage the tile's rows of plane z into a shared plane of packed segments.
__device__ __forceinline__ void load_potts_plane(uint4* pl, const int8_t* src, int z, const BitsGeom& g) {
  if (g.row0 >= g.rstep) return;
  const int gs = wrap_i(g.s0 + g.col - g.xh, g.nseg);
  const size_t zrow = (size_t)z * g.ly;
  for (int it = 0; it < g.iters_load; ++it) {
    const int r = g.row0 + it * g.rstep;
    if (r >= g.R) break;
    const size_t off = (zrow + wrap_i(g.y0 - g.yo + r, g.ly)) * g.pitch + 64 * gs;
    const uint4* p = (const uint4*)(src + off);
    const bool in = GPUMC_IN(off + 63, g.gbytes);
    const uint4 z4 = make_uint4(0, 0, 0, 0);
    const uint4 a = in ? __ldg(p) : z4, b = in ? __ldg(p + 1) : z4, c = in ? __ldg(p + 2) : z4,
                d = in ? __ldg(p + 3) : z4;
    st_chk(pl, r * g.NC + g.col, g.pw, pack_potts(a, b, c, d));
  }
}

// Full and half adders on bit masks.
__device__ __forceinline__ void fa(uint32_t a, uint32_t b, uint32_t c, uint32_t& s, uint32_t& co) {
  s = a ^ b ^ c;
  co = (a & b) | (c & (a ^ b));
}
__device__ __forceinline__ void ha(uint32_t a, uint32_t b, uint32_t& s, uint32_t& co) {
  s = a ^ b;
  co = a & b;
}

// 4-bit count of 2z one-bit masks (z = 4: 8 inputs, z = 6: 12 inputs).
template <int DIM>
__device__ __forceinline__ void count_masks(const uint32_t* m, uint32_t& b0, uint32_t& b1, uint32_t& b2,
                                            uint32_t& b3) {
  if (DIM == 2) {
    uint32_t s1, c1, s2, c2, s3, c3, c4, s5, c5, c6;
    fa(m[0], m[1], m[2], s1, c1);
    fa(m[3], m[4], m[5], s2, c2);
    ha(m[6], m[7], s3, c3);
    fa(s1, s2, s3, b0, c4);    // weight 1
    fa(c1, c2, c3, s5, c5);    // weight 2
    ha(s5, c4, b1, c6);
    ha(c5, c6, b2, b3);        // weight 4
  } else {
    uint32_t s1, s2, s3, s4, c1, c2, c3, c4, t1, d1, d2, u1, u2, e1, e2, e3;
    fa(m[0], m[1], m[2], s1, c1);
    fa(m[3], m[4], m[5], s2, c2);
    fa(m[6], m[7], m[8], s3, c3);
    fa(m[9], m[10], m[11], s4, c4);
    fa(s1, s2, s3, t1, d1);
    ha(t1, s4, b0, d2);
    fa(c1, c2, c3, u1, e1);    // weight 2
    fa(c4, d1, d2, u2, e2);
    ha(u1, u2, b1, e3);
    fa(e1, e2, e3, b2, b3);    // weight 4 (and 8)
  }
}

struct PottsAcc {
  int nacc, clsum;
  int counts[4];
};

// One colour pass over rows [rlo, rlo + nrows) of plane `pl` (in place); for
// 3D, pm / pp are the planes below and above.
template <int DIM>
__device__ __forceinline__ void potts_pass(uint4* pl, const uint4* pm, const uint4* pp, const BitsGeom& g,
                                           int z, int colour, int rlo, int nrows, int iters,
                                           bool owned_plane, int out_mode, int8_t* dst, int q,
                                           const PottsTab& tab, const BitsPhilox& P, PottsAcc& acc) {
  constexpr int NB = 2 * DIM;
  constexpr int NP = DIM == 2 ? 4 : 6;  // pending classes on the square / cubic lattice
  const unsigned full = 0xFFFFFFFFu;
  const int cc = g.col;
  const bool col_ok = g.row0 < g.rstep && (colour == 0 || (cc >= g.xh && cc < g.xh + g.ns));
  const int gs = wrap_i(g.s0 + cc - g.xh, g.nseg);
  const bool last_seg = gs == g.nseg - 1;
  const bool first_seg = gs == 0;
  const uint32_t valid = (last_seg && g.hlast < 32) ? ((1u << g.hlast) - 1u) : 0xFFFFFFFFu;
  const bool owned_col = cc >= g.xh && cc < g.xh + g.ns;
  const int cprev = g.xh ? cc - 1 : (cc == 0 ? g.NC - 1 : cc - 1);
  const int cnext = g.xh ? cc + 1 : (cc == g.NC - 1 ? 0 : cc + 1);
  const bool has_prev = cprev >= 0, has_next = cnext < g.NC;
  const uint32_t ctrl_p = (uint32_t)colour | (TAG_PBITS << 1);
  const uint32_t ctrl_a = (uint32_t)colour | (TAG_PACC << 1);
  for (int it = 0; it < iters; ++it) {
    const int r = rlo + g.row0 + it * g.rstep;
    const bool active = col_ok && r < rlo + nrows;
    uint32_t own0 = 0, own1 = 0, segid = 0, b0 = 0, b1 = 0, b2 = 0, b3 = 0, pending = 0, always = 0;
    uint32_t m[NP];
#pragma unroll
    for (int i = 0; i < NP; ++i) m[i] = 0;
    uint32_t n0[NB], n1[NB];
    int P_ = 0;
    if (active) {
      const int y = wrap_i(g.y0 - g.yo + r, g.ly);
      P_ = (colour + y + z) & 1;  // x parity of this colour's sites in the row
      const uint4 me = ld_chk(pl, r * g.NC + cc, g.pw);
      const int ru = g.yw && r == 0 ? g.R - 1 : r - 1;
      const int rd = g.yw && r == g.R - 1 ? 0 : r + 1;
      const uint4 up = ld_chk(pl, ru * g.NC + cc, g.pw);
      const uint4 dn = ld_chk(pl, rd * g.NC + cc, g.pw);
      own0 = P_ ? me.z : me.x;
      own1 = P_ ? me.w : me.y;
      const uint32_t ot0 = P_ ? me.x : me.z, ot1 = P_ ? me.y : me.w;
      if (P_ == 0) {
        // even x = 2i: left = odd 2i-1 (index i-1), right = odd 2i+1 (index i)
        uint32_t c0 = 0, c1 = 0;
        if (has_prev) {
          const uint4 po = ld_chk(pl, r * g.NC + cprev, g.pw);
          const int sh = first_seg ? g.hlast - 1 : 31;
          c0 = (po.z >> sh) & 1u;
          c1 = (po.w >> sh) & 1u;
        }
        n0[0] = (ot0 << 1) | c0;
        n1[0] = (ot1 << 1) | c1;
        n0[1] = ot0;
        n1[1] = ot1;
      } else {
        // odd x = 2i+1: left = even 2i (index i), right = even 2i+2 (index i+1)
        n0[0] = ot0;
        n1[0] = ot1;
        uint32_t e0 = 0, e1 = 0;
        if (has_next) {
          const uint4 ne = ld_chk(pl, r * g.NC + cnext, g.pw);
          e0 = ne.x & 1u;
          e1 = ne.y & 1u;
        }
        const int hb = last_seg ? g.hlast - 1 : 31;
        n0[1] = ((ot0 >> 1) & ~(1u << hb)) | (e0 << hb);
        n1[1] = ((ot1 >> 1) & ~(1u << hb)) | (e1 << hb);
      }
      n0[2] = P_ ? up.z : up.x;
      n1[2] = P_ ? up.w : up.y;
      n0[3] = P_ ? dn.z : dn.x;
      n1[3] = P_ ? dn.w : dn.y;
      if (DIM == 3) {
        const uint4 zm = pm[r * g.NC + cc], zp = pp[r * g.NC + cc];
        n0[NB - 2] = P_ ? zm.z : zm.x;
        n1[NB - 2] = P_ ? zm.w : zm.y;
        n0[NB - 1] = P_ ? zp.z : zp.x;
        n1[NB - 1] = P_ ? zp.w : zp.y;
      }
      segid = (uint32_t)(y + g.ly * z) * (uint32_t)g.nseg + (uint32_t)gs;
    }
    // proposal planes v (uniform in [0, q-1))
    uint32_t v0 = 0, v1 = 0;
    if (q == 3) {
      v0 = bits_philox(P, segid, ctrl_p).x;
    } else if (q == 4) {
      uint32_t und = active ? valid : 0u;
      uint4 o = make_uint4(0, 0, 0, 0);
      int rr = 0;
      do {
        if ((rr & 1) == 0) o = bits_philox(P, segid, ctrl_p | ((uint32_t)(rr >> 1) << 8));
        const uint32_t w0 = (rr & 1) ? o.z : o.x, w1 = (rr & 1) ? o.w : o.y;
        const uint32_t take = und & ~(w0 & w1);
        v0 |= take & w0;
        v1 |= take & w1;
        und &= ~take;
        ++rr;
      } while (rr < kPottsPropRounds && __any_sync(full, und));
    }
    uint32_t new0 = 0, new1 = 0;
    if (active) {
      // new = v < s ? v : v + 1 on two bit planes (v <= q - 2 <= 2)
      const uint32_t lt = (~v1 & own1) | (~(v1 ^ own1) & ~v0 & own0);
      new0 = v0 ^ ~lt;
      new1 = v1 ^ (~lt & v0);
      uint32_t cm[2 * NB];
#pragma unroll
      for (int i = 0; i < NB; ++i) {
        cm[i] = ~((n1[i] ^ new1) | (n0[i] ^ new0));  // neighbour equals the new state
        cm[NB + i] = (n1[i] ^ own1) | (n0[i] ^ own0); // neighbour differs from the old state
      }
      count_masks<DIM>(cm, b0, b1, b2, b3);
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        if (i < tab.npend) {
          m[i] = (b0 ^ tab.pend_neg[i][0]) & (b1 ^ tab.pend_neg[i][1]) & (b2 ^ tab.pend_neg[i][2]) &
                 (b3 ^ tab.pend_neg[i][3]) & valid;
          pending |= m[i];
        }
      }
      always = valid & ~pending;
    }
    // bit-serial comparison of the 32 uniforms against their thresholds
    uint32_t lt = 0, eq = pending;
    int qq = 0;
    do {
      const uint4 o = bits_philox(P, segid, ctrl_a | ((uint32_t)qq << 8));
      uint4 tj = make_uint4(0, 0, 0, 0);
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        const uint4 t = tab.tq[qq][i];
        tj.x += m[i] * t.x;
        tj.y += m[i] * t.y;
        tj.z += m[i] * t.z;
        tj.w += m[i] * t.w;
      }
      lt |= eq & tj.x & ~o.x;
      eq &= ~(tj.x ^ o.x);
      lt |= eq & tj.y & ~o.y;
      eq &= ~(tj.y ^ o.y);
      lt |= eq & tj.z & ~o.z;
      eq &= ~(tj.z ^ o.z);
      lt |= eq & tj.w & ~o.w;
      eq &= ~(tj.w ^ o.w);
      ++qq;
    } while (qq < 20 && __any_sync(full, eq));
    if (active) {
      const uint32_t acc_m = (always | lt) & valid;
      const uint32_t f0 = (own0 & ~acc_m) | (new0 & acc_m);
      const uint32_t f1 = (own1 & ~acc_m) | (new1 & acc_m);
      const bool in_me = GPUMC_IN(r * g.NC + cc, g.pw);
      uint4& me = pl[in_me ? r * g.NC + cc : 0];
      if (in_me) {
        if (P_) {
          me.z = f0;
          me.w = f1;
        } else {
          me.x = f0;
          me.y = f1;
        }
      }
      const bool owned = owned_plane && owned_col && r >= g.yo && r < g.yo + g.hv;
      if (owned) {
        acc.nacc += __popc(acc_m);
        acc.clsum += __popc(acc_m & b0) + 2 * __popc(acc_m & b1) + 4 * __popc(acc_m & b2) + 8 * __popc(acc_m & b3);
      }
      if (out_mode != 0) {
        // both colours of this segment are final: state histogram and
        // (mode 1) the int8 row segment
        const uint4 fin = P_ ? make_uint4(me.x, me.y, f0, f1) : make_uint4(f0, f1, me.z, me.w);
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          const uint32_t mE = ((v & 1) ? fin.x : ~fin.x) & ((v & 2) ? fin.y : ~fin.y);
          const uint32_t mO = ((v & 1) ? fin.z : ~fin.z) & ((v & 2) ? fin.w : ~fin.w);
          acc.counts[v] += __popc(mE & valid) + __popc(mO & valid);
        }
        if (out_mode == 1) {
          const int y = wrap_i(g.y0 - g.yo + r, g.ly);
          uint4 o0, o1, o2, o3;
          unpack_potts(fin, o0, o1, o2, o3);
          const size_t off = ((size_t)z * g.ly + y) * g.pitch + 64 * gs;
          uint4* out = (uint4*)(dst + off);
          if (GPUMC_IN(off + 63, g.gbytes)) {
            out[0] = o0;
            out[1] = o1;
            out[2] = o2;
            out[3] = o3;
          }
        }
      }
    }
  }
}

__device__ __forceinline__ void flush_potts(Accum* A, const PottsAcc& a, int zc) {
  // dE = -(sum of d), d = cls - z
  long long v[6] = {-((long long)a.clsum - (long long)zc * a.nacc), a.nacc, a.counts[0], a.counts[1],
                    a.counts[2], a.counts[3]};
  cta_sum(v);
  if (threadIdx.x == 0) {
    if (v[0]) atomic_add_i64(&A->dE, v[0]);
    if (v[1]) atomic_add_i64(&A->accepted, v[1]);
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (v[2 + k]) atomic_add_i64(&A->counts[k], v[2 + k]);
  }
}

// 2D: four CTAs per SM (64 registers, 12 spilled bytes) measured 1.8 %
// faster on the uneven mix than three at 80 registers
template <int DIM>
__global__ void __launch_bounds__(kThreads, DIM == 2 ? 4 : 2)
    k_sweep_potts_bits(const TileItem* __restrict__ tiles, LatDesc* __restrict__ lats,
                       GroupDesc* __restrict__ groups, LaunchCtl* __restrict__ ctl) {
  extern __shared__ __align__(16) uint4 psm[];
  __shared__ PottsTab tab;
  const TileItem t = tiles[blockIdx.x];
  LatDesc* L = &lats[t.lat];
  const GroupDesc* G = &groups[L->group];
  const uint64_t sweep = L->sweep;
  if (sweep >= L->target) {
    group_epilogue(t.pad, lats, groups, ctl);
    return;
  }
  const int8_t* cur = (const int8_t*)L->buf[sweep & 1];
  int8_t* nxt = (int8_t*)L->buf[(sweep & 1) ^ 1];
  const BitsGeom g = make_bits_geom(t, L);
  const int q = L->q;
  load_potts_table(tab, L, G);
  const BitsPhilox P = make_bits_philox(L->key, sweep);
  PottsAcc acc = {0, 0, {0, 0, 0, 0}};
  if (DIM == 2) {
    load_potts_plane(psm, cur, 0, g);
    __syncthreads();
    potts_pass<2>(psm, psm, psm, g, 0, 0, 1, g.R - 2, g.iters_black, true, 0, nxt, q, tab, P, acc);
    __syncthreads();
    potts_pass<2>(psm, psm, psm, g, 0, 1, 2, g.hv, g.iters_white, true, 1, nxt, q, tab, P, acc);
  } else {
    const int lz = L->lz;
    const int dv = min(t.tz, lz - t.z0);
    const int pw = g.R * g.NC;
    for (int s = 0; s < dv + 4; ++s) {
      const int zl = t.z0 - 2 + s;
      uint4* Pl = psm + (s & 3) * pw;
      load_potts_plane(Pl, cur, wrap_i(zl, lz), g);
      __syncthreads();
      if (s >= 2) {
        const int zb = zl - 1;
        potts_pass<3>(psm + ((s - 1) & 3) * pw, psm + ((s - 2) & 3) * pw, Pl, g, wrap_i(zb, lz), 0,
                      g.yo / 2, g.yw ? g.R : g.R - 2, g.iters_black, zb >= t.z0 && zb < t.z0 + dv, 0, nxt,
                      q, tab, P, acc);
        __syncthreads();
      }
      if (s >= 4) {
        const int zw = zl - 2;
        potts_pass<3>(psm + ((s - 2) & 3) * pw, psm + ((s - 3) & 3) * pw, psm + ((s - 1) & 3) * pw, g,
                      wrap_i(zw, lz), 1, g.yo, g.hv, g.iters_white, true, 1, nxt, q, tab, P, acc);
      }
      __syncthreads();  // the next load overwrites the plane slot read above
    }
  }
  flush_potts(&L->acc, acc, 2 * DIM);
  group_epilogue(t.pad, lats, groups, ctl);
}

template __global__ void k_sweep_potts_bits<2>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template __global__ void k_sweep_potts_bits<3>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);

GPUMC_BOUNDS_MODULE(sweep_potts_bits)

}  // namespace gpumc
