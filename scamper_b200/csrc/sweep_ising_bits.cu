// Bit-sliced fused checkerboard sweep for int8 Ising spins on periodic square
// (2D) and cubic (3D) lattices.
//
// The int8 lattice is read and written once per sweep (2 B of HBM traffic per
// attempt), but the update runs on bits: each 64-site row segment is packed
// into two 32-bit masks, E (even x) and O (odd x), bit = 1 for spin -1.  In a
// row the two colours of the checkerboard are exactly the two x parities, so
// a colour pass updates one 32-bit mask per segment:
//   * neighbour spins are shifts of the other-parity mask of the same row and
//     the same-parity masks of the rows above/below (and planes in 3D), so the
//     anti-aligned count of all 32 sites comes from a bit-sliced adder;
//   * the 32 Metropolis decisions u_i < T[k_i] (T = 80-bit fixed point of
//     exp(-beta dE), from the host table) are made together by a bit-serial
//     comparator over Philox bit planes, most significant plane first; the
//     warp stops drawing planes once every lane's sites are decided.
// A colour pass reads only the other colour's masks and writes only its own,
// so both passes update the shared tile in place without races.
//
// Random stream (also restated by the oracle): plane j of segment g = rho *
// ceil(Lx/64) + x/64 (rho = y + Ly z), colour c, is word j & 3 of
// Philox4x32-10(key, ctr = (g, c | TAG_BITS << 1 | (j >> 2) << 8, sweep));
// bit i of a plane belongs to the colour site (x & 63) >> 1 = i.
//
// Reference semantics: Ising dE = 2J(z - 2k) (CMC.rs/src/lattice/
// interaction.rs:73-84), acceptance min(1, exp(-beta dE))
// (Carlo.rs/src/acceptance.rs:11-22), energy cache += dE
// (CMC.rs/src/lattice/state.rs:127-136), |M| observable
// (CMC.rs/src/lattice/models.rs:103-110).
//
// Heat bath (ALG = 1; HeatBathCore, CMC.rs/src/algorithms/heat_bath.rs:41-66,
// with IsingModel::heat_bath_sample_site, CMC.rs/src/lattice/models.rs:158-186):
// the new spin is +1 with probability p(x) = 1 / (1 + exp(-x)), x = 2 beta J h,
// h = sum of the neighbour spins = z - 2k with k the number of DOWN neighbours
// (the adder counts neighbour bits, not anti-aligned ones).  The host table
// holds T[k] = p(|x_k|) as 80-bit fixed point; classes k and z - k have the
// same |x| and share one comparator slot.  For the member whose field is
// positive the site goes up iff u < T; for the negative one it goes down iff
// ~u < T (the complemented uniform, same distribution), so one threshold and
// one bit-serial comparison serve both.  The zero-field class k = z/2 goes up
// iff the first bit of u is 0 (u < 1/2).  The planes come from tag
// TAG_HBITS.  "Accepted" counts the sites whose spin changed.
#include "bits_common.cuh"
#include "epilogue.cuh"

namespace gpumc {

// Acceptance table of the pass in the form the comparator uses.  For Ising
// the classes with p < 1 are those with dE > 0: at most z/2 of them (two on
// the square lattice, three on the cubic), so the comparator handles up to
// three "pending" classes; every other class is accepted outright.  The
// 80-bit thresholds are stored as one 0/1 value per (plane, class), grouped
// four planes to a 16-byte word so that one shared load serves a Philox
// draw; the comparator selects a plane's threshold bits with integer
// multiply-adds of the disjoint class masks.
struct BitsTab {
  int npend;                  // pending classes (0..3)
  uint32_t pend_neg[3][3];    // pend_neg[i][b] = ~0 if bit b of class pc[i] is 0 (heat
                              // bath: of the positive-field member of pair i)
  uint32_t pair_neg[3][3];    // heat bath: the same for the negative-field member
  uint32_t half_neg[3];       // heat bath: the same for the zero-field class z/2
  uint4 tq[20][3];            // tq[q][i].{x,y,z,w} = bit 4q+{0,1,2,3} (MSB first) of T[pc[i]]
};

// 64 int8 spins (x order) -> parity masks (bit set for spin -1).
__device__ __forceinline__ uint2 pack_segment(const uint4 v0, const uint4 v1, const uint4 v2,
                                              const uint4 v3) {
  const uint32_t w[16] = {v0.x, v0.y, v0.z, v0.w, v1.x, v1.y, v1.z, v1.w,
                          v2.x, v2.y, v2.z, v2.w, v3.x, v3.y, v3.z, v3.w};
  uint32_t E = 0, O = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint32_t ev = __byte_perm(w[2 * k], w[2 * k + 1], 0x6420);
    const uint32_t od = __byte_perm(w[2 * k], w[2 * k + 1], 0x7531);
    // sign bits of the four bytes gathered into bits 28..31 by one multiply
    E |= (((ev & 0x80808080u) * 0x00204081u) >> (28 - 4 * k)) & (0xFu << (4 * k));
    O |= (((od & 0x80808080u) * 0x00204081u) >> (28 - 4 * k)) & (0xFu << (4 * k));
  }
  return make_uint2(E, O);
}

// Parity masks -> 64 int8 spins (+1 = 0x01, -1 = 0xFF).
__device__ __forceinline__ void unpack_segment(uint32_t E, uint32_t O, uint4& v0, uint4& v1,
                                               uint4& v2, uint4& v3) {
  uint32_t w[16];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint32_t e4 = (E >> (4 * k)) & 0xFu, o4 = (O >> (4 * k)) & 0xFu;
    const uint32_t es = 0x01010101u ^ (((e4 * 0x00204081u) & 0x01010101u) * 0xFEu);
    const uint32_t os = 0x01010101u ^ (((o4 * 0x00204081u) & 0x01010101u) * 0xFEu);
    w[2 * k] = __byte_perm(es, os, 0x5140);
    w[2 * k + 1] = __byte_perm(es, os, 0x7362);
  }
  v0 = make_uint4(w[0], w[1], w[2], w[3]);
  v1 = make_uint4(w[4], w[5], w[6], w[7]);
  v2 = make_uint4(w[8], w[9], w[10], w[11]);
  v3 = make_uint4(w[12], w[13], w[14], w[15]);
}

// Stage rows y0-2 .. y0+hv+1 of plane z into a shared mask plane.
__device__ __forceinline__ void load_bits_plane(uint2* pl, const int8_t* src, int z,
                                                const BitsGeom& g) {
  if (g.row0 >= g.rstep) return;
  const int gs = wrap_i(g.s0 + g.col - g.xh, g.nseg);
  const size_t zrow = (size_t)z * g.ly;
  for (int it = 0; it < g.iters_load; it += 2) {
    const int r0 = g.row0 + it * g.rstep, r1 = r0 + g.rstep;
    uint4 a[4], b[4];
    const bool ok0 = r0 < g.R, ok1 = r1 < g.R && it + 1 < g.iters_load;
    if (ok0) {
      const size_t off = (zrow + wrap_i(g.y0 - g.yo + r0, g.ly)) * g.pitch + 64 * gs;
      const uint4* p = (const uint4*)(src + off);
#pragma unroll
      for (int k = 0; k < 4; ++k) a[k] = GPUMC_IN(off + 63, g.gbytes) ? __ldg(p + k) : make_uint4(0, 0, 0, 0);
    }
    if (ok1) {
      const size_t off = (zrow + wrap_i(g.y0 - g.yo + r1, g.ly)) * g.pitch + 64 * gs;
      const uint4* p = (const uint4*)(src + off);
#pragma unroll
      for (int k = 0; k < 4; ++k) b[k] = GPUMC_IN(off + 63, g.gbytes) ? __ldg(p + k) : make_uint4(0, 0, 0, 0);
    }
    if (ok0) st_chk(pl, r0 * g.NC + g.col, g.pw, pack_segment(a[0], a[1], a[2], a[3]));
    if (ok1) st_chk(pl, r1 * g.NC + g.col, g.pw, pack_segment(b[0], b[1], b[2], b[3]));
  }
}

struct PassAcc {
  int nacc, ksum, down, owned_sites;
};

// One colour pass over rows [rlo, rlo + nrows) and columns [c_lo, c_hi) of
// plane `pl` (in place).  For 3D, pm/pp are the neighbouring planes.
template <int DIM, int ALG>
__device__ __forceinline__ void bits_pass(uint2* pl, const uint2* pm, const uint2* pp,
                                          const BitsGeom& g, int z, int colour, int rlo,
                                          int nrows, int iters, bool owned_plane, int out_mode,
                                          int8_t* dst, const BitsTab& tab, const BitsPhilox& P,
                                          PassAcc& acc) {
  const unsigned full = 0xFFFFFFFFu;
  const int cc = g.col;
  // columns this pass covers: colour 0 also updates the halo columns
  const bool col_ok = g.row0 < g.rstep && (colour == 0 || (cc >= g.xh && cc < g.xh + g.ns));
  const int gs = wrap_i(g.s0 + cc - g.xh, g.nseg);
  const bool last_seg = gs == g.nseg - 1;
  const bool first_seg = gs == 0;
  const uint32_t valid = (last_seg && g.hlast < 32) ? ((1u << g.hlast) - 1u) : 0xFFFFFFFFu;
  const bool owned_col = cc >= g.xh && cc < g.xh + g.ns;
  // neighbour columns inside the plane (full-row tiles wrap around the row)
  const int cprev = g.xh ? cc - 1 : (cc == 0 ? g.NC - 1 : cc - 1);
  const int cnext = g.xh ? cc + 1 : (cc == g.NC - 1 ? 0 : cc + 1);
  const bool has_prev = cprev >= 0, has_next = cnext < g.NC;
  // the class patterns of the pass in registers: the loop stores to the
  // shared plane, so reads of the shared table would be repeated per word
  constexpr int kPend = DIM == 2 ? 2 : 3;  // pending slots: z/2
  const int npend = tab.npend;
  uint32_t pn[kPend][3], qn[kPend][3], hn[3];
#pragma unroll
  for (int i = 0; i < kPend; ++i)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      pn[i][b] = tab.pend_neg[i][b];
      qn[i][b] = ALG ? tab.pair_neg[i][b] : 0u;
    }
#pragma unroll
  for (int b = 0; b < 3; ++b) hn[b] = ALG ? tab.half_neg[b] : 0u;
  for (int it = 0; it < iters; ++it) {
    const int r = rlo + g.row0 + it * g.rstep;
    const bool active = col_ok && r < rlo + nrows;
    uint32_t own = 0, pending = 0, always = 0, flip = 0;
    uint32_t b0 = 0, b1 = 0, b2 = 0, segid = 0;
    uint32_t m[3] = {0, 0, 0};
    uint32_t negm = 0, half = 0;  // heat bath: negative-field and zero-field lanes
    int P_ = 0;
    if (active) {
      const int y = wrap_i(g.y0 - g.yo + r, g.ly);
      P_ = (colour + y + z) & 1;  // x parity of this colour's sites in the row
      const uint2 me = ld_chk(pl, r * g.NC + cc, g.pw);
      const int ru = g.yw && r == 0 ? g.R - 1 : r - 1;
      const int rd = g.yw && r == g.R - 1 ? 0 : r + 1;
      const uint2 up = ld_chk(pl, ru * g.NC + cc, g.pw);
      const uint2 dn = ld_chk(pl, rd * g.NC + cc, g.pw);
      own = P_ ? me.y : me.x;
      const uint32_t other = P_ ? me.x : me.y;
      uint32_t lft, rgt;
      if (P_ == 0) {
        // even x = 2i: left = odd 2i-1 (index i-1), right = odd 2i+1 (index i)
        uint32_t carry = 0;
        if (has_prev) {
          const uint32_t po = ld_chk(pl, r * g.NC + cprev, g.pw).y;
          carry = first_seg ? (po >> (g.hlast - 1)) & 1u : po >> 31;
        }
        lft = (other << 1) | carry;
        rgt = other;
      } else {
        // odd x = 2i+1: left = even 2i (index i), right = even 2i+2 (index i+1)
        lft = other;
        const uint32_t ne = has_next ? ld_chk(pl, r * g.NC + cnext, g.pw).x & 1u : 0u;
        const int hb = last_seg ? g.hlast - 1 : 31;
        rgt = ((other >> 1) & ~(1u << hb)) | (ne << hb);
      }
      // Metropolis counts anti-aligned neighbours, the heat bath down ones
      const uint32_t ox = ALG ? 0u : own;
      uint32_t x0 = ox ^ lft, x1 = ox ^ rgt, x2 = ox ^ (P_ ? up.y : up.x), x3 = ox ^ (P_ ? dn.y : dn.x);
      if (DIM == 2) {
        const uint32_t s0 = x0 ^ x1 ^ x2;
        const uint32_t c0 = (x0 & x1) | (x2 & (x0 ^ x1));
        b0 = s0 ^ x3;
        const uint32_t c1 = s0 & x3;
        b1 = c0 ^ c1;
        b2 = c0 & c1;
      } else {
        const uint2 zm = pm[r * g.NC + cc], zp = pp[r * g.NC + cc];
        const uint32_t x4 = ox ^ (P_ ? zm.y : zm.x), x5 = ox ^ (P_ ? zp.y : zp.x);
        const uint32_t s0 = x0 ^ x1 ^ x2;
        const uint32_t c0 = (x0 & x1) | (x2 & (x0 ^ x1));
        const uint32_t s1 = x3 ^ x4 ^ x5;
        const uint32_t c1 = (x3 & x4) | (x5 & (x3 ^ x4));
        b0 = s0 ^ s1;
        const uint32_t c2 = s0 & s1;
        b1 = c0 ^ c1 ^ c2;
        b2 = (c0 & c1) | (c2 & (c0 ^ c1));
      }
      // masks of the pending classes (class index k = b2 b1 b0 in bits)
#pragma unroll
      for (int i = 0; i < kPend; ++i) {
        if (i < npend) {
          m[i] = (b0 ^ pn[i][0]) & (b1 ^ pn[i][1]) & (b2 ^ pn[i][2]) & valid;
          if (ALG) {
            const uint32_t mn = (b0 ^ qn[i][0]) & (b1 ^ qn[i][1]) & (b2 ^ qn[i][2]) & valid;
            m[i] |= mn;
            negm |= mn;
          }
          pending |= m[i];
        }
      }
      if (ALG) half = (b0 ^ hn[0]) & (b1 ^ hn[1]) & (b2 ^ hn[2]) & valid;
      always = valid & ~pending;
      segid = (uint32_t)(y + g.ly * z) * (uint32_t)g.nseg + (uint32_t)gs;
    }
    // bit-serial comparison of the 32 uniforms against their thresholds
    uint32_t lt = 0, eq = pending;
    const uint32_t ctrl0 = (uint32_t)colour | ((ALG ? TAG_HBITS : TAG_BITS) << 1);
    int q = 0;
    do {
      uint4 o = bits_philox(P, segid, ctrl0 | ((uint32_t)q << 8));
      if (ALG) {
        if (q == 0) lt = half & ~o.x;  // zero field: up iff u < 1/2
        o.x ^= negm;                   // negative field: compare ~u
        o.y ^= negm;
        o.z ^= negm;
        o.w ^= negm;
      }
      const uint4 t0 = tab.tq[q][0], t1 = tab.tq[q][1];
      uint4 tj = make_uint4(m[0] * t0.x + m[1] * t1.x, m[0] * t0.y + m[1] * t1.y,
                            m[0] * t0.z + m[1] * t1.z, m[0] * t0.w + m[1] * t1.w);
      if (DIM == 3) {  // a third pending class exists only for z = 6
        const uint4 t2 = tab.tq[q][2];
        tj.x += m[2] * t2.x;
        tj.y += m[2] * t2.y;
        tj.z += m[2] * t2.z;
        tj.w += m[2] * t2.w;
      }
      lt |= eq & tj.x & ~o.x;
      eq &= ~(tj.x ^ o.x);
      lt |= eq & tj.y & ~o.y;
      eq &= ~(tj.y ^ o.y);
      lt |= eq & tj.z & ~o.z;
      eq &= ~(tj.z ^ o.z);
      lt |= eq & tj.w & ~o.w;
      eq &= ~(tj.w ^ o.w);
      ++q;
    } while (q < 20 && __any_sync(full, eq));
    if (active) {
      // heat bath: the new spin is down iff (lt == neg), i.e. ~(lt ^ neg)
      flip = ALG ? (own ^ ~(lt ^ negm)) & valid : (always | lt) & valid;
      const uint32_t nw = own ^ flip;
      const int mi = GPUMC_IN(r * g.NC + cc, g.pw) ? r * g.NC + cc : 0;
      uint2& me = pl[mi];
      if (GPUMC_IN(r * g.NC + cc, g.pw)) {
        if (P_) me.y = nw;
        else me.x = nw;
      }
      const bool owned = owned_plane && owned_col && r >= g.yo && r < g.yo + g.hv;
      if (owned) {
        acc.nacc += __popc(flip);
        if (ALG) {
          // anti-aligned neighbours of a flipped site: k if it was up, z - k if down
          const uint32_t fu = flip & ~own, fd = flip & own;
          acc.ksum += __popc(fu & b0) + 2 * __popc(fu & b1) + 4 * __popc(fu & b2) - __popc(fd & b0) -
                      2 * __popc(fd & b1) - 4 * __popc(fd & b2) + 2 * DIM * __popc(fd);
        } else {
          acc.ksum += __popc(flip & b0) + 2 * __popc(flip & b1) + 4 * __popc(flip & b2);
        }
      }
      if (out_mode != 0) {
        // both colours of this segment are final now: count its down spins
        // and (mode 1) store the int8 row segment
        const uint2 fin = P_ ? make_uint2(me.x, nw) : make_uint2(nw, me.y);
        if (out_mode == 1) {
          const int y = wrap_i(g.y0 - g.yo + r, g.ly);
          uint4 v0, v1, v2, v3;
          unpack_segment(fin.x, fin.y, v0, v1, v2, v3);
          const size_t off = ((size_t)z * g.ly + y) * g.pitch + 64 * gs;
          uint4* out = (uint4*)(dst + off);
          if (GPUMC_IN(off + 63, g.gbytes)) {
            out[0] = v0;
            out[1] = v1;
            out[2] = v2;
            out[3] = v3;
          }
        }
        acc.down += __popc(fin.x & valid) + __popc(fin.y & valid);
        acc.owned_sites += 2 * __popc(valid);
      }
    }
  }
}

template <int ALG>
__device__ __forceinline__ void load_bits_table(BitsTab& tab, const LatDesc* L, const GroupDesc* G) {
  // the label can change between the sweeps of a resident launch: read it
  // from L2, not from a possibly stale L1 line
  const int label = __ldcg(&G->label[L->replica]);
  const int n = min(G->n_cls, 7);
  const uint32_t* head = G->head + label * G->n_cls;
  const unsigned long long* tail = G->tail + label * G->n_cls;
  // Metropolis: pending classes in increasing k (at most three for the
  // Ising table).  Heat bath: pair i = classes {i, z - i} (i < z/2) with the
  // threshold T[i]; its positive-field member is i for J >= 0, else z - i.
  int pc[3] = {0, 0, 0}, pn[3] = {0, 0, 0}, np = 0;
  const int zc = n - 1;
  if (ALG) {
    const bool jpos = G->J >= 0.0;
    for (int i = 0; i < zc / 2 && i < 3; ++i) {
      pc[i] = jpos ? i : zc - i;
      pn[i] = jpos ? zc - i : i;
      ++np;
    }
  } else {
    for (int k = 0; k < n; ++k)
      if (head[k] < 65536u && np < 3) pc[np++] = k;
  }
  if (threadIdx.x == 0) {
    tab.npend = np;
    for (int i = 0; i < 3; ++i)
      for (int b = 0; b < 3; ++b) {
        tab.pend_neg[i][b] = (i < np && ((pc[i] >> b) & 1)) ? 0u : 0xFFFFFFFFu;
        tab.pair_neg[i][b] = (i < np && ((pn[i] >> b) & 1)) ? 0u : 0xFFFFFFFFu;
      }
    for (int b = 0; b < 3; ++b) tab.half_neg[b] = (((zc / 2) >> b) & 1) ? 0u : 0xFFFFFFFFu;
  }
  for (int e = threadIdx.x; e < 80 * 3; e += kThreads) {
    const int j = e / 3, i = e - 3 * j;
    uint32_t v = 0;
    if (i < np) {
      const int k = ALG ? i : pc[i];
      const uint32_t h = head[k];
      const unsigned long long t = tail[k];
      v = j < 16 ? (h >> (15 - j)) & 1u : (uint32_t)((t >> (79 - j)) & 1ull);
    }
    reinterpret_cast<uint32_t*>(&tab.tq[j >> 2][i])[j & 3] = v;
  }
}

__device__ __forceinline__ void flush_bits(Accum* A, const PassAcc& a, int zc) {
  long long v[3] = {2LL * zc * a.nacc - 4LL * a.ksum, (long long)a.owned_sites - 2LL * a.down, a.nacc};
  cta_sum(v);
  if (threadIdx.x == 0) {
    if (v[0]) atomic_add_i64(&A->dE, v[0]);
    if (v[1]) atomic_add_i64(&A->mag, v[1]);
    if (v[2]) atomic_add_i64(&A->accepted, v[2]);
  }
}

template <int DIM, int ALG>
__global__ void __launch_bounds__(kThreads, DIM == 2 ? 4 : 3)
    k_sweep_ising_bits(const TileItem* __restrict__ tiles, LatDesc* __restrict__ lats,
                       GroupDesc* __restrict__ groups, LaunchCtl* __restrict__ ctl) {
  extern __shared__ __align__(16) uint2 bsm[];
  __shared__ BitsTab tab;
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
  load_bits_table<ALG>(tab, L, G);
  const BitsPhilox P = make_bits_philox(L->key, sweep);
  PassAcc acc = {0, 0, 0, 0};
  if (DIM == 2) {
    load_bits_plane(bsm, cur, 0, g);
    __syncthreads();
    bits_pass<2, ALG>(bsm, bsm, bsm, g, 0, 0, 1, g.R - 2, g.iters_black, true, 0, nxt, tab, P, acc);
    __syncthreads();
    bits_pass<2, ALG>(bsm, bsm, bsm, g, 0, 1, 2, g.hv, g.iters_white, true, 1, nxt, tab, P, acc);
  } else {
    const int lz = L->lz;
    const int dv = min(t.tz, lz - t.z0);
    const int pw = g.R * g.NC;
    for (int s = 0; s < dv + 4; ++s) {
      const int zl = t.z0 - 2 + s;
      uint2* Pl = bsm + (s & 3) * pw;
      load_bits_plane(Pl, cur, wrap_i(zl, lz), g);
      __syncthreads();
      if (s >= 2) {
        const int zb = zl - 1;
        bits_pass<3, ALG>(bsm + ((s - 1) & 3) * pw, bsm + ((s - 2) & 3) * pw, Pl, g, wrap_i(zb, lz), 0,
                     g.yo / 2, g.yw ? g.R : g.R - 2, g.iters_black, zb >= t.z0 && zb < t.z0 + dv, 0, nxt,
                     tab, P, acc);
        __syncthreads();
      }
      if (s >= 4) {
        const int zw = zl - 2;
        bits_pass<3, ALG>(bsm + ((s - 2) & 3) * pw, bsm + ((s - 3) & 3) * pw, bsm + ((s - 1) & 3) * pw, g,
                     wrap_i(zw, lz), 1, g.yo, g.hv, g.iters_white, true, 1, nxt, tab, P, acc);
      }
      __syncthreads();  // the next load overwrites the plane slot read above
    }
  }
  flush_bits(&L->acc, acc, 2 * DIM);
  group_epilogue(t.pad, lats, groups, ctl);
}

// ---------------------------------------------------------------------------
// Resident whole-row 2D tiles: temporal blocking across the sweeps of a launch.
//
// The packed parity masks of a tile (1 bit per site, 1/8 of the int8 rows)
// stay in shared memory for all the sweeps of one cooperative launch; with
// whole-row tiles sized to the device's CTA slots, every tile of the three
// headline lattices (3 x 8 MiB of bits) is resident at once.  A sweep is the
// same black and white pass as k_sweep_ising_bits, on the same random
// stream, so the trajectory is bit-identical to the per-sweep kernel.  The
// int8 buffer is read once at the start of the launch and the owned rows are
// written once at the end (to the buffer of the final sweep count), so HBM
// traffic per sweep is only the edge rows exchanged between tiles:
//   * after its white pass a tile publishes its first two and last two owned
//     rows (packed) to its exchange slot for that sweep's parity;
//   * a grid barrier ends the sweep; block 0 then runs the sweep epilogue of
//     every group (records, energy caches, sweep counters, PT exchange) and
//     publishes its completion in ctl->epi, which the other CTAs wait for
//     only before a sweep that follows a PT exchange (the labels, and so the
//     acceptance tables, change there);
//   * the next sweep refreshes the tile's four halo rows from the two
//     neighbours' slots (tile above: its last two rows; tile below: its first
//     two) and recomputes the black halo rows as usual.
// Every barrier wait is bounded by `spin_limit` polls (128 ns sleeps; the
// host's default is 2^22, about half a second): a CTA that waits too long (or
// sees another CTA's error) sets ctl->err and returns, every other CTA then
// leaves at its next barrier, and the host reports the error.  The
// cooperative launch guarantees that all CTAs are co-resident.
// ---------------------------------------------------------------------------

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ uint64_t ld_volatile_u64(const uint64_t* p) {
  return *(const volatile uint64_t*)p;
}

__device__ bool resident_grid_sync(LaunchCtl* ctl, unsigned int target, long long spin_limit) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(&ctl->bar, 1u);
    int good = 1;
    long long it = 0;
    while (ld_acquire_u32(&ctl->bar) < target) {
      if (*(volatile int32_t*)&ctl->err != 0 || ++it > spin_limit) {
        atomicExch(&ctl->err, 1);
        good = 0;
        break;
      }
      __nanosleep(128);
    }
    if (good && *(volatile int32_t*)&ctl->err != 0) good = 0;
    ok = good;
  }
  __syncthreads();
  return ok != 0;
}

// Bounded wait until block 0 has finished the epilogue of launch-local sweep
// `k1 - 1` (ctl->epi >= k1); on giving up, flags the error like a barrier.
__device__ bool resident_wait_epilogue(LaunchCtl* ctl, unsigned int k1, long long spin_limit) {
  __shared__ int ok;
  if (threadIdx.x == 0) {
    int good = 1;
    long long it = 0;
    while (ld_acquire_u32(&ctl->epi) < k1) {
      if (*(volatile int32_t*)&ctl->err != 0 || ++it > spin_limit) {
        atomicExch(&ctl->err, 1);
        good = 0;
        break;
      }
      __nanosleep(128);
    }
    ok = good;
  }
  __syncthreads();
  return ok != 0;
}

// Owned rows (local rows 2 .. hv+1) of a whole-row tile to int8 spins.
__device__ __forceinline__ void store_owned_rows(const uint2* pl, const BitsGeom& g, int8_t* dst) {
  if (g.row0 >= g.rstep) return;
  const int gs = wrap_i(g.s0 + g.col - g.xh, g.nseg);
  for (int it = 0; it < g.iters_white; ++it) {
    const int r = 2 + g.row0 + it * g.rstep;
    if (r >= 2 + g.hv) break;
    const uint2 fin = ld_chk(pl, r * g.NC + g.col, g.pw);
    const int y = wrap_i(g.y0 - 2 + r, g.ly);
    uint4 v0, v1, v2, v3;
    unpack_segment(fin.x, fin.y, v0, v1, v2, v3);
    const size_t off = (size_t)y * g.pitch + 64 * gs;
    uint4* out = (uint4*)(dst + off);
    if (GPUMC_IN(off + 63, g.gbytes)) {
      out[0] = v0;
      out[1] = v1;
      out[2] = v2;
      out[3] = v3;
    }
  }
}

template <int ALG>
__global__ void __launch_bounds__(kThreads, 4)
    k_sweep_ising_resident(const TileItem* __restrict__ tiles, LatDesc* __restrict__ lats,
                           GroupDesc* __restrict__ groups, LaunchCtl* __restrict__ ctl,
                           const int2* __restrict__ nbr, uint2* __restrict__ xchg, int xstride,
                           int n_sweeps, long long spin_limit) {
  extern __shared__ __align__(16) uint2 bsm[];
  __shared__ BitsTab tab;
  const TileItem t = tiles[blockIdx.x];
  LatDesc* L = &lats[t.lat];
  const GroupDesc* G = &groups[L->group];
  const BitsGeom g = make_bits_geom(t, L);
  const int W = g.NC;  // whole rows: one column per segment, no column halo
  const size_t slot = (size_t)4 * W;
  uint2* mine = xchg + (size_t)blockIdx.x * xstride;  // [parity][4 rows][W]
  const int2 nb = nbr[blockIdx.x];
  // sweep index of launch-local iteration k: s0 + k (the epilogue advances
  // L->sweep the same way, stopping at the target)
  const uint64_t s0 = ld_volatile_u64(&L->sweep);
  const uint64_t target = L->target;
  load_bits_plane(bsm, (const int8_t*)L->buf[s0 & 1], 0, g);
  unsigned int phase = 0;
  for (int k = 0; k < n_sweeps; ++k) {
    const uint64_t sweep = s0 + (uint64_t)k;
    if (sweep < target) {
      if (k > 0) {
        const uint2* up = xchg + (size_t)nb.x * xstride + ((k - 1) & 1) * slot;
        const uint2* dn = xchg + (size_t)nb.y * xstride + ((k - 1) & 1) * slot;
        for (int i = threadIdx.x; i < 4 * W; i += kThreads) {
          const int sl = i / W, c = i - sl * W;
          const int row = sl < 2 ? sl : g.hv + sl;  // local rows 0, 1, hv+2, hv+3
          const long long xn = (long long)gridDim.x * xstride;  // exchange buffer words
          (void)xn;
          const long long iu = (long long)(up - xchg) + (long long)(2 + sl) * W + c;
          const long long id = (long long)(dn - xchg) + (long long)(sl - 2) * W + c;
          const uint2 v = sl < 2 ? (GPUMC_IN(iu, xn) ? __ldcg(xchg + iu) : make_uint2(0, 0))
                                 : (GPUMC_IN(id, xn) ? __ldcg(xchg + id) : make_uint2(0, 0));
          st_chk(bsm, (long long)row * W + c, (long long)g.pw, v);
        }
      }
      // the acceptance table depends only on the label, which within a
      // launch only a PT exchange changes (after sweep s with
      // (s + 1) % interval == 0, i.e. before a sweep with sweep % interval
      // == 0); reloading it every sweep cost 1.3 % of the headline
      if (k == 0 || (G->pt_interval > 0 && sweep % (uint64_t)G->pt_interval == 0))
        load_bits_table<ALG>(tab, L, G);
      __syncthreads();
      const BitsPhilox P = make_bits_philox(L->key, sweep);
      PassAcc acc = {0, 0, 0, 0};
      bits_pass<2, ALG>(bsm, bsm, bsm, g, 0, 0, 1, g.R - 2, g.iters_black, true, 0, nullptr, tab, P, acc);
      __syncthreads();
      bits_pass<2, ALG>(bsm, bsm, bsm, g, 0, 1, 2, g.hv, g.iters_white, true, 2, nullptr, tab, P, acc);
      flush_bits((k & 1) ? &L->acc2 : &L->acc, acc, 4);
      __syncthreads();
      uint2* out = mine + (size_t)(k & 1) * slot;
      for (int i = threadIdx.x; i < 4 * W; i += kThreads) {
        const int sl = i / W, c = i - sl * W;
        const int row = sl < 2 ? 2 + sl : g.hv + sl - 2;  // local rows 2, 3, hv, hv+1
        const long long io = (long long)(out - xchg) + (long long)sl * W + c;
        if (GPUMC_IN(io, (long long)gridDim.x * xstride)) __stcg(xchg + io, ld_chk(bsm, (long long)row * W + c, (long long)g.pw));
      }
    }
    if (!resident_grid_sync(ctl, ++phase * gridDim.x, spin_limit)) return;
    if (blockIdx.x == 0) {
      // the epilogue of sweep k drains accumulator slot k & 1, which no CTA
      // touches again before the next barrier (its next use is sweep k + 2)
      finish_groups(lats, groups, ctl->group_ids, ctl->n_groups, k & 1);
      __syncthreads();
      if (threadIdx.x == 0) {
        __threadfence();
        atomicExch(&ctl->epi, (unsigned int)(k + 1));
      }
    } else if (G->pt_interval > 0 && sweep < target && ((sweep + 1) % (uint64_t)G->pt_interval) == 0) {
      // a PT exchange after this sweep changes this group's labels (its
      // acceptance tables for the next sweep): wait for the epilogue
      if (!resident_wait_epilogue(ctl, (unsigned int)(k + 1), spin_limit)) return;
    }
  }
  const uint64_t s_end = s0 + (uint64_t)n_sweeps < target ? s0 + (uint64_t)n_sweeps : (s0 > target ? s0 : target);
  store_owned_rows(bsm, g, (int8_t*)L->buf[s_end & 1]);
}

// ---------------------------------------------------------------------------
// Resident 3D tiles: the same temporal blocking for cubic lattices.  A tile is
// a slab of whole planes z0 .. z0+dz-1 (dz >= 2; rows wrap inside a plane, no
// y halo), held with two halo planes on each side: local planes 0 .. dz+3,
// plane p at z0 - 2 + p.  A sweep runs the black pass on planes 1 .. dz+2
// (the halo planes next to the slab too, so the white pass of the slab's end
// planes sees final black neighbours) and the white pass on the owned planes
// 2 .. dz+1, the same passes and stream as the streaming 3D kernel, so the
// trajectory is bit-identical to it.  After the white pass a tile publishes
// its first two and last two owned planes to its exchange slot (parity k & 1)
// and, after the grid barrier, refreshes halo planes 0, 1 from the slab below
// (its last two owned planes) and dz+2, dz+3 from the slab above (its first
// two).  The epilogue, the PT exchange and the bounded waits are those of the
// 2D resident kernel.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void store_plane(const uint2* pl, const BitsGeom& g, int z, int8_t* dst) {
  if (g.row0 >= g.rstep) return;
  const int gs = wrap_i(g.s0 + g.col - g.xh, g.nseg);
  for (int it = 0; it < g.iters_load; ++it) {
    const int r = g.row0 + it * g.rstep;
    if (r >= g.R) break;
    const uint2 fin = ld_chk(pl, r * g.NC + g.col, g.pw);
    uint4 v0, v1, v2, v3;
    unpack_segment(fin.x, fin.y, v0, v1, v2, v3);
    const size_t off = ((size_t)z * g.ly + r) * g.pitch + 64 * gs;
    uint4* out = (uint4*)(dst + off);
    if (GPUMC_IN(off + 63, g.gbytes)) {
      out[0] = v0;
      out[1] = v1;
      out[2] = v2;
      out[3] = v3;
    }
  }
}

template <int ALG>
__global__ void __launch_bounds__(kThreads, 3)
    k_sweep_ising_resident3(const TileItem* __restrict__ tiles, LatDesc* __restrict__ lats,
                            GroupDesc* __restrict__ groups, LaunchCtl* __restrict__ ctl,
                            const int2* __restrict__ nbr, uint2* __restrict__ xchg, int xstride,
                            int n_sweeps, long long spin_limit) {
  extern __shared__ __align__(16) uint2 bsm[];
  __shared__ BitsTab tab;
  const TileItem t = tiles[blockIdx.x];
  LatDesc* L = &lats[t.lat];
  const GroupDesc* G = &groups[L->group];
  const BitsGeom g = make_bits_geom(t, L);  // whole planes: yw, R = hv = ly
  const int lz = L->lz;
  const int dz = min(t.tz, lz - t.z0);
  const int pw = g.pw;
  const long long np = (long long)(dz + 4) * pw;  // words of the resident slab
  const size_t slot = (size_t)4 * pw;
  const long long xn = (long long)gridDim.x * xstride;  // words of the exchange buffer
  (void)xn;
  uint2* mine = xchg + (size_t)blockIdx.x * xstride;  // [parity][4 planes][pw]
  const int2 nb = nbr[blockIdx.x];  // (slab below, slab above)
  const uint64_t s0 = ld_volatile_u64(&L->sweep);
  const uint64_t target = L->target;
  auto zof = [&](int p) { return wrap_i(t.z0 - 2 + p, lz); };
  for (int p = 0; p < dz + 4; ++p) load_bits_plane(bsm + (size_t)p * pw, (const int8_t*)L->buf[s0 & 1], zof(p), g);
  unsigned int phase = 0;
  for (int k = 0; k < n_sweeps; ++k) {
    const uint64_t sweep = s0 + (uint64_t)k;
    if (sweep < target) {
      if (k > 0) {
        const long long dn = (long long)nb.x * xstride + (long long)((k - 1) & 1) * slot;
        const long long up = (long long)nb.y * xstride + (long long)((k - 1) & 1) * slot;
        for (int i = threadIdx.x; i < 4 * pw; i += kThreads) {
          const int sl = i / pw, w = i - sl * pw;
          const int p = sl < 2 ? sl : dz + sl;  // local planes 0, 1, dz+2, dz+3
          const long long src = sl < 2 ? dn + (long long)(2 + sl) * pw + w : up + (long long)(sl - 2) * pw + w;
          const uint2 v = GPUMC_IN(src, xn) ? __ldcg(xchg + src) : make_uint2(0, 0);
          st_chk(bsm, (long long)p * pw + w, np, v);
        }
      }
      if (k == 0 || (G->pt_interval > 0 && sweep % (uint64_t)G->pt_interval == 0))
        load_bits_table<ALG>(tab, L, G);
      __syncthreads();
      const BitsPhilox P = make_bits_philox(L->key, sweep);
      PassAcc acc = {0, 0, 0, 0};
      for (int p = 1; p <= dz + 2; ++p)
        bits_pass<3, ALG>(bsm + (size_t)p * pw, bsm + (size_t)(p - 1) * pw, bsm + (size_t)(p + 1) * pw, g, zof(p),
                          0, 0, g.R, g.iters_black, p >= 2 && p <= dz + 1, 0, nullptr, tab, P, acc);
      __syncthreads();
      for (int p = 2; p <= dz + 1; ++p)
        bits_pass<3, ALG>(bsm + (size_t)p * pw, bsm + (size_t)(p - 1) * pw, bsm + (size_t)(p + 1) * pw, g, zof(p),
                          1, 0, g.hv, g.iters_white, true, 2, nullptr, tab, P, acc);
      flush_bits((k & 1) ? &L->acc2 : &L->acc, acc, 6);
      __syncthreads();
      const long long out = (long long)blockIdx.x * xstride + (long long)(k & 1) * slot;
      for (int i = threadIdx.x; i < 4 * pw; i += kThreads) {
        const int sl = i / pw, w = i - sl * pw;
        const int p = sl < 2 ? 2 + sl : dz + sl - 2;  // local planes 2, 3, dz, dz+1
        if (GPUMC_IN(out + (long long)sl * pw + w, xn))
          __stcg(xchg + out + (long long)sl * pw + w, ld_chk(bsm, (long long)p * pw + w, np));
      }
    }
    if (!resident_grid_sync(ctl, ++phase * gridDim.x, spin_limit)) return;
    if (blockIdx.x == 0) {
      finish_groups(lats, groups, ctl->group_ids, ctl->n_groups, k & 1);
      __syncthreads();
      if (threadIdx.x == 0) {
        __threadfence();
        atomicExch(&ctl->epi, (unsigned int)(k + 1));
      }
    } else if (G->pt_interval > 0 && sweep < target && ((sweep + 1) % (uint64_t)G->pt_interval) == 0) {
      if (!resident_wait_epilogue(ctl, (unsigned int)(k + 1), spin_limit)) return;
    }
  }
  (void)mine;
  const uint64_t s_end = s0 + (uint64_t)n_sweeps < target ? s0 + (uint64_t)n_sweeps : (s0 > target ? s0 : target);
  for (int p = 2; p <= dz + 1; ++p) store_plane(bsm + (size_t)p * pw, g, zof(p), (int8_t*)L->buf[s_end & 1]);
}

template __global__ void k_sweep_ising_bits<2, 0>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template __global__ void k_sweep_ising_bits<3, 0>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template __global__ void k_sweep_ising_bits<2, 1>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template __global__ void k_sweep_ising_bits<3, 1>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template __global__ void k_sweep_ising_resident<0>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*,
                                                   const int2*, uint2*, int, int, long long);
template __global__ void k_sweep_ising_resident<1>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*,
                                                   const int2*, uint2*, int, int, long long);
template __global__ void k_sweep_ising_resident3<0>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*,
                                                    const int2*, uint2*, int, int, long long);
template __global__ void k_sweep_ising_resident3<1>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*,
                                                    const int2*, uint2*, int, int, long long);

GPUMC_BOUNDS_MODULE(sweep_ising_bits)

}  // namespace gpumc
