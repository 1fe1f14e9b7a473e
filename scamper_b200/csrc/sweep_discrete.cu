// Fused two-colour checkerboard sweep for int8 q-state Potts spins on
// periodic square (2D) and cubic (3D) lattices (int8 Ising runs on the
// bit-sliced kernel of sweep_ising_bits.cu).
//
// Method (one kernel launch = one full sweep of every lattice in the launch):
//   * each CTA owns a tile of one lattice: tile_cx 16-site chunks x tile_y
//     rows (x tile_z planes in 3D, marched plane by plane through shared-memory
//     rings);
//   * the tile plus a 2-site halo is staged from the read buffer into shared
//     memory with cp.async; colour 0 is updated on the tile and a 1-site halo
//     ring into a second shared plane (halo sites are recomputed redundantly:
//     the counter-based RNG makes them identical to the owner's result), then
//     colour 1 on the tile straight to the other ping-pong buffer in HBM.  HBM
//     traffic is one read and one write of every byte per sweep.
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
//
// Heat bath (ALG = 1; HeatBathCore, CMC.rs/src/algorithms/heat_bath.rs:41-66,
// with PottsModel::heat_bath_sample_site, CMC.rs/src/lattice/models.rs:
// 340-380): the new state of a site is drawn from all q states with weights
// exp(beta J n_s), n_s = neighbours in state s.  As in the reference the
// weights are taken relative to the site's largest one, here as 64-bit
// integers W[d] = floor(2^60 exp(-beta |J| d)) from the host table (d = the
// state's count distance from the site's most favoured count), so the draw is
// exact integer arithmetic: x = floor(u * total / 2^64) for a 64-bit uniform
// u, then the first state whose cumulative weight exceeds x in state order.
// Word w (0..3) of a 16-site chunk draws one Philox block, counter (chunk,
// colour | TAG_HB << 1 | w << 8, sweep): words 0-1 are the uniform of its
// first pass-colour site, words 2-3 of its second.  "Accepted" counts the
// sites whose state changed.
#include "device_common.cuh"
#include "epilogue.cuh"

namespace gpumc {

struct SiteTab {
  uint32_t head[kMaxClasses];
  unsigned long long tail[kMaxClasses];  // heat bath: the weights W[d]
  int32_t jneg;                          // heat bath: J < 0 (favoured = fewest neighbours)
};

// Heat-bath draw of one Potts site from its neighbour counts n[0..Q-1], old
// state s and 64-bit uniform u; returns the new state t and sets dn = n[t] -
// n[s] (dE = -J dn).  Exact integer arithmetic (restated by the oracle).
template <int Q>
__device__ __forceinline__ uint32_t potts_hb_pick(const int (&n)[kMaxPottsCounts], uint32_t s,
                                                  unsigned long long u, const SiteTab& tab, int& dn) {
  int nmax = 0, nmin = 64;
#pragma unroll
  for (int k = 0; k < Q; ++k) {
    nmax = max(nmax, n[k]);
    nmin = min(nmin, n[k]);
  }
  const int ref = tab.jneg ? nmin : nmax, sg = tab.jneg ? 1 : -1;  // d = |n - ref|
  unsigned long long w[Q], tot = 0;
#pragma unroll
  for (int k = 0; k < Q; ++k) {
    w[k] = tab.tail[sg * (n[k] - ref)];
    tot += w[k];
  }
  unsigned long long x = __umul64hi(u, tot);
  uint32_t t = (uint32_t)(Q - 1);
  int nt = n[Q - 1], ns = 0;
  bool found = false;
#pragma unroll
  for (int k = 0; k < Q; ++k) {
    if (!found) {
      if (x < w[k]) {
        t = (uint32_t)k;
        nt = n[k];
        found = true;
      } else {
        x -= w[k];
      }
    }
    if ((uint32_t)k == s) ns = n[k];
  }
  dn = nt - ns;
  return t;
}

// Heat bath of the two pass-colour sites of one word (bytes 0 and 2 after the
// pre-shift), from one Philox block r.
template <int DIM, int Q>
__device__ __forceinline__ uint32_t potts_hb_word(uint32_t o, uint32_t lw, uint32_t rw, uint32_t u,
                                                  uint32_t d, uint32_t a, uint32_t b, int bsh,
                                                  const uint4 r, const SiteTab& tab,
                                                  uint32_t own2, int& nacc, int& dsum) {
  constexpr int zc = 2 * DIM;
  const uint32_t os = o >> bsh;
  const uint32_t sA = os & 0xFFu, sB = (os >> 16) & 0xFFu;
  const uint32_t nbw[6] = {lw >> bsh, rw >> bsh, u >> bsh, d >> bsh, a >> bsh, b >> bsh};
  int nA[kMaxPottsCounts], nB[kMaxPottsCounts];
#pragma unroll
  for (int k = 0; k < Q; ++k) {
    const uint32_t pat = (uint32_t)k * 0x00010001u;
    uint32_t c = 0;  // bytes 0 and 2: neighbours NOT in state k
#pragma unroll
    for (int i = 0; i < zc; ++i) {
      const uint32_t x = (nbw[i] ^ pat) & 0x00FF00FFu;
      c += ((x + 0x00FF00FFu) >> 8) & 0x00010001u;
    }
    nA[k] = zc - (int)(c & 0xFFu);
    nB[k] = zc - (int)(c >> 16);
  }
  int dA, dB;
  const uint32_t tA = potts_hb_pick<Q>(nA, sA, (unsigned long long)r.x | ((unsigned long long)r.y << 32), tab, dA);
  const uint32_t tB = potts_hb_pick<Q>(nB, sB, (unsigned long long)r.z | ((unsigned long long)r.w << 32), tab, dB);
  const int oA = (int)((tA != sA) & (own2 & 1u)), oB = (int)((tB != sB) & ((own2 >> 1) & 1u));
  nacc += oA + oB;
  dsum += oA * dA + oB * dB;
  const uint32_t ns = (os & ~0x00FF00FFu) | tA | (tB << 16);
  const uint32_t keep = bsh ? 0x00FF00FFu : 0xFF00FF00u;
  return (o & keep) | (ns << bsh);
}

// Philox4x32-10 with the per-sweep uniform part hoisted: the counter words
// 1..3 (colour/tag, sweep) are the same for every draw of a pass, so round 1
// needs one multiply, and the bumped keys are computed once per CTA.
struct PhiloxCtx {
  uint32_t a, b, c;  // round-1 terms: hi(M1*c2) ^ k0, lo(M1*c2), c3 ^ k1
  uint32_t k0[10], k1[10];
};

__device__ __forceinline__ PhiloxCtx make_philox(uint64_t key, uint64_t sweep) {
  PhiloxCtx P;
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

// draw(key, index, colour, tag, 0, sweep) for index < 2^32; ctrl = colour |
// tag << 1 (counter word 1).
__device__ __forceinline__ uint4 philox_fast(const PhiloxCtx& P, uint32_t index, uint32_t ctrl) {
  uint4 c = make_uint4(P.a ^ ctrl, P.b, __umulhi(0xD2511F53u, index) ^ P.c, 0xD2511F53u * index);
#pragma unroll
  for (int r = 1; r < 10; ++r) {
    const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
    const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
    c = make_uint4(hi1 ^ c.y ^ P.k0[r], lo1, hi0 ^ c.w ^ P.k1[r], lo0);
  }
  return c;
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// Per-word update of the two sites of the pass colour.  Words are pre-shifted
// right by `bsh` (0 or 8) so the two sites sit in bytes 0 and 2.
// Potts: returns the new word (sites of the pass colour replaced on accept).
template <int DIM>
__device__ __forceinline__ uint32_t potts_word(uint32_t o, uint32_t lw, uint32_t rw, uint32_t u,
                                               uint32_t d, uint32_t a, uint32_t b, int bsh,
                                               uint32_t rnd, uint32_t rprop, const SiteTab& tab,
                                               int q, uint64_t key, uint32_t site0,
                                               uint32_t colour, uint64_t sweep, uint32_t own2,
                                               int& nacc, int& dsum) {
  constexpr int zc = 2 * DIM;
  const uint32_t os = o >> bsh;
  const uint32_t sA = os & 0xFFu, sB = (os >> 16) & 0xFFu;
  const uint32_t n = (uint32_t)(q - 1);
  const uint32_t rej = 65536u % n;
  const uint32_t pA = rprop & 0xFFFFu, pB = rprop >> 16;
  const uint32_t mA = pA * n, mB = pB * n;
  uint32_t rA = mA >> 16, rB = mB >> 16;
  const uint32_t siteA = site0 + (uint32_t)(bsh >> 3), siteB = siteA + 2u;
  if (__builtin_expect(((mA & 0xFFFFu) < rej) | ((mB & 0xFFFFu) < rej), 0)) {
    if ((mA & 0xFFFFu) < rej) rA = potts_refine(key, siteA, colour, sweep, n);
    if ((mB & 0xFFFFu) < rej) rB = potts_refine(key, siteB, colour, sweep, n);
  }
  const uint32_t tA = rA < sA ? rA : rA + 1u, tB = rB < sB ? rB : rB + 1u;
  // byte-equality counts of the neighbours against s and t at bytes 0 and 2
  const uint32_t S = sA | (sB << 16), T = tA | (tB << 16);
  uint32_t cs = 0, ct = 0;
  const uint32_t nbw[6] = {lw >> bsh, rw >> bsh, u >> bsh, d >> bsh, a >> bsh, b >> bsh};
#pragma unroll
  for (int i = 0; i < zc; ++i) {
    const uint32_t xs = (nbw[i] ^ S) & 0x00FF00FFu;
    const uint32_t xt = (nbw[i] ^ T) & 0x00FF00FFu;
    cs += ((xs + 0x00FF00FFu) >> 8) & 0x00010001u;  // 1 where the byte is nonzero
    ct += ((xt + 0x00FF00FFu) >> 8) & 0x00010001u;
  }
  // counts of equal neighbours = zc - nonzero counts
  const int nsA = zc - (int)(cs & 0xFFu), nsB = zc - (int)(cs >> 16);
  const int ntA = zc - (int)(ct & 0xFFu), ntB = zc - (int)(ct >> 16);
  const int dA = ntA - nsA, dB = ntB - nsB;
  const uint32_t cA = (uint32_t)(dA + zc), cB = (uint32_t)(dB + zc);
  const uint32_t thA = tab.head[cA], thB = tab.head[cB];
  const uint32_t uA = rnd & 0xFFFFu, uB = rnd >> 16;
  bool aA = uA < thA, aB = uB < thB;
  if (__builtin_expect((uA == thA) | (uB == thB), 0)) {
    if (uA == thA) aA = refine_accept(key, siteA, colour, sweep, tab.tail[cA]);
    if (uB == thB) aB = refine_accept(key, siteB, colour, sweep, tab.tail[cB]);
  }
  const int oA = (int)(aA & (own2 & 1u)), oB = (int)(aB & ((own2 >> 1) & 1u));
  nacc += oA + oB;
  dsum += oA * dA + oB * dB;
  uint32_t ns = os;
  if (aA) ns = (ns & ~0xFFu) | tA;
  if (aB) ns = (ns & ~0xFF0000u) | (tB << 16);
  // bytes 1 and 3 of the shifted word are the other colour: untouched
  const uint32_t keep = bsh ? 0x00FF00FFu : 0xFF00FF00u;
  return (o & keep) | (ns << bsh);
}

template <int MODEL, int DIM>
__device__ __forceinline__ uint4 update_chunk(const uint4 own, const uint4 up, const uint4 dn,
                                              const uint4 zm, const uint4 zp, uint32_t wprev,
                                              uint32_t wnext, int bsh, const uint4 rnd,
                                              const uint4 rprop, const SiteTab& tab, int q,
                                              uint64_t key, uint32_t site0, uint32_t colour,
                                              uint64_t sweep, uint32_t owned16, int& nacc,
                                              int& acc2) {
  const uint32_t o[4] = {own.x, own.y, own.z, own.w};
  const uint32_t uu[4] = {up.x, up.y, up.z, up.w};
  const uint32_t dd[4] = {dn.x, dn.y, dn.z, dn.w};
  const uint32_t aa[4] = {zm.x, zm.y, zm.z, zm.w};
  const uint32_t bb[4] = {zp.x, zp.y, zp.z, zp.w};
  const uint32_t rr[4] = {rnd.x, rnd.y, rnd.z, rnd.w};
  const uint32_t rp[4] = {rprop.x, rprop.y, rprop.z, rprop.w};
  const int bp = bsh >> 3;
  uint32_t res[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint32_t lw = __funnelshift_l(i == 0 ? wprev : o[i - 1], o[i], 8);
    const uint32_t rw = __funnelshift_r(o[i], i == 3 ? wnext : o[i + 1], 8);
    const uint32_t own2 = ((owned16 >> (4 * i + bp)) & 1u) | (((owned16 >> (4 * i + bp + 2)) & 1u) << 1);
    res[i] = potts_word<DIM>(o[i], lw, rw, uu[i], dd[i], aa[i], bb[i], bsh, rr[i], rp[i], tab, q, key,
                             site0 + 4u * i, colour, sweep, own2, nacc, acc2);
  }
  return make_uint4(res[0], res[1], res[2], res[3]);
}

template <int DIM>
__device__ __forceinline__ uint4 update_chunk_hb(const uint4 own, const uint4 up, const uint4 dn,
                                                 const uint4 zm, const uint4 zp, uint32_t wprev,
                                                 uint32_t wnext, int bsh, const PhiloxCtx& P,
                                                 uint32_t chunk, uint32_t colour, const SiteTab& tab,
                                                 int q, uint32_t owned16, int& nacc, int& acc2) {
  const uint32_t o[4] = {own.x, own.y, own.z, own.w};
  const uint32_t uu[4] = {up.x, up.y, up.z, up.w};
  const uint32_t dd[4] = {dn.x, dn.y, dn.z, dn.w};
  const uint32_t aa[4] = {zm.x, zm.y, zm.z, zm.w};
  const uint32_t bb[4] = {zp.x, zp.y, zp.z, zp.w};
  const int bp = bsh >> 3;
  uint32_t res[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint32_t lw = __funnelshift_l(i == 0 ? wprev : o[i - 1], o[i], 8);
    const uint32_t rw = __funnelshift_r(o[i], i == 3 ? wnext : o[i + 1], 8);
    const uint32_t own2 = ((owned16 >> (4 * i + bp)) & 1u) | (((owned16 >> (4 * i + bp + 2)) & 1u) << 1);
    const uint4 r = philox_fast(P, chunk, colour | (TAG_HB << 1) | ((uint32_t)i << 8));
    // q is uniform over the launch's tile: one branch, loops of exactly q states
    switch (q) {
#define HB_CASE(QQ) \
  case QQ: res[i] = potts_hb_word<DIM, QQ>(o[i], lw, rw, uu[i], dd[i], aa[i], bb[i], bsh, r, tab, own2, nacc, acc2); break;
      HB_CASE(2) HB_CASE(3) HB_CASE(4) HB_CASE(5) HB_CASE(6) HB_CASE(7)
      default: HB_CASE(8)
#undef HB_CASE
    }
  }
  return make_uint4(res[0], res[1], res[2], res[3]);
}

// Scalar update of one halo site (positions x0-1 and x0+Wv, whose draws come
// from chunks the vector pass does not cover), reading plane `src`.
template <int MODEL, int DIM, int ALG>
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
  if (ALG) {
    int n[kMaxPottsCounts];
#pragma unroll
    for (int k = 0; k < kMaxPottsCounts; ++k) {
      n[k] = 0;
#pragma unroll
      for (int i = 0; i < zc; ++i) n[k] += nb[i] == k ? 1 : 0;
    }
    const uint4 hv = draw(key, chunk, colour, TAG_HB, (uint32_t)(slot >> 1), sweep);
    const unsigned long long u = (slot & 1) ? ((unsigned long long)hv.z | ((unsigned long long)hv.w << 32))
                                            : ((unsigned long long)hv.x | ((unsigned long long)hv.y << 32));
    int dn;
    switch (q) {
      case 2: return (int8_t)potts_hb_pick<2>(n, (uint32_t)s, u, tab, dn);
      case 3: return (int8_t)potts_hb_pick<3>(n, (uint32_t)s, u, tab, dn);
      case 4: return (int8_t)potts_hb_pick<4>(n, (uint32_t)s, u, tab, dn);
      case 5: return (int8_t)potts_hb_pick<5>(n, (uint32_t)s, u, tab, dn);
      case 6: return (int8_t)potts_hb_pick<6>(n, (uint32_t)s, u, tab, dn);
      case 7: return (int8_t)potts_hb_pick<7>(n, (uint32_t)s, u, tab, dn);
      default: return (int8_t)potts_hb_pick<8>(n, (uint32_t)s, u, tab, dn);
    }
  }
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
  if (remaining >= 16) return 0xFFFFu;
  if (remaining <= 0) return 0u;
  return (1u << remaining) - 1u;
}

// Tile geometry shared by the passes.  Shared planes hold rows y0-2 ..
// y0+hv+1; logical x maps to byte x - x0 + 16 of a row of S bytes.
struct TileGeom {
  int x0, y0, W, S, Wv, ncv, hv, R;
  int lx, ly, pitch, pc;
  long long gbytes;  // bytes of one int8 buffer of the lattice (bounds checks)
  // thread mapping of the vector passes: fixed chunk column, rows strided
  int col, row0, rstep;
  bool active;
};

__device__ __forceinline__ int wrap_row(int y, int ly) {
  return y < 0 ? y + ly : (y >= ly ? y - ly : y);
}

// Stage rows y0-2 .. y0+hv+1 of plane z (cp.async, 16 B per chunk) and fetch
// the wrapped halo bytes into registers (written by stage_halo after the wait).
__device__ __forceinline__ void stage_plane(uint8_t* plane, const int8_t* src, int z,
                                            const TileGeom& g) {
  if (!g.active) return;
  const size_t zoff = (size_t)z * g.ly;
  const int c = g.col;
  for (int r = g.row0; r < g.R; r += g.rstep) {
    const int y = wrap_row(g.y0 - 2 + r, g.ly);
    const size_t so = (zoff + y) * (size_t)g.pitch + g.x0 + 16 * c;
    if (GPUMC_IN(so + 15, g.gbytes) && GPUMC_IN(r * g.S + 31 + 16 * c, (long long)g.R * g.S))
      cp_async16(plane + r * g.S + 16 + 16 * c, src + so);
  }
}
struct HaloBytes {
  int8_t v[2];
  int off[2];
};
__device__ __forceinline__ HaloBytes fetch_halo(const int8_t* src, int z, const TileGeom& g) {
  // thread t < 2R handles row t>>1, side t&1 (two bytes each)
  HaloBytes h;
  h.off[0] = h.off[1] = -1;
  const int t = threadIdx.x;
  if (t < 2 * g.R) {
    const int r = t >> 1, side = t & 1;
    const int y = wrap_row(g.y0 - 2 + r, g.ly);
    const size_t row = ((size_t)z * g.ly + y) * (size_t)g.pitch;
    const int p0 = side ? g.x0 + g.Wv : g.x0 - 2;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      int xr = p0 + j;
      xr = xr < 0 ? xr + g.lx : (xr >= g.lx ? xr - g.lx : xr);
      h.v[j] = ld_chk(src, (long long)(row + xr), g.gbytes);
      h.off[j] = r * g.S + 16 + (p0 + j - g.x0);
    }
  }
  return h;
}
__device__ __forceinline__ void store_halo(uint8_t* plane, const HaloBytes& h, const TileGeom& g) {
  if (h.off[0] >= 0) {
    st_chk(plane, h.off[0], (long long)g.R * g.S, (uint8_t)h.v[0]);
    st_chk(plane, h.off[1], (long long)g.R * g.S, (uint8_t)h.v[1]);
  }
}

// Colour 0 on rows [1, R-1) of plane A, written to plane B (all bytes of the
// chunk: colour-1 bytes are copied unchanged).
template <int MODEL, int DIM, int ALG>
__device__ __forceinline__ void black_pass(const uint8_t* A, const uint8_t* Azm, const uint8_t* Azp,
                                           uint8_t* B, const TileGeom& g, int z, int lz_wrapped_z,
                                           const SiteTab& tab, int q, uint64_t key, uint64_t sweep,
                                           const PhiloxCtx& P, bool owned_plane, int& nacc,
                                           int& acc2) {
  (void)lz_wrapped_z;
  const uint4 zero4 = make_uint4(0, 0, 0, 0);
  if (g.active) {
    const int c = g.col;
    const uint32_t owned_full = owned_bytes(g.Wv - 16 * c);
    for (int r = 1 + g.row0; r < g.R - 1; r += g.rstep) {
      const int off = r * g.S + 16 + 16 * c;
      const uint8_t* p = A + off;
      const int y = wrap_row(g.y0 - 2 + r, g.ly);
      const uint32_t rho = (uint32_t)y + (uint32_t)g.ly * (uint32_t)z;
      const uint32_t chunk = rho * (uint32_t)g.pc + (uint32_t)((g.x0 >> 4) + c);
      const uint4 own = *(const uint4*)p;
      const uint4 up = *(const uint4*)(p - g.S);
      const uint4 dn = *(const uint4*)(p + g.S);
      const uint4 zmv = DIM == 3 ? *(const uint4*)(Azm + off) : zero4;
      const uint4 zpv = DIM == 3 ? *(const uint4*)(Azp + off) : zero4;
      const uint32_t wprev = *(const uint32_t*)(p - 4);
      const uint32_t wnext = *(const uint32_t*)(p + 16);
      const int bsh = ((y + z) & 1) << 3;
      const bool row_owned = owned_plane && r >= 2 && r < 2 + g.hv;
      const uint32_t owned = row_owned ? owned_full : 0u;
      if (ALG) {
        *(uint4*)(B + off) = update_chunk_hb<DIM>(own, up, dn, zmv, zpv, wprev, wnext, bsh, P, chunk, 0u,
                                                  tab, q, owned, nacc, acc2);
      } else {
        const uint4 rnd = philox_fast(P, chunk, 0u | (TAG_ACC << 1));
        const uint4 rpr = MODEL == POTTS ? philox_fast(P, chunk, 0u | (TAG_PROP << 1)) : zero4;
        *(uint4*)(B + off) = update_chunk<MODEL, DIM>(own, up, dn, zmv, zpv, wprev, wnext, bsh, rnd,
                                                      rpr, tab, q, key,
                                                      rho * (uint32_t)g.lx + (uint32_t)(g.x0 + 16 * c),
                                                      0u, sweep, owned, nacc, acc2);
      }
    }
  }
}

// Scalar halo sites of colour 0 (x0-1 and x0+Wv on rows [1, R-1)), A -> B.
template <int MODEL, int DIM, int ALG>
__device__ __forceinline__ void black_halo(const uint8_t* A, const uint8_t* Azm, const uint8_t* Azp,
                                           uint8_t* B, const TileGeom& g, int z,
                                           const SiteTab& tab, int q, uint64_t key,
                                           uint64_t sweep) {
  const int t = threadIdx.x;
  if (t < 2 * (g.R - 2)) {
    const int r = 1 + (t >> 1);
    const int pos = (t & 1) ? g.x0 + g.Wv : g.x0 - 1;
    const int y = wrap_row(g.y0 - 2 + r, g.ly);
    const int xr = pos < 0 ? pos + g.lx : (pos >= g.lx ? pos - g.lx : pos);
    const int off = r * g.S + 16 + (pos - g.x0);
    if (((xr + y + z) & 1) == 0)
      B[off] = (uint8_t)update_site<MODEL, DIM, ALG>((const int8_t*)A + off, g.S, (const int8_t*)Azm + off,
                                                (const int8_t*)Azp + off, xr, y, z, g.ly, g.lx, g.pc,
                                                tab, q, key, 0u, sweep);
    else
      B[off] = A[off];
  }
}

// Colour 1 on the tile rows of plane B, written to HBM; magnetisation or
// Potts histogram of the owned (finished) sites.
template <int MODEL, int DIM, int ALG>
__device__ __forceinline__ void white_pass(const uint8_t* B, const uint8_t* Bzm, const uint8_t* Bzp,
                                           const TileGeom& g, int z, const SiteTab& tab, int q,
                                           uint64_t key, uint64_t sweep, const PhiloxCtx& P,
                                           int8_t* dst, int& nacc, int& acc2, int& mag, int* cnt) {
  const uint4 zero4 = make_uint4(0, 0, 0, 0);
  if (!g.active) return;
  const int c = g.col;
  const uint32_t owned = owned_bytes(g.Wv - 16 * c);
  for (int r = 2 + g.row0; r < 2 + g.hv; r += g.rstep) {
    const int off = r * g.S + 16 + 16 * c;
    const uint8_t* p = B + off;
    const int y = wrap_row(g.y0 - 2 + r, g.ly);
    const uint32_t rho = (uint32_t)y + (uint32_t)g.ly * (uint32_t)z;
    const uint32_t chunk = rho * (uint32_t)g.pc + (uint32_t)((g.x0 >> 4) + c);
    const uint4 own = *(const uint4*)p;
    const uint4 up = *(const uint4*)(p - g.S);
    const uint4 dn = *(const uint4*)(p + g.S);
    const uint4 zmv = DIM == 3 ? *(const uint4*)(Bzm + off) : zero4;
    const uint4 zpv = DIM == 3 ? *(const uint4*)(Bzp + off) : zero4;
    const uint32_t wprev = *(const uint32_t*)(p - 4);
    const uint32_t wnext = *(const uint32_t*)(p + 16);
    const int bsh = ((1 + y + z) & 1) << 3;
    uint4 res;
    if (ALG) {
      res = update_chunk_hb<DIM>(own, up, dn, zmv, zpv, wprev, wnext, bsh, P, chunk, 1u, tab, q, owned,
                                 nacc, acc2);
    } else {
      const uint4 rnd = philox_fast(P, chunk, 1u | (TAG_ACC << 1));
      const uint4 rpr = MODEL == POTTS ? philox_fast(P, chunk, 1u | (TAG_PROP << 1)) : zero4;
      res = update_chunk<MODEL, DIM>(own, up, dn, zmv, zpv, wprev, wnext, bsh, rnd, rpr, tab, q, key,
                                     rho * (uint32_t)g.lx + (uint32_t)(g.x0 + 16 * c), 1u, sweep, owned,
                                     nacc, acc2);
    }
    const size_t doff = (size_t)rho * (size_t)g.pitch + g.x0 + 16 * c;
    if (GPUMC_IN(doff + 15, g.gbytes)) *(uint4*)(dst + doff) = res;
    const uint32_t w[4] = {res.x, res.y, res.z, res.w};
    if (owned == 0xFFFFu) {
      if (MODEL == ISING) {
#pragma unroll
        for (int k = 0; k < 4; ++k) mag = __dp4a((int)w[k], 0x01010101, mag);
      } else {
#pragma unroll
        for (int s = 0; s < kMaxPottsCounts; ++s) {
          if (s < q) {
            const uint32_t pat = 0x01010101u * (uint32_t)s;
            int n0 = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              const uint32_t x8 = w[k] ^ pat;
              const uint32_t t8 = (x8 & 0x7F7F7F7Fu) + 0x7F7F7F7Fu;
              n0 += __popc(~(t8 | x8 | 0x7F7F7F7Fu));
            }
            cnt[s] += n0;
          }
        }
      }
    } else {
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
              const uint32_t t8 = (x8 & 0x7F7F7F7Fu) + 0x7F7F7F7Fu;
              cnt[s] += __popc(~(t8 | x8 | 0x7F7F7F7Fu) & bm);
            }
          }
        }
      }
    }
  }
}

template <int MODEL, int DIM>
__device__ __forceinline__ void flush_accumulators(LatDesc* L, int nacc, int acc2, int mag,
                                                   const int* cnt, int q) {
  constexpr int zc = 2 * DIM;
  // Ising: dE = sum over accepted owned flips of 2(z - 2k) = 2 z n - 4 sum k;
  // Potts: dE = -sum d.
  long long v[3 + kMaxPottsCounts];
  v[0] = MODEL == ISING ? 2LL * zc * nacc - 4LL * acc2 : -(long long)acc2;
  v[1] = nacc;
  v[2] = mag;
#pragma unroll
  for (int s = 0; s < kMaxPottsCounts; ++s) v[3 + s] = MODEL == POTTS ? cnt[s] : 0;
  cta_sum(v);
  if (threadIdx.x == 0) {
    if (v[0]) atomic_add_i64(&L->acc.dE, v[0]);
    if (v[1]) atomic_add_i64(&L->acc.accepted, v[1]);
    if (MODEL == ISING) {
      if (v[2]) atomic_add_i64(&L->acc.mag, v[2]);
    } else {
      for (int s = 0; s < kMaxPottsCounts && s < q; ++s)
        if (v[3 + s]) atomic_add_i64(&L->acc.counts[s], v[3 + s]);
    }
  }
}

__device__ __forceinline__ void load_table(SiteTab& tab, const LatDesc* L, const GroupDesc* G) {
  const int label = G->label[L->replica];
  for (int i = threadIdx.x; i < G->n_cls; i += kThreads) {
    tab.head[i] = G->head[label * G->n_cls + i];
    tab.tail[i] = G->tail[label * G->n_cls + i];
  }
  if (threadIdx.x == 0) tab.jneg = G->J < 0.0 ? 1 : 0;
}

__device__ __forceinline__ TileGeom make_geom(const TileItem& t, const LatDesc* L) {
  TileGeom g;
  g.x0 = t.x0;
  g.y0 = t.y0;
  g.lx = L->lx;
  g.ly = L->ly;
  g.pitch = L->pitch;
  g.pc = L->pitch >> 4;
  g.W = t.cx * 16;
  g.S = g.W + 32;
  g.Wv = min(g.W, g.lx - t.x0);
  g.ncv = (g.Wv + 15) >> 4;
  g.hv = min(t.ty, g.ly - t.y0);
  g.R = g.hv + 4;
  g.rstep = kThreads / g.ncv;
  g.col = threadIdx.x % g.ncv;
  g.row0 = threadIdx.x / g.ncv;
  g.active = g.row0 < g.rstep;
  g.gbytes = (long long)L->pitch * L->ly * (L->dims == 3 ? L->lz : 1);
  return g;
}

template <int MODEL, int ALG>
__global__ void __launch_bounds__(kThreads)
    k_sweep_discrete_2d(const TileItem* __restrict__ tiles, LatDesc* __restrict__ lats,
                        GroupDesc* __restrict__ groups, LaunchCtl* __restrict__ ctl) {
  extern __shared__ __align__(16) uint8_t smem[];
  __shared__ SiteTab tab;
  const TileItem t = tiles[blockIdx.x];
  LatDesc* L = &lats[t.lat];
  const GroupDesc* G = &groups[L->group];
  const uint64_t sweep = L->sweep;
  if (sweep >= L->target) {  // finished lattice: nothing to do this launch
    group_epilogue(t.pad, lats, groups, ctl);
    return;
  }
  const uint64_t key = L->key;
  const int q = L->q;
  const int8_t* cur = (const int8_t*)L->buf[sweep & 1];
  int8_t* nxt = (int8_t*)L->buf[(sweep & 1) ^ 1];
  const TileGeom g = make_geom(t, L);
  uint8_t* A = smem;
  uint8_t* B = smem + g.R * g.S;
  stage_plane(A, cur, 0, g);
  const HaloBytes hb = fetch_halo(cur, 0, g);
  load_table(tab, L, G);
  const PhiloxCtx P = make_philox(key, sweep);
  cp_async_wait_all();
  __syncthreads();
  store_halo(A, hb, g);
  __syncthreads();
  int nacc = 0, acc2 = 0, mag = 0;
  int cnt[kMaxPottsCounts] = {0, 0, 0, 0, 0, 0, 0, 0};
  black_pass<MODEL, 2, ALG>(A, A, A, B, g, 0, 0, tab, q, key, sweep, P, true, nacc, acc2);
  __syncthreads();
  black_halo<MODEL, 2, ALG>(A, A, A, B, g, 0, tab, q, key, sweep);
  __syncthreads();
  white_pass<MODEL, 2, ALG>(B, B, B, g, 0, tab, q, key, sweep, P, nxt, nacc, acc2, mag, cnt);
  flush_accumulators<MODEL, 2>(L, nacc, acc2, mag, cnt, q);
  group_epilogue(t.pad, lats, groups, ctl);
}

// 3D: the tile is tile_cx chunks x tile_y rows in the xy plane, marched over
// tile_z planes.  Step s stages plane z0-2+s into the A ring, updates colour 0
// of plane z0-3+s (its z neighbours are still-old A planes) into the B ring,
// and colour 1 of plane z0-4+s from the B ring (its z neighbours have
// finished colour 0) to HBM.
template <int MODEL, int ALG>
__global__ void __launch_bounds__(kThreads)
    k_sweep_discrete_3d(const TileItem* __restrict__ tiles, LatDesc* __restrict__ lats,
                        GroupDesc* __restrict__ groups, LaunchCtl* __restrict__ ctl) {
  extern __shared__ __align__(16) uint8_t smem[];
  __shared__ SiteTab tab;
  const TileItem t = tiles[blockIdx.x];
  LatDesc* L = &lats[t.lat];
  const GroupDesc* G = &groups[L->group];
  const uint64_t sweep = L->sweep;
  if (sweep >= L->target) {
    group_epilogue(t.pad, lats, groups, ctl);
    return;
  }
  const uint64_t key = L->key;
  const int q = L->q, lz = L->lz;
  const int8_t* cur = (const int8_t*)L->buf[sweep & 1];
  int8_t* nxt = (int8_t*)L->buf[(sweep & 1) ^ 1];
  const TileGeom g = make_geom(t, L);
  const int dv = min(t.tz, lz - t.z0);
  const int pb = g.R * g.S;  // bytes per plane
  uint8_t* Aring = smem;          // 3 planes
  uint8_t* Bring = smem + 3 * pb; // 3 planes
  load_table(tab, L, G);
  const PhiloxCtx P = make_philox(key, sweep);
  int nacc = 0, acc2 = 0, mag = 0;
  int cnt[kMaxPottsCounts] = {0, 0, 0, 0, 0, 0, 0, 0};
  auto slot = [](int v) { return ((v % 3) + 3) % 3; };
  for (int s = 0; s < dv + 4; ++s) {
    const int zl = t.z0 - 2 + s;
    const int zlw = zl < 0 ? zl + lz : (zl >= lz ? zl - lz : zl);
    uint8_t* Al = Aring + slot(s) * pb;
    stage_plane(Al, cur, zlw, g);
    const HaloBytes hb = fetch_halo(cur, zlw, g);
    cp_async_wait_all();
    __syncthreads();
    store_halo(Al, hb, g);
    __syncthreads();
    if (s >= 2) {
      const int zb = zl - 1;
      const int zbw = zb < 0 ? zb + lz : (zb >= lz ? zb - lz : zb);
      const uint8_t* Ab = Aring + slot(s - 1) * pb;
      const uint8_t* Am = Aring + slot(s - 2) * pb;
      uint8_t* Bb = Bring + slot(s - 1) * pb;
      const bool owned_plane = zb >= t.z0 && zb < t.z0 + dv;
      black_pass<MODEL, 3, ALG>(Ab, Am, Al, Bb, g, zbw, 0, tab, q, key, sweep, P, owned_plane, nacc, acc2);
      __syncthreads();
      black_halo<MODEL, 3, ALG>(Ab, Am, Al, Bb, g, zbw, tab, q, key, sweep);
      __syncthreads();
    }
    if (s >= 4) {
      const int zw = zl - 2;
      const int zww = zw < 0 ? zw + lz : (zw >= lz ? zw - lz : zw);
      white_pass<MODEL, 3, ALG>(Bring + slot(s - 2) * pb, Bring + slot(s - 3) * pb, Bring + slot(s - 1) * pb,
                           g, zww, tab, q, key, sweep, P, nxt, nacc, acc2, mag, cnt);
    }
    __syncthreads();  // the next stage overwrites A and B slots read in this step
  }
  flush_accumulators<MODEL, 3>(L, nacc, acc2, mag, cnt, q);
  group_epilogue(t.pad, lats, groups, ctl);
}

template __global__ void k_sweep_discrete_2d<POTTS, 0>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template __global__ void k_sweep_discrete_3d<POTTS, 0>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template __global__ void k_sweep_discrete_2d<POTTS, 1>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template __global__ void k_sweep_discrete_3d<POTTS, 1>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);

GPUMC_BOUNDS_MODULE(sweep_discrete)

}  // namespace gpumc
