// Checkerboard sweep for O(3) Heisenberg spins (float32 unit vectors, three
// component planes) on periodic square and cubic lattices.
//
// The O(3) update costs ~200 arithmetic instructions per attempt against 24 B
// of compulsory traffic, so it is bound by instruction throughput, not HBM.
// It therefore runs in place as two launches per sweep (colour 0, then colour
// 1), one thread per site: a colour pass reads only the other colour, whose
// values stay fixed during the pass, so no tiles, halos or barriers are needed
// and neighbour reads are served by L1/L2.  The colour-1 launch ends with the
// sweep epilogue.
//
// Energy: on the bipartite periodic lattice every bond has exactly one
// colour-1 end, so the colour-1 pass sums s . h over its sites with their
// final spins (fp64 neighbour sums of the fp32 components, exact products)
// and the epilogue sets E = -J times that sum: the energy after each sweep is
// computed afresh rather than carried by a cache of per-move changes, so it
// cannot drift, and the colour-0 pass does no fp64 work.
//
// Proposal: a uniform point on the spherical cap of half-angle alpha around
// the current spin (w = 1 - cos(alpha) stored per lattice, adapted toward 50 %
// acceptance during thermalisation only, mirroring the adaptation contract of
// the reference's OPSSStrategy, CMC.rs/src/lattice/proposal.rs:72-167).  The
// cap proposal is symmetric, so acceptance is min(1, exp(-beta dE)) with
// dE = -J (s' - s) . h, h the sum of the neighbour spins
// (ONModel::bond_energy, CMC.rs/src/lattice/models.rs:440-452).
//
// Other proposals of the Metropolis step (ALG = 2, 3): the reference's
// StandardStrategy (an independent uniform unit vector, ONModel::propose_from,
// CMC.rs/src/lattice/proposal.rs:45-63; here z = 1 - 2u, phi from word 1, one
// Newton renormalisation) and OPSSStrategy (proposal.rs:72-167: a rotation by
// theta uniform in (-sigma, sigma) in a random coordinate plane, then
// normalised; sigma adapted during thermalisation by exp(0.08 (rate - 0.5)),
// clamped to [1e-4, pi]).  OPSS takes the plane floor(3 w0 / 2^32) of
// {(x,y), (y,z), (z,x)} (rotating in (j,i) by theta is rotating in (i,j) by
// -theta, so unordered planes with a symmetric angle are the reference's
// ordered pairs) and theta = sigma (2u - 1), u from word 1, its sine and
// cosine by the engine's own turn polynomials; sigma is the lattice's `omc`.
//
// Heat bath (ALG = 1; ContinuousHeatBathCore, CMC.rs/src/algorithms/
// heat_bath.rs:75-134, with ContinuousHeatBathable for ONModel<3>,
// CMC.rs/src/lattice/models.rs:617-663): the new spin is drawn from
// p(s) ~ exp(beta f . s), f = J h the local field, by inverting the CDF of
// w = 1 - cos(theta) around f: w = -ln(1 - v (1 - exp(-2 kappa))) / kappa,
// kappa = beta |f|, v uniform in [0, 1), phi uniform; below kappa = 2^-20 the
// draw is uniform on the sphere (w = 2v), as the reference's kappa < 1e-12
// branch.  The sample is placed with the same basis and renormalisation as
// the cap proposal.  Draws come from tag TAG_O3HB (word 0: v, word 1: phi);
// there is no cone to adapt, and "accepted" counts the sites that changed.
//
// Every fp32 operation is an explicitly rounded intrinsic and exp / log /
// sin / cos are the engine's own polynomials, so a CPU replay in the same
// operation order reproduces the device trajectory bit for bit.
#include "device_common.cuh"
#include "epilogue.cuh"

namespace gpumc {

// Cap proposal around a = (ax, ay, az): local sample v = (st cos phi,
// st sin phi, ct) mapped through the orthonormal basis {e1, e2, a} of Duff,
// Burgess, Christensen, Hery, Kensler, Liani, Villemin, "Building an
// Orthonormal Basis, Revisited" (JCGT 6(1), 2017): with s = sign(az),
// k = -1 / (s + az), b = ax ay k,
//   e1 = (1 + s ax^2 k, s b, -s ax),  e2 = (b, s + ay^2 k, -ay),
// one division and no square root, never singular since |s + az| >= 1.  The
// result is renormalised by one Newton step of 1/sqrt(n2) from 1
// (f = 1.5 - 0.5 n2; n2 is within a few ulp of 1, so f is exact to fp32).
__device__ __forceinline__ void o3_place(float ax, float ay, float az, float ct, float st, float cp,
                                         float sp, float& px, float& py, float& pz) {
  const float vx = fmul(st, cp), vy = fmul(st, sp);
  const float sg = az >= 0.0f ? 1.0f : -1.0f;
  const float k = fdiv(-1.0f, fadd(sg, az));
  const float b = fmul(fmul(ax, ay), k);
  const float e1x = fadd(1.0f, fmul(fmul(sg, fmul(ax, ax)), k));
  const float e1y = fmul(sg, b);
  const float e1z = -fmul(sg, ax);
  const float e2x = b;
  const float e2y = fadd(sg, fmul(fmul(ay, ay), k));
  const float e2z = -ay;
  px = fadd(fadd(fmul(vx, e1x), fmul(vy, e2x)), fmul(ct, ax));
  py = fadd(fadd(fmul(vx, e1y), fmul(vy, e2y)), fmul(ct, ay));
  pz = fadd(fadd(fmul(vx, e1z), fmul(vy, e2z)), fmul(ct, az));
  const float n2 = fadd(fadd(fmul(px, px), fmul(py, py)), fmul(pz, pz));
  const float f = fsub(1.5f, fmul(0.5f, n2));
  px = fmul(px, f);
  py = fmul(py, f);
  pz = fmul(pz, f);
}

// Renormalisation by one Newton step of 1/sqrt(n2) from 1.
__device__ __forceinline__ void o3_renorm(float& px, float& py, float& pz) {
  const float n2 = fadd(fadd(fmul(px, px), fmul(py, py)), fmul(pz, pz));
  const float f = fsub(1.5f, fmul(0.5f, n2));
  px = fmul(px, f);
  py = fmul(py, f);
  pz = fmul(pz, f);
}

// Metropolis step: PROP 0 cap proposal (w = 1 - cos(alpha) in omc), 1
// uniform unit vector, 2 OPSS plane rotation (sigma in omc).  Returns the
// decision and the proposed spin and its fp32 dE.
template <int PROP>
__device__ __forceinline__ bool o3_update(float ax, float ay, float az, float hx, float hy,
                                          float hz, uint4 o, float omc, float mJ, float beta,
                                          float& nx, float& ny, float& nz, float& dE) {
  float px, py, pz;
  if (PROP == 0) {
    const float w = fmul(fmul((float)(o.x >> 8), 0x1p-24f), omc);
    const float ct = fsub(1.0f, w);
    const float st = fsqrt(fmul(w, fsub(2.0f, w)));
    float cp, sp;
    sincos_turn(o.y, cp, sp);
    o3_place(ax, ay, az, ct, st, cp, sp, px, py, pz);
  } else if (PROP == 1) {
    pz = fsub(1.0f, fmul(2.0f, fmul((float)(o.x >> 8), 0x1p-24f)));
    const float rho = fsqrt(fmul(fsub(1.0f, pz), fadd(1.0f, pz)));
    float cp, sp;
    sincos_turn(o.y, cp, sp);
    px = fmul(rho, cp);
    py = fmul(rho, sp);
    o3_renorm(px, py, pz);
  } else {
    const uint32_t plane = __umulhi(o.x, 3u);
    const float u = fmul(fadd((float)(o.y >> 8), 0.5f), 0x1p-24f);
    const float theta = fmul(omc, fsub(fmul(2.0f, u), 1.0f));
    // theta as a signed fraction of a turn, 32-bit fixed point
    const float turns = fmul(theta, 0x1.45f306p-3f);  // 1 / (2 pi)
    const uint32_t tu = (uint32_t)(long long)__float2ll_rn(fmul(turns, 0x1p32f));
    float c, s;
    sincos_turn(tu, c, s);
    const float a0 = plane == 0 ? ax : (plane == 1 ? ay : az);
    const float a1 = plane == 0 ? ay : (plane == 1 ? az : ax);
    const float r0 = fsub(fmul(c, a0), fmul(s, a1)), r1 = fadd(fmul(s, a0), fmul(c, a1));
    px = plane == 0 ? r0 : (plane == 1 ? ax : r1);
    py = plane == 0 ? r1 : (plane == 1 ? r0 : ay);
    pz = plane == 0 ? az : (plane == 1 ? r1 : r0);
    o3_renorm(px, py, pz);
  }
  const float dot =
      fadd(fadd(fmul(fsub(px, ax), hx), fmul(fsub(py, ay), hy)), fmul(fsub(pz, az), hz));
  const float de = fmul(mJ, dot);
  bool ok;
  if (de <= 0.0f) {
    ok = true;
  } else {
    const float p = exp_neg(-fmul(beta, de));
    const float u = fmul(fadd((float)(o.z >> 8), 0.5f), 0x1p-24f);
    ok = u < p;
  }
  nx = px;
  ny = py;
  nz = pz;
  dE = de;
  return ok;
}

// Heat-bath draw of a site with neighbour sum h (fp32) under coupling Jf.
__device__ __forceinline__ void o3_heat_bath(float hx, float hy, float hz, uint4 o, float Jf, float beta,
                                             float& nx, float& ny, float& nz) {
  const float fx = fmul(Jf, hx), fy = fmul(Jf, hy), fz = fmul(Jf, hz);
  const float nrm = fsqrt(fadd(fadd(fmul(fx, fx), fmul(fy, fy)), fmul(fz, fz)));
  const float kap = fmul(beta, nrm);
  const float v = fmul((float)(o.x >> 8), 0x1p-24f);
  float w, ax = 0.0f, ay = 0.0f, az = 1.0f;
  if (!(kap >= 0x1p-20f)) {
    w = fmul(2.0f, v);
  } else {
    const float y = fmul(v, one_minus_exp_neg(fmul(2.0f, kap)));
    w = fdiv(-log_one_minus(y), kap);
    if (w > 2.0f) w = 2.0f;
    ax = fdiv(fx, nrm);
    ay = fdiv(fy, nrm);
    az = fdiv(fz, nrm);
  }
  const float ct = fsub(1.0f, w);
  const float st = fsqrt(fmul(w, fsub(2.0f, w)));
  float cp, sp;
  sincos_turn(o.y, cp, sp);
  o3_place(ax, ay, az, ct, st, cp, sp, nx, ny, nz);
}

// Philox4x32-10 of counter (site, colour | TAG_O3 << 1, sweep) with the
// sweep-uniform part of round 1 precomputed; the round keys are bumped on the
// fly (two adds per round instead of twenty live registers: resident warps
// matter more here), and each round multiply is one 32x32->64 wide product.
struct O3Philox {
  uint32_t a, b, c, k0, k1;
};
__device__ __forceinline__ O3Philox make_o3_philox(uint64_t key, uint64_t sweep, uint32_t ctrl) {
  O3Philox P;
  P.k0 = (uint32_t)key;
  P.k1 = (uint32_t)(key >> 32);
  const uint32_t c2 = (uint32_t)sweep, c3 = (uint32_t)(sweep >> 32);
  P.a = __umulhi(0xCD9E8D57u, c2) ^ P.k0 ^ ctrl;
  P.b = 0xCD9E8D57u * c2;
  P.c = c3 ^ P.k1;
  return P;
}
__device__ __forceinline__ uint4 o3_philox(const O3Philox& P, uint32_t index) {
  const uint64_t p00 = (uint64_t)0xD2511F53u * index;
  uint4 c = make_uint4(P.a, P.b, (uint32_t)(p00 >> 32) ^ P.c, (uint32_t)p00);
  uint32_t k0 = P.k0, k1 = P.k1;
#pragma unroll
  for (int r = 1; r < 10; ++r) {
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
    const uint64_t p0 = (uint64_t)0xD2511F53u * c.x;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c.z;
    c = make_uint4((uint32_t)(p1 >> 32) ^ c.y ^ k0, (uint32_t)p1, (uint32_t)(p0 >> 32) ^ c.w ^ k1,
                   (uint32_t)p0);
  }
  return c;
}

// One site of a colour pass: its own spin and the fp32 sum of its
// neighbours (the decision), plus, in the colour-1 pass, their exact fp64 sum
// (the sweep's bond sum), loaded before any update of the thread's sites so
// that the loads of two sites overlap.
struct O3Site {
  uint32_t me, site;
  float ax, ay, az, hx, hy, hz;
  double hxd, hyd, hzd;
};

template <int DIM, bool EXACT>
__device__ __forceinline__ void o3_load_site(O3Site& q, const float* S, const float* S1, const float* S2,
                                             int x, int y, int z, int lx, int ly, int lz, int pitch) {
  const uint32_t rowoff = ((uint32_t)z * ly + y) * (uint32_t)pitch;
  const int ym = y ? y - 1 : ly - 1, yp = y + 1 < ly ? y + 1 : 0;
  const int xm = x ? x - 1 : lx - 1, xp = x + 1 < lx ? x + 1 : 0;
  uint32_t zmo = 0, zpo = 0;
  if (DIM == 3) {
    const int zm = z ? z - 1 : lz - 1, zp = z + 1 < lz ? z + 1 : 0;
    zmo = ((uint32_t)zm * ly + y) * (uint32_t)pitch + x;
    zpo = ((uint32_t)zp * ly + y) * (uint32_t)pitch + x;
  }
  // neighbour sum in the fixed order x-1, x+1, y-1, y+1, z-1, z+1
  const uint32_t nb[6] = {rowoff + xm, rowoff + xp, ((uint32_t)z * ly + ym) * (uint32_t)pitch + x,
                          ((uint32_t)z * ly + yp) * (uint32_t)pitch + x, zmo, zpo};
  float hx = __ldg(S + nb[0]), hy = __ldg(S1 + nb[0]), hz = __ldg(S2 + nb[0]);
  double hxd = 0.0, hyd = 0.0, hzd = 0.0;
  if (EXACT) {
    hxd = (double)hx;
    hyd = (double)hy;
    hzd = (double)hz;
  }
#pragma unroll
  for (int i = 1; i < 2 * DIM; ++i) {
    const float vx = __ldg(S + nb[i]), vy = __ldg(S1 + nb[i]), vz = __ldg(S2 + nb[i]);
    hx = fadd(hx, vx);
    hy = fadd(hy, vy);
    hz = fadd(hz, vz);
    if (EXACT) {
      hxd += (double)vx;
      hyd += (double)vy;
      hzd += (double)vz;
    }
  }
  q.me = rowoff + x;
  q.ax = S[q.me];
  q.ay = S1[q.me];
  q.az = S2[q.me];
  q.hx = hx;
  q.hy = hy;
  q.hz = hz;
  q.hxd = hxd;
  q.hyd = hyd;
  q.hzd = hzd;
  q.site = (uint32_t)((size_t)(z * ly + y) * lx + x);
}

// One colour pass over a tile of full rows (y0 .. y0+hv-1, planes z0 ..
// z0+dv-1), one thread per site of the colour.
template <int DIM, int COLOUR, int ALG>
__global__ void __launch_bounds__(kThreads, 4)
    k_sweep_o3(const TileItem* __restrict__ tiles, LatDesc* __restrict__ lats,
               GroupDesc* __restrict__ groups, LaunchCtl* __restrict__ ctl) {
  const TileItem t = tiles[blockIdx.x];
  LatDesc* L = &lats[t.lat];
  const GroupDesc* G = &groups[L->group];
  const uint64_t sweep = L->sweep;
  if (sweep >= L->target) {
    if (COLOUR == 1) launch_epilogue(lats, groups, ctl);
    return;
  }
  const int lx = L->lx, ly = L->ly, lz = DIM == 3 ? L->lz : 1, pitch = L->pitch;
  const uint32_t cs = (uint32_t)pitch * ly * lz;  // component plane stride (< 2^32 elements)
  float* S = (float*)L->buf[0];  // in place; component planes S, S1, S2
  float* S1 = S + (size_t)cs;
  float* S2 = S + 2 * (size_t)cs;
  const float* Sr = S;
  const float* Sr1 = S1;
  const float* Sr2 = S2;
  const int label = G->label[L->replica];
  const float beta = G->betas_f[label];
  const float mJ = -G->Jf;
  const float omc = L->omc;
  const O3Philox P = make_o3_philox(L->key, sweep, (uint32_t)COLOUR | ((ALG == 1 ? TAG_O3HB : TAG_O3) << 1));
  const int hv = min(t.ty, ly - t.y0);
  const int dv = DIM == 3 ? min(t.tz, lz - t.z0) : 1;
  const int half = lx >> 1;
  const int rows = hv * dv;
  // thread mapping: fixed column (or column stride) per thread, rows strided
  int col0, cstep, r0, rstep;
  if (half >= kThreads) {
    col0 = threadIdx.x;
    cstep = kThreads;
    r0 = 0;
    rstep = 1;
  } else {
    col0 = threadIdx.x % half;
    cstep = half;
    r0 = threadIdx.x / half;
    rstep = kThreads / half;
  }
  double eb = 0.0, mx = 0.0, my = 0.0, mz = 0.0;  // eb: colour 1's sum of s . h
  int nacc = 0;
  // this thread's sites, row-major: rows r0, r0 + rstep, ... of the tile's
  // rows (y fastest, then z), columns col0, col0 + cstep, ...; taken two at a
  // time, with the (row, column) cursor advanced without divisions
  const int nc = (r0 < rstep && col0 < half) ? (half - col0 + cstep - 1) / cstep : 0;
  const int nr = r0 < rstep ? (rows - r0 + rstep - 1) / rstep : 0;
  const int n_items = nc * nr;
  int cy = t.y0 + (DIM == 3 ? r0 % hv : r0), cz = DIM == 3 ? t.z0 + r0 / hv : 0, cc = 0;
  const int ry = DIM == 3 ? rstep % hv : rstep, rz = DIM == 3 ? rstep / hv : 0;
  auto next_site = [&](int& x, int& y, int& z) {
    y = cy;
    z = cz;
    x = 2 * (col0 + cc * cstep) + ((y + z + COLOUR) & 1);
    if (++cc == nc) {
      cc = 0;
      cy += ry;
      cz += rz;
      if (cy >= t.y0 + hv) {
        cy -= hv;
        cz += 1;
      }
    }
  };
  auto update = [&](const O3Site& q) {
    float nx, ny, nz, de;
    bool ok;
    if (ALG == 1) {
      o3_heat_bath(q.hx, q.hy, q.hz, o3_philox(P, q.site), -mJ, beta, nx, ny, nz);
      ok = (nx != q.ax) | (ny != q.ay) | (nz != q.az);
    } else {
      ok = o3_update<ALG == 2 ? 1 : (ALG == 3 ? 2 : 0)>(q.ax, q.ay, q.az, q.hx, q.hy, q.hz, o3_philox(P, q.site),
                                                         omc, mJ, beta, nx, ny, nz, de);
    }
    float fx = q.ax, fy = q.ay, fz = q.az;
    if (ok) {
      ++nacc;
      fx = nx;
      fy = ny;
      fz = nz;
      S[q.me] = fx;
      S1[q.me] = fy;
      S2[q.me] = fz;
    }
    mx += (double)fx;
    my += (double)fy;
    mz += (double)fz;
    // every bond has one colour-1 end: the sweep's energy is -J times the
    // colour-1 pass's sum of s . h over the final spins (exact products of
    // fp32 components and fp64 neighbour sums)
    if (COLOUR == 1) eb += ((double)fx * q.hxd + (double)fy * q.hyd) + (double)fz * q.hzd;
  };
  for (int k = 0; k < n_items; k += 2) {
    int x, y, z;
    O3Site qa, qb;
    next_site(x, y, z);
    o3_load_site<DIM, COLOUR == 1>(qa, Sr, Sr1, Sr2, x, y, z, lx, ly, lz, pitch);
    const bool two = k + 1 < n_items;
    if (two) {
      next_site(x, y, z);
      o3_load_site<DIM, COLOUR == 1>(qb, Sr, Sr1, Sr2, x, y, z, lx, ly, lz, pitch);
    }
    update(qa);
    if (two) update(qb);
  }
  double v[4] = {eb, mx, my, mz};
  long long n[1] = {nacc};
  cta_sum(v);
  cta_sum(n);
  if (threadIdx.x == 0) {
    if (COLOUR == 1) {
      atomicAdd(&L->acc.ebond, v[0]);
      L->acc.fresh = 1;
    }
    atomicAdd(&L->acc.mx, v[1]);
    atomicAdd(&L->acc.my, v[2]);
    atomicAdd(&L->acc.mz, v[3]);
    if (n[0]) atomic_add_i64(&L->acc.accepted, n[0]);
  }
  if (COLOUR == 1) launch_epilogue(lats, groups, ctl);
}

// ---------------------------------------------------------------------------
// 3D colour pass marched along z through a ring of four shared-memory planes.
//
// A tile is whole rows y0 .. y0+hv-1 of planes z0 .. z0+dv-1.  Each plane the
// tile touches (z0-1 .. z0+dv) is copied once, rows y0-1 .. y0+hv with all
// three components, by 16-byte cp.async into a ring slot, and serves as the
// z-1, z and z+1 plane of three consecutive steps; the copy of plane z+2 is in
// flight while plane z is computed.  Every neighbour read is then a
// shared-memory read.  The pass reads only the other colour's values (and its
// own sites' old values, which only this tile writes), so copying planes that
// other tiles update in place is race-free.  The site arithmetic and its
// operation order are those of k_sweep_o3.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void o3_cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

// Colour 1 also carries the sweep epilogue's shared memory, so three CTAs
// fit an SM: its register budget is that of three CTAs (no spills of the fp64
// neighbour sums).
template <int COLOUR, int ALG>
__global__ void __launch_bounds__(kThreads, COLOUR == 1 ? 3 : 4)
    k_sweep_o3_march(const TileItem* __restrict__ tiles, LatDesc* __restrict__ lats,
                     GroupDesc* __restrict__ groups, LaunchCtl* __restrict__ ctl) {
  extern __shared__ __align__(16) float osm[];
  const TileItem t = tiles[blockIdx.x];
  LatDesc* L = &lats[t.lat];
  const GroupDesc* G = &groups[L->group];
  const uint64_t sweep = L->sweep;
  if (sweep >= L->target) {
    if (COLOUR == 1) launch_epilogue(lats, groups, ctl);
    return;
  }
  const int lx = L->lx, ly = L->ly, lz = L->lz, pitch = L->pitch;
  const size_t cs = (size_t)pitch * ly * lz;  // component plane stride
  float* S = (float*)L->buf[0];
  const int label = G->label[L->replica];
  const float beta = G->betas_f[label];
  const float mJ = -G->Jf;
  const float omc = L->omc;
  const O3Philox P = make_o3_philox(L->key, sweep, (uint32_t)COLOUR | ((ALG == 1 ? TAG_O3HB : TAG_O3) << 1));
  const int hv = min(t.ty, ly - t.y0);
  const int dv = min(t.tz, lz - t.z0);
  const int RW = hv + 2;                    // slot rows: y0-1 .. y0+hv
  const int cstr = RW * pitch;              // floats per component in a slot
  const int slot = 3 * cstr;                // floats per ring slot
  const int nvec = pitch >> 2;              // 16-byte chunks per row
  // Plane copies: thread k copies chunks k, k + kThreads, ... of the
  // 3 x RW x nvec chunks (component c, slot row r, chunk v), walked by a
  // division-free cursor that advances kThreads chunks per step.
  const int cv0 = threadIdx.x % nvec, ccr0 = threadIdx.x / nvec;
  const int cc0 = ccr0 / RW, cr0 = ccr0 - cc0 * RW;
  const int step_v = kThreads % nvec, step_r = kThreads / nvec;
  float* S1 = S + cs;
  float* S2 = S + 2 * cs;
  auto copy_plane = [&](int sl, int z) {
    const int zz = z < 0 ? z + lz : (z >= lz ? z - lz : z);
    float* dst = osm + sl * slot;
    const float* src = S + (size_t)zz * ly * pitch;
    int v = cv0, r = cr0, c = cc0;
    while (c < 3) {
      int y = t.y0 - 1 + r;
      y = y < 0 ? y + ly : (y >= ly ? y - ly : y);
      o3_cp_async16(dst + c * cstr + r * pitch + 4 * v, src + c * cs + y * pitch + 4 * v);
      v += step_v;
      r += step_r;
      if (v >= nvec) {
        v -= nvec;
        ++r;
      }
      while (r >= RW) {
        r -= RW;
        ++c;
      }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  double eb = 0.0, mx = 0.0, my = 0.0, mz = 0.0;  // eb: colour 1's sum of s . h
  int nacc = 0;
  const int half = lx >> 1;
  const int n_items = hv * half;  // colour sites of the tile's rows in one plane
  const int dr = kThreads / half, dj = kThreads - dr * half;  // cursor step of kThreads items
  auto update = [&](const O3Site& q) {
    float nx, ny, nz, de;
    bool ok;
    if (ALG == 1) {
      o3_heat_bath(q.hx, q.hy, q.hz, o3_philox(P, q.site), -mJ, beta, nx, ny, nz);
      ok = (nx != q.ax) | (ny != q.ay) | (nz != q.az);
    } else {
      ok = o3_update<ALG == 2 ? 1 : (ALG == 3 ? 2 : 0)>(q.ax, q.ay, q.az, q.hx, q.hy, q.hz, o3_philox(P, q.site),
                                                         omc, mJ, beta, nx, ny, nz, de);
    }
    float fx = q.ax, fy = q.ay, fz = q.az;
    if (ok) {
      ++nacc;
      fx = nx;
      fy = ny;
      fz = nz;
      S[q.me] = fx;
      S1[q.me] = fy;
      S2[q.me] = fz;
    }
    mx += (double)fx;
    my += (double)fy;
    mz += (double)fz;
    if (COLOUR == 1) eb += ((double)fx * q.hxd + (double)fy * q.hyd) + (double)fz * q.hzd;
  };
  copy_plane(0, t.z0 - 1);
  copy_plane(1, t.z0);
  copy_plane(2, t.z0 + 1);
  for (int k = 0; k < dv; ++k) {
    const int z = t.z0 + k;
    // plane z+2 (needed as z+1 of the next step) into the slot freed by the
    // previous step; an empty group keeps the count when it is not needed
    if (k + 1 < dv) {
      copy_plane((k + 3) & 3, z + 2);
    } else {
      asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");  // planes z-1, z, z+1 landed
    __syncthreads();
    const float* pm = osm + (k & 3) * slot;
    const float* pc = osm + ((k + 1) & 3) * slot;
    const float* pp = osm + ((k + 2) & 3) * slot;
    auto load_site = [&](O3Site& q, int rl, int j) {  // local owned row, colour column
      const int y = t.y0 + rl;
      const int x = 2 * j + ((y + z + COLOUR) & 1);
      const int xm = x ? x - 1 : lx - 1, xp = x + 1 < lx ? x + 1 : 0;
      const int oc = (rl + 1) * pitch;  // slot row of y
      // neighbour order x-1, x+1, y-1, y+1, z-1, z+1 (as k_sweep_o3)
      float h[3];
      double hd[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float* P = pc + c * cstr;
        const float v0 = P[oc + xm], v1 = P[oc + xp];
        const float v2 = P[oc - pitch + x];
        const float v3 = P[oc + pitch + x];
        const float v4 = pm[c * cstr + oc + x];
        const float v5 = pp[c * cstr + oc + x];
        h[c] = fadd(fadd(fadd(fadd(fadd(v0, v1), v2), v3), v4), v5);
        hd[c] = COLOUR == 1
                    ? (((((double)v0 + (double)v1) + (double)v2) + (double)v3) + (double)v4) + (double)v5
                    : 0.0;
      }
      q.ax = pc[oc + x];
      q.ay = pc[cstr + oc + x];
      q.az = pc[2 * cstr + oc + x];
      q.hx = h[0];
      q.hy = h[1];
      q.hz = h[2];
      q.hxd = hd[0];
      q.hyd = hd[1];
      q.hzd = hd[2];
      // 32-bit index arithmetic: the same values as the 64-bit products
      // truncated to the 32-bit fields
      q.me = ((uint32_t)z * (uint32_t)ly + (uint32_t)y) * (uint32_t)pitch + (uint32_t)x;
      q.site = ((uint32_t)z * (uint32_t)ly + (uint32_t)y) * (uint32_t)lx + (uint32_t)x;
    };
    // items i = threadIdx.x, + kThreads, ... as (row, column) cursors
    int ra = threadIdx.x / half, ja = threadIdx.x - ra * half;
    for (int i = threadIdx.x; i < n_items; i += 2 * kThreads) {
      O3Site qa, qb;
      load_site(qa, ra, ja);
      int rb = ra + dr, jb = ja + dj;
      if (jb >= half) {
        jb -= half;
        rb += 1;
      }
      const bool two = i + kThreads < n_items;
      if (two) load_site(qb, rb, jb);
      update(qa);
      if (two) update(qb);
      ra = rb + dr;
      ja = jb + dj;
      if (ja >= half) {
        ja -= half;
        ra += 1;
      }
    }
    __syncthreads();  // the next copy overwrites the z-1 slot read above
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  double v[4] = {eb, mx, my, mz};
  long long n[1] = {nacc};
  cta_sum(v);
  cta_sum(n);
  if (threadIdx.x == 0) {
    if (COLOUR == 1) {
      atomicAdd(&L->acc.ebond, v[0]);
      L->acc.fresh = 1;
    }
    atomicAdd(&L->acc.mx, v[1]);
    atomicAdd(&L->acc.my, v[2]);
    atomicAdd(&L->acc.mz, v[3]);
    if (n[0]) atomic_add_i64(&L->acc.accepted, n[0]);
  }
  if (COLOUR == 1) launch_epilogue(lats, groups, ctl);
}

#define O3_INSTANTIATE(ALG)                                                                          \
  template __global__ void k_sweep_o3_march<0, ALG>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*); \
  template __global__ void k_sweep_o3_march<1, ALG>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*); \
  template __global__ void k_sweep_o3<2, 0, ALG>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);    \
  template __global__ void k_sweep_o3<2, 1, ALG>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);    \
  template __global__ void k_sweep_o3<3, 0, ALG>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);    \
  template __global__ void k_sweep_o3<3, 1, ALG>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
O3_INSTANTIATE(0)
O3_INSTANTIATE(1)
O3_INSTANTIATE(2)
O3_INSTANTIATE(3)

}  // namespace gpumc
