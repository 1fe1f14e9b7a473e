// Checkerboard sweep for O(3) Heisenberg spins (float32 unit vectors, three
// component planes) on periodic square and cubic lattices.
//
// The O(3) update costs some 245-255 instructions per site against 24 B of
// compulsory traffic, so it is bound by instruction issue and dependency
// latency, not HBM.  It runs in place as two launches per sweep (colour 0,
// then colour 1): a colour pass reads only the other colour, whose values
// stay fixed during the pass, so tiles need no coordination.  3D lattices are
// marched along z through shared-memory planes (k_sweep_o3_march); 2D
// lattices and 3D lattices too small for the march use k_sweep_o3, whose
// neighbour reads are served by L1/L2.  Both take the sites of a colour in
// pairs.  The colour-1 launch ends with the sweep epilogue.
//
// Observables: on the bipartite periodic lattice every bond has exactly one
// colour-1 end, so the colour-1 pass sums s . h over its sites with their
// final spins and the epilogue sets E = -J times that sum: the energy after
// each sweep is computed afresh rather than carried by a cache of per-move
// changes, so it cannot drift.  The sum is taken in fixed point: each site
// adds rint(2^19 s . h) (the fp32 dot with its fp32 neighbour sum h, the
// decision's h) to an integer accumulator, and the magnetisation components
// add rint(2^21 s_c); integer sums do not depend on the order in which
// threads and CTAs combine them, so the records are bit-identical to the CPU
// replay.  Accuracy: a few 1e-7 per bond from the fp32 products, i.e. the
// precision of the fp32 spins themselves (relative 1e-9 on the total energy
// of a 64^3 lattice).
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
// ALG = 4, the fast cap: the cap proposal on the same draws with the
// hardware approximations of sqrt, reciprocal, sin / cos and exp in place of
// the exactly rounded operations and the engine's polynomials (about 40
// instructions per site fewer).  Its spins follow the exact cap's to a few
// 1e-7 and its decisions differ only where a uniform falls within about 1e-6
// of its acceptance probability, so its parity is float32 tolerance and
// statistics, not bit identity with the CPU replay.
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
// (Word 0 and word 1 here are a site's first and second draw.)
//
// Random draws: one Philox4x32-10 call per pair of sites of the colour that
// are adjacent in a row (x0 = 4m + parity and x0 + 2: the kernels' unit of
// work), counter (x0's site, colour | tag << 1, sweep); the first site takes
// words 0-1 and the second words 2-3, each site's two words split into its
// three draws (o3_split: 21, 21 and 22 bits).
//
// Arithmetic of the Metropolis step (ALG 0, 2, 3): two sites per thread
// evaluated together with Blackwell's packed fp32 pair instructions
// (fma/add/mul.rn.f32x2: one instruction, two IEEE-rounded lane results),
// uniforms built from Philox bits (1.m - 1 with the draw's top bits as m, no
// integer-to-float conversion), products fused where the CPU replay fuses
// them (fmaf), square root and division IEEE-rounded, and exp / sin / cos the
// engine's own polynomials; the CPU replay (oracle/oracle.c,
// orc_o3_propose / orc_o3_accept) performs the same operations per site and
// reproduces the device trajectory bit for bit.  The heat bath (ALG 1) keeps
// its scalar per-site arithmetic.
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
  const float k = -__frcp_rn(fadd(sg, az));  // = fdiv(-1, sg + az) bit for bit (|sg + az| >= 1)
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

// ---- packed fp32 pairs (lane 0: the thread's first site, lane 1: its second)
struct f2 {
  unsigned long long v;
};
__device__ __forceinline__ f2 F2(float a, float b) {
  return f2{((unsigned long long)__float_as_uint(b) << 32) | __float_as_uint(a)};
}
__device__ __forceinline__ f2 F2s(float a) { return F2(a, a); }
__device__ __forceinline__ float lo(f2 x) { return __uint_as_float((uint32_t)x.v); }
__device__ __forceinline__ float hi(f2 x) { return __uint_as_float((uint32_t)(x.v >> 32)); }
__device__ __forceinline__ f2 add2(f2 a, f2 b) {
  f2 d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
  return d;
}
__device__ __forceinline__ f2 sub2(f2 a, f2 b) {
  f2 d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
  return d;
}
__device__ __forceinline__ f2 mul2(f2 a, f2 b) {
  f2 d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
  return d;
}
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) {
  f2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d.v) : "l"(a.v), "l"(b.v), "l"(c.v));
  return d;
}

// Uniforms from Philox bits without an integer-to-float conversion:
// unit23 = 1.m - 1 with the top 23 bits of u as m (multiples of 2^-23 in
// [0, 1)); half23 = unit23 + 2^-24 (in (0, 1)).  Both subtractions are exact.
__device__ __forceinline__ float bits23(uint32_t u) { return __uint_as_float(0x3F800000u | (u >> 9)); }
__device__ __forceinline__ f2 unit23_2(uint32_t a, uint32_t b) { return sub2(F2(bits23(a), bits23(b)), F2s(1.0f)); }
__device__ __forceinline__ f2 half23_2(uint32_t a, uint32_t b) {
  return sub2(F2(bits23(a), bits23(b)), F2s(0x1.fffffep-1f));
}

// (cos, sin) of 2 pi u / 2^32 for both lanes: octant from the top 3 bits, the
// next 23 bits as the fraction t of the octant (1.m - 1), Taylor polynomials
// of degree 9 / 10 on [0, pi/4] (fused Horner, packed), swaps and signs per
// lane by octant.
__device__ __forceinline__ void sincos23_2(uint32_t ua, uint32_t ub, f2& c, f2& s) {
  const uint32_t oa = ua >> 29, ob = ub >> 29;
  f2 t = sub2(F2(__uint_as_float(0x3F800000u | ((ua >> 6) & 0x7FFFFFu)),
                 __uint_as_float(0x3F800000u | ((ub >> 6) & 0x7FFFFFu))),
              F2s(1.0f));
  const f2 t1 = sub2(F2s(1.0f), t);
  t = F2((oa & 1u) ? lo(t1) : lo(t), (ob & 1u) ? hi(t1) : hi(t));
  const f2 th = mul2(t, F2s(0x1.921fb6p-1f));
  const f2 t2 = mul2(th, th);
  f2 sp = fma2(F2s(0x1.71de3ap-19f), t2, F2s(-0x1.a01a02p-13f));
  sp = fma2(sp, t2, F2s(0x1.111112p-7f));
  sp = fma2(sp, t2, F2s(-0x1.555556p-3f));
  sp = fma2(sp, t2, F2s(1.0f));
  const f2 sn = mul2(th, sp);
  f2 cp = fma2(F2s(-0x1.27e4fcp-22f), t2, F2s(0x1.a01a02p-16f));
  cp = fma2(cp, t2, F2s(-0x1.6c16c2p-10f));
  cp = fma2(cp, t2, F2s(0x1.555556p-5f));
  cp = fma2(cp, t2, F2s(-0.5f));
  const f2 cs = fma2(cp, t2, F2s(1.0f));
  // octants 1, 2, 5, 6 swap; cos < 0 in octants 2..5, sin < 0 in 4..7
  const bool swa = ((oa + 1u) & 2u) != 0u, swb = ((ob + 1u) & 2u) != 0u;
  const float aa = swa ? lo(sn) : lo(cs), ba = swa ? lo(cs) : lo(sn);
  const float ab = swb ? hi(sn) : hi(cs), bb = swb ? hi(cs) : hi(sn);
  c = F2(((oa + 2u) & 4u) ? -aa : aa, ((ob + 2u) & 4u) ? -ab : ab);
  s = F2((oa & 4u) ? -ba : ba, (ob & 4u) ? -bb : bb);
}

// exp(x) for -87 <= x <= 0, both lanes (lanes below -87 are clamped there,
// where the result is below every acceptance draw; lanes above 0 are not
// used): x log2(e) = n + f, n = rint by the 1.5 2^23 shifter, f in
// [-1/2, 1/2], e^(f ln 2) by the degree-7 Taylor polynomial, times 2^n.
__device__ __forceinline__ f2 exp_neg2_2(f2 x) {
  x = F2(fmaxf(lo(x), -87.0f), fmaxf(hi(x), -87.0f));
  const f2 y = mul2(x, F2s(0x1.715476p+0f));
  const f2 r = add2(y, F2s(0x1.8p23f));
  const f2 n = sub2(r, F2s(0x1.8p23f));
  const f2 t = mul2(sub2(y, n), F2s(0x1.62e430p-1f));
  f2 p = fma2(F2s(0x1.a01a02p-13f), t, F2s(0x1.6c16c2p-10f));
  p = fma2(p, t, F2s(0x1.111112p-7f));
  p = fma2(p, t, F2s(0x1.555556p-5f));
  p = fma2(p, t, F2s(0x1.555556p-3f));
  p = fma2(p, t, F2s(0.5f));
  p = fma2(p, t, F2s(1.0f));
  p = fma2(p, t, F2s(1.0f));
  // 2^n: (bits(r) - 0x4B400000 + 127) << 23
  const f2 sc = F2(__uint_as_float((__float_as_uint(lo(r)) - 0x4B3FFF81u) << 23),
                   __uint_as_float((__float_as_uint(hi(r)) - 0x4B3FFF81u) << 23));
  return mul2(p, sc);
}

// Hardware approximations (PTX sqrt.approx / rcp.approx, the sin / cos / exp
// intrinsics) for the fast cap proposal.
__device__ __forceinline__ float sqrt_approx(float x) {
  float r;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Metropolis step of two sites (PROP 0 cap of 1 - cos(alpha) = omc, 1
// uniform unit vector, 2 OPSS rotation with bound omc, 3 the cap with the
// hardware approximations of sqrt, reciprocal, sin / cos and exp): proposals
// n and the decisions.  Per lane (PROP 0-2) the operations of
// orc_o3_propose / orc_o3_accept; PROP 3 takes the same draws and differs from
// PROP 0 only by the approximations' rounding (float32-tolerance parity).
template <int PROP>
__device__ __forceinline__ void o3_metropolis_2(f2 ax, f2 ay, f2 az, f2 hx, f2 hy, f2 hz, const uint4& oa,
                                                const uint4& ob, float omc, float mJ, float beta, f2& nx,
                                                f2& ny, f2& nz, bool& ok_a, bool& ok_b) {
  f2 px, py, pz;
  if (PROP == 0 || PROP == 3) {
    const f2 w = mul2(unit23_2(oa.x, ob.x), F2s(omc));
    const f2 ct = sub2(F2s(1.0f), w);
    const f2 s2 = fma2(mul2(w, F2s(-1.0f)), w, add2(w, w));
    f2 st, cp, sp;
    if (PROP == 0) {
      st = F2(__fsqrt_rn(lo(s2)), __fsqrt_rn(hi(s2)));
      sincos23_2(oa.y, ob.y, cp, sp);
    } else {
      st = F2(sqrt_approx(lo(s2)), sqrt_approx(hi(s2)));
      // phi = 2 pi u / 2^32 taken in [-pi, pi) (u as a signed word): the
      // same angle modulo 2 pi, where the intrinsics are most accurate
      float sa, ca, sb, cb;
      __sincosf((float)(int32_t)oa.y * 0x1.921fb6p-30f, &sa, &ca);
      __sincosf((float)(int32_t)ob.y * 0x1.921fb6p-30f, &sb, &cb);
      cp = F2(ca, cb);
      sp = F2(sa, sb);
    }
    const f2 vx = mul2(st, cp), vy = mul2(st, sp);
    // Duff et al. (JCGT 2017) basis {e1, e2, a}: sg = sign(az), k = -1/(sg + az)
    const f2 sg = F2(lo(az) >= 0.0f ? 1.0f : -1.0f, hi(az) >= 0.0f ? 1.0f : -1.0f);
    const f2 d = add2(sg, az);
    // -1 / d as the negated correctly rounded reciprocal: round-to-nearest
    // is symmetric in sign, so this is the IEEE quotient bit for bit (|d| >= 1)
    const f2 k = PROP == 0 ? F2(-__frcp_rn(lo(d)), -__frcp_rn(hi(d))) : F2(-rcp_approx(lo(d)), -rcp_approx(hi(d)));
    const f2 axk = mul2(ax, k);
    const f2 b = mul2(ay, axk);
    const f2 sax = mul2(sg, ax);
    const f2 e1x = fma2(sax, axk, F2s(1.0f)), e1y = mul2(sg, b), e1z = mul2(sax, F2s(-1.0f));
    const f2 e2x = b, e2y = fma2(mul2(ay, k), ay, sg), e2z = mul2(ay, F2s(-1.0f));
    px = fma2(ct, ax, fma2(vy, e2x, mul2(vx, e1x)));
    py = fma2(ct, ay, fma2(vy, e2y, mul2(vx, e1y)));
    pz = fma2(ct, az, fma2(vy, e2z, mul2(vx, e1z)));
  } else if (PROP == 1) {
    pz = fma2(F2s(-2.0f), unit23_2(oa.x, ob.x), F2s(1.0f));
    const f2 r2 = fma2(mul2(pz, F2s(-1.0f)), pz, F2s(1.0f));
    const f2 rho = F2(__fsqrt_rn(lo(r2)), __fsqrt_rn(hi(r2)));
    f2 cp, sp;
    sincos23_2(oa.y, ob.y, cp, sp);
    px = mul2(rho, cp);
    py = mul2(rho, sp);
  } else {
    const f2 theta = mul2(F2s(omc), fma2(F2s(2.0f), half23_2(oa.y, ob.y), F2s(-1.0f)));
    const f2 turns = mul2(mul2(theta, F2s(0x1.45f306p-3f)), F2s(0x1p32f));
    const uint32_t ta = (uint32_t)(long long)__float2ll_rn(lo(turns));
    const uint32_t tb = (uint32_t)(long long)__float2ll_rn(hi(turns));
    f2 c, sn;
    sincos23_2(ta, tb, c, sn);
    const uint32_t pa = __umulhi(oa.x, 3u), pb = __umulhi(ob.x, 3u);
    const f2 a0 = F2(pa == 0 ? lo(ax) : (pa == 1 ? lo(ay) : lo(az)), pb == 0 ? hi(ax) : (pb == 1 ? hi(ay) : hi(az)));
    const f2 a1 = F2(pa == 0 ? lo(ay) : (pa == 1 ? lo(az) : lo(ax)), pb == 0 ? hi(ay) : (pb == 1 ? hi(az) : hi(ax)));
    const f2 r0 = fma2(c, a0, mul2(mul2(sn, a1), F2s(-1.0f))), r1 = fma2(sn, a0, mul2(c, a1));
    px = F2(pa == 0 ? lo(r0) : (pa == 1 ? lo(ax) : lo(r1)), pb == 0 ? hi(r0) : (pb == 1 ? hi(ax) : hi(r1)));
    py = F2(pa == 0 ? lo(r1) : (pa == 1 ? lo(r0) : lo(ay)), pb == 0 ? hi(r1) : (pb == 1 ? hi(r0) : hi(ay)));
    pz = F2(pa == 0 ? lo(az) : (pa == 1 ? lo(r1) : lo(r0)), pb == 0 ? hi(az) : (pb == 1 ? hi(r1) : hi(r0)));
  }
  // one Newton step of 1/sqrt(n2) from 1
  const f2 n2 = fma2(pz, pz, fma2(py, py, mul2(px, px)));
  const f2 f = fma2(F2s(-0.5f), n2, F2s(1.5f));
  px = mul2(px, f);
  py = mul2(py, f);
  pz = mul2(pz, f);
  const f2 dot = fma2(sub2(pz, az), hz, fma2(sub2(py, ay), hy, mul2(sub2(px, ax), hx)));
  const f2 de = mul2(F2s(mJ), dot);
  const f2 bde = mul2(F2s(-beta), de);
  const f2 p = PROP == 3 ? F2(__expf(fmaxf(lo(bde), -87.0f)), __expf(fmaxf(hi(bde), -87.0f))) : exp_neg2_2(bde);
  const f2 u = half23_2(oa.z, ob.z);
  ok_a = lo(de) <= 0.0f || lo(u) < lo(p);
  ok_b = hi(de) <= 0.0f || hi(u) < hi(p);
  nx = px;
  ny = py;
  nz = pz;
}

// Fixed-point observables of a site's final spin (s) and, in the colour-1
// pass, its bond sum with the fp32 neighbour sum h: rint(2^21 s_c) and
// rint(2^19 s . h) by the 1.5 2^23 shifter (|2^21 s_c| <= 2^21,
// |2^19 s . h| <= 6 2^19 < 2^22), summed in 32-bit integers.
// The shifter's bit patterns are summed as they are (modulo 2^32) and the
// shifter's own pattern, once per term, is taken off at the flush: one
// three-input add per value and pair.  A pair with one site scales its second
// lane by zero, so that lane adds exactly the shifter.
struct O3Fix {
  uint32_t m[3], e;
  uint32_t n;  // terms per value since the last flush
};
__device__ __forceinline__ int32_t fix_shift(float v) { return (int32_t)(__float_as_uint(v) - 0x4B400000u); }
template <bool BOND>
__device__ __forceinline__ void o3_fix_add_2(O3Fix& q, f2 sx, f2 sy, f2 sz, f2 hx, f2 hy, f2 hz, bool use_b) {
  const f2 X = F2s(0x1.8p23f);
  const f2 sm = F2(0x1p21f, use_b ? 0x1p21f : 0.0f);
  const f2 mx = fma2(sx, sm, X), my = fma2(sy, sm, X), mz = fma2(sz, sm, X);
  q.m[0] += __float_as_uint(lo(mx)) + __float_as_uint(hi(mx));
  q.m[1] += __float_as_uint(lo(my)) + __float_as_uint(hi(my));
  q.m[2] += __float_as_uint(lo(mz)) + __float_as_uint(hi(mz));
  if (BOND) {
    const f2 se = F2(0x1p19f, use_b ? 0x1p19f : 0.0f);
    const f2 e = fma2(fma2(sz, hz, fma2(sy, hy, mul2(sx, hx))), se, X);
    q.e += __float_as_uint(lo(e)) + __float_as_uint(hi(e));
  }
  q.n += 2;
}

// Philox4x32-10 of counter (site, colour | TAG_O3 << 1, sweep) with the
// sweep-uniform part of round 1 and the ten round keys precomputed once per
// tile (the key is the lattice's, the same for the whole CTA, so the compiler
// holds the schedule in uniform registers: measured 15 fewer instructions per
// site than bumping the keys every round, at the same 64 registers).
struct O3Philox {
  uint32_t a, b, c;
  uint32_t k0[10], k1[10];
};
__device__ __forceinline__ O3Philox make_o3_philox(uint64_t key, uint64_t sweep, uint32_t ctrl) {
  O3Philox P;
  const uint32_t k0 = (uint32_t)key, k1 = (uint32_t)(key >> 32);
  const uint32_t c2 = (uint32_t)sweep, c3 = (uint32_t)(sweep >> 32);
  P.a = __umulhi(0xCD9E8D57u, c2) ^ k0 ^ ctrl;
  P.b = 0xCD9E8D57u * c2;
  P.c = c3 ^ k1;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    P.k0[r] = k0 + (uint32_t)r * 0x9E3779B9u;
    P.k1[r] = k1 + (uint32_t)r * 0xBB67AE85u;
  }
  return P;
}
__device__ __forceinline__ uint4 o3_philox(const O3Philox& P, uint32_t index) {
  const uint64_t p00 = (uint64_t)0xD2511F53u * index;
  uint4 c = make_uint4(P.a, P.b, (uint32_t)(p00 >> 32) ^ P.c, (uint32_t)p00);
#pragma unroll
  for (int r = 1; r < 10; ++r) {
    // separate high and low products: 10 fewer instructions per site here
    // than one 32x32->64 wide product (which the bit-sliced kernels keep)
    const uint32_t h0 = __umulhi(0xD2511F53u, c.x), l0 = 0xD2511F53u * c.x;
    const uint32_t h1 = __umulhi(0xCD9E8D57u, c.z), l1 = 0xCD9E8D57u * c.z;
    c = make_uint4(h1 ^ c.y ^ P.k0[r], l1, h0 ^ c.w ^ P.k1[r], l0);
  }
  return c;
}

// The three draw words of a site from two Philox words u, v: the top 21
// bits of u and of v (low bits zero), and the two low 11-bit fields joined
// into the top 22 bits of the third word (orc_o3_split).
__device__ __forceinline__ uint4 o3_split(uint32_t u, uint32_t v) {
  return make_uint4(u & ~0x7FFu, v & ~0x7FFu, (u << 21) | ((v & 0x7FFu) << 10), 0u);
}

// One site of a colour pass: its own spin and the fp32 sum of its
// neighbours (in the fixed order x-1, x+1, y-1, y+1, z-1, z+1).
struct O3Site {
  uint32_t me, site;
  float ax, ay, az, hx, hy, hz;
};

template <int DIM>
__device__ __forceinline__ void o3_load_site(O3Site& q, const float* S, const float* S1, const float* S2,
                                             int x, int y, int z, int lx, int ly, int lz, int pitch,
                                             uint32_t cs) {
  const uint32_t rowoff = ((uint32_t)z * ly + y) * (uint32_t)pitch;
  const int ym = y ? y - 1 : ly - 1, yp = y + 1 < ly ? y + 1 : 0;
  const int xm = x ? x - 1 : lx - 1, xp = x + 1 < lx ? x + 1 : 0;
  uint32_t zmo = 0, zpo = 0;
  if (DIM == 3) {
    const int zm = z ? z - 1 : lz - 1, zp = z + 1 < lz ? z + 1 : 0;
    zmo = ((uint32_t)zm * ly + y) * (uint32_t)pitch + x;
    zpo = ((uint32_t)zp * ly + y) * (uint32_t)pitch + x;
  }
  const uint32_t nb[6] = {rowoff + xm, rowoff + xp, ((uint32_t)z * ly + ym) * (uint32_t)pitch + x,
                          ((uint32_t)z * ly + yp) * (uint32_t)pitch + x, zmo, zpo};
  float hx = ld_chk(S, nb[0], cs), hy = ld_chk(S1, nb[0], cs), hz = ld_chk(S2, nb[0], cs);
#pragma unroll
  for (int i = 1; i < 2 * DIM; ++i) {
    hx = fadd(hx, ld_chk(S, nb[i], cs));
    hy = fadd(hy, ld_chk(S1, nb[i], cs));
    hz = fadd(hz, ld_chk(S2, nb[i], cs));
  }
  q.me = rowoff + x;
  q.ax = ld_chk(S, q.me, cs);
  q.ay = ld_chk(S1, q.me, cs);
  q.az = ld_chk(S2, q.me, cs);
  q.hx = hx;
  q.hy = hy;
  q.hz = hz;
  q.site = (uint32_t)((size_t)(z * ly + y) * lx + x);
}

// Stores spin (x, y, z) at element `me` of the three component planes of S
// (plane stride cs).
__device__ __forceinline__ void o3_store3(float* S, uint32_t cs, uint32_t me, float x, float y, float z) {
  if (GPUMC_IN(me, cs)) {
    float* p = S + me;
    p[0] = x;
    p[cs] = y;
    p[2 * (size_t)cs] = z;
  }
}

// Updates the pair (qa, qb) of a colour pass (qb only when `two`): writes
// the final spins in place, counts acceptances and adds the fixed-point
// observables of the final spins.
template <int COLOUR, int ALG>
__device__ __forceinline__ void o3_update_pair(const O3Site& qa, const O3Site& qb, bool two, const O3Philox& P,
                                               float omc, float mJ, float beta, float* S, uint32_t cs, O3Fix& fx,
                                               int& nacc) {
  // one draw per pair (keyed by its first site, qa): words 0-1 for qa,
  // 2-3 for qb
  const uint4 w = o3_philox(P, qa.site);
  const uint4 oa = o3_split(w.x, w.y), ob = o3_split(w.z, w.w);
  f2 fx2 = F2(qa.ax, qb.ax), fy2 = F2(qa.ay, qb.ay), fz2 = F2(qa.az, qb.az);
  const f2 hx = F2(qa.hx, qb.hx), hy = F2(qa.hy, qb.hy), hz = F2(qa.hz, qb.hz);
  bool ok_a, ok_b;
  if (ALG == 1) {
    float nx, ny, nz, mx, my, mz;
    o3_heat_bath(qa.hx, qa.hy, qa.hz, oa, -mJ, beta, nx, ny, nz);
    o3_heat_bath(qb.hx, qb.hy, qb.hz, ob, -mJ, beta, mx, my, mz);
    ok_a = (nx != qa.ax) | (ny != qa.ay) | (nz != qa.az);
    ok_b = (mx != qb.ax) | (my != qb.ay) | (mz != qb.az);
    fx2 = F2(nx, mx);
    fy2 = F2(ny, my);
    fz2 = F2(nz, mz);
  } else {
    f2 nx, ny, nz;
    constexpr int PROP = ALG == 2 ? 1 : (ALG == 3 ? 2 : (ALG == 4 ? 3 : 0));
    o3_metropolis_2<PROP>(fx2, fy2, fz2, hx, hy, hz, oa, ob, omc, mJ, beta, nx, ny, nz, ok_a, ok_b);
    fx2 = F2(ok_a ? lo(nx) : qa.ax, ok_b ? hi(nx) : qb.ax);
    fy2 = F2(ok_a ? lo(ny) : qa.ay, ok_b ? hi(ny) : qb.ay);
    fz2 = F2(ok_a ? lo(nz) : qa.az, ok_b ? hi(nz) : qb.az);
  }
  ok_b = ok_b && two;
  // every site of the pair is stored, rejected ones with their old spin: a
  // colour pass reads only the other colour, so the rewrite is invisible,
  // and the stores no longer branch on the decisions (measured 1-2 % faster;
  // the DRAM writes barely change, as a sector of four colour sites almost
  // always holds an accepted one)
  o3_store3(S, cs, qa.me, lo(fx2), lo(fy2), lo(fz2));
  if (two) o3_store3(S, cs, qb.me, hi(fx2), hi(fy2), hi(fz2));
  nacc += (int)ok_a + (int)ok_b;
  // every bond has one colour-1 end: the colour-1 pass also sums s . h
  o3_fix_add_2<COLOUR == 1>(fx, fx2, fy2, fz2, hx, hy, hz, two);
}

// Per-thread fixed-point sums into 64-bit totals (flushed often enough that
// the 32-bit partial sums cannot overflow), then CTA sums and one atomic each.
struct O3Totals {
  long long m[3], e;
};
template <bool BOND>
__device__ __forceinline__ void o3_flush(O3Totals& t, O3Fix& q) {
  const uint32_t off = q.n * 0x4B400000u;  // the shifter's pattern, once per term (mod 2^32)
  t.m[0] += (int32_t)(q.m[0] - off);
  t.m[1] += (int32_t)(q.m[1] - off);
  t.m[2] += (int32_t)(q.m[2] - off);
  if (BOND) t.e += (int32_t)(q.e - off);
  q = O3Fix{{0, 0, 0}, 0, 0};
}
template <int COLOUR>
__device__ __forceinline__ void o3_commit(LatDesc* L, O3Totals& t, int nacc) {
  long long v[5] = {t.m[0], t.m[1], t.m[2], t.e, (long long)nacc};
  cta_sum(v);
  if (threadIdx.x == 0) {
    atomic_add_i64(&L->acc.mq[0], v[0]);
    atomic_add_i64(&L->acc.mq[1], v[1]);
    atomic_add_i64(&L->acc.mq[2], v[2]);
    if (COLOUR == 1) {
      atomic_add_i64(&L->acc.ebq, v[3]);
      L->acc.fresh = 1;
    }
    if (v[4]) atomic_add_i64(&L->acc.accepted, v[4]);
  }
}

// One colour pass over a tile of full rows (y0 .. y0+hv-1, planes z0 ..
// z0+dv-1), one thread per site of the colour, two sites at a time.
template <int DIM, int COLOUR, int ALG>
__global__ void __launch_bounds__(kThreads, 4)
    k_sweep_o3(const TileItem* __restrict__ tiles, LatDesc* __restrict__ lats,
               GroupDesc* __restrict__ groups, LaunchCtl* __restrict__ ctl) {
  const TileItem t = tiles[blockIdx.x];
  LatDesc* L = &lats[t.lat];
  const GroupDesc* G = &groups[L->group];
  const uint64_t sweep = L->sweep;
  if (sweep >= L->target) {
    if (COLOUR == 1) group_epilogue(t.pad, lats, groups, ctl);
    return;
  }
  const int lx = L->lx, ly = L->ly, lz = DIM == 3 ? L->lz : 1, pitch = L->pitch;
  const uint32_t cs = (uint32_t)pitch * ly * lz;  // component plane stride (< 2^32 elements)
  float* S = (float*)L->buf[0];  // in place; component planes S, S1, S2
  float* S1 = S + (size_t)cs;
  float* S2 = S + 2 * (size_t)cs;
  const int label = G->label[L->replica];
  const float beta = G->betas_f[label];
  const float mJ = -G->Jf;
  const float omc = L->omc;
  const O3Philox P = make_o3_philox(L->key, sweep, (uint32_t)COLOUR | ((ALG == 1 ? TAG_O3HB : TAG_O3) << 1));
  const int hv = min(t.ty, ly - t.y0);
  const int dv = DIM == 3 ? min(t.tz, lz - t.z0) : 1;
  const int half = lx >> 1;        // sites of the colour per row
  const int np = (half + 1) >> 1;  // pairs per row (the last may be single)
  const int rows = hv * dv;
  // Work items are pairs of horizontally adjacent sites of the colour in one
  // row (x and x + 2, x = 4m + parity), one draw per pair, as in the z-march
  // kernel.  Thread mapping: fixed pair column (or column stride) per thread,
  // rows strided.
  int col0, cstep, r0, rstep;
  if (np >= kThreads) {
    col0 = threadIdx.x;
    cstep = kThreads;
    r0 = 0;
    rstep = 1;
  } else {
    col0 = threadIdx.x % np;
    cstep = np;
    r0 = threadIdx.x / np;
    rstep = kThreads / np;
  }
  O3Fix fx = {{0, 0, 0}, 0, 0};
  O3Totals tot = {{0, 0, 0}, 0};
  int nacc = 0;
  // this thread's pairs, row-major: rows r0, r0 + rstep, ... of the tile's
  // rows (y fastest, then z), pair columns col0, col0 + cstep, ...; the
  // (row, column) cursor advances without divisions
  const int nc = (r0 < rstep && col0 < np) ? (np - col0 + cstep - 1) / cstep : 0;
  const int nr = r0 < rstep ? (rows - r0 + rstep - 1) / rstep : 0;
  const int n_items = nc * nr;
  int cy = t.y0 + (DIM == 3 ? r0 % hv : r0), cz = DIM == 3 ? t.z0 + r0 / hv : 0, cc = 0;
  const int ry = DIM == 3 ? rstep % hv : rstep, rz = DIM == 3 ? rstep / hv : 0;
  for (int k = 0; k < n_items; ++k) {
    const int y = cy, z = cz, m = col0 + cc * cstep;
    if (++cc == nc) {
      cc = 0;
      cy += ry;
      cz += rz;
      if (cy >= t.y0 + hv) {
        cy -= hv;
        cz += 1;
      }
    }
    const int xa = 4 * m + ((y + z + COLOUR) & 1);
    const bool two = 2 * m + 1 < half;
    O3Site qa, qb;
    o3_load_site<DIM>(qa, S, S1, S2, xa, y, z, lx, ly, lz, pitch, cs);
    if (two)
      o3_load_site<DIM>(qb, S, S1, S2, xa + 2, y, z, lx, ly, lz, pitch, cs);
    else
      qb = qa;
    o3_update_pair<COLOUR, ALG>(qa, qb, two, P, omc, mJ, beta, S, cs, fx, nacc);
    if ((k & 31) == 31) o3_flush<COLOUR == 1>(tot, fx);  // every 64 sites: 32-bit partials stay far from overflow
  }
  o3_flush<COLOUR == 1>(tot, fx);
  o3_commit<COLOUR>(L, tot, nacc);
  if (COLOUR == 1) group_epilogue(t.pad, lats, groups, ctl);
}

// ---------------------------------------------------------------------------
// 3D colour pass marched along z through a ring of shared-memory planes.
//
// A tile is whole rows y0 .. y0+hv-1 of planes z0 .. z0+dv-1.  Each plane the
// tile touches (z0-1 .. z0+dv) is copied once, rows y0-1 .. y0+hv with all
// three components, into a ring slot and serves as the z-1, z and z+1 plane
// of three consecutive steps.  A slot holds the three components one after
// another, each as the tile's rows at the lattice's pitch; for pitches 32, 64
// and 128 the pitch and the component stride are compiled in
// (o3_row_class), so every neighbour of a thread's sites is a fixed offset
// from one index per plane and the loads take the offsets as immediates.
//
// The copies are bulk asynchronous copies (cp.async.bulk, no multicast), one
// per component and contiguous run of rows (at most three: split where the
// rows wrap), issued by three lanes of one warp; each slot's mbarrier counts
// the bytes in (expect_tx / complete_tx).  (One copy per row and component
// measured 1.65x slower: many small copies queue in the copy engine.)  Plane p of a
// tile's march (p = 0 for z0-1) goes to slot p % S (S = kO3RingSlots) as that
// slot's (p / S)-th fill, so a step waits for phase parity (p / S) & 1 of its
// three slots.  The warps are not synchronised per plane: each warp waits for
// the planes of its step, computes its pairs and then releases the plane it
// no longer needs (a per-slot arrival counter in shared memory); the warp
// whose arrival completes a slot's count refills the slot with plane p + S.
// A warp can thus run up to S - 3 steps ahead of the slowest one, and no
// step ends in a CTA-wide barrier.  Every wait is bounded; one that gives up
// flags the launch (ctl->err), stops the other warps' waits, waits (bounded
// again) for the copies in flight and leaves the tile.  The pass reads only
// the other colour's values (and its own sites' old values, which only this
// tile writes), so copying planes that other tiles update in place is
// race-free.  The site arithmetic and its operation order are those of
// k_sweep_o3.
// ---------------------------------------------------------------------------
constexpr long long kRingWaitPolls = 1ll << 20;  // try_wait polls per ring wait
constexpr int kWarps = kThreads / 32;

__device__ __forceinline__ void ring_init(unsigned long long* bar) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(a) : "memory");
}
__device__ __forceinline__ void ring_expect(unsigned long long* bar, uint32_t bytes) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}\n" ::"r"(a),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void ring_bulk_copy(void* dst, const void* src, uint32_t bytes, unsigned long long* bar) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(d),
               "l"(src), "r"(bytes), "r"(a)
               : "memory");
}
__device__ __forceinline__ bool ring_test(unsigned long long* bar, uint32_t parity) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
  uint32_t done;
  asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
               : "=r"(done)
               : "r"(a), "r"(parity)
               : "memory");
  return done != 0;
}
// Bounded wait for the completion of phase `parity` of a slot's mbarrier;
// gives up early when another warp has flagged the ring (`abort`).
__device__ __forceinline__ bool ring_wait(unsigned long long* bar, uint32_t parity, const volatile int* abort) {
  for (long long it = 0; it < kRingWaitPolls; ++it) {
    if (ring_test(bar, parity)) return true;
    if ((it & 63) == 63 && *abort) return false;
  }
  return false;
}

// Ring state of a CTA: per-slot fill barriers and arrival counters, and the
// tile's observable totals (kept here rather than in registers).
struct O3Ring {
  unsigned long long full[kO3RingSlots];
  unsigned int freed[kO3RingSlots];
  int abort;
  int issued;        // march planes whose copies were issued (this tile)
  long long tot[5];  // magnetisation x, y, z, bond sum, accepted
};

// Adds the warp's fixed-point partial sums (and acceptances) to the CTA
// totals: 64-bit butterfly over the lanes, one shared atomic per value.  All
// 32 lanes call.  The 32-bit partials are exact modulo 2^32 and their true
// values stay below 2^31 in magnitude (fewer than 512 terms of at most
// 6 2^19 each), so each lane's value is recovered exactly.
template <bool BOND>
__device__ __forceinline__ void o3_flush_warp(O3Ring& R, O3Fix& q, int& nacc) {
  const uint32_t off = q.n * 0x4B400000u;
  long long v[5] = {(int32_t)(q.m[0] - off), (int32_t)(q.m[1] - off), (int32_t)(q.m[2] - off),
                    BOND ? (long long)(int32_t)(q.e - off) : 0ll, (long long)nacc};
#pragma unroll
  for (int i = 0; i < 5; ++i)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_xor_sync(0xFFFFFFFFu, v[i], o);
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int i = 0; i < 5; ++i)
      if (v[i]) atomicAdd((unsigned long long*)&R.tot[i], (unsigned long long)v[i]);
  q = O3Fix{{0, 0, 0}, 0, 0};
  nacc = 0;
}

// Issues the copy of march plane p of tile t into its slot: per component,
// the tile's rows y0-1 .. y0+hv as one contiguous run of the plane (split
// where the rows wrap), by lanes 0..2 of the calling warp (all 32 lanes
// call).  `crows` is the slot's rows per component.  The geometry is read
// again from the lattice descriptor (cached), so none of it stays live in
// registers across the march.
__device__ __forceinline__ void o3_issue_plane(const TileItem& t, const LatDesc* L, O3Ring& R, float* osm, int p,
                                               int crows, int lane) {
  const int ly = L->ly, lz = L->lz, pitch = L->pitch;
  const long long cs = (long long)pitch * ly * lz;
  const int hv = min(t.ty, ly - t.y0);
  const int RW = hv + 2;
  const long long cstr = (long long)crows * pitch;
  const long long slot = 3 * cstr;
  const int sl = p % kO3RingSlots;
  if (lane == 0) {
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");  // generic reads of the slot before the refill
    ring_expect(&R.full[sl], (uint32_t)(RW * 3 * pitch) * 4u);
  }
  __syncwarp();
  if (lane < 3) {
    const int c = lane;
    const float* S = (const float*)L->buf[0];
    int zz = t.z0 - 1 + p;
    zz = zz < 0 ? zz + lz : (zz >= lz ? zz - lz : zz);
    int r = 0;
    while (r < RW) {
      int y = t.y0 - 1 + r;
      y = y < 0 ? y + ly : (y >= ly ? y - ly : y);
      const int n = min(RW - r, ly - y);  // rows contiguous up to the plane's last row
      const long long so = (long long)c * cs + ((long long)zz * ly + y) * pitch;
      const long long dof = (long long)sl * slot + (long long)c * cstr + (long long)r * pitch;
      if (GPUMC_IN(so + (long long)n * pitch - 1, 3 * cs) && GPUMC_IN(dof + (long long)n * pitch - 1, kO3RingSlots * slot))
        ring_bulk_copy(osm + dof, S + so, (uint32_t)(n * pitch) * 4u, &R.full[sl]);
      r += n;
    }
  }
}

// Shared-memory load of slot element i (checked in bounds-checked builds).
__device__ __forceinline__ float o3_lds(const float* base, int i, int lim) {
#ifdef GPUMC_DEBUG_BOUNDS
  return GPUMC_IN(i, lim) ? base[i] : 0.0f;
#else
  (void)lim;
  return base[i];
#endif
}

// One tile of a colour pass; RP_ is the compiled row pitch and CROWS_ the
// compiled rows per component of a slot (0: the lattice's pitch and the
// tile's rows at run time).
template <int COLOUR, int ALG, int RP_, int CROWS_>
__device__ __forceinline__ void o3_march_tile(const TileItem& t, LatDesc* L, const GroupDesc* G, LaunchCtl* ctl,
                                              float* osm, O3Ring& R) {
  O3Fix fx = {{0, 0, 0}, 0, 0};
  int nacc = 0;
  const int lx = L->lx, ly = L->ly, lz = L->lz, pitch = L->pitch;
  const long long csl = (long long)pitch * ly * lz;
  float* S = (float*)L->buf[0];
  const int hv = min(t.ty, ly - t.y0);
  const int dv = min(t.tz, lz - t.z0);
  const int RP = RP_ > 0 ? RP_ : pitch;               // floats per slot row (= pitch)
  const int crows = CROWS_ > 0 ? CROWS_ : hv + 2;     // slot rows per component
  const int cstr = crows * RP;                        // floats per component in a slot
  const int slot = 3 * cstr;                          // floats per slot
  const int lim = slot;                  // every index below is within its plane's slot
  const uint32_t cs = (uint32_t)csl;     // < 2^32 elements
  const uint64_t sweep = L->sweep;
  const int label = G->label[L->replica];
  const float beta = G->betas_f[label];
  const float mJ = -G->Jf;
  const float omc = L->omc;
  const O3Philox P = make_o3_philox(L->key, sweep, (uint32_t)COLOUR | ((ALG == 1 ? TAG_O3HB : TAG_O3) << 1));
  const int lane = threadIdx.x & 31;
  // Work items are pairs of horizontally adjacent sites of the colour in one
  // row (x and x + 2, x = 4m + parity): both sites' neighbours then sit at
  // fixed offsets from one row position (the x + 1 site is shared), and a
  // thread's pairs are found once per tile, not per plane.
  const int half = lx >> 1;        // sites of the colour per row
  const int np = (half + 1) >> 1;  // pairs per row (the last may be single)
  const int n_pairs = hv * np;     // pairs of the tile's rows in one plane
  const int rs = RP;               // floats per slot row
  const int r0 = threadIdx.x / np, m0 = threadIdx.x - r0 * np;
  const int dr = kThreads / np, dm = kThreads - dr * np;  // cursor step of kThreads pairs
  bool ok = true;
  for (int k = 0; k < dv && ok; ++k) {
    const int z = t.z0 + k;
    // planes z-1, z, z+1 = march planes k, k+1, k+2; after the first step
    // only plane k+2 is new to this warp (a wait on a completed phase still
    // costs some hundred cycles, so the others are not waited for again)
    for (int i = k == 0 ? 0 : 2; i < 3 && ok; ++i)
      ok = ring_wait(&R.full[(k + i) % kO3RingSlots], (uint32_t)((k + i) / kO3RingSlots) & 1u, &R.abort);
    ok = __all_sync(0xFFFFFFFFu, ok);  // one decision per warp
    if (!ok) break;
    const float* pm = osm + (k % kO3RingSlots) * slot;
    const float* pc = osm + ((k + 1) % kO3RingSlots) * slot;
    const float* pp = osm + ((k + 2) % kO3RingSlots) * slot;
    int rl = r0, m = m0;
    for (int i = threadIdx.x; i < n_pairs; i += kThreads) {
      const int y = t.y0 + rl;
      const int xa = 4 * m + ((y + z + COLOUR) & 1), xb = xa + 2;
      const bool two = 2 * m + 1 < half;
      const int row = (rl + 1) * rs;  // slot row of y (component 0; component c at + c cstr)
      const int ia = row + xa;
      const int ib = two ? ia + 2 : ia;
      // x-1 of a and x+1 of b wrap at the row's ends; x+1 of a = x-1 of b
      // (x+1 of a wraps only for a single last site, x = lx - 1)
      const int iam = xa ? ia - 1 : row + lx - 1;
      const int iap = xa + 1 < lx ? ia + 1 : row;
      const int ibp = two ? (xb + 1 < lx ? ia + 3 : row) : iap;
      const int ibm = two ? iap : iam;
      O3Site qa, qb;
      float ha[3], hb[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int o = c * cstr;
        // both sites' sums in one packed chain, neighbour order x-1, x+1,
        // y-1, y+1, z-1, z+1 per lane (as k_sweep_o3); a single site's
        // second lane repeats the first
        const f2 h2 = add2(add2(add2(add2(add2(F2(o3_lds(pc, iam + o, lim), o3_lds(pc, ibm + o, lim)),
                                               F2(o3_lds(pc, iap + o, lim), o3_lds(pc, ibp + o, lim))),
                                          F2(o3_lds(pc, ia - rs + o, lim), o3_lds(pc, ib - rs + o, lim))),
                                     F2(o3_lds(pc, ia + rs + o, lim), o3_lds(pc, ib + rs + o, lim))),
                                F2(o3_lds(pm, ia + o, lim), o3_lds(pm, ib + o, lim))),
                           F2(o3_lds(pp, ia + o, lim), o3_lds(pp, ib + o, lim)));
        ha[c] = lo(h2);
        hb[c] = hi(h2);
      }
      qa.ax = o3_lds(pc, ia, lim);
      qa.ay = o3_lds(pc, ia + cstr, lim);
      qa.az = o3_lds(pc, ia + 2 * cstr, lim);
      qb.ax = o3_lds(pc, ib, lim);
      qb.ay = o3_lds(pc, ib + cstr, lim);
      qb.az = o3_lds(pc, ib + 2 * cstr, lim);
      qa.hx = ha[0];
      qa.hy = ha[1];
      qa.hz = ha[2];
      qb.hx = hb[0];
      qb.hy = hb[1];
      qb.hz = hb[2];
      // 32-bit index arithmetic: the same values as the 64-bit products
      // truncated to the 32-bit fields
      const uint32_t grow = (uint32_t)z * (uint32_t)ly + (uint32_t)y;
      qa.me = grow * (uint32_t)pitch + (uint32_t)xa;
      qa.site = grow * (uint32_t)lx + (uint32_t)xa;
      qb.me = two ? qa.me + 2 : qa.me;
      o3_update_pair<COLOUR, ALG>(qa, qb, two, P, omc, mJ, beta, S, cs, fx, nacc);
      rl += dr;
      m += dm;
      if (m >= np) {
        m -= np;
        rl += 1;
      }
    }
    // a thread adds at most 8 terms per plane (n_pairs <= 4 kThreads), so
    // flushing at 256 keeps every 32-bit partial below 2^31
    if (__any_sync(0xFFFFFFFFu, fx.n >= 256u)) o3_flush_warp<COLOUR == 1>(R, fx, nacc);
    // release the planes this warp no longer needs: plane k after step k,
    // and the last three after the last step
    __syncwarp();
    const int p_lo = k, p_hi = k + 1 < dv ? k : dv + 1;
    for (int p = p_lo; p <= p_hi; ++p) {
      const int sl = p % kO3RingSlots;
      int last = 0;
      if (lane == 0) {
        __threadfence_block();
        last = atomicAdd(&R.freed[sl], 1u) == (unsigned)(kWarps - 1);
        if (last) {
          atomicExch(&R.freed[sl], 0u);
          __threadfence_block();
        }
      }
      last = __shfl_sync(0xFFFFFFFFu, last, 0);
      if (last && p + kO3RingSlots <= dv + 1) {
        o3_issue_plane(t, L, R, osm, p + kO3RingSlots, crows, lane);
        if (lane == 0) atomicMax(&R.issued, p + kO3RingSlots + 1);
      }
    }
  }
  o3_flush_warp<COLOUR == 1>(R, fx, nacc);
  if (!ok && lane == 0) {
    atomicExch(&ctl->err, 2);
    *(volatile int*)&R.abort = 1;
  }
  __syncthreads();
  if (R.abort) {
    // a copy did not land in time: wait (bounded) for the last copy issued
    // into each slot, so none is in flight when the CTA leaves
    if (threadIdx.x == 0)
      for (int p = max(0, R.issued - kO3RingSlots); p < R.issued; ++p) {
        for (long long it = 0; it < kRingWaitPolls; ++it)
          if (ring_test(&R.full[p % kO3RingSlots], (uint32_t)(p / kO3RingSlots) & 1u)) break;
      }
    __syncthreads();
  }
}

// Four CTAs per SM for both colours (64 registers, 55 KB of ring each):
// colour 1's sweep epilogue takes its scratch arrays from the ring.
template <int COLOUR, int ALG, int CLS>
__global__ void __launch_bounds__(kThreads, kO3RingSlots > 4 ? 3 : 4)
    k_sweep_o3_march(const TileItem* __restrict__ tiles, LatDesc* __restrict__ lats,
                     GroupDesc* __restrict__ groups, LaunchCtl* __restrict__ ctl) {
  extern __shared__ __align__(16) float osm[];
  __shared__ O3Ring R;
  const TileItem t = tiles[blockIdx.x];
  LatDesc* L = &lats[t.lat];
  const GroupDesc* G = &groups[L->group];
  if (L->sweep >= L->target) {
    if (COLOUR == 1) group_epilogue<true>(t.pad, lats, groups, ctl, (int*)osm);
    return;
  }
  // warp 0 initialises the ring and issues the first planes' copies right
  // away, before the rest of the tile's set-up (its loads of the group's
  // labels and temperatures): a CTA's first planes are its longest wait
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    if (lane == 0) {
      for (int i = 0; i < kO3RingSlots; ++i) {
        ring_init(&R.full[i]);
        R.freed[i] = 0;
      }
      for (int i = 0; i < 5; ++i) R.tot[i] = 0;
      R.abort = 0;
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");  // the inits, visible to the copy engine
    }
    __syncwarp();
    const int dv = min(t.tz, L->lz - t.z0);
    const int crows = o3_class_rows(CLS) > 0 ? o3_class_rows(CLS) : min(t.ty, L->ly - t.y0) + 2;
    for (int p = 0; p < kO3RingSlots && p <= dv + 1; ++p) o3_issue_plane(t, L, R, osm, p, crows, lane);
    if (lane == 0) R.issued = min(kO3RingSlots, dv + 2);
  }
  __syncthreads();
  o3_march_tile<COLOUR, ALG, o3_class_row(CLS), o3_class_rows(CLS)>(t, L, G, ctl, osm, R);
  // the tile function ends with a CTA barrier after the last flush
  if (threadIdx.x == 0) {
    atomic_add_i64(&L->acc.mq[0], R.tot[0]);
    atomic_add_i64(&L->acc.mq[1], R.tot[1]);
    atomic_add_i64(&L->acc.mq[2], R.tot[2]);
    if (COLOUR == 1) {
      atomic_add_i64(&L->acc.ebq, R.tot[3]);
      L->acc.fresh = 1;
    }
    if (R.tot[4]) atomic_add_i64(&L->acc.accepted, R.tot[4]);
  }
  // the epilogue's scratch is the ring, whose copies have all landed
  if (COLOUR == 1) group_epilogue<true>(t.pad, lats, groups, ctl, (int*)osm);
}
#define O3_INSTANTIATE_MARCH(ALG, CLS)                                                                     \
  template __global__ void k_sweep_o3_march<0, ALG, CLS>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*); \
  template __global__ void k_sweep_o3_march<1, ALG, CLS>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
#define O3_INSTANTIATE(ALG)                                                                          \
  O3_INSTANTIATE_MARCH(ALG, 0)                                                                       \
  O3_INSTANTIATE_MARCH(ALG, 1)                                                                       \
  O3_INSTANTIATE_MARCH(ALG, 2)                                                                       \
  O3_INSTANTIATE_MARCH(ALG, 3)                                                                       \
  template __global__ void k_sweep_o3<2, 0, ALG>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);    \
  template __global__ void k_sweep_o3<2, 1, ALG>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);    \
  template __global__ void k_sweep_o3<3, 0, ALG>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);    \
  template __global__ void k_sweep_o3<3, 1, ALG>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
O3_INSTANTIATE(0)
O3_INSTANTIATE(1)
O3_INSTANTIATE(2)
O3_INSTANTIATE(3)
O3_INSTANTIATE(4)

GPUMC_BOUNDS_MODULE(sweep_o3)

}  // namespace gpumc
