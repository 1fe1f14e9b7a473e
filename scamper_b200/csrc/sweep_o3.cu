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
// Arithmetic of the Metropolis step (ALG 0, 2, 3): two sites per thread
// evaluated together with Blackwell's packed fp32 pair instructions
// (fma/add/mul.rn.f32x2: one instruction, two IEEE-rounded lane results),
// uniforms built from Philox bits (1.m - 1 with 23 bits of the word, no
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

// Metropolis step of two sites (PROP 0 cap of 1 - cos(alpha) = omc, 1
// uniform unit vector, 2 OPSS rotation with bound omc): proposals n and the
// decisions.  Per lane the operations of orc_o3_propose / orc_o3_accept.
template <int PROP>
__device__ __forceinline__ void o3_metropolis_2(f2 ax, f2 ay, f2 az, f2 hx, f2 hy, f2 hz, const uint4& oa,
                                                const uint4& ob, float omc, float mJ, float beta, f2& nx,
                                                f2& ny, f2& nz, bool& ok_a, bool& ok_b) {
  f2 px, py, pz;
  if (PROP == 0) {
    const f2 w = mul2(unit23_2(oa.x, ob.x), F2s(omc));
    const f2 ct = sub2(F2s(1.0f), w);
    const f2 s2 = fma2(mul2(w, F2s(-1.0f)), w, add2(w, w));
    const f2 st = F2(__fsqrt_rn(lo(s2)), __fsqrt_rn(hi(s2)));
    f2 cp, sp;
    sincos23_2(oa.y, ob.y, cp, sp);
    const f2 vx = mul2(st, cp), vy = mul2(st, sp);
    // Duff et al. (JCGT 2017) basis {e1, e2, a}: sg = sign(az), k = -1/(sg + az)
    const f2 sg = F2(lo(az) >= 0.0f ? 1.0f : -1.0f, hi(az) >= 0.0f ? 1.0f : -1.0f);
    const f2 d = add2(sg, az);
    const f2 k = F2(__fdiv_rn(-1.0f, lo(d)), __fdiv_rn(-1.0f, hi(d)));
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
  const f2 p = exp_neg2_2(mul2(F2s(-beta), de));
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
// site than bumping the keys every round, at the same 64 registers), and each
// round multiply one 32x32->64 wide product.
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
    const uint64_t p0 = (uint64_t)0xD2511F53u * c.x;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c.z;
    c = make_uint4((uint32_t)(p1 >> 32) ^ c.y ^ P.k0[r], (uint32_t)p1, (uint32_t)(p0 >> 32) ^ c.w ^ P.k1[r],
                   (uint32_t)p0);
  }
  return c;
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

// Updates the pair (qa, qb) of a colour pass (qb only when `two`): writes
// accepted spins in place, counts acceptances and adds the fixed-point
// observables of the final spins.
template <int COLOUR, int ALG>
__device__ __forceinline__ void o3_update_pair(const O3Site& qa, const O3Site& qb, bool two, const O3Philox& P,
                                               float omc, float mJ, float beta, float* S, float* S1, float* S2,
                                               uint32_t cs, O3Fix& fx, int& nacc) {
  const uint4 oa = o3_philox(P, qa.site);
  const uint4 ob = o3_philox(P, two ? qb.site : qa.site);
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
    o3_metropolis_2<ALG == 2 ? 1 : (ALG == 3 ? 2 : 0)>(fx2, fy2, fz2, hx, hy, hz, oa, ob, omc, mJ, beta, nx, ny, nz,
                                                        ok_a, ok_b);
    fx2 = F2(ok_a ? lo(nx) : qa.ax, ok_b ? hi(nx) : qb.ax);
    fy2 = F2(ok_a ? lo(ny) : qa.ay, ok_b ? hi(ny) : qb.ay);
    fz2 = F2(ok_a ? lo(nz) : qa.az, ok_b ? hi(nz) : qb.az);
  }
  ok_b = ok_b && two;
  if (ok_a) {
    st_chk(S, qa.me, cs, lo(fx2));
    st_chk(S1, qa.me, cs, lo(fy2));
    st_chk(S2, qa.me, cs, lo(fz2));
  }
  if (ok_b) {
    st_chk(S, qb.me, cs, hi(fx2));
    st_chk(S1, qb.me, cs, hi(fy2));
    st_chk(S2, qb.me, cs, hi(fz2));
  }
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
    if (COLOUR == 1) launch_epilogue(lats, groups, ctl);
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
  O3Fix fx = {{0, 0, 0}, 0, 0};
  O3Totals tot = {{0, 0, 0}, 0};
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
  for (int k = 0; k < n_items; k += 2) {
    int x, y, z;
    O3Site qa, qb;
    next_site(x, y, z);
    o3_load_site<DIM>(qa, S, S1, S2, x, y, z, lx, ly, lz, pitch, cs);
    const bool two = k + 1 < n_items;
    if (two) {
      next_site(x, y, z);
      o3_load_site<DIM>(qb, S, S1, S2, x, y, z, lx, ly, lz, pitch, cs);
    } else {
      qb = qa;
    }
    o3_update_pair<COLOUR, ALG>(qa, qb, two, P, omc, mJ, beta, S, S1, S2, cs, fx, nacc);
    if ((k & 62) == 62) o3_flush<COLOUR == 1>(tot, fx);  // every 64 sites: 32-bit partials stay far from overflow
  }
  o3_flush<COLOUR == 1>(tot, fx);
  o3_commit<COLOUR>(L, tot, nacc);
  if (COLOUR == 1) launch_epilogue(lats, groups, ctl);
}

// ---------------------------------------------------------------------------
// 3D colour pass marched along z through a ring of four shared-memory planes.
//
// A tile is whole rows y0 .. y0+hv-1 of planes z0 .. z0+dv-1.  Each plane the
// tile touches (z0-1 .. z0+dv) is copied once, rows y0-1 .. y0+hv with all
// three components, into a ring slot and serves as the z-1, z and z+1 plane
// of three consecutive steps; the copy of plane z+2 is in flight while plane
// z is computed.  The copies are bulk asynchronous copies (cp.async.bulk, no
// multicast) issued by one thread: per component the slot's rows are at most
// three contiguous runs of the plane (split where the rows wrap), and each
// slot's mbarrier counts the bytes in (expect_tx / complete_tx).  Plane p of
// the march (p = 0 for z0-1) goes to slot p % S as that slot's (p / S)-th
// fill (S = kO3RingSlots), so a step waits for phase parity (p / S) & 1 of its
// three slots; the copy of a plane is issued S - 3 steps before its first use.
// Every wait is bounded; one that gives up flags the launch (ctl->err), waits
// (bounded again) for the copies in flight and leaves the tile.  Every
// neighbour read is a shared-memory read.  The pass reads only the other
// colour's values (and its own sites' old values, which only this tile
// writes), so copying planes that other tiles update in place is race-free.
// The site arithmetic and its operation order are those of k_sweep_o3.
// ---------------------------------------------------------------------------
constexpr long long kRingWaitPolls = 1ll << 20;  // try_wait polls per ring wait

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
// Bounded wait for the completion of phase `parity` of a slot's mbarrier.
__device__ __forceinline__ bool ring_wait(unsigned long long* bar, uint32_t parity) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
  for (long long it = 0; it < kRingWaitPolls; ++it) {
    uint32_t done;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(done)
                 : "r"(a), "r"(parity)
                 : "memory");
    if (done) return true;
  }
  return false;
}

// Colour 1 also carries the sweep epilogue's shared memory, so three CTAs
// fit an SM: its register budget is that of three CTAs (no spills of the fp64
// neighbour sums).
template <int COLOUR, int ALG>
__global__ void __launch_bounds__(kThreads, COLOUR == 1 || kO3RingSlots > 4 ? 3 : 4)
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
  const uint32_t cs = (uint32_t)pitch * ly * lz;  // component plane stride (< 2^32 elements)
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
  float* S1 = S + (size_t)cs;
  float* S2 = S + 2 * (size_t)cs;
  constexpr int NS = kO3RingSlots;
  __shared__ __align__(8) unsigned long long ring_bar[NS];
  if (threadIdx.x == 0) {
    for (int i = 0; i < NS; ++i) ring_init(&ring_bar[i]);
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");  // the inits, visible to the copy engine
  }
  __syncthreads();
  // plane p of the march (z0 - 1 + p) into slot p % NS, by thread 0
  auto copy_plane = [&](int p) {
    if (threadIdx.x != 0) return;
    const int sl = p % NS;
    int zz = t.z0 - 1 + p;
    zz = zz < 0 ? zz + lz : (zz >= lz ? zz - lz : zz);
    ring_expect(&ring_bar[sl], (uint32_t)(3 * cstr) * 4u);
    for (int c = 0; c < 3; ++c) {
      int r = 0;
      while (r < RW) {
        int y = t.y0 - 1 + r;
        y = y < 0 ? y + ly : (y >= ly ? y - ly : y);
        const int n = min(RW - r, ly - y);  // rows contiguous up to the plane's last row
        const long long so = (long long)c * cs + ((long long)zz * ly + y) * pitch;
        const long long dof = (long long)sl * slot + (long long)c * cstr + (long long)r * pitch;
        if (GPUMC_IN(so + (long long)n * pitch - 1, 3ll * cs) && GPUMC_IN(dof + (long long)n * pitch - 1, (long long)NS * slot))
          ring_bulk_copy(osm + dof, S + so, (uint32_t)(n * pitch) * 4u, &ring_bar[sl]);
        r += n;
      }
    }
  };
  O3Fix fx = {{0, 0, 0}, 0, 0};
  O3Totals tot = {{0, 0, 0}, 0};
  int nacc = 0;
  // Work items are pairs of horizontally adjacent sites of the colour in one
  // row (x and x + 2, x = 4m + parity): both sites' neighbours then sit at
  // fixed offsets from one row position (the x + 1 site is shared), and a
  // thread's pair is found once per tile, not per plane.
  const int half = lx >> 1;             // sites of the colour per row
  const int np = (half + 1) >> 1;       // pairs per row (the last may be single)
  const int n_pairs = hv * np;          // pairs of the tile's rows in one plane
  const int r0 = threadIdx.x / np, m0 = threadIdx.x - r0 * np;
  const int dr = kThreads / np, dm = kThreads - dr * np;  // cursor step of kThreads pairs
  int issued = 0;  // planes whose copies were issued: march planes 0 .. dv + 1 in all
  for (; issued <= NS - 2 && issued <= dv + 1; ++issued) copy_plane(issued);
  bool ok_ring = true;
  for (int k = 0; k < dv && ok_ring; ++k) {
    const int z = t.z0 + k;
    // plane z+2 (needed as z+1 of the next step) into the slot freed by the
    // previous step
    if (k + NS - 1 <= dv + 1) {
      copy_plane(k + NS - 1);
      issued = k + NS;
    }
    // planes z-1, z, z+1 = march planes k, k+1, k+2
    for (int i = 0; i < 3 && ok_ring; ++i)
      ok_ring = ring_wait(&ring_bar[(k + i) % NS], (uint32_t)((k + i) / NS) & 1u);
    ok_ring = __syncthreads_and(ok_ring) != 0;  // one decision for the whole CTA
    if (!ok_ring) break;
    const float* pm = osm + (k % NS) * slot;
    const float* pc = osm + ((k + 1) % NS) * slot;
    const float* pp = osm + ((k + 2) % NS) * slot;
    int rl = r0, m = m0;
    for (int i = threadIdx.x; i < n_pairs; i += kThreads) {
      const int y = t.y0 + rl;
      const int xa = 4 * m + ((y + z + COLOUR) & 1), xb = xa + 2;
      const bool two = 2 * m + 1 < half;
      const int oc = (rl + 1) * pitch;  // slot row of y
      // x-1 of a and x+1 of b wrap at the row's ends; x+1 of a = x-1 of b
      // (x+1 of a wraps only for a single last site, x = lx - 1)
      const int xam = xa ? xa - 1 : lx - 1;
      const int xap = xa + 1 < lx ? xa + 1 : 0;
      const int xbp = xb + 1 < lx ? xb + 1 : 0;
      O3Site qa, qb;
      float ha[3], hb[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float* P = pc + c * cstr;
        const float* M = pm + c * cstr;
        const float* Q = pp + c * cstr;
        const float mid = ld_chk(P, oc + xap, cstr);
        // neighbour order x-1, x+1, y-1, y+1, z-1, z+1 (as k_sweep_o3)
        ha[c] = fadd(fadd(fadd(fadd(fadd(ld_chk(P, oc + xam, cstr), mid), ld_chk(P, oc - pitch + xa, cstr)),
                                ld_chk(P, oc + pitch + xa, cstr)),
                           ld_chk(M, oc + xa, cstr)),
                      ld_chk(Q, oc + xa, cstr));
        if (two)
          hb[c] = fadd(fadd(fadd(fadd(fadd(mid, ld_chk(P, oc + xbp, cstr)), ld_chk(P, oc - pitch + xb, cstr)),
                                  ld_chk(P, oc + pitch + xb, cstr)),
                             ld_chk(M, oc + xb, cstr)),
                        ld_chk(Q, oc + xb, cstr));
        else
          hb[c] = ha[c];
      }
      qa.ax = ld_chk(pc, oc + xa, cstr);
      qa.ay = ld_chk(pc + cstr, oc + xa, cstr);
      qa.az = ld_chk(pc + 2 * cstr, oc + xa, cstr);
      qa.hx = ha[0];
      qa.hy = ha[1];
      qa.hz = ha[2];
      // 32-bit index arithmetic: the same values as the 64-bit products
      // truncated to the 32-bit fields
      const uint32_t row = (uint32_t)z * (uint32_t)ly + (uint32_t)y;
      qa.me = row * (uint32_t)pitch + (uint32_t)xa;
      qa.site = row * (uint32_t)lx + (uint32_t)xa;
      if (two) {
        qb.ax = ld_chk(pc, oc + xb, cstr);
        qb.ay = ld_chk(pc + cstr, oc + xb, cstr);
        qb.az = ld_chk(pc + 2 * cstr, oc + xb, cstr);
        qb.me = qa.me + 2;
        qb.site = qa.site + 2;
      } else {
        qb.ax = qa.ax;
        qb.ay = qa.ay;
        qb.az = qa.az;
        qb.me = qa.me;
        qb.site = qa.site;
      }
      qb.hx = hb[0];
      qb.hy = hb[1];
      qb.hz = hb[2];
      o3_update_pair<COLOUR, ALG>(qa, qb, two, P, omc, mJ, beta, S, S1, S2, cs, fx, nacc);
      rl += dr;
      m += dm;
      if (m >= np) {
        m -= np;
        rl += 1;
      }
    }
    o3_flush<COLOUR == 1>(tot, fx);  // per plane: at most one pair per thread per 256 pairs since the last flush
    __syncthreads();  // the next copy overwrites the z-1 slot read above
  }
  if (!ok_ring) {
    // a copy did not land in time: flag the launch, wait (bounded) for every
    // copy still in flight into this CTA's ring, and leave the tile
    atomicExch(&ctl->err, 2);
    for (int p = max(0, issued - NS); p < issued; ++p) ring_wait(&ring_bar[p % NS], (uint32_t)(p / NS) & 1u);
  }
  o3_commit<COLOUR>(L, tot, nacc);
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

GPUMC_BOUNDS_MODULE(sweep_o3)

}  // namespace gpumc
