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
// Proposal: a uniform point on the spherical cap of half-angle alpha around
// the current spin (w = 1 - cos(alpha) stored per lattice, adapted toward 50 %
// acceptance during thermalisation only, mirroring the adaptation contract of
// the reference's OPSSStrategy, CMC.rs/src/lattice/proposal.rs:72-167).  The
// cap proposal is symmetric, so acceptance is min(1, exp(-beta dE)) with
// dE = -J (s' - s) . h, h the sum of the neighbour spins
// (ONModel::bond_energy, CMC.rs/src/lattice/models.rs:440-452).
//
// Every fp32 operation is an explicitly rounded intrinsic and exp / sin / cos
// are the engine's own polynomials, so a CPU replay in the same operation
// order reproduces the device trajectory bit for bit.
#include "device_common.cuh"
#include "epilogue.cuh"

namespace gpumc {

__device__ __forceinline__ bool o3_update(float ax, float ay, float az, float hx, float hy,
                                          float hz, uint4 o, float omc, float mJ, float beta,
                                          float& nx, float& ny, float& nz, float& dE) {
  const float w = fmul(fmul((float)(o.x >> 8), 0x1p-24f), omc);
  const float ct = fsub(1.0f, w);
  const float st = fsqrt(fmul(w, fsub(2.0f, w)));
  float cp, sp;
  sincos_turn(o.y, cp, sp);
  float e1x, e1y, e1z;
  if (fabsf(az) < 0.9f) {
    const float a = fsqrt(fadd(fmul(ax, ax), fmul(ay, ay)));
    e1x = fdiv(ay, a);
    e1y = fdiv(-ax, a);
    e1z = 0.0f;
  } else {
    const float a = fsqrt(fadd(fmul(ay, ay), fmul(az, az)));
    e1x = 0.0f;
    e1y = fdiv(az, a);
    e1z = fdiv(-ay, a);
  }
  const float e2x = fsub(fmul(ay, e1z), fmul(az, e1y));
  const float e2y = fsub(fmul(az, e1x), fmul(ax, e1z));
  const float e2z = fsub(fmul(ax, e1y), fmul(ay, e1x));
  float px = fadd(fmul(ct, ax), fmul(st, fadd(fmul(cp, e1x), fmul(sp, e2x))));
  float py = fadd(fmul(ct, ay), fmul(st, fadd(fmul(cp, e1y), fmul(sp, e2y))));
  float pz = fadd(fmul(ct, az), fmul(st, fadd(fmul(cp, e1z), fmul(sp, e2z))));
  const float r = fsqrt(fadd(fadd(fmul(px, px), fmul(py, py)), fmul(pz, pz)));
  px = fdiv(px, r);
  py = fdiv(py, r);
  pz = fdiv(pz, r);
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

// Philox4x32-10 of counter (site, colour | TAG_O3 << 1, sweep) with the
// sweep-uniform part of round 1 and the bumped keys precomputed.
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
  uint4 c = make_uint4(P.a, P.b, __umulhi(0xD2511F53u, index) ^ P.c, 0xD2511F53u * index);
#pragma unroll
  for (int r = 1; r < 10; ++r) {
    const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
    const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
    c = make_uint4(hi1 ^ c.y ^ P.k0[r], lo1, hi0 ^ c.w ^ P.k1[r], lo0);
  }
  return c;
}

// One colour pass over a tile of full rows (y0 .. y0+hv-1, planes z0 ..
// z0+dv-1), one thread per site of the colour.
template <int DIM, int COLOUR>
__global__ void __launch_bounds__(kThreads, 3)
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
  const double Jd = G->J;
  const float omc = L->omc;
  const O3Philox P = make_o3_philox(L->key, sweep, (uint32_t)COLOUR | (TAG_O3 << 1));
  const int hv = min(L->tile_y, ly - t.y0);
  const int dv = DIM == 3 ? min(L->tile_z, lz - t.z0) : 1;
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
  double dE = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
  int nacc = 0;
  if (r0 < rstep) {
    for (int r = r0; r < rows; r += rstep) {
      const int y = t.y0 + (DIM == 3 ? r % hv : r);
      const int z = DIM == 3 ? t.z0 + r / hv : 0;
      const uint32_t rowoff = ((uint32_t)z * ly + y) * (uint32_t)pitch;
      const int ym = y ? y - 1 : ly - 1, yp = y + 1 < ly ? y + 1 : 0;
      const uint32_t rm = ((uint32_t)z * ly + ym) * (uint32_t)pitch;
      const uint32_t rp = ((uint32_t)z * ly + yp) * (uint32_t)pitch;
      uint32_t zmo = 0, zpo = 0;
      if (DIM == 3) {
        const int zm = z ? z - 1 : lz - 1, zp = z + 1 < lz ? z + 1 : 0;
        zmo = ((uint32_t)zm * ly + y) * (uint32_t)pitch;
        zpo = ((uint32_t)zp * ly + y) * (uint32_t)pitch;
      }
      const int par = (y + z + COLOUR) & 1;
      for (int c = col0; c < half; c += cstep) {
        const int x = 2 * c + par;
        const int xm = x ? x - 1 : lx - 1, xp = x + 1 < lx ? x + 1 : 0;
        // neighbour sum in the fixed order x-1, x+1, y-1, y+1, z-1, z+1
        const uint32_t nb[6] = {rowoff + xm, rowoff + xp, rm + x, rp + x, zmo + x, zpo + x};
        float hx = __ldg(Sr + nb[0]), hy = __ldg(Sr1 + nb[0]), hz = __ldg(Sr2 + nb[0]);
#pragma unroll
        for (int i = 1; i < 2 * DIM; ++i) {
          hx = fadd(hx, __ldg(Sr + nb[i]));
          hy = fadd(hy, __ldg(Sr1 + nb[i]));
          hz = fadd(hz, __ldg(Sr2 + nb[i]));
        }
        const uint32_t me = rowoff + x;
        const float ax = S[me], ay = S1[me], az = S2[me];
        const uint32_t site = (uint32_t)((size_t)(z * ly + y) * lx + x);
        float nx, ny, nz, de;
        const bool ok = o3_update(ax, ay, az, hx, hy, hz, o3_philox(P, site), omc, mJ, beta, nx, ny,
                                  nz, de);
        float fx = ax, fy = ay, fz = az;
        if (ok) {
          // energy cache: exact fp64 change of the fp32 configuration (the
          // decision used the fp32 dE)
          double hxd = 0.0, hyd = 0.0, hzd = 0.0;
#pragma unroll
          for (int i = 0; i < 2 * DIM; ++i) {
            hxd += (double)__ldg(Sr + nb[i]);
            hyd += (double)__ldg(Sr1 + nb[i]);
            hzd += (double)__ldg(Sr2 + nb[i]);
          }
          dE += -Jd * (((double)nx - (double)ax) * hxd + ((double)ny - (double)ay) * hyd +
                       ((double)nz - (double)az) * hzd);
          ++nacc;
          fx = nx;
          fy = ny;
          fz = nz;
          S[me] = fx;
          S1[me] = fy;
          S2[me] = fz;
        }
        mx += (double)fx;
        my += (double)fy;
        mz += (double)fz;
      }
    }
  }
  const unsigned full = 0xFFFFFFFFu;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    dE += __shfl_xor_sync(full, dE, o);
    nacc += __shfl_xor_sync(full, nacc, o);
    mx += __shfl_xor_sync(full, mx, o);
    my += __shfl_xor_sync(full, my, o);
    mz += __shfl_xor_sync(full, mz, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&L->acc.dEf, dE);
    atomicAdd(&L->acc.mx, mx);
    atomicAdd(&L->acc.my, my);
    atomicAdd(&L->acc.mz, mz);
    if (nacc) atomic_add_i64(&L->acc.accepted, nacc);
  }
  if (COLOUR == 1) launch_epilogue(lats, groups, ctl);
}

template __global__ void k_sweep_o3<2, 0>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template __global__ void k_sweep_o3<2, 1>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template __global__ void k_sweep_o3<3, 0>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template __global__ void k_sweep_o3<3, 1>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);

}  // namespace gpumc
