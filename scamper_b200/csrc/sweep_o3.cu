// Fused two-colour checkerboard sweep for O(3) Heisenberg spins (float32 unit
// vectors, three component planes) on periodic square and cubic lattices.
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

constexpr int kO3MaxItems = 6;

struct O3Geom {
  int x0, Wv, S, R, hv;  // S = row stride (floats), R = rows per plane buffer
};

struct O3Site {
  float x, y, z;
};

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

// Shared-memory plane: three component planes of R rows x S floats; logical
// position x maps to column x - x0 + 2.
__device__ __forceinline__ void o3_load_plane(float* pl, int plane_floats, const float* src,
                                              size_t comp_stride, int pitch, int lx, int ly,
                                              int y0, int z, const O3Geom& g) {
  const int cols = g.Wv + 4;
  for (int i = threadIdx.x; i < g.R * cols; i += kThreads) {
    const int r = i / cols, c = i - r * cols;
    const int y = wrapi(y0 - 2 + r, ly);
    const int x = wrapi(g.x0 - 2 + c, lx);
    const size_t off = ((size_t)z * ly + y) * (size_t)pitch + x;
    pl[r * g.S + c] = src[off];
    pl[plane_floats + r * g.S + c] = src[comp_stride + off];
    pl[2 * plane_floats + r * g.S + c] = src[2 * comp_stride + off];
  }
}

template <int DIM>
__device__ __forceinline__ void o3_pass(float* pl, const float* pzm, const float* pzp,
                                        int plane_floats, const O3Geom& g, int colour, int y0,
                                        int z, int ly, int lx, int pitch, uint64_t key,
                                        uint64_t sweep, float omc, float mJ, float beta,
                                        double Jd, bool owned_plane, float* dst, size_t comp_stride,
                                        double& dEsum, int& nacc, double& mx, double& my,
                                        double& mz) {
  // colour 0 covers rows [1, R-1) and positions [x0-1, x0+Wv]; colour 1 the tile
  const int rlo = colour == 0 ? 1 : 2;
  const int nrows = colour == 0 ? g.hv + 2 : g.hv;
  const int xlo = colour == 0 ? g.x0 - 1 : g.x0;
  const int half = colour == 0 ? (g.Wv + 2) / 2 : g.Wv / 2;
  const int nitems = nrows * half;
  float rx[kO3MaxItems], ry[kO3MaxItems], rz[kO3MaxItems];
  int roff[kO3MaxItems];
#pragma unroll
  for (int it = 0; it < kO3MaxItems; ++it) {
    roff[it] = -1;
    const int i = threadIdx.x + it * kThreads;
    if (i < nitems) {
      const int r = rlo + i / half;
      const int k = i - (r - rlo) * half;
      const int y = wrapi(y0 - 2 + r, ly);
      const int par = ((xlo + y + z + colour) & 1);
      const int pos = xlo + 2 * k + par;
      const int c = pos - g.x0 + 2;
      const int off = r * g.S + c;
      const float* P0 = pl;
      const float* P1 = pl + plane_floats;
      const float* P2 = pl + 2 * plane_floats;
      float hx = P0[off - 1], hy = P1[off - 1], hz = P2[off - 1];
      hx = fadd(hx, P0[off + 1]); hy = fadd(hy, P1[off + 1]); hz = fadd(hz, P2[off + 1]);
      hx = fadd(hx, P0[off - g.S]); hy = fadd(hy, P1[off - g.S]); hz = fadd(hz, P2[off - g.S]);
      hx = fadd(hx, P0[off + g.S]); hy = fadd(hy, P1[off + g.S]); hz = fadd(hz, P2[off + g.S]);
      if (DIM == 3) {
        hx = fadd(hx, pzm[off]);
        hy = fadd(hy, pzm[plane_floats + off]);
        hz = fadd(hz, pzm[2 * plane_floats + off]);
        hx = fadd(hx, pzp[off]);
        hy = fadd(hy, pzp[plane_floats + off]);
        hz = fadd(hz, pzp[2 * plane_floats + off]);
      }
      const float ax = P0[off], ay = P1[off], az = P2[off];
      const int xr = wrapi(pos, lx);
      const uint64_t site = ((uint64_t)z * ly + y) * (uint64_t)lx + (uint64_t)xr;
      const uint4 o = draw(key, site, (uint32_t)colour, TAG_O3, 0, sweep);
      float nx, ny, nz, de;
      const bool ok = o3_update(ax, ay, az, hx, hy, hz, o, omc, mJ, beta, nx, ny, nz, de);
      const bool owned = owned_plane && r >= 2 && r < 2 + g.hv && pos >= g.x0 && pos < g.x0 + g.Wv;
      float fx = ax, fy = ay, fz = az;
      if (ok) {
        fx = nx; fy = ny; fz = nz;
        if (owned) {
          // energy cache: exact fp64 change of the fp32 configuration (the
          // decision above used the fp32 dE)
          double hxd = (double)P0[off - 1] + (double)P0[off + 1] + (double)P0[off - g.S] + (double)P0[off + g.S];
          double hyd = (double)P1[off - 1] + (double)P1[off + 1] + (double)P1[off - g.S] + (double)P1[off + g.S];
          double hzd = (double)P2[off - 1] + (double)P2[off + 1] + (double)P2[off - g.S] + (double)P2[off + g.S];
          if (DIM == 3) {
            hxd += (double)pzm[off] + (double)pzp[off];
            hyd += (double)pzm[plane_floats + off] + (double)pzp[plane_floats + off];
            hzd += (double)pzm[2 * plane_floats + off] + (double)pzp[2 * plane_floats + off];
          }
          dEsum += -(double)Jd * (((double)nx - (double)ax) * hxd + ((double)ny - (double)ay) * hyd +
                                  ((double)nz - (double)az) * hzd);
          ++nacc;
        }
      }
      rx[it] = fx; ry[it] = fy; rz[it] = fz;
      roff[it] = off;
      if (owned) {
        const size_t goff = ((size_t)z * ly + y) * (size_t)pitch + xr;
        dst[goff] = fx;
        dst[comp_stride + goff] = fy;
        dst[2 * comp_stride + goff] = fz;
        mx += (double)fx;
        my += (double)fy;
        mz += (double)fz;
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < kO3MaxItems; ++it) {
    if (roff[it] >= 0) {
      pl[roff[it]] = rx[it];
      pl[plane_floats + roff[it]] = ry[it];
      pl[2 * plane_floats + roff[it]] = rz[it];
    }
  }
  __syncthreads();
}

__device__ __forceinline__ void o3_flush(LatDesc* L, double dE, int nacc, double mx, double my,
                                         double mz) {
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
}

template <int DIM>
__global__ void __launch_bounds__(kThreads)
    k_sweep_o3(const TileItem* __restrict__ tiles, LatDesc* __restrict__ lats,
               GroupDesc* __restrict__ groups, LaunchCtl* __restrict__ ctl) {
  extern __shared__ __align__(16) float fsm[];
  const TileItem t = tiles[blockIdx.x];
  LatDesc* L = &lats[t.lat];
  const GroupDesc* G = &groups[L->group];
  const uint64_t sweep = L->sweep;
  if (sweep >= L->target) {
    launch_epilogue(lats, groups, ctl);
    return;
  }
  const int lx = L->lx, ly = L->ly, lz = DIM == 3 ? L->lz : 1, pitch = L->pitch;
  const uint64_t key = L->key;
  const size_t comp_stride = (size_t)pitch * ly * lz;
  const float* cur = (const float*)L->buf[sweep & 1];
  float* nxt = (float*)L->buf[(sweep & 1) ^ 1];
  const int label = G->label[L->replica];
  const float beta = G->betas_f[label];
  const float mJ = -G->Jf;
  const float omc = L->omc;
  O3Geom g;
  g.x0 = t.x0;
  g.Wv = min(L->tile_cx * 4, lx - t.x0);
  g.hv = min(L->tile_y, ly - t.y0);
  g.S = g.Wv + 4;
  g.R = g.hv + 4;
  const int plane_floats = g.R * g.S;
  double dE = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
  int nacc = 0;
  if (DIM == 2) {
    o3_load_plane(fsm, plane_floats, cur, comp_stride, pitch, lx, ly, t.y0, 0, g);
    __syncthreads();
    o3_pass<2>(fsm, fsm, fsm, plane_floats, g, 0, t.y0, 0, ly, lx, pitch, key, sweep, omc, mJ,
               beta, G->J, true, nxt, comp_stride, dE, nacc, mx, my, mz);
    o3_pass<2>(fsm, fsm, fsm, plane_floats, g, 1, t.y0, 0, ly, lx, pitch, key, sweep, omc, mJ,
               beta, G->J, true, nxt, comp_stride, dE, nacc, mx, my, mz);
  } else {
    const int dv = min(L->tile_z, lz - t.z0);
    const int slot_floats = 3 * plane_floats;
    for (int s = 0; s < dv + 4; ++s) {
      const int zl = t.z0 - 2 + s;
      float* pl = fsm + (s & 3) * slot_floats;
      o3_load_plane(pl, plane_floats, cur, comp_stride, pitch, lx, ly, t.y0, wrapi(zl, lz), g);
      __syncthreads();
      if (s >= 2) {
        const int zb = zl - 1;
        o3_pass<3>(fsm + ((s - 1) & 3) * slot_floats, fsm + ((s - 2) & 3) * slot_floats, pl,
                   plane_floats, g, 0, t.y0, wrapi(zb, lz), ly, lx, pitch, key, sweep, omc, mJ,
                   beta, G->J, zb >= t.z0 && zb < t.z0 + dv, nxt, comp_stride, dE, nacc, mx, my, mz);
      }
      if (s >= 4) {
        const int zw = zl - 2;
        o3_pass<3>(fsm + ((s - 2) & 3) * slot_floats, fsm + ((s - 3) & 3) * slot_floats,
                   fsm + ((s - 1) & 3) * slot_floats, plane_floats, g, 1, t.y0, wrapi(zw, lz), ly,
                   lx, pitch, key, sweep, omc, mJ, beta, G->J, true, nxt, comp_stride, dE, nacc, mx,
                   my, mz);
      }
      __syncthreads();
    }
  }
  o3_flush(L, dE, nacc, mx, my, mz);
  launch_epilogue(lats, groups, ctl);
}

template __global__ void k_sweep_o3<2>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template __global__ void k_sweep_o3<3>(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);

}  // namespace gpumc
