// Initial states, exact energy recomputation (the reference's
// System::recompute_energy / audit_lattice_cache, CMC.rs/src/lattice/
// state.rs:75-78 and CMC.rs/src/audit.rs:41-52) and helpers used by the host
// engine outside the sweep.
#include "device_common.cuh"

namespace gpumc {

// Hot start: site s takes word (s & 3) of the Philox block (s >> 2) of its
// replica's initialisation stream.  Ising: spin +1 iff the top bit is set;
// Potts: floor(u * q / 2^32).  Cold start: all +1 / all state 0.
__global__ void k_init_discrete(int8_t* buf, int model, int lx, int ly, int lz, int pitch, int q,
                                uint64_t key, int hot) {
  const long long n = (long long)lx * ly * lz;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n; s += stride) {
    const int x = (int)(s % lx);
    const long long rho = s / lx;
    int8_t v;
    if (!hot) {
      v = model == ISING ? 1 : 0;
    } else {
      const uint4 o = draw(key, (uint64_t)s >> 2, 0u, TAG_INIT, 0u, 0ull);
      const uint32_t u = (s & 3) == 0 ? o.x : (s & 3) == 1 ? o.y : (s & 3) == 2 ? o.z : o.w;
      v = model == ISING ? ((u >> 31) ? 1 : -1)
                         : (int8_t)(((unsigned long long)u * (unsigned long long)q) >> 32);
    }
    buf[rho * pitch + x] = v;
  }
}

// O(3) hot start: z uniform in (-1, 1], azimuth uniform, in the engine's
// exactly rounded arithmetic.  Cold start: (1, 0, 0) as the reference's
// ONModel::ordered_spin.
__global__ void k_init_o3(float* buf, int lx, int ly, int lz, int pitch, uint64_t key, int hot) {
  const long long n = (long long)lx * ly * lz;
  const size_t comp = (size_t)pitch * ly * lz;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n; s += stride) {
    const int x = (int)(s % lx);
    const long long rho = s / lx;
    const size_t off = (size_t)rho * pitch + x;
    if (!hot) {
      buf[off] = 1.0f;
      buf[comp + off] = 0.0f;
      buf[2 * comp + off] = 0.0f;
      continue;
    }
    const uint4 o = draw(key, (uint64_t)s, 0u, TAG_INIT, 0u, 0ull);
    const float t = fmul((float)(o.x >> 8), 0x1p-24f);
    const float zz = fsub(1.0f, fmul(2.0f, t));
    const float r = fsqrt(fmul(fsub(1.0f, zz), fadd(1.0f, zz)));
    float c, sn;
    sincos_turn(o.y, c, sn);
    buf[off] = fmul(r, c);
    buf[comp + off] = fmul(r, sn);
    buf[2 * comp + off] = zz;
  }
}

// Multi-spin hot start: bit r of every word is replica r's own Ising hot start
// (keys[r] = replica r's initialisation stream).
__global__ void k_init_msc(unsigned long long* buf, int lx, int ly, int lz, int pitch,
                           const uint64_t* keys, int hot) {
  const long long n = (long long)lx * ly * lz;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n; s += stride) {
    const int x = (int)(s % lx);
    const long long rho = s / lx;
    unsigned long long w = ~0ull;
    if (hot) {
      w = 0;
      for (int r = 0; r < 64; ++r) {
        const uint4 o = draw(keys[r], (uint64_t)s >> 2, 0u, TAG_INIT, 0u, 0ull);
        const uint32_t u = (s & 3) == 0 ? o.x : (s & 3) == 1 ? o.y : (s & 3) == 2 ? o.z : o.w;
        w |= (unsigned long long)(u >> 31) << r;
      }
    }
    buf[rho * pitch + x] = w;
  }
}

// Exact integer energy (units of J) over the +x/+y/+z bonds.  For the
// multi-spin model: the joint energy of all 64 replicas.
__global__ void k_energy_int(const void* buf, int model, int lx, int ly, int lz, int pitch,
                             unsigned long long* out) {
  const long long n = (long long)lx * ly * lz;
  const long long stride = (long long)gridDim.x * blockDim.x;
  long long e = 0;
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n; s += stride) {
    const int x = (int)(s % lx);
    const long long rho = s / lx;
    const int y = (int)(rho % ly);
    const int z = (int)(rho / ly);
    const int xp = x + 1 < lx ? x + 1 : 0, yp = y + 1 < ly ? y + 1 : 0, zp = z + 1 < lz ? z + 1 : 0;
    const long long o0 = rho * pitch + x;
    const long long o1 = rho * pitch + xp;
    const long long o2 = ((long long)z * ly + yp) * pitch + x;
    const long long o3 = ((long long)zp * ly + y) * pitch + x;
    if (model == MSC) {
      const unsigned long long* w = (const unsigned long long*)buf;
      const unsigned long long a = w[o0];
      int anti = __popcll(a ^ w[o1]) + __popcll(a ^ w[o2]);
      int bonds = 128;
      if (lz > 1) {
        anti += __popcll(a ^ w[o3]);
        bonds += 64;
      }
      e -= (long long)(bonds - 2 * anti);
    } else {
      const int8_t* b = (const int8_t*)buf;
      const int8_t a = b[o0];
      if (model == ISING) {
        e -= (long long)a * b[o1] + (long long)a * b[o2];
        if (lz > 1) e -= (long long)a * b[o3];
      } else {
        e -= (long long)(a == b[o1]) + (long long)(a == b[o2]);
        if (lz > 1) e -= (long long)(a == b[o3]);
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xFFFFFFFFu, e, o);
  if ((threadIdx.x & 31) == 0 && e) atomicAdd(out, (unsigned long long)e);
}

__global__ void k_energy_o3(const float* buf, int lx, int ly, int lz, int pitch, double J,
                            double* out) {
  const long long n = (long long)lx * ly * lz;
  const size_t comp = (size_t)pitch * ly * lz;
  const long long stride = (long long)gridDim.x * blockDim.x;
  double e = 0.0;
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n; s += stride) {
    const int x = (int)(s % lx);
    const long long rho = s / lx;
    const int y = (int)(rho % ly);
    const int z = (int)(rho / ly);
    const int xp = x + 1 < lx ? x + 1 : 0, yp = y + 1 < ly ? y + 1 : 0, zp = z + 1 < lz ? z + 1 : 0;
    const size_t o0 = rho * pitch + x;
    size_t nb[3] = {(size_t)(rho * pitch + xp), (size_t)(((long long)z * ly + yp) * pitch + x),
                    (size_t)(((long long)zp * ly + y) * pitch + x)};
    const int nn = lz > 1 ? 3 : 2;
    for (int i = 0; i < nn; ++i)
      e -= J * ((double)buf[o0] * buf[nb[i]] + (double)buf[comp + o0] * buf[comp + nb[i]] +
                (double)buf[2 * comp + o0] * buf[2 * comp + nb[i]]);
  }
  for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xFFFFFFFFu, e, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, e);
}

// Device self-check of the random stream: Philox4x32-10 outputs for given
// counters/keys (compared on the host against the oracle and the published
// known-answer vectors).
__global__ void k_philox_probe(const uint4* ctr, const uint2* key, uint4* out, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = philox10(ctr[i], key[i].x, key[i].y);
}

}  // namespace gpumc
