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

// Exact integer energy (units of J) over the +x/+y/+z bonds of an int8
// lattice (Ising: -sum s_i s_j; Potts: -sum delta(s_i, s_j)), with the
// reference's spin validation (validate_spin, CMC.rs/src/lattice/
// state.rs:114-124) folded in: `bad` counts 16-site chunks holding a value
// that is not +-1 (Ising) or not in [0, q) (Potts).
//
// Work is split into (row, 16-site chunk) items; a chunk is one 16-byte load
// of its row, of the row above (+y) and of the next plane (+z), and its +x
// neighbours are the same bytes shifted by one with the next chunk's first
// byte (or the row's first byte at the periodic edge).  Ising products of
// +-1 bytes are summed four at a time with dp4a; Potts counts equal bytes
// with a carry-free zero-byte test.
__device__ __forceinline__ uint32_t equal_bytes(uint32_t a, uint32_t b) {
  const uint32_t t = a ^ b;
  return __popc(~(((t & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | t | 0x7F7F7F7Fu));
}

__device__ __forceinline__ bool bad_word(uint32_t w, int model, uint32_t qk) {
  if (model == ISING) return w != (0x01010101u | (((w >> 7) & 0x01010101u) * 0xFEu));
  return ((((w & 0x7F7F7F7Fu) + qk) | w) & 0x80808080u) != 0u;  // byte < 0 or >= q
}

__device__ __forceinline__ int bond_i8(int model, int8_t a, int8_t b) {
  return model == ISING ? (int)a * (int)b : (int)(a == b);
}

__device__ __forceinline__ void energy_chunk_i8(const int8_t* __restrict__ buf, int model, int q,
                                                uint32_t qk, int lx, int ly, int lz, int pitch,
                                                uint32_t row, int c, long long& e, uint32_t& bad) {
  const uint32_t y = row % (uint32_t)ly, z = row / (uint32_t)ly;
  const uint32_t yp = y + 1 < (uint32_t)ly ? y + 1 : 0, zp = z + 1 < (uint32_t)lz ? z + 1 : 0;
  const int8_t* r0 = buf + (size_t)row * pitch;
  const int8_t* ry = buf + ((size_t)z * ly + yp) * pitch;
  const int8_t* rz = buf + ((size_t)zp * ly + y) * pitch;
  const int x0 = 16 * c;
  if (x0 + 16 <= lx) {
    const uint4 a = *(const uint4*)(r0 + x0);
    const uint4 b = *(const uint4*)(ry + x0);
    const uint32_t nb = (uint32_t)(uint8_t)(x0 + 16 < lx ? r0[x0 + 16] : r0[0]);
    const uint4 sx = make_uint4(__funnelshift_r(a.x, a.y, 8), __funnelshift_r(a.y, a.z, 8),
                                __funnelshift_r(a.z, a.w, 8), __funnelshift_r(a.w, nb, 8));
    uint4 cz = make_uint4(0, 0, 0, 0);
    if (lz > 1) cz = *(const uint4*)(rz + x0);
    if (model == ISING) {
      int s = __dp4a((int)a.x, (int)sx.x, 0);
      s = __dp4a((int)a.y, (int)sx.y, s);
      s = __dp4a((int)a.z, (int)sx.z, s);
      s = __dp4a((int)a.w, (int)sx.w, s);
      s = __dp4a((int)a.x, (int)b.x, s);
      s = __dp4a((int)a.y, (int)b.y, s);
      s = __dp4a((int)a.z, (int)b.z, s);
      s = __dp4a((int)a.w, (int)b.w, s);
      if (lz > 1) {
        s = __dp4a((int)a.x, (int)cz.x, s);
        s = __dp4a((int)a.y, (int)cz.y, s);
        s = __dp4a((int)a.z, (int)cz.z, s);
        s = __dp4a((int)a.w, (int)cz.w, s);
      }
      e -= s;
    } else {
      uint32_t s = equal_bytes(a.x, sx.x) + equal_bytes(a.y, sx.y) + equal_bytes(a.z, sx.z) +
                   equal_bytes(a.w, sx.w) + equal_bytes(a.x, b.x) + equal_bytes(a.y, b.y) +
                   equal_bytes(a.z, b.z) + equal_bytes(a.w, b.w);
      if (lz > 1)
        s += equal_bytes(a.x, cz.x) + equal_bytes(a.y, cz.y) + equal_bytes(a.z, cz.z) + equal_bytes(a.w, cz.w);
      e -= (long long)s;
    }
    bad += (bad_word(a.x, model, qk) || bad_word(a.y, model, qk) || bad_word(a.z, model, qk) ||
            bad_word(a.w, model, qk)) ? 1u : 0u;
  } else {
    // ragged last chunk of a row whose length is not a multiple of 16
    for (int x = x0; x < lx; ++x) {
      const int8_t a = r0[x];
      int s = bond_i8(model, a, r0[x + 1 < lx ? x + 1 : 0]) + bond_i8(model, a, ry[x]);
      if (lz > 1) s += bond_i8(model, a, rz[x]);
      e -= s;
      const bool ok = model == ISING ? (a == 1 || a == -1) : (a >= 0 && a < q);
      bad += ok ? 0u : 1u;
    }
  }
}

__global__ void __launch_bounds__(256)
    k_energy_i8(const int8_t* __restrict__ buf, int model, int q, int lx, int ly, int lz, int pitch,
                unsigned long long* e_out, unsigned int* bad_out) {
  const int nch = (lx + 15) >> 4;
  const uint32_t rows = (uint32_t)ly * (uint32_t)lz;
  const uint32_t qk = (uint32_t)(0x80 - q) * 0x01010101u;
  long long e = 0;
  uint32_t bad = 0;
  if (nch <= (int)blockDim.x) {
    // several rows per block step: thread t takes chunk t % nch of row t / nch
    const uint32_t rpi = blockDim.x / nch;
    const uint32_t my_r = threadIdx.x / nch, my_c = threadIdx.x % nch;
    if (my_r < rpi)
      for (uint32_t row = blockIdx.x * rpi + my_r; row < rows; row += gridDim.x * rpi)
        energy_chunk_i8(buf, model, q, qk, lx, ly, lz, pitch, row, (int)my_c, e, bad);
  } else {
    for (uint32_t row = blockIdx.x; row < rows; row += gridDim.x)
      for (int c = threadIdx.x; c < nch; c += blockDim.x)
        energy_chunk_i8(buf, model, q, qk, lx, ly, lz, pitch, row, c, e, bad);
  }
  for (int o = 16; o > 0; o >>= 1) {
    e += __shfl_xor_sync(0xFFFFFFFFu, e, o);
    bad += __shfl_xor_sync(0xFFFFFFFFu, bad, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (e) atomicAdd(e_out, (unsigned long long)e);
    if (bad && bad_out) atomicAdd(bad_out, bad);
  }
}

// Joint energy of the 64 replicas of a multi-spin lattice (units of J):
// each bond contributes -(64 - 2 popcount(a ^ b)).
__global__ void __launch_bounds__(256)
    k_energy_msc(const unsigned long long* __restrict__ w, int lx, int ly, int lz, int pitch,
                 unsigned long long* e_out) {
  const uint32_t rows = (uint32_t)ly * (uint32_t)lz;
  const int bonds = lz > 1 ? 192 : 128;
  long long e = 0;
  for (uint32_t row = blockIdx.x; row < rows; row += gridDim.x) {
    const uint32_t y = row % (uint32_t)ly, z = row / (uint32_t)ly;
    const uint32_t yp = y + 1 < (uint32_t)ly ? y + 1 : 0, zp = z + 1 < (uint32_t)lz ? z + 1 : 0;
    const unsigned long long* r0 = w + (size_t)row * pitch;
    const unsigned long long* ry = w + ((size_t)z * ly + yp) * pitch;
    const unsigned long long* rz = w + ((size_t)zp * ly + y) * pitch;
    for (int x = threadIdx.x; x < lx; x += blockDim.x) {
      const unsigned long long a = r0[x];
      int anti = __popcll(a ^ r0[x + 1 < lx ? x + 1 : 0]) + __popcll(a ^ ry[x]);
      if (lz > 1) anti += __popcll(a ^ rz[x]);
      e -= (long long)(bonds - 2 * anti);
    }
  }
  for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xFFFFFFFFu, e, o);
  if ((threadIdx.x & 31) == 0 && e) atomicAdd(e_out, (unsigned long long)e);
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

GPUMC_BOUNDS_MODULE(lattice_ops)

}  // namespace gpumc
