// Allocation-free exact energy of caller-provided int8 lattices.
//
// gpumc_recompute_energy reduces into a device accumulator it allocates with
// cudaMalloc on every call (and frees with cudaFree, which synchronizes the
// device).  Some callers cannot allow that: a host application whose device
// memory is owned by another allocator (a framework's caching allocator or a
// fixed memory pool under a hard budget), where a stray cudaMalloc either
// fails or fragments the pool, and latency-sensitive loops that cannot absorb
// the device-wide synchronization of cudaFree.  For them this file provides
// gpumc_energy_int8_noalloc: the same exact bond-sum reduction, with its
// scratch (per-block partial sums) in a file-scope __device__ array instead
// of allocated memory.  The caller passes the spins and the output.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/gpumc.h"
#include "engine.h"
#include "host_internal.h"

namespace gpumc {

constexpr int kNoAllocBlocksPerLattice = 256;
constexpr int kNoAllocMaxLattices = 64;
constexpr int kNoAllocMaxDevices = 64;

// Scratch for the first reduction stage: one int64 partial sum per
// (lattice, block), 64 x 256 x 8 B = 128 KiB.  Every GPU that loads the
// library holds it until the process exits.
static __device__ __align__(256) long long g_noalloc_partials[kNoAllocMaxLattices * kNoAllocBlocksPerLattice];

// Stage 1: block (b, l) sums -J-free bond terms over a grid-stride slice of
// lattice l and writes its partial into partials[l * 256 + b].  Every slot a
// call reads is written by the same call, so nothing needs clearing.
__global__ void __launch_bounds__(256)
    k_noalloc_energy_partials(int model, int dims, int lx, int ly, int lz, const int8_t* spins,
                              long long* partials) {
  const int l = blockIdx.y;
  const long long n = (long long)lx * ly * lz;
  const int8_t* s = spins + (size_t)l * (size_t)n;
  long long e = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int x = (int)(i % lx);
    const long long rho = i / lx;
    const int y = (int)(rho % ly);
    const int z = (int)(rho / ly);
    const int8_t a = s[i];
    // one +1 bond per axis, wrapping at the far face; an axis of extent 1 has
    // no bond at all (a site is not its own neighbour)
    if (lx > 1) {
      const int xp = x + 1 < lx ? x + 1 : 0;
      const int8_t b = s[rho * lx + xp];
      e -= model == ISING ? (long long)a * b : (long long)(a == b);
    }
    if (ly > 1) {
      const int yp = y + 1 < ly ? y + 1 : 0;
      const int8_t b = s[((long long)z * ly + yp) * lx + x];
      e -= model == ISING ? (long long)a * b : (long long)(a == b);
    }
    if (dims == 3 && lz > 1) {
      const int zp = z + 1 < lz ? z + 1 : 0;
      const int8_t b = s[((long long)zp * ly + y) * lx + x];
      e -= model == ISING ? (long long)a * b : (long long)(a == b);
    }
  }
  __shared__ long long red[256 / 32];
  for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xFFFFFFFFu, e, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    partials[(size_t)l * kNoAllocBlocksPerLattice + blockIdx.x] = t;
  }
}

// Stage 2: one block per lattice adds its 256 partials in a fixed order.
__global__ void __launch_bounds__(256)
    k_noalloc_energy_finish(const long long* partials, long long* energy_out) {
  const int l = blockIdx.x;
  long long v = partials[(size_t)l * kNoAllocBlocksPerLattice + threadIdx.x];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
  __shared__ long long red[8];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long t = 0;
    for (int w = 0; w < 8; ++w) t += red[w];
    energy_out[l] = t;
  }
}

// Device address of the scratch array, looked up with the device current
// (the array's host-side name is not a device address).  The address belongs
// to the device's current context: it is cached together with that context's
// unique id and looked up again when the id changes (after cudaDeviceReset the
// runtime creates a new primary context and reloads the module).
struct ScratchSlot {
  long long* ptr = nullptr;
  unsigned long long ctx_id = 0;
};
static ScratchSlot g_scratch[kNoAllocMaxDevices];
static std::mutex g_scratch_mu;

// Unique id of the calling thread's current context (cuCtxGetId through the
// runtime's driver entry point, so the library needs no link to libcuda).
static bool current_context_id(unsigned long long* id) {
  typedef CUresult (*CtxGetId)(CUcontext, unsigned long long*);
  static CtxGetId fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return (CtxGetId)p;
  }();
  return fn && fn(nullptr, id) == CUDA_SUCCESS;
}

static int scratch_for_current_device(long long** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(GPUMC_ENODEV, std::string("no usable CUDA device: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(GPUMC_ENODEV, "device index beyond 64");
  unsigned long long ctx = 0;
  const bool have_ctx = current_context_id(&ctx);
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  ScratchSlot& slot = g_scratch[dev];
  if (!have_ctx || !slot.ptr || slot.ctx_id != ctx) {
    long long* p = nullptr;
    e = cudaGetSymbolAddress((void**)&p, g_noalloc_partials);  // creates the context if needed
    if (e != cudaSuccess)
      return fail(GPUMC_ECUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    if (!current_context_id(&ctx))
      return fail(GPUMC_ECUDA, "no current CUDA context after looking up the scratch array");
    slot.ptr = p;
    slot.ctx_id = ctx;
  }
  *out = slot.ptr;
  return GPUMC_OK;
}

}  // namespace gpumc

using namespace gpumc;

int gpumc_energy_int8_noalloc(int32_t model, int32_t dims, int64_t lx, int64_t ly, int64_t lz,
                              const int8_t* spins, int32_t n_lattices, long long* energy_out,
                              void* stream) {
  if (model != GPUMC_ISING && model != GPUMC_POTTS)
    return fail(GPUMC_EINVAL, "model: the allocation-free energy handles int8 Ising and Potts lattices");
  if (dims != 2 && dims != 3) return fail(GPUMC_EINVAL, "dims: expected 2 or 3");
  const int64_t lzz = dims == 3 ? lz : 1;
  if (lx < 1 || ly < 1 || lzz < 1 || lx > (1 << 20) || ly > (1 << 20) || lzz > (1 << 20))
    return fail(GPUMC_EINVAL, "Lx/Ly/Lz: extents must be in 1..2^20");
  if ((double)lx * (double)ly * (double)lzz > 4.0e9)
    return fail(GPUMC_EINVAL, "lattice: more than 4e9 sites");
  if (n_lattices < 1 || n_lattices > kNoAllocMaxLattices)
    return fail(GPUMC_EINVAL,
                "n_lattices: the allocation-free energy handles 1..64 lattices per call "
                "(its fixed scratch holds 64 x 256 partial sums)");
  if (!spins || !energy_out) return fail(GPUMC_EINVAL, "spins/energy_out: null device pointer");
  long long* scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc) return rc;
  // An error left pending by the caller's earlier work is reported as such
  // (and left pending), so the check after the launches sees only their own.
  cudaError_t pending = cudaPeekAtLastError();
  if (pending != cudaSuccess)
    return fail(GPUMC_ECUDA, std::string("CUDA error pending before the call: ") + cudaGetErrorString(pending));
  cudaStream_t st = (cudaStream_t)stream;
  const dim3 grid(kNoAllocBlocksPerLattice, (unsigned)n_lattices);
  k_noalloc_energy_partials<<<grid, 256, 0, st>>>(model, dims, (int)lx, (int)ly, (int)lzz, spins, scratch);
  k_noalloc_energy_finish<<<n_lattices, kNoAllocBlocksPerLattice, 0, st>>>(scratch, energy_out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(GPUMC_ECUDA, std::string("noalloc energy launch: ") + cudaGetErrorString(e));
  return GPUMC_OK;
}
