// Host side of the engine and the C ABI declared in include/gpumc.h.
//
// A gpumc_engine owns a CUDA stream and two device-resident descriptor pools
// (lattices and groups).  A gpumc_sim takes one lattice slot per replica and
// one group slot; its sweep kernels read the descriptors directly, and the
// last CTA of every launch updates them (energy cache, records, sweep count,
// PT labels), so a launch sequence can be captured once in a CUDA graph and
// replayed without host involvement.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <string>
#include <vector>

#include "../../include/gpumc.h"
#include "engine.h"
#include "host_internal.h"

namespace gpumc {

template <int DIM, int ALG>
__global__ void k_sweep_ising_bits(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template <int MODEL, int ALG>
__global__ void k_sweep_discrete_2d(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template <int MODEL, int ALG>
__global__ void k_sweep_discrete_3d(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template <int DIM, int COLOUR, int ALG>
__global__ void k_sweep_o3(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template <int DIM>
__global__ void k_sweep_msc(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template <int DIM>
__global__ void k_sweep_potts_bits(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template <int COLOUR, int ALG, int CLS>
__global__ void k_sweep_o3_march(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template <int DIM, int MODEL, int WOLFF>
__global__ void k_cluster_local(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template <int DIM, int MODEL, int WOLFF>
__global__ void k_cluster_global(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template <int DIM, int MODEL, int WOLFF>
__global__ void k_cluster_flip(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template <int DIM, int MODEL, int WOLFF>
__global__ void k_cluster_account(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template <int DIM, int WOLFF>
__global__ void k_cluster_o3_local(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template <int DIM, int WOLFF>
__global__ void k_cluster_o3_global(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template <int DIM, int WOLFF>
__global__ void k_cluster_o3_flip(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template <int DIM, int WOLFF>
__global__ void k_cluster_o3_account(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
template <int ALG>
__global__ void k_sweep_ising_resident(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*, const int2*,
                                       uint2*, int, int, long long);
template <int ALG>
__global__ void k_sweep_ising_resident3(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*, const int2*,
                                        uint2*, int, int, long long);
template <int DIM>
__global__ void k_msc_measure(const LatDesc*, int, unsigned long long*);
__global__ void k_msc_record(LatDesc*, GroupDesc*, int, unsigned long long*);
__global__ void k_init_discrete(int8_t*, int, int, int, int, int, int, uint64_t, int);
__global__ void k_init_o3(float*, int, int, int, int, uint64_t, int);
__global__ void k_init_msc(unsigned long long*, int, int, int, int, const uint64_t*, int);
__global__ void k_energy_o3(const float*, int, int, int, int, double, double*);
__global__ void k_philox_probe(const uint4*, const uint2*, uint4*, int);

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}
const std::string& last_error_ref() { return g_last_error; }
size_t g_last_error_size() { return g_last_error.size(); }

#define CUDA_TRY(expr)                                                            \
  do {                                                                            \
    cudaError_t e_ = (expr);                                                      \
    if (e_ != cudaSuccess)                                                        \
      return fail(e_ == cudaErrorMemoryAllocation ? GPUMC_ENOMEM : GPUMC_ECUDA,   \
                  std::string(#expr) + ": " + cudaGetErrorString(e_));            \
  } while (0)

// ---------------------------------------------------------------------------
// stream keys: restatement of RngStreamKey::seed (Carlo.rs/src/rng_stream.rs:
// 126-154): domain-separated SplitMix64 folding of the stream coordinates.
// ---------------------------------------------------------------------------
static uint64_t mix64(uint64_t v) {
  v += 0x9E3779B97F4A7C15ull;
  v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ull;
  v = (v ^ (v >> 27)) * 0x94D049BB133111EBull;
  return v ^ (v >> 31);
}
static uint64_t fold(uint64_t state, uint64_t domain, uint64_t value) {
  const uint64_t rot = (domain << 17) | (domain >> 47);
  return mix64(state ^ domain ^ mix64(value + rot));
}
uint64_t stream_key(uint64_t base, uint64_t replica, uint64_t phase, uint64_t substream) {
  uint64_t s = mix64(base ^ 0x53435554544C4552ull);  // "SCUTTLER"
  s = fold(s, 0x5441534Bull, 0);                     // task
  s = fold(s, 0x52554E00ull, 0);                     // run
  s = fold(s, 0x434841494E00ull, 0);                 // chain
  s = fold(s, 0x5245504C49434100ull, replica);       // replica
  s = fold(s, 0x544852454144ull, 0);                 // thread
  s = fold(s, 0x504841534500ull, phase);             // phase
  return fold(s, 0x535542535452ull, substream);      // substream
}

// 80-bit acceptance threshold of probability p: head = floor(p 2^16) (65536
// = always), tail = next 64 bits of p's binary expansion.
void threshold80(double p, uint32_t& head, unsigned long long& tail) {
  if (!(p > 0.0)) {
    head = 0;
    tail = 0;
    return;
  }
  if (p >= 1.0) {
    head = 65536u;
    tail = 0;
    return;
  }
  const double s = std::ldexp(p, 16);
  const double h = std::floor(s);
  head = (uint32_t)h;
  tail = (unsigned long long)std::ldexp(s - h, 64);
}

// Class tables.  Ising / multi-spin: class k = anti-aligned neighbours,
// dE = 2J(z - 2k) (multi_spin.rs:84-91 indexes by aligned count z - k).
// Potts: class d + z with d = n(new) - n(old), dE = -J d.
//
// Heat bath.  Ising: class k = down neighbours, T[k] = p(|x|) with
// x = 2 beta J (z - 2k) and p(x) = 1 / (1 + exp(-x)) (IsingModel::
// heat_bath_sample_site, CMC.rs/src/lattice/models.rs:158-186), clamped below
// 1 so that every class stays a comparison.  Potts: the weight exp(beta J n)
// of a state held by n neighbours (PottsModel::heat_bath_sample_site,
// models.rs:340-380) relative to the site's largest one, as a 64-bit integer:
// tail[d] = W[d] = floor(2^60 exp(-beta |J| d)), d = 0..z the distance of
// the state's count from the site's most favoured count (n_max - n for
// J >= 0, n - n_min for J < 0).  The favoured state weighs exactly 2^60, so
// a site's total weight is in [2^60, 2^63) for q <= 8.
int n_classes(int model, int dims) {
  const int z = 2 * dims;
  return (model == POTTS) ? 2 * z + 1 : z + 1;
}
void build_table(int model, int dims, double J, double beta, uint32_t* head,
                 unsigned long long* tail, int alg) {
  const int z = 2 * dims;
  const int n = n_classes(model, dims);
  if (alg == SWENDSEN_WANG || alg == WOLFF) {
    // cluster bond activation (ClusterModel::cluster_bond_probability,
    // models.rs:130-147, :312-329): tail[0] = floor(p 2^64), active iff a
    // 64-bit uniform is below it (p >= 1: all ones)
    for (int c = 0; c < n; ++c) {
      head[c] = 0;
      tail[c] = 0;
    }
    double p = model == POTTS ? 1.0 - std::exp(-beta * J) : 1.0 - std::exp(-2.0 * beta * J);
    p = p < 0.0 ? 0.0 : p;
    tail[0] = p >= 1.0 ? ~0ull : (unsigned long long)std::ldexp(p, 64);
    return;
  }
  if (alg == HEAT_BATH) {
    for (int c = 0; c < n; ++c) {
      head[c] = 0;
      tail[c] = 0;
    }
    if (model == POTTS) {
      for (int d = 0; d <= z; ++d)
        tail[d] = (unsigned long long)std::ldexp(std::exp(-(beta * std::fabs(J)) * (double)d), 60);
    } else {
      for (int k = 0; k <= z; ++k) {
        const double ax = std::fabs(2.0 * beta * J * (double)(z - 2 * k));
        double p = 1.0 / (1.0 + std::exp(-ax));
        if (p >= 1.0) p = 1.0 - 0x1p-53;
        threshold80(p, head[k], tail[k]);
      }
    }
    return;
  }
  for (int c = 0; c < n; ++c) {
    const double dE = (model == POTTS) ? -J * (double)(c - z) : 2.0 * J * (double)(z - 2 * c);
    const double logA = -beta * dE;
    threshold80(logA >= 0.0 ? 1.0 : std::exp(logA), head[c], tail[c]);
  }
}

// ---------------------------------------------------------------------------
// spec validation and layout planning
// ---------------------------------------------------------------------------
int validate_spec(const gpumc_spec* s) {
  if (!s) return fail(GPUMC_EINVAL, "spec: null pointer");
  if (s->model < GPUMC_ISING || s->model > GPUMC_ISING_MSC64)
    return fail(GPUMC_EINVAL, "model: unknown model id");
  if (s->dims != 2 && s->dims != 3)
    return fail(GPUMC_EINVAL, "lattice_type: expected square (dims=2) or cubic (dims=3)");
  if (!s->pbc) return fail(GPUMC_EINVAL, "pbc: the checkerboard engine requires periodic boundaries");
  const int64_t lz = s->dims == 3 ? s->lz : 1;
  const int64_t ext[3] = {s->lx, s->ly, lz};
  for (int a = 0; a < s->dims; ++a) {
    if (ext[a] < 4 || (ext[a] & 1))
      return fail(GPUMC_EINVAL,
                  "Lx/Ly/Lz: extents must be even and >= 4 (a periodic checkerboard needs a "
                  "bipartite lattice)");
    if (ext[a] > (1 << 20)) return fail(GPUMC_EINVAL, "Lx/Ly/Lz: extent too large");
  }
  if ((double)s->lx * (double)s->ly * (double)lz > 4.0e9)
    return fail(GPUMC_EINVAL, "lattice: more than 4e9 sites");
  if (s->model == GPUMC_ISING && s->lx > 16384 && s->lx % 64 != 0)
    return fail(GPUMC_EINVAL, "Lx: Ising rows longer than 16384 sites must be a multiple of 64");
  if (s->model == GPUMC_ISING && s->dims == 3 && s->lx > 16384)
    return fail(GPUMC_EINVAL, "Lx: cubic Ising rows are limited to 16384 sites");
  if (!std::isfinite(s->J)) return fail(GPUMC_EINVAL, "J: must be finite");
  if (s->model == GPUMC_POTTS && (s->q < 2 || s->q > kMaxPottsCounts))
    return fail(GPUMC_EINVAL, "q: Potts q must be in 2..8");
  if (s->n_replicas < 1 || s->n_replicas > 4096) return fail(GPUMC_EINVAL, "n_replicas: 1..4096");
  if (s->n_temps != 1 && s->n_temps != s->n_replicas)
    return fail(GPUMC_EINVAL, "n_temps: must be 1 or n_replicas");
  if (!s->betas) return fail(GPUMC_EINVAL, "beta: missing");
  for (int i = 0; i < s->n_temps; ++i)
    if (!std::isfinite(s->betas[i]) || s->betas[i] < 0.0)
      return fail(GPUMC_EINVAL, "beta: must be finite and non-negative");
  if (s->init != GPUMC_INIT_HOT && s->init != GPUMC_INIT_COLD)
    return fail(GPUMC_EINVAL, "initial_state: expected hot/random or cold/ordered");
  if (s->model == GPUMC_O3 && !(s->cone_half_angle > 0.0 && s->cone_half_angle <= M_PI))
    return fail(GPUMC_EINVAL, "cone_half_angle: must be in (0, pi]");
  if (s->o3_proposal < GPUMC_O3_CAP || s->o3_proposal > GPUMC_O3_CAP_FAST)
    return fail(GPUMC_EINVAL, "o3_proposal: expected cap, uniform (standard), opss or cap_fast");
  if (s->record_capacity < 1) return fail(GPUMC_EINVAL, "record_capacity: must be >= 1");
  if (s->algorithm < GPUMC_METROPOLIS || s->algorithm > GPUMC_WOLFF)
    return fail(GPUMC_EINVAL, "algorithm: expected metropolis, heat_bath, swendsen_wang or wolff");
  if (s->algorithm != GPUMC_METROPOLIS && s->model == GPUMC_ISING_MSC64)
    return fail(GPUMC_EINVAL, "algorithm: the multi-spin model has Metropolis sweeps only");
  if (s->algorithm >= GPUMC_SWENDSEN_WANG) {
    if (s->model != GPUMC_ISING && s->model != GPUMC_POTTS && s->model != GPUMC_O3)
      return fail(GPUMC_EINVAL, "algorithm: cluster updates are for Ising, Potts and O(3)");
    if (s->J < 0.0)
      return fail(GPUMC_EINVAL, "J: ferromagnetic cluster updates require J >= 0");
  }
  if (!layout_ok(plan_layout(s)))
    return fail(GPUMC_EINVAL, "lattice: no tile plan fits this geometry (row too long for shared memory)");
  return GPUMC_OK;
}

// Shared memory a bit-sliced tile needs, with the geometry the kernels derive
// from it (make_bits_geom): packed segments of 8 B (Ising) or 16 B (Potts
// q <= 4), NC columns (owned + halo), R rows (two halo rows each side unless
// a 3D tile spans whole planes), four planes in 3D.
static size_t bits_tile_smem(const Layout& L, const TileItem& t) {
  const int nseg = L.pitch / 64;
  const int s0 = t.x0 >> 6;
  const int ns = std::min(L.tile_cx, nseg - s0);
  const int xh = ns < nseg ? 1 : 0;
  const int nc = ns + 2 * xh;
  const int hv = std::min(L.tile_y, L.ly - t.y0);
  const bool yw = L.dims == 3 && t.y0 == 0 && L.tile_y >= L.ly && xh == 0;
  const int r = yw ? hv : hv + 4;
  if (nc > kThreads) return ~(size_t)0;  // a CTA covers at least one whole tile row
  const size_t elem = L.model == ISING ? 8 : 16;
  return elem * (size_t)r * nc * (L.dims == 3 ? 4 : 1);
}

// Every tile step must be positive and the shared-memory plan must fit, for
// every tile the plan enumerates.
bool layout_ok(const Layout& L) {
  if (!(L.buf_bytes > 0 && L.tile_cx > 0 && L.tile_y > 0 && L.tile_z > 0 &&
        (L.smem > 0 || L.model == O3 || L.cluster) && L.smem <= 200 * 1024))
    return false;
  if (!L.cluster && (L.model == ISING || (L.model == POTTS && L.bits))) {
    std::vector<TileItem> tiles;
    enumerate_tiles(L, 0, tiles);
    for (const TileItem& t : tiles)
      if (t.x0 % 64 != 0 || bits_tile_smem(L, t) > L.smem) return false;
  }
  return true;
}

// Rows per whole-row Ising tile.  A tile of hv rows costs its CTA
// ceil((hv+4)/r) + ceil((hv+2)/r) + ceil(hv/r) row steps (load, black pass
// with its halo rows, white pass; r = rows the CTA covers per step), and the
// n_rep lattices of ly rows run in ceil(tiles / slots) waves of the device's
// resident CTA slots.  The height minimising waves x steps is chosen (the
// taller one on a tie, which does less halo work), among heights that fit
// the shared-memory budget and are at least 8 rows unless the lattice is
// smaller.
int ising_tile_rows(int ly, int n_rep, int nseg, int hv_max, int slots) {
  const int r = std::max(1, kThreads / nseg);
  int best = std::min(ly, hv_max);
  double best_t = 1e300;
  int last_hv = -1;
  for (int nty = 1; nty <= ly; ++nty) {
    const int hv = (ly + nty - 1) / nty;
    if (hv == last_hv) continue;
    last_hv = hv;
    if (hv > hv_max) continue;
    if (hv < 8 && hv < ly) break;
    const int tiles = ((ly + hv - 1) / hv) * n_rep;
    const double waves = std::max(1.0, std::ceil((double)tiles / slots));
    const double steps = std::ceil((hv + 4.0) / r) + std::ceil((hv + 2.0) / r) + std::ceil((double)hv / r);
    const double t = waves * steps;
    if (t < best_t - 1e-9) {
      best_t = t;
      best = hv;
    }
  }
  return best;
}

// Tile knobs of the planner (gpumc_set_tile_knobs): 0 = the analytic
// choice; a positive value replaces it for layouts planned afterwards.
static gpumc_tile_knobs g_knobs = {0, 0, 0, 0, 0, 0};
static std::mutex g_knobs_mu;

static gpumc_tile_knobs current_knobs() {
  std::lock_guard<std::mutex> lock(g_knobs_mu);
  return g_knobs;
}

Layout plan_layout(const gpumc_spec* s, int slots, int slots3) {
  const gpumc_tile_knobs kn = current_knobs();
  Layout L;
  L.model = s->model;
  L.alg = s->algorithm == GPUMC_HEAT_BATH ? HEAT_BATH
          : s->algorithm == GPUMC_SWENDSEN_WANG ? SWENDSEN_WANG
          : s->algorithm == GPUMC_WOLFF ? WOLFF : METROPOLIS;
  L.cluster = L.alg == SWENDSEN_WANG || L.alg == WOLFF;
  L.prop = (L.model == O3 && L.alg == METROPOLIS) ? s->o3_proposal : 0;
  L.q = (int)s->q;
  L.dims = s->dims;
  L.lx = (int)s->lx;
  L.ly = (int)s->ly;
  L.lz = s->dims == 3 ? (int)s->lz : 1;
  const int lx = L.lx, ly = L.ly, lz = L.lz;
  L.n_sites = (int64_t)lx * ly * lz;
  const size_t rows = (size_t)ly * lz;
  if (L.model == ISING) {
    // bit-sliced kernel: 64-site row segments.  2D lattices whose rows are at
    // most 256 segments use whole-row tiles (no column halo, the threads of a
    // CTA cover whole rows); the tile height trades the two halo rows of the
    // black pass against filling the GPU's CTA slots in whole waves.  Longer
    // rows (and 3D) use x-split tiles of 32 segments plus one halo segment
    // per side when the row is a whole number of segments.
    L.pitch = (lx + 63) / 64 * 64;
    L.buf_bytes = (size_t)L.pitch * rows;
    const int nseg = L.pitch / 64;
    if (L.dims == 2 && nseg <= 256) {
      L.tile_cx = nseg;
      const int hv_max = std::max(1, (int)(kIsingTileSmem / (8 * (size_t)nseg)) - 4);
      L.tile_y = kn.ising2d_rows > 0 ? std::min({kn.ising2d_rows, hv_max, ly})
                                     : ising_tile_rows(ly, std::max<int>(1, (int)s->n_replicas), nseg, hv_max, slots);
      L.tile_z = 1;
      L.smem = 8 * (size_t)(L.tile_y + 4) * nseg;
    } else if (L.dims == 3 && nseg <= 256 && (size_t)ly * nseg * 8 * 4 <= kIsingTileSmem) {
      // whole-plane 3D tiles: four packed planes in the ring, rows wrap
      // inside the tile (no y halo); the z extent per tile minimises
      // (CTA waves) x (planes loaded + black-updated + white-updated)
      L.tile_cx = nseg;
      L.tile_y = ly;
      const int n_rep = std::max<int>(1, (int)s->n_replicas);
      int best = std::min(lz, 16);
      double best_t = 1e300;
      for (int ntz = 1; ntz <= lz; ++ntz) {
        const int dv = (lz + ntz - 1) / ntz;
        if (dv < 4 && dv < lz) break;
        const int tiles = ((lz + dv - 1) / dv) * n_rep;
        const double waves = std::max(1.0, std::ceil((double)tiles / slots3));
        const double t = waves * (3.0 * dv + 6.0);
        if (t < best_t - 1e-9) {
          best_t = t;
          best = dv;
        }
      }
      L.tile_z = kn.ising3d_planes > 0 ? std::min(kn.ising3d_planes, lz) : best;
      L.smem = 4 * 8 * (size_t)ly * nseg;
    } else {
      const bool xsplit = (lx % 64 == 0) && nseg > 32;
      L.tile_cx = xsplit ? 32 : nseg;
      const int nc = L.tile_cx + (xsplit ? 2 : 0);
      const int items = L.dims == 2 ? 2048 : 1024;
      const int hv_max = std::max(1, items / nc - 2);
      const int nty = (ly + hv_max - 1) / hv_max;
      L.tile_y = (ly + nty - 1) / nty;
      if (L.dims == 2) {
        L.tile_z = 1;
        L.smem = 8 * (size_t)(L.tile_y + 4) * nc;
      } else {
        const int ntz = (lz + 15) / 16;
        L.tile_z = (lz + ntz - 1) / ntz;
        L.smem = 4 * 8 * (size_t)(L.tile_y + 4) * nc;
      }
    }
  } else if (L.model == POTTS && L.alg == METROPOLIS && s->q <= 4 && ((lx + 63) / 64 <= 128 || lx % 64 == 0)) {
    // bit-sliced kernel (two bit planes per parity, 16 B per packed 64-site
    // segment): whole-row tiles up to 128 segments per row, else x-split
    // tiles of 32 segments plus one halo segment per side; about 1536
    // packed segments per tile (2D) or per plane (3D), y halo of two rows
    // unless a 3D tile spans whole planes
    L.bits = true;
    L.pitch = (lx + 63) / 64 * 64;
    L.buf_bytes = (size_t)L.pitch * rows;
    const int nseg = L.pitch / 64;
    if (L.dims == 3 && nseg <= 128 && (size_t)ly * nseg * 16 * 4 <= kIsingTileSmem) {
      L.tile_cx = nseg;
      L.tile_y = ly;
      const int zmax = kn.potts3d_planes > 0 ? kn.potts3d_planes : 16;
      const int ntz = (lz + zmax - 1) / zmax;
      L.tile_z = (lz + ntz - 1) / ntz;
      L.smem = 4 * 16 * (size_t)ly * nseg;
    } else {
      const bool xsplit = (lx % 64 == 0) && nseg > 128;
      L.tile_cx = xsplit ? 32 : nseg;
      const int nc = L.tile_cx + (xsplit ? 2 : 0);
      const int items = L.dims == 2 ? (kn.potts_segments > 0 ? std::min(kn.potts_segments, 3072) : 1536) : 768;
      const int hv_max = std::max(1, items / nc - 4);
      const int nty = (ly + hv_max - 1) / hv_max;
      L.tile_y = (ly + nty - 1) / nty;
      if (L.dims == 2) {
        L.tile_z = 1;
        L.smem = 16 * (size_t)(L.tile_y + 4) * nc;
      } else {
        const int ntz = (lz + 15) / 16;
        L.tile_z = (lz + ntz - 1) / ntz;
        L.smem = 4 * 16 * (size_t)(L.tile_y + 4) * nc;
      }
    }
  } else if (L.model == POTTS) {
    L.pitch = (lx + 15) / 16 * 16;
    L.buf_bytes = (size_t)L.pitch * rows;
    const int ncol = L.pitch / 16;
    // a pass maps threads to (row, chunk column) with rstep rows per sweep of
    // the CTA; tile heights are multiples of rstep minus the 2 halo rows
    if (L.dims == 2) {
      L.tile_cx = ncol <= 64 ? ncol : 32;
      const int rstep = kThreads / L.tile_cx;
      const int m = std::max(1, (16384 + 16 * L.tile_cx * rstep - 1) / (16 * L.tile_cx * rstep));
      L.tile_y = std::max(1, std::min(std::min(m * rstep - 2, 124), ly));
      L.tile_z = 1;
      L.smem = 2 * (size_t)(L.tile_y + 4) * (16 * L.tile_cx + 32);
    } else {
      L.tile_cx = ncol <= 16 ? ncol : 16;
      const int rstep = kThreads / L.tile_cx;
      L.tile_y = std::max(1, std::min(std::min(2 * rstep - 2, 124), ly));
      L.tile_z = std::min(lz, 32);
      L.smem = 6 * (size_t)(L.tile_y + 4) * (16 * L.tile_cx + 32);
    }
  } else if (L.model == O3) {
    // in place, one thread per site of the colour, tiles of whole rows with
    // about 2048 sites of each colour
    L.pitch = (lx + 3) / 4 * 4;
    // 3D rows within 15 % of a compiled z-march row class (32, 64, 128
    // floats) are padded to it, for its compile-time neighbour offsets
    // (measured on 12.6 M sites: L = 64 at 67.7 attempts/ns, L = 56 / 60 / 72
    // at 53.9 / 54.5 / 57.5 with the offsets at run time)
    if (L.dims == 3)
      for (int c : {32, 64, 128})
        if (L.pitch <= c && 100 * c <= 115 * L.pitch) {
          L.pitch = c;
          break;
        }
    L.buf_bytes = 3 * sizeof(float) * (size_t)L.pitch * rows;
    L.inplace = true;
    L.tile_cx = (lx + 3) / 4;
    // 3D: tiles of whole rows marched along z through a ring of four shared
    // planes (3 components x (rows + 2 halo rows) x pitch floats) of at
    // most 56 KB (four CTAs per SM), rows x 8 planes per tile (for 32
    // lattices of 64^3: 16 rows, 1024 tiles, 1.7 waves of 148 x 4 CTAs).  Deeper
    // tiles re-read fewer halo planes but leave the last wave ragged: on
    // that mix 22 planes ran at 41.2 attempts/ns, 11 at 42.7, 8 at 47.5,
    // 6 at 44.1 and 4 at 45.2.
    const int ty_max = (int)(kO3MarchSmem / (12 * (size_t)kO3RingSlots * L.pitch)) - 2;
    if (L.dims == 3 && ty_max >= 1) {
      L.march = true;
      // rows per tile: about one site pair per thread per plane (16 rows
      // at L = 64; fewer pairs per row, more rows)
      const int np = std::max(1, ((lx >> 1) + 1) >> 1);
      const int rows = std::min(kn.o3_rows > 0 ? kn.o3_rows : std::max(1, kThreads / np), ty_max);
      const int nty = (ly + rows - 1) / rows;
      L.tile_y = (ly + nty - 1) / nty;
      const int planes = kn.o3_planes > 0 ? kn.o3_planes : 8;
      const int ntz = (lz + planes - 1) / planes;
      L.tile_z = (lz + ntz - 1) / ntz;
      const int cls = o3_row_class(L.pitch);
      L.smem = 12 * (size_t)kO3RingSlots * L.pitch * (cls ? o3_class_rows(cls) : L.tile_y + 2);
      L.smem = std::max(L.smem, sizeof(int) * (size_t)kEpiScratchInts);  // colour 1's epilogue scratch
    } else {
      L.tile_y = std::max(1, std::min(ly, 4096 / lx));
      L.tile_z = L.dims == 3 ? std::max(1, std::min(lz, 4096 / (lx * L.tile_y))) : 1;
      L.smem = 0;
    }
  } else {  // MSC
    L.pitch = (lx + 1) / 2 * 2;
    L.buf_bytes = sizeof(unsigned long long) * (size_t)L.pitch * rows;
    const int w = std::min(lx, L.dims == 2 ? 64 : 32);
    L.tile_cx = (w + 1) / 2;
    const int W = std::min(lx, L.tile_cx * 2);
    const int ty_max = 2 * 4 * 256 / (W + 2) - 2;
    if (L.dims == 2) {
      L.tile_y = std::max(1, std::min(ty_max, ly));
      L.tile_z = 1;
      L.smem = 8 * (size_t)(L.tile_y + 4) * (W + 4);
    } else {
      L.tile_y = std::max(1, std::min(std::min(ty_max, 16), ly));
      L.tile_z = std::min(lz, 16);
      L.smem = 4 * 8 * (size_t)(L.tile_y + 4) * (W + 4);
    }
  }
  if (L.cluster) {
    // cluster updates keep the model's buffer layout; their kernels take
    // tiles of 16 x 16 (2D) or 8 x 8 x 4 (3D) sites, one thread per site
    L.tile_cx = L.dims == 2 ? 16 : 8;  // sites
    L.tile_y = L.dims == 2 ? 16 : 8;
    L.tile_z = L.dims == 2 ? 1 : 4;
    L.smem = 0;
    L.inplace = false;  // O(3) too: the flip writes the other buffer
  }
  return L;
}

int tile_width_sites(const Layout& L) {
  if (L.cluster) return L.tile_cx;
  if (L.model == ISING) return 64 * L.tile_cx;
  if (L.model == POTTS) return (L.bits ? 64 : 16) * L.tile_cx;
  if (L.model == O3) return 4 * L.tile_cx;
  return 2 * L.tile_cx;
}

void enumerate_tiles(const Layout& L, int lat, std::vector<TileItem>& out) {
  const int tw = tile_width_sites(L);
  if (tw <= 0 || L.tile_y <= 0 || L.tile_z <= 0) return;  // rejected by layout_ok()
  for (int z0 = 0; z0 < L.lz; z0 += L.tile_z)
    for (int y0 = 0; y0 < L.ly; y0 += L.tile_y)
      for (int x0 = 0; x0 < L.lx; x0 += tw) out.push_back(TileItem{lat, x0, y0, z0, L.tile_cx, L.tile_y, L.tile_z, 0});
}

// Kernel of a layout: model x dims; Potts planned on bit planes (q <= 4)
// runs the bit-sliced kernel (kinds 8 / 9); heat-bath layouts add
// kKindHeatBath to the kind of the same model and geometry.
int kernel_kind(const Layout& L) {
  if (L.cluster && L.model == O3) return kKindCluster + 8 + (L.dims - 2) + (L.alg == WOLFF ? 2 : 0);
  if (L.cluster) return kKindCluster + (L.model == POTTS ? 2 : 0) + (L.dims - 2) + (L.alg == WOLFF ? 4 : 0);
  const int hb = L.alg == HEAT_BATH ? kKindHeatBath
                 : L.prop == GPUMC_O3_UNIFORM ? kKindO3Uniform
                 : L.prop == GPUMC_O3_OPSS ? kKindO3Opss
                 : L.prop == GPUMC_O3_CAP_FAST ? kKindO3Fast : 0;
  if (L.model == POTTS && L.bits) return 8 + (L.dims - 2);
  if (L.model == O3 && L.march) return 10 + o3_row_class(L.pitch) + hb;
  return L.model * 2 + (L.dims - 2) + hb;
}

// ---------------------------------------------------------------------------
// Launch-dependent tile shapes.  plan_layout sizes a lattice's tiles for a
// launch with plenty of tiles (halo and staging work amortised over large
// tiles).  A launch with far fewer tiles than the device has CTA slots (a
// lone lattice, a few serving jobs) would run on a fraction of the SMs with
// each CTA stepping through a large tile, so refine_layouts splits tiles,
// the simulation whose tiles hold the most sites first, until the launch has
// at least half a wave of CTAs or nothing can be split further.  Results do
// not depend on tile shapes: a colour pass reads only the other colour, and
// every draw is keyed by site or row segment, not by tile.
// ---------------------------------------------------------------------------
int64_t count_tiles(const Layout& L) {
  const int tw = tile_width_sites(L);
  if (tw <= 0 || L.tile_y <= 0 || L.tile_z <= 0) return 0;
  return (int64_t)((L.lx + tw - 1) / tw) * ((L.ly + L.tile_y - 1) / L.tile_y) *
         ((L.lz + L.tile_z - 1) / L.tile_z);
}

// One step of refinement (about halving the tile volume); false when the
// layout's tiles cannot be split further.  2D Ising tiles are already sized
// against the device's slots (ising_tile_rows) and feed the resident kernel;
// multi-spin and cluster layouts keep their shapes.
static bool split_tiles(Layout& L) {
  if (L.cluster || L.model == MSC || (L.model == ISING && L.dims == 2)) return false;
  if (L.model == O3) {
    if (L.march && L.tile_z >= 8) {
      L.tile_z = (L.tile_z + 1) / 2;
      return true;
    }
    if (L.march) {
      // the plain kernel with its own full-launch tiles (about 2048 sites of
      // each colour), split further by the steps below
      L.march = false;
      L.smem = 0;
      L.tile_y = std::max(1, std::min(L.ly, 4096 / L.lx));
      L.tile_z = L.tile_y < L.ly ? 1 : std::max(1, std::min(L.lz, 4096 / (L.lx * L.ly)));
      return true;
    }
    if (L.tile_z > 1) {
      L.tile_z = (L.tile_z + 1) / 2;
      return true;
    }
    if (L.tile_y > 1 && (int64_t)L.tile_y * L.lx > 256) {
      L.tile_y = (L.tile_y + 1) / 2;
      return true;
    }
    return false;
  }
  // bit-sliced Ising / Potts and int8 Potts: tiles with two-row y halos
  const bool bits = L.model == ISING || L.bits;
  if (bits && L.dims == 3 && L.tile_y >= L.ly) {
    if (L.ly < 8) return false;
    L.tile_y = (L.ly + 1) / 2;  // whole-plane tiles -> row bands with halos
  } else if (L.tile_y > 4) {
    L.tile_y = (L.tile_y + 1) / 2;
  } else if (L.dims == 3 && L.tile_z > 2) {
    L.tile_z = (L.tile_z + 1) / 2;
  } else {
    return false;
  }
  if (bits) {
    L.smem = bits_tile_smem(L, TileItem{0, 0, 0, 0, L.tile_cx, L.tile_y, L.tile_z, 0});
  } else {
    L.smem = (L.dims == 2 ? 2 : 6) * (size_t)(L.tile_y + 4) * (16 * L.tile_cx + 32);
  }
  return true;
}

void refine_layouts(std::vector<Layout>& lays, const std::vector<int>& reps, int slots) {
  const size_t n = lays.size();
  std::vector<bool> fixed(n, false);
  int64_t total = 0;
  for (size_t i = 0; i < n; ++i) total += count_tiles(lays[i]) * reps[i];
  const int64_t target = std::max(1, slots / 2);
  while (total < target) {
    size_t best = n;
    double most = 0.0;
    for (size_t i = 0; i < n; ++i) {
      if (fixed[i]) continue;
      const double per = (double)lays[i].n_sites / (double)std::max<int64_t>(1, count_tiles(lays[i]));
      if (per > most) {
        most = per;
        best = i;
      }
    }
    if (best == n) break;
    Layout t = lays[best];
    if (!split_tiles(t) || !layout_ok(t)) {
      fixed[best] = true;
      continue;
    }
    total += (count_tiles(t) - count_tiles(lays[best])) * reps[best];
    lays[best] = t;
  }
}

// CTA slots a launch of this layout's family fills: the 3D bit-sliced
// kernels run fewer CTAs per SM.
int family_slots(const Layout& L, int slots, int slots3) {
  return (L.dims == 3 && (L.model == ISING || L.bits)) ? slots3 : slots;
}

size_t footprint_bytes(const gpumc_spec* s) {
  const Layout L = plan_layout(s);
  const size_t per = (L.inplace ? 1 : 2) * L.buf_bytes;
  const size_t rec_entries = (size_t)s->record_capacity * s->n_replicas * (L.model == MSC ? 64 : 1);
  const size_t labels = L.cluster ? 4 * (size_t)L.n_sites : 0;
  return (per + labels) * s->n_replicas + rec_entries * sizeof(Record) +
         (size_t)s->n_temps * kMaxClasses * 12 + 4096;
}

// ---------------------------------------------------------------------------
// kernel launch table
// ---------------------------------------------------------------------------
typedef void (*SweepKernel)(const TileItem*, LatDesc*, GroupDesc*, LaunchCtl*);
// The O(3) z-march kernel of a colour for kind 10..13 (+ algorithm offset).
#define O3_MARCH_ROW(C, A) \
  {k_sweep_o3_march<C, A, 0>, k_sweep_o3_march<C, A, 1>, k_sweep_o3_march<C, A, 2>, k_sweep_o3_march<C, A, 3>}
static const SweepKernel kO3March[2][5][4] = {
    {O3_MARCH_ROW(0, 0), O3_MARCH_ROW(0, 1), O3_MARCH_ROW(0, 2), O3_MARCH_ROW(0, 3), O3_MARCH_ROW(0, 4)},
    {O3_MARCH_ROW(1, 0), O3_MARCH_ROW(1, 1), O3_MARCH_ROW(1, 2), O3_MARCH_ROW(1, 3), O3_MARCH_ROW(1, 4)}};
#undef O3_MARCH_ROW
static SweepKernel o3_march_kernel(int colour, int kind) {
  if (!is_o3_march_kind(kind)) return nullptr;
  const int off = kind - kind % 16;
  const int alg = off == kKindHeatBath ? 1 : off == kKindO3Uniform ? 2 : off == kKindO3Opss ? 3
                  : off == kKindO3Fast ? 4 : 0;
  return kO3March[colour][alg][kind % 16 - 10];
}
static SweepKernel kernel_for(int kind) {
  if (is_o3_march_kind(kind)) return o3_march_kernel(1, kind);
  switch (kind) {
    case 0: return k_sweep_ising_bits<2, 0>;
    case 1: return k_sweep_ising_bits<3, 0>;
    case 2: return k_sweep_discrete_2d<POTTS, 0>;
    case 3: return k_sweep_discrete_3d<POTTS, 0>;
    case 4: return k_sweep_o3<2, 1, 0>;
    case 5: return k_sweep_o3<3, 1, 0>;
    case 6: return k_sweep_msc<2>;
    case 7: return k_sweep_msc<3>;
    case 8: return k_sweep_potts_bits<2>;
    case 9: return k_sweep_potts_bits<3>;
    case kKindHeatBath + 0: return k_sweep_ising_bits<2, 1>;
    case kKindHeatBath + 1: return k_sweep_ising_bits<3, 1>;
    case kKindHeatBath + 2: return k_sweep_discrete_2d<POTTS, 1>;
    case kKindHeatBath + 3: return k_sweep_discrete_3d<POTTS, 1>;
    case kKindHeatBath + 4: return k_sweep_o3<2, 1, 1>;
    case kKindHeatBath + 5: return k_sweep_o3<3, 1, 1>;
    case kKindO3Uniform + 4: return k_sweep_o3<2, 1, 2>;
    case kKindO3Uniform + 5: return k_sweep_o3<3, 1, 2>;
    case kKindO3Opss + 4: return k_sweep_o3<2, 1, 3>;
    case kKindO3Opss + 5: return k_sweep_o3<3, 1, 3>;
    case kKindO3Fast + 4: return k_sweep_o3<2, 1, 4>;
    case kKindO3Fast + 5: return k_sweep_o3<3, 1, 4>;
    default: return nullptr;
  }
}

constexpr size_t kMaxDynSmem = 200 * 1024;

static int prepare_kernels() {
  static std::once_flag once;
  static cudaError_t status = cudaSuccess;
  std::call_once(once, [] {
    for (int k = 0; k < kKindO3Fast + 16; ++k) {
      if (!kernel_for(k)) continue;
      cudaError_t e = cudaFuncSetAttribute(kernel_for(k), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)kMaxDynSmem);
      if (e != cudaSuccess) status = e;
    }
    const void* extra[] = {(const void*)k_sweep_ising_resident<0>, (const void*)k_sweep_ising_resident<1>};
    for (const void* f : extra) {
      cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kIsingTileSmem);
      if (e != cudaSuccess) status = e;
    }
    const void* extra3[] = {(const void*)k_sweep_ising_resident3<0>, (const void*)k_sweep_ising_resident3<1>};
    for (const void* f : extra3) {
      cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxDynSmem);
      if (e != cudaSuccess) status = e;
    }
    for (int a = 0; a < 5; ++a)
      for (int c = 0; c < 4; ++c) {
        cudaError_t e = cudaFuncSetAttribute(kO3March[0][a][c], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)kMaxDynSmem);
        if (e != cudaSuccess) status = e;
      }
  });
  if (status != cudaSuccess)
    return fail(GPUMC_ECUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(status));
  return GPUMC_OK;
}

int launch_sweep_kernel(cudaStream_t st, int kind, const TileItem* tiles, int n_tiles,
                        LatDesc* lats, GroupDesc* groups, LaunchCtl* ctl, size_t smem) {
  if (n_tiles <= 0) return GPUMC_OK;
  if (is_cluster_kind(kind)) {
    // local bonds + union, global union across tiles, flip, account (+ epilogue)
#define CLUSTER_ROW(D, M, W) \
  {k_cluster_local<D, M, W>, k_cluster_global<D, M, W>, k_cluster_flip<D, M, W>, k_cluster_account<D, M, W>}
#define CLUSTER_O3_ROW(D, W) \
  {k_cluster_o3_local<D, W>, k_cluster_o3_global<D, W>, k_cluster_o3_flip<D, W>, k_cluster_o3_account<D, W>}
    static const SweepKernel ck[12][4] = {CLUSTER_ROW(2, ISING, 0), CLUSTER_ROW(3, ISING, 0),
                                          CLUSTER_ROW(2, POTTS, 0), CLUSTER_ROW(3, POTTS, 0),
                                          CLUSTER_ROW(2, ISING, 1), CLUSTER_ROW(3, ISING, 1),
                                          CLUSTER_ROW(2, POTTS, 1), CLUSTER_ROW(3, POTTS, 1),
                                          CLUSTER_O3_ROW(2, 0),     CLUSTER_O3_ROW(3, 0),
                                          CLUSTER_O3_ROW(2, 1),     CLUSTER_O3_ROW(3, 1)};
#undef CLUSTER_ROW
#undef CLUSTER_O3_ROW
    const int c = kind - kKindCluster;
    if (c < 0 || c >= 12) return fail(GPUMC_EINVAL, "internal: no cluster kernel for this layout");
    for (int i = 0; i < 3; ++i) ck[c][i]<<<n_tiles, kThreads, 0, st>>>(tiles, lats, groups, ctl);
    // the accounting kernel strides over the tiles, about eight per CTA
    ck[c][3]<<<std::max(1, std::min(n_tiles, (n_tiles + 7) / 8)), kThreads, 0, st>>>(tiles, lats, groups, ctl);
    CUDA_TRY(cudaGetLastError());
    return GPUMC_OK;
  }
  const SweepKernel k = kernel_for(kind);
  if (!k) return fail(GPUMC_EINVAL, "internal: no sweep kernel for this layout");
  // O(3) sweeps in place: colour 0, then colour 1 (which runs the epilogue)
  if (kind == 4) k_sweep_o3<2, 0, 0><<<n_tiles, kThreads, 0, st>>>(tiles, lats, groups, ctl);
  if (kind == 5) k_sweep_o3<3, 0, 0><<<n_tiles, kThreads, 0, st>>>(tiles, lats, groups, ctl);
  if (kind == kKindHeatBath + 4) k_sweep_o3<2, 0, 1><<<n_tiles, kThreads, 0, st>>>(tiles, lats, groups, ctl);
  if (kind == kKindHeatBath + 5) k_sweep_o3<3, 0, 1><<<n_tiles, kThreads, 0, st>>>(tiles, lats, groups, ctl);
  if (kind == kKindO3Uniform + 4) k_sweep_o3<2, 0, 2><<<n_tiles, kThreads, 0, st>>>(tiles, lats, groups, ctl);
  if (kind == kKindO3Uniform + 5) k_sweep_o3<3, 0, 2><<<n_tiles, kThreads, 0, st>>>(tiles, lats, groups, ctl);
  if (kind == kKindO3Opss + 4) k_sweep_o3<2, 0, 3><<<n_tiles, kThreads, 0, st>>>(tiles, lats, groups, ctl);
  if (kind == kKindO3Opss + 5) k_sweep_o3<3, 0, 3><<<n_tiles, kThreads, 0, st>>>(tiles, lats, groups, ctl);
  if (kind == kKindO3Fast + 4) k_sweep_o3<2, 0, 4><<<n_tiles, kThreads, 0, st>>>(tiles, lats, groups, ctl);
  if (kind == kKindO3Fast + 5) k_sweep_o3<3, 0, 4><<<n_tiles, kThreads, 0, st>>>(tiles, lats, groups, ctl);
  if (is_o3_march_kind(kind)) o3_march_kernel(0, kind)<<<n_tiles, kThreads, smem, st>>>(tiles, lats, groups, ctl);
  k<<<n_tiles, kThreads, smem, st>>>(tiles, lats, groups, ctl);
  CUDA_TRY(cudaGetLastError());
  return GPUMC_OK;
}

int launch_msc_measure(cudaStream_t st, const Layout& L, const LatDesc* lats, int lat,
                       unsigned long long* counters) {
  const int blocks = (int)std::min<int64_t>(1184, (L.n_sites + kThreads - 1) / kThreads);
  if (L.dims == 2)
    k_msc_measure<2><<<blocks, kThreads, 0, st>>>(lats, lat, counters);
  else
    k_msc_measure<3><<<blocks, kThreads, 0, st>>>(lats, lat, counters);
  CUDA_TRY(cudaGetLastError());
  return GPUMC_OK;
}

int launch_msc_record(cudaStream_t st, LatDesc* lats, GroupDesc* groups, int group,
                      unsigned long long* counters) {
  k_msc_record<<<1, 256, 0, st>>>(lats, groups, group, counters);
  CUDA_TRY(cudaGetLastError());
  return GPUMC_OK;
}

}  // namespace gpumc

using namespace gpumc;

// ===========================================================================
// engine
// ===========================================================================
static int check_device(int device) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0)
    return fail(GPUMC_ENODEV, std::string("no usable CUDA device: ") +
                                  (e == cudaSuccess ? "device count is 0" : cudaGetErrorString(e)));
  if (device < 0 || device >= n) return fail(GPUMC_ENODEV, "device index out of range");
  return GPUMC_OK;
}

int gpumc_engine_create(int32_t device, gpumc_engine** out) {
  if (!out) return fail(GPUMC_EINVAL, "out: null pointer");
  int rc = check_device(device);
  if (rc) return rc;
  CUDA_TRY(cudaSetDevice(device));
  rc = prepare_kernels();
  if (rc) return rc;
  gpumc_engine* e = new gpumc_engine();
  e->device = device;
  cudaError_t err = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
  if (err == cudaSuccess) err = cudaMalloc(&e->d_lats, sizeof(LatDesc) * e->lat_cap);
  if (err == cudaSuccess) err = cudaMalloc(&e->d_groups, sizeof(GroupDesc) * e->group_cap);
  if (err == cudaSuccess) err = cudaMemset(e->d_lats, 0, sizeof(LatDesc) * e->lat_cap);
  if (err == cudaSuccess) err = cudaMemset(e->d_groups, 0, sizeof(GroupDesc) * e->group_cap);
  if (err != cudaSuccess) {
    delete e;
    return fail(GPUMC_ECUDA, std::string("engine allocation: ") + cudaGetErrorString(err));
  }
  // Simulations allocate from the device's stream-ordered pool: keep freed
  // memory pooled (no release to the driver at synchronisation points), so
  // admitting a job after another retired reuses its memory without mapping
  // pages or synchronising the device.  The pool setting belongs to this
  // process; destroying the engine trims the pool again.
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  int n_sm = 0, per_sm = 0;
  err = cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, device);
  if (err == cudaSuccess)
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep_ising_bits<2, 0>, kThreads, kIsingTileSmem);
  if (err != cudaSuccess) {
    delete e;
    return fail(GPUMC_ECUDA, std::string("device query: ") + cudaGetErrorString(err));
  }
  e->slots = std::max(1, n_sm * std::max(1, per_sm));
  int per_sm3 = 0;
  err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm3, k_sweep_ising_bits<3, 0>, kThreads, 16 * 1024);
  if (err != cudaSuccess) {
    delete e;
    return fail(GPUMC_ECUDA, std::string("device query: ") + cudaGetErrorString(err));
  }
  e->slots3 = std::max(1, n_sm * std::max(1, per_sm3));
  e->lat_used.assign(e->lat_cap, false);
  e->group_used.assign(e->group_cap, false);
  *out = e;
  return GPUMC_OK;
}

gpumc_engine::~gpumc_engine() {
  cudaSetDevice(device);
  drop_graphs();
  for (auto& p : batch_plans) p.release(stream);
  if (stream) cudaStreamSynchronize(stream);
  for (cudaStream_t s2 : side) {
    cudaStreamSynchronize(s2);
    cudaStreamDestroy(s2);
  }
  for (cudaEvent_t ev : side_done) cudaEventDestroy(ev);
  if (fork) cudaEventDestroy(fork);
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
  if (d_lats) cudaFree(d_lats);
  if (d_groups) cudaFree(d_groups);
  if (stream) cudaStreamDestroy(stream);
}

void gpumc_engine::drop_graphs() {
  for (auto& kv : batch_graphs) cudaGraphExecDestroy(kv.second);
  batch_graphs.clear();
}

int gpumc_engine_destroy(gpumc_engine* eng) {
  if (!eng) return GPUMC_OK;
  if (!eng->sims.empty()) return fail(GPUMC_ESTATE, "engine still has simulations");
  delete eng;
  return GPUMC_OK;
}

int gpumc_engine_synchronize(gpumc_engine* eng) {
  if (!eng) return fail(GPUMC_EINVAL, "engine: null");
  CUDA_TRY(cudaSetDevice(eng->device));
  CUDA_TRY(cudaStreamSynchronize(eng->stream));
  return GPUMC_OK;
}

int gpumc_engine_stream(gpumc_engine* eng, void** stream) {
  if (!eng || !stream) return fail(GPUMC_EINVAL, "null argument");
  *stream = (void*)eng->stream;
  return GPUMC_OK;
}

int gpumc_sim_engine(gpumc_sim* sim, gpumc_engine** eng) {
  if (!sim || !eng) return fail(GPUMC_EINVAL, "null argument");
  *eng = sim->eng;
  return GPUMC_OK;
}

int gpumc_engine_set_temporal_blocking(gpumc_engine* eng, int32_t enable) {
  if (!eng) return fail(GPUMC_EINVAL, "engine: null");
  if (eng->blocking != (enable != 0)) {
    eng->blocking = enable != 0;
    eng->drop_graphs();  // captured sweeps depend on which plans run resident
  }
  return GPUMC_OK;
}

int gpumc_engine_set_concurrent_kinds(gpumc_engine* eng, int32_t enable) {
  if (!eng) return fail(GPUMC_EINVAL, "engine: null");
  if (eng->concurrent != (enable != 0)) {
    eng->concurrent = enable != 0;
    eng->drop_graphs();  // captured sweeps depend on the stream layout
  }
  return GPUMC_OK;
}

int gpumc_engine_set_tile_refinement(gpumc_engine* eng, int32_t enable) {
  if (!eng) return fail(GPUMC_EINVAL, "engine: null");
  if (eng->refine != (enable != 0)) {
    eng->refine = enable != 0;
    eng->batch_dirty = true;  // the next engine sweep re-plans the batch
  }
  return GPUMC_OK;
}

int gpumc_engine_launch_count(gpumc_engine* eng, uint64_t* n) {
  if (!eng || !n) return fail(GPUMC_EINVAL, "null argument");
  *n = eng->launches;
  return GPUMC_OK;
}

int gpumc_launches_per_sweep(gpumc_sim* sim, int32_t* n) {
  if (!sim || !n) return fail(GPUMC_EINVAL, "null argument");
  *n = (sim->lay.cluster ? 4 : sim->lay.model == O3 ? 2 : 1) +
       ((sim->lay.model == MSC && sim->phase == GPUMC_PHASE_MEASUREMENT) ? sim->n_rep + 1 : 0);
  return GPUMC_OK;
}

void BatchPlan::release(cudaStream_t st) {
  dev_free(d_tiles, st);
  dev_free(d_gids, st);
  dev_free(d_ctl, st);
  d_tiles = nullptr;
  d_gids = nullptr;
  d_ctl = nullptr;
  res.release(st);
}

void ResidentPlan::release(cudaStream_t st) {
  dev_free(d_nbr, st);
  dev_free(d_xchg, st);
  d_nbr = nullptr;
  d_xchg = nullptr;
  on = false;
}

// 3D path of build_resident: whole-plane slabs of at least two planes, each
// lattice's slabs consecutive in z order (enumerate_tiles), neighbours the
// previous and next slab of its run, cyclically.
static int build_resident3(int device, cudaStream_t st, const std::vector<TileItem>& tiles,
                           const std::map<int, const Layout*>& layout_of_lat, ResidentPlan& rp) {
  int pwmax = 0;
  size_t smem = 0;
  std::vector<int2> nbr(tiles.size());
  for (size_t i = 0; i < tiles.size();) {
    auto it = layout_of_lat.find(tiles[i].lat);
    if (it == layout_of_lat.end()) return GPUMC_OK;
    const Layout& L = *it->second;
    const int nseg = L.pitch / 64;
    if (L.model != ISING || L.dims != 3 || L.tile_cx != nseg || L.tile_y != L.ly) return GPUMC_OK;
    if (i == 0) rp.alg = L.alg;
    if (L.alg != rp.alg) return GPUMC_OK;
    size_t j = i;
    while (j < tiles.size() && tiles[j].lat == tiles[i].lat) ++j;
    const int n = (int)(j - i);
    for (int k = 0; k < n; ++k) {
      const TileItem& t = tiles[i + k];
      if (t.x0 != 0 || t.y0 != 0 || t.ty < L.ly || t.cx != nseg || t.z0 != k * t.tz ||
          std::min(t.tz, L.lz - t.z0) < 2)
        return GPUMC_OK;
      smem = std::max(smem, (size_t)8 * (size_t)(std::min(t.tz, L.lz) + 4) * L.ly * nseg);
      nbr[i + k] = make_int2((int)i + (k + n - 1) % n, (int)i + (k + 1) % n);
    }
    pwmax = std::max(pwmax, L.ly * nseg);
    i = j;
  }
  if (smem > kMaxDynSmem) return GPUMC_OK;
  int coop = 0, n_sm = 0, per_sm = 0;
  CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
  CUDA_TRY(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, device));
  CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, rp.alg == HEAT_BATH ? k_sweep_ising_resident3<1> : k_sweep_ising_resident3<0>, kThreads, smem));
  if (!coop || (int64_t)per_sm * n_sm < (int64_t)tiles.size()) return GPUMC_OK;
  rp.dims = 3;
  rp.smem = smem;
  rp.xstride = 2 * 4 * pwmax;
  CUDA_TRY(cudaMallocAsync(&rp.d_nbr, sizeof(int2) * nbr.size(), st));
  CUDA_TRY(cudaMemcpyAsync(rp.d_nbr, nbr.data(), sizeof(int2) * nbr.size(), cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMallocAsync(&rp.d_xchg, sizeof(uint2) * (size_t)rp.xstride * tiles.size(), st));
  rp.on = true;
  return GPUMC_OK;
}

int gpumc::build_resident(int device, cudaStream_t st, const std::vector<TileItem>& tiles,
                          const std::map<int, const Layout*>& layout_of_lat, size_t smem, ResidentPlan& rp) {
  rp.release(st);
  if (tiles.empty()) return GPUMC_OK;
  {
    auto it = layout_of_lat.find(tiles[0].lat);
    if (it != layout_of_lat.end() && it->second->dims == 3) return build_resident3(device, st, tiles, layout_of_lat, rp);
  }
  if (smem > kIsingTileSmem) return GPUMC_OK;
  // every tile a whole-row 2D Ising tile of >= 2 rows; a lattice's tiles are
  // consecutive in y order (enumerate_tiles), so its neighbours are the
  // previous and next tile of its run, cyclically
  int wmax = 0;
  std::vector<int2> nbr(tiles.size());
  for (size_t i = 0; i < tiles.size();) {
    auto it = layout_of_lat.find(tiles[i].lat);
    if (it == layout_of_lat.end()) return GPUMC_OK;
    const Layout& L = *it->second;
    if (L.model != ISING || L.dims != 2 || L.tile_cx != L.pitch / 64) return GPUMC_OK;
    if (i == 0) rp.alg = L.alg;
    if (L.alg != rp.alg) return GPUMC_OK;
    size_t j = i;
    while (j < tiles.size() && tiles[j].lat == tiles[i].lat) ++j;
    const int n = (int)(j - i);
    for (int k = 0; k < n; ++k) {
      const TileItem& t = tiles[i + k];
      if (t.x0 != 0 || t.y0 != k * L.tile_y || std::min(L.tile_y, L.ly - t.y0) < 2) return GPUMC_OK;
      nbr[i + k] = make_int2((int)i + (k + n - 1) % n, (int)i + (k + 1) % n);
    }
    wmax = std::max(wmax, L.pitch / 64);
    i = j;
  }
  int coop = 0, n_sm = 0, per_sm = 0;
  CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
  CUDA_TRY(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, device));
  CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, rp.alg == HEAT_BATH ? k_sweep_ising_resident<1> : k_sweep_ising_resident<0>, kThreads, smem));
  if (!coop || (int64_t)per_sm * n_sm < (int64_t)tiles.size()) return GPUMC_OK;
  rp.dims = 2;
  rp.smem = smem;
  rp.xstride = 2 * 4 * wmax;
  CUDA_TRY(cudaMallocAsync(&rp.d_nbr, sizeof(int2) * nbr.size(), st));
  CUDA_TRY(cudaMemcpyAsync(rp.d_nbr, nbr.data(), sizeof(int2) * nbr.size(), cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMallocAsync(&rp.d_xchg, sizeof(uint2) * (size_t)rp.xstride * tiles.size(), st));
  rp.on = true;
  return GPUMC_OK;
}

// Zeroes the per-sweep accumulators of every lattice of a tile list (after a
// resident launch gave up, its partial sums must not reach a later epilogue).
__global__ void k_reset_accumulators(const TileItem* __restrict__ tiles, int n_tiles, LatDesc* __restrict__ lats) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_tiles; i += gridDim.x * blockDim.x) {
    LatDesc* L = &lats[tiles[i].lat];
    L->acc = Accum{};
    L->acc2 = Accum{};
  }
}

int gpumc::launch_resident(cudaStream_t st, const TileItem* tiles, int n_tiles, LatDesc* lats,
                           GroupDesc* groups, LaunchCtl* ctl, const ResidentPlan& rp, size_t smem,
                           int n_sweeps, long long spin_limit) {
  // bar, err and epi are adjacent: one memset clears them
  CUDA_TRY(cudaMemsetAsync(&ctl->bar, 0, 2 * sizeof(unsigned int) + sizeof(int32_t), st));
  const int2* nbr = rp.d_nbr;
  uint2* xchg = rp.d_xchg;
  int xstride = rp.xstride;
  void* args[] = {(void*)&tiles, (void*)&lats, (void*)&groups, (void*)&ctl,
                  (void*)&nbr, (void*)&xchg, (void*)&xstride, (void*)&n_sweeps, (void*)&spin_limit};
  const void* kern = rp.dims == 3 ? (rp.alg == HEAT_BATH ? (const void*)k_sweep_ising_resident3<1>
                                                         : (const void*)k_sweep_ising_resident3<0>)
                                  : (rp.alg == HEAT_BATH ? (const void*)k_sweep_ising_resident<1>
                                                         : (const void*)k_sweep_ising_resident<0>);
  CUDA_TRY(cudaLaunchCooperativeKernel(kern, dim3(n_tiles), dim3(kThreads),
                                       args, rp.smem ? rp.smem : smem, st));
  int32_t err = 0;
  CUDA_TRY(cudaMemcpyAsync(&err, &ctl->err, sizeof(err), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  if (err) {
    // the CTAs left at their next wait: no state was stored by the CTAs that
    // gave up, and the launch's sweep counters and caches are not a
    // trajectory; clear the partial sums so the handle can be restored
    k_reset_accumulators<<<(n_tiles + 255) / 256, 256, 0, st>>>(tiles, n_tiles, lats);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(st));
    return fail(GPUMC_ECUDA,
                "resident sweep: a grid-barrier wait gave up after " + std::to_string(spin_limit) +
                    " polls; the handle's spins, sweep count and energy cache must be restored "
                    "(gpumc_set_spins / gpumc_set_sweep_count or a snapshot)");
  }
  return GPUMC_OK;
}

namespace gpumc {
int bounds_read_sweep_o3(unsigned long long*, unsigned int*);
int bounds_read_sweep_ising_bits(unsigned long long*, unsigned int*);
int bounds_read_sweep_potts_bits(unsigned long long*, unsigned int*);
int bounds_read_sweep_discrete(unsigned long long*, unsigned int*);
int bounds_read_sweep_msc(unsigned long long*, unsigned int*);
int bounds_read_cluster(unsigned long long*, unsigned int*);
int bounds_read_lattice_ops(unsigned long long*, unsigned int*);
}  // namespace gpumc

int gpumc_debug_bounds(uint64_t* hits, int32_t* first_module, int32_t* first_line, int32_t* compiled) {
  if (!hits || !first_module || !first_line || !compiled) return fail(GPUMC_EINVAL, "null argument");
  int (*const readers[])(unsigned long long*, unsigned int*) = {
      bounds_read_sweep_o3,   bounds_read_sweep_ising_bits, bounds_read_sweep_potts_bits,
      bounds_read_sweep_discrete, bounds_read_sweep_msc,    bounds_read_cluster,
      bounds_read_lattice_ops};
  *hits = 0;
  *first_module = -1;
  *first_line = 0;
  *compiled = 1;
  for (int m = 0; m < (int)(sizeof(readers) / sizeof(readers[0])); ++m) {
    unsigned long long h = 0;
    unsigned int line = 0;
    const int rc = readers[m](&h, &line);
    if (rc < 0) return fail(GPUMC_ECUDA, "bounds counters: symbol copy failed");
    if (rc > 0) *compiled = 0;  // release build: no checks compiled in
    if (h && *first_module < 0) {
      *first_module = m;
      *first_line = (int32_t)line;
    }
    *hits += h;
  }
  return GPUMC_OK;
}

int gpumc_set_tile_knobs(const gpumc_tile_knobs* knobs) {
  if (!knobs) return fail(GPUMC_EINVAL, "knobs: null");
  const int32_t v[6] = {knobs->ising2d_rows, knobs->ising3d_planes, knobs->potts_segments,
                        knobs->potts3d_planes, knobs->o3_rows, knobs->o3_planes};
  for (int32_t x : v)
    if (x < 0 || x > 4096) return fail(GPUMC_EINVAL, "knobs: each value must be in 0..4096 (0 = analytic)");
  std::lock_guard<std::mutex> lock(g_knobs_mu);
  g_knobs = *knobs;
  return GPUMC_OK;
}

int gpumc_get_tile_knobs(gpumc_tile_knobs* knobs) {
  if (!knobs) return fail(GPUMC_EINVAL, "knobs: null");
  *knobs = current_knobs();
  return GPUMC_OK;
}

int gpumc::check_launch_flag(cudaStream_t st, LaunchCtl* ctl) {
  int32_t err = 0;
  CUDA_TRY(cudaMemcpyAsync(&err, &ctl->err, sizeof(err), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  if (!err) return GPUMC_OK;
  CUDA_TRY(cudaMemsetAsync(&ctl->err, 0, sizeof(int32_t), st));
  CUDA_TRY(cudaStreamSynchronize(st));
  return fail(GPUMC_ECUDA, "O(3) sweep: a shared-memory plane copy did not complete in time; the launch's "
                           "spins, energies and records are not a trajectory and must be restored");
}

int gpumc_engine_set_wait_limit(gpumc_engine* eng, int64_t polls) {
  if (!eng) return fail(GPUMC_EINVAL, "engine: null");
  if (polls < 0) return fail(GPUMC_EINVAL, "polls: must be >= 0");
  eng->wait_limit = polls;
  return GPUMC_OK;
}


int gpumc_engine::rebuild_batch() {
  if (!batch_dirty) return GPUMC_OK;
  drop_graphs();
  for (auto& p : batch_plans) p.release(stream);
  batch_plans.clear();
  std::map<int, BatchPlan> plans;
  std::map<int, std::vector<TileItem>> tiles;
  std::map<int, std::vector<int32_t>> gids;
  std::map<int, std::vector<int32_t>> gtiles;  // tiles of each group of a plan
  std::map<int, const Layout*> layout_of_lat;
  // tile shapes for this batch: the simulations of one kernel family (kind
  // of the creation-time plan) share its launch and are refined together
  std::map<int, std::vector<gpumc_sim*>> family;
  for (gpumc_sim* s : sims) family[kernel_kind(s->base)].push_back(s);
  for (auto& kv : family) {
    std::vector<Layout> lays;
    std::vector<int> reps;
    for (gpumc_sim* s : kv.second) {
      lays.push_back(s->base);
      reps.push_back(s->n_rep);
    }
    if (refine) refine_layouts(lays, reps, family_slots(lays[0], slots, slots3));
    for (size_t i = 0; i < kv.second.size(); ++i) kv.second[i]->blay = lays[i];
  }
  for (gpumc_sim* s : sims) {
    const int kind = kernel_kind(s->blay);
    BatchPlan& p = plans[kind];
    p.kind = kind;
    p.smem = std::max(p.smem, s->blay.smem);
    const size_t first = tiles[kind].size();
    for (int r = 0; r < s->n_rep; ++r) {
      enumerate_tiles(s->blay, s->lat0 + r, tiles[kind]);
      layout_of_lat[s->lat0 + r] = &s->blay;
    }
    const int32_t pos = (int32_t)gids[kind].size();  // the group's position in the plan
    for (size_t i = first; i < tiles[kind].size(); ++i) tiles[kind][i].pad = pos;
    gids[kind].push_back(s->group);
    gtiles[kind].push_back((int32_t)(tiles[kind].size() - first));
  }
  for (auto& kv : plans) {
    BatchPlan p = kv.second;
    auto& tv = tiles[kv.first];
    auto& gv = gids[kv.first];
    p.n_tiles = (int)tv.size();
    p.n_groups = (int)gv.size();
    // group ids, tiles per group, done counters (zero) in one buffer
    std::vector<int32_t> gbuf(gv);
    gbuf.insert(gbuf.end(), gtiles[kv.first].begin(), gtiles[kv.first].end());
    gbuf.resize(3 * gv.size(), 0);
    CUDA_TRY(cudaMallocAsync(&p.d_tiles, sizeof(TileItem) * tv.size(), stream));
    CUDA_TRY(cudaMallocAsync(&p.d_gids, sizeof(int32_t) * gbuf.size(), stream));
    CUDA_TRY(cudaMallocAsync(&p.d_ctl, sizeof(LaunchCtl), stream));
    CUDA_TRY(cudaMemcpyAsync(p.d_tiles, tv.data(), sizeof(TileItem) * tv.size(), cudaMemcpyHostToDevice, stream));
    CUDA_TRY(cudaMemcpyAsync(p.d_gids, gbuf.data(), sizeof(int32_t) * gbuf.size(), cudaMemcpyHostToDevice, stream));
    LaunchCtl c;
    c.done = 0;
    c.n_groups = p.n_groups;
    c.group_ids = p.d_gids;
    c.group_tiles = p.d_gids + gv.size();
    c.group_done = (unsigned int*)(p.d_gids + 2 * gv.size());
    c.n_tiles = p.n_tiles;
    CUDA_TRY(cudaMemcpyAsync(p.d_ctl, &c, sizeof(c), cudaMemcpyHostToDevice, stream));
    if (is_ising_bits_kind(p.kind)) {
      int rc = build_resident(device, stream, tv, layout_of_lat, p.smem, p.res);
      if (rc) {
        p.release(stream);
        return rc;
      }
    }
    batch_plans.push_back(p);
  }
  batch_dirty = false;
  return GPUMC_OK;
}

bool gpumc_engine::has_per_sweep_work() const { return launches_per_batch_sweep() > 0; }

// Kernel launches of one launch_batch_sweep (resident plans excluded).
uint64_t gpumc_engine::launches_per_batch_sweep() const {
  uint64_t n = 0;
  for (const auto& p : batch_plans)
    if (!(p.res.on && blocking)) {
      const int base = p.kind % kKindHeatBath;  // O(3) sweeps are two colour launches
      n += is_cluster_kind(p.kind) ? 4 : (base == 4 || base == 5 || is_o3_march_kind(p.kind)) ? 2 : 1;
    }
  for (gpumc_sim* s : sims)
    if (s->lay.model == MSC && s->phase == GPUMC_PHASE_MEASUREMENT) n += (uint64_t)s->n_rep + 1;
  return n;
}

int gpumc_engine::launch_batch_sweep() {
  for (auto& p : batch_plans) {
    if (p.res.on && blocking) continue;  // resident plans run whole chunks in one launch
    int rc = launch_sweep_kernel(stream, p.kind, p.d_tiles, p.n_tiles, d_lats, d_groups, p.d_ctl, p.smem);
    if (rc) return rc;
  }
  for (gpumc_sim* s : sims) {
    if (s->lay.model == MSC && s->phase == GPUMC_PHASE_MEASUREMENT) {
      int rc = s->launch_msc_measurement();
      if (rc) return rc;
    }
  }
  return GPUMC_OK;
}

int gpumc_engine_sweep(gpumc_engine* eng, uint32_t n_sweeps) {
  if (!eng) return fail(GPUMC_EINVAL, "engine: null");
  CUDA_TRY(cudaSetDevice(eng->device));
  int rc = eng->rebuild_batch();
  if (rc) return rc;
  if (eng->sims.empty() || n_sweeps == 0) return GPUMC_OK;
  uint32_t left = n_sweeps;
  while (left > 0) {
    // never outrun the smallest free record space of a measuring simulation
    uint32_t room = left;
    for (gpumc_sim* s : eng->sims) {
      rc = s->measure_room(room);
      if (rc) return rc;
    }
    uint32_t chunk = std::min<uint32_t>(room, 64);
    for (gpumc_sim* s : eng->sims)
      if (const uint32_t to_audit = s->sweeps_to_audit()) chunk = std::min(chunk, to_audit);
    if (eng->has_per_sweep_work()) {
      rc = eng->use_graphs ? eng->run_graph(chunk) : eng->launch_batch_sweeps(chunk);
      eng->launches += (uint64_t)chunk * eng->launches_per_batch_sweep();
    }
    for (auto& p : eng->batch_plans)
      if (rc == GPUMC_OK && p.res.on && eng->blocking) {
        rc = launch_resident(eng->stream, p.d_tiles, p.n_tiles, eng->d_lats, eng->d_groups, p.d_ctl, p.res,
                             p.smem, (int)chunk, eng->wait_limit);
        eng->launches += 1;
      }
    if (rc) return rc;
    for (gpumc_sim* s : eng->sims) {
      s->sweeps = std::min<uint64_t>(s->sweeps + chunk, s->target);
      s->note_measured(chunk);
    }
    for (gpumc_sim* s : eng->sims)
      if (s->audit_interval && s->sweeps % s->audit_interval == 0 && (rc = s->audit()) != GPUMC_OK) return rc;
    left -= chunk;
  }
  for (auto& p : eng->batch_plans)
    if (is_o3_march_kind(p.kind) && (rc = check_launch_flag(eng->stream, p.d_ctl)) != GPUMC_OK) return rc;
  return GPUMC_OK;
}

int gpumc_engine::ensure_side(size_t n) {
  if (!fork) CUDA_TRY(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
  while (side.size() < n) {
    cudaStream_t s2 = nullptr;
    cudaEvent_t ev = nullptr;
    CUDA_TRY(cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking));
    cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e != cudaSuccess) {
      cudaStreamDestroy(s2);
      return fail(GPUMC_ECUDA, std::string("event create: ") + cudaGetErrorString(e));
    }
    side.push_back(s2);
    side_done.push_back(ev);
  }
  return GPUMC_OK;
}

static bool is_msc_kind(int kind) { return kind == MSC * 2 || kind == MSC * 2 + 1; }

// n sweeps of every plan that runs per sweep.  The plans of a batch touch
// disjoint lattices (one kernel kind each, each with its own launch control
// and groups), so with `concurrent` every plan runs its n sweeps on a stream
// of its own, forked from and joined back into the engine stream by events
// (the same inside graph capture), and the kinds fill each other's idle SMs.
// Multi-spin plans and their measurement kernels stay on the engine stream,
// in sweep order.
int gpumc_engine::launch_batch_sweeps(uint32_t n) {
  std::vector<size_t> fan;
  for (size_t i = 0; i < batch_plans.size(); ++i) {
    const BatchPlan& p = batch_plans[i];
    if (!(p.res.on && blocking) && !is_msc_kind(p.kind)) fan.push_back(i);
  }
  if (!concurrent || fan.size() < 2) {
    for (uint32_t k = 0; k < n; ++k) {
      const int rc = launch_batch_sweep();
      if (rc) return rc;
    }
    return GPUMC_OK;
  }
  int rc = ensure_side(fan.size());
  if (rc) return rc;
  CUDA_TRY(cudaEventRecord(fork, stream));
  size_t forked = 0;  // side streams that wait on the fork and must be joined
  for (size_t j = 0; j < fan.size() && rc == GPUMC_OK; ++j) {
    const BatchPlan& p = batch_plans[fan[j]];
    if (cudaStreamWaitEvent(side[j], fork, 0) != cudaSuccess) {
      rc = fail(GPUMC_ECUDA, "stream fork failed");
      break;
    }
    ++forked;
    for (uint32_t k = 0; k < n && rc == GPUMC_OK; ++k)
      rc = launch_sweep_kernel(side[j], p.kind, p.d_tiles, p.n_tiles, d_lats, d_groups, p.d_ctl, p.smem);
  }
  for (uint32_t k = 0; k < n && rc == GPUMC_OK; ++k) {
    for (const BatchPlan& p : batch_plans) {
      if (!is_msc_kind(p.kind) || (p.res.on && blocking) || rc) continue;
      rc = launch_sweep_kernel(stream, p.kind, p.d_tiles, p.n_tiles, d_lats, d_groups, p.d_ctl, p.smem);
    }
    for (gpumc_sim* s : sims)
      if (!rc && s->lay.model == MSC && s->phase == GPUMC_PHASE_MEASUREMENT) rc = s->launch_msc_measurement();
  }
  // join every forked stream, on success and on error alike, so that the
  // engine stream (and a capture in progress) never leaves work behind
  for (size_t j = 0; j < forked; ++j) {
    if (cudaEventRecord(side_done[j], side[j]) != cudaSuccess ||
        cudaStreamWaitEvent(stream, side_done[j], 0) != cudaSuccess) {
      if (!rc) rc = fail(GPUMC_ECUDA, "stream join failed");
    }
  }
  return rc;
}

int gpumc_engine::run_graph(uint32_t n) {
  auto it = batch_graphs.find(n);
  if (it == batch_graphs.end()) {
    cudaGraph_t g;
    if (concurrent) {  // create the side streams outside the capture
      const int rs = ensure_side(batch_plans.size());
      if (rs) return rs;
    }
    CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    const int rc = launch_batch_sweeps(n);
    cudaError_t e = cudaStreamEndCapture(stream, &g);
    if (rc) return rc;
    if (e != cudaSuccess) return fail(GPUMC_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    cudaGraphExec_t ex;
    e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(GPUMC_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    it = batch_graphs.emplace(n, ex).first;
  }
  CUDA_TRY(cudaGraphLaunch(it->second, stream));
  return GPUMC_OK;
}

int gpumc_engine::alloc_slots(int n, int& first) {
  // first fit of n consecutive free lattice slots
  int run = 0;
  for (int i = 0; i < lat_cap; ++i) {
    run = lat_used[i] ? 0 : run + 1;
    if (run == n) {
      first = i - n + 1;
      for (int j = first; j <= i; ++j) lat_used[j] = true;
      return GPUMC_OK;
    }
  }
  return fail(GPUMC_ENOMEM, "lattice descriptor pool exhausted");
}

int gpumc_engine::alloc_group(int& g) {
  for (int i = 0; i < group_cap; ++i)
    if (!group_used[i]) {
      group_used[i] = true;
      g = i;
      return GPUMC_OK;
    }
  return fail(GPUMC_ENOMEM, "group descriptor pool exhausted");
}

int gpumc_last_error(char* buf, size_t cap) {
  if (!buf || cap == 0) return (int)gpumc::g_last_error_size();
  const std::string& m = gpumc::last_error_ref();
  const size_t k = std::min(cap - 1, m.size());
  std::memcpy(buf, m.data(), k);
  buf[k] = 0;
  return GPUMC_OK;
}
