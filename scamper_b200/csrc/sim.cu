// Simulation handles: ClassicalMC-style construction, sweeps, observables,
// spin I/O and the parallel-tempering contract over the C ABI.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gpumc.h"
#include "engine.h"
#include "host_internal.h"

namespace gpumc {
__global__ void k_init_discrete(int8_t*, int, int, int, int, int, int, uint64_t, int);
__global__ void k_init_o3(float*, int, int, int, int, uint64_t, int);
__global__ void k_init_msc(unsigned long long*, int, int, int, int, const uint64_t*, int);
__global__ void k_energy_i8(const int8_t*, int, int, int, int, int, int, unsigned long long*, unsigned int*);
__global__ void k_energy_msc(const unsigned long long*, int, int, int, int, unsigned long long*);
__global__ void k_energy_o3(const float*, int, int, int, int, double, double*);
__global__ void k_philox_probe(const uint4*, const uint2*, uint4*, int);
}  // namespace gpumc

using namespace gpumc;

#define CUDA_TRY(expr)                                                            \
  do {                                                                            \
    cudaError_t e_ = (expr);                                                      \
    if (e_ != cudaSuccess)                                                        \
      return fail(e_ == cudaErrorMemoryAllocation ? GPUMC_ENOMEM : GPUMC_ECUDA,   \
                  std::string(#expr) + ": " + cudaGetErrorString(e_));            \
  } while (0)

#define RC_TRY(expr)      \
  do {                    \
    int rc_ = (expr);     \
    if (rc_) return rc_;  \
  } while (0)

static const int kInitBlocks = 1184;

gpumc_sim::~gpumc_sim() {
  cudaSetDevice(eng->device);
  cudaStreamSynchronize(eng->stream);
  drop_graphs();
  // stream-ordered frees: no device-wide synchronisation, the memory goes
  // back to the pool for the next simulation
  const cudaStream_t st = eng->stream;
  for (size_t i = 0; i < bufs.size(); ++i)
    if (bufs[i] && (i % 2 == 0 || bufs[i] != bufs[i - 1])) dev_free(bufs[i], st);
  dev_free(d_head, st);
  dev_free(d_tail, st);
  dev_free(d_betas, st);
  dev_free(d_betas_f, st);
  dev_free(d_label, st);
  dev_free(d_rep_at, st);
  dev_free(d_records, st);
  for (void* p : aux) dev_free(p, st);
  dev_free(d_bin_open, st);
  dev_free(d_bins, st);
  dev_free(d_msc_counters, st);
  dev_free(d_tiles, st);
  dev_free(d_gid, st);
  dev_free(d_ctl, st);
  res.release(st);
}

// The tile list of the simulation's own launches, from `lay`; a launch
// control block that exists already gets the new tile count.
int gpumc_sim::upload_own_tiles(std::vector<TileItem>& tiles) {
  tiles.clear();
  for (int r = 0; r < n_rep; ++r) enumerate_tiles(lay, lat0 + r, tiles);
  TileItem* d = nullptr;
  CUDA_TRY(cudaMallocAsync(&d, sizeof(TileItem) * tiles.size(), eng->stream));
  CUDA_TRY(cudaMemcpyAsync(d, tiles.data(), sizeof(TileItem) * tiles.size(), cudaMemcpyHostToDevice, eng->stream));
  dev_free(d_tiles, eng->stream);
  d_tiles = d;
  n_tiles = (int)tiles.size();
  if (d_ctl) {
    const int32_t n = n_tiles;
    CUDA_TRY(cudaMemcpyAsync(&d_ctl->n_tiles, &n, sizeof(n), cudaMemcpyHostToDevice, eng->stream));
    CUDA_TRY(cudaMemcpyAsync(d_gid + 1, &n, sizeof(n), cudaMemcpyHostToDevice, eng->stream));  // the group's tiles
    CUDA_TRY(cudaStreamSynchronize(eng->stream));  // `n` lives on this stack frame
  }
  return GPUMC_OK;
}

void gpumc_sim::drop_graphs() {
  for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
  graphs.clear();
}

int gpumc_sim::upload_tables() {
  std::vector<uint32_t> head((size_t)n_temps * n_cls);
  std::vector<unsigned long long> tail((size_t)n_temps * n_cls);
  std::vector<float> bf(n_temps);
  for (int t = 0; t < n_temps; ++t) {
    build_table(lay.model == MSC ? ISING : lay.model, lay.dims, spec.J, betas[t], &head[(size_t)t * n_cls],
                &tail[(size_t)t * n_cls], lay.alg);
    bf[t] = (float)betas[t];
  }
  CUDA_TRY(cudaMemcpyAsync(d_head, head.data(), head.size() * 4, cudaMemcpyHostToDevice, eng->stream));
  CUDA_TRY(cudaMemcpyAsync(d_tail, tail.data(), tail.size() * 8, cudaMemcpyHostToDevice, eng->stream));
  CUDA_TRY(cudaMemcpyAsync(d_betas, betas.data(), betas.size() * 8, cudaMemcpyHostToDevice, eng->stream));
  CUDA_TRY(cudaMemcpyAsync(d_betas_f, bf.data(), bf.size() * 4, cudaMemcpyHostToDevice, eng->stream));
  CUDA_TRY(cudaStreamSynchronize(eng->stream));
  return GPUMC_OK;
}

int gpumc_sim::push_phase_flags() {
  const int32_t measure = phase == GPUMC_PHASE_MEASUREMENT ? 1 : 0;
  RC_TRY(set_group_field(offsetof(GroupDesc, measure), measure));
  if (lay.model == O3) {
    // the cone adapts during thermalization; the heat bath has no cone
    const int32_t adapt =
        phase == GPUMC_PHASE_THERMALIZATION && lay.alg == METROPOLIS && lay.prop != GPUMC_O3_UNIFORM ? 1 : 0;
    for (int r = 0; r < n_rep; ++r) RC_TRY(set_lat_field(r, offsetof(LatDesc, adapt), adapt));
  }
  CUDA_TRY(cudaStreamSynchronize(eng->stream));
  return GPUMC_OK;
}

int gpumc_sim::launch_msc_measurement() {
  for (int r = 0; r < n_rep; ++r)
    RC_TRY(launch_msc_measure(eng->stream, lay, eng->d_lats, lat0 + r, d_msc_counters + (size_t)r * 128));
  return launch_msc_record(eng->stream, eng->d_lats, eng->d_groups, group, d_msc_counters);
}

int gpumc_sim::launch_one_sweep() {
  RC_TRY(launch_sweep_kernel(eng->stream, kernel_kind(lay), d_tiles, n_tiles,
                             eng->d_lats, eng->d_groups, d_ctl, lay.smem));
  return GPUMC_OK;
}

int gpumc_sim::run_graph(uint32_t n) {
  const uint32_t key = n;
  auto it = graphs.find(key);
  if (it == graphs.end()) {
    cudaGraph_t g;
    CUDA_TRY(cudaStreamBeginCapture(eng->stream, cudaStreamCaptureModeThreadLocal));
    int rc = GPUMC_OK;
    for (uint32_t i = 0; i < n && rc == GPUMC_OK; ++i) {
      rc = launch_one_sweep();
      if (rc == GPUMC_OK && lay.model == MSC && phase == GPUMC_PHASE_MEASUREMENT)
        rc = launch_msc_measurement();
    }
    cudaError_t e = cudaStreamEndCapture(eng->stream, &g);
    if (rc) return rc;
    if (e != cudaSuccess) return fail(GPUMC_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    cudaGraphExec_t ex;
    e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(GPUMC_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    it = graphs.emplace(key, ex).first;
  }
  CUDA_TRY(cudaGraphLaunch(it->second, eng->stream));
  return GPUMC_OK;
}

int gpumc_sim::drain_records() {
  CUDA_TRY(cudaStreamSynchronize(eng->stream));
  GroupDesc g;
  CUDA_TRY(cudaMemcpy(&g, eng->d_groups + group, sizeof(GroupDesc), cudaMemcpyDeviceToHost));
  if (g.overflow) return fail(GPUMC_ESTATE, "record buffer overflow (internal scheduling error)");
  const int cnt = g.rec_count;
  if (cnt > 0) {
    std::vector<Record> recs((size_t)cnt * rec_stride);
    CUDA_TRY(cudaMemcpy(recs.data(), d_records, recs.size() * sizeof(Record), cudaMemcpyDeviceToHost));
    const double n = (double)lay.n_sites;
    for (int i = 0; i < cnt; ++i) {
      for (int r = 0; r < rec_stride; ++r) {
        const Record& R = recs[(size_t)i * rec_stride + r];
        gpumc_obs o;
        o.sweep = R.sweep;
        o.replica = r;
        o.temp_index = R.label;
        o.beta = betas[std::min(std::max(R.label, 0), n_temps - 1)];
        o.energy = R.energy;
        if (lay.model == POTTS)
          o.magnetization = ((double)spec.q * R.m[0] - n) / (n * (double)(spec.q - 1));
        else if (lay.model == O3)
          o.magnetization = std::sqrt(R.m[0] * R.m[0] + R.m[1] * R.m[1] + R.m[2] * R.m[2]) / n;
        else
          o.magnetization = std::fabs(R.m[0]) / n;
        o.acceptance = R.accepted / n;
        pending.push_back(o);
      }
    }
    const int32_t zero = 0;
    RC_TRY(set_group_field(offsetof(GroupDesc, rec_count), zero));
    CUDA_TRY(cudaStreamSynchronize(eng->stream));
  }
  rec_used = 0;
  return GPUMC_OK;
}

// Moves the completed bins of the device ring to pending_bins; the open bin
// stays on the device.
int gpumc_sim::drain_bins() {
  CUDA_TRY(cudaStreamSynchronize(eng->stream));
  GroupDesc g;
  CUDA_TRY(cudaMemcpy(&g, eng->d_groups + group, sizeof(GroupDesc), cudaMemcpyDeviceToHost));
  if (g.bin_overflow) return fail(GPUMC_ESTATE, "bin buffer overflow (internal scheduling error)");
  if (g.bin_count > 0) {
    const size_t n = (size_t)g.bin_count * n_rep * kBinObs;
    const size_t at = pending_bins.size();
    pending_bins.resize(at + n);
    CUDA_TRY(cudaMemcpy(pending_bins.data() + at, d_bins, n * sizeof(double), cudaMemcpyDeviceToHost));
    const int32_t zero = 0;
    RC_TRY(set_group_field(offsetof(GroupDesc, bin_count), zero));
    CUDA_TRY(cudaStreamSynchronize(eng->stream));
  }
  bin_total = (uint64_t)g.bin_fill;
  return GPUMC_OK;
}

// Clamps `room` to the measured sweeps the device can take before its record
// ring (or bin ring) is full, draining it first when it already is.
int gpumc_sim::measure_room(uint32_t& room) {
  if (phase != GPUMC_PHASE_MEASUREMENT || device_schedule) return GPUMC_OK;
  if (binsize > 0) {
    const uint64_t cap = (uint64_t)bin_cap * (uint64_t)binsize;
    if (bin_total >= cap) RC_TRY(drain_bins());
    room = (uint32_t)std::min<uint64_t>(room, cap - bin_total);
  } else {
    if (rec_used >= rec_cap) RC_TRY(drain_records());
    room = std::min<uint32_t>(room, (uint32_t)(rec_cap - rec_used));
  }
  return GPUMC_OK;
}

void gpumc_sim::note_measured(uint32_t chunk) {
  if (phase != GPUMC_PHASE_MEASUREMENT || device_schedule) return;
  if (binsize > 0)
    bin_total += chunk;
  else
    rec_used += (int)chunk;
}

// Launches the exact energy reduction of one buffer into d_e (int64 units of
// J for the integer models, f64 for O(3)); for int8 models also counts
// chunks with invalid spin values into d_bad (if given).
int gpumc_sim::launch_energy(const void* buf, unsigned long long* d_e, unsigned int* d_bad) {
  const Layout& L = lay;
  const int rows = L.ly * L.lz;
  if (L.model == O3) {
    const int blocks = (int)std::min<int64_t>(kInitBlocks, (L.n_sites + 255) / 256);
    k_energy_o3<<<blocks, 256, 0, eng->stream>>>((const float*)buf, L.lx, L.ly, L.lz, L.pitch, spec.J,
                                                  (double*)d_e);
  } else if (L.model == MSC) {
    const int blocks = std::min(kInitBlocks, rows);
    k_energy_msc<<<blocks, 256, 0, eng->stream>>>((const unsigned long long*)buf, L.lx, L.ly, L.lz,
                                                   L.pitch, d_e);
  } else {
    const int nch = (L.lx + 15) / 16;
    const int rpi = nch <= 256 ? 256 / nch : 1;
    const int blocks = std::min(kInitBlocks, (rows + rpi - 1) / rpi);
    k_energy_i8<<<blocks, 256, 0, eng->stream>>>((const int8_t*)buf, L.model, (int)spec.q, L.lx, L.ly,
                                                  L.lz, L.pitch, d_e, d_bad);
  }
  CUDA_TRY(cudaGetLastError());
  return GPUMC_OK;
}

int gpumc_sim::recompute(std::vector<double>& out, bool store) {
  out.assign(n_rep, 0.0);
  unsigned long long* d_acc = nullptr;
  CUDA_TRY(cudaMallocAsync(&d_acc, 8 * (size_t)n_rep, eng->stream));
  int rc = GPUMC_OK;
  cudaError_t e = cudaMemsetAsync(d_acc, 0, 8 * (size_t)n_rep, eng->stream);
  for (int r = 0; r < n_rep && e == cudaSuccess && rc == GPUMC_OK; ++r)
    rc = launch_energy(bufs[2 * r + (sweeps & 1)], d_acc + r, nullptr);
  std::vector<unsigned long long> h(n_rep);
  if (e == cudaSuccess && rc == GPUMC_OK)
    e = cudaMemcpyAsync(h.data(), d_acc, 8 * (size_t)n_rep, cudaMemcpyDeviceToHost, eng->stream);
  dev_free(d_acc, eng->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(eng->stream);
  if (rc != GPUMC_OK) return rc;
  if (e != cudaSuccess) return fail(GPUMC_ECUDA, std::string("energy recompute: ") + cudaGetErrorString(e));
  for (int r = 0; r < n_rep; ++r) {
    if (lay.model == O3) {
      double v;
      std::memcpy(&v, &h[r], 8);
      out[r] = v;
      if (store) RC_TRY(set_lat_field(r, offsetof(LatDesc, e_f), v));
    } else {
      const long long ei = (long long)h[r];
      out[r] = spec.J * (double)ei;
      if (store) RC_TRY(set_lat_field(r, offsetof(LatDesc, e_int), ei));
    }
  }
  if (store) CUDA_TRY(cudaStreamSynchronize(eng->stream));
  return GPUMC_OK;
}

// Cache audit (audit_lattice_cache, CMC.rs/src/audit.rs:41-52): the cached
// energy of every replica against an exact recomputation from the spins,
// with the reference's tolerance 1e-10 (1 + |exact|).
int gpumc_sim::audit() {
  std::vector<LatDesc> d(n_rep);
  CUDA_TRY(cudaStreamSynchronize(eng->stream));
  CUDA_TRY(cudaMemcpy(d.data(), eng->d_lats + lat0, sizeof(LatDesc) * n_rep, cudaMemcpyDeviceToHost));
  std::vector<double> exact;
  RC_TRY(recompute(exact, false));
  for (int r = 0; r < n_rep; ++r) {
    const double cached = lay.model == O3 ? d[r].e_f : spec.J * (double)d[r].e_int;
    // O(3) sweeps record the energy as a fixed-point sum of fp32 bond
    // products (each within 4e-6 of exact on a colour-1 site: the fp32
    // neighbour sum, the fused dot and the 2^-19 rounding), so the audit
    // allows that rounding on top of the reference's tolerance
    const double fp32_bound = lay.model == O3 && !lay.cluster ? 2e-6 * std::fabs(spec.J) * (double)lay.n_sites : 0.0;
    if (std::fabs(cached - exact[r]) > 1e-10 * (1.0 + std::fabs(exact[r])) + fp32_bound) {
      char msg[256];
      std::snprintf(msg, sizeof(msg),
                    "lattice energy cache mismatch: replica %d after sweep %llu: cached=%.17g, exact=%.17g", r,
                    (unsigned long long)sweeps, cached, exact[r]);
      return fail(GPUMC_ESTATE, msg);
    }
  }
  return GPUMC_OK;
}

// Sweeps a chunk may run before the next audit point (0 = no audit due).
uint32_t gpumc_sim::sweeps_to_audit() const {
  if (!audit_interval) return 0;
  return (uint32_t)std::min<uint64_t>(audit_interval - sweeps % audit_interval, 1u << 30);
}

// ===========================================================================
// C ABI
// ===========================================================================
int gpumc_validate(const gpumc_spec* spec) { return validate_spec(spec); }

int gpumc_footprint(const gpumc_spec* spec, size_t* bytes) {
  RC_TRY(validate_spec(spec));
  if (!bytes) return fail(GPUMC_EINVAL, "bytes: null");
  *bytes = footprint_bytes(spec);
  return GPUMC_OK;
}

int gpumc_plan_tiles(const gpumc_spec* spec, int32_t slots, int32_t slots3, int32_t refine,
                     int64_t* n_tiles, int32_t* kind) {
  RC_TRY(validate_spec(spec));
  if (!n_tiles || !kind) return fail(GPUMC_EINVAL, "null argument");
  if (slots < 1 || slots3 < 1) return fail(GPUMC_EINVAL, "slots: must be >= 1");
  std::vector<Layout> one{plan_layout(spec, slots, slots3)};
  const int n_rep = std::max<int>(1, (int)spec->n_replicas);
  if (refine) refine_layouts(one, {n_rep}, family_slots(one[0], slots, slots3));
  *n_tiles = count_tiles(one[0]) * n_rep;
  *kind = kernel_kind(one[0]);
  return GPUMC_OK;
}

int gpumc_create(gpumc_engine* eng, const gpumc_spec* spec, uint64_t base_seed, gpumc_sim** out) {
  RC_TRY(validate_spec(spec));
  if (!out) return fail(GPUMC_EINVAL, "out: null pointer");
  bool priv = false;
  if (!eng) {
    RC_TRY(gpumc_engine_create(0, &eng));
    priv = true;
  }
  CUDA_TRY(cudaSetDevice(eng->device));
  gpumc_sim* s = new gpumc_sim();
  s->eng = eng;
  s->private_engine = priv;
  s->spec = *spec;
  s->betas.assign(spec->betas, spec->betas + spec->n_temps);
  s->spec.betas = nullptr;
  s->base = plan_layout(spec, eng->slots, eng->slots3);
  {
    // the simulation's own launches: tiles split until they fill the device
    std::vector<Layout> one{s->base};
    refine_layouts(one, {std::max<int>(1, (int)spec->n_replicas)},
                   family_slots(s->base, eng->slots, eng->slots3));
    s->lay = one[0];
  }
  s->blay = s->lay;
  s->n_rep = spec->n_replicas;
  s->n_temps = spec->n_temps;
  s->n_cls = n_classes(s->lay.model == MSC ? ISING : s->lay.model, s->lay.dims);
  s->base_seed = base_seed;
  s->rec_cap = spec->record_capacity;
  s->rec_stride = s->lay.model == MSC ? 64 * s->n_rep : s->n_rep;
  auto cleanup = [&](int rc) {
    if (s->lat0 >= 0)
      for (int r = 0; r < s->n_rep; ++r) eng->lat_used[s->lat0 + r] = false;
    if (s->group >= 0) eng->group_used[s->group] = false;
    delete s;
    if (priv) gpumc_engine_destroy(eng);
    return rc;
  };
  int rc = eng->alloc_slots(s->n_rep, s->lat0);
  if (rc) return cleanup(rc);
  rc = eng->alloc_group(s->group);
  if (rc) return cleanup(rc);
#define CUDA_CLEAN(expr)                                                              \
  do {                                                                                \
    cudaError_t e_ = (expr);                                                          \
    if (e_ != cudaSuccess)                                                            \
      return cleanup(fail(e_ == cudaErrorMemoryAllocation ? GPUMC_ENOMEM : GPUMC_ECUDA, \
                          std::string(#expr) + ": " + cudaGetErrorString(e_)));        \
  } while (0)
  // device buffers
  s->bufs.assign(2 * s->n_rep, nullptr);
  for (int i = 0; i < 2 * s->n_rep; ++i) {
    if (s->lay.inplace && (i & 1)) {  // in-place models: both slots name one buffer
      s->bufs[i] = s->bufs[i - 1];
      continue;
    }
    CUDA_CLEAN(cudaMallocAsync(&s->bufs[i], s->lay.buf_bytes, eng->stream));
    CUDA_CLEAN(cudaMemsetAsync(s->bufs[i], 0, s->lay.buf_bytes, eng->stream));
  }
  if (s->lay.cluster) {  // union-find labels of the cluster updates, one array per replica
    s->aux.assign(s->n_rep, nullptr);
    for (int r = 0; r < s->n_rep; ++r) CUDA_CLEAN(cudaMallocAsync(&s->aux[r], 4 * (size_t)s->lay.n_sites, eng->stream));
  }
  CUDA_CLEAN(cudaMallocAsync(&s->d_head, 4 * (size_t)s->n_temps * s->n_cls, eng->stream));
  CUDA_CLEAN(cudaMallocAsync(&s->d_tail, 8 * (size_t)s->n_temps * s->n_cls, eng->stream));
  CUDA_CLEAN(cudaMallocAsync(&s->d_betas, 8 * (size_t)s->n_temps, eng->stream));
  CUDA_CLEAN(cudaMallocAsync(&s->d_betas_f, 4 * (size_t)s->n_temps, eng->stream));
  CUDA_CLEAN(cudaMallocAsync(&s->d_label, 4 * (size_t)s->n_rep, eng->stream));
  CUDA_CLEAN(cudaMallocAsync(&s->d_rep_at, 4 * (size_t)s->n_rep, eng->stream));
  CUDA_CLEAN(cudaMallocAsync(&s->d_records, sizeof(Record) * (size_t)s->rec_cap * s->rec_stride, eng->stream));
  if (s->lay.model == MSC) {
    CUDA_CLEAN(cudaMallocAsync(&s->d_msc_counters, 8 * 128 * (size_t)s->n_rep, eng->stream));
    CUDA_CLEAN(cudaMemsetAsync(s->d_msc_counters, 0, 8 * 128 * (size_t)s->n_rep, eng->stream));
  }
  rc = s->upload_tables();
  if (rc) return cleanup(rc);
  std::vector<int32_t> labels(s->n_rep);
  for (int r = 0; r < s->n_rep; ++r) labels[r] = s->n_temps == 1 ? 0 : r;
  CUDA_CLEAN(cudaMemcpyAsync(s->d_label, labels.data(), 4 * (size_t)s->n_rep, cudaMemcpyHostToDevice, eng->stream));
  // tiles and launch control of the plain path
  std::vector<TileItem> tiles;
  rc = s->upload_own_tiles(tiles);
  if (rc) return cleanup(rc);
  // the group id, its tile count and its done counter (tiles are the group's
  // only: TileItem::pad = 0)
  const int32_t gbuf[3] = {s->group, s->n_tiles, 0};
  CUDA_CLEAN(cudaMallocAsync(&s->d_gid, sizeof(gbuf), eng->stream));
  CUDA_CLEAN(cudaMemcpyAsync(s->d_gid, gbuf, sizeof(gbuf), cudaMemcpyHostToDevice, eng->stream));
  CUDA_CLEAN(cudaMallocAsync(&s->d_ctl, sizeof(LaunchCtl), eng->stream));
  LaunchCtl c;
  c.done = 0;
  c.n_groups = 1;
  c.group_ids = s->d_gid;
  c.group_tiles = s->d_gid + 1;
  c.group_done = (unsigned int*)(s->d_gid + 2);
  c.n_tiles = s->n_tiles;
  CUDA_CLEAN(cudaMemcpyAsync(s->d_ctl, &c, sizeof(c), cudaMemcpyHostToDevice, eng->stream));
  if (is_ising_bits_kind(kernel_kind(s->lay))) {
    std::map<int, const Layout*> lay_of;
    for (int r = 0; r < s->n_rep; ++r) lay_of[s->lat0 + r] = &s->lay;
    rc = build_resident(eng->device, eng->stream, tiles, lay_of, s->lay.smem, s->res);
    if (rc) return cleanup(rc);
  }
  // descriptors
  const float omc = (float)(2.0 * std::sin(0.5 * spec->cone_half_angle) * std::sin(0.5 * spec->cone_half_angle));
  for (int r = 0; r < s->n_rep; ++r) {
    LatDesc d;
    std::memset(&d, 0, sizeof(d));
    d.model = s->lay.model;
    d.dims = s->lay.dims;
    d.lx = s->lay.lx;
    d.ly = s->lay.ly;
    d.lz = s->lay.lz;
    d.pitch = s->lay.pitch;
    d.q = spec->q;
    d.z = 2 * s->lay.dims;
    d.tile_cx = s->lay.tile_cx;
    d.tile_y = s->lay.tile_y;
    d.tile_z = s->lay.tile_z;
    d.group = s->group;
    d.replica = r;
    d.n_sites = s->lay.n_sites;
    d.buf[0] = s->bufs[2 * r];
    d.buf[1] = s->bufs[2 * r + 1];
    d.aux = s->lay.cluster ? s->aux[r] : nullptr;
    const uint64_t rid = s->lay.model == MSC ? 64ull * r : (uint64_t)r;
    d.key = stream_key(base_seed, rid, 0, 1);
    d.sweep = 0;
    d.target = ~0ull;
    d.prop = s->lay.prop;
    // OPSS keeps its bound sigma where the cap keeps 1 - cos(alpha)
    d.omc = s->lay.prop == GPUMC_O3_OPSS ? (float)spec->cone_half_angle : omc;
    // the cap and OPSS adapt while thermalizing; the uniform proposal and the
    // heat bath have nothing to adapt
    d.adapt = (s->lay.alg == METROPOLIS && s->lay.prop != GPUMC_O3_UNIFORM) ? 1 : 0;
    CUDA_CLEAN(cudaMemcpyAsync(eng->d_lats + s->lat0 + r, &d, sizeof(d), cudaMemcpyHostToDevice, eng->stream));
  }
  GroupDesc g;
  std::memset(&g, 0, sizeof(g));
  g.first_lat = s->lat0;
  g.n_rep = s->n_rep;
  g.n_cls = s->n_cls;
  g.pt_interval = 0;
  g.measure = 0;
  g.rec_cap = s->rec_cap;
  g.label = s->d_label;
  g.rep_at = s->d_rep_at;
  g.head = s->d_head;
  g.tail = s->d_tail;
  g.betas = s->d_betas;
  g.betas_f = s->d_betas_f;
  g.J = spec->J;
  g.Jf = (float)spec->J;
  g.measure_from = 0;
  g.adapt_until = ~0ull;
  g.pt_key = stream_key(base_seed, 0, 3, 0);
  g.records = s->d_records;
  CUDA_CLEAN(cudaMemcpyAsync(eng->d_groups + s->group, &g, sizeof(g), cudaMemcpyHostToDevice, eng->stream));
  // initial state
  const int blocks = (int)std::min<int64_t>(kInitBlocks, (s->lay.n_sites + 255) / 256);
  const int hot = spec->init == GPUMC_INIT_HOT;
  uint64_t* d_keys = nullptr;
  if (s->lay.model == MSC) CUDA_CLEAN(cudaMallocAsync(&d_keys, 8 * 64, eng->stream));
  for (int r = 0; r < s->n_rep; ++r) {
    const uint64_t kinit = stream_key(base_seed, (uint64_t)r, 0, 0);
    if (s->lay.model == ISING || s->lay.model == POTTS) {
      k_init_discrete<<<blocks, 256, 0, eng->stream>>>((int8_t*)s->bufs[2 * r], s->lay.model, s->lay.lx,
                                                        s->lay.ly, s->lay.lz, s->lay.pitch, spec->q,
                                                        kinit, hot);
    } else if (s->lay.model == O3) {
      k_init_o3<<<blocks, 256, 0, eng->stream>>>((float*)s->bufs[2 * r], s->lay.lx, s->lay.ly, s->lay.lz,
                                                  s->lay.pitch, kinit, hot);
    } else {
      uint64_t keys[64];
      for (int b = 0; b < 64; ++b) keys[b] = stream_key(base_seed, 64ull * r + b, 0, 0);
      CUDA_CLEAN(cudaMemcpyAsync(d_keys, keys, sizeof(keys), cudaMemcpyHostToDevice, eng->stream));
      k_init_msc<<<blocks, 256, 0, eng->stream>>>((unsigned long long*)s->bufs[2 * r], s->lay.lx,
                                                   s->lay.ly, s->lay.lz, s->lay.pitch, d_keys, hot);
      CUDA_CLEAN(cudaStreamSynchronize(eng->stream));
    }
  }
  CUDA_CLEAN(cudaGetLastError());
  CUDA_CLEAN(cudaStreamSynchronize(eng->stream));
  if (d_keys) dev_free(d_keys, eng->stream);
  std::vector<double> e0;
  rc = s->recompute(e0, true);
  if (rc) return cleanup(rc);
  rc = s->push_phase_flags();
  if (rc) return cleanup(rc);
#undef CUDA_CLEAN
  eng->sims.insert(s);
  eng->batch_dirty = true;
  *out = s;
  return GPUMC_OK;
}

int gpumc_destroy(gpumc_sim* sim) {
  if (!sim) return GPUMC_OK;
  gpumc_engine* eng = sim->eng;
  const bool priv = sim->private_engine;
  eng->sims.erase(sim);
  eng->batch_dirty = true;
  for (int r = 0; r < sim->n_rep; ++r) eng->lat_used[sim->lat0 + r] = false;
  eng->group_used[sim->group] = false;
  delete sim;
  if (priv) gpumc_engine_destroy(eng);
  return GPUMC_OK;
}

int gpumc_set_phase(gpumc_sim* sim, int32_t phase) {
  if (!sim) return fail(GPUMC_EINVAL, "sim: null");
  if (phase != GPUMC_PHASE_THERMALIZATION && phase != GPUMC_PHASE_MEASUREMENT)
    return fail(GPUMC_EINVAL, "phase: expected THERMALIZATION or MEASUREMENT");
  CUDA_TRY(cudaSetDevice(sim->eng->device));
  if (phase == sim->phase) return GPUMC_OK;
  sim->phase = phase;
  sim->drop_graphs();
  sim->eng->drop_graphs();
  return sim->push_phase_flags();
}

int gpumc_set_tile_refinement(gpumc_sim* sim, int32_t enable) {
  if (!sim) return fail(GPUMC_EINVAL, "sim: null");
  CUDA_TRY(cudaSetDevice(sim->eng->device));
  std::vector<Layout> one{sim->base};
  if (enable) refine_layouts(one, {sim->n_rep}, family_slots(sim->base, sim->eng->slots, sim->eng->slots3));
  const Layout& want = one[0];
  if (want.tile_cx == sim->lay.tile_cx && want.tile_y == sim->lay.tile_y && want.tile_z == sim->lay.tile_z &&
      want.march == sim->lay.march)
    return GPUMC_OK;
  const Layout old = sim->lay;
  sim->lay = want;
  std::vector<TileItem> tiles;
  const int rc = sim->upload_own_tiles(tiles);
  if (rc) {
    sim->lay = old;
    return rc;
  }
  sim->drop_graphs();
  // the resident plan follows the new tiles (whole-row or whole-plane Ising
  // tiles may qualify now, or no longer)
  sim->res.release(sim->eng->stream);
  if (is_ising_bits_kind(kernel_kind(sim->lay))) {
    std::map<int, const Layout*> lay_of;
    for (int r = 0; r < sim->n_rep; ++r) lay_of[sim->lat0 + r] = &sim->lay;
    RC_TRY(build_resident(sim->eng->device, sim->eng->stream, tiles, lay_of, sim->lay.smem, sim->res));
  }
  CUDA_TRY(cudaStreamSynchronize(sim->eng->stream));
  return GPUMC_OK;
}

int gpumc_tile_count(gpumc_sim* sim, int32_t* n_tiles) {
  if (!sim || !n_tiles) return fail(GPUMC_EINVAL, "null argument");
  *n_tiles = sim->n_tiles;
  return GPUMC_OK;
}

int gpumc_sweep(gpumc_sim* sim, uint32_t n_sweeps) {
  if (!sim) return fail(GPUMC_EINVAL, "sim: null");
  CUDA_TRY(cudaSetDevice(sim->eng->device));
  uint32_t left = n_sweeps;
  while (left > 0) {
    uint32_t room = left;
    RC_TRY(sim->measure_room(room));
    uint32_t chunk = std::min<uint32_t>(room, 64);
    if (const uint32_t to_audit = sim->sweeps_to_audit()) chunk = std::min(chunk, to_audit);
    if (sim->res.on && sim->blocking) {
      RC_TRY(launch_resident(sim->eng->stream, sim->d_tiles, sim->n_tiles, sim->eng->d_lats, sim->eng->d_groups,
                             sim->d_ctl, sim->res, sim->lay.smem, (int)chunk, sim->eng->wait_limit));
      sim->launches += 1;
    } else {
      RC_TRY(sim->run_graph(chunk));
      int32_t lps = 0;
      gpumc_launches_per_sweep(sim, &lps);
      sim->launches += (uint64_t)chunk * (uint64_t)lps;
    }
    sim->sweeps += chunk;
    sim->note_measured(chunk);
    left -= chunk;
    if (sim->audit_interval && sim->sweeps % sim->audit_interval == 0) RC_TRY(sim->audit());
  }
  if (is_o3_march_kind(kernel_kind(sim->lay))) RC_TRY(check_launch_flag(sim->eng->stream, sim->d_ctl));
  return GPUMC_OK;
}

int gpumc_set_audit_interval(gpumc_sim* sim, uint64_t interval) {
  if (!sim) return fail(GPUMC_EINVAL, "sim: null");
  if (interval && sim->device_schedule) return fail(GPUMC_ESTATE, "audit: not available for server jobs");
  sim->audit_interval = interval;
  return GPUMC_OK;
}

int gpumc_perturb_energy_cache(gpumc_sim* sim, int32_t replica, double delta) {
  if (!sim) return fail(GPUMC_EINVAL, "sim: null");
  if (replica < 0 || replica >= sim->n_rep) return fail(GPUMC_EINVAL, "replica: out of range");
  if (!std::isfinite(delta)) return fail(GPUMC_EINVAL, "delta: must be finite");
  CUDA_TRY(cudaSetDevice(sim->eng->device));
  CUDA_TRY(cudaStreamSynchronize(sim->eng->stream));
  LatDesc d;
  CUDA_TRY(cudaMemcpy(&d, sim->eng->d_lats + sim->lat0 + replica, sizeof(d), cudaMemcpyDeviceToHost));
  if (sim->lay.model == O3) {
    RC_TRY(sim->set_lat_field(replica, offsetof(LatDesc, e_f), d.e_f + delta));
  } else {
    if (delta != std::floor(delta)) return fail(GPUMC_EINVAL, "delta: integer models take a whole number of J");
    RC_TRY(sim->set_lat_field(replica, offsetof(LatDesc, e_int), d.e_int + (long long)delta));
  }
  CUDA_TRY(cudaStreamSynchronize(sim->eng->stream));
  return GPUMC_OK;
}

int gpumc_set_binning(gpumc_sim* sim, int32_t binsize, int32_t bin_capacity) {
  if (!sim) return fail(GPUMC_EINVAL, "sim: null");
  if (binsize < 0) return fail(GPUMC_EINVAL, "binsize: must be >= 0 (0 = per-sweep records)");
  if (binsize > 0 && bin_capacity < 1) return fail(GPUMC_EINVAL, "bin_capacity: must be >= 1");
  if (binsize > 0 && sim->lay.model == MSC)
    return fail(GPUMC_EINVAL, "binsize: the multi-spin model reports per-replica records only");
  if (sim->device_schedule) return fail(GPUMC_ESTATE, "binning: not available for server jobs");
  CUDA_TRY(cudaSetDevice(sim->eng->device));
  RC_TRY(sim->drain_records());  // records measured so far stay available
  CUDA_TRY(cudaStreamSynchronize(sim->eng->stream));
  dev_free(sim->d_bin_open, sim->eng->stream);
  dev_free(sim->d_bins, sim->eng->stream);
  sim->d_bin_open = sim->d_bins = nullptr;
  sim->pending_bins.clear();
  sim->bin_total = 0;
  sim->binsize = 0;
  sim->bin_cap = 0;
  const size_t per = (size_t)sim->n_rep * kBinObs;
  if (binsize > 0) {
    CUDA_TRY(cudaMallocAsync(&sim->d_bin_open, per * sizeof(double), sim->eng->stream));
    CUDA_TRY(cudaMemsetAsync(sim->d_bin_open, 0, per * sizeof(double), sim->eng->stream));
    if (cudaMallocAsync(&sim->d_bins, per * (size_t)bin_capacity * sizeof(double), sim->eng->stream) !=
        cudaSuccess) {
      cudaGetLastError();
      dev_free(sim->d_bin_open, sim->eng->stream);
      sim->d_bin_open = nullptr;
      return fail(GPUMC_ENOMEM, "bin_capacity: device memory exhausted");
    }
    sim->binsize = binsize;
    sim->bin_cap = bin_capacity;
  }
  const int32_t zero = 0, by_label = (sim->n_temps == sim->n_rep && sim->n_rep > 1) ? 1 : 0;
  RC_TRY(sim->set_group_field(offsetof(GroupDesc, binsize), (int32_t)sim->binsize));
  RC_TRY(sim->set_group_field(offsetof(GroupDesc, bin_cap), (int32_t)sim->bin_cap));
  RC_TRY(sim->set_group_field(offsetof(GroupDesc, bin_count), zero));
  RC_TRY(sim->set_group_field(offsetof(GroupDesc, bin_fill), zero));
  RC_TRY(sim->set_group_field(offsetof(GroupDesc, bin_by_label), by_label));
  RC_TRY(sim->set_group_field(offsetof(GroupDesc, bin_overflow), zero));
  RC_TRY(sim->set_group_field(offsetof(GroupDesc, bin_open), sim->d_bin_open));
  RC_TRY(sim->set_group_field(offsetof(GroupDesc, bins), sim->d_bins));
  CUDA_TRY(cudaStreamSynchronize(sim->eng->stream));
  return GPUMC_OK;
}

int gpumc_drain_bins(gpumc_sim* sim, double* out, size_t cap_bins, size_t* n_bins) {
  if (!sim || !n_bins) return fail(GPUMC_EINVAL, "sim/n_bins: null");
  if (sim->binsize <= 0) return fail(GPUMC_ESTATE, "binning: not enabled (gpumc_set_binning)");
  CUDA_TRY(cudaSetDevice(sim->eng->device));
  RC_TRY(sim->drain_bins());
  const size_t per = (size_t)sim->n_rep * kBinObs;
  const size_t k = std::min(cap_bins, sim->pending_bins.size() / per);
  if (k && !out) return fail(GPUMC_EINVAL, "out: null");
  std::copy(sim->pending_bins.begin(), sim->pending_bins.begin() + k * per, out);
  sim->pending_bins.erase(sim->pending_bins.begin(), sim->pending_bins.begin() + k * per);
  *n_bins = k;
  return GPUMC_OK;
}

int gpumc_open_bin(gpumc_sim* sim, double* sums, int32_t* fill) {
  if (!sim || !sums || !fill) return fail(GPUMC_EINVAL, "sim/sums/fill: null");
  if (sim->binsize <= 0) return fail(GPUMC_ESTATE, "binning: not enabled (gpumc_set_binning)");
  CUDA_TRY(cudaSetDevice(sim->eng->device));
  CUDA_TRY(cudaStreamSynchronize(sim->eng->stream));
  GroupDesc g;
  CUDA_TRY(cudaMemcpy(&g, sim->eng->d_groups + sim->group, sizeof(GroupDesc), cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemcpy(sums, sim->d_bin_open, (size_t)sim->n_rep * kBinObs * sizeof(double),
                      cudaMemcpyDeviceToHost));
  *fill = g.bin_fill;
  return GPUMC_OK;
}

int gpumc_observables(gpumc_sim* sim, gpumc_obs* out, size_t cap, size_t* n) {
  if (!sim || !n) return fail(GPUMC_EINVAL, "sim/n: null");
  CUDA_TRY(cudaSetDevice(sim->eng->device));
  RC_TRY(sim->drain_records());
  const size_t k = std::min(cap, sim->pending.size());
  if (k && !out) return fail(GPUMC_EINVAL, "out: null");
  std::copy(sim->pending.begin(), sim->pending.begin() + k, out);
  sim->pending.erase(sim->pending.begin(), sim->pending.begin() + k);
  *n = k;
  return GPUMC_OK;
}

static size_t host_site_bytes(int model) {
  return model == GPUMC_O3 ? 12 : model == GPUMC_ISING_MSC64 ? 8 : 1;
}

int gpumc_get_spins(gpumc_sim* sim, int32_t replica, void* host, size_t nbytes) {
  if (!sim || !host) return fail(GPUMC_EINVAL, "sim/host: null");
  if (replica < 0 || replica >= sim->n_rep) return fail(GPUMC_EINVAL, "replica: out of range");
  const Layout& L = sim->lay;
  const size_t need = host_site_bytes(L.model) * (size_t)L.n_sites;
  if (nbytes < need) return fail(GPUMC_EINVAL, "nbytes: buffer too small");
  CUDA_TRY(cudaSetDevice(sim->eng->device));
  CUDA_TRY(cudaStreamSynchronize(sim->eng->stream));
  const void* buf = sim->bufs[2 * replica + (sim->sweeps & 1)];
  const size_t rows = (size_t)L.ly * L.lz;
  if (L.model == ISING || L.model == POTTS) {
    CUDA_TRY(cudaMemcpy2D(host, L.lx, buf, L.pitch, L.lx, rows, cudaMemcpyDeviceToHost));
  } else if (L.model == MSC) {
    CUDA_TRY(cudaMemcpy2D(host, 8 * (size_t)L.lx, buf, 8 * (size_t)L.pitch, 8 * (size_t)L.lx, rows,
                          cudaMemcpyDeviceToHost));
  } else {
    std::vector<float> comp((size_t)L.n_sites * 3);
    for (int c = 0; c < 3; ++c)
      CUDA_TRY(cudaMemcpy2D(comp.data() + (size_t)c * L.n_sites, 4 * (size_t)L.lx,
                            (const float*)buf + (size_t)c * L.pitch * rows, 4 * (size_t)L.pitch,
                            4 * (size_t)L.lx, rows, cudaMemcpyDeviceToHost));
    float* h = (float*)host;
    for (int64_t i = 0; i < L.n_sites; ++i)
      for (int c = 0; c < 3; ++c) h[3 * i + c] = comp[(size_t)c * L.n_sites + i];
  }
  return GPUMC_OK;
}

int gpumc_set_spins(gpumc_sim* sim, int32_t replica, const void* host, size_t nbytes) {
  if (!sim || !host) return fail(GPUMC_EINVAL, "sim/host: null");
  if (replica < 0 || replica >= sim->n_rep) return fail(GPUMC_EINVAL, "replica: out of range");
  const Layout& L = sim->lay;
  const size_t need = host_site_bytes(L.model) * (size_t)L.n_sites;
  if (nbytes != need) return fail(GPUMC_EINVAL, "nbytes: does not match the lattice");
  CUDA_TRY(cudaSetDevice(sim->eng->device));
  CUDA_TRY(cudaStreamSynchronize(sim->eng->stream));
  const size_t rows = (size_t)L.ly * L.lz;
  void* cur = sim->bufs[2 * replica + (sim->sweeps & 1)];
  if (L.model == ISING || L.model == POTTS) {
    // The state lands in the replica's other ping-pong buffer (rewritten by
    // the next sweep anyway) and is validated on the device together with
    // the exact energy (validate_spin, CMC.rs/src/lattice/models.rs:62-75,
    // :238-252); only a valid state replaces the current one.
    void* stage = sim->bufs[2 * replica + ((sim->sweeps & 1) ^ 1)];
    unsigned long long* d_acc = nullptr;
    cudaStream_t st = sim->eng->stream;
    CUDA_TRY(cudaMallocAsync(&d_acc, 16, st));
    unsigned long long h[2] = {0, 0};
    cudaError_t e = cudaMemcpy2DAsync(stage, L.pitch, host, L.lx, L.lx, rows, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_acc, 0, 16, st);
    int rc = e == cudaSuccess ? sim->launch_energy(stage, d_acc, (unsigned int*)(d_acc + 1)) : GPUMC_OK;
    if (e == cudaSuccess && rc == GPUMC_OK) e = cudaMemcpyAsync(h, d_acc, 16, cudaMemcpyDeviceToHost, st);
    dev_free(d_acc, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (rc != GPUMC_OK) return rc;
    if (e != cudaSuccess) return fail(GPUMC_ECUDA, std::string("set_spins: ") + cudaGetErrorString(e));
    if ((unsigned int)h[1] != 0)
      return fail(GPUMC_EINVAL, L.model == ISING ? "spins: Ising spin must be exactly -1 or +1"
                                                 : "spins: Potts spin must be in [0, q)");
    CUDA_TRY(cudaMemcpyAsync(cur, stage, L.buf_bytes, cudaMemcpyDeviceToDevice, st));
    RC_TRY(sim->set_lat_field(replica, offsetof(LatDesc, e_int), (long long)h[0]));
    CUDA_TRY(cudaStreamSynchronize(st));
    return GPUMC_OK;
  }
  if (L.model == O3) {
    // validate_spin of ONModel (unit norm, CMC.rs/src/lattice/models.rs:454-475)
    const float* v = (const float*)host;
    for (int64_t i = 0; i < L.n_sites; ++i) {
      const double n2 = (double)v[3 * i] * v[3 * i] + (double)v[3 * i + 1] * v[3 * i + 1] +
                        (double)v[3 * i + 2] * v[3 * i + 2];
      if (!std::isfinite(n2) || std::fabs(n2 - 1.0) > 1e-5)
        return fail(GPUMC_EINVAL, "spins: O(3) spin must have unit norm (|n^2 - 1| <= 1e-5 in float32)");
    }
    std::vector<float> comp((size_t)L.n_sites * 3);
    for (int64_t i = 0; i < L.n_sites; ++i)
      for (int c = 0; c < 3; ++c) comp[(size_t)c * L.n_sites + i] = v[3 * i + c];
    for (int c = 0; c < 3; ++c)
      CUDA_TRY(cudaMemcpy2D((float*)cur + (size_t)c * L.pitch * rows, 4 * (size_t)L.pitch,
                            comp.data() + (size_t)c * L.n_sites, 4 * (size_t)L.lx, 4 * (size_t)L.lx, rows,
                            cudaMemcpyHostToDevice));
  } else {  // multi-spin: every 64-bit word is a valid state
    CUDA_TRY(cudaMemcpy2D(cur, 8 * (size_t)L.pitch, host, 8 * (size_t)L.lx, 8 * (size_t)L.lx, rows,
                          cudaMemcpyHostToDevice));
  }
  std::vector<double> e;
  return sim->recompute(e, true);
}

int gpumc_energy(gpumc_sim* sim, double* energies) {
  if (!sim || !energies) return fail(GPUMC_EINVAL, "sim/energies: null");
  CUDA_TRY(cudaSetDevice(sim->eng->device));
  CUDA_TRY(cudaStreamSynchronize(sim->eng->stream));
  std::vector<LatDesc> d(sim->n_rep);
  CUDA_TRY(cudaMemcpy(d.data(), sim->eng->d_lats + sim->lat0, sizeof(LatDesc) * sim->n_rep,
                      cudaMemcpyDeviceToHost));
  for (int r = 0; r < sim->n_rep; ++r)
    energies[r] = sim->lay.model == O3 ? d[r].e_f : sim->spec.J * (double)d[r].e_int;
  return GPUMC_OK;
}

int gpumc_recompute_energy(gpumc_sim* sim, double* energies) {
  if (!sim || !energies) return fail(GPUMC_EINVAL, "sim/energies: null");
  CUDA_TRY(cudaSetDevice(sim->eng->device));
  CUDA_TRY(cudaStreamSynchronize(sim->eng->stream));
  std::vector<double> e;
  RC_TRY(sim->recompute(e, false));
  std::copy(e.begin(), e.end(), energies);
  return GPUMC_OK;
}

int gpumc_msc_replica_observables(gpumc_sim* sim, int32_t word_lattice, double* energy64,
                                  double* mag64) {
  if (!sim || !energy64 || !mag64) return fail(GPUMC_EINVAL, "null argument");
  if (sim->lay.model != MSC) return fail(GPUMC_EINVAL, "model: not a multi-spin simulation");
  if (word_lattice < 0 || word_lattice >= sim->n_rep) return fail(GPUMC_EINVAL, "word_lattice: out of range");
  CUDA_TRY(cudaSetDevice(sim->eng->device));
  CUDA_TRY(cudaStreamSynchronize(sim->eng->stream));
  unsigned long long* d = nullptr;
  CUDA_TRY(cudaMallocAsync(&d, 8 * 128, sim->eng->stream));
  CUDA_TRY(cudaMemsetAsync(d, 0, 8 * 128, sim->eng->stream));
  int rc = launch_msc_measure(sim->eng->stream, sim->lay, sim->eng->d_lats, sim->lat0 + word_lattice, d);
  unsigned long long h[128];
  cudaError_t e = cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, sim->eng->stream);
  dev_free(d, sim->eng->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(sim->eng->stream);
  if (rc) return rc;
  if (e != cudaSuccess) return fail(GPUMC_ECUDA, cudaGetErrorString(e));
  const double n = (double)sim->lay.n_sites;
  const double bonds = (double)sim->lay.dims * n;
  for (int r = 0; r < 64; ++r) {
    energy64[r] = -sim->spec.J * (bonds - 2.0 * (double)h[64 + r]);
    mag64[r] = std::fabs(2.0 * (double)h[r] - n) / n;
  }
  return GPUMC_OK;
}

int gpumc_set_temporal_blocking(gpumc_sim* sim, int32_t enable) {
  if (!sim) return fail(GPUMC_EINVAL, "sim: null");
  sim->blocking = enable != 0;
  return GPUMC_OK;
}

int gpumc_launch_count(gpumc_sim* sim, uint64_t* n) {
  if (!sim || !n) return fail(GPUMC_EINVAL, "null argument");
  *n = sim->launches;
  return GPUMC_OK;
}

int gpumc_sweep_count(gpumc_sim* sim, uint64_t* out) {
  if (!sim || !out) return fail(GPUMC_EINVAL, "null argument");
  *out = sim->sweeps;
  return GPUMC_OK;
}

int gpumc_acceptance(gpumc_sim* sim, int32_t replica, double* cone_half_angle) {
  if (!sim || !cone_half_angle) return fail(GPUMC_EINVAL, "null argument");
  if (replica < 0 || replica >= sim->n_rep) return fail(GPUMC_EINVAL, "replica: out of range");
  CUDA_TRY(cudaSetDevice(sim->eng->device));
  CUDA_TRY(cudaStreamSynchronize(sim->eng->stream));
  LatDesc d;
  CUDA_TRY(cudaMemcpy(&d, sim->eng->d_lats + sim->lat0 + replica, sizeof(d), cudaMemcpyDeviceToHost));
  if (sim->lay.prop == GPUMC_O3_OPSS)
    *cone_half_angle = (double)d.omc;  // the rotation bound sigma itself
  else  // cap: omc = 1 - cos(alpha) = 2 sin^2(alpha / 2)
    *cone_half_angle = 2.0 * std::asin(std::sqrt(std::min(1.0, 0.5 * (double)d.omc)));
  return GPUMC_OK;
}

int gpumc_set_sweep_count(gpumc_sim* sim, uint64_t sweeps) {
  if (!sim) return fail(GPUMC_EINVAL, "sim: null");
  CUDA_TRY(cudaSetDevice(sim->eng->device));
  CUDA_TRY(cudaStreamSynchronize(sim->eng->stream));
  std::vector<LatDesc> d(sim->n_rep);
  CUDA_TRY(cudaMemcpy(d.data(), sim->eng->d_lats + sim->lat0, sizeof(LatDesc) * sim->n_rep,
                      cudaMemcpyDeviceToHost));
  for (int r = 0; r < sim->n_rep; ++r) {
    if (sweeps > d[r].target) return fail(GPUMC_EINVAL, "sweeps: beyond the handle's target");
    // the current state lives in buf[sweep & 1]: keep it current across the change
    if (((d[r].sweep ^ sweeps) & 1) && !sim->lay.inplace) {
      void* from = sim->bufs[2 * r + (d[r].sweep & 1)];
      void* to = sim->bufs[2 * r + (sweeps & 1)];
      CUDA_TRY(cudaMemcpy(to, from, sim->lay.buf_bytes, cudaMemcpyDeviceToDevice));
    }
    RC_TRY(sim->set_lat_field(r, offsetof(LatDesc, sweep), sweeps));
  }
  // exchange steps attempted up to this count (the device derives each
  // exchange's step from the sweep count; this keeps gpumc_pt_stats in line)
  const uint64_t steps = sim->pt_interval > 0 ? sweeps / sim->pt_interval : 0;
  RC_TRY(sim->set_group_field(offsetof(GroupDesc, pt_step), steps));
  CUDA_TRY(cudaStreamSynchronize(sim->eng->stream));
  sim->sweeps = sweeps;
  return GPUMC_OK;
}

int gpumc_get_cone_omc(gpumc_sim* sim, int32_t replica, float* omc) {
  if (!sim || !omc) return fail(GPUMC_EINVAL, "null argument");
  if (replica < 0 || replica >= sim->n_rep) return fail(GPUMC_EINVAL, "replica: out of range");
  CUDA_TRY(cudaSetDevice(sim->eng->device));
  CUDA_TRY(cudaStreamSynchronize(sim->eng->stream));
  CUDA_TRY(cudaMemcpy(omc, (char*)(sim->eng->d_lats + sim->lat0 + replica) + offsetof(LatDesc, omc),
                      sizeof(float), cudaMemcpyDeviceToHost));
  return GPUMC_OK;
}

int gpumc_set_cone_omc(gpumc_sim* sim, int32_t replica, float omc) {
  if (!sim) return fail(GPUMC_EINVAL, "sim: null");
  if (replica < 0 || replica >= sim->n_rep) return fail(GPUMC_EINVAL, "replica: out of range");
  if (sim->lay.prop == GPUMC_O3_OPSS ? !(omc >= 1e-4f && omc <= 0x1.921fb6p+1f) : !(omc > 0.0f && omc <= 2.0f))
    return fail(GPUMC_EINVAL, "omc: must be in (0, 2] (cap) or [1e-4, pi] (OPSS sigma)");
  CUDA_TRY(cudaSetDevice(sim->eng->device));
  RC_TRY(sim->set_lat_field(replica, offsetof(LatDesc, omc), omc));
  CUDA_TRY(cudaStreamSynchronize(sim->eng->stream));
  return GPUMC_OK;
}

int gpumc_log_weight_ratio(gpumc_sim* sim, int32_t replica, double new_beta, double* out) {
  if (!sim || !out) return fail(GPUMC_EINVAL, "null argument");
  if (replica < 0 || replica >= sim->n_rep) return fail(GPUMC_EINVAL, "replica: out of range");
  std::vector<double> e(sim->n_rep);
  RC_TRY(gpumc_energy(sim, e.data()));
  std::vector<int32_t> lab(sim->n_rep);
  CUDA_TRY(cudaMemcpy(lab.data(), sim->d_label, 4 * (size_t)sim->n_rep, cudaMemcpyDeviceToHost));
  // ClassicalMC::log_weight_ratio: (beta - beta') * E (classical_mc.rs:209-214)
  *out = (sim->betas[lab[replica]] - new_beta) * e[replica];
  return GPUMC_OK;
}

int gpumc_change_parameter(gpumc_sim* sim, int32_t replica, double new_beta) {
  if (!sim) return fail(GPUMC_EINVAL, "sim: null");
  if (replica < 0 || replica >= sim->n_rep) return fail(GPUMC_EINVAL, "replica: out of range");
  if (!std::isfinite(new_beta) || new_beta < 0.0)
    return fail(GPUMC_EINVAL, "beta: must be finite and non-negative");
  CUDA_TRY(cudaSetDevice(sim->eng->device));
  CUDA_TRY(cudaStreamSynchronize(sim->eng->stream));
  std::vector<int32_t> lab(sim->n_rep);
  CUDA_TRY(cudaMemcpy(lab.data(), sim->d_label, 4 * (size_t)sim->n_rep, cudaMemcpyDeviceToHost));
  sim->betas[lab[replica]] = new_beta;
  RC_TRY(sim->upload_tables());
  // ClassicalMC::change_parameter recomputes the energy exactly (classical_mc.rs:216-228)
  std::vector<double> e;
  return sim->recompute(e, true);
}

int gpumc_pt_configure(gpumc_sim* sim, uint32_t interval) {
  if (!sim) return fail(GPUMC_EINVAL, "sim: null");
  if (interval > 0 && sim->n_temps != sim->n_rep)
    return fail(GPUMC_EINVAL, "parallel tempering needs one ladder entry per replica (n_temps = n_replicas)");
  if (interval > 0 && sim->n_rep > 256) return fail(GPUMC_EINVAL, "parallel tempering: at most 256 replicas");
  CUDA_TRY(cudaSetDevice(sim->eng->device));
  sim->pt_interval = interval;
  RC_TRY(sim->set_group_field(offsetof(GroupDesc, pt_interval), (int32_t)interval));
  CUDA_TRY(cudaStreamSynchronize(sim->eng->stream));
  return GPUMC_OK;
}

int gpumc_pt_labels(gpumc_sim* sim, int32_t* labels) {
  if (!sim || !labels) return fail(GPUMC_EINVAL, "null argument");
  CUDA_TRY(cudaSetDevice(sim->eng->device));
  CUDA_TRY(cudaStreamSynchronize(sim->eng->stream));
  CUDA_TRY(cudaMemcpy(labels, sim->d_label, 4 * (size_t)sim->n_rep, cudaMemcpyDeviceToHost));
  return GPUMC_OK;
}

int gpumc_pt_set_labels(gpumc_sim* sim, const int32_t* labels) {
  if (!sim || !labels) return fail(GPUMC_EINVAL, "null argument");
  if (sim->n_temps != sim->n_rep)
    return fail(GPUMC_EINVAL, "labels: the handle needs one ladder entry per replica (n_temps = n_replicas)");
  std::vector<char> seen(sim->n_rep, 0);
  for (int r = 0; r < sim->n_rep; ++r) {
    if (labels[r] < 0 || labels[r] >= sim->n_rep || seen[labels[r]])
      return fail(GPUMC_EINVAL, "labels: must be a permutation of 0..n_replicas-1");
    seen[labels[r]] = 1;
  }
  CUDA_TRY(cudaSetDevice(sim->eng->device));
  CUDA_TRY(cudaStreamSynchronize(sim->eng->stream));
  CUDA_TRY(cudaMemcpy(sim->d_label, labels, 4 * (size_t)sim->n_rep, cudaMemcpyHostToDevice));
  return GPUMC_OK;
}

int gpumc_pt_stats(gpumc_sim* sim, uint64_t* exchange_steps, uint64_t* accepted_swaps) {
  if (!sim || !exchange_steps || !accepted_swaps) return fail(GPUMC_EINVAL, "null argument");
  CUDA_TRY(cudaSetDevice(sim->eng->device));
  CUDA_TRY(cudaStreamSynchronize(sim->eng->stream));
  GroupDesc g;
  CUDA_TRY(cudaMemcpy(&g, sim->eng->d_groups + sim->group, sizeof(g), cudaMemcpyDeviceToHost));
  *exchange_steps = g.pt_step;
  *accepted_swaps = g.pt_accepted;
  return GPUMC_OK;
}

int gpumc_philox_probe(const uint32_t* ctr4, const uint32_t* key2, uint32_t* out4, int32_t n) {
  if (!ctr4 || !key2 || !out4 || n <= 0) return fail(GPUMC_EINVAL, "null argument");
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return fail(GPUMC_ENODEV, "no usable CUDA device");
  uint4 *dc = nullptr, *dout = nullptr;
  uint2* dk = nullptr;
  CUDA_TRY(cudaMalloc(&dc, 16 * (size_t)n));
  CUDA_TRY(cudaMalloc(&dk, 8 * (size_t)n));
  CUDA_TRY(cudaMalloc(&dout, 16 * (size_t)n));
  CUDA_TRY(cudaMemcpy(dc, ctr4, 16 * (size_t)n, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(dk, key2, 8 * (size_t)n, cudaMemcpyHostToDevice));
  k_philox_probe<<<(n + 255) / 256, 256>>>(dc, dk, dout, n);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(out4, dout, 16 * (size_t)n, cudaMemcpyDeviceToHost);
  cudaFree(dc);
  cudaFree(dk);
  cudaFree(dout);
  if (e != cudaSuccess) return fail(GPUMC_ECUDA, cudaGetErrorString(e));
  return GPUMC_OK;
}
