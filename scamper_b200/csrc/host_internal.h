// Host-side structures of the engine (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <set>
#include <string>
#include <vector>

#include "../../include/gpumc.h"
#include "engine.h"

namespace gpumc {

struct Layout {
  int model = 0, dims = 2, lx = 0, ly = 0, lz = 1, pitch = 0;
  int q = 2;             // Potts states
  int alg = METROPOLIS;  // sweep algorithm (METROPOLIS / HEAT_BATH / SWENDSEN_WANG / WOLFF)
  bool cluster = false;  // cluster update (label scratch per lattice, 4 launches per sweep)
  int prop = 0;          // O(3) Metropolis proposal (GPUMC_O3_*)
  bool bits = false;     // Potts on the bit-sliced kernel (q <= 4, Metropolis)
  bool march = false;    // 3D O(3) on the shared-memory z-march kernel
  int64_t n_sites = 0;
  size_t buf_bytes = 0;  // one ping-pong buffer
  int tile_cx = 0, tile_y = 0, tile_z = 1;
  size_t smem = 0;
  bool inplace = false;  // one buffer, updated in place (O(3)); else ping-pong
};

int fail(int code, const std::string& msg);
// Stream-ordered release into the device's memory pool (no device-wide
// synchronisation; the engine keeps freed memory pooled for reuse).
inline void dev_free(void* p, cudaStream_t st) {
  if (p) cudaFreeAsync(p, st);
}
uint64_t stream_key(uint64_t base, uint64_t replica, uint64_t phase, uint64_t substream);
void threshold80(double p, uint32_t& head, unsigned long long& tail);
int n_classes(int model, int dims);
void build_table(int model, int dims, double J, double beta, uint32_t* head,
                 unsigned long long* tail, int alg);
// kernel kinds of heat-bath layouts: the Metropolis kind of the same model and
// geometry plus this offset
constexpr int kKindHeatBath = 16;
// kernel kinds of cluster layouts: kKindCluster + 2 (Potts) + (dims - 2) + 4 (Wolff);
// O(3): kKindCluster + 8 + (dims - 2) + 2 (Wolff)
constexpr int kKindCluster = 32;
inline bool is_cluster_kind(int kind) { return kind >= kKindCluster && kind < kKindCluster + 16; }
// O(3) Metropolis with the uniform / OPSS / fast-cap proposal: the cap kind
// plus these
constexpr int kKindO3Uniform = 48, kKindO3Opss = 64, kKindO3Fast = 80;
// 2D Ising on the bit-sliced kernel (either single-site algorithm): the kinds
// the resident multi-sweep launch can take
inline bool is_ising2d_bits_kind(int kind) { return kind == 0 || kind == kKindHeatBath; }
// O(3) z-march kernels (any proposal or the heat bath): their ring copies
// flag a wait that gave up in LaunchCtl::err
// O(3) z-march kinds: 10 + the row class (o3_row_class) of the lattices
inline bool is_o3_march_kind(int kind) { return !is_cluster_kind(kind) && kind % 16 >= 10 && kind % 16 <= 13; }
// Reads and clears LaunchCtl::err after the stream's work; a set flag (a
// ring copy that did not land in time) becomes GPUMC_ECUDA.
int check_launch_flag(cudaStream_t st, LaunchCtl* ctl);
inline bool is_ising_bits_kind(int kind) {
  return kind == 0 || kind == 1 || kind == kKindHeatBath || kind == kKindHeatBath + 1;
}
int validate_spec(const gpumc_spec* s);
// CTA slots of one B200 (148 SMs x 4 resident sweep CTAs); the engine
// passes its device's own count.
constexpr int kDefaultSlots = 148 * 4;
constexpr size_t kIsingTileSmem = 48 * 1024;  // whole-row Ising tile budget
// O(3) z-march ring: the shared-memory budget that bounds a tile's rows

constexpr int kDefaultSlots3 = 148 * 2;  // resident 3D Ising sweep CTAs of one B200
Layout plan_layout(const gpumc_spec* s, int slots = kDefaultSlots, int slots3 = kDefaultSlots3);
int ising_tile_rows(int ly, int n_rep, int nseg, int hv_max, int slots);
bool layout_ok(const Layout& L);
void enumerate_tiles(const Layout& L, int lat, std::vector<TileItem>& out);
int kernel_kind(const Layout& L);
int64_t count_tiles(const Layout& L);
// Split the tiles of the layouts of one launch (n_rep lattices each) until the
// launch has at least half of `slots` CTAs or no tile can be split further.
void refine_layouts(std::vector<Layout>& lays, const std::vector<int>& reps, int slots);
int family_slots(const Layout& L, int slots, int slots3);
size_t footprint_bytes(const gpumc_spec* s);
int launch_sweep_kernel(cudaStream_t st, int kind, const TileItem* tiles, int n_tiles,
                        LatDesc* lats, GroupDesc* groups, LaunchCtl* ctl, size_t smem);
int launch_msc_measure(cudaStream_t st, const Layout& L, const LatDesc* lats, int lat,
                       unsigned long long* counters);
const std::string& last_error_ref();
size_t g_last_error_size();
int launch_msc_record(cudaStream_t st, LatDesc* lats, GroupDesc* groups, int group,
                      unsigned long long* counters);

// Resident (temporally blocked) launch of whole-row 2D Ising tiles: the
// neighbour table (tile above / below of each tile) and the edge-row
// exchange buffer of a tile list that qualifies (see build_resident).
struct ResidentPlan {
  bool on = false;
  int alg = METROPOLIS;  // kernel variant (all tiles of a plan share it)
  int dims = 2;          // 2: whole-row square tiles; 3: whole-plane cubic slabs
  size_t smem = 0;       // dynamic shared memory of the resident launch
  int2* d_nbr = nullptr;
  uint2* d_xchg = nullptr;
  int xstride = 0;  // uint2 words of exchange space per tile
  void release(cudaStream_t st);
};

struct BatchPlan {
  int kind = 0;
  size_t smem = 0;
  TileItem* d_tiles = nullptr;
  int n_tiles = 0;
  int32_t* d_gids = nullptr;
  int n_groups = 0;
  LaunchCtl* d_ctl = nullptr;
  ResidentPlan res;
  void release(cudaStream_t st);
};

// Qualifies a tile list for the resident Ising kernels (every tile a
// whole-row 2D Ising tile of at least two rows, or every tile a whole-plane
// 3D Ising slab of at least two planes; all tiles co-resident on the device)
// and allocates its neighbour table and exchange buffer; leaves rp.on false
// when the list does not qualify.
int build_resident(int device, cudaStream_t st, const std::vector<TileItem>& tiles,
                   const std::map<int, const Layout*>& layout_of_lat, size_t smem, ResidentPlan& rp);
// n_sweeps sweeps of every tile in one cooperative launch whose inter-CTA
// waits give up after spin_limit polls; waits for it and reports a wait that
// gave up as an error.
int launch_resident(cudaStream_t st, const TileItem* tiles, int n_tiles, LatDesc* lats,
                    GroupDesc* groups, LaunchCtl* ctl, const ResidentPlan& rp, size_t smem,
                    int n_sweeps, long long spin_limit);
constexpr long long kDefaultWaitLimit = 1ll << 22;  // polls of 128 ns, about half a second

}  // namespace gpumc

struct gpumc_sim;

struct gpumc_engine {
  int device = 0;
  cudaStream_t stream = nullptr;
  gpumc::LatDesc* d_lats = nullptr;
  gpumc::GroupDesc* d_groups = nullptr;
  int lat_cap = 16384;
  int group_cap = 8192;
  std::vector<bool> lat_used, group_used;
  std::set<gpumc_sim*> sims;
  bool batch_dirty = true;
  bool use_graphs = true;
  bool blocking = true;       // temporal blocking of qualifying Ising plans
  bool refine = true;         // split tiles of batches that leave CTA slots idle
  bool concurrent = true;     // each plan's sweeps on a stream of its own (disjoint lattices)
  std::vector<cudaStream_t> side;     // per-plan streams, created on first use
  std::vector<cudaEvent_t> side_done; // per-plan join events
  cudaEvent_t fork = nullptr;         // fork point on the engine stream
  uint64_t launches = 0;      // kernel launches issued by gpumc_engine_sweep
  long long wait_limit = gpumc::kDefaultWaitLimit;  // polls before an inter-CTA wait gives up
  int slots = gpumc::kDefaultSlots;  // resident sweep CTAs of the device (tile planning)
  int slots3 = gpumc::kDefaultSlots3;  // the same for the 3D Ising kernel
  std::vector<gpumc::BatchPlan> batch_plans;
  std::map<uint32_t, cudaGraphExec_t> batch_graphs;

  ~gpumc_engine();
  int rebuild_batch();
  int launch_batch_sweep();
  int launch_batch_sweeps(uint32_t n);
  int ensure_side(size_t n);
  bool has_per_sweep_work() const;
  uint64_t launches_per_batch_sweep() const;
  int run_graph(uint32_t n);
  void drop_graphs();
  int alloc_slots(int n, int& first);
  int alloc_group(int& g);
};

struct gpumc_sim {
  gpumc_engine* eng = nullptr;
  bool private_engine = false;
  gpumc_spec spec{};
  std::vector<double> betas;
  gpumc::Layout base;  // creation-time plan (tiles sized for a full launch)
  gpumc::Layout lay;   // plan of the simulation's own launches (base refined for it alone)
  gpumc::Layout blay;  // plan inside the engine's current batch (base refined for the batch)
  int n_rep = 1, n_temps = 1, n_cls = 0;
  int lat0 = -1, group = -1;
  uint64_t base_seed = 0;
  std::vector<void*> bufs;  // 2 per replica
  std::vector<void*> aux;   // cluster updates: label array per replica
  uint32_t* d_head = nullptr;
  unsigned long long* d_tail = nullptr;
  double* d_betas = nullptr;
  float* d_betas_f = nullptr;
  int32_t* d_label = nullptr;
  int32_t* d_rep_at = nullptr;
  gpumc::Record* d_records = nullptr;
  int rec_cap = 0, rec_used = 0;
  int rec_stride = 1;  // records per sweep
  unsigned long long* d_msc_counters = nullptr;
  gpumc::TileItem* d_tiles = nullptr;
  int n_tiles = 0;
  int32_t* d_gid = nullptr;
  gpumc::LaunchCtl* d_ctl = nullptr;
  gpumc::ResidentPlan res;  // plain path: resident Ising launch, when it qualifies
  bool blocking = true;      // plain path: use `res` when it is on
  uint64_t launches = 0;     // kernel launches issued by gpumc_sweep
  std::map<uint32_t, cudaGraphExec_t> graphs;
  uint64_t sweeps = 0;  // host mirror of the device sweep counter
  uint64_t audit_interval = 0;  // cache audit every this many sweeps (0 = off)
  uint64_t target = ~0ull;        // sweep target (serving)
  bool device_schedule = false;   // phases driven by measure_from / target on the device
  int phase = GPUMC_PHASE_THERMALIZATION;
  uint32_t pt_interval = 0;
  std::vector<gpumc_obs> pending;
  // device-side binning (gpumc_set_binning)
  int binsize = 0, bin_cap = 0;
  double* d_bin_open = nullptr;      // [n_rep][kBinObs]
  double* d_bins = nullptr;          // [bin_cap][n_rep][kBinObs]
  uint64_t bin_total = 0;            // measured sweeps in the device ring + open bin
  std::vector<double> pending_bins;  // drained bins, [bin][n_rep][kBinObs]

  ~gpumc_sim();
  int measure_room(uint32_t& room);
  void note_measured(uint32_t chunk);
  int drain_bins();
  int launch_one_sweep();
  int launch_msc_measurement();
  int run_graph(uint32_t n);
  int drain_records();
  int push_phase_flags();
  int upload_tables();
  int upload_own_tiles(std::vector<gpumc::TileItem>& tiles);
  void drop_graphs();
  int recompute(std::vector<double>& out, bool store);
  int audit();
  uint32_t sweeps_to_audit() const;
  int launch_energy(const void* buf, unsigned long long* d_e, unsigned int* d_bad);
  template <class T>
  int set_lat_field(int r, size_t offset, const T& v) {
    return cudaMemcpyAsync(reinterpret_cast<char*>(eng->d_lats + lat0 + r) + offset, &v, sizeof(T),
                           cudaMemcpyHostToDevice, eng->stream) == cudaSuccess
               ? GPUMC_OK
               : gpumc::fail(GPUMC_ECUDA, "descriptor update failed");
  }
  template <class T>
  int set_group_field(size_t offset, const T& v) {
    return cudaMemcpyAsync(reinterpret_cast<char*>(eng->d_groups + group) + offset, &v, sizeof(T),
                           cudaMemcpyHostToDevice, eng->stream) == cudaSuccess
               ? GPUMC_OK
               : gpumc::fail(GPUMC_ECUDA, "descriptor update failed");
  }
};
