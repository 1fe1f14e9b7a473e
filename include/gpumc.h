/*
 * gpumc.h - C ABI of the B200 lattice Metropolis engine.
 *
 * The engine replaces the hot path of the scamper workspace's classical crate
 * (cmc-rs): the single-site Metropolis sweep of Ising, q-state Potts and O(3)
 * spins on periodic square and cubic lattices, the 64-replica multi-spin
 * Ising variant, and the parallel-tempering exchange that carlo-rs schedules
 * around the sweep.  Each entry point below names the reference interface it
 * stands in for (paths within the scamper workspace).
 *
 * Conventions (mirroring the reference's contract, Carlo.rs/src/monte_carlo.rs
 * and Carlo.rs/src/error.rs):
 *   - every call returns an int status: 0 = ok, negative = GPUMC_E* code;
 *     gpumc_last_error() gives the message of the calling thread's last error
 *     (the reference's CarloError::InvalidConfig {field, reason} text);
 *   - handles are opaque; a handle is not thread-safe (the reference's
 *     `&mut self` ownership), distinct handles may be used from distinct host
 *     threads;
 *   - device memory is owned by the engine; host buffers passed in are
 *     caller-owned and copied;
 *   - there is no CPU fallback: without a usable CUDA device every call that
 *     needs one returns GPUMC_ENODEV.
 */
#ifndef GPUMC_H
#define GPUMC_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define GPUMC_OK 0
#define GPUMC_EINVAL -1   /* invalid configuration or argument          */
#define GPUMC_ENODEV -2   /* no usable CUDA device                      */
#define GPUMC_ECUDA -3    /* CUDA runtime error                         */
#define GPUMC_ENOMEM -4   /* device memory exhausted                    */
#define GPUMC_EAGAIN -5   /* server: job does not fit the HBM budget now */
#define GPUMC_ESTATE -6   /* call not valid in the handle's current state */
#define GPUMC_ENOTFOUND -7

/* models (cmc-rs IsingModel, PottsModel, HeisenbergModel = ONModel<3>,
 * MultiSpinIsing: CMC.rs/src/lattice/models.rs:29-595, CMC.rs/src/multi_spin.rs) */
#define GPUMC_ISING 0
#define GPUMC_POTTS 1
#define GPUMC_O3 2
#define GPUMC_ISING_MSC64 3

/* sweep algorithms: MetropolisCore (CMC.rs/src/algorithms/metropolis.rs) and
 * the heat bath, HeatBathCore (Ising, Potts) / ContinuousHeatBathCore (O(3))
 * (CMC.rs/src/algorithms/heat_bath.rs:12-134), the algorithm type parameter
 * of ClassicalMC<H, A> (CMC.rs/src/classical_mc.rs:21-31).  The multi-spin
 * model has Metropolis only. */
#define GPUMC_METROPOLIS 0
#define GPUMC_HEAT_BATH 1
/* cluster updates, Ising and Potts with J >= 0: one Swendsen-Wang update of
 * every cluster (SWCore, CMC.rs/src/algorithms/swendsen_wang.rs:73-138) or one
 * Wolff cluster flip (WolffCore, CMC.rs/src/algorithms/wolff.rs:73-135) per
 * sweep */
#define GPUMC_SWENDSEN_WANG 2
#define GPUMC_WOLFF 3

/* O(3) Metropolis proposals: the engine's cap around the current spin
 * (adapted half-angle), the reference's StandardStrategy (independent uniform
 * unit vector, CMC.rs/src/lattice/proposal.rs:45-63) and OPSSStrategy (random
 * plane rotation with adapted bound, proposal.rs:72-167).  GPUMC_O3_CAP_FAST
 * is the cap on the same random stream with the hardware approximations of
 * sqrt, reciprocal, sin / cos and exp: float32-tolerance parity (spins within
 * a few 1e-7 of the exact cap's, decisions equal except within about 1e-6 of
 * a threshold), not bit-identical to the CPU replay. */
#define GPUMC_O3_CAP 0
#define GPUMC_O3_UNIFORM 1
#define GPUMC_O3_OPSS 2
#define GPUMC_O3_CAP_FAST 3

#define GPUMC_INIT_HOT 0  /* "hot" / "random" initial_state */
#define GPUMC_INIT_COLD 1 /* "cold" / "ordered" */

/* run phases (Carlo.rs/src/phase.rs:11-35): proposal adaptation only while
 * thermalizing, records only while measuring */
#define GPUMC_PHASE_THERMALIZATION 1
#define GPUMC_PHASE_MEASUREMENT 2

typedef struct gpumc_engine gpumc_engine;
typedef struct gpumc_sim gpumc_sim;
typedef struct gpumc_server gpumc_server;

/* Simulation spec: the reference's Params keys for this path
 * (CMC.rs/src/classical_mc.rs:336-489: L|Lx,Ly,Lz, lattice_type
 * square|cubic, pbc, J, q, beta, initial_state) plus the replica ladder of
 * ParallelTemperingConfig (Carlo.rs/src/parallel_tempering.rs:53-60). */
typedef struct {
  int32_t model;            /* GPUMC_ISING / POTTS / O3 / ISING_MSC64          */
  int32_t dims;             /* 2 = square, 3 = cubic                           */
  int64_t lx, ly, lz;       /* even extents >= 4 (lz ignored for dims = 2)     */
  int32_t pbc;              /* must be 1: periodic boundaries                  */
  int32_t q;                /* Potts states, 2..8                              */
  double J;                 /* coupling, finite                                */
  int32_t n_replicas;       /* lattices in this handle (MSC: 64-bit words     */
                            /* lattices, 64 bit-replicas each)                 */
  int32_t n_temps;          /* entries in betas: 1 (shared) or n_replicas      */
  const double* betas;      /* inverse temperatures, finite and >= 0           */
  int32_t init;             /* GPUMC_INIT_HOT / GPUMC_INIT_COLD                */
  double cone_half_angle;   /* O(3): initial cap half-angle, or the OPSS bound  */
                            /* sigma (radians), (0, pi]                        */
  int32_t record_capacity;  /* measured sweeps buffered on the device (>= 1)   */
  int32_t algorithm;        /* GPUMC_METROPOLIS / HEAT_BATH / SWENDSEN_WANG / WOLFF */
  int32_t o3_proposal;      /* GPUMC_O3_CAP / UNIFORM / OPSS / CAP_FAST        */
} gpumc_spec;

/* One measured sweep of one replica (Context::measure of Energy, E2,
 * Magnetization, M2, M4: CMC.rs/src/observables/common.rs:81-95).  Energy is
 * the total physical energy, not per site.  For the multi-spin model there is
 * one record per bit-replica (64 per word lattice). */
typedef struct {
  uint64_t sweep;        /* 0-based index of the sweep that produced it       */
  int32_t replica;       /* lattice (or bit-replica) index                    */
  int32_t temp_index;    /* parameter-chain index held during the sweep       */
  double beta;
  double energy;
  double magnetization;  /* |M|/N (Ising, O(3)); Potts order parameter        */
  double acceptance;     /* accepted / attempted in this sweep                */
} gpumc_obs;

/* ---- engine (device context, stream, batched launches) ---------------- */
int gpumc_engine_create(int32_t device, gpumc_engine** out);
int gpumc_engine_destroy(gpumc_engine* eng);
/* One batched launch per sweep over every simulation in the engine (all
 * sizes, all replicas): the batched form of Scheduler::run_parallel's
 * independent chains (Carlo.rs/src/scheduler.rs:345-405).  measure != 0
 * records observables of every simulation whose phase is MEASUREMENT.
 * Sweeps are captured in CUDA graphs of up to 64 launches. */
int gpumc_engine_sweep(gpumc_engine* eng, uint32_t n_sweeps);
int gpumc_engine_synchronize(gpumc_engine* eng);
/* The CUDA stream (cudaStream_t) the engine launches on, for callers that
 * time or order work around the engine with their own events. */
int gpumc_engine_stream(gpumc_engine* eng, void** stream);
/* The engine a simulation handle runs on (its private one if created with
 * eng = NULL). */
int gpumc_sim_engine(gpumc_sim* sim, gpumc_engine** eng);
/* Kernel launches one sweep of this handle issues (sweep kernel plus, for a
 * measuring multi-spin handle, its measurement kernels). */
int gpumc_launches_per_sweep(gpumc_sim* sim, int32_t* n);
/* Temporal blocking of 2D Ising sweeps (default on): when every tile of the
 * handle's lattices fits on the device at once, a run of up to 64 sweeps is
 * one persistent launch that keeps the packed lattice in shared memory and
 * touches HBM only at its ends; off = one streaming launch per sweep.  Both
 * give identical spins, energies and records.  The _engine_ form applies to
 * gpumc_engine_sweep, the other to gpumc_sweep of one handle.  (The
 * reference has no counterpart: its sweep is one CPU loop per chain.) */
int gpumc_set_temporal_blocking(gpumc_sim* sim, int32_t enable);
int gpumc_engine_set_temporal_blocking(gpumc_engine* eng, int32_t enable);
/* Tile refinement (default on): a launch with fewer tiles than half the
 * device's CTA slots (a lone lattice, a few serving jobs) splits its 3D
 * Ising, Potts and O(3) tiles, largest first, until it fills them; off =
 * every lattice keeps the tiles sized for a full launch.  Both give identical
 * spins, energies and records.  The _engine_ form applies to the batches of
 * gpumc_engine_sweep, the other to gpumc_sweep of one handle; `n_tiles` of
 * gpumc_tile_count is the CTA count of one sweep launch of the handle's own
 * path.  (No counterpart in the reference: its sweep is one CPU loop.) */
int gpumc_set_tile_refinement(gpumc_sim* sim, int32_t enable);
int gpumc_engine_set_tile_refinement(gpumc_engine* eng, int32_t enable);
/* Concurrent kernel kinds (default on): the plans of an engine batch (one
 * per kernel kind) touch disjoint lattices, so gpumc_engine_sweep runs each
 * plan's sweeps on a stream of its own, forked from and joined back into the
 * engine stream; off = all plans in sequence on the engine stream.  Both
 * give identical results. */
int gpumc_engine_set_concurrent_kinds(gpumc_engine* eng, int32_t enable);
/* Polls (128 ns apart) after which an inter-CTA wait of the resident Ising
 * kernel (its per-sweep grid barrier, the wait for a PT exchange) gives up
 * (default 2^22, about half a second; 0 = give up at the first unsuccessful
 * poll).  A wait that gives up makes every CTA leave, the sweep call returns
 * GPUMC_ECUDA, and the handles of that launch must be restored (spins, sweep
 * count) before they continue: the failure path of a lost CTA, where the
 * reference's sweep panics (CMC.rs/src/classical_mc.rs:181-184). */
int gpumc_engine_set_wait_limit(gpumc_engine* eng, int64_t polls);
int gpumc_tile_count(gpumc_sim* sim, int32_t* n_tiles);
/* Tile knobs of the planner, for the autotuner (scamper_b200/autotune.py):
 * 0 keeps the analytic choice, a positive value replaces it in every layout
 * planned afterwards (simulations created, batches rebuilt): rows of the
 * whole-row 2D Ising tiles, planes of the whole-plane 3D Ising tiles, packed
 * 64-site segments per bit-sliced 2D Potts tile (at most 3072), planes per
 * whole-plane 3D Potts tile, and the rows / planes of the O(3) z-march tiles.
 * Results never depend on tiles (a colour pass reads only the other colour
 * and every draw is keyed by site or segment).  Process-wide.  (The
 * reference has no counterpart: its sweep is one CPU loop.) */
typedef struct {
  int32_t ising2d_rows, ising3d_planes, potts_segments, potts3d_planes, o3_rows, o3_planes;
} gpumc_tile_knobs;
int gpumc_set_tile_knobs(const gpumc_tile_knobs* knobs);
int gpumc_get_tile_knobs(gpumc_tile_knobs* knobs);
/* Kernel launches issued so far by gpumc_sweep of this handle / by
 * gpumc_engine_sweep of this engine (sweep, measurement and resident
 * launches; host copies excluded). */
int gpumc_launch_count(gpumc_sim* sim, uint64_t* n);
int gpumc_engine_launch_count(gpumc_engine* eng, uint64_t* n);

/* ---- simulation handle: ClassicalMC<H, MetropolisCore, _> ------------- */
/* FromParams::from_params (Carlo.rs/src/monte_carlo.rs:80-88;
 * CMC.rs/src/classical_mc.rs:443-489).  eng may be NULL (private engine). */
int gpumc_create(gpumc_engine* eng, const gpumc_spec* spec, uint64_t base_seed, gpumc_sim** out);
/* FromParams::validate_params: checks a spec without allocating. */
int gpumc_validate(const gpumc_spec* spec);
int gpumc_destroy(gpumc_sim* sim);
/* MonteCarlo::on_phase_start (Carlo.rs/src/monte_carlo.rs:31-77). */
int gpumc_set_phase(gpumc_sim* sim, int32_t phase);
/* MonteCarlo::sweep (+ measure after each sweep while measuring):
 * n_sweeps full sweeps of every replica of this handle, launched alone
 * (the plain single-simulation path). */
int gpumc_sweep(gpumc_sim* sim, uint32_t n_sweeps);
/* Drains recorded measurements (oldest first); *n receives the count. */
int gpumc_observables(gpumc_sim* sim, gpumc_obs* out, size_t cap, size_t* n);
/* Device-side binning of the measured observables (the carlo-rs Accumulator,
 * Carlo.rs/src/measurements.rs:60-183, fed on the device): while measuring,
 * each sweep adds Energy, E2, Magnetization, M2, M4 (powi moments: e*e, m*m,
 * (m*m)*(m*m)) of every slot to its open bin in sample order, and a full bin
 * of `binsize` samples becomes one bin mean (sum / binsize) - the values a
 * host Accumulator of the same bin size computes from the records.  A slot is
 * a temperature index when the handle has one beta per replica (PT chains),
 * else a replica index.  Per-sweep records are not written while binning is
 * on.  binsize 0 switches back to records; enabling resets the bin state
 * (records measured before stay available to gpumc_observables).
 * bin_capacity = completed bins buffered on the device (drained by the host
 * as needed).  Not for the multi-spin model or server jobs. */
int gpumc_set_binning(gpumc_sim* sim, int32_t binsize, int32_t bin_capacity);
/* Completed bins, oldest first: out[bin][slot][5] (slots = n_replicas);
 * *n_bins receives the count (at most cap_bins). */
int gpumc_drain_bins(gpumc_sim* sim, double* out, size_t cap_bins, size_t* n_bins);
/* The open (partial) bin: sums[slot][5] of its samples and their count *fill
 * (the reference's trailing partial bin, counted at finalize). */
int gpumc_open_bin(gpumc_sim* sim, double* sums, int32_t* fill);
/* Spin state of one replica in the reference's site order (x fastest,
 * CMC.rs/src/lattice/graph.rs:417-451): int8 (+-1 Ising, 0..q-1 Potts),
 * float32[3] per site (O(3)), uint64 per site (multi-spin). */
int gpumc_get_spins(gpumc_sim* sim, int32_t replica, void* host, size_t nbytes);
int gpumc_set_spins(gpumc_sim* sim, int32_t replica, const void* host, size_t nbytes);
/* Cached physical energies (System::energy, CMC.rs/src/lattice/state.rs:19-27)
 * of every replica (multi-spin: joint energy of the 64 bit-replicas). */
int gpumc_energy(gpumc_sim* sim, double* energies);
/* Exact recomputation compared with the cache (audit_lattice_cache,
 * CMC.rs/src/audit.rs:41-52); writes recomputed energies. */
int gpumc_recompute_energy(gpumc_sim* sim, double* energies);
/* Per-bit-replica energies and |M|/N of a multi-spin lattice
 * (MultiSpinIsing::measure, CMC.rs/src/multi_spin.rs:220-286). */
int gpumc_msc_replica_observables(gpumc_sim* sim, int32_t word_lattice, double* energy64,
                                  double* mag64);
/* Periodic cache audit (should_audit_cache / audit_lattice_cache,
 * CMC.rs/src/audit.rs:35-52, which the reference runs every 1024 completed
 * sweeps in debug builds): after every `interval`-th completed sweep,
 * gpumc_sweep and gpumc_engine_sweep compare each replica's cached energy with
 * an exact recomputation (tolerance 1e-10 (1 + |exact|)) and return
 * GPUMC_ESTATE with both values on a mismatch (the reference panics).  0 = off
 * (default).  Not for server jobs. */
int gpumc_set_audit_interval(gpumc_sim* sim, uint64_t interval);
int gpumc_sweep_count(gpumc_sim* sim, uint64_t* out);
/* O(3) proposal step of a replica: the cap half-angle (cap proposal) or the
 * rotation bound sigma (OPSS, OPSSStrategy::sigma). */
int gpumc_acceptance(gpumc_sim* sim, int32_t replica, double* cone_half_angle);
/* Resume support for state snapshots (the cmc-rs-snapshot-v2 format of
 * ClassicalMC::save_snapshot / load_snapshot, CMC.rs/src/classical_mc.rs:
 * 63-165, carries spins and beta; these carry the rest of this engine's
 * state).  The sweep counter of every replica (the position of the
 * counter-based random stream: resuming at the same count continues the same
 * trajectory), and one replica's O(3) cone parameter 1 - cos(alpha) as the
 * exact float the device holds. */
int gpumc_set_sweep_count(gpumc_sim* sim, uint64_t sweeps);
int gpumc_get_cone_omc(gpumc_sim* sim, int32_t replica, float* omc);
int gpumc_set_cone_omc(gpumc_sim* sim, int32_t replica, float omc);

/* ---- ParallelTemperingCompatible (Carlo.rs/src/parallel_tempering.rs:71-84;
 * CMC.rs/src/classical_mc.rs:203-229) ------------------------------------ */
int gpumc_log_weight_ratio(gpumc_sim* sim, int32_t replica, double new_beta, double* out);
int gpumc_change_parameter(gpumc_sim* sim, int32_t replica, double new_beta);
/* Device-side exchange every `interval` sweeps between ladder neighbours
 * (PtExchange::try_exchange, parallel_tempering.rs:362-419).  0 disables. */
int gpumc_pt_configure(gpumc_sim* sim, uint32_t interval);
/* labels[r] = ladder index held by replica r (always a permutation). */
int gpumc_pt_labels(gpumc_sim* sim, int32_t* labels);
/* Restores the labels of a resumed ensemble (labels[r] = ladder index held
 * by replica r; a permutation), the parameter-chain indices that
 * ParallelTemperingCompatible chains carry across a checkpoint
 * (set_chain_idx, Carlo.rs/src/parallel_tempering.rs:159-163).  Each
 * exchange's step and pairing follow from the sweep count (sweep / interval,
 * parallel_tempering.rs:372-373), so restoring the sweep count with
 * gpumc_set_sweep_count and the labels continues the same exchanges. */
int gpumc_pt_set_labels(gpumc_sim* sim, const int32_t* labels);
int gpumc_pt_stats(gpumc_sim* sim, uint64_t* exchange_steps, uint64_t* accepted_swaps);

/* ---- serving: continuous batching of simulation jobs ------------------ */
typedef struct {
  gpumc_spec spec;
  uint64_t base_seed;
  uint64_t n_sweeps;         /* measurement sweeps (each recorded)            */
  uint64_t n_therm;          /* thermalization sweeps before them             */
} gpumc_job;

typedef struct {
  uint64_t job_id;
  int32_t status;            /* 0 done, GPUMC_E* on failure, 1 cancelled      */
  int32_t n_replicas;
  double submit_s, start_s, finish_s;  /* server clock (seconds)             */
  double mean_energy;        /* per site, averaged over replicas and sweeps   */
  double mean_abs_m;
  double attempts;           /* spin-flip attempts performed                  */
} gpumc_job_result;

/* hbm_budget: bytes of device memory the server may hold for resident
 * lattices; chunk: sweeps per batched launch group (admission granularity). */
int gpumc_server_create(int32_t device, size_t hbm_budget, uint32_t chunk, gpumc_server** out);
/* Queues the job; gpumc_server_step admits queued jobs in arrival order as
 * their footprint fits the free budget.  The spec (its betas included) is
 * copied.  GPUMC_EAGAIN when the admission queue is full, GPUMC_EINVAL when
 * the footprint exceeds the whole budget. */
int gpumc_submit(gpumc_server* srv, const gpumc_job* job, uint64_t* job_id);
/* Runs one scheduling round: packs admitted jobs into the running batch,
 * launches `chunk` sweeps, retires finished jobs.  Returns the number of
 * active jobs in *active. */
int gpumc_server_step(gpumc_server* srv, int32_t* active);
int gpumc_poll(gpumc_server* srv, gpumc_job_result* out, size_t cap, size_t* n);
int gpumc_cancel(gpumc_server* srv, uint64_t job_id);
/* Final spins of a finished job's replica (kept until polled). */
int gpumc_job_spins(gpumc_server* srv, uint64_t job_id, int32_t replica, void* host, size_t nbytes);
int gpumc_server_stats(gpumc_server* srv, double* attempts_total, double* busy_s, size_t* bytes_in_use);
/* Host seconds the server's steps spent admitting jobs, sweeping (launches
 * and the wait for them) and retiring jobs, summed over all steps. */
int gpumc_server_timing(gpumc_server* srv, double* admit_s, double* sweep_s, double* retire_s);
/* Final spins are kept for gpumc_job_spins for jobs of at most this many
 * sites over all replicas (default 2^20); larger jobs skip the copy. */
int gpumc_server_set_keep_spins(gpumc_server* srv, size_t max_sites);
int gpumc_server_destroy(gpumc_server* srv);

/* ---- diagnostics ------------------------------------------------------- */
int gpumc_last_error(char* buf, size_t cap);
/* Adds `delta` to a replica's cached energy (integer models: a whole number
 * of J) without touching its spins: a host-made cache fault for testing the
 * audit.  gpumc_set_spins or gpumc_change_parameter restores the cache. */
int gpumc_perturb_energy_cache(gpumc_sim* sim, int32_t replica, double delta);
/* Bounds-checked builds (libgpumc_bounds.so, compiled with
 * -DGPUMC_DEBUG_BOUNDS): every checked global and shared-memory access of the
 * sweep, cluster and lattice kernels that falls outside its buffer is
 * skipped and counted.  Returns the violations counted since the last call
 * (and clears them), the module (0 O(3) sweep, 1 Ising bits, 2 Potts bits,
 * 3 int8 Potts, 4 multi-spin, 5 cluster, 6 lattice ops) and source line of
 * the first, and compiled = 0 for a release library (no checks). */
int gpumc_debug_bounds(uint64_t* hits, int32_t* first_module, int32_t* first_line, int32_t* compiled);
/* Device Philox4x32-10 outputs for n (counter, key) pairs (4 + 2 words each). */
int gpumc_philox_probe(const uint32_t* ctr4, const uint32_t* key2, uint32_t* out4, int32_t n);
/* Bytes of device memory a spec needs (both ping-pong buffers, tables,
 * records): the admission footprint. */
int gpumc_footprint(const gpumc_spec* spec, size_t* bytes);
/* Host-side tile plan of a spec's own sweep launch on a device with `slots`
 * CTA slots (`slots3` for the 3D bit-sliced kernels): the CTA count and the
 * kernel kind, with or without tile refinement.  Needs no device. */
int gpumc_plan_tiles(const gpumc_spec* spec, int32_t slots, int32_t slots3, int32_t refine,
                     int64_t* n_tiles, int32_t* kind);

/* ---- allocation-free exact energy ---------------------------------------
 * No counterpart in the reference: an engine-specific entry point for callers
 * that must not allocate device memory (their memory belongs to another
 * allocator under a fixed budget, or they cannot absorb the device-wide
 * synchronization of cudaFree).  Computes what gpumc_recompute_energy computes
 * - the exact energy in units of J (physical energy = J * value) of int8 Ising
 * (+-1) or Potts (0..q-1) lattices on periodic square / cubic lattices - but
 * allocates nothing: no cudaMalloc, cudaFree or allocating library call.
 *   spins      device pointer: n_lattices lattices back to back, each in the
 *              reference's site order (x fastest, no padding)
 *   energy_out device pointer: n_lattices int64 results
 *   stream     cudaStream_t to run on (NULL = default stream); the call is
 *              asynchronous with respect to the host
 * Extents are 1..2^20 (any parity); bonds follow the reference's periodic
 * hypercubic builder (CMC.rs/src/lattice/graph.rs:417-451): one +1 bond per
 * axis and site, wrapping at the far face, and none along an axis of extent 1
 * (extent 2 gives the two parallel bonds the builder makes).
 * Limits: 1 <= n_lattices <= 64, at most 4e9 sites per lattice; larger
 * requests return GPUMC_EINVAL.  Its reduction scratch is one file-scope
 * device array of 128 KiB (64 lattices x 256 partial sums) that every GPU
 * which loads the library holds until exit.  The first call in a context
 * (per device, and again after cudaDeviceReset) looks up that array's device
 * address; make it before any stream capture.  All calls on a device share
 * the array: calls that overlap on the GPU (different streams without
 * ordering between them) race and must not be issued.  A CUDA error already
 * pending when the call starts is returned as GPUMC_ECUDA and left pending. */
int gpumc_energy_int8_noalloc(int32_t model, int32_t dims, int64_t lx, int64_t ly, int64_t lz,
                              const int8_t* spins, int32_t n_lattices, long long* energy_out,
                              void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GPUMC_H */
