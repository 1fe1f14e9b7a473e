/*
 * CPU oracle for the lattice Metropolis engine.  TEST INFRASTRUCTURE ONLY:
 * the parity tests compare the device against it and the benchmark times it
 * as the CPU baseline; it is never a product code path.
 *
 * Two parts:
 *  1. A bit-exact replay of the engine's method (checkerboard colour order,
 *     Philox4x32-10 counter-based stream keyed by (seed, replica, sweep,
 *     site)).  Spin configurations produced by the CUDA kernels must equal
 *     these byte for byte (Ising, Potts, multi-spin) and bit for bit (O(3)).
 *  2. A restatement of the reference sampler (cmc-rs MetropolisCore +
 *     ClassicalMC): f64 spins on a CSR multigraph, a fresh Fisher-Yates visit
 *     order every sweep, Xoshiro256++, log-space acceptance.  Used for the
 *     |z|<3 statistical cross-checks and as the timed CPU baseline.
 *
 * Parity at the RNG boundary with the reference itself is unpinned: the
 * reference draws from rand 0.10.2 / rand_xoshiro 0.8.0 (not vendored, no
 * Rust toolchain here), so its raw stream cannot be replayed.  Everything
 * above the RNG (stream-key derivation, energies, LUTs, exchange rule,
 * observables) is pinned against the reference's own tests.
 */
#ifndef SCAMPER_ORACLE_H
#define SCAMPER_ORACLE_H
#include <stdint.h>
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_ISING = 0, ORC_POTTS = 1, ORC_O3 = 2, ORC_MSC = 3 };

/* Stream-tag values placed in counter word 1 (bits 1..7); bit 0 = colour. */
enum {
    ORC_TAG_ACC = 0,        /* 16-bit acceptance draws, 8 per 16-site chunk */
    ORC_TAG_PROP = 1,       /* 16-bit Potts proposal draws, 8 per chunk     */
    ORC_TAG_ACC_REFINE = 2, /* per-site 64 extra acceptance bits            */
    ORC_TAG_PROP_REFINE = 3,/* per-site 32-bit Lemire retries (Potts)       */
    ORC_TAG_INIT = 4,       /* hot initial state                            */
    ORC_TAG_O3 = 5,         /* O(3): cos-theta, phi, acceptance             */
    ORC_TAG_MSC = 6,        /* multi-spin bit planes (plane pair in bits 8+) */
    ORC_TAG_PT = 7,         /* replica exchange decisions                   */
    ORC_TAG_BITS = 8,       /* Ising bit planes of a 64-site row segment    */
    ORC_TAG_PBITS = 9,      /* Potts (q <= 4) proposal bit planes           */
    ORC_TAG_PACC = 10,      /* Potts (q <= 4) acceptance bit planes         */
    ORC_TAG_HBITS = 11,     /* heat bath: Ising bit planes                  */
    ORC_TAG_HB = 12,        /* heat bath: 64-bit uniforms of int8 Potts sites */
    ORC_TAG_O3HB = 13,      /* heat bath: O(3) (cos theta, phi) draws       */
    ORC_TAG_SW = 14,        /* cluster updates: bond activations            */
    ORC_TAG_SWFLIP = 15,    /* Swendsen-Wang: cluster decisions             */
    ORC_TAG_WOLFF = 16,     /* Wolff: seed site and target state            */
    ORC_TAG_O3CL = 17       /* O(3) cluster updates: reflection axis        */
};

/* Substream ids used with RngStreamKey::with_substream. */
enum { ORC_SUB_INIT = 0, ORC_SUB_SWEEP = 1 };

/* Threads of the discrete and multi-spin replays (rows of a colour pass are
 * split; results do not depend on the count).  Default 1. */
void orc_set_threads(int n);

/* --- RNG ---------------------------------------------------------------- */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
uint64_t orc_stream_seed(uint64_t base_seed, uint64_t task, uint64_t run, uint64_t chain,
                         uint64_t replica, uint64_t thread, uint64_t phase, uint64_t substream);
uint64_t orc_replica_key(uint64_t base_seed, uint64_t replica, uint64_t substream);
uint64_t orc_exchange_key(uint64_t base_seed);

/* Xoshiro256++ seeded like rand_core's seed_from_u64 (SplitMix64 fill). */
typedef struct { uint64_t s[4]; } orc_xoshiro;
void orc_xoshiro_seed(orc_xoshiro* g, uint64_t seed);
uint64_t orc_xoshiro_next(orc_xoshiro* g);

/* --- acceptance thresholds ---------------------------------------------- */
/* p -> 80-bit fixed point threshold T = floor(p * 2^80), split as a 17-bit
 * head (0..65536; 65536 means "always accept") and a 64-bit tail. */
void orc_threshold(double p, uint32_t* head, uint64_t* tail);
/* Acceptance table for a discrete model.  Ising: class = number of
 * anti-aligned neighbours k in 0..z, dE = 2J(z-2k).  Potts: class = d + z,
 * d = n(new) - n(old) in -z..z, dE = -J d.  Returns number of classes. */
int orc_build_table(int model, int dims, double J, double beta, uint32_t* head, uint64_t* tail);
/* Heat-bath tables (HeatBathable for IsingModel / PottsModel, CMC.rs/src/
 * lattice/models.rs:158-186, :340-380).  Ising: T[k] = p(|x_k|) as 80-bit
 * thresholds, k = down neighbours, x_k = 2 beta J (z - 2k), p(x) = 1 / (1 +
 * exp(-x)) clamped to 1 - 2^-53.  Potts: tail[d] = floor(2^60 exp(-beta |J|
 * d)), d = 0..z, head = 0.  Returns the entry count. */
int orc_build_table_hb(int model, int dims, double J, double beta, uint32_t* head, uint64_t* tail);

/* --- checkerboard replay: int8 Ising / Potts -----------------------------
 * Ising decisions use bit planes: a row is cut into 64-site segments
 * (segment id g = rho * ceil(Lx/64) + x/64, rho = y + Ly*z); the 32 sites of
 * one colour in a segment are numbered i = (x & 63) >> 1; plane j (0 = most
 * significant) is word j & 3 of Philox(g, colour | TAG_BITS << 1 |
 * (j >> 2) << 8, sweep), and its bit i is bit j of site i's uniform u.  A site
 * flips iff u < T[k] compared most-significant bit first over 80 planes.
 * Potts decisions use the 16-bit chunk draws (TAG_ACC / TAG_PROP). */
void orc_init_discrete(int model, int dims, int64_t lx, int64_t ly, int64_t lz, int q,
                       uint64_t base_seed, uint64_t replica, int hot, int8_t* spins);
/* One full sweep (colour 0 then colour 1).  Returns the integer energy change
 * in units of J (E = J * E_int); *accepted receives the accepted count. */
int64_t orc_sweep_discrete(int model, int dims, int64_t lx, int64_t ly, int64_t lz, int q,
                           const uint32_t* head, const uint64_t* tail, uint64_t key64,
                           uint64_t sweep, int8_t* spins, int64_t* accepted);
int64_t orc_energy_int(int model, int dims, int64_t lx, int64_t ly, int64_t lz, const int8_t* spins);

/* --- checkerboard replay: O(3) fp32 -------------------------------------- */
void orc_init_o3(int dims, int64_t lx, int64_t ly, int64_t lz, uint64_t base_seed,
                 uint64_t replica, int hot, float* sx, float* sy, float* sz);
/* omc = 1 - cos(alpha) of the cone; beta and J as float.  Returns the
 * accumulated energy change (sum of fp32 dE in double). */
/* One heat-bath sweep (HeatBathCore, CMC.rs/src/algorithms/heat_bath.rs:41-66)
 * of an int8 Ising or Potts lattice in the engine's checkerboard order and
 * random streams; returns dE in units of J, *changed = sites whose spin
 * changed. */
int64_t orc_sweep_discrete_hb(int model, int dims, int64_t lx, int64_t ly, int64_t lz, int q,
                              double J, const uint32_t* head, const uint64_t* tail, uint64_t key64,
                              uint64_t sweep, int8_t* spins, int64_t* changed);
/* One O(3) heat-bath sweep (ContinuousHeatBathCore, heat_bath.rs:75-134, with
 * the Langevin inverse CDF of models.rs:617-663) with the engine's fp32
 * arithmetic; returns the exact fp64 dE. */
double orc_sweep_o3_hb(int dims, int64_t lx, int64_t ly, int64_t lz, float J, float beta,
                       uint64_t key64, uint64_t sweep, float* sx, float* sy, float* sz,
                       int64_t* changed);
/* Cluster updates (SWCore, CMC.rs/src/algorithms/swendsen_wang.rs:73-138;
 * WolffCore, CMC.rs/src/algorithms/wolff.rs:73-135) of an int8 Ising / Potts
 * lattice in the engine's random streams: bonds between equal neighbours
 * active iff a 64-bit uniform is below `thr` (orc_cluster_threshold),
 * components by union-find with the minimum site as root, one decision per
 * root (SW) or the seed's component flipped to the target (Wolff).  Returns
 * dE in units of J; *changed = sites whose spin changed. */
uint64_t orc_cluster_threshold(int model, double J, double beta);
int64_t orc_sweep_cluster(int model, int dims, int64_t lx, int64_t ly, int64_t lz, int q, int wolff,
                          uint64_t thr, uint64_t key64, uint64_t sweep, int8_t* spins, int64_t* changed);
/* O(3) cluster updates (ClusterModel for ONModel, CMC.rs/src/lattice/
 * models.rs:516-579): embedded Ising variables along a random axis per sweep,
 * bonds p = 1 - exp(-2 beta J s_i.r s_j.r) for positive products, clusters
 * reflected (SW: each with probability 1/2; Wolff: the seed's), in the
 * engine's fp32 arithmetic; returns the exact fp64 dE. */
double orc_sweep_cluster_o3(int dims, int64_t lx, int64_t ly, int64_t lz, float J, float beta, int wolff,
                            uint64_t key64, uint64_t sweep, float* sx, float* sy, float* sz, int64_t* changed);
float orc_one_minus_exp_neg(float x);
float orc_log_one_minus(float y);
/* O(3) Metropolis with proposal prop: 0 the cap (omc = 1 - cos(alpha)), 1
 * StandardStrategy's uniform unit vector, 2 OPSSStrategy's plane rotation
 * (omc = sigma); CMC.rs/src/lattice/proposal.rs:45-167. */
/* O(3) Metropolis arithmetic of the sweep kernels (bit-identical): 23-bit
 * uniforms from bits, (cos, sin) of a turn, exp(x) for x <= 0, the proposal
 * and the decision of one site, and the fixed-point observables (energy from
 * colour-1 bond sums at 2^-19, magnetisation components at 2^-21). */
float orc_unit23(uint32_t u);
float orc_half23(uint32_t u);
/* The three draw words of an O(3) site from two Philox words (one Philox
 * call per pair of adjacent sites of a colour in a row, keyed by the pair's
 * first site; the first site takes words 0-1, the second words 2-3). */
void orc_o3_split(uint32_t u, uint32_t v, uint32_t o[4]);
void orc_sincos23(uint32_t u, float* c, float* s);
float orc_exp_neg2(float x);
void orc_o3_propose(int prop, float ax, float ay, float az, const uint32_t o[4], float omc,
                    float* nx, float* ny, float* nz);
int orc_o3_accept(float ax, float ay, float az, float px, float py, float pz, float hx, float hy,
                  float hz, float mJ, float beta, uint32_t o2);
void orc_o3_fixed_observables(int dims, int64_t lx, int64_t ly, int64_t lz, double J, const float* sx,
                              const float* sy, const float* sz, double* energy, double m[3]);
double orc_sweep_o3_prop(int dims, int64_t lx, int64_t ly, int64_t lz, float J, float beta,
                         float omc, int prop, uint64_t key64, uint64_t sweep, float* sx, float* sy,
                         float* sz, int64_t* accepted);
/* OPSSStrategy::finish_sweep (proposal.rs:156-167) in fp32 */
float orc_opss_adapt(float sigma, int64_t accepted, int64_t attempted);
double orc_sweep_o3(int dims, int64_t lx, int64_t ly, int64_t lz, float J, float beta,
                    float omc, uint64_t key64, uint64_t sweep, float* sx, float* sy,
                    float* sz, int64_t* accepted);
double orc_energy_o3(int dims, int64_t lx, int64_t ly, int64_t lz, double J, const float* sx,
                     const float* sy, const float* sz);
float orc_o3_adapt(float omc, int64_t accepted, int64_t attempted);
float orc_exp_neg(float x);                       /* engine's exp for x <= 0 */
void orc_sincos_turn(uint32_t u, float* c, float* s); /* cos/sin(2 pi u 2^-32) */

/* --- checkerboard replay: 64-replica multi-spin Ising --------------------- */
void orc_init_msc(int dims, int64_t lx, int64_t ly, int64_t lz, uint64_t base_seed, int hot,
                  uint64_t* words);
void orc_sweep_msc(int dims, int64_t lx, int64_t ly, int64_t lz, const uint32_t* head,
                   const uint64_t* tail, uint64_t key64, uint64_t sweep, uint64_t* words,
                   int64_t* accepted);
/* Per-replica energy (units of J) and magnetisation sums. */
void orc_msc_observables(int dims, int64_t lx, int64_t ly, int64_t lz, const uint64_t* words,
                         int64_t* e_int, int64_t* m_sum);

/* --- parallel tempering exchange ----------------------------------------- */
/* label[r] = temperature index held by replica r; energies[r] = physical
 * energy of replica r; betas[t] = ladder.  exchange_step is 1-based
 * (sweep_count / interval).  Returns number of accepted swaps. */
int orc_pt_exchange(int n, const double* betas, const double* energies, int32_t* label,
                    uint64_t exchange_key, uint64_t exchange_step, int32_t* accepted_pairs);
int orc_accept_log(double log_acceptance, uint64_t u64);

/* --- reference-semantics sampler (restated cmc-rs MetropolisCore) --------- */
typedef struct orc_ref orc_ref;
orc_ref* orc_ref_create(int model, int dims, int64_t lx, int64_t ly, int64_t lz, int q, double J,
                        double beta, uint64_t base_seed, uint64_t chain, int hot);
void orc_ref_destroy(orc_ref* r);
void orc_ref_sweep(orc_ref* r, int adapt);
/* observables of the current state: E (total), |M|/N (order parameter for
 * Potts), energy from cache */
void orc_ref_measure(const orc_ref* r, double* energy, double* mag);
/* therm sweeps, then meas measured sweeps: per-sweep E/N and |M| (or the
 * Potts order parameter) into the caller's arrays */
void orc_ref_series(orc_ref* r, int therm, int meas, double* e_per_site, double* mag);
double orc_ref_recompute_energy(const orc_ref* r);
void orc_ref_set_beta(orc_ref* r, double beta);
int64_t orc_ref_n_sites(const orc_ref* r);
/* Run n chains on up to n_threads threads (one chain per thread, like the
 * reference's Rayon task backend): therm + meas sweeps each, measuring every
 * measured sweep.  Returns the sweep seconds of the slowest thread (lattice
 * construction excluded); attempts written to *attempts. */
double orc_ref_run_parallel(int model, int dims, int64_t lx, int64_t ly, int64_t lz, int q,
                            double J, double beta, uint64_t base_seed, int n_chains, int n_threads,
                            int therm, int meas, double* attempts, double* mean_e, double* mean_m);
/* Restated MultiSpinIsing sweep + measure (64 replicas, shared order). */
double orc_ref_msc_run(int dims, int64_t lx, int64_t ly, int64_t lz, double J, double beta,
                       uint64_t base_seed, int sweeps, int measure, double* attempts);

#ifdef __cplusplus
}
#endif
#endif
