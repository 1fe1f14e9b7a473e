// Shared host/device definitions of the lattice engine.
//
// A "lattice" is one spin configuration (one replica) resident in HBM.  Its
// state lives in two ping-pong buffers: sweep t reads buf[t & 1] and writes
// buf[(t + 1) & 1], so every tile of a sweep reads an immutable snapshot and
// the two colour half-sweeps of the checkerboard can be fused in one pass
// (2 bytes of compulsory HBM traffic per int8 attempt instead of 3-4).
//
// Layout in HBM:
//   int8 models : rows of `pitch` = round_up(Lx, 16) bytes; row rho = y + Ly*z.
//   O(3)        : three float planes (x, y, z components), each rows of
//                 `pitch` = round_up(Lx, 4) floats.
//   multi-spin  : rows of `pitch` = round_up(Lx, 2) uint64 words (bit r =
//                 replica r, 1 = spin up), as in the reference's
//                 MultiSpinIsing::packed_spins (CMC.rs/src/multi_spin.rs:28-43).
#pragma once
#include <stdint.h>

namespace gpumc {

enum Model : int32_t { ISING = 0, POTTS = 1, O3 = 2, MSC = 3 };

// Stream tags (counter word 1, bits 1..7; bit 0 holds the colour).
enum Tag : uint32_t {
  TAG_ACC = 0, TAG_PROP = 1, TAG_ACC_REFINE = 2, TAG_PROP_REFINE = 3,
  TAG_INIT = 4, TAG_O3 = 5, TAG_MSC = 6, TAG_PT = 7, TAG_BITS = 8, TAG_PBITS = 9, TAG_PACC = 10,
  TAG_HBITS = 11,  // heat bath: Ising bit planes
  TAG_HB = 12,     // heat bath: 64-bit uniforms of int8 Potts sites
  TAG_O3HB = 13,   // heat bath: O(3) (cos theta, phi) draws
  TAG_SW = 14,     // cluster updates: bond activations
  TAG_SWFLIP = 15, // Swendsen-Wang: cluster decisions (counter = root site)
  TAG_WOLFF = 16,  // Wolff: seed site and target state
  TAG_O3CL = 17    // O(3) cluster updates: reflection axis of the sweep
};

enum Algorithm : int32_t { METROPOLIS = 0, HEAT_BATH = 1, SWENDSEN_WANG = 2, WOLFF = 3 };

constexpr int kMaxClasses = 13;    // 2z+1 for z = 6 (Potts on the cubic lattice)
constexpr int kMaxPottsCounts = 8; // fused order-parameter histogram (q <= 8)
constexpr int kThreads = 256;      // CTA size of the sweep kernels
constexpr int kEpiScratchInts = 3 * kThreads + 1;  // scratch of an epilogue in a kernel's dynamic shared memory
// O(3) z-march ring slots per tile: the copy of a plane is issued
// kO3RingSlots - 3 planes ahead of its first use
#ifndef GPUMC_O3_RING_SLOTS
#define GPUMC_O3_RING_SLOTS 4
#endif
constexpr int kO3RingSlots = GPUMC_O3_RING_SLOTS;
// O(3) z-march ring slots: a slot holds the three component planes of the
// tile's rows (y0-1 .. y0+hv) one after another, rows at the lattice's
// pitch, so each component's rows are one contiguous copy (split only where
// the rows wrap).  For the row pitches 32, 64 and 128 (row classes 1, 2, 3)
// the kernel is compiled with the pitch and a component stride of
// o3_class_rows(class) rows (the most rows a ring of kO3RingSlots slots of
// kO3MarchSmem bytes holds), so every neighbour offset is a compile-time constant;
// class 0 takes both at run time.
__host__ __device__ constexpr int o3_row_class(int pitch) {
  return pitch == 32 ? 1 : pitch == 64 ? 2 : pitch == 128 ? 3 : 0;
}
__host__ __device__ constexpr int o3_class_row(int cls) { return cls == 1 ? 32 : cls == 2 ? 64 : cls == 3 ? 128 : 0; }
constexpr int kO3MarchSmem = kO3RingSlots == 4 ? 56 * 1024 : 72 * 1024;  // ring bytes per CTA at most
__host__ __device__ constexpr int o3_class_rows(int cls) {
  return cls == 0 ? 0 : kO3MarchSmem / (12 * kO3RingSlots * o3_class_row(cls));
}
// observables binned on the device, in this order: Energy, E2, Magnetization,
// M2, M4 (DefaultObservableSet, CMC.rs/src/observables/common.rs:81-95)
constexpr int kBinObs = 5;

// Per-sweep accumulators, filled with atomics by the sweep kernels and
// drained by the epilogue (last CTA of the launch).
struct Accum {
  unsigned long long dE;        // int64 energy change (units of J), two's complement
  unsigned long long mag;       // int64 sum of spins (Ising)
  unsigned long long accepted;  // accepted moves
  unsigned long long counts[kMaxPottsCounts];
  double dEf;                   // O(3) cluster updates: accumulated energy change
  double mx, my, mz;            // O(3) cluster updates: magnetisation components
  unsigned long long ebq;       // O(3) sweeps: int64 sum over colour-1 sites of rint(2^19 s . h)
  unsigned long long mq[3];     // O(3) sweeps: int64 sums of rint(2^21 s_c) over all sites
  int32_t fresh;                // set when ebq holds the full bond sum of a sweep
  int32_t pad;
};

// One measured sweep of one lattice, as recorded on the device.
struct Record {
  double energy;       // physical energy after the sweep
  double m[3];         // Ising: {sum s}; Potts: {max count, -, -}; O(3): sum vector
  double accepted;     // accepted moves in the sweep
  int32_t label;       // temperature index held during the sweep
  int32_t pad;
  uint64_t sweep;      // sweep index (0-based) of this record
};

struct LatDesc {
  // geometry / model (immutable after creation)
  int32_t model, dims, lx, ly, lz, pitch, q, z;
  int32_t tile_cx, tile_y, tile_z;  // creation-time tile shape (kernels read TileItem's)
  int32_t group;                    // index into the group array (PT / records)
  int32_t replica;                  // replica index within its group
  int32_t prop;                     // O(3) Metropolis proposal: 0 cap, 1 uniform, 2 OPSS, 3 fast cap
  int64_t n_sites;
  void* buf[2];
  void* aux;                        // cluster updates: uint32 label per site
  uint64_t key;                     // Philox key of the sweep stream
  // mutable device state
  uint64_t sweep;                   // sweeps completed
  uint64_t target;                  // stop once sweep reaches this count (serving)
  long long e_int;                  // discrete: energy in units of J
  double e_f;                       // O(3): running energy
  float omc;                        // O(3): 1 - cos(cap half-angle); OPSS: rotation bound sigma
  int32_t adapt;                    // O(3): adapt omc during this sweep
  Accum acc;
  Accum acc2;                       // resident kernel: accumulators of odd launch-local sweeps
};

// A group is a set of lattices that share a temperature ladder and a record
// stream: the replicas of one simulation handle (a PT ensemble, or independent
// replicas with their own ladders).
struct GroupDesc {
  int32_t first_lat, n_rep, n_cls, pt_interval;  // pt_interval 0 = no exchange
  int32_t measure;                // record every sweep of this launch
  int32_t rec_cap, rec_count, overflow;
  int32_t* label;                 // [n_rep] temperature index of each replica
  int32_t* rep_at;                // [n_rep] scratch: replica holding each index
  const uint32_t* head;           // [n_temps][n_cls] 17-bit threshold heads
  const unsigned long long* tail; // [n_temps][n_cls] 64-bit threshold tails
  const double* betas;            // [n_temps]
  const float* betas_f;           // [n_temps] (O(3))
  double J;
  float Jf;
  int32_t pad1;
  uint64_t measure_from;          // record only sweeps with index >= this
  uint64_t adapt_until;           // O(3): adapt the cone only below this sweep
  uint64_t msc_recorded;          // multi-spin: sweep count of the last record
  uint64_t pt_key;                // exchange stream key
  uint64_t pt_step;               // exchanges attempted so far
  unsigned long long pt_accepted; // accepted swaps (all pairs)
  Record* records;                // [rec_cap][n_rep]
  // device-side binning of the measured observables (binsize 0: records)
  int32_t binsize;                // samples per bin
  int32_t bin_cap;                // completed bins the ring holds
  int32_t bin_count;              // completed bins not yet drained
  int32_t bin_fill;               // samples in the open bin (all slots alike)
  int32_t bin_by_label;           // slot = temperature label (else replica index)
  int32_t bin_overflow;
  double* bin_open;               // [n_rep][kBinObs] sums of the open bin
  double* bins;                   // [bin_cap][n_rep][kBinObs] completed bin means
};

// One CTA's work: the tile's origin and the tile shape of its lattice in the
// launch (chunks x rows x planes, the units of LatDesc's tile fields).  The
// shape travels with the tile because it depends on the launch: a batch that
// leaves CTA slots idle splits its lattices into smaller tiles.
struct TileItem {
  int32_t lat, x0, y0, z0;
  int32_t cx, ty, tz, pad;  // pad: position of the tile's group in the launch (LaunchCtl::group_ids)
};

// Device-side bookkeeping of one launch (last-CTA epilogue; grid barrier of
// the resident Ising kernel).
struct LaunchCtl {
  unsigned int done;
  int32_t n_groups;
  const int32_t* group_ids;  // [n_groups] indices into the group pool
  // per-group epilogues (group_epilogue): the tiles of each group of the
  // launch (TileItem::pad of a tile = its group's position) and how many of
  // them are done; null: one epilogue for the whole launch
  const int32_t* group_tiles = nullptr;  // [n_groups]
  unsigned int* group_done = nullptr;    // [n_groups]
  unsigned int bar = 0;      // resident kernel: grid-barrier arrivals of this launch
  int32_t err = 0;           // resident kernel: 1 = a barrier wait gave up
  unsigned int epi = 0;      // resident kernel: launch-local sweeps whose epilogue is done
  int32_t n_tiles = 0;       // tiles of the launch (kernels that stride over them)
};

}  // namespace gpumc
