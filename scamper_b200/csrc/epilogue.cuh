// Per-launch epilogue, run by the last CTA of a sweep launch: folds the
// per-sweep accumulators into each lattice's cached energy (the reference's
// System::commit_trial energy cache, CMC.rs/src/lattice/state.rs:127-136),
// appends a measurement record, advances the sweep counter, adapts the O(3)
// cone during thermalisation, and performs the parallel-tempering exchange
// when the sweep count reaches a multiple of the exchange interval
// (Carlo.rs/src/parallel_tempering.rs:346-419: even/odd neighbour pairing by
// parameter index, combined log ratio (b_i - b_j)(E_i - E_j), temperatures
// move and configurations stay).
#pragma once
#include "device_common.cuh"

namespace gpumc {

constexpr int kMaxPtReplicas = 256;

__device__ __forceinline__ long long take_i64(unsigned long long* p) {
  return (long long)atomicExch(p, 0ull);
}
__device__ __forceinline__ double take_f64(double* p) {
  return __longlong_as_double((long long)atomicExch((unsigned long long*)p, 0ull));
}

__device__ __forceinline__ float o3_adapt(float omc, long long accepted, long long attempted) {
  // Multiplicative adaptation of w = 1 - cos(alpha) toward 50 % acceptance.
  // First-order form of OPSSStrategy::finish_sweep (CMC.rs/src/lattice/
  // proposal.rs:156-167, sigma *= exp(0.08 (rate - target))), with the rate
  // doubled because w grows as alpha^2.
  if (attempted <= 0) return omc;
  const float rate = __fdiv_rn((float)accepted, (float)attempted);
  const float f = __fadd_rn(1.0f, __fmul_rn(0.16f, __fsub_rn(rate, 0.5f)));
  float w = __fmul_rn(omc, f);
  w = w < 5.0e-9f ? 5.0e-9f : w;
  w = w > 2.0f ? 2.0f : w;
  return w;
}

__device__ __forceinline__ float opss_adapt(float sigma, long long accepted, long long attempted) {
  // OPSSStrategy::finish_sweep (CMC.rs/src/lattice/proposal.rs:156-167):
  // sigma *= exp(0.08 (rate - 0.5)), clamped to [1e-4, pi]; |x| <= 0.04, so
  // exp(x) is exp_neg(x) or 1 / exp_neg(-x)
  if (attempted <= 0) return sigma;
  const float rate = __fdiv_rn((float)accepted, (float)attempted);
  const float x = __fmul_rn(0.08f, __fsub_rn(rate, 0.5f));
  const float f = x <= 0.0f ? exp_neg(x) : __fdiv_rn(1.0f, exp_neg(-x));
  float s = __fmul_rn(sigma, f);
  s = s < 1e-4f ? 1e-4f : s;
  s = s > 0x1.921fb6p+1f ? 0x1.921fb6p+1f : s;
  return s;
}

// Epilogue flags of a group for the sweep being finished (GroupDesc::epi).
constexpr int32_t kEpiFinished = 1, kEpiMeasuring = 2, kEpiRecord = 4, kEpiMsc = 8, kEpiExchange = 16,
                  kEpiBin = 32;

// One measured sample of a replica into the open bin of its slot: the values
// Context::measure receives for Energy, E2, Magnetization, M2, M4 (the moments
// as powi computes them: e*e, m*m, (m*m)*(m*m)), summed in sample order with
// one rounding per operation, so that the bin means equal a host Accumulator's
// (Carlo.rs/src/measurements.rs:60-183: sum of the bin's samples / binsize).
// Magnetization as the records report it: |M|/N (Ising), (q max_s n_s - N) /
// (N (q - 1)) (Potts), |sum s|/N (O(3)).
static __device__ void bin_sample(const LatDesc* L, GroupDesc* G, int r, const Record& R) {
  const int s = G->bin_by_label ? R.label : r;
  double* acc = G->bin_open + (size_t)s * kBinObs;
  const double n = (double)L->n_sites;
  double m;
  if (L->model == POTTS)
    m = __ddiv_rn(__dsub_rn(__dmul_rn((double)L->q, R.m[0]), n), __dmul_rn(n, (double)(L->q - 1)));
  else if (L->model == O3)
    m = __ddiv_rn(__dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(R.m[0], R.m[0]), __dmul_rn(R.m[1], R.m[1])),
                                       __dmul_rn(R.m[2], R.m[2]))),
                  n);
  else
    m = __ddiv_rn(fabs(R.m[0]), n);
  const double m2 = __dmul_rn(m, m);
  const double v[kBinObs] = {R.energy, __dmul_rn(R.energy, R.energy), m, m2, __dmul_rn(m2, m2)};
  const bool close = G->bin_fill + 1 >= G->binsize;
  const bool room = G->bin_count < G->bin_cap;
#pragma unroll
  for (int k = 0; k < kBinObs; ++k) {
    const double a = __dadd_rn(acc[k], v[k]);
    if (close) {
      if (room) G->bins[((size_t)G->bin_count * G->n_rep + s) * kBinObs + k] = __ddiv_rn(a, (double)G->binsize);
      acc[k] = 0.0;
    } else {
      acc[k] = a;
    }
  }
}

// Per-replica part of the sweep epilogue: drain the accumulators of slot
// `slot`, update the cached energy, write the record, advance the sweep.
static __device__ void finish_replica(LatDesc* lats, GroupDesc* G, int r, int32_t flags, int slot) {
  LatDesc* L = &lats[G->first_lat + r];
  Accum* A = slot ? &L->acc2 : &L->acc;
  const long long dE = take_i64(&A->dE);
  const long long nacc = take_i64(&A->accepted);
  const long long mag = take_i64(&A->mag);
  Record R;
  R.m[0] = R.m[1] = R.m[2] = 0.0;
  if (L->model == O3) {
    const double dEf = take_f64(&A->dEf);
    if (A->fresh) {
      // sweeps: every bond has exactly one colour-1 end, so the energy after
      // the sweep is -J times the colour-1 pass's sum of s . h, accumulated
      // in fixed point (2^-19) from the fp32 dot products; the magnetisation
      // components likewise at 2^-21 (integer sums: independent of order)
      A->fresh = 0;
      L->e_f = -G->J * ((double)take_i64(&A->ebq) * 0x1p-19);
      R.m[0] = (double)take_i64(&A->mq[0]) * 0x1p-21;
      R.m[1] = (double)take_i64(&A->mq[1]) * 0x1p-21;
      R.m[2] = (double)take_i64(&A->mq[2]) * 0x1p-21;
    } else {
      L->e_f += dEf;  // cluster updates: exact change of the flipped clusters
      R.m[0] = take_f64(&A->mx);
      R.m[1] = take_f64(&A->my);
      R.m[2] = take_f64(&A->mz);
    }
    R.energy = L->e_f;
    if (L->adapt && L->sweep < G->adapt_until)
      L->omc = L->prop == 2 ? opss_adapt(L->omc, nacc, L->n_sites) : o3_adapt(L->omc, nacc, L->n_sites);
  } else {
    L->e_int += dE;
    R.energy = G->J * (double)L->e_int;
    if (L->model == POTTS) {
      long long best = 0;
      for (int s = 0; s < kMaxPottsCounts; ++s) {
        const long long c = take_i64(&A->counts[s]);
        best = c > best ? c : best;
      }
      R.m[0] = (double)best;
    } else {
      R.m[0] = (double)mag;
    }
  }
  R.accepted = (double)nacc;
  R.label = G->label[r];
  R.pad = 0;
  R.sweep = L->sweep;
  if (flags & kEpiRecord) G->records[(size_t)G->rec_count * G->n_rep + r] = R;
  if (flags & kEpiBin) bin_sample(L, G, r, R);
  L->sweep += 1;
}

// Sweep epilogue of the groups ids[0..ng), run by one whole CTA of kThreads
// threads (every thread must call it).  Groups are taken kThreads at a time;
// per batch, phases separated by block barriers:
//   0. one thread per group decides (from the state before the sweep
//      counter moves) whether the group is finished, measuring, recording,
//      and the batch's replica counts are prefix-summed in shared memory;
//   1. one thread per (group, replica) runs finish_replica (the group of a
//      flattened replica index is found by binary search over the offsets);
//   2. one thread per group counts the record and decides whether a PT
//      exchange is due (sweep count a multiple of the interval);
//   3. for each group with an exchange due, one thread per neighbour pair:
//      the pairs of one exchange step are disjoint and their decisions
//      independent, so they run in parallel with the same outcome as a
//      sequential loop over t = offset, offset + 2, ...
// Multi-spin records (64 per word lattice) are written by k_msc_record.
// EXT: the three per-group arrays live in `ext` (kEpiScratchInts ints of the
// caller's shared memory, e.g. a kernel's dynamic shared memory that is free
// by the time of the epilogue) instead of static shared memory of their own,
// so the kernel needs no more shared memory than its own.
template <bool EXT>
static __device__ void finish_groups_in(LatDesc* lats, GroupDesc* groups, const int32_t* ids, int ng, int slot,
                                        int* ext) {
  int* s_off;
  int32_t* s_f;
  int* s_due;
  if (EXT) {
    s_off = ext;
    s_f = ext + kThreads + 1;
    s_due = ext + 2 * kThreads + 1;
  } else {
    __shared__ int own_off[kThreads + 1];
    __shared__ int32_t own_f[kThreads];
    __shared__ int own_due[kThreads];
    s_off = own_off;
    s_f = own_f;
    s_due = own_due;
  }
  __shared__ int s_ndue;
  __shared__ unsigned long long s_acc;
  const int t = threadIdx.x;
  for (int base = 0; base < ng; base += kThreads) {
    const int nb = min(kThreads, ng - base);
    GroupDesc* G = t < nb ? &groups[ids[base + t]] : nullptr;
    int n = 0;
    if (G) {
      const LatDesc* L0 = &lats[G->first_lat];
      int32_t f = 0;
      if (L0->sweep >= L0->target) {
        f = kEpiFinished;
      } else {
        const bool msc = L0->model == MSC;
        const bool measuring = G->measure && L0->sweep >= G->measure_from;
        const bool binning = !msc && G->binsize > 0;
        f = (msc ? kEpiMsc : 0) | (measuring ? kEpiMeasuring : 0) |
            ((!msc && !binning && measuring && G->rec_count < G->rec_cap) ? kEpiRecord : 0) |
            ((binning && measuring) ? kEpiBin : 0);
        n = G->n_rep;
      }
      s_f[t] = f;
    }
    // inclusive scan of n over the batch: warp scans, then warp totals
    int v = n;
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xFFFFFFFFu, v, o);
      if ((t & 31) >= o) v += u;
    }
    __shared__ int s_warp[kThreads / 32];
    if ((t & 31) == 31) s_warp[t >> 5] = v;
    if (t == 0) {
      s_ndue = 0;
      s_off[0] = 0;
    }
    __syncthreads();
    int add = 0;
    for (int w = 0; w < (t >> 5); ++w) add += s_warp[w];
    s_off[t + 1] = v + add;  // s_off[i] = replicas of groups base .. base + i - 1
    __syncthreads();
    const int total = s_off[nb];
    for (int fi = t; fi < total; fi += kThreads) {
      int lo = 0, hi = nb - 1;  // last group index with s_off[g] <= fi
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (s_off[mid] <= fi) lo = mid;
        else hi = mid - 1;
      }
      finish_replica(lats, &groups[ids[base + lo]], fi - s_off[lo], s_f[lo], slot);
    }
    __syncthreads();
    if (G) {
      const int32_t f = s_f[t];
      if (!(f & kEpiFinished)) {
        if (f & kEpiBin) {
          if (++G->bin_fill >= G->binsize) {
            G->bin_fill = 0;
            if (G->bin_count < G->bin_cap) G->bin_count += 1;
            else G->bin_overflow = 1;
          }
        } else if ((f & kEpiMeasuring) && !(f & kEpiMsc)) {
          if (f & kEpiRecord) G->rec_count += 1;
          else G->overflow = 1;
        }
        const uint64_t sweep_after = lats[G->first_lat].sweep;
        if (G->pt_interval > 0 && sweep_after > 0 && (sweep_after % (uint64_t)G->pt_interval) == 0 &&
            G->n_rep >= 2 && G->n_rep <= kMaxPtReplicas) {
          G->pt_step += 1;
          s_due[atomicAdd(&s_ndue, 1)] = base + t;
        }
      }
    }
    __syncthreads();
    const int ndue = s_ndue;
    for (int i = 0; i < ndue; ++i) {
      GroupDesc* H = &groups[ids[s_due[i]]];
      const int m = H->n_rep;
      // exchange step = sweep count / interval, as PtExchange::try_exchange
      // derives it (Carlo.rs/src/parallel_tempering.rs:372-373), so a handle
      // resumed at a sweep count continues the pairing and the stream
      const uint64_t step = lats[H->first_lat].sweep / (uint64_t)H->pt_interval;
      int32_t* at = H->rep_at;
      if (t == 0) s_acc = 0;
      for (int r = t; r < m; r += kThreads) at[H->label[r]] = r;
      __syncthreads();
      const int offset = (int)((step - 1) & 1u);
      for (int p = t; offset + 2 * p + 1 < m; p += kThreads) {
        const int tt = offset + 2 * p;
        const int a = at[tt], b = at[tt + 1];
        const LatDesc* La = &lats[H->first_lat + a];
        const LatDesc* Lb = &lats[H->first_lat + b];
        const double ea = La->model == O3 ? La->e_f : H->J * (double)La->e_int;
        const double eb = Lb->model == O3 ? Lb->e_f : H->J * (double)Lb->e_int;
        const double wa = (H->betas[tt] - H->betas[tt + 1]) * ea;
        const double wb = (H->betas[tt + 1] - H->betas[tt]) * eb;
        const uint4 o = draw(H->pt_key, (uint64_t)tt, 0u, TAG_PT, 0u, step);
        const unsigned long long u = (unsigned long long)o.x | ((unsigned long long)o.y << 32);
        if (accept_log(wa + wb, u)) {
          H->label[a] = tt + 1;
          H->label[b] = tt;
          at[tt] = b;
          at[tt + 1] = a;
          atomicAdd(&s_acc, 1ull);
        }
      }
      __syncthreads();
      if (t == 0) H->pt_accepted += s_acc;
      __syncthreads();
    }
    __syncthreads();  // the next batch rewrites the shared arrays read above
  }
}

// The sweep epilogue of one group as soon as its last tile of the launch is
// done: each CTA (one tile) adds itself to its group's count, and the CTA
// completing the count finishes that group, so the epilogues of most groups
// overlap the tiles of the others and only the last group's remains at the
// end of the launch (measured: ~11 us per launch of one last-CTA epilogue
// over 32 to 256 groups, on the critical path of every sweep).  A launch
// without per-group counts falls back to launch_epilogue.
static __device__ void finish_groups(LatDesc* lats, GroupDesc* groups, const int32_t* ids, int ng, int slot) {
  finish_groups_in<false>(lats, groups, ids, ng, slot, nullptr);
}

template <bool EXT = false>
__device__ __forceinline__ void launch_epilogue(LatDesc* lats, GroupDesc* groups, LaunchCtl* ctl,
                                                int* ext = nullptr);
template <bool EXT = false>
__device__ __forceinline__ void group_epilogue(int pos, LatDesc* lats, GroupDesc* groups, LaunchCtl* ctl,
                                               int* ext = nullptr) {
  if (ctl->group_tiles == nullptr) {
    launch_epilogue<EXT>(lats, groups, ctl, ext);
    return;
  }
  __shared__ bool is_last_of_group;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned ticket = atomicAdd(&ctl->group_done[pos], 1u);
    is_last_of_group = ticket == (unsigned)ctl->group_tiles[pos] - 1u;
  }
  __syncthreads();
  if (!is_last_of_group) return;
  __threadfence();
  finish_groups_in<EXT>(lats, groups, ctl->group_ids + pos, 1, 0, ext);
  __syncthreads();
  if (threadIdx.x == 0) ctl->group_done[pos] = 0;
}

template <bool EXT>
__device__ __forceinline__ void launch_epilogue(LatDesc* lats, GroupDesc* groups, LaunchCtl* ctl, int* ext) {
  __shared__ bool is_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned ticket = atomicAdd(&ctl->done, 1u);
    is_last = ticket == gridDim.x - 1;
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  finish_groups_in<EXT>(lats, groups, ctl->group_ids, ctl->n_groups, 0, ext);
  __syncthreads();
  if (threadIdx.x == 0) ctl->done = 0;
}

}  // namespace gpumc
