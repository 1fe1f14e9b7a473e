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

static __device__ void pt_exchange(LatDesc* lats, GroupDesc* G) {
  const int n = G->n_rep;
  if (n < 2 || n > kMaxPtReplicas) return;
  const uint64_t step = ++G->pt_step;
  int32_t* at = G->rep_at;
  for (int r = 0; r < n; ++r) at[G->label[r]] = r;
  const int offset = (int)((step - 1) & 1u);
  unsigned long long accepted = 0;
  for (int t = offset; t + 1 < n; t += 2) {
    const int a = at[t], b = at[t + 1];
    const LatDesc* La = &lats[G->first_lat + a];
    const LatDesc* Lb = &lats[G->first_lat + b];
    const double ea = La->model == O3 ? La->e_f : G->J * (double)La->e_int;
    const double eb = Lb->model == O3 ? Lb->e_f : G->J * (double)Lb->e_int;
    const double wa = (G->betas[t] - G->betas[t + 1]) * ea;
    const double wb = (G->betas[t + 1] - G->betas[t]) * eb;
    const uint4 o = draw(G->pt_key, (uint64_t)t, 0u, TAG_PT, 0u, step);
    const unsigned long long u = (unsigned long long)o.x | ((unsigned long long)o.y << 32);
    if (accept_log(wa + wb, u)) {
      G->label[a] = t + 1;
      G->label[b] = t;
      at[t] = b;
      at[t + 1] = a;
      ++accepted;
    }
  }
  G->pt_accepted += accepted;
}

// slot 1 drains the second accumulator set (odd sweeps of a resident launch).
static __device__ void finish_group(LatDesc* lats, GroupDesc* G, int slot = 0) {
  if (lats[G->first_lat].sweep >= lats[G->first_lat].target) return;  // finished job
  // multi-spin records (64 per word lattice) are written by k_msc_record
  const bool msc = lats[G->first_lat].model == MSC;
  const bool measuring = G->measure && lats[G->first_lat].sweep >= G->measure_from;
  const bool rec = !msc && measuring && G->rec_count < G->rec_cap;
  uint64_t sweep_after = 0;
  for (int r = 0; r < G->n_rep; ++r) {
    LatDesc* L = &lats[G->first_lat + r];
    Accum* A = slot ? &L->acc2 : &L->acc;
    const long long dE = take_i64(&A->dE);
    const long long nacc = take_i64(&A->accepted);
    const long long mag = take_i64(&A->mag);
    Record R;
    R.m[0] = R.m[1] = R.m[2] = 0.0;
    if (L->model == O3) {
      const double dEf = take_f64(&A->dEf);
      L->e_f += dEf;
      R.energy = L->e_f;
      R.m[0] = take_f64(&A->mx);
      R.m[1] = take_f64(&A->my);
      R.m[2] = take_f64(&A->mz);
      if (L->adapt && L->sweep < G->adapt_until) L->omc = o3_adapt(L->omc, nacc, L->n_sites);
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
    if (rec) G->records[(size_t)G->rec_count * G->n_rep + r] = R;
    L->sweep += 1;
    sweep_after = L->sweep;
  }
  if (measuring && !msc) {
    if (rec) G->rec_count += 1;
    else G->overflow = 1;
  }
  if (G->pt_interval > 0 && sweep_after > 0 && (sweep_after % (uint64_t)G->pt_interval) == 0)
    pt_exchange(lats, G);
}

__device__ __forceinline__ void launch_epilogue(LatDesc* lats, GroupDesc* groups, LaunchCtl* ctl) {
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
  const int ng = ctl->n_groups;
  for (int gi = threadIdx.x; gi < ng; gi += blockDim.x) finish_group(lats, &groups[ctl->group_ids[gi]]);
  __syncthreads();
  if (threadIdx.x == 0) ctl->done = 0;
}

}  // namespace gpumc
