// Serving: continuous batching of simulation jobs.
//
// Jobs (model, lattice, beta ladder, thermalization + measurement sweeps)
// arrive through gpumc_submit.  Each scheduling round (gpumc_server_step)
//   1. admits waiting jobs in arrival order while their HBM footprint fits the
//      free part of the budget (lattices are created resident and stay on the
//      device until the job retires),
//   2. runs `chunk` sweeps of every active job in one batched launch per
//      kernel kind and sweep (jobs admitted in this round join the running
//      batch; each job's thermalize -> measure switch and its stop at its own
//      sweep target happen on the device, so unequal jobs share launches),
//   3. retires jobs that reached their target: drains their records, reduces
//      them, frees their memory and records the completion time.
// Results depend only on (seed, replica, sweep, site) keys, never on batch
// composition, so a job's spins are identical alone and in the mix.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstddef>
#include <cstring>
#include <deque>
#include <map>
#include <string>
#include <vector>

#include "../../include/gpumc.h"
#include "engine.h"
#include "host_internal.h"

using namespace gpumc;

namespace {

double now_s() {
  using clk = std::chrono::steady_clock;
  static const clk::time_point t0 = clk::now();
  return std::chrono::duration<double>(clk::now() - t0).count();
}

struct JobState {
  uint64_t id = 0;
  gpumc_job job{};
  std::vector<double> betas;
  size_t bytes = 0;
  gpumc_sim* sim = nullptr;
  double submit = 0, start = 0, finish = 0;
  uint64_t target = 0;
  int32_t status = 0;
  std::vector<std::vector<uint8_t>> spins;  // kept for finished jobs until polled
};

}  // namespace

struct gpumc_server {
  gpumc_engine* eng = nullptr;
  size_t budget = 0, in_use = 0;
  uint32_t chunk = 10;
  uint64_t next_id = 1;
  std::deque<JobState*> waiting;
  std::vector<JobState*> active;
  std::map<uint64_t, JobState*> finished;
  std::vector<gpumc_job_result> results;
  double attempts_total = 0.0, busy_s = 0.0;
  double admit_s = 0.0, sweep_s = 0.0, retire_s = 0.0;  // host time of the step's phases
  size_t max_waiting = 1u << 20;
  // final spins of jobs up to this many sites (all replicas) are kept for
  // gpumc_job_spins; larger jobs skip the device-to-host copy at retirement
  size_t keep_spins_sites = 1u << 20;
};

static int retire(gpumc_server* srv, JobState* js) {
  gpumc_sim* s = js->sim;
  gpumc_job_result r;
  std::memset(&r, 0, sizeof(r));
  r.job_id = js->id;
  r.status = js->status;
  r.n_replicas = s->n_rep;
  r.submit_s = js->submit;
  r.start_s = js->start;
  std::vector<gpumc_obs> obs(4096);
  double se = 0, sm = 0;
  size_t cnt = 0, n = 0;
  do {
    int rc = gpumc_observables(s, obs.data(), obs.size(), &n);
    if (rc) return rc;
    for (size_t i = 0; i < n; ++i) {
      se += obs[i].energy / (double)s->lay.n_sites;
      sm += obs[i].magnetization;
    }
    cnt += n;
  } while (n == obs.size());
  r.mean_energy = cnt ? se / (double)cnt : 0.0;
  r.mean_abs_m = cnt ? sm / (double)cnt : 0.0;
  const double per_sweep = (double)s->lay.n_sites * (double)s->n_rep * (s->lay.model == MSC ? 64.0 : 1.0);
  r.attempts = per_sweep * (double)js->target;
  srv->attempts_total += r.attempts;
  if ((size_t)s->lay.n_sites * s->n_rep <= srv->keep_spins_sites) {
    const size_t per = (size_t)s->lay.n_sites * (s->lay.model == O3 ? 12 : s->lay.model == MSC ? 8 : 1);
    js->spins.resize(s->n_rep);
    for (int k = 0; k < s->n_rep; ++k) {
      js->spins[k].resize(per);
      int rc = gpumc_get_spins(s, k, js->spins[k].data(), per);
      if (rc) return rc;
    }
  }
  js->finish = now_s();
  r.finish_s = js->finish;
  gpumc_destroy(s);
  js->sim = nullptr;
  srv->in_use -= js->bytes;
  srv->results.push_back(r);
  srv->finished[js->id] = js;
  return GPUMC_OK;
}

static int admit(gpumc_server* srv, JobState* js) {
  gpumc_spec spec = js->job.spec;
  spec.betas = js->betas.data();
  spec.record_capacity = (int32_t)std::max<uint64_t>(1, js->job.n_sweeps);
  gpumc_sim* s = nullptr;
  int rc = gpumc_create(srv->eng, &spec, js->job.base_seed, &s);
  if (rc) return rc;
  js->sim = s;
  js->start = now_s();
  js->target = js->job.n_therm + js->job.n_sweeps;
  // device-side phase schedule: records from sweep n_therm on, cone adaptation
  // below it, stop at the target
  s->phase = GPUMC_PHASE_MEASUREMENT;
  s->device_schedule = true;
  s->target = js->target;
  const int32_t one = 1;
  rc = s->set_group_field(offsetof(GroupDesc, measure), one);
  if (!rc) rc = s->set_group_field(offsetof(GroupDesc, measure_from), (uint64_t)js->job.n_therm);
  if (!rc) rc = s->set_group_field(offsetof(GroupDesc, adapt_until), (uint64_t)js->job.n_therm);
  for (int r = 0; r < s->n_rep && !rc; ++r) {
    rc = s->set_lat_field(r, offsetof(LatDesc, target), js->target);
    if (!rc && s->lay.model == O3 && s->lay.alg == METROPOLIS && s->lay.prop != GPUMC_O3_UNIFORM)
      rc = s->set_lat_field(r, offsetof(LatDesc, adapt), one);
  }
  if (!rc && cudaStreamSynchronize(srv->eng->stream) != cudaSuccess)
    rc = fail(GPUMC_ECUDA, "job admission: stream synchronize failed");
  return rc;
}

int gpumc_server_create(int32_t device, size_t hbm_budget, uint32_t chunk, gpumc_server** out) {
  if (!out) return fail(GPUMC_EINVAL, "out: null pointer");
  if (chunk == 0) return fail(GPUMC_EINVAL, "chunk: must be >= 1");
  gpumc_engine* eng = nullptr;
  int rc = gpumc_engine_create(device, &eng);
  if (rc) return rc;
  eng->use_graphs = false;  // the batch changes every round
  gpumc_server* srv = new gpumc_server();
  srv->eng = eng;
  srv->budget = hbm_budget;
  srv->chunk = chunk;
  *out = srv;
  return GPUMC_OK;
}

int gpumc_submit(gpumc_server* srv, const gpumc_job* job, uint64_t* job_id) {
  if (!srv || !job || !job_id) return fail(GPUMC_EINVAL, "null argument");
  gpumc_spec spec = job->spec;
  spec.record_capacity = (int32_t)std::max<uint64_t>(1, job->n_sweeps);
  int rc = validate_spec(&spec);
  if (rc) return rc;
  if (job->n_sweeps + job->n_therm == 0) return fail(GPUMC_EINVAL, "n_sweeps: job has no sweeps");
  const size_t bytes = footprint_bytes(&spec);
  if (bytes > srv->budget) return fail(GPUMC_EINVAL, "job footprint exceeds the server's HBM budget");
  if (srv->waiting.size() >= srv->max_waiting) return fail(GPUMC_EAGAIN, "admission queue is full");
  JobState* js = new JobState();
  js->id = srv->next_id++;
  js->job = *job;
  js->betas.assign(job->spec.betas, job->spec.betas + job->spec.n_temps);
  js->job.spec.betas = nullptr;
  js->bytes = bytes;
  js->submit = now_s();
  srv->waiting.push_back(js);
  *job_id = js->id;
  return GPUMC_OK;
}

int gpumc_server_step(gpumc_server* srv, int32_t* active) {
  if (!srv) return fail(GPUMC_EINVAL, "server: null");
  const double t0 = now_s();
  // 1. admission by footprint, arrival order
  while (!srv->waiting.empty() && srv->in_use + srv->waiting.front()->bytes <= srv->budget) {
    JobState* js = srv->waiting.front();
    srv->waiting.pop_front();
    int rc = admit(srv, js);
    if (rc) {
      js->status = rc;
      gpumc_job_result r;
      std::memset(&r, 0, sizeof(r));
      r.job_id = js->id;
      r.status = rc;
      r.submit_s = js->submit;
      r.finish_s = now_s();
      srv->results.push_back(r);
      delete js;
      continue;
    }
    srv->in_use += js->bytes;
    srv->active.push_back(js);
  }
  const double t1 = now_s();
  srv->admit_s += t1 - t0;
  // 2. one chunk of batched sweeps over every active job
  if (!srv->active.empty()) {
    int rc = gpumc_engine_sweep(srv->eng, srv->chunk);
    if (rc) return rc;
    if (cudaStreamSynchronize(srv->eng->stream) != cudaSuccess)
      return fail(GPUMC_ECUDA, "server step: stream synchronize failed");
  }
  const double t2 = now_s();
  srv->sweep_s += t2 - t1;
  // 3. retire finished jobs
  std::vector<JobState*> still;
  for (JobState* js : srv->active) {
    if (js->sim->sweeps >= js->target) {
      int rc = retire(srv, js);
      if (rc) return rc;
    } else {
      still.push_back(js);
    }
  }
  srv->active.swap(still);
  const double t3 = now_s();
  srv->retire_s += t3 - t2;
  srv->busy_s += t3 - t0;
  if (active) *active = (int32_t)(srv->active.size() + srv->waiting.size());
  return GPUMC_OK;
}

int gpumc_poll(gpumc_server* srv, gpumc_job_result* out, size_t cap, size_t* n) {
  if (!srv || !n) return fail(GPUMC_EINVAL, "null argument");
  const size_t k = std::min(cap, srv->results.size());
  if (k && !out) return fail(GPUMC_EINVAL, "out: null");
  std::copy(srv->results.begin(), srv->results.begin() + k, out);
  srv->results.erase(srv->results.begin(), srv->results.begin() + k);
  *n = k;
  return GPUMC_OK;
}

int gpumc_cancel(gpumc_server* srv, uint64_t job_id) {
  if (!srv) return fail(GPUMC_EINVAL, "server: null");
  for (auto it = srv->waiting.begin(); it != srv->waiting.end(); ++it) {
    if ((*it)->id == job_id) {
      gpumc_job_result r;
      std::memset(&r, 0, sizeof(r));
      r.job_id = job_id;
      r.status = 1;
      r.submit_s = (*it)->submit;
      r.finish_s = now_s();
      srv->results.push_back(r);
      delete *it;
      srv->waiting.erase(it);
      return GPUMC_OK;
    }
  }
  for (size_t i = 0; i < srv->active.size(); ++i) {
    JobState* js = srv->active[i];
    if (js->id == job_id) {
      cudaStreamSynchronize(srv->eng->stream);
      gpumc_job_result r;
      std::memset(&r, 0, sizeof(r));
      r.job_id = job_id;
      r.status = 1;
      r.submit_s = js->submit;
      r.start_s = js->start;
      r.finish_s = now_s();
      gpumc_destroy(js->sim);
      srv->in_use -= js->bytes;
      srv->results.push_back(r);
      srv->active.erase(srv->active.begin() + i);
      delete js;
      return GPUMC_OK;
    }
  }
  return fail(GPUMC_ENOTFOUND, "job_id: not waiting or running");
}

int gpumc_job_spins(gpumc_server* srv, uint64_t job_id, int32_t replica, void* host, size_t nbytes) {
  if (!srv || !host) return fail(GPUMC_EINVAL, "null argument");
  auto it = srv->finished.find(job_id);
  if (it == srv->finished.end()) return fail(GPUMC_ENOTFOUND, "job_id: not a finished job");
  JobState* js = it->second;
  if (replica < 0 || replica >= (int32_t)js->spins.size())
    return fail(GPUMC_ENOTFOUND, "replica: spins not kept for this job");
  const auto& v = js->spins[replica];
  if (nbytes < v.size()) return fail(GPUMC_EINVAL, "nbytes: buffer too small");
  std::memcpy(host, v.data(), v.size());
  return GPUMC_OK;
}

int gpumc_server_stats(gpumc_server* srv, double* attempts_total, double* busy_s, size_t* bytes_in_use) {
  if (!srv) return fail(GPUMC_EINVAL, "server: null");
  if (attempts_total) *attempts_total = srv->attempts_total;
  if (busy_s) *busy_s = srv->busy_s;
  if (bytes_in_use) *bytes_in_use = srv->in_use;
  return GPUMC_OK;
}

int gpumc_server_timing(gpumc_server* srv, double* admit_s, double* sweep_s, double* retire_s) {
  if (!srv) return fail(GPUMC_EINVAL, "server: null");
  if (admit_s) *admit_s = srv->admit_s;
  if (sweep_s) *sweep_s = srv->sweep_s;
  if (retire_s) *retire_s = srv->retire_s;
  return GPUMC_OK;
}

int gpumc_server_set_keep_spins(gpumc_server* srv, size_t max_sites) {
  if (!srv) return fail(GPUMC_EINVAL, "server: null");
  srv->keep_spins_sites = max_sites;
  return GPUMC_OK;
}

int gpumc_server_destroy(gpumc_server* srv) {
  if (!srv) return GPUMC_OK;
  for (JobState* js : srv->active) {
    gpumc_destroy(js->sim);
    delete js;
  }
  for (JobState* js : srv->waiting) delete js;
  for (auto& kv : srv->finished) delete kv.second;
  gpumc_engine_destroy(srv->eng);
  delete srv;
  return GPUMC_OK;
}
