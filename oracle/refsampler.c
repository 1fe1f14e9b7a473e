/*
 * CPU oracle, part 2: restatement of the reference sampler.  TEST
 * INFRASTRUCTURE ONLY: the statistical cross-check and the timed CPU
 * baseline, never a product code path.
 *
 * Follows the reference's single-site Metropolis path step for step:
 *   ClassicalMC::from_params hot init     CMC.rs/src/classical_mc.rs:443-489
 *   build_hypercubic + CsrLattice          CMC.rs/src/lattice/graph.rs:112-184, :417-451
 *   MetropolisCore::sweep_with_phase       CMC.rs/src/algorithms/metropolis.rs:67-106
 *   SiteOrder::prepare (Fisher-Yates)      CMC.rs/src/core/visit.rs:30-59
 *   metropolis_hastings_step               CMC.rs/src/core/trial.rs:68-101
 *   System::evaluate_trial / commit_trial  CMC.rs/src/lattice/state.rs:104-137
 *   local_energy over CSR incidences       CMC.rs/src/lattice/interaction.rs:149-181
 *   accept_log_probability                 Carlo.rs/src/acceptance.rs:11-22
 *   measure: Energy (cached), |M|          CMC.rs/src/observables/{energy,magnetization}.rs
 *   MultiSpinIsing sweep / measure         CMC.rs/src/multi_spin.rs:107-151, :220-286
 *   run_parallel (one chain per task)      Carlo.rs/src/scheduler.rs:345-405
 * Random numbers come from Xoshiro256++ seeded through the restated
 * RngStreamKey; the raw reference stream (rand 0.10.2) cannot be replayed
 * here, so parity with this sampler is statistical (|z| < 3).
 */
#include "oracle.h"
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef struct {
    size_t source, target;
    uint8_t bond_type;
    double weight;
} bond_t; /* same 32-byte footprint as the reference's Bond */

struct orc_ref {
    int model, dims, q;
    int64_t n;
    double J, beta, energy;
    double* spins; /* site-major, spin_dim components per site */
    int spin_dim;
    size_t* offsets;   /* n + 1 */
    size_t* nbr;       /* incidences: neighbour */
    size_t* edge_id;   /* incidences: edge */
    bond_t* edges;
    size_t n_edges;
    size_t* order;
    orc_xoshiro rng;
    double prop[3];
};

static double rng_f64(orc_xoshiro* g) { return (double)(orc_xoshiro_next(g) >> 11) * 0x1p-53; }

/* uniform integer in [0, range) (range >= 1): widening multiply + rejection */
static uint64_t rng_below(orc_xoshiro* g, uint64_t range) {
    uint64_t threshold = (0 - range) % range;
    for (;;) {
        __uint128_t m = (__uint128_t)orc_xoshiro_next(g) * range;
        if ((uint64_t)m >= threshold) return (uint64_t)(m >> 64);
    }
}

static int accept_log_probability(double logA, orc_xoshiro* g) {
    if (isnan(logA)) return 0;
    if (logA >= 0.0) return 1;
    if (isinf(logA)) return 0;
    double u = rng_f64(g);
    if (u < 2.2250738585072014e-308) u = 2.2250738585072014e-308;
    return log(u) < logA;
}

static void build_lattice(orc_ref* r, int64_t lx, int64_t ly, int64_t lz) {
    int64_t dims[3] = {lx, ly, lz};
    int nd = r->dims;
    int64_t strides[3] = {1, lx, lx * ly};
    r->n_edges = 0;
    r->edges = (bond_t*)malloc(sizeof(bond_t) * (size_t)(r->n * nd));
    for (int64_t site = 0; site < r->n; ++site) {
        int64_t coords[3], rem = site;
        for (int a = nd - 1; a >= 0; --a) {
            coords[a] = rem / strides[a];
            rem %= strides[a];
        }
        for (int a = 0; a < nd; ++a) {
            int64_t c = coords[a], next;
            if (c + 1 < dims[a]) next = c + 1;
            else if (dims[a] > 1) next = 0;
            else continue;
            bond_t b = {(size_t)site, (size_t)(site - c * strides[a] + next * strides[a]),
                        (uint8_t)a, 1.0};
            r->edges[r->n_edges++] = b;
        }
    }
    /* CSR incidences at both ends, edges stored once */
    size_t* deg = (size_t*)calloc((size_t)r->n, sizeof(size_t));
    for (size_t e = 0; e < r->n_edges; ++e) {
        deg[r->edges[e].source]++;
        deg[r->edges[e].target]++;
    }
    r->offsets = (size_t*)malloc(sizeof(size_t) * (size_t)(r->n + 1));
    r->offsets[0] = 0;
    for (int64_t s = 0; s < r->n; ++s) r->offsets[s + 1] = r->offsets[s] + deg[s];
    r->nbr = (size_t*)malloc(sizeof(size_t) * r->offsets[r->n]);
    r->edge_id = (size_t*)malloc(sizeof(size_t) * r->offsets[r->n]);
    memset(deg, 0, sizeof(size_t) * (size_t)r->n);
    for (size_t e = 0; e < r->n_edges; ++e) {
        size_t a = r->edges[e].source, b = r->edges[e].target;
        size_t ia = r->offsets[a] + deg[a]++;
        r->nbr[ia] = b; r->edge_id[ia] = e;
        size_t ib = r->offsets[b] + deg[b]++;
        r->nbr[ib] = a; r->edge_id[ib] = e;
    }
    free(deg);
}

static double bond_energy(const orc_ref* r, const double* a, const double* b, const bond_t* e) {
    switch (r->model) {
        case ORC_ISING: return -r->J * e->weight * a[0] * b[0];
        case ORC_POTTS: return ((size_t)a[0] == (size_t)b[0]) ? -r->J * e->weight : 0.0;
        default: return -r->J * e->weight * (a[0] * b[0] + a[1] * b[1] + a[2] * b[2]);
    }
}

static double local_energy(const orc_ref* r, size_t site, const double* proposed) {
    double energy = 0.0;
    int d = r->spin_dim;
    for (size_t i = r->offsets[site]; i < r->offsets[site + 1]; ++i) {
        const bond_t* e = &r->edges[r->edge_id[i]];
        if (e->source == site && e->target == site) {
            energy += 0.5 * bond_energy(r, proposed, proposed, e);
            continue;
        }
        if (e->source == site)
            energy += bond_energy(r, proposed, &r->spins[e->target * d], e);
        else
            energy += bond_energy(r, &r->spins[e->source * d], proposed, e);
    }
    return energy;
}

static int validate_spin(const orc_ref* r, const double* s) {
    switch (r->model) {
        case ORC_ISING: return s[0] == -1.0 || s[0] == 1.0;
        case ORC_POTTS: return isfinite(s[0]) && s[0] == floor(s[0]) && s[0] >= 0.0 && s[0] < r->q;
        default: {
            double n2 = s[0] * s[0] + s[1] * s[1] + s[2] * s[2];
            return fabs(n2 - 1.0) <= 3e-10;
        }
    }
}

static void random_unit_vector(orc_xoshiro* g, double out[3]) {
    int len = 0;
    while (len < 3) {
        double u1 = rng_f64(g);
        if (u1 < 2.2250738585072014e-308) u1 = 2.2250738585072014e-308;
        double u2 = rng_f64(g);
        double radius = sqrt(-2.0 * log(u1));
        double angle = 6.283185307179586 * u2;
        out[len++] = radius * cos(angle);
        if (len < 3) out[len++] = radius * sin(angle);
    }
    double norm = sqrt(out[0] * out[0] + out[1] * out[1] + out[2] * out[2]);
    if (norm > 1e-15)
        for (int i = 0; i < 3; ++i) out[i] /= norm;
}

double orc_ref_recompute_energy(const orc_ref* r) {
    double e = 0.0;
    int d = r->spin_dim;
    for (size_t i = 0; i < r->n_edges; ++i) {
        const bond_t* b = &r->edges[i];
        e += bond_energy(r, &r->spins[b->source * d], &r->spins[b->target * d], b);
    }
    return e;
}

orc_ref* orc_ref_create(int model, int dims, int64_t lx, int64_t ly, int64_t lz, int q, double J,
                        double beta, uint64_t base_seed, uint64_t chain, int hot) {
    orc_ref* r = (orc_ref*)calloc(1, sizeof(orc_ref));
    r->model = model;
    r->dims = dims;
    r->q = q;
    r->J = J;
    r->beta = beta;
    r->n = lx * ly * (dims == 3 ? lz : 1);
    r->spin_dim = model == ORC_O3 ? 3 : 1;
    build_lattice(r, lx, ly, dims == 3 ? lz : 1);
    r->spins = (double*)malloc(sizeof(double) * (size_t)(r->n * r->spin_dim));
    r->order = (size_t*)malloc(sizeof(size_t) * (size_t)r->n);
    for (int64_t s = 0; s < r->n; ++s) r->order[s] = (size_t)s;
    orc_xoshiro_seed(&r->rng, orc_stream_seed(base_seed, chain, 0, chain, 0, 0, 0, 0));
    for (int64_t s = 0; s < r->n; ++s) {
        double* sp = &r->spins[s * r->spin_dim];
        if (model == ORC_ISING) sp[0] = hot ? ((orc_xoshiro_next(&r->rng) >> 63) ? 1.0 : -1.0) : 1.0;
        else if (model == ORC_POTTS) sp[0] = hot ? (double)rng_below(&r->rng, (uint64_t)q) : 0.0;
        else if (hot) random_unit_vector(&r->rng, sp);
        else { sp[0] = 1.0; sp[1] = 0.0; sp[2] = 0.0; }
    }
    r->energy = orc_ref_recompute_energy(r);
    return r;
}

void orc_ref_destroy(orc_ref* r) {
    if (!r) return;
    free(r->spins); free(r->offsets); free(r->nbr); free(r->edge_id); free(r->edges);
    free(r->order); free(r);
}

void orc_ref_set_beta(orc_ref* r, double beta) { r->beta = beta; r->energy = orc_ref_recompute_energy(r); }
int64_t orc_ref_n_sites(const orc_ref* r) { return r->n; }

void orc_ref_sweep(orc_ref* r, int adapt) {
    (void)adapt;
    int64_t n = r->n;
    int d = r->spin_dim;
    for (int64_t i = n - 1; i >= 1; --i) {
        size_t j = (size_t)rng_below(&r->rng, (uint64_t)i + 1);
        size_t t = r->order[i]; r->order[i] = r->order[j]; r->order[j] = t;
    }
    double old[3];
    for (int64_t idx = 0; idx < n; ++idx) {
        size_t site = r->order[idx];
        double* cur = &r->spins[site * d];
        double* p = r->prop;
        if (r->model == ORC_ISING) p[0] = -cur[0];
        else if (r->model == ORC_POTTS) {
            uint64_t st = rng_below(&r->rng, (uint64_t)(r->q - 1));
            if (st >= (uint64_t)cur[0]) st += 1;
            p[0] = (double)st;
        } else random_unit_vector(&r->rng, p);
        if (!validate_spin(r, p)) abort();
        memcpy(old, cur, sizeof(double) * (size_t)d);
        double dE = local_energy(r, site, p) - local_energy(r, site, old);
        if (!isfinite(dE)) abort();
        double logA = -r->beta * dE;
        if (accept_log_probability(logA, &r->rng)) {
            memcpy(cur, p, sizeof(double) * (size_t)d);
            r->energy += dE;
        }
    }
}

void orc_ref_measure(const orc_ref* r, double* energy, double* mag) {
    *energy = r->energy;
    int64_t n = r->n;
    if (r->model == ORC_ISING) {
        double s = 0.0;
        for (int64_t i = 0; i < n; ++i) s += r->spins[i];
        *mag = fabs(s) / (double)n;
    } else if (r->model == ORC_POTTS) {
        int64_t counts[128] = {0};
        for (int64_t i = 0; i < n; ++i) counts[(int)r->spins[i]]++;
        int64_t best = 0;
        for (int k = 0; k < r->q; ++k) if (counts[k] > best) best = counts[k];
        *mag = ((double)r->q * (double)best - (double)n) / ((double)n * (double)(r->q - 1));
    } else {
        double sx = 0, sy = 0, sz = 0;
        for (int64_t i = 0; i < n; ++i) {
            sx += r->spins[3 * i]; sy += r->spins[3 * i + 1]; sz += r->spins[3 * i + 2];
        }
        *mag = sqrt(sx * sx + sy * sy + sz * sz) / (double)n;
    }
}

/* One chain's run: `therm` sweeps, then `meas` sweeps each followed by a
 * measurement (Energy per site and Magnetization, ClassicalMC::measure). */
void orc_ref_series(orc_ref* r, int therm, int meas, double* e_per_site, double* mag) {
    for (int s = 0; s < therm; ++s) orc_ref_sweep(r, 1);
    for (int s = 0; s < meas; ++s) {
        orc_ref_sweep(r, 0);
        double e, m;
        orc_ref_measure(r, &e, &m);
        e_per_site[s] = e / (double)r->n;
        mag[s] = m;
    }
}

/* ---- one chain per thread (Scheduler::run_parallel + RayonBackend) ------ */
typedef struct {
    int model, dims, q, therm, meas, tid, n_threads, n_chains;
    int64_t lx, ly, lz;
    double J, beta;
    uint64_t seed;
    double sum_e, sum_m, attempts, sweep_seconds;
} job_t;

static double now_s(void);

static void* chain_worker(void* arg) {
    job_t* j = (job_t*)arg;
    for (int c = j->tid; c < j->n_chains; c += j->n_threads) {
        orc_ref* r = orc_ref_create(j->model, j->dims, j->lx, j->ly, j->lz, j->q, j->J, j->beta,
                                    j->seed, (uint64_t)c, 1);
        double t0 = now_s(); /* lattice construction is not part of the timed sweeps */
        for (int s = 0; s < j->therm; ++s) orc_ref_sweep(r, 1);
        for (int s = 0; s < j->meas; ++s) {
            orc_ref_sweep(r, 0);
            double e, m;
            orc_ref_measure(r, &e, &m);
            j->sum_e += e / (double)r->n;
            j->sum_m += m;
        }
        j->sweep_seconds += now_s() - t0;
        j->attempts += (double)r->n * (double)(j->therm + j->meas);
        orc_ref_destroy(r);
    }
    return NULL;
}

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

double orc_ref_run_parallel(int model, int dims, int64_t lx, int64_t ly, int64_t lz, int q,
                            double J, double beta, uint64_t base_seed, int n_chains, int n_threads,
                            int therm, int meas, double* attempts, double* mean_e, double* mean_m) {
    if (n_threads < 1) n_threads = 1;
    if (n_threads > n_chains) n_threads = n_chains;
    pthread_t th[256];
    job_t jobs[256];
    if (n_threads > 256) n_threads = 256;
    for (int t = 0; t < n_threads; ++t) {
        job_t j = {model, dims, q, therm, meas, t, n_threads, n_chains, lx, ly, lz, J, beta,
                   base_seed, 0, 0, 0, 0};
        jobs[t] = j;
        pthread_create(&th[t], NULL, chain_worker, &jobs[t]);
    }
    double att = 0, se = 0, sm = 0, dt = 0;
    for (int t = 0; t < n_threads; ++t) {
        pthread_join(th[t], NULL);
        att += jobs[t].attempts; se += jobs[t].sum_e; sm += jobs[t].sum_m;
        if (jobs[t].sweep_seconds > dt) dt = jobs[t].sweep_seconds; /* slowest thread */
    }
    if (attempts) *attempts = att;
    double denom = (double)n_chains * (meas > 0 ? meas : 1);
    if (mean_e) *mean_e = se / denom;
    if (mean_m) *mean_m = sm / denom;
    return dt;
}

/* ---- restated MultiSpinIsing (shared order, 64 draws per site) ---------- */
double orc_ref_msc_run(int dims, int64_t lx, int64_t ly, int64_t lz, double J, double beta,
                       uint64_t base_seed, int sweeps, int measure, double* attempts) {
    orc_ref* r = orc_ref_create(ORC_ISING, dims, lx, ly, lz, 2, J, beta, base_seed, 0, 1);
    int64_t n = r->n;
    uint64_t* packed = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
    for (int64_t s = 0; s < n; ++s) packed[s] = r->spins[s] > 0 ? ~0ull : 0ull;
    int z = 2 * dims;
    double lut[7];
    for (int k = 0; k <= z; ++k) {
        double dE = 2.0 * J * (2.0 * k - z);
        double v = -beta * dE;
        lut[k] = v < 0.0 ? v : 0.0;
    }
    double t0 = now_s();
    for (int sw = 0; sw < sweeps; ++sw) {
        for (int64_t i = n - 1; i >= 1; --i) {
            size_t j = (size_t)rng_below(&r->rng, (uint64_t)i + 1);
            size_t t = r->order[i]; r->order[i] = r->order[j]; r->order[j] = t;
        }
        for (int64_t idx = 0; idx < n; ++idx) {
            size_t site = r->order[idx];
            uint64_t w = packed[site];
            uint8_t anti[64] = {0};
            for (size_t i = r->offsets[site]; i < r->offsets[site + 1]; ++i) {
                uint64_t x = w ^ packed[r->nbr[i]];
                for (int b = 0; b < 64; ++b) anti[b] += (uint8_t)((x >> b) & 1u);
            }
            uint64_t flip = 0;
            for (int b = 0; b < 64; ++b)
                if (accept_log_probability(lut[z - anti[b]], &r->rng)) flip |= 1ull << b;
            packed[site] = w ^ flip;
        }
        /* replica 0 extraction and exact energy, as the reference does per sweep */
        for (int64_t s = 0; s < n; ++s) r->spins[s] = (packed[s] & 1u) ? 1.0 : -1.0;
        r->energy = orc_ref_recompute_energy(r);
        if (measure) {
            volatile double acc = 0;
            for (int b = 0; b < 64; ++b) {
                double sum = 0, e = 0;
                for (int64_t s = 0; s < n; ++s) sum += ((packed[s] >> b) & 1u) ? 1.0 : -1.0;
                for (size_t i = 0; i < r->n_edges; ++i) {
                    double a = ((packed[r->edges[i].source] >> b) & 1u) ? 1.0 : -1.0;
                    double c = ((packed[r->edges[i].target] >> b) & 1u) ? 1.0 : -1.0;
                    e += -J * a * c;
                }
                acc += e + fabs(sum / (double)n);
            }
        }
    }
    double dt = now_s() - t0;
    if (attempts) *attempts = 64.0 * (double)n * (double)sweeps;
    free(packed);
    orc_ref_destroy(r);
    return dt;
}
