/*
 * CPU oracle, part 1: bit-exact replay of the engine's checkerboard method.
 * TEST INFRASTRUCTURE ONLY (parity checker and CPU baseline), never shipped
 * on a product path.  Compiled with -ffp-contract=off so that every float
 * operation below is individually rounded, exactly like the device code.
 *
 * Reference anchors (paths relative to the scamper workspace):
 *   stream keys      Carlo.rs/src/rng_stream.rs:126-154 (seed/fold/mix64)
 *   acceptance       Carlo.rs/src/acceptance.rs:11-22
 *   Ising dE / LUT   CMC.rs/src/lattice/interaction.rs:73-84, :149-181;
 *                    CMC.rs/src/multi_spin.rs:84-91
 *   Potts proposal   CMC.rs/src/lattice/models.rs:212-218, :271-273
 *   site indexing    CMC.rs/src/lattice/graph.rs:417-451 (x fastest, +1 bonds)
 *   PT exchange      Carlo.rs/src/parallel_tempering.rs:362-419
 *   OPSS adaptation  CMC.rs/src/lattice/proposal.rs:156-167
 * Third-party algorithms restated from their publications: Philox4x32-10
 * (Salmon, Moraes, Dror, Shaw, SC'11); SplitMix64 and Xoshiro256++
 * (Steele/Lea/Flood 2014; Blackman & Vigna 2018) as pinned by the reference's
 * Cargo.lock (rand_core 0.10.0, rand_xoshiro 0.8.0).
 */
#include "oracle.h"
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* Philox4x32-10                                                             */
/* ------------------------------------------------------------------------ */
void orc_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int round = 0; round < 10; ++round) {
        if (round > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* ------------------------------------------------------------------------ */
/* RngStreamKey::seed restated                                               */
/* ------------------------------------------------------------------------ */
static uint64_t mix64(uint64_t v) {
    v += 0x9E3779B97F4A7C15ull;
    v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ull;
    v = (v ^ (v >> 27)) * 0x94D049BB133111EBull;
    return v ^ (v >> 31);
}
static uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
static uint64_t fold(uint64_t state, uint64_t domain, uint64_t value) {
    return mix64(state ^ domain ^ mix64(value + rotl64(domain, 17)));
}
uint64_t orc_stream_seed(uint64_t base_seed, uint64_t task, uint64_t run, uint64_t chain,
                         uint64_t replica, uint64_t thread, uint64_t phase, uint64_t substream) {
    uint64_t s = mix64(base_seed ^ 0x53435554544C4552ull);
    s = fold(s, 0x5441534Bull, task);
    s = fold(s, 0x52554E00ull, run);
    s = fold(s, 0x434841494E00ull, chain);
    s = fold(s, 0x5245504C49434100ull, replica);
    s = fold(s, 0x544852454144ull, thread);
    s = fold(s, 0x504841534500ull, phase);
    return fold(s, 0x535542535452ull, substream);
}
uint64_t orc_replica_key(uint64_t base_seed, uint64_t replica, uint64_t substream) {
    return orc_stream_seed(base_seed, 0, 0, 0, replica, 0, 0, substream);
}
uint64_t orc_exchange_key(uint64_t base_seed) {
    return orc_stream_seed(base_seed, 0, 0, 0, 0, 0, 3 /* RngPhase::Exchange */, 0);
}

/* ------------------------------------------------------------------------ */
/* Xoshiro256++                                                              */
/* ------------------------------------------------------------------------ */
void orc_xoshiro_seed(orc_xoshiro* g, uint64_t seed) {
    uint64_t st = seed;
    for (int i = 0; i < 4; ++i) {
        st += 0x9E3779B97F4A7C15ull;
        uint64_t z = st;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        g->s[i] = z ^ (z >> 31);
    }
}
uint64_t orc_xoshiro_next(orc_xoshiro* g) {
    uint64_t* s = g->s;
    uint64_t result = rotl64(s[0] + s[3], 23) + s[0];
    uint64_t t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl64(s[3], 45);
    return result;
}

/* ------------------------------------------------------------------------ */
/* thresholds                                                                */
/* ------------------------------------------------------------------------ */
void orc_threshold(double p, uint32_t* head, uint64_t* tail) {
    if (!(p > 0.0)) { *head = 0; *tail = 0; return; }        /* NaN or <= 0 */
    if (p >= 1.0) { *head = 65536u; *tail = 0; return; }
    double s = p * 65536.0;                                  /* exact scaling */
    double h = floor(s);
    double frac = s - h;                                     /* exact */
    *head = (uint32_t)h;
    *tail = (uint64_t)ldexp(frac, 64);                       /* exact, < 2^64 */
}

int orc_build_table(int model, int dims, double J, double beta, uint32_t* head, uint64_t* tail) {
    int z = 2 * dims;
    if (model == ORC_ISING || model == ORC_MSC) {
        for (int k = 0; k <= z; ++k) {
            double dE = 2.0 * J * (double)(z - 2 * k);
            double logA = -beta * dE;
            orc_threshold(logA >= 0.0 ? 1.0 : exp(logA), &head[k], &tail[k]);
        }
        return z + 1;
    }
    for (int d = -z; d <= z; ++d) {
        double dE = -J * (double)d;
        double logA = -beta * dE;
        orc_threshold(logA >= 0.0 ? 1.0 : exp(logA), &head[d + z], &tail[d + z]);
    }
    return 2 * z + 1;
}

/* Heat-bath tables: the host side of the engine's heat-bath kernels. */
int orc_build_table_hb(int model, int dims, double J, double beta, uint32_t* head, uint64_t* tail) {
    int z = 2 * dims;
    int n = model == ORC_POTTS ? 2 * z + 1 : z + 1;
    for (int c = 0; c < n; ++c) { head[c] = 0; tail[c] = 0; }
    if (model == ORC_POTTS) {
        for (int d = 0; d <= z; ++d)
            tail[d] = (uint64_t)ldexp(exp(-(beta * fabs(J)) * (double)d), 60);
        return n;
    }
    for (int k = 0; k <= z; ++k) {
        double ax = fabs(2.0 * beta * J * (double)(z - 2 * k));
        double p = 1.0 / (1.0 + exp(-ax));
        if (p >= 1.0) p = 1.0 - 0x1p-53;
        orc_threshold(p, &head[k], &tail[k]);
    }
    return n;
}

/* ------------------------------------------------------------------------ */
/* row-parallel colour passes                                                */
/* ------------------------------------------------------------------------ */
/* Within one checkerboard colour every site reads only sites of the other
 * colour and writes only itself, and every draw is keyed by site or row
 * segment, so the rows of a colour pass can be split across threads without
 * changing any result (integer sums are order-free).  orc_set_threads sets
 * the thread count of the discrete and multi-spin replays (default 1). */
static int g_threads = 1;
void orc_set_threads(int n) { g_threads = n < 1 ? 1 : (n > 256 ? 256 : n); }

typedef void (*rows_fn)(void* ctx, uint32_t colour, int64_t r0, int64_t r1, int64_t* dE,
                        int64_t* acc);
typedef struct {
    rows_fn fn;
    void* ctx;
    uint32_t colour;
    int64_t r0, r1, dE, acc;
} rows_job;

static void* rows_worker(void* p) {
    rows_job* j = (rows_job*)p;
    j->fn(j->ctx, j->colour, j->r0, j->r1, &j->dE, &j->acc);
    return NULL;
}

static void run_rows(rows_fn fn, void* ctx, uint32_t colour, int64_t nrows, int64_t* dE,
                     int64_t* acc) {
    int nt = g_threads;
    if (nt > nrows) nt = (int)nrows;
    if (nt <= 1) {
        int64_t d = 0, a = 0;
        fn(ctx, colour, 0, nrows, &d, &a);
        *dE += d;
        *acc += a;
        return;
    }
    rows_job jobs[256];
    pthread_t th[256];
    for (int t = 0; t < nt; ++t) {
        rows_job j = {fn, ctx, colour, nrows * t / nt, nrows * (t + 1) / nt, 0, 0};
        jobs[t] = j;
        pthread_create(&th[t], NULL, rows_worker, &jobs[t]);
    }
    for (int t = 0; t < nt; ++t) {
        pthread_join(th[t], NULL);
        *dE += jobs[t].dE;
        *acc += jobs[t].acc;
    }
}

/* ------------------------------------------------------------------------ */
/* geometry helpers                                                          */
/* ------------------------------------------------------------------------ */
typedef struct { int dims; int64_t lx, ly, lz; } geom;

static inline int64_t site_of(const geom* g, int64_t x, int64_t y, int64_t z) {
    return x + g->lx * (y + g->ly * z);
}
/* neighbours in the fixed order (x-1, x+1, y-1, y+1[, z-1, z+1]) */
static inline int neighbours(const geom* g, int64_t x, int64_t y, int64_t z, int64_t nb[6]) {
    int64_t xm = x ? x - 1 : g->lx - 1, xp = x + 1 < g->lx ? x + 1 : 0;
    int64_t ym = y ? y - 1 : g->ly - 1, yp = y + 1 < g->ly ? y + 1 : 0;
    nb[0] = site_of(g, xm, y, z);
    nb[1] = site_of(g, xp, y, z);
    nb[2] = site_of(g, x, ym, z);
    nb[3] = site_of(g, x, yp, z);
    if (g->dims == 2) return 4;
    int64_t zm = z ? z - 1 : g->lz - 1, zp = z + 1 < g->lz ? z + 1 : 0;
    nb[4] = site_of(g, x, y, zm);
    nb[5] = site_of(g, x, y, zp);
    return 6;
}
static inline void make_ctr(uint32_t ctr[4], uint64_t index, uint32_t colour, uint32_t tag,
                            uint32_t plane_pair, uint64_t sweep) {
    ctr[0] = (uint32_t)index;
    ctr[1] = colour | (tag << 1) | (plane_pair << 8) | ((uint32_t)(index >> 32) << 16);
    ctr[2] = (uint32_t)sweep;
    ctr[3] = (uint32_t)(sweep >> 32);
}
static inline void key_of(uint64_t k64, uint32_t key[2]) {
    key[0] = (uint32_t)k64;
    key[1] = (uint32_t)(k64 >> 32);
}

/* 16-bit draw of a site from the 16-site chunk batch (x & 15 selects slot) */
static uint32_t chunk_u16(const geom* g, int64_t x, int64_t y, int64_t z, uint32_t colour,
                          uint32_t tag, const uint32_t key[2], uint64_t sweep) {
    int64_t pc = (g->lx + 15) / 16;
    uint64_t chunk = (uint64_t)((y + g->ly * z) * pc + (x >> 4));
    uint32_t ctr[4], out[4];
    make_ctr(ctr, chunk, colour, tag, 0, sweep);
    orc_philox4x32_10(ctr, key, out);
    int slot = (int)((x & 15) >> 1);
    return (out[slot >> 1] >> (16 * (slot & 1))) & 0xFFFFu;
}

static int accept_discrete(uint32_t u16, uint32_t head, uint64_t tail, uint64_t site,
                           uint32_t colour, const uint32_t key[2], uint64_t sweep) {
    if (u16 < head) return 1;
    if (u16 > head) return 0;
    uint32_t ctr[4], out[4];
    make_ctr(ctr, site, colour, ORC_TAG_ACC_REFINE, 0, sweep);
    orc_philox4x32_10(ctr, key, out);
    uint64_t r = (uint64_t)out[0] | ((uint64_t)out[1] << 32);
    return r < tail;
}

/* Ising decision on bit planes of the site's 64-site row segment */
static int accept_bits(const geom* g, int64_t x, int64_t y, int64_t z, uint32_t head,
                       uint64_t tail, uint32_t colour, const uint32_t key[2], uint64_t sweep) {
    if (head >= 65536u) return 1;
    int64_t ps = (g->lx + 63) / 64;
    uint64_t seg = (uint64_t)((y + g->ly * z) * ps + (x >> 6));
    int bit = (int)((x & 63) >> 1);
    uint32_t out[4];
    for (int j = 0; j < 80; ++j) {
        if ((j & 3) == 0) {
            uint32_t ctr[4];
            make_ctr(ctr, seg, colour, ORC_TAG_BITS, (uint32_t)(j >> 2), sweep);
            orc_philox4x32_10(ctr, key, out);
        }
        int ub = (int)((out[j & 3] >> bit) & 1u);
        int tb = j < 16 ? (int)((head >> (15 - j)) & 1u) : (int)((tail >> (79 - j)) & 1u);
        if (ub != tb) return ub < tb;
    }
    return 0;
}

/* Heat-bath Ising decision on the bit planes (tag HBITS) of the site's
 * segment: u < T, with u's bits complemented when `flip` (the negative-field
 * member of a class pair compares ~u). */
static int hb_bits_below(const geom* g, int64_t x, int64_t y, int64_t z, uint32_t head,
                         uint64_t tail, int flip, uint32_t colour, const uint32_t key[2],
                         uint64_t sweep) {
    int64_t ps = (g->lx + 63) / 64;
    uint64_t seg = (uint64_t)((y + g->ly * z) * ps + (x >> 6));
    int bit = (int)((x & 63) >> 1);
    uint32_t out[4];
    for (int j = 0; j < 80; ++j) {
        if ((j & 3) == 0) {
            uint32_t ctr[4];
            make_ctr(ctr, seg, colour, ORC_TAG_HBITS, (uint32_t)(j >> 2), sweep);
            orc_philox4x32_10(ctr, key, out);
        }
        int ub = (int)((out[j & 3] >> bit) & 1u) ^ (flip ? 1 : 0);
        int tb = j < 16 ? (int)((head >> (15 - j)) & 1u) : (int)((tail >> (79 - j)) & 1u);
        if (ub != tb) return ub < tb;
    }
    return 0;
}

/* first bit of the site's heat-bath uniform (plane 0) */
static int hb_bits_first(const geom* g, int64_t x, int64_t y, int64_t z, uint32_t colour,
                         const uint32_t key[2], uint64_t sweep) {
    int64_t ps = (g->lx + 63) / 64;
    uint64_t seg = (uint64_t)((y + g->ly * z) * ps + (x >> 6));
    uint32_t ctr[4], out[4];
    make_ctr(ctr, seg, colour, ORC_TAG_HBITS, 0, sweep);
    orc_philox4x32_10(ctr, key, out);
    return (int)((out[0] >> ((x & 63) >> 1)) & 1u);
}

/* Potts (q <= 4) on bit planes of the site's 64-site row segment: the
 * proposal v in [0, q-1) (q = 2: 0; q = 3: one bit; q = 4: two bits, v = 3
 * redrawn from the next pair of planes, at most 32 rounds, then 0) and the
 * bit-serial acceptance against the 80-bit threshold of the class. */
static uint64_t potts_segment(const geom* g, int64_t x, int64_t y, int64_t z) {
    int64_t ps = (g->lx + 63) / 64;
    return (uint64_t)((y + g->ly * z) * ps + (x >> 6));
}

static uint32_t potts_bits_proposal(const geom* g, int64_t x, int64_t y, int64_t z, int q,
                                    uint32_t colour, const uint32_t key[2], uint64_t sweep) {
    if (q == 2) return 0;
    uint64_t seg = potts_segment(g, x, y, z);
    int bit = (int)((x & 63) >> 1);
    uint32_t ctr[4], out[4];
    if (q == 3) {
        make_ctr(ctr, seg, colour, ORC_TAG_PBITS, 0, sweep);
        orc_philox4x32_10(ctr, key, out);
        return (out[0] >> bit) & 1u;
    }
    for (int r = 0; r < 32; ++r) {
        if ((r & 1) == 0) {
            make_ctr(ctr, seg, colour, ORC_TAG_PBITS, (uint32_t)(r >> 1), sweep);
            orc_philox4x32_10(ctr, key, out);
        }
        uint32_t b0 = (out[2 * (r & 1)] >> bit) & 1u, b1 = (out[2 * (r & 1) + 1] >> bit) & 1u;
        uint32_t v = 2 * b1 + b0;
        if (v < 3) return v;
    }
    return 0;
}

static int potts_bits_accept(const geom* g, int64_t x, int64_t y, int64_t z, uint32_t head,
                             uint64_t tail, uint32_t colour, const uint32_t key[2], uint64_t sweep) {
    if (head >= 65536u) return 1;
    uint64_t seg = potts_segment(g, x, y, z);
    int bit = (int)((x & 63) >> 1);
    uint32_t out[4];
    for (int j = 0; j < 80; ++j) {
        if ((j & 3) == 0) {
            uint32_t ctr[4];
            make_ctr(ctr, seg, colour, ORC_TAG_PACC, (uint32_t)(j >> 2), sweep);
            orc_philox4x32_10(ctr, key, out);
        }
        int ub = (int)((out[j & 3] >> bit) & 1u);
        int tb = j < 16 ? (int)((head >> (15 - j)) & 1u) : (int)((tail >> (79 - j)) & 1u);
        if (ub != tb) return ub < tb;
    }
    return 0;
}

/* uniform r in [0, n) for the Potts proposal, Lemire multiply-shift with
 * exact rejection (16-bit first draw, 32-bit retries from a refine batch) */
static uint32_t potts_draw(uint32_t u16, uint32_t n, uint64_t site, uint32_t colour,
                           const uint32_t key[2], uint64_t sweep) {
    uint32_t m = u16 * n;
    uint32_t low = m & 0xFFFFu;
    uint32_t reject16 = 65536u % n;
    if (low >= reject16) return m >> 16;
    uint32_t ctr[4], out[4];
    make_ctr(ctr, site, colour, ORC_TAG_PROP_REFINE, 0, sweep);
    orc_philox4x32_10(ctr, key, out);
    uint32_t reject32 = (uint32_t)((0x100000000ull) % n);
    uint64_t mm = 0;
    for (int i = 0; i < 4; ++i) {
        mm = (uint64_t)out[i] * n;
        if ((uint32_t)mm >= reject32) return (uint32_t)(mm >> 32);
    }
    return (uint32_t)(mm >> 32);
}

/* ------------------------------------------------------------------------ */
/* discrete models                                                           */
/* ------------------------------------------------------------------------ */
void orc_init_discrete(int model, int dims, int64_t lx, int64_t ly, int64_t lz, int q,
                       uint64_t base_seed, uint64_t replica, int hot, int8_t* spins) {
    int64_t n = lx * ly * (dims == 3 ? lz : 1);
    if (!hot) {
        memset(spins, model == ORC_ISING ? 1 : 0, (size_t)n);
        return;
    }
    uint32_t key[2];
    key_of(orc_replica_key(base_seed, replica, ORC_SUB_INIT), key);
    for (int64_t s = 0; s < n; ++s) {
        uint32_t ctr[4], out[4];
        make_ctr(ctr, (uint64_t)s >> 2, 0, ORC_TAG_INIT, 0, 0);
        orc_philox4x32_10(ctr, key, out);
        uint32_t u = out[s & 3];
        if (model == ORC_ISING)
            spins[s] = (u >> 31) ? 1 : -1;
        else
            spins[s] = (int8_t)(((uint64_t)u * (uint64_t)q) >> 32);
    }
}

typedef struct {
    int model, q, zc, potts_bits;
    geom g;
    const uint32_t* head;
    const uint64_t* tail;
    uint32_t key[2];
    uint64_t sweep;
    int8_t* spins;
} discrete_ctx;

static void discrete_rows(void* p, uint32_t colour, int64_t r0, int64_t r1, int64_t* dE_out,
                          int64_t* acc_out) {
    const discrete_ctx* c = (const discrete_ctx*)p;
    const geom* g = &c->g;
    const int model = c->model, q = c->q, zc = c->zc;
    const uint32_t* head = c->head;
    const uint64_t* tail = c->tail;
    const uint32_t* key = c->key;
    const uint64_t sweep = c->sweep;
    int8_t* spins = c->spins;
    int64_t dE = 0, acc = 0;
    for (int64_t rho = r0; rho < r1; ++rho) {
        const int64_t z = rho / g->ly, y = rho % g->ly;
        for (int64_t x = 0; x < g->lx; ++x) {
            if ((uint32_t)((x + y + z) & 1) != colour) continue;
            int64_t site = site_of(g, x, y, z);
            int64_t nb[6];
            int nn = neighbours(g, x, y, z, nb);
            int8_t s = spins[site];
            if (model == ORC_ISING) {
                int k = 0;
                for (int i = 0; i < nn; ++i) k += spins[nb[i]] != s;
                if (accept_bits(g, x, y, z, head[k], tail[k], colour, key, sweep)) {
                    spins[site] = (int8_t)-s;
                    dE += 2 * (zc - 2 * k);
                    ++acc;
                }
            } else if (c->potts_bits) {
                uint32_t v = potts_bits_proposal(g, x, y, z, q, colour, key, sweep);
                int8_t t = (int8_t)((int)v < s ? (int)v : (int)v + 1);
                int nold = 0, nnew = 0;
                for (int i = 0; i < nn; ++i) {
                    nold += spins[nb[i]] == s;
                    nnew += spins[nb[i]] == t;
                }
                int d = nnew - nold;
                if (potts_bits_accept(g, x, y, z, head[d + zc], tail[d + zc], colour, key, sweep)) {
                    spins[site] = t;
                    dE += -d;
                    ++acc;
                }
            } else {
                uint32_t u = chunk_u16(g, x, y, z, colour, ORC_TAG_ACC, key, sweep);
                uint32_t pu = chunk_u16(g, x, y, z, colour, ORC_TAG_PROP, key, sweep);
                uint32_t r = potts_draw(pu, (uint32_t)(q - 1), (uint64_t)site, colour, key, sweep);
                int8_t t = (int8_t)((int)r < s ? (int)r : (int)r + 1);
                int nold = 0, nnew = 0;
                for (int i = 0; i < nn; ++i) {
                    nold += spins[nb[i]] == s;
                    nnew += spins[nb[i]] == t;
                }
                int d = nnew - nold;
                if (accept_discrete(u, head[d + zc], tail[d + zc], (uint64_t)site, colour, key, sweep)) {
                    spins[site] = t;
                    dE += -d;
                    ++acc;
                }
            }
        }
    }
    *dE_out = dE;
    *acc_out = acc;
}

int64_t orc_sweep_discrete(int model, int dims, int64_t lx, int64_t ly, int64_t lz, int q,
                           const uint32_t* head, const uint64_t* tail, uint64_t key64,
                           uint64_t sweep, int8_t* spins, int64_t* accepted) {
    discrete_ctx c;
    geom g = {dims, lx, ly, dims == 3 ? lz : 1};
    c.model = model;
    c.q = q;
    c.zc = 2 * dims;
    /* Potts on bit planes when q <= 4 and rows are at most 128 segments of 64
     * sites or a whole number of segments; else the 16-bit chunk method */
    c.potts_bits = q <= 4 && ((lx + 63) / 64 <= 128 || lx % 64 == 0);
    c.g = g;
    c.head = head;
    c.tail = tail;
    key_of(key64, c.key);
    c.sweep = sweep;
    c.spins = spins;
    int64_t dE = 0, acc = 0;
    for (uint32_t colour = 0; colour < 2; ++colour)
        run_rows(discrete_rows, &c, colour, g.ly * g.lz, &dE, &acc);
    if (accepted) *accepted = acc;
    return dE;
}

int64_t orc_sweep_discrete_hb(int model, int dims, int64_t lx, int64_t ly, int64_t lz, int q,
                              double J, const uint32_t* head, const uint64_t* tail, uint64_t key64,
                              uint64_t sweep, int8_t* spins, int64_t* changed) {
    geom g = {dims, lx, ly, dims == 3 ? lz : 1};
    int zc = 2 * dims;
    uint32_t key[2];
    key_of(key64, key);
    int64_t dE = 0, nch = 0;
    int64_t pc = (lx + 15) / 16;
    for (uint32_t colour = 0; colour < 2; ++colour) {
        for (int64_t z = 0; z < g.lz; ++z)
            for (int64_t y = 0; y < g.ly; ++y)
                for (int64_t x = 0; x < g.lx; ++x) {
                    if ((uint32_t)((x + y + z) & 1) != colour) continue;
                    int64_t site = site_of(&g, x, y, z);
                    int64_t nb[6];
                    int nn = neighbours(&g, x, y, z, nb);
                    int8_t s = spins[site];
                    if (model == ORC_ISING) {
                        /* k = down neighbours; field h = z - 2k; class pair
                         * {k, z-k} shares T[k] = p(|x|); the member with
                         * negative field compares ~u, zero field is u < 1/2 */
                        int k = 0;
                        for (int i = 0; i < nn; ++i) k += spins[nb[i]] == -1;
                        int up;
                        if (2 * k == zc) {
                            up = hb_bits_first(&g, x, y, z, colour, key, sweep) == 0;
                        } else {
                            int neg = J >= 0.0 ? 2 * k > zc : 2 * k < zc;
                            int lt = hb_bits_below(&g, x, y, z, head[k], tail[k], neg, colour, key,
                                                   sweep);
                            up = neg ? !lt : lt;
                        }
                        int8_t t = up ? 1 : -1;
                        if (t != s) {
                            spins[site] = t;
                            dE += 2 * (int64_t)s * (zc - 2 * k);
                            ++nch;
                        }
                    } else {
                        /* state weights exp(beta J n_t) relative to the site's
                         * favoured count, as 64-bit integers; x = u * total
                         * / 2^64; first state whose cumulative weight
                         * exceeds x */
                        int n[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                        for (int i = 0; i < nn; ++i)
                            if (spins[nb[i]] >= 0 && spins[nb[i]] < q) ++n[spins[nb[i]]];
                        int nmax = 0, nmin = 64;
                        for (int t = 0; t < q; ++t) {
                            if (n[t] > nmax) nmax = n[t];
                            if (n[t] < nmin) nmin = n[t];
                        }
                        uint64_t w[8], tot = 0;
                        for (int t = 0; t < q; ++t) {
                            w[t] = tail[J < 0.0 ? n[t] - nmin : nmax - n[t]];
                            tot += w[t];
                        }
                        uint64_t chunk = (uint64_t)((y + g.ly * z) * pc + (x >> 4));
                        int slot = (int)((x & 15) >> 1);
                        uint32_t ctr[4], out[4];
                        make_ctr(ctr, chunk, colour, ORC_TAG_HB, (uint32_t)(slot >> 1), sweep);
                        orc_philox4x32_10(ctr, key, out);
                        uint64_t u = (slot & 1) ? ((uint64_t)out[2] | ((uint64_t)out[3] << 32))
                                                : ((uint64_t)out[0] | ((uint64_t)out[1] << 32));
                        uint64_t r = (uint64_t)(((unsigned __int128)u * tot) >> 64);
                        int t = q - 1;
                        for (int c = 0; c < q; ++c) {
                            if (r < w[c]) { t = c; break; }
                            r -= w[c];
                        }
                        if (t != s) {
                            spins[site] = (int8_t)t;
                            dE += -(int64_t)(n[t] - n[s]);
                            ++nch;
                        }
                    }
                }
    }
    if (changed) *changed = nch;
    return dE;
}

uint64_t orc_cluster_threshold(int model, double J, double beta) {
    double p = model == ORC_POTTS ? 1.0 - exp(-beta * J) : 1.0 - exp(-2.0 * beta * J);
    p = p < 0.0 ? 0.0 : p;
    return p >= 1.0 ? ~(uint64_t)0 : (uint64_t)ldexp(p, 64);
}

static uint32_t uf_find(uint32_t* par, uint32_t a) {
    while (par[a] != a) {
        par[a] = par[par[a]];
        a = par[a];
    }
    return a;
}

/* the larger root under the smaller: every root is its component's minimum */
static void uf_union(uint32_t* par, uint32_t a, uint32_t b) {
    a = uf_find(par, a);
    b = uf_find(par, b);
    if (a < b) par[b] = a;
    else if (b < a) par[a] = b;
}

/* integer in [0, n) by 32-bit multiply-shift with exact rejection over the
 * four words of a block; 0 if all are rejected */
static uint32_t uniform_below4(const uint32_t w[4], uint32_t n) {
    uint32_t rej = (uint32_t)(0x100000000ull % n);
    for (int i = 0; i < 4; ++i) {
        uint64_t m = (uint64_t)w[i] * n;
        if ((uint32_t)m >= rej) return (uint32_t)(m >> 32);
    }
    return 0;
}

int64_t orc_sweep_cluster(int model, int dims, int64_t lx, int64_t ly, int64_t lz, int q, int wolff,
                          uint64_t thr, uint64_t key64, uint64_t sweep, int8_t* spins, int64_t* changed) {
    geom g = {dims, lx, ly, dims == 3 ? lz : 1};
    int64_t n = lx * ly * g.lz;
    uint32_t key[2];
    key_of(key64, key);
    uint32_t* par = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n);
    int8_t* sn = (int8_t*)malloc((size_t)n);
    for (int64_t i = 0; i < n; ++i) par[i] = (uint32_t)i;
    /* bonds: Philox(site, TAG_SW, plane 0): +x words 0-1, +y words 2-3;
     * plane 1: +z words 0-1 */
    for (int64_t z = 0; z < g.lz; ++z)
        for (int64_t y = 0; y < ly; ++y)
            for (int64_t x = 0; x < lx; ++x) {
                int64_t s = site_of(&g, x, y, z);
                uint32_t ctr[4], o[4], o2[4];
                make_ctr(ctr, (uint64_t)s, 0, ORC_TAG_SW, 0, sweep);
                orc_philox4x32_10(ctr, key, o);
                if (dims == 3) {
                    make_ctr(ctr, (uint64_t)s, 0, ORC_TAG_SW, 1, sweep);
                    orc_philox4x32_10(ctr, key, o2);
                }
                for (int d = 0; d < dims; ++d) {
                    int64_t nb = d == 0 ? site_of(&g, x + 1 < lx ? x + 1 : 0, y, z)
                               : d == 1 ? site_of(&g, x, y + 1 < ly ? y + 1 : 0, z)
                                        : site_of(&g, x, y, z + 1 < g.lz ? z + 1 : 0);
                    uint64_t u = d == 0 ? ((uint64_t)o[0] | ((uint64_t)o[1] << 32))
                               : d == 1 ? ((uint64_t)o[2] | ((uint64_t)o[3] << 32))
                                        : ((uint64_t)o2[0] | ((uint64_t)o2[1] << 32));
                    if (spins[nb] == spins[s] && u < thr) uf_union(par, (uint32_t)s, (uint32_t)nb);
                }
            }
    uint32_t seed_root = 0;
    int8_t target = 0;
    if (wolff) {
        uint32_t ctr[4], o[4];
        make_ctr(ctr, 0, 0, ORC_TAG_WOLFF, 0, sweep);
        orc_philox4x32_10(ctr, key, o);
        uint64_t nn = (uint64_t)n, rej = (0 - nn) % nn, seed = 0;
        uint64_t u[2] = {(uint64_t)o[0] | ((uint64_t)o[1] << 32), (uint64_t)o[2] | ((uint64_t)o[3] << 32)};
        for (int i = 0; i < 2; ++i)
            if (u[i] * nn >= rej) {
                seed = (uint64_t)(((unsigned __int128)u[i] * nn) >> 64);
                break;
            }
        int8_t ss = spins[seed];
        if (model == ORC_ISING) {
            target = (int8_t)-ss;
        } else {
            make_ctr(ctr, 0, 0, ORC_TAG_WOLFF, 1, sweep);
            orc_philox4x32_10(ctr, key, o);
            uint32_t r = uniform_below4(o, (uint32_t)(q - 1));
            target = (int8_t)((int)r < ss ? (int)r : (int)r + 1);
        }
        seed_root = uf_find(par, (uint32_t)seed);
    }
    int64_t nch = 0;
    for (int64_t s = 0; s < n; ++s) {
        uint32_t r = uf_find(par, (uint32_t)s);
        int8_t v;
        if (wolff) {
            v = r == seed_root ? target : spins[s];
        } else {
            uint32_t ctr[4], o[4];
            make_ctr(ctr, r, 0, ORC_TAG_SWFLIP, 0, sweep);
            orc_philox4x32_10(ctr, key, o);
            v = model == ORC_ISING ? ((o[0] >> 31) ? 1 : -1) : (int8_t)uniform_below4(o, (uint32_t)q);
        }
        sn[s] = v;
        nch += v != spins[s];
    }
    int64_t e0 = orc_energy_int(model, dims, lx, ly, lz, spins);
    memcpy(spins, sn, (size_t)n);
    int64_t e1 = orc_energy_int(model, dims, lx, ly, lz, spins);
    free(par);
    free(sn);
    if (changed) *changed = nch;
    return e1 - e0;
}

int64_t orc_energy_int(int model, int dims, int64_t lx, int64_t ly, int64_t lz,
                       const int8_t* spins) {
    geom g = {dims, lx, ly, dims == 3 ? lz : 1};
    int64_t e = 0;
    for (int64_t z = 0; z < g.lz; ++z)
        for (int64_t y = 0; y < g.ly; ++y)
            for (int64_t x = 0; x < g.lx; ++x) {
                int64_t nb[6];
                int nn = neighbours(&g, x, y, z, nb);
                int8_t s = spins[site_of(&g, x, y, z)];
                /* +1 bonds only: entries 1, 3, 5 of the neighbour list */
                for (int i = 1; i < nn; i += 2) {
                    int8_t t = spins[nb[i]];
                    e -= (model == ORC_ISING) ? (int64_t)s * t : (int64_t)(s == t);
                }
            }
    return e;
}

/* ------------------------------------------------------------------------ */
/* O(3): engine arithmetic, one rounding per operation                       */
/* ------------------------------------------------------------------------ */
float orc_exp_neg(float x) {
    if (!(x <= 0.0f)) return 1.0f;
    if (x < -87.0f) return 0.0f;
    float y = x * 0x1.715476p+0f;           /* log2(e) */
    float n = floorf(y + 0.5f);
    float f = y - n;
    float t = f * 0x1.62e430p-1f;           /* ln 2 */
    float p = 0x1.a01a02p-13f;              /* 1/7! ; Horner steps fused (fmaf) */
    p = fmaf(p, t, 0x1.6c16c2p-10f);        /* 1/6! */
    p = fmaf(p, t, 0x1.111112p-7f);         /* 1/5! */
    p = fmaf(p, t, 0x1.555556p-5f);         /* 1/4! */
    p = fmaf(p, t, 0x1.555556p-3f);         /* 1/3! */
    p = fmaf(p, t, 0.5f);
    p = fmaf(p, t, 1.0f);
    p = fmaf(p, t, 1.0f);
    int ni = (int)n;                        /* -126 <= ni <= 0 */
    uint32_t bits = (uint32_t)(ni + 127) << 23;
    float scale;
    memcpy(&scale, &bits, 4);
    return p * scale;
}

void orc_sincos_turn(uint32_t u, float* c, float* s) {
    uint32_t octant = u >> 29;
    float t = (float)((u >> 5) & 0xFFFFFFu) * 0x1p-24f;
    if (octant & 1u) t = 1.0f - t;
    float th = t * 0x1.921fb6p-1f;          /* pi / 4 */
    float t2 = th * th;
    float sp = 0x1.71de3ap-19f;             /* 1/9! ; Horner steps fused (fmaf) */
    sp = fmaf(sp, t2, -0x1.a01a02p-13f);    /* 1/7! */
    sp = fmaf(sp, t2, 0x1.111112p-7f);      /* 1/5! */
    sp = fmaf(sp, t2, -0x1.555556p-3f);     /* 1/3! */
    sp = fmaf(sp, t2, 1.0f);
    float sn = th * sp;
    float cp = -0x1.27e4fcp-22f;            /* -1/10! */
    cp = fmaf(cp, t2, 0x1.a01a02p-16f);     /* 1/8! */
    cp = fmaf(cp, t2, -0x1.6c16c2p-10f);    /* 1/6! */
    cp = fmaf(cp, t2, 0x1.555556p-5f);      /* 1/4! */
    cp = fmaf(cp, t2, -0.5f);
    float cs = fmaf(cp, t2, 1.0f);
    float rc, rs;
    switch (octant) {
        case 0: rc = cs;  rs = sn;  break;
        case 1: rc = sn;  rs = cs;  break;
        case 2: rc = -sn; rs = cs;  break;
        case 3: rc = -cs; rs = sn;  break;
        case 4: rc = -cs; rs = -sn; break;
        case 5: rc = -sn; rs = -cs; break;
        case 6: rc = sn;  rs = -cs; break;
        default: rc = cs; rs = -sn; break;
    }
    *c = rc;
    *s = rs;
}

void orc_init_o3(int dims, int64_t lx, int64_t ly, int64_t lz, uint64_t base_seed,
                 uint64_t replica, int hot, float* sx, float* sy, float* sz) {
    int64_t n = lx * ly * (dims == 3 ? lz : 1);
    uint32_t key[2];
    key_of(orc_replica_key(base_seed, replica, ORC_SUB_INIT), key);
    for (int64_t s = 0; s < n; ++s) {
        if (!hot) { sx[s] = 1.0f; sy[s] = 0.0f; sz[s] = 0.0f; continue; }
        uint32_t ctr[4], out[4];
        make_ctr(ctr, (uint64_t)s, 0, ORC_TAG_INIT, 0, 0);
        orc_philox4x32_10(ctr, key, out);
        float t = (float)(out[0] >> 8) * 0x1p-24f;
        float zz = 1.0f - 2.0f * t;
        float r = sqrtf((1.0f - zz) * (1.0f + zz));
        float c, sn;
        orc_sincos_turn(out[1], &c, &sn);
        sx[s] = r * c;
        sy[s] = r * sn;
        sz[s] = zz;
    }
}

double orc_sweep_o3(int dims, int64_t lx, int64_t ly, int64_t lz, float J, float beta,
                    float omc, uint64_t key64, uint64_t sweep, float* sx, float* sy,
                    float* sz, int64_t* accepted) {
    return orc_sweep_o3_prop(dims, lx, ly, lz, J, beta, omc, 0, key64, sweep, sx, sy, sz, accepted);
}

/* ---- O(3) Metropolis arithmetic of the sweep kernels ----------------------
 * Uniforms are built from bits, not by integer-to-float conversion:
 * unit23(u) = 1.m - 1 with the top 23 bits of u as m (multiples of 2^-23 in
 * [0, 1)), half23(u) = unit23(u) + 2^-24 (in (0, 1)); both exact.  Products
 * are fused where the kernel fuses them (fmaf: one rounding, as the device's
 * fma.rn), every other operation is one IEEE rounding. */
static inline float bits_f(uint32_t b) { float f; memcpy(&f, &b, 4); return f; }
static inline uint32_t f_bits(float f) { uint32_t b; memcpy(&b, &f, 4); return b; }
float orc_unit23(uint32_t u) { return bits_f(0x3F800000u | (u >> 9)) - 1.0f; }
float orc_half23(uint32_t u) { return bits_f(0x3F800000u | (u >> 9)) - 0x1.fffffep-1f; }

/* The three draw words of one O(3) site from two Philox words u, v: the top
 * 21 bits of u and of v (low bits zero), and the two low 11-bit fields
 * joined into the top 22 bits of the third word. */
void orc_o3_split(uint32_t u, uint32_t v, uint32_t o[4]) {
    o[0] = u & ~0x7FFu;
    o[1] = v & ~0x7FFu;
    o[2] = (u << 21) | ((v & 0x7FFu) << 10);
    o[3] = 0;
}

/* The draw of an O(3) site update: one Philox call per pair of sites of the
 * colour adjacent in a row (x0 = 4m + parity and x0 + 2, the sweep kernels'
 * unit of work), counter (x0's site, colour | tag << 1, sweep); the pair's
 * first site takes words 0-1, the second words 2-3 (orc_o3_split). */
static void o3_site_draw(const geom* g, int64_t x, int64_t y, int64_t z, uint32_t colour, uint32_t tag,
                         const uint32_t key[2], uint64_t sweep, uint32_t o[4]) {
    int64_t lane = (x >> 1) & 1;
    uint32_t ctr[4], w[4];
    make_ctr(ctr, (uint64_t)site_of(g, x - 2 * lane, y, z), colour, tag, 0, sweep);
    orc_philox4x32_10(ctr, key, w);
    orc_o3_split(w[2 * lane], w[2 * lane + 1], o);
}

/* (cos, sin) of 2 pi u / 2^32: octant from the top 3 bits, the next 23 bits
 * as the fraction t of the octant, Taylor polynomials of degree 9 / 10 on
 * [0, pi/4] (Horner, fused), swaps and signs by octant. */
void orc_sincos23(uint32_t u, float* c, float* s) {
    uint32_t octant = u >> 29;
    float t = bits_f(0x3F800000u | ((u >> 6) & 0x7FFFFFu)) - 1.0f;
    if (octant & 1u) t = 1.0f - t;
    float th = t * 0x1.921fb6p-1f;          /* pi / 4 */
    float t2 = th * th;
    float sp = 0x1.71de3ap-19f;
    sp = fmaf(sp, t2, -0x1.a01a02p-13f);
    sp = fmaf(sp, t2, 0x1.111112p-7f);
    sp = fmaf(sp, t2, -0x1.555556p-3f);
    sp = fmaf(sp, t2, 1.0f);
    float sn = th * sp;
    float cp = -0x1.27e4fcp-22f;
    cp = fmaf(cp, t2, 0x1.a01a02p-16f);
    cp = fmaf(cp, t2, -0x1.6c16c2p-10f);
    cp = fmaf(cp, t2, 0x1.555556p-5f);
    cp = fmaf(cp, t2, -0.5f);
    float cs = fmaf(cp, t2, 1.0f);
    int sw = ((octant + 1u) & 2u) != 0u;
    float a = sw ? sn : cs, b = sw ? cs : sn;
    *c = ((octant + 2u) & 4u) ? -a : a;
    *s = (octant & 4u) ? -b : b;
}

/* exp(x) for -87 <= x <= 0 (smaller x are clamped to -87, where the result is
 * below every acceptance draw): x log2(e) = n + f with n = rint by the
 * 1.5 * 2^23 shifter, f in [-1/2, 1/2], e^(f ln 2) by the degree-7 Taylor
 * polynomial (fused Horner), times 2^n. */
float orc_exp_neg2(float x) {
    if (x < -87.0f) x = -87.0f;
    float y = x * 0x1.715476p+0f;
    float r = y + 0x1.8p23f;
    float n = r - 0x1.8p23f;
    int ni = (int)f_bits(r) - 0x4B400000;
    float t = (y - n) * 0x1.62e430p-1f;
    float p = 0x1.a01a02p-13f;
    p = fmaf(p, t, 0x1.6c16c2p-10f);
    p = fmaf(p, t, 0x1.111112p-7f);
    p = fmaf(p, t, 0x1.555556p-5f);
    p = fmaf(p, t, 0x1.555556p-3f);
    p = fmaf(p, t, 0.5f);
    p = fmaf(p, t, 1.0f);
    p = fmaf(p, t, 1.0f);
    return p * bits_f((uint32_t)(ni + 127) << 23);
}

static void o3_renorm2(float* px, float* py, float* pz) {
    float n2 = fmaf(*pz, *pz, fmaf(*py, *py, *px * *px));
    float f = fmaf(-0.5f, n2, 1.5f);
    *px = *px * f; *py = *py * f; *pz = *pz * f;
}

/* Proposal of the Metropolis step from the site's draw o: 0 the cap of
 * 1 - cos(alpha) = omc around a (Duff et al. 2017 basis), 1 a uniform unit
 * vector (StandardStrategy), 2 a rotation by theta = omc (2u - 1) in plane
 * floor(3 o0 / 2^32) (OPSSStrategy). */
void orc_o3_propose(int prop, float ax, float ay, float az, const uint32_t o[4], float omc,
                    float* nx, float* ny, float* nz) {
    float px, py, pz;
    if (prop == 0) {
        float w = orc_unit23(o[0]) * omc;
        float ct = 1.0f - w;
        float st = sqrtf(fmaf(-w, w, w + w));
        float cp, sp;
        orc_sincos23(o[1], &cp, &sp);
        float vx = st * cp, vy = st * sp;
        float sg = az >= 0.0f ? 1.0f : -1.0f;
        float k = -1.0f / (sg + az);
        float axk = ax * k;
        float b = ay * axk;
        float sax = sg * ax;
        float e1x = fmaf(sax, axk, 1.0f), e1y = sg * b, e1z = -sax;
        float e2x = b, e2y = fmaf(ay * k, ay, sg), e2z = -ay;
        px = fmaf(ct, ax, fmaf(vy, e2x, vx * e1x));
        py = fmaf(ct, ay, fmaf(vy, e2y, vx * e1y));
        pz = fmaf(ct, az, fmaf(vy, e2z, vx * e1z));
    } else if (prop == 1) {
        pz = fmaf(-2.0f, orc_unit23(o[0]), 1.0f);
        float rho = sqrtf(fmaf(-pz, pz, 1.0f));
        float cp, sp;
        orc_sincos23(o[1], &cp, &sp);
        px = rho * cp;
        py = rho * sp;
    } else {
        uint32_t plane = (uint32_t)(((uint64_t)o[0] * 3u) >> 32);
        float theta = omc * fmaf(2.0f, orc_half23(o[1]), -1.0f);
        float turns = theta * 0x1.45f306p-3f;
        uint32_t tu = (uint32_t)(int64_t)llrintf(turns * 0x1p32f);
        float c, sn;
        orc_sincos23(tu, &c, &sn);
        float a0 = plane == 0 ? ax : (plane == 1 ? ay : az);
        float a1 = plane == 0 ? ay : (plane == 1 ? az : ax);
        float r0 = fmaf(c, a0, -(sn * a1)), r1 = fmaf(sn, a0, c * a1);
        px = plane == 0 ? r0 : (plane == 1 ? ax : r1);
        py = plane == 0 ? r1 : (plane == 1 ? r0 : ay);
        pz = plane == 0 ? az : (plane == 1 ? r1 : r0);
    }
    o3_renorm2(&px, &py, &pz);
    *nx = px; *ny = py; *nz = pz;
}

/* Decision: dE = -J (p - a) . h (fused); accept when dE <= 0, else when
 * half23(o2) < exp(-beta dE). */
int orc_o3_accept(float ax, float ay, float az, float px, float py, float pz, float hx, float hy,
                  float hz, float mJ, float beta, uint32_t o2) {
    float dot = fmaf(pz - az, hz, fmaf(py - ay, hy, (px - ax) * hx));
    float de = mJ * dot;
    if (de <= 0.0f) return 1;
    return orc_half23(o2) < orc_exp_neg2(-(beta * de));
}

/* Fixed-point observables of an O(3) configuration as the sweep kernels
 * accumulate them: every site's components as rint(s 2^21), and for every
 * site of colour 1 the bond sum rint(2^19 s . h) with h its fp32 neighbour
 * sum (order x-1, x+1, y-1, y+1, z-1, z+1) and the dot fused; integer sums,
 * so the order of accumulation does not matter.  Every bond has exactly one
 * colour-1 end: energy = -J 2^-19 sum. */
void orc_o3_fixed_observables(int dims, int64_t lx, int64_t ly, int64_t lz, double J, const float* sx,
                              const float* sy, const float* sz, double* energy, double m[3]) {
    geom g = {dims, lx, ly, dims == 3 ? lz : 1};
    int64_t eq = 0, mq[3] = {0, 0, 0};
    for (int64_t z = 0; z < g.lz; ++z)
        for (int64_t y = 0; y < g.ly; ++y)
            for (int64_t x = 0; x < g.lx; ++x) {
                int64_t site = site_of(&g, x, y, z);
                float v[3] = {sx[site], sy[site], sz[site]};
                for (int c = 0; c < 3; ++c)
                    mq[c] += (int32_t)(f_bits(fmaf(v[c], 0x1p21f, 0x1.8p23f)) - 0x4B400000u);
                if (((x + y + z) & 1) != 1) continue;
                int64_t nb[6];
                int nn = neighbours(&g, x, y, z, nb);
                float hx = sx[nb[0]], hy = sy[nb[0]], hz = sz[nb[0]];
                for (int i = 1; i < nn; ++i) {
                    hx = hx + sx[nb[i]];
                    hy = hy + sy[nb[i]];
                    hz = hz + sz[nb[i]];
                }
                float e = fmaf(v[2], hz, fmaf(v[1], hy, v[0] * hx));
                eq += (int32_t)(f_bits(fmaf(e, 0x1p19f, 0x1.8p23f)) - 0x4B400000u);
            }
    *energy = -J * ((double)eq * 0x1p-19);
    for (int c = 0; c < 3; ++c) m[c] = (double)mq[c] * 0x1p-21;
}

double orc_sweep_o3_prop(int dims, int64_t lx, int64_t ly, int64_t lz, float J, float beta,
                         float omc, int prop, uint64_t key64, uint64_t sweep, float* sx, float* sy,
                         float* sz, int64_t* accepted) {
    geom g = {dims, lx, ly, dims == 3 ? lz : 1};
    uint32_t key[2];
    key_of(key64, key);
    double dEsum = 0.0;
    int64_t acc = 0;
    float mJ = -J;
    for (uint32_t colour = 0; colour < 2; ++colour) {
        for (int64_t z = 0; z < g.lz; ++z)
            for (int64_t y = 0; y < g.ly; ++y)
                for (int64_t x = 0; x < g.lx; ++x) {
                    if ((uint32_t)((x + y + z) & 1) != colour) continue;
                    int64_t site = site_of(&g, x, y, z);
                    int64_t nb[6];
                    int nn = neighbours(&g, x, y, z, nb);
                    float hx = sx[nb[0]], hy = sy[nb[0]], hz = sz[nb[0]];
                    for (int i = 1; i < nn; ++i) {
                        hx = hx + sx[nb[i]];
                        hy = hy + sy[nb[i]];
                        hz = hz + sz[nb[i]];
                    }
                    float ax = sx[site], ay = sy[site], az = sz[site];
                    uint32_t o[4];
                    o3_site_draw(&g, x, y, z, colour, ORC_TAG_O3, key, sweep, o);
                    float nx, ny, nz;
                    orc_o3_propose(prop, ax, ay, az, o, omc, &nx, &ny, &nz);
                    if (orc_o3_accept(ax, ay, az, nx, ny, nz, hx, hy, hz, mJ, beta, o[2])) {
                        /* the reference's energy cache: exact fp64 change of
                         * the fp32 configuration */
                        double hxd = 0.0, hyd = 0.0, hzd = 0.0;
                        for (int i = 0; i < nn; ++i) {
                            hxd += (double)sx[nb[i]];
                            hyd += (double)sy[nb[i]];
                            hzd += (double)sz[nb[i]];
                        }
                        dEsum += -(double)J * (((double)nx - (double)ax) * hxd +
                                               ((double)ny - (double)ay) * hyd +
                                               ((double)nz - (double)az) * hzd);
                        sx[site] = nx; sy[site] = ny; sz[site] = nz;
                        ++acc;
                    }
                }
    }
    if (accepted) *accepted = acc;
    return dEsum;
}

/* 1 - exp(-x), x >= 0: Taylor series x (1 - x/2 + ... + x^8/9!) below 1/2
 * (Horner steps fused), else 1 - exp_neg(-x). */
float orc_one_minus_exp_neg(float x) {
    if (x < 0.5f) {
        float p = 0x1.71de3ap-19f;              /* 1/9! */
        p = fmaf(p, x, -0x1.a01a02p-16f);       /* -1/8! */
        p = fmaf(p, x, 0x1.a01a02p-13f);        /* 1/7! */
        p = fmaf(p, x, -0x1.6c16c2p-10f);       /* -1/6! */
        p = fmaf(p, x, 0x1.111112p-7f);         /* 1/5! */
        p = fmaf(p, x, -0x1.555556p-5f);        /* -1/4! */
        p = fmaf(p, x, 0x1.555556p-3f);         /* 1/3! */
        p = fmaf(p, x, -0.5f);
        p = fmaf(p, x, 1.0f);
        return x * p;
    }
    return 1.0f - orc_exp_neg(-x);
}

/* 2 atanh(s), |s| <= 0.1716: 2 s (1 + s^2/3 + ... + s^10/11) */
static float two_atanh_small(float s) {
    float s2 = s * s;
    float q = 0x1.745d18p-4f;                   /* 1/11 */
    q = fmaf(q, s2, 0x1.c71c72p-4f);            /* 1/9 */
    q = fmaf(q, s2, 0x1.24924ap-3f);            /* 1/7 */
    q = fmaf(q, s2, 0x1.99999ap-3f);            /* 1/5 */
    q = fmaf(q, s2, 0x1.555556p-2f);            /* 1/3 */
    q = fmaf(q, s2, 1.0f);
    return (2.0f * s) * q;
}

/* ln(1 - y), 0 <= y < 1: from y directly below 1/4, else from z = 1 - y =
 * m 2^e, m in [sqrt(1/2), sqrt(2)]: e ln 2 + 2 atanh((m - 1) / (m + 1)) */
float orc_log_one_minus(float y) {
    if (y < 0.25f) return two_atanh_small(-y / (2.0f - y));
    float z = 1.0f - y;
    uint32_t bits;
    memcpy(&bits, &z, 4);
    int e = (int)(bits >> 23) - 127;
    uint32_t mb = (bits & 0x7FFFFFu) | 0x3F800000u;
    float m;
    memcpy(&m, &mb, 4);
    if (m > 0x1.6a09e6p+0f) {                   /* sqrt(2) */
        m = m * 0.5f;
        e += 1;
    }
    float sm = (m - 1.0f) / (m + 1.0f);
    return (float)e * 0x1.62e430p-1f + two_atanh_small(sm);
}

double orc_sweep_o3_hb(int dims, int64_t lx, int64_t ly, int64_t lz, float J, float beta,
                       uint64_t key64, uint64_t sweep, float* sx, float* sy, float* sz,
                       int64_t* changed) {
    geom g = {dims, lx, ly, dims == 3 ? lz : 1};
    uint32_t key[2];
    key_of(key64, key);
    double dEsum = 0.0;
    int64_t nch = 0;
    for (uint32_t colour = 0; colour < 2; ++colour) {
        for (int64_t z = 0; z < g.lz; ++z)
            for (int64_t y = 0; y < g.ly; ++y)
                for (int64_t x = 0; x < g.lx; ++x) {
                    if ((uint32_t)((x + y + z) & 1) != colour) continue;
                    int64_t site = site_of(&g, x, y, z);
                    int64_t nb[6];
                    int nn = neighbours(&g, x, y, z, nb);
                    float hx = sx[nb[0]], hy = sy[nb[0]], hz = sz[nb[0]];
                    for (int i = 1; i < nn; ++i) {
                        hx = hx + sx[nb[i]];
                        hy = hy + sy[nb[i]];
                        hz = hz + sz[nb[i]];
                    }
                    uint32_t o[4];
                    o3_site_draw(&g, x, y, z, colour, ORC_TAG_O3HB, key, sweep, o);
                    /* w = 1 - cos(theta) by the inverse CDF of exp(kappa cos) */
                    float fx = J * hx, fy = J * hy, fz = J * hz;
                    float nrm = sqrtf((fx * fx + fy * fy) + fz * fz);
                    float kap = beta * nrm;
                    float v = (float)(o[0] >> 8) * 0x1p-24f;
                    float w, ax = 0.0f, ay = 0.0f, az = 1.0f;
                    if (!(kap >= 0x1p-20f)) {
                        w = 2.0f * v;                    /* uniform on the sphere */
                    } else {
                        float yv = v * orc_one_minus_exp_neg(2.0f * kap);
                        w = -orc_log_one_minus(yv) / kap;
                        if (w > 2.0f) w = 2.0f;
                        ax = fx / nrm;
                        ay = fy / nrm;
                        az = fz / nrm;
                    }
                    float ct = 1.0f - w;
                    float st = sqrtf(w * (2.0f - w));
                    float cp, sp;
                    orc_sincos_turn(o[1], &cp, &sp);
                    /* placed around the field direction with the Duff et al.
                     * (2017) basis and one Newton renormalisation, as the
                     * cap proposal */
                    float vx = st * cp, vy = st * sp;
                    float sg = az >= 0.0f ? 1.0f : -1.0f;
                    float k = -1.0f / (sg + az);
                    float b = (ax * ay) * k;
                    float e1x = 1.0f + (sg * (ax * ax)) * k;
                    float e1y = sg * b;
                    float e1z = -(sg * ax);
                    float e2x = b;
                    float e2y = sg + (ay * ay) * k;
                    float e2z = -ay;
                    float nx = (vx * e1x + vy * e2x) + ct * ax;
                    float ny = (vx * e1y + vy * e2y) + ct * ay;
                    float nz = (vx * e1z + vy * e2z) + ct * az;
                    float n2 = (nx * nx + ny * ny) + nz * nz;
                    float f = 1.5f - 0.5f * n2;
                    nx = nx * f; ny = ny * f; nz = nz * f;
                    float ox = sx[site], oy = sy[site], oz = sz[site];
                    if (nx != ox || ny != oy || nz != oz) {
                        double hxd = 0.0, hyd = 0.0, hzd = 0.0;
                        for (int i = 0; i < nn; ++i) {
                            hxd += (double)sx[nb[i]];
                            hyd += (double)sy[nb[i]];
                            hzd += (double)sz[nb[i]];
                        }
                        dEsum += -(double)J * (((double)nx - (double)ox) * hxd +
                                               ((double)ny - (double)oy) * hyd +
                                               ((double)nz - (double)oz) * hzd);
                        sx[site] = nx; sy[site] = ny; sz[site] = nz;
                        ++nch;
                    }
                }
    }
    if (changed) *changed = nch;
    return dEsum;
}

double orc_sweep_cluster_o3(int dims, int64_t lx, int64_t ly, int64_t lz, float J, float beta, int wolff,
                            uint64_t key64, uint64_t sweep, float* sx, float* sy, float* sz, int64_t* changed) {
    geom g = {dims, lx, ly, dims == 3 ? lz : 1};
    int64_t n = lx * ly * g.lz;
    uint32_t key[2];
    key_of(key64, key);
    /* reflection axis of the sweep */
    uint32_t ctr[4], o[4];
    make_ctr(ctr, 0, 0, ORC_TAG_O3CL, 0, sweep);
    orc_philox4x32_10(ctr, key, o);
    float t = (float)(o[0] >> 8) * 0x1p-24f;
    float rz = 1.0f - 2.0f * t;
    float rho = sqrtf((1.0f - rz) * (1.0f + rz));
    float c, s;
    orc_sincos_turn(o[1], &c, &s);
    float rx = rho * c, ry = rho * s;
    float c2bj = (2.0f * beta) * J;
    uint32_t* par = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n);
    float* sig = (float*)malloc(sizeof(float) * (size_t)n);
    for (int64_t i = 0; i < n; ++i) {
        par[i] = (uint32_t)i;
        sig[i] = (sx[i] * rx + sy[i] * ry) + sz[i] * rz;
    }
    for (int64_t z = 0; z < g.lz; ++z)
        for (int64_t y = 0; y < ly; ++y)
            for (int64_t x = 0; x < lx; ++x) {
                int64_t st = site_of(&g, x, y, z);
                uint32_t o1[4], o2[4];
                make_ctr(ctr, (uint64_t)st, 0, ORC_TAG_SW, 0, sweep);
                orc_philox4x32_10(ctr, key, o1);
                make_ctr(ctr, (uint64_t)st, 0, ORC_TAG_SW, 1, sweep);
                orc_philox4x32_10(ctr, key, o2);
                for (int d = 0; d < dims; ++d) {
                    int64_t nb = d == 0 ? site_of(&g, x + 1 < lx ? x + 1 : 0, y, z)
                               : d == 1 ? site_of(&g, x, y + 1 < ly ? y + 1 : 0, z)
                                        : site_of(&g, x, y, z + 1 < g.lz ? z + 1 : 0);
                    float prod = sig[st] * sig[nb];
                    if (!(prod > 0.0f)) continue;
                    float p = orc_one_minus_exp_neg(c2bj * prod);
                    uint64_t thr = p >= 1.0f ? ~(uint64_t)0 : (uint64_t)((double)p * 18446744073709551616.0);
                    uint64_t u = d == 0 ? ((uint64_t)o1[0] | ((uint64_t)o1[1] << 32))
                               : d == 1 ? ((uint64_t)o1[2] | ((uint64_t)o1[3] << 32))
                                        : ((uint64_t)o2[0] | ((uint64_t)o2[1] << 32));
                    if (u < thr) uf_union(par, (uint32_t)st, (uint32_t)nb);
                }
            }
    uint32_t seed_root = 0;
    if (wolff) {
        make_ctr(ctr, 0, 0, ORC_TAG_WOLFF, 0, sweep);
        orc_philox4x32_10(ctr, key, o);
        uint64_t nn = (uint64_t)n, rej = (0 - nn) % nn, seed = 0;
        uint64_t u[2] = {(uint64_t)o[0] | ((uint64_t)o[1] << 32), (uint64_t)o[2] | ((uint64_t)o[3] << 32)};
        for (int i = 0; i < 2; ++i)
            if (u[i] * nn >= rej) {
                seed = (uint64_t)(((unsigned __int128)u[i] * nn) >> 64);
                break;
            }
        seed_root = uf_find(par, (uint32_t)seed);
    }
    float* nx = (float*)malloc(sizeof(float) * (size_t)n);
    float* ny = (float*)malloc(sizeof(float) * (size_t)n);
    float* nz = (float*)malloc(sizeof(float) * (size_t)n);
    int64_t nch = 0;
    for (int64_t i = 0; i < n; ++i) {
        uint32_t r = uf_find(par, (uint32_t)i);
        int refl;
        if (wolff) {
            refl = r == seed_root;
        } else {
            make_ctr(ctr, r, 0, ORC_TAG_SWFLIP, 0, sweep);
            orc_philox4x32_10(ctr, key, o);
            refl = (o[0] >> 31) != 0;
        }
        float vx = sx[i], vy = sy[i], vz = sz[i];
        if (refl) {
            float k = 2.0f * sig[i];
            float px = vx - k * rx, py = vy - k * ry, pz = vz - k * rz;
            float n2 = (px * px + py * py) + pz * pz;
            float f = 1.5f - 0.5f * n2;
            vx = px * f; vy = py * f; vz = pz * f;
        }
        nx[i] = vx; ny[i] = vy; nz[i] = vz;
        nch += (vx != sx[i]) | (vy != sy[i]) | (vz != sz[i]);
    }
    double e0 = orc_energy_o3(dims, lx, ly, lz, (double)J, sx, sy, sz);
    memcpy(sx, nx, sizeof(float) * (size_t)n);
    memcpy(sy, ny, sizeof(float) * (size_t)n);
    memcpy(sz, nz, sizeof(float) * (size_t)n);
    double e1 = orc_energy_o3(dims, lx, ly, lz, (double)J, sx, sy, sz);
    free(par); free(sig); free(nx); free(ny); free(nz);
    if (changed) *changed = nch;
    return e1 - e0;
}

double orc_energy_o3(int dims, int64_t lx, int64_t ly, int64_t lz, double J, const float* sx,
                     const float* sy, const float* sz) {
    geom g = {dims, lx, ly, dims == 3 ? lz : 1};
    double e = 0.0;
    for (int64_t z = 0; z < g.lz; ++z)
        for (int64_t y = 0; y < g.ly; ++y)
            for (int64_t x = 0; x < g.lx; ++x) {
                int64_t nb[6];
                int nn = neighbours(&g, x, y, z, nb);
                int64_t s = site_of(&g, x, y, z);
                for (int i = 1; i < nn; i += 2)
                    e -= J * ((double)sx[s] * sx[nb[i]] + (double)sy[s] * sy[nb[i]] +
                              (double)sz[s] * sz[nb[i]]);
            }
    return e;
}

float orc_opss_adapt(float sigma, int64_t accepted, int64_t attempted) {
    if (attempted <= 0) return sigma;
    float rate = (float)accepted / (float)attempted;
    float x = 0.08f * (rate - 0.5f);
    float f = x <= 0.0f ? orc_exp_neg(x) : 1.0f / orc_exp_neg(-x);
    float s = sigma * f;
    s = s < 1e-4f ? 1e-4f : s;
    s = s > 0x1.921fb6p+1f ? 0x1.921fb6p+1f : s;
    return s;
}

float orc_o3_adapt(float omc, int64_t accepted, int64_t attempted) {
    if (attempted <= 0) return omc;
    float rate = (float)accepted / (float)attempted;
    float f = 1.0f + 0.16f * (rate - 0.5f);
    float w = omc * f;
    const float lo = 5.0e-9f; /* 1 - cos(1e-4) */
    if (w < lo) w = lo;
    if (w > 2.0f) w = 2.0f;
    return w;
}

/* ------------------------------------------------------------------------ */
/* multi-spin coding                                                         */
/* ------------------------------------------------------------------------ */
void orc_init_msc(int dims, int64_t lx, int64_t ly, int64_t lz, uint64_t base_seed, int hot,
                  uint64_t* words) {
    int64_t n = lx * ly * (dims == 3 ? lz : 1);
    if (!hot) {
        for (int64_t s = 0; s < n; ++s) words[s] = ~0ull;
        return;
    }
    memset(words, 0, (size_t)n * 8);
    for (int r = 0; r < 64; ++r) {
        uint32_t key[2];
        key_of(orc_replica_key(base_seed, (uint64_t)r, ORC_SUB_INIT), key);
        for (int64_t s = 0; s < n; ++s) {
            uint32_t ctr[4], out[4];
            make_ctr(ctr, (uint64_t)s >> 2, 0, ORC_TAG_INIT, 0, 0);
            orc_philox4x32_10(ctr, key, out);
            if (out[s & 3] >> 31) words[s] |= 1ull << r;
        }
    }
}

static int t_bit(uint32_t head, uint64_t tail, int j) {
    return j < 16 ? (int)((head >> (15 - j)) & 1u) : (int)((tail >> (79 - j)) & 1u);
}

typedef struct {
    geom g;
    const uint32_t* head;
    const uint64_t* tail;
    uint32_t key[2];
    uint64_t sweep;
    uint64_t* words;
} msc_ctx;

static void msc_rows(void* p, uint32_t colour, int64_t r0, int64_t r1, int64_t* dE_out,
                     int64_t* acc_out) {
    const msc_ctx* c = (const msc_ctx*)p;
    const geom* g = &c->g;
    const uint32_t* head = c->head;
    const uint64_t* tail = c->tail;
    const uint32_t* key = c->key;
    const uint64_t sweep = c->sweep;
    uint64_t* words = c->words;
    int64_t acc = 0;
    for (int64_t rho = r0; rho < r1; ++rho) {
        const int64_t z = rho / g->ly, y = rho % g->ly;
        for (int64_t x = 0; x < g->lx; ++x) {
            if ((uint32_t)((x + y + z) & 1) != colour) continue;
            int64_t site = site_of(g, x, y, z);
            int64_t nb[6];
            int nn = neighbours(g, x, y, z, nb);
            uint64_t w = words[site];
            uint64_t planes[80];
            int have = 0;
            uint64_t flip = 0;
            for (int r = 0; r < 64; ++r) {
                int k = 0;
                for (int i = 0; i < nn; ++i) k += (int)(((w ^ words[nb[i]]) >> r) & 1u);
                if (head[k] >= 65536u) { flip |= 1ull << r; continue; }
                int decided = 0, less = 0;
                for (int j = 0; j < 80 && !decided; ++j) {
                    while (have <= j) {
                        uint32_t ctr[4], out[4];
                        make_ctr(ctr, (uint64_t)site, colour, ORC_TAG_MSC, (uint32_t)(have >> 1), sweep);
                        orc_philox4x32_10(ctr, key, out);
                        planes[have] = (uint64_t)out[0] | ((uint64_t)out[1] << 32);
                        planes[have + 1] = (uint64_t)out[2] | ((uint64_t)out[3] << 32);
                        have += 2;
                    }
                    int ub = (int)((planes[j] >> r) & 1u);
                    int tb = t_bit(head[k], tail[k], j);
                    if (ub != tb) { decided = 1; less = ub < tb; }
                }
                if (less) flip |= 1ull << r;
            }
            words[site] = w ^ flip;
            acc += __builtin_popcountll(flip);
        }
    }
    *dE_out = 0;
    *acc_out = acc;
}

void orc_sweep_msc(int dims, int64_t lx, int64_t ly, int64_t lz, const uint32_t* head,
                   const uint64_t* tail, uint64_t key64, uint64_t sweep, uint64_t* words,
                   int64_t* accepted) {
    msc_ctx c;
    geom g = {dims, lx, ly, dims == 3 ? lz : 1};
    c.g = g;
    c.head = head;
    c.tail = tail;
    key_of(key64, c.key);
    c.sweep = sweep;
    c.words = words;
    int64_t dE = 0, acc = 0;
    for (uint32_t colour = 0; colour < 2; ++colour)
        run_rows(msc_rows, &c, colour, g.ly * g.lz, &dE, &acc);
    if (accepted) *accepted = acc;
}

void orc_msc_observables(int dims, int64_t lx, int64_t ly, int64_t lz, const uint64_t* words,
                         int64_t* e_int, int64_t* m_sum) {
    geom g = {dims, lx, ly, dims == 3 ? lz : 1};
    for (int r = 0; r < 64; ++r) { e_int[r] = 0; m_sum[r] = 0; }
    for (int64_t z = 0; z < g.lz; ++z)
        for (int64_t y = 0; y < g.ly; ++y)
            for (int64_t x = 0; x < g.lx; ++x) {
                int64_t nb[6];
                int nn = neighbours(&g, x, y, z, nb);
                uint64_t w = words[site_of(&g, x, y, z)];
                for (int r = 0; r < 64; ++r) m_sum[r] += ((w >> r) & 1u) ? 1 : -1;
                for (int i = 1; i < nn; i += 2) {
                    uint64_t a = w ^ words[nb[i]];
                    for (int r = 0; r < 64; ++r) e_int[r] += ((a >> r) & 1u) ? 1 : -1;
                }
            }
}

/* ------------------------------------------------------------------------ */
/* replica exchange                                                          */
/* ------------------------------------------------------------------------ */
int orc_accept_log(double logA, uint64_t u64) {
    if (isnan(logA)) return 0;
    if (logA >= 0.0) return 1;
    if (isinf(logA)) return 0;
    double u = (double)(u64 >> 11) * 0x1p-53;
    if (u < 2.2250738585072014e-308) u = 2.2250738585072014e-308;
    return log(u) < logA;
}

int orc_pt_exchange(int n, const double* betas, const double* energies, int32_t* label,
                    uint64_t exchange_key, uint64_t exchange_step, int32_t* accepted_pairs) {
    if (n < 2 || exchange_step == 0) return 0;
    int32_t* at = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    for (int r = 0; r < n; ++r) at[label[r]] = r;
    uint32_t key[2];
    key_of(exchange_key, key);
    int offset = (int)((exchange_step - 1) & 1u);
    int count = 0;
    for (int t = offset; t + 1 < n; t += 2) {
        int a = at[t], b = at[t + 1];
        double wa = (betas[t] - betas[t + 1]) * energies[a];
        double wb = (betas[t + 1] - betas[t]) * energies[b];
        uint32_t ctr[4], out[4];
        make_ctr(ctr, (uint64_t)t, 0, ORC_TAG_PT, 0, exchange_step);
        orc_philox4x32_10(ctr, key, out);
        uint64_t u = (uint64_t)out[0] | ((uint64_t)out[1] << 32);
        int ok = orc_accept_log(wa + wb, u);
        if (accepted_pairs) accepted_pairs[t] = ok;
        if (ok) {
            label[a] = t + 1;
            label[b] = t;
            at[t] = b;
            at[t + 1] = a;
            ++count;
        }
    }
    free(at);
    return count;
}
