/* TEST INFRASTRUCTURE ONLY: CPU restatement of the reference SCA golden model (the checker; never shipped).
 * Each function cites the reference lines it restates (paths relative to the reference project root).
 * Parity status: pinned for n <= 2048 by tests/golden (generated by the reference itself); n > 2048 uses this
 * project's slot generalisation (orc_np) and is not pinned by the reference. */
#include "sca_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define ORC_LANES 256

int orc_np(int n) {
    int np = ((n + ORC_LANES - 1) / ORC_LANES) * ORC_LANES;
    return np < 2048 ? 2048 : np;
}

/* Floor division by 2^k of a signed 64-bit value (the reference relies on an arithmetic >>, sca_ref.hpp:128). */
static int64_t floor_shift(int64_t v, int k) { return v >= 0 ? (v >> k) : ~((~v) >> k); }

/* ---- tables: restates v80host::geom/build_tables (tables.hpp:14-40), sca::make_tables (sca_ref.hpp:57-68) and the
 * scale folding of mb::tables (mb_common.hpp:141-154) ---- */
int orc_tables(int S, double t0, double t1, double q, double lam, double jv, double kappa, int ramp, double scale,
               int32_t* fourT, int32_t* qo, int64_t* kcorr, int32_t* kconst) {
    if (S < 1 || !fourT || !qo || !kcorr || !kconst) return -1;
    double* T = (double*)malloc(sizeof(double) * (size_t)S);
    if (!T) return -1;
    const int den = S - 1 > 1 ? S - 1 : 1;
    for (int t = 0; t < S; ++t) T[t] = t0 * pow(t1 / t0, (double)t / den);
    const double rden = (double)(S - 1) - 0.7 * S > 1.0 ? (double)(S - 1) - 0.7 * S : 1.0;
    for (int t = 0; t < S; ++t) {
        double L = lam;
        if (ramp && t >= 0.7 * S) L = lam * (S - 1 - t) / rden;
        if (scale != 1.0) L *= scale;
        fourT[t] = (int32_t)llround(4.0 * T[t] * 65536.0);
        qo[t] = (int32_t)llround(q * 65536.0);
        kcorr[t] = t == 0 ? 0 : (int64_t)llround(L / (2.0 * T[t - 1]) * 16777216.0);
        kconst[t] = t == 0 ? 0 : (int32_t)llround(-jv * 65536.0);
    }
    if (kappa > 0) {
        for (int t = 1; t < S; ++t) {
            const double rf = (ramp && t >= 0.7 * S) ? (S - 1 - t) / rden : 1.0;
            /* build_tables uses kappa * T * rf; mb::tables uses kappa * scale * T * rf (identical when scale == 1) */
            const double k = scale != 1.0 ? kappa * scale : kappa;
            kconst[t] = (int32_t)llround(k * T[t - 1] * rf * 65536.0);
            kcorr[t] = 0;
        }
    }
    free(T);
    return 0;
}

/* ---- RNG: xoshiro128** seeded by splitmix64(seed ^ trial << 20 ^ lane << 48 ^ 0x5CA0F00D), sca_ref.hpp:70-91 ---- */
typedef struct { uint32_t s[4]; } orc_rng;

static uint64_t splitmix64(uint64_t* x) {
    uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static void rng_seed(orc_rng* r, uint64_t seed, uint32_t trial, uint32_t lane) {
    uint64_t x = seed ^ ((uint64_t)trial << 20) ^ ((uint64_t)lane << 48) ^ 0x5CA0F00Dull;
    const uint64_t a = splitmix64(&x), b = splitmix64(&x);
    r->s[0] = (uint32_t)a; r->s[1] = (uint32_t)(a >> 32); r->s[2] = (uint32_t)b; r->s[3] = (uint32_t)(b >> 32);
    if (!(r->s[0] | r->s[1] | r->s[2] | r->s[3])) r->s[0] = 1;
}

static uint32_t rotl32(uint32_t x, int k) { return (x << k) | (x >> (32 - k)); }

static uint32_t rng_next(orc_rng* r) {
    const uint32_t out = rotl32(r->s[1] * 5u, 7) * 9u, t = r->s[1] << 9;
    r->s[2] ^= r->s[0]; r->s[3] ^= r->s[1]; r->s[1] ^= r->s[2]; r->s[0] ^= r->s[3]; r->s[2] ^= t;
    r->s[3] = rotl32(r->s[3], 11);
    return out;
}

/* h[y] += mult * J[x][y] for every y of row x (J[x][x] == 0). */
static void add_row(const orc_instance* in, int x, int32_t mult, int32_t* h) {
    if (in->dense) {
        const int8_t* row = in->dense + (size_t)x * (size_t)in->n;
        for (int y = 0; y < in->n; ++y) h[y] += mult * (int32_t)row[y];
    } else {
        for (int k = in->row_ptr[x]; k < in->row_ptr[x + 1]; ++k) h[in->col[k]] += mult * (int32_t)in->val[k];
    }
}

/* ---- one anneal: restates sca::run_trial_bias (sca_ref_bias.hpp:25-75), which is sca::run_trial (sca_ref.hpp:101-155)
 * with a bias and a runtime n. Slot i = k * 256 + l is decided by RNG lane l in round k; padding slots still consume
 * their draw. ---- */
int orc_run(const orc_instance* in, const orc_tables_t* tb, uint64_t seed, uint32_t trial, int trace, uint64_t* spins,
            int64_t* sum_sh, int64_t* sum_bs, int64_t* flips_out, int32_t* nlin_out, int32_t* h_out) {
    const int n = in->n;
    if (n < 1 || (!in->dense && !in->row_ptr) || tb->S < 1) return -1;
    const int NP = orc_np(n), R = NP / ORC_LANES, S = tb->S;
    orc_rng rng[ORC_LANES];
    int8_t* s = (int8_t*)malloc((size_t)NP);
    int8_t* sp = (int8_t*)malloc((size_t)NP);
    int32_t* h = (int32_t*)calloc((size_t)NP, 4);
    int32_t* fl = (int32_t*)malloc(sizeof(int32_t) * (size_t)NP);
    if (!s || !sp || !h || !fl) { free(s); free(sp); free(h); free(fl); return -1; }
    for (int l = 0; l < ORC_LANES; ++l) rng_seed(&rng[l], seed, trial, (uint32_t)l);
    memset(s, 1, (size_t)NP);
    memset(sp, 1, (size_t)NP);
    /* initial spins: draw >> 31, round-major (sca_ref_bias.hpp:31-36) */
    for (int k = 0; k < R; ++k)
        for (int l = 0; l < ORC_LANES; ++l) {
            const int i = k * ORC_LANES + l;
            const uint32_t r = rng_next(&rng[l]);
            if (i < n) s[i] = (r >> 31) ? 1 : -1;
        }
    /* initial fields h = b + J s (sca_ref_bias.hpp:37-41) */
    for (int y = 0; y < n; ++y) h[y] = in->bias ? in->bias[y] : 0;
    for (int x = 0; x < n; ++x) add_row(in, x, s[x], h);
    int32_t nlin_prev = 0;
    int64_t flips = 0;
    for (int t = 0; t < S; ++t) {
        /* decision (sca_ref_bias.hpp:45-57) */
        const int64_t corr = floor_shift((int64_t)nlin_prev * tb->kcorr[t], 8) + tb->kconst[t];
        const int32_t fourT = tb->fourT[t], twoT = fourT >> 1;
        int32_t nlin = 0, nf = 0;
        for (int k = 0; k < R; ++k)
            for (int l = 0; l < ORC_LANES; ++l) {
                const int i = k * ORC_LANES + l;
                const uint32_t u16 = rng_next(&rng[l]) >> 16;
                if (i >= n) continue;
                const int64_t z = ((int64_t)s[i] * h[i]) * 65536 + tb->q[t] - (s[i] == sp[i] ? corr : -corr);
                const int64_t r = floor_shift(((int64_t)u16 - 32768) * fourT, 16);
                if (z > -twoT && z < twoT) ++nlin;
                if (z < r) fl[nf++] = i;
            }
        /* commit and field update (sca_ref_bias.hpp:58-65) */
        memcpy(sp, s, (size_t)n);
        for (int f = 0; f < nf; ++f) s[fl[f]] = (int8_t)-s[fl[f]];
        for (int f = 0; f < nf; ++f) add_row(in, fl[f], 2 * s[fl[f]], h);
        flips += nf;
        nlin_prev = nlin;
        if (trace && nlin_out) nlin_out[t] = nlin;
    }
    /* score (sca_ref_bias.hpp:69-73) */
    int64_t sh = 0, bs = 0;
    memset(spins, 0, sizeof(uint64_t) * (size_t)(NP / 64));
    for (int i = 0; i < n; ++i) {
        sh += (int64_t)s[i] * h[i];
        if (in->bias) bs += (int64_t)in->bias[i] * s[i];
        if (s[i] > 0) spins[i >> 6] |= (uint64_t)1 << (i & 63);
    }
    *sum_sh = sh; *sum_bs = bs; *flips_out = flips;
    if (h_out) memcpy(h_out, h, sizeof(int32_t) * (size_t)n);
    free(s); free(sp); free(h); free(fl);
    return 0;
}

typedef struct {
    const orc_instance* in;
    const orc_tables_t* tb;
    uint64_t seed;
    uint32_t off;
    int ntrials, trace;
    uint64_t* spins;
    int64_t *sh, *bs, *flips;
    int32_t* nlin;
    int next;
    int bad;
    pthread_mutex_t mu;
} orc_job;

static void* orc_worker(void* arg) {
    orc_job* j = (orc_job*)arg;
    const int words = orc_np(j->in->n) / 64;
    for (;;) {
        pthread_mutex_lock(&j->mu);
        const int c = j->next++;
        pthread_mutex_unlock(&j->mu);
        if (c >= j->ntrials) break;
        const int rc = orc_run(j->in, j->tb, j->seed, j->off + (uint32_t)c, j->trace, j->spins + (size_t)c * words,
                               j->sh + c, j->bs + c, j->flips + c, j->trace ? j->nlin + (size_t)c * j->tb->S : NULL, NULL);
        if (rc) {
            pthread_mutex_lock(&j->mu);
            j->bad = 1;
            pthread_mutex_unlock(&j->mu);
        }
    }
    return NULL;
}

int orc_run_batch(const orc_instance* in, const orc_tables_t* tb, uint64_t seed, uint32_t trial_offset, int ntrials,
                  int trace, int threads, uint64_t* spins, int64_t* sum_sh, int64_t* sum_bs, int64_t* flips, int32_t* nlin) {
    if (ntrials < 0) return -1;
    orc_job j;
    memset(&j, 0, sizeof j);
    j.in = in; j.tb = tb; j.seed = seed; j.off = trial_offset; j.ntrials = ntrials; j.trace = trace;
    j.spins = spins; j.sh = sum_sh; j.bs = sum_bs; j.flips = flips; j.nlin = nlin;
    pthread_mutex_init(&j.mu, NULL);
    int nth = threads < 1 ? 1 : threads;
    if (nth > ntrials) nth = ntrials > 0 ? ntrials : 1;
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)nth);
    if (!th) return -1;
    for (int i = 0; i < nth; ++i) pthread_create(&th[i], NULL, orc_worker, &j);
    for (int i = 0; i < nth; ++i) pthread_join(th[i], NULL);
    free(th);
    pthread_mutex_destroy(&j.mu);
    return j.bad ? -1 : 0;
}
