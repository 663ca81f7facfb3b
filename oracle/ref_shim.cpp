// TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// C-ABI shim over the reference's own golden model, compiled from the reference headers where they lie
// (include path set by oracle/Makefile; nothing is copied). Functions wrapped:
//   sca::run_trial            gpu/multibit_bias_20261008/src/sca_ref.hpp:101-155
//   sca::run_trial_bias       gpu/multibit_bias_20261008/src/sca_ref_bias.hpp:25-75
//   v80host::build_tables     gpu/multibit_bias_20261008/src/tables.hpp:24-40
//   mb::tables (with scale)   gpu/multibit_bias_20261008/src/mb_common.hpp:141-154
// Built with -DSCA_LANES=256 (the GPU engines' lane count; the header default of 128 is the V80 v4 board image).
#include "sca_ref_bias.hpp"
#include "tables.hpp"
#include "mb_common.hpp"

#include <atomic>
#include <cstring>
#include <thread>
#include <vector>

static_assert(sca::LANES == 256, "build with -DSCA_LANES=256");

namespace {

sca::Tables tables_of(const int32_t* fourT, const int32_t* q, const int64_t* kcorr, const int32_t* kconst, int S) {
    sca::Tables tb;
    tb.fourT.assign(fourT, fourT + S);
    tb.q.assign(q, q + S);
    tb.kcorr.assign(kcorr, kcorr + S);
    tb.kconst.assign(kconst, kconst + S);
    return tb;
}

void tables_out(const sca::Tables& tb, int32_t* fourT, int32_t* q, int64_t* kcorr, int32_t* kconst) {
    const size_t S = tb.fourT.size();
    std::memcpy(fourT, tb.fourT.data(), S * 4);
    std::memcpy(q, tb.q.data(), S * 4);
    std::memcpy(kcorr, tb.kcorr.data(), S * 8);
    std::memcpy(kconst, tb.kconst.data(), S * 4);
}

}  // namespace

extern "C" {

int ref_np(void) { return sca::NP; }
int ref_lanes(void) { return sca::LANES; }

// v80host::build_tables (the flag-built tables of sca_gpu / sca_gpu_bias).
int ref_build_tables(int S, double t0, double t1, double q, double lam, double jv, double kappa, int ramp, int32_t* fourT,
                     int32_t* qo, int64_t* kcorr, int32_t* kconst) {
    try {
        v80host::Schedule sc;
        sc.S = S; sc.t0 = t0; sc.t1 = t1; sc.q = q; sc.lam = lam; sc.jv = jv; sc.kappa = kappa; sc.ramp = ramp != 0;
        tables_out(v80host::build_tables(sc), fourT, qo, kcorr, kconst);
        return 0;
    } catch (...) { return -1; }
}

// mb::tables (correction scale folded into lambda / kappa).
int ref_mb_tables(int S, double t0, double t1, double q, double lam, double jv, double kappa, int ramp, double scale,
                  int32_t* fourT, int32_t* qo, int64_t* kcorr, int32_t* kconst) {
    try {
        mb::Sched sc;
        sc.S = S; sc.t0 = t0; sc.t1 = t1; sc.q = q; sc.lam = lam; sc.jv = jv; sc.kappa = kappa; sc.ramp = ramp != 0; sc.scale = scale;
        tables_out(mb::tables(sc), fourT, qo, kcorr, kconst);
        return 0;
    } catch (...) { return -1; }
}

// sca::run_trial_bias on a dense NP x NP int8 matrix (dense[x * NP + y], zero diagonal and padding).
// spins: 32 words; nlin: S entries when trace != 0.
int ref_run_trial_bias(int n, const int8_t* dense, const int32_t* bias, const int32_t* fourT, const int32_t* q,
                       const int64_t* kcorr, const int32_t* kconst, int S, uint64_t seed, uint32_t trial, int trace,
                       uint64_t* spins, int64_t* sum_sh, int64_t* sum_bs, int64_t* flips, int32_t* nlin) {
    try {
        const sca::Tables tb = tables_of(fourT, q, kcorr, kconst, S);
        const sca::ResultBias r = sca::run_trial_bias(n, dense, bias, tb, seed, trial, trace != 0);
        std::memcpy(spins, r.spins.data(), sizeof(uint64_t) * sca::WORDS);
        *sum_sh = r.sum_sh; *sum_bs = r.sum_bs; *flips = r.flips;
        if (trace) std::memcpy(nlin, r.n_lin.data(), size_t(S) * 4);
        return 0;
    } catch (...) { return -1; }
}

// sca::run_trial (N = 2000 only) on the same dense matrix; sumw is passed in (run_trial reads only g.sumw when dense is set).
int ref_run_trial(const int8_t* dense, int64_t sumw, const int32_t* fourT, const int32_t* q, const int64_t* kcorr,
                  const int32_t* kconst, int S, uint64_t seed, uint32_t trial, int trace, uint64_t* spins, int64_t* cut,
                  int64_t* flips, int32_t* nlin) {
    try {
        const sca::Tables tb = tables_of(fourT, q, kcorr, kconst, S);
        sca::Graph g; g.sumw = sumw;
        const sca::Result r = sca::run_trial(g, tb, seed, trial, trace != 0, dense);
        std::memcpy(spins, r.spins.data(), sizeof(uint64_t) * sca::WORDS);
        *cut = r.cut; *flips = r.flips;
        if (trace) std::memcpy(nlin, r.n_lin.data(), size_t(S) * 4);
        return 0;
    } catch (...) { return -1; }
}

// Many trials of run_trial_bias on a std::thread pool (the pattern of check_ref_bias.cpp). Trial c uses trial id
// trial_offset + c. Outputs are per trial: spins[c * 32 ...], sum_sh[c], sum_bs[c], flips[c], nlin[c * S ...].
int ref_run_batch_bias(int n, const int8_t* dense, const int32_t* bias, const int32_t* fourT, const int32_t* q,
                       const int64_t* kcorr, const int32_t* kconst, int S, uint64_t seed, uint32_t trial_offset, int ntrials,
                       int trace, int threads, uint64_t* spins, int64_t* sum_sh, int64_t* sum_bs, int64_t* flips,
                       int32_t* nlin) {
    try {
        const sca::Tables tb = tables_of(fourT, q, kcorr, kconst, S);
        std::atomic<int> next{0}, bad{0};
        auto work = [&]() {
            for (int c; (c = next++) < ntrials;) {
                try {
                    const sca::ResultBias r = sca::run_trial_bias(n, dense, bias, tb, seed, trial_offset + uint32_t(c), trace != 0);
                    std::memcpy(spins + size_t(c) * sca::WORDS, r.spins.data(), sizeof(uint64_t) * sca::WORDS);
                    sum_sh[c] = r.sum_sh; sum_bs[c] = r.sum_bs; flips[c] = r.flips;
                    if (trace) std::memcpy(nlin + size_t(c) * S, r.n_lin.data(), size_t(S) * 4);
                } catch (...) { ++bad; }
            }
        };
        const int nth = threads < 1 ? 1 : threads;
        std::vector<std::thread> th;
        for (int i = 0; i < nth; ++i) th.emplace_back(work);
        for (auto& t : th) t.join();
        return bad.load() ? -1 : 0;
    } catch (...) { return -1; }
}

}  // extern "C"
