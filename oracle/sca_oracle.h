/* TEST INFRASTRUCTURE ONLY: CPU restatement of the reference SCA golden model, used by tests/, smoke() and bench.py's
 * CPU-baseline leg as the checker. The product (anechoic_b200/) never links or calls it.
 *
 * Parity: pinned for N <= 2048 against the reference's own golden model (sca_ref.hpp / sca_ref_bias.hpp, compiled
 * unmodified into oracle/_ref by oracle/Makefile) through the committed fixtures in tests/golden/. For N > 2048 the
 * slot layout is this project's generalisation (see orc_np) and parity rests on this restatement alone. */
#ifndef ANECHOIC_SCA_ORACLE_H
#define ANECHOIC_SCA_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Padded spin count: max(2048, ceil(n / 256) * 256). 256 RNG lanes, NP / 256 rounds (8 for n <= 2048, as the reference). */
int orc_np(int n);

/* Schedule -> fixed-point tables, restating v80host::build_tables (tables.hpp:24-40) and mb::tables
 * (mb_common.hpp:141-154; scale == 1 gives build_tables). Returns 0, or -1 on bad arguments. */
int orc_tables(int S, double t0, double t1, double q, double lam, double jv, double kappa, int ramp, double scale,
               int32_t* fourT, int32_t* qo, int64_t* kcorr, int32_t* kconst);

/* One coupling source: either dense (J[x * n + y], int8, symmetric, zero diagonal) or CSR rows (row_ptr[n + 1],
 * col[], val[]; every nonzero of row x, each pair stored in both rows). Exactly one of dense / row_ptr is non-NULL. */
typedef struct {
    int n;
    const int8_t* dense;
    const int32_t* row_ptr;
    const int32_t* col;
    const int8_t* val;
    const int32_t* bias; /* n entries or NULL */
} orc_instance;

typedef struct {
    const int32_t* fourT;
    const int32_t* q;
    const int64_t* kcorr;
    const int32_t* kconst;
    int S;
} orc_tables_t;

/* One anneal (restating sca::run_trial_bias, sca_ref_bias.hpp:25-75, generalised to any n).
 * spins: orc_np(n) / 64 words, bit i set iff s_i = +1 (active spins only). nlin: S entries if trace. h_out: n entries
 * (final fields) or NULL. Returns 0 or -1. */
int orc_run(const orc_instance* inst, const orc_tables_t* tb, uint64_t seed, uint32_t trial, int trace, uint64_t* spins,
            int64_t* sum_sh, int64_t* sum_bs, int64_t* flips, int32_t* nlin, int32_t* h_out);

/* ntrials anneals with trial ids trial_offset + c on `threads` POSIX threads. Per-trial output strides:
 * spins orc_np(n) / 64 words, nlin S entries. */
int orc_run_batch(const orc_instance* inst, const orc_tables_t* tb, uint64_t seed, uint32_t trial_offset, int ntrials,
                  int trace, int threads, uint64_t* spins, int64_t* sum_sh, int64_t* sum_bs, int64_t* flips, int32_t* nlin);

#ifdef __cplusplus
}
#endif
#endif
