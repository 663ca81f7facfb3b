// Plain SCA engine ("bit-column" path): one CTA of 512 threads runs one anneal at a time; a persistent grid pulls
// (job, trial) items from a queue, so one launch carries many anneals and many instances of uneven size.
//
// Per step (exactly sca::run_trial_bias, reference gpu/multibit_bias_20261008/src/sca_ref_bias.hpp:44-68):
//   1. Warps 0..7 own RNG lanes 0..255. For each round k, lane l decides slot i = k*256 + l. The 32 slots of a warp
//      in one round are spin word k*8 + warp, so one __ballot_sync gives the flip word, one gives the n_lin band word
//      (n_lin = sum of __popc over them), and flipped slots are appended to a compact flip list in shared memory.
//   2. Field update h_y += 2 * s'_x * J_xy over the flipped x only.
//      Dense couplings are bit planes, row x = NWJ 32-bit words (32 couplings each): K = 1 one plane (bit = [J = +1]);
//      K = 2, 4 a sign plane and K-1 magnitude planes. Thread (group g, word w) reads word w of each flipped row of
//      its group (coalesced: a warp reads 128 contiguous bytes of one row) and adds it into bit-sliced counters with
//      carry-save adders (a Harley-Seal tree over batches of 8 rows, LOP3 arithmetic, 32 couplings per op). The
//      groups' counters are summed by a bit-sliced adder tree in shared memory; the deciding thread of slot y
//      extracts y's count at the start of the next step, when it reads h_y. When the counters of all 2(K-1)
//      sign/magnitude sets do not fit in shared memory (N = 16384, K = 4), each set is added into the fields as soon
//      as it is complete (streaming layout, one result buffer).
//      Sparse couplings (CSR rows) are scattered with shared-memory atomics: a group of lanes per flipped row (an
//      eighth of the rows' mean degree, rounded up to a power of two), each lane fetching up to 8 edges before it
//      applies any, so many L2 fetches are in flight per warp.
//   The initial field h = b + J s0 reuses step 2 with F = all active slots and factor 1.
// All arithmetic is integer and order-independent, so the result is bit-exact with the golden model.
#pragma once
#include <cstdint>

#include "anc_common.cuh"

namespace anc {

constexpr int kPlainThreads = 512;

struct PlainJob {
    // instance
    int n, np, nw, nwj, K;             // K = 0: sparse CSR
    const uint32_t* planes;            // dense: [max(K,1)][np][nwj]
    const int32_t* row_ptr;            // sparse: [n + 1] (csr16: in words of two edges)
    const uint32_t* adj;               // sparse: (y << 8) | uint8(J_xy); csr16: two 16-bit edges per word
    int csr16;                         // sparse, every J_xy = +-1 and n < 32767: edge = y | [J_xy = -1] << 15, rows
                                       // padded to whole words with the skip edge 0x7fff
    const int32_t* bias;               // [n] or null
    DevTables tab;
    uint64_t seed;
    uint32_t trial_offset;
    int ntrials;
    int trace;
    int32_t hclamp;                    // > 0: clamp s*h to +-hclamp in the decision (exact; host range plan)
    // outputs (device pointers)
    uint32_t* out_spins;               // [ntrials][nw]: bit i of word i/32 = [s_i = +1], active spins only
    int64_t* out_sum_sh;               // [ntrials]
    int64_t* out_sum_bs;               // [ntrials]
    int64_t* out_flips;                // [ntrials]
    int32_t* out_trace;                // [ntrials][S] or null
    int32_t* out_h;                    // [ntrials][n] or null (final fields)
    // cluster engine only: error word (a bounded wait that gave up sets it; may be null) and the limit of each wait
    int* err;
    uint64_t wait_ns;
};

// Error codes of the cluster engine's error word.
constexpr int kClusterErrRecv = 1;     // a step's exchange words did not all arrive within the wait limit

struct PlainLaunch {
    PlainJob job0;                     // the job when items == nullptr (item index = trial index)
    const PlainJob* jobs;              // device array when items != nullptr
    const int2* items;                 // (job, trial index), or nullptr
    int nitems;
    int* next_item;                    // queue head (zeroed before launch)
    int np_max, nwj_max;               // shared-memory layout
    int stream;                        // 1: dense counts go into the fields set by set (one result buffer)
    int sparse_variant;                // CSR pass variant (kSparseVariants index; 0 = rows 1 x edges 8 per lane)
    int dense_variant;                 // dense pass variant (dense_variants(K) of them; 0 = the default)
};

// CSR pass variants the host's tuner chooses among: {lane groups' rows in flight, edges per lane fetched before any
// is applied}. Every variant computes the same fields (integer atomics into shared memory), only the time differs.
constexpr int kSparseVariants = 4;
constexpr int kSparseVariantShape[kSparseVariants][2] = {{1, 8}, {1, 4}, {2, 4}, {1, 16}};

// Compiled variants of the dense pass (rows of bit planes each thread counts per batch):
//   K = 1: 0 = 8 rows with the next 8 fetched ahead, 1 = 8 rows, 2 = 16 rows;
//   K = 2: 0 = 8 rows, 1 = 16 rows;
//   K = 4 and the streaming layout: 8 rows only (16 rows of 6 counter sets exceed the 128 registers a thread has).
constexpr int kDenseVariantsMax = 3;
inline int dense_variants(int K, bool stream) { return stream ? 1 : K == 1 ? 3 : K == 2 ? 2 : 1; }

// Shared-memory bytes for a launch (P = counter planes).
inline size_t plain_smem_bytes(int np_max, int nwj_max, int K, int P, bool stream = false) {
    const size_t C = (K <= 1 || stream) ? 1 : size_t(2 * (K - 1));
    size_t b = size_t(np_max) * 4 * 2 + size_t(nwj_max) * 4 * 2;
    if (K != 0) {
        const size_t comb = size_t(nwj_max > kPlainThreads ? nwj_max : kPlainThreads);
        b += comb * P * 4 + C * size_t(nwj_max) * P * 4;
    }
    return b;
}

// Shared-memory plan of a launch: the full layout when it fits in 227 KB; otherwise, for K = 2 / 4 with at most one
// counter word per thread (N <= 16384), the streaming layout, where each of the 2(K-1) sign/magnitude counter sets
// is added into the fields as soon as it is complete, so one result buffer serves them all (*stream = true).
inline size_t plain_smem_plan(int np_max, int nwj_max, int K, int P, bool* stream) {
    constexpr size_t kLimit = 227 * 1024;
    const size_t full = plain_smem_bytes(np_max, nwj_max, K, P, false);
    *stream = K >= 2 && full > kLimit && nwj_max <= kPlainThreads;
    return *stream ? plain_smem_bytes(np_max, nwj_max, K, P, true) : full;
}

// Host launcher (plain_engine.cu). Returns a cudaError_t value.
int plain_launch(const PlainLaunch& L, int K, int P, int grid, size_t smem, cudaStream_t stream);
int plain_max_blocks_per_sm(int K, int P, size_t smem, int* out, bool stream = false);

// Cluster variant (plain_engine.cu): one anneal per cluster of 8 CTAs, dense K = 1 couplings with NP = 2048 only.
// job.ntrials anneals, trial c = job.trial_offset + c; every output is written (no zeroing needed).
bool plain_cluster_supported(int K, int np);
// One anneal per cluster of `ctas` CTAs (8, or 16: half the slots per SM, a non-portable cluster size)
int plain_cluster_launch(const PlainJob& job, cudaStream_t stream, int ctas = 8);
int plain_cluster_max_active(int* out, int ctas = 8);      // clusters of `ctas` co-resident on this device

}  // namespace anc
