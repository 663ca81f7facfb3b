// Batched SCA engine for replicas that share J: the field update is a dense int8 contraction on the tcgen05 tensor
// cores, exact with int32 accumulation in TMEM.
//
// Per step of the reference algorithm (sca::run_trial_bias, gpu/multibit_bias_20261008/src/sca_ref_bias.hpp:44-68):
//   h_y += sum_x D_x J_xy  with  D_x = 2 s'_x for flipped x and 0 otherwise  (D = s0 with factor 1 for h(0) = b + J s0).
// Layout: a thread-block cluster of C = 16 CTAs runs a group of 128 replicas (one TMEM lane each). Spin slot
// i = k*256 + l (RNG lane l, round k) is owned by CTA c = l / 16 and held at permuted index
// p(i) = c*NC + (l % 16)*R + k (NC = NP/16 slots per CTA, R = NP/256 rounds); J is stored permuted the same way
// (J_perm[p(x)][p(y)] = J_xy), so CTA c's slots are the contiguous column slice [c*NC, (c+1)*NC).
//   * 16 decision warps: thread (replica r, quarter q) owns RNG lanes 16c + 4q .. 16c + 4q + 3 of replica r, i.e.
//     4R slots = TMEM columns [4Rq, 4R(q+1)). It reads h with tcgen05.ld, decides exactly as the golden model
//     (Q16.16 integer threshold from the replica's own xoshiro128** stream, counted / temperature-scaled correction),
//     and writes its D bytes to a global exchange buffer D[group][parity][r][p]; n_lin partials go to a small buffer.
//   * barrier.cluster (release / acquire) publishes every CTA's slice of D and n_lin.
//   * 1 TMA warp streams K-chunks of 128: A = D[group][parity][0..127][chunk] (128 x 128 B) and
//     B = J_perm[c*NC .. +NC][chunk] (NC x 128 B), 128-byte swizzled, into a 4-stage shared-memory ring
//     (no multicast anywhere).
//   * 1 MMA thread issues tcgen05.mma.cta_group::1.kind::i8 (M = 128, N = NC, K = 32) accumulating into h in TMEM,
//     frees each stage with tcgen05.commit, and signals "h ready" after the last chunk.
// Every mbarrier wait is bounded by %globaltimer: on expiry the kernel records an error code, skips the remaining
// work but keeps every cluster barrier, so all CTAs finish; the host reports ANC_ETIMEOUT.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "anc_ptx.cuh"
#include "anc_tensor.cuh"

namespace anc {
namespace {

using namespace ptx;

constexpr int kC = 16;                  // CTAs per cluster (replica group)
constexpr int kM = 128;                 // replicas per group (MMA M, TMEM lanes)
constexpr int kDW = 16;                 // decision warps
constexpr int kThreads = (kDW + 2) * 32;
constexpr int kTmaWarp = kDW, kMmaWarp = kDW + 1;
constexpr int kStages = 4;
constexpr int kKChunk = 128;            // bytes (= int8 elements) of K per stage

// error codes written to the run's error word
constexpr int kErrFull = 1, kErrEmpty = 2, kErrHready = 3;

struct TensorParams {
    int n, np, R, nc;                   // active spins, padded, rounds, slots per CTA
    int S;
    const int32_t* fourT;
    const int32_t* q;
    const int64_t* kcorr;
    const int32_t* kconst;
    int32_t hclamp;
    const int32_t* bias_perm;           // [np] bias at permuted index, or null
    uint64_t seed;
    uint32_t trial_offset;
    int nchains;
    int8_t* dbuf;                       // [groups][2][128][np]
    int32_t* nlbuf;                     // [groups][2][16][128]
    uint32_t* out_spins;                // [nchains][np/32] (zeroed by the host)
    unsigned long long* out_sum_sh;     // [nchains] (zeroed)
    unsigned long long* out_sum_bs;     // [nchains] (zeroed)
    unsigned long long* out_flips;      // [nchains] (zeroed)
    int32_t* out_trace;                 // [nchains][S] or null
    int32_t* out_h;                     // [nchains][n] or null
    int* err;                           // error word (zeroed)
    long long* prof;                    // [gridDim.x][kProfSlots] clock64 phase totals, or null (off)
};

// opt-in phase profile (clock64 cycles summed over the steps, per CTA):
//   0 decision warps waiting for h   1 TMEM load + decide + D store   2 named barrier + n_lin publish (fp4 kernel:
//     named barrier + flag release)   3 cluster barrier (fp4 kernel: the next step's draws)   4 n_lin read (fp4
//     kernel: the exchange, flags to last tile stored and n_lin summed)   5 MMA thread waiting for stages
//   6 MMA thread: barrier end -> last commit issued   7 TMA thread waiting for free stages   8 whole step loop
//   9 MMA issue   10 MMA commits
//   fp4 kernel, measured from this CTA's own publish: 11 first D tile full, 12 last D tile full, 14 fields-ready
//     commit issued, 15 / 16 flags of D tile 0 / 7 seen by decision thread 0, 17 / 18 its copies of D tile 0 / 7
//     landed and arrived
constexpr int kProfSlots = kTensorProfSlots;

// ------------------------------------------------------------------------------------------------ helpers
__device__ __forceinline__ void flag_publish(uint32_t* p, uint32_t v) {
    asm volatile("fence.acq_rel.gpu;\n\tst.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Release store alone: the writes of the CTA's other threads are ordered before it by the preceding bar.sync, and
// release is cumulative over them.
__device__ __forceinline__ void flag_release(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

__device__ __forceinline__ uint32_t cluster_id_x() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
    return r;
}

// ------------------------------------------------------------------------------------------------ the kernel
template <int R>
__global__ void __launch_bounds__(kThreads, 1)
    tensor_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                  const __grid_constant__ TensorParams P) {
    constexpr int NC = 16 * R;            // slots (TMEM columns) per CTA
    constexpr int COLS = 4 * R;           // columns per decision thread (4 RNG lanes x R rounds)
    constexpr int NCHUNK = 2 * R;         // K chunks of 128 over NP = 256 R
    constexpr uint32_t A_BYTES = kM * kKChunk;
    constexpr uint32_t B_BYTES = NC * kKChunk;
    constexpr uint32_t STAGE = A_BYTES + B_BYTES;
    constexpr int TMEM_COLS = NC <= 32 ? 32 : NC <= 64 ? 64 : NC <= 128 ? 128 : 256;
    constexpr uint32_t IDESC = (2u << 4) | (1u << 7) | (1u << 10) | (uint32_t(NC >> 3) << 17) | (uint32_t(kM >> 4) << 24);

    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* stages = smem;                                        // kStages x STAGE, 1024-aligned
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kStages * STAGE);
    // bars: full[kStages], empty[kStages], hready
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kStages + 1);
    int* nl_s = reinterpret_cast<int*>(tmem_slot + 4);           // [128] n_lin partial of this CTA per replica

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int c = int(cluster_rank());
    const int g = int(cluster_id_x());                            // replica group
    const int n = P.n, S = P.S;
    int* err = P.err;

    const uint32_t bar_full = smem_u32(bars), bar_empty = smem_u32(bars + kStages);
    const uint32_t bar_h = smem_u32(bars + 2 * kStages);

    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(bar_full + 8 * s, 1);
            mbar_init(bar_empty + 8 * s, 1);
        }
        mbar_init(bar_h, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (tid < kM) nl_s[tid] = 0;
    if (warp == kMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    // ---------------- decision warps ----------------
    // replica r = lane quarter (warp % 4) * 32 + lane; column quarter qq = warp / 4
    const int r = (warp & 3) * 32 + lane;
    const int qq = warp >> 2;
    const int chain = g * kM + r;
    const bool writer = chain < P.nchains;
    Xoshiro rng[4];
    uint32_t sw[2] = {0u, 0u}, dw[2] = {0u, 0u};   // spin (1 = +1) and flipped-last-step bits of the COLS slots
    long long flips = 0;
    int32_t nlin_prev = 0;
    const uint32_t taddr = tmem + (uint32_t((warp & 3) * 32) << 16) + uint32_t(qq * COLS);
    int8_t* drow0 = P.dbuf + (size_t(g) * 2 * kM + r) * P.np + size_t(c) * NC + size_t(qq) * COLS;
    const size_t dpar_stride = size_t(kM) * P.np;

    // slot of column col (= j*R + k) of this thread: RNG lane l = 16c + 4qq + j, round k, i = k*256 + l
    auto slot_of = [&](int col) { return (col % R) * 256 + 16 * c + 4 * qq + col / R; };

    if (warp < kDW) {
        // seeds, initial spins (draw >> 31, padding +1), s_prev = +1 (so "flipped" = [s0 = -1]); h := bias
        for (int j = 0; j < 4; ++j) rng_seed(rng[j], P.seed, P.trial_offset + uint32_t(chain), uint32_t(16 * c + 4 * qq + j));
        uint32_t dbytes[COLS / 4];
#pragma unroll
        for (int w = 0; w < COLS / 4; ++w) dbytes[w] = 0u;
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const int col = j * R + k;
                const uint32_t rv = rng_next(rng[j]);
                const int i = k * 256 + 16 * c + 4 * qq + j;
                const bool valid = i < n;
                const uint32_t up = valid ? (rv >> 31) : 1u;
                sw[col >> 5] |= up << (col & 31);
                if (valid && !up) dw[col >> 5] |= 1u << (col & 31);
                const uint32_t b = valid ? (up ? 0x01u : 0xFFu) : 0u;
                dbytes[col >> 2] |= b << (8 * (col & 3));
            }
        // D(-1) = s0 into parity 1 (the step index -1 is odd)
        int8_t* drow = drow0 + dpar_stride;
#pragma unroll
        for (int w = 0; w < COLS / 16; ++w)
            reinterpret_cast<uint4*>(drow)[w] = make_uint4(dbytes[4 * w], dbytes[4 * w + 1], dbytes[4 * w + 2], dbytes[4 * w + 3]);
        // TMEM h := bias (per column)
#pragma unroll
        for (int cb = 0; cb < COLS; cb += 16) {
            uint32_t v[16];
#pragma unroll
            for (int e = 0; e < 16; ++e) {
                const int col = qq * COLS + cb + e;
                v[e] = P.bias_perm ? uint32_t(P.bias_perm[c * NC + col]) : 0u;
            }
            tmem_st16(taddr + cb, v);
        }
        tmem_wait_st();
        if (qq == 0) P.nlbuf[((size_t(g) * 2 + 1) * kC + c) * kM + r] = 0;
        asm volatile("fence.proxy.async.global;" ::: "memory");
        tc_fence_before();
    }

    // step index m = -1 (initial field), 0 .. S-1; after each: cluster barrier, then the MMA applies D(m)
    uint32_t stage_it = 0;                     // running stage counter (TMA and MMA threads)
    const bool prof = P.prof != nullptr;
    long long pr[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    long long tq = clock64();
    const long long t_loop0 = tq;
    auto mark = [&](int slot) {
        if (prof) {
            const long long now = clock64();
            pr[slot] += now - tq;
            tq = now;
        }
    };
    for (int m = -1; m < S; ++m) {
        const int par = m & 1;
        if (m >= 0 && warp < kDW) {
            // wait for h (after D(m-1)), read it, decide step m
            if (prof) tq = clock64();
            if (!err_set(err)) mbar_wait(bar_h, uint32_t(m & 1), err, kErrHready);
            tc_fence_after();
            mark(0);
            const int t = m;
            const int32_t fourT = __ldg(P.fourT + t), twoT = fourT >> 1, qv = __ldg(P.q + t);
            const int32_t corr = step_corr(nlin_prev, __ldg(P.kcorr + t), __ldg(P.kconst + t));
            const uint32_t lw = uint32_t(2 * twoT - 1);
            const int32_t hcl = P.hclamp;
            uint32_t dbytes[COLS / 4];
#pragma unroll
            for (int w = 0; w < COLS / 4; ++w) dbytes[w] = 0u;
            int nl = 0;
            uint32_t nsw[2] = {sw[0], sw[1]}, ndw[2] = {0u, 0u};
#pragma unroll
            for (int cb = 0; cb < COLS; cb += 16) {
                uint32_t hv[16];
                tmem_ld16(taddr + cb, hv);
                tmem_wait_ld();
                // draws follow each lane's round order: columns are j*R + k, so 16-column blocks taken in order
                // visit every lane's rounds in increasing k
#pragma unroll
                for (int e = 0; e < 16; ++e) {
                    const int col = cb + e;
                    const int j = col / R, k = col % R;
                    const uint32_t u = rng_next(rng[j]);
                    const int i = k * 256 + 16 * c + 4 * qq + j;
                    const bool valid = i < n;
                    const bool up = (sw[col >> 5] >> (col & 31)) & 1u;
                    const bool dif = (dw[col >> 5] >> (col & 31)) & 1u;
                    const int32_t h = int32_t(hv[e]);
                    int32_t hs = up ? h : -h;
                    if (hcl > 0) hs = max(-hcl, min(hs, hcl));
                    const int32_t x = qv + (dif ? corr : -corr);
                    const int32_t zt = hs * 65536 + x;
                    const int32_t thr = threshold16(u, fourT);
                    const bool fl = valid && (zt - thr < 0);
                    nl += (valid && (uint32_t(zt + twoT - 1) < lw)) ? 1 : 0;
                    if (fl) {
                        nsw[col >> 5] ^= 1u << (col & 31);
                        ndw[col >> 5] |= 1u << (col & 31);
                        dbytes[col >> 2] |= (up ? 0xFEu : 0x02u) << (8 * (col & 3));   // 2 * s' with s' = -s
                        ++flips;
                    }
                }
            }
            sw[0] = nsw[0]; sw[1] = nsw[1];
            dw[0] = ndw[0]; dw[1] = ndw[1];
            int8_t* drow = drow0 + size_t(par) * dpar_stride;
#pragma unroll
            for (int w = 0; w < COLS / 16; ++w)
                reinterpret_cast<uint4*>(drow)[w] =
                    make_uint4(dbytes[4 * w], dbytes[4 * w + 1], dbytes[4 * w + 2], dbytes[4 * w + 3]);
            mark(1);
            atomicAdd(&nl_s[r], nl);
            tc_fence_before();
            asm volatile("bar.sync 1, %0;" ::"r"(kDW * 32) : "memory");
            if (qq == 0) {
                P.nlbuf[((size_t(g) * 2 + par) * kC + c) * kM + r] = nl_s[r];
                nl_s[r] = 0;
            }
            asm volatile("fence.proxy.async.global;" ::: "memory");
            mark(2);
        }
        if (prof) tq = clock64();
        cluster_sync();
        asm volatile("fence.proxy.async.global;" ::: "memory");
        if (warp < kDW) mark(3);
        else if (prof) tq = clock64();
        if (warp < kDW && m >= 0) {
            // n_lin of step m for replica r: sum of the 16 CTAs' partials
            const int32_t* nlp = P.nlbuf + (size_t(g) * 2 + par) * kC * kM + r;
            int32_t tot = 0;
#pragma unroll
            for (int cc = 0; cc < kC; ++cc) tot += __ldcg(nlp + cc * kM);
            nlin_prev = tot;
            if (c == 0 && qq == 0 && writer && P.out_trace) P.out_trace[size_t(chain) * S + m] = tot;
            mark(4);
        }
        if (warp == kTmaWarp) {
            if (lane == 0) {
                const int ay = (g * 2 + (par & 1)) * kM;
                for (int kc = 0; kc < NCHUNK; ++kc, ++stage_it) {
                    const int s = int(stage_it % kStages);
                    const uint32_t ph = (stage_it / kStages) & 1u;
                    if (err_set(err)) continue;   // after a failed wait: issue nothing more
                    const long long w0 = prof ? clock64() : 0;
                    if (stage_it >= kStages && !mbar_wait(bar_empty + 8 * s, ph ^ 1u, err, kErrEmpty)) continue;
                    if (prof) pr[7] += clock64() - w0;
                    const uint32_t dst = smem_u32(stages + size_t(s) * STAGE);
                    mbar_arrive_expect_tx(bar_full + 8 * s, STAGE);
                    tma_load_2d(dst, &mapA, kc * kKChunk, ay, bar_full + 8 * s);
                    tma_load_2d(dst + A_BYTES, &mapB, kc * kKChunk, c * NC, bar_full + 8 * s);
                }
            } else {
                stage_it += NCHUNK;
            }
            __syncwarp();
        } else if (warp == kMmaWarp) {
            if (lane == 0) {
                tc_fence_after();
                for (int kc = 0; kc < NCHUNK; ++kc, ++stage_it) {
                    const int s = int(stage_it % kStages);
                    const uint32_t ph = (stage_it / kStages) & 1u;
                    const long long w0 = prof ? clock64() : 0;
                    const bool ok = !err_set(err) && mbar_wait(bar_full + 8 * s, ph, err, kErrFull);
                    if (prof) pr[5] += clock64() - w0;
                    tc_fence_after();
                    if (ok) {
                        const uint32_t a0 = smem_u32(stages + size_t(s) * STAGE), b0 = a0 + A_BYTES;
#pragma unroll
                        for (int kk = 0; kk < kKChunk / 32; ++kk)
                            mma_i8(tmem, sw128_desc(a0 + 32 * kk), sw128_desc(b0 + 32 * kk), IDESC, 1u);
                    }
                    mma_commit(bar_empty + 8 * s);     // frees the stage once the MMAs above have read it
                }
                mma_commit(bar_h);                     // h ready for the next decision
                mark(6);
            } else {
                stage_it += NCHUNK;
            }
            __syncwarp();
        }
    }
    if (prof) {
        pr[8] = clock64() - t_loop0;
        long long* dst = P.prof + size_t(blockIdx.x) * kProfSlots;
        if (warp == 0 && lane == 0)
            for (int s = 0; s < 5; ++s) dst[s] = pr[s];
        if (warp == kMmaWarp && lane == 0) { dst[5] = pr[5]; dst[6] = pr[6]; dst[8] = pr[8]; }
        if (warp == kTmaWarp && lane == 0) dst[7] = pr[7];
    }

    // ---------------- final fields and outputs ----------------
    if (warp < kDW) {
        if (!err_set(err)) mbar_wait(bar_h, uint32_t(S & 1), err, kErrHready);
        tc_fence_after();
        long long sh = 0, bs = 0;
        const int words = P.np / 32;
#pragma unroll
        for (int cb = 0; cb < COLS; cb += 16) {
            uint32_t hv[16];
            tmem_ld16(taddr + cb, hv);
            tmem_wait_ld();
#pragma unroll
            for (int e = 0; e < 16; ++e) {
                const int col = cb + e;
                const int i = slot_of(col);
                if (i >= n) continue;
                const bool up = (sw[col >> 5] >> (col & 31)) & 1u;
                const int32_t h = int32_t(hv[e]);
                sh += up ? h : -h;
                if (P.bias_perm) {
                    const int32_t b = P.bias_perm[c * NC + qq * COLS + col];
                    bs += up ? b : -b;
                }
                if (writer) {
                    if (up) atomicOr(P.out_spins + size_t(chain) * words + (i >> 5), 1u << (i & 31));
                    if (P.out_h) P.out_h[size_t(chain) * n + i] = h;
                }
            }
        }
        if (writer) {
            atomicAdd(P.out_sum_sh + chain, static_cast<unsigned long long>(sh));
            atomicAdd(P.out_sum_bs + chain, static_cast<unsigned long long>(bs));
            atomicAdd(P.out_flips + chain, static_cast<unsigned long long>(flips));
        }
        tc_fence_before();
    }
    __syncthreads();
    cluster_sync();   // no CTA leaves while a peer may still read its D slice through L2 (and keeps TMEM until done)
    if (warp == kMmaWarp) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

// ------------------------------------------------------------------------------------------------ resident-J kernel
// For NP = 2048 (n <= 2048): a cooperative persistent grid of 32 y-slices x P group-pairs. CTA (pair slot gp,
// slice cs) owns spin slots with RNG lanes 8cs .. 8cs+7 (64 columns at permuted indices p = 8l + k) and keeps its
// J column slice (2048 x 64 int8 = 128 KB, 128-byte swizzled) resident in shared memory for the whole launch.
// It runs TWO replica groups of 128 (a pair) and alternates between them, so the decisions of one group overlap
// the tensor-core update of the other:
//   decision warps (16): for group g: wait "h ready", tcgen05.ld 16 field columns + the n_lin accumulator, decide,
//     write D(m) (16 bytes) and the thread's n_lin partial (1 byte) to the exchange buffers, then one thread
//     publishes flag[g][cs] = m + 2 (st.release.gpu).
//   producer warps (4): for every K chunk (128 x-values = two source slices) wait for both slices' flags
//     (ld.acquire.gpu), then TMA the 128 x 128-byte D tile into the stage ring; a 17th chunk carries the 128
//     n_lin partials of all slices. Each warp issues every fourth chunk: one thread's bulk copies are serviced one
//     at a time, so four issuers keep four copies in flight.
//   MMA thread: per chunk 4 x tcgen05.mma.kind::i8 (M 128, N 64, K 32) into the group's field accumulator with B
//     = the resident J chunk; the n_lin chunk is multiplied by a ones row (N 16) into a per-group accumulator,
//     so sum_slices n_lin partials comes out of the tensor core with the fields.
// No cluster barrier exists: the flags make the exchange a dataflow, chunks are consumed as slices finish.
constexpr int kResSlices = 32;            // y-slices for NP = 2048
constexpr int kResYS = 64;                // columns per slice (MMA N)
constexpr int kResPW = 4;                 // producer warps
constexpr int kResStages = 5;
constexpr int kResMmaWarp = kDW + kResPW;
constexpr int kResThreads = (kDW + kResPW + 1) * 32;
constexpr int kResChunks = 17;            // 16 D chunks + 1 n_lin chunk per (step, group)
constexpr int kErrFlag = 4, kErrJ = 5, kErrInit = 6, kErrRead = 7;

struct ResParams {
    int n, S, npairs;
    const int32_t* fourT;
    const int32_t* q;
    const int64_t* kcorr;
    const int32_t* kconst;
    int32_t hclamp;
    const int32_t* bias_perm;           // [2048] or null
    uint64_t seed;
    uint32_t trial_offset;
    int nchains;
    uint32_t* flags;                    // [2 * npairs][32] (zeroed)
    int8_t* dbuf;                       // [2 * npairs][2][128][2048]
    int8_t* nlx;                        // [2 * npairs][2][128][128]
    uint64_t wait_ns;                   // limit of each wait of the exchange (the drain at exit keeps its own)
    uint32_t* out_spins;                // [nchains][64] (zeroed)
    unsigned long long* out_sum_sh;
    unsigned long long* out_sum_bs;
    unsigned long long* out_flips;
    int32_t* out_trace;
    int32_t* out_h;
    int* err;
    long long* prof;
};

__global__ void __launch_bounds__(kResThreads, 1)
    tensor_res_kernel(const __grid_constant__ CUtensorMap mapD, const __grid_constant__ CUtensorMap mapNL,
                      const __grid_constant__ CUtensorMap mapJ, const __grid_constant__ ResParams P) {
    constexpr int R = 8, NPAD = 2048;
    constexpr uint32_t TILE = kM * kKChunk;                 // 16 KB D / n_lin tile
    constexpr uint32_t JCHUNK = kResYS * kKChunk;           // 8 KB of resident J per K chunk
    constexpr uint32_t IDESC_H = (2u << 4) | (1u << 7) | (1u << 10) | (uint32_t(kResYS >> 3) << 17) | (uint32_t(kM >> 4) << 24);
    constexpr uint32_t IDESC_NL = (2u << 4) | (1u << 7) | (1u << 10) | (uint32_t(16 >> 3) << 17) | (uint32_t(kM >> 4) << 24);

    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* jres = smem;                                   // 16 x 8 KB
    uint8_t* ones = smem + 16 * JCHUNK;                     // 2 KB: row 0 = 128 x int8(1), rows 1..15 = 0
    uint8_t* stages = ones + 2048;                          // kResStages x 16 KB (1024-aligned)
    uint64_t* bars = reinterpret_cast<uint64_t*>(stages + kResStages * TILE);
    // bars: full[5], empty[5], hready[2], jbar, init, fields read[2], drain
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kResStages + 7);
    uint32_t* s_issued = tmem_slot + 1;                     // [kResStages] copies issued into each stage (drain)

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int cs = int(blockIdx.x % kResSlices);
    const int gp0 = int(blockIdx.x / kResSlices), gstride = int(gridDim.x / kResSlices);
    const int n = P.n, S = P.S;
    int* err = P.err;
    const uint32_t bar_full = smem_u32(bars), bar_empty = smem_u32(bars + kResStages);
    const uint32_t bar_h0 = smem_u32(bars + 2 * kResStages), bar_j = smem_u32(bars + 2 * kResStages + 2);
    const uint32_t bar_init = smem_u32(bars + 2 * kResStages + 3);   // decision warps: fields of a new pair set
    // decision warps: group g's fields for step m have been read, so its step-m tiles may now be accumulated (other
    // slices can publish step m before this CTA has read the fields it decides step m from)
    const uint32_t bar_rd0 = smem_u32(bars + 2 * kResStages + 4);
    const uint32_t bar_fin = smem_u32(bars + 2 * kResStages + 6);    // MMA thread: drain before TMEM is freed

    if (tid == 0) {
        for (int s = 0; s < kResStages; ++s) {
            mbar_init(bar_full + 8 * s, 1);
            mbar_init(bar_empty + 8 * s, 1);
        }
        mbar_init(bar_h0, 1);
        mbar_init(bar_h0 + 8, 1);
        mbar_init(bar_rd0, 1);
        mbar_init(bar_rd0 + 8, 1);
        mbar_init(bar_j, 1);
        mbar_init(bar_init, 1);
        mbar_init(bar_fin, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (tid < kResStages) s_issued[tid] = 0u;
    for (int i = tid; i < 2048; i += blockDim.x) ones[i] = i < 128 ? 1 : 0;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (warp == kResMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(256)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    // resident J slice: rows cs*64 .. +64 of J_perm, 16 chunks of 128 columns
    if (warp == kDW && lane == 0) {
        mbar_arrive_expect_tx(bar_j, 16 * JCHUNK);
        for (int kc = 0; kc < 16; ++kc) tma_load_2d(smem_u32(jres + kc * JCHUNK), &mapJ, kc * kKChunk, cs * kResYS, bar_j);
    }

    // decision-thread geometry: replica r (TMEM lane), column quarter qq: RNG lanes 8cs + 2qq + j, columns qq*16 ..
    const int r = (warp & 3) * 32 + lane, qq = warp >> 2;
    const uint32_t tl = uint32_t((warp & 3) * 32) << 16;
    uint32_t hph[2] = {0u, 0u};            // decision side: completed "h ready" phases per group
    uint32_t q = 0;                        // running chunk index (producers, MMA)
    bool jready = false;
    uint32_t iph = 0u;                     // MMA thread: completed "fields set" phases
    uint32_t rph[2] = {0u, 0u};            // MMA thread: completed "fields read" phases per group
    uint32_t q_ok = 0;                     // MMA thread: chunks 0 .. q_ok - 1 were waited for and consumed
    const bool prof = P.prof != nullptr;
    long long pr[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    const long long t_loop0 = clock64();

    for (int pw = gp0; pw < P.npairs; pw += gstride) {
        const int G[2] = {2 * pw, 2 * pw + 1};
        if (warp < kDW) {
            // ---------------- decision warps ----------------
            Xoshiro rng[2][2];
            uint32_t sw[2], dw[2], nlacc_prev[2] = {0u, 0u};
            int32_t nlin_prev[2] = {0, 0};
            long long flips[2] = {0, 0};
            const int chain[2] = {G[0] * kM + r, G[1] * kM + r};
#pragma unroll
            for (int g = 0; g < 2; ++g) {
                sw[g] = 0u;
                dw[g] = 0u;
                uint32_t db[4] = {0u, 0u, 0u, 0u};
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    rng_seed(rng[g][j], P.seed, P.trial_offset + uint32_t(chain[g]), uint32_t(8 * cs + 2 * qq + j));
#pragma unroll
                    for (int k = 0; k < R; ++k) {
                        const int col = j * R + k, i = k * 256 + 8 * cs + 2 * qq + j;
                        const uint32_t rv = rng_next(rng[g][j]);
                        const bool valid = i < n;
                        const uint32_t up = valid ? (rv >> 31) : 1u;
                        sw[g] |= up << col;
                        if (valid && !up) dw[g] |= 1u << col;
                        db[col >> 2] |= (valid ? (up ? 0x01u : 0xFFu) : 0u) << (8 * (col & 3));
                    }
                }
                int8_t* drow = P.dbuf + ((size_t(G[g]) * 2 + 1) * kM + r) * NPAD + cs * kResYS + qq * 16;
                *reinterpret_cast<uint4*>(drow) = make_uint4(db[0], db[1], db[2], db[3]);
                P.nlx[((size_t(G[g]) * 2 + 1) * kM + r) * 128 + cs * 4 + qq] = 0;
                // fields := bias, n_lin accumulator := 0
                uint32_t v[16];
#pragma unroll
                for (int e = 0; e < 16; ++e)
                    v[e] = P.bias_perm ? uint32_t(P.bias_perm[cs * kResYS + qq * 16 + e]) : 0u;
                tmem_st16(tmem + tl + uint32_t(g * kResYS + qq * 16), v);
                if (qq == 0) {
#pragma unroll
                    for (int e = 0; e < 16; ++e) v[e] = 0u;
                    tmem_st16(tmem + tl + uint32_t(128 + g * 16), v);
                }
            }
            tmem_wait_st();
            writer_fence();
            tc_fence_before();
            asm volatile("bar.sync 1, %0;" ::"r"(kDW * 32) : "memory");
            if (tid == 0) {
                // the MMA thread may accumulate into these fields only after they are set: tiles of other slices
                // can land before this CTA leaves its previous pair
                mbar_arrive(bar_init);
                flag_publish(P.flags + G[0] * kResSlices + cs, 1u);
                flag_publish(P.flags + G[1] * kResSlices + cs, 1u);
            }
            for (int m = 0; m <= S; ++m) {
#pragma unroll
                for (int g = 0; g < 2; ++g) {
                    long long t0 = prof ? clock64() : 0;
                    if (!err_set(err)) mbar_wait_for(bar_h0 + 8 * g, hph[g] & 1u, err, kErrHready, P.wait_ns);
                    ++hph[g];
                    tc_fence_after();
                    if (prof) { const long long t1 = clock64(); pr[0] += t1 - t0; t0 = t1; }
                    uint32_t hv[16], nv;
                    tmem_ld16(tmem + tl + uint32_t(g * kResYS + qq * 16), hv);
                    asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];"
                                 : "=r"(nv)
                                 : "r"(tmem + tl + uint32_t(128 + g * 16)));
                    tmem_wait_ld();
                    const int32_t nlin = int32_t(nv - nlacc_prev[g]);   // n_lin of step m - 1 (0 before step 0)
                    nlacc_prev[g] = nv;
                    const bool writer = chain[g] < P.nchains;
                    if (m >= 1 && writer && cs == 0 && qq == 0 && P.out_trace) P.out_trace[size_t(chain[g]) * S + (m - 1)] = nlin;
                    nlin_prev[g] = nlin;
                    if (m == S) {
                        // final fields: outputs
                        long long sh = 0, bs = 0;
#pragma unroll
                        for (int e = 0; e < 16; ++e) {
                            const int j = e / R, k = e % R, i = k * 256 + 8 * cs + 2 * qq + j;
                            if (i >= n) continue;
                            const bool up = (sw[g] >> e) & 1u;
                            const int32_t h = int32_t(hv[e]);
                            sh += up ? h : -h;
                            if (P.bias_perm) {
                                const int32_t b = P.bias_perm[cs * kResYS + qq * 16 + e];
                                bs += up ? b : -b;
                            }
                            if (writer) {
                                if (up) atomicOr(P.out_spins + size_t(chain[g]) * 64 + (i >> 5), 1u << (i & 31));
                                if (P.out_h) P.out_h[size_t(chain[g]) * n + i] = h;
                            }
                        }
                        if (writer) {
                            atomicAdd(P.out_sum_sh + chain[g], static_cast<unsigned long long>(sh));
                            atomicAdd(P.out_sum_bs + chain[g], static_cast<unsigned long long>(bs));
                            atomicAdd(P.out_flips + chain[g], static_cast<unsigned long long>(flips[g]));
                        }
                        continue;
                    }
                    const int t = m;
                    const int32_t fourT = __ldg(P.fourT + t), twoT = fourT >> 1, qv = __ldg(P.q + t);
                    const int32_t corr = step_corr(nlin_prev[g], __ldg(P.kcorr + t), __ldg(P.kconst + t));
                    const uint32_t lw = uint32_t(2 * twoT - 1);
                    const int32_t hcl = P.hclamp;
                    uint32_t db[4] = {0u, 0u, 0u, 0u};
                    uint32_t nsw = sw[g], ndw = 0u;
                    int nl = 0;
#pragma unroll
                    for (int e = 0; e < 16; ++e) {
                        const int j = e / R, k = e % R, i = k * 256 + 8 * cs + 2 * qq + j;
                        const uint32_t u = rng_next(rng[g][j]);
                        const bool valid = i < n;
                        const bool up = (sw[g] >> e) & 1u, dif = (dw[g] >> e) & 1u;
                        const int32_t h = int32_t(hv[e]);
                        int32_t hs = up ? h : -h;
                        if (hcl > 0) hs = max(-hcl, min(hs, hcl));
                        const int32_t x = qv + (dif ? corr : -corr);
                        const int32_t zt = hs * 65536 + x;
                        const int32_t thr = threshold16(u, fourT);
                        const bool fl = valid && (zt - thr < 0);
                        nl += (valid && (uint32_t(zt + twoT - 1) < lw)) ? 1 : 0;
                        if (fl) {
                            nsw ^= 1u << e;
                            ndw |= 1u << e;
                            db[e >> 2] |= (up ? 0xFEu : 0x02u) << (8 * (e & 3));
                            ++flips[g];
                        }
                    }
                    sw[g] = nsw;
                    dw[g] = ndw;
                    const int par = m & 1;
                    int8_t* drow = P.dbuf + ((size_t(G[g]) * 2 + par) * kM + r) * NPAD + cs * kResYS + qq * 16;
                    *reinterpret_cast<uint4*>(drow) = make_uint4(db[0], db[1], db[2], db[3]);
                    P.nlx[((size_t(G[g]) * 2 + par) * kM + r) * 128 + cs * 4 + qq] = int8_t(nl);
                    writer_fence();
                    tc_fence_before();
                    if (prof) { const long long t1 = clock64(); pr[1] += t1 - t0; t0 = t1; }
                    asm volatile("bar.sync 1, %0;" ::"r"(kDW * 32) : "memory");
                    if (tid == 0) {
                        mbar_arrive(bar_rd0 + 8 * g);
                        flag_publish(P.flags + G[g] * kResSlices + cs, uint32_t(m + 2));
                    }
                    if (prof) pr[2] += clock64() - t0;
                }
            }
            tc_fence_before();
        } else if (warp < kDW + kResPW) {
            // ---------------- producer warps (all lanes poll the 32 slice flags at once; lane 0 issues) ----------
            const int pwid = warp - kDW;
            uint32_t ready = 0u;                   // slices known to have published (m, g)
            for (int m = -1; m < S; ++m) {
                const int par = m & 1;
                for (int g = 0; g < 2; ++g) {
                    const int ay = (G[g] * 2 + par) * kM;
                    const uint32_t* fl = P.flags + G[g] * kResSlices;
                    const uint32_t target = uint32_t(m + 2);
                    ready = 0u;
                    for (int c = 0; c < kResChunks; ++c, ++q) {
                        if (int(q % kResPW) != pwid) continue;
                        // every branch below is warp-uniform: lane 0 decides and broadcasts
                        if (__shfl_sync(0xffffffffu, err_set(err) ? 1 : 0, 0)) continue;
                        const int s = int(q % kResStages);
                        const uint32_t u = q / kResStages;
                        const long long w0 = prof ? clock64() : 0;
                        if (u >= 1) {
                            const int w = lane == 0 ? (mbar_wait_for(bar_empty + 8 * s, (u - 1) & 1u, err, kErrEmpty, P.wait_ns) ? 1 : 0) : 1;
                            if (!__shfl_sync(0xffffffffu, w, 0)) continue;
                        }
                        const uint32_t need = c < 16 ? (3u << (2 * c)) : 0xffffffffu;
                        bool ok = (ready & need) == need;
                        if (!ok) {
                            const uint64_t t0 = globaltimer();
                            for (uint32_t k = 1;; ++k) {
                                uint32_t v;
                                asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(fl + lane) : "memory");
                                ready = __ballot_sync(0xffffffffu, v >= target);
                                if ((ready & need) == need) { ok = true; break; }
                                if ((k & 63u) == 0 && __shfl_sync(0xffffffffu, globaltimer() - t0 > P.wait_ns, 0)) {
                                    if (lane == 0) atomicCAS(err, 0, kErrFlag);
                                    break;
                                }
                            }
                        }
                        if (prof) pr[7] += clock64() - w0;
                        if (!ok) continue;
                        if (lane == 0) {
                            asm volatile("fence.proxy.async.global;" ::: "memory");
                            const uint32_t dst = smem_u32(stages + size_t(s) * TILE);
                            mbar_arrive_expect_tx(bar_full + 8 * s, TILE);
                            if (c < 16) tma_load_2d(dst, &mapD, c * kKChunk, ay, bar_full + 8 * s);
                            else tma_load_2d(dst, &mapNL, 0, ay, bar_full + 8 * s);
                            atomicAdd(s_issued + s, 1u);
                        }
                        __syncwarp();
                    }
                }
            }
        } else if (warp == kResMmaWarp) {
            // ---------------- MMA thread ----------------
            if (lane == 0) {
                // jready only once the J copy is seen landed: after a wait that gave up, the drain at exit waits
                // for it (a copy must not land in shared memory the CTA has released)
                if (!jready && !err_set(err)) jready = mbar_wait_for(bar_j, 0u, err, kErrJ, P.wait_ns);
                if (!err_set(err)) mbar_wait_for(bar_init, iph & 1u, err, kErrInit, P.wait_ns);
                ++iph;
                tc_fence_after();
                for (int m = -1; m < S; ++m) {
                    for (int g = 0; g < 2; ++g) {
                        const long long t0 = prof ? clock64() : 0;
                        if (m >= 0) {
                            if (!err_set(err)) mbar_wait_for(bar_rd0 + 8 * g, rph[g] & 1u, err, kErrRead, P.wait_ns);
                            ++rph[g];
                            tc_fence_after();
                        }
                        for (int c = 0; c < kResChunks; ++c, ++q) {
                            const int s = int(q % kResStages);
                            const uint32_t u = q / kResStages;
                            const long long w0 = prof ? clock64() : 0;
                            const bool ok = !err_set(err) && mbar_wait_for(bar_full + 8 * s, u & 1u, err, kErrFull, P.wait_ns);
                            if (ok) q_ok = q + 1;
                            if (prof) pr[5] += clock64() - w0;
                            tc_fence_after();
                            const long long i0 = prof ? clock64() : 0;
                            if (ok) {
                                const uint32_t a0 = smem_u32(stages + size_t(s) * TILE);
                                if (c < 16) {
                                    const uint32_t b0 = smem_u32(jres + c * JCHUNK);
#pragma unroll
                                    for (int kk = 0; kk < kKChunk / 32; ++kk)
                                        mma_i8(tmem + uint32_t(g * kResYS), sw128_desc(a0 + 32 * kk), sw128_desc(b0 + 32 * kk),
                                               IDESC_H, 1u);
                                } else {
                                    const uint32_t b0 = smem_u32(ones);
#pragma unroll
                                    for (int kk = 0; kk < kKChunk / 32; ++kk)
                                        mma_i8(tmem + uint32_t(128 + g * 16), sw128_desc(a0 + 32 * kk),
                                               sw128_desc(b0 + 32 * kk), IDESC_NL, 1u);
                                }
                            }
                            const long long i1 = prof ? clock64() : 0;
                            mma_commit(bar_empty + 8 * s);
                            if (prof) { const long long i2 = clock64(); pr[9] += i1 - i0; pr[10] += i2 - i1; }
                        }
                        mma_commit(bar_h0 + 8 * g);
                        if (prof) pr[6] += clock64() - t0;
                    }
                }
            } else {
                q += uint32_t(S + 1) * 2 * kResChunks;
            }
            __syncwarp();
        }
    }
    // every warp has left the loop, so no copy or MMA is issued after this barrier: the MMA thread waits (fixed
    // bound) for the copies still in flight -- after a wait that gave up, some were issued but never consumed -- and
    // for every MMA it issued, before the CTA releases shared memory and TMEM
    __syncthreads();
    if (warp == kResMmaWarp && lane == 0) {
        if (!jready) mbar_wait_for(bar_j, 0u, nullptr, 0, kWaitNs);
        for (int s = 0; s < kResStages; ++s) {
            // uses of stage s consumed (chunks q < q_ok with q mod stages = s), then the issued ones not consumed
            uint32_t u = q_ok > uint32_t(s) ? (q_ok - uint32_t(s) + kResStages - 1) / kResStages : 0u;
            for (uint32_t k = 0; u < s_issued[s] && k < 64; ++k, ++u) mbar_wait_for(bar_full + 8 * s, u & 1u, nullptr, 0, kWaitNs);
        }
        mma_commit(bar_fin);
        mbar_wait_for(bar_fin, 0u, nullptr, 0, kWaitNs);
    }
    if (prof) {
        long long* dst = P.prof + size_t(blockIdx.x) * kProfSlots;
        if (warp == 0 && lane == 0) {
            dst[0] = pr[0]; dst[1] = pr[1]; dst[2] = pr[2];
        }
        if (warp == kResMmaWarp && lane == 0) {
            dst[5] = pr[5]; dst[6] = pr[6]; dst[8] = clock64() - t_loop0; dst[9] = pr[9]; dst[10] = pr[10];
        }
        if (warp == kDW && lane == 0) dst[7] = pr[7];
    }
    __syncthreads();
    if (warp == kResMmaWarp) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256) : "memory");
    }
}

// ------------------------------------------------------------------------------------------------ fp4 kernel
// For NP = 2048 and couplings in {-1, 0, +1}: J and D are exact in e2m1 (packed fp4, two per byte), so the update
// runs as tcgen05.mma.kind::mxf4.block_scale (M 128, N 128, K 64) with every block scale 1.0 (ue8m0 0x7F) and fp32
// accumulation, exact for these integer fields. A cooperative persistent grid of 16 y-slices x G replica groups:
// CTA (group slot, slice cs) owns RNG lanes 16cs .. 16cs+15 (128 columns at p = 8l + k), keeps its J slice
// (128 rows x 2048 fp4 = 128 KB) resident, and runs one group of 128 replicas at a time. Per step:
//   8 decision warps: thread (replica r, half hf) owns quarters qq = 2hf, 2hf+1; quarter qq is lanes
//     16cs + 4qq + j (j < 4) x 8 rounds = 32 slots = TMEM columns qq*32 + j*8 + k. The step's draws were made while
//     the previous step's MMAs ran (the lane states live in TMEM); the thread reads its 64 fields, decides,
//     writes its 64 D nibbles (32 bytes) and two n_lin partial bytes to the group's exchange buffers, and after a
//     named barrier one thread publishes flag[g][cs] = m + 2 with a release store (the barrier orders every
//     writer's stores before it, and release is cumulative over them).
//   The same warps then fetch the step's D: tile t (128 replicas x 256 K, the slices of CTAs 2t and 2t+1) is
//     loaded once both slice flags are seen, with 16-byte asynchronous L2 copies (four per thread, up to 6 tiles in flight),
//     into a stage of an NS-deep shared-memory ring (NS = 6, 5, 4 or 3: compiled variants the host's tuner picks from) in the 128-byte-swizzled K-major layout the MMA reads; each
//     thread fences the async proxy and one lane per warp arrives on the stage's barrier. Each thread also sums
//     its replica's 64 n_lin partial bytes for the next step's correction.
//   The MMA thread: 4 mxf4 MMAs per tile into the fp32 fields in TMEM, a commit per stage to free it, and a commit
//     of "fields ready" after the 8th tile.
//   The poller warp: watches the 16 slice flags of the group in L2 and mirrors what it sees into shared memory
//     (acquire at gpu scope, release at cta scope), so the decision warps wait on shared memory.
// The exchange crosses L2 through the generic proxy only; the async proxy reads shared memory alone, after the
// loaders' proxy fence. 10 warps leave 168 registers per thread (a fifth warp on an SM sub-partition would cap
// them at 96).
constexpr int kF4Slices = 16;
constexpr int kF4YS = 128;
constexpr int kF4DW = 8;                  // decision warps (two quarters of 32 columns per thread)
constexpr int kF4Tiles = 8;               // D tiles per step (2048 fp4 = 1024 bytes per row, 128 bytes per tile)
constexpr int kF4MmaWarp = kF4DW;
constexpr int kF4PollWarp = kF4DW + 1;   // watches the group's 16 slice flags for the whole CTA
constexpr int kF4Threads = (kF4DW + 2) * 32;
constexpr int kF4Cluster = 1;            // CTAs per cluster (1: the scheduler spreads a group's slices; 4 GPC-local measured slower)
constexpr int kF4SfCol = 160;             // TMEM columns 144..255 hold scale factors 0x7F (1.0)
constexpr int kF4RngCol = 256;            // TMEM columns 256..319: RNG lane states, 32 per half hf
constexpr int kF4TmemCols = 512;
// mbarriers of an NS-stage ring: full[NS], empty[NS], fields ready, J loaded, drain
__host__ __device__ constexpr int f4_bars(int ns) { return 2 * ns + 3; }

struct F4Params {
    int n, S, ngroups;
    const int32_t* fourT;
    const int32_t* q;
    const int64_t* kcorr;
    const int32_t* kconst;
    int32_t hclamp;
    const int32_t* bias_perm;           // [2048] or null
    uint64_t seed;
    uint32_t trial_offset;
    int nchains;
    uint32_t* flags;                    // [ngroups][16] (zeroed)
    uint8_t* dbuf;                      // [ngroups][2][128][1024] packed e2m1
    int8_t* nlx;                        // [ngroups][2][128][128]: byte 4 cs + qq = partial n_lin
    uint64_t wait_ns;                   // limit of each wait of the exchange (the drain at exit keeps its own)
    uint32_t* out_spins;                // [nchains][64] (zeroed)
    unsigned long long* out_sum_sh;
    unsigned long long* out_sum_bs;
    unsigned long long* out_flips;
    int32_t* out_trace;
    int32_t* out_h;
    int* err;
    long long* prof;
};

// The step's draws for the thread's eight RNG lanes (quarter e = jj / 4, lane j = jj % 4; 8 rounds each, every
// lane's stream in round order), kept as their top 16 bits with the top bit flipped (u16 - 32768 as a signed
// 16-bit value): pk[16e + 4j + k/2] holds column j*8 + k of quarter e in its high half for even k and in its low half
// for odd k. The lane states live in TMEM (32 columns at taddr: a, b, c, d of lanes jj = 0..7), loaded, advanced and
// stored back here.
__device__ __forceinline__ void f4_draw(uint32_t taddr, uint32_t (&pk)[32]) {
    uint32_t st[32];
    tmem_ld32(taddr, st);
    tmem_wait_ld();
    Xoshiro rng[8];
#pragma unroll
    for (int jj = 0; jj < 8; ++jj) rng[jj] = Xoshiro{st[4 * jj], st[4 * jj + 1], st[4 * jj + 2], st[4 * jj + 3]};
#pragma unroll
    for (int k = 0; k < 8; ++k)
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) {
            const uint32_t u = rng_next(rng[jj]);
            uint32_t& w = pk[16 * (jj >> 2) + 4 * (jj & 3) + k / 2];
            if (k & 1) w |= (u >> 16) ^ 0x8000u;
            else w = (u & 0xffff0000u) ^ 0x80000000u;
        }
#pragma unroll
    for (int jj = 0; jj < 8; ++jj) {
        st[4 * jj] = rng[jj].a;
        st[4 * jj + 1] = rng[jj].b;
        st[4 * jj + 2] = rng[jj].c;
        st[4 * jj + 3] = rng[jj].d;
    }
    tmem_st32(taddr, st);
    tmem_wait_st();
}

// One decision pass over quarter E's 32 columns (fields hv, packed draws pk[16E ..]). Outputs the flip mask and
// the mask of slots inside the linear band -2T < z < 2T.
//   r = floor((u16 - 32768) * 4T / 65536) = mulhi((u16 - 32768) << 16, 4T);
//   s*h: the field in f32 with its sign flipped for s = -1 (bit 31 of ~sw), clamped when the range plan asks;
//   z = s*h*65536 + q -/+ corr through the exact conversion 1.5*2^23 + x (|x| < 2^22): the low 16 bits of that
//   encoding are x, so encoding << 16 = x * 65536 modulo 2^32.
template <bool CLAMP, int E>
__device__ __forceinline__ void f4_decide(const uint32_t (&pk)[32], const uint32_t (&hv)[32], uint32_t downs,
                                          uint32_t dw, int32_t xs, int32_t twocorr, int32_t fourT, int32_t c1,
                                          uint32_t lw, float hclf, uint32_t& fm, uint32_t& lm) {
    fm = 0u;
    lm = 0u;
#pragma unroll
    for (int col = 0; col < 32; ++col) {
        const int j = col >> 3, k = col & 7;
        const uint32_t w = pk[16 * E + 4 * j + k / 2];
        const uint32_t a16 = (k & 1) ? (w << 16) : (w & 0xffff0000u);     // (u16 - 32768) << 16
        const int32_t thr = __mulhi(int32_t(a16), fourT);
        float hsf = __uint_as_float(hv[col] ^ ((downs << (31 - col)) & 0x80000000u));
        if (CLAMP) hsf = fminf(fmaxf(hsf, -hclf), hclf);
        const int32_t zb = __float_as_int(hsf + 12582912.0f);
        int32_t zt = (zb << 16) + xs;
        if ((dw >> col) & 1u) zt += twocorr;
        if (zt < thr) fm |= 1u << col;
        if (uint32_t(zt + c1) < lw) lm |= 1u << col;
    }
}

// dS nibbles of 8 columns: flipped down->up = +2 (0x4), up->down = -2 (0xC); word w holds columns 8w .. 8w+7.
__device__ __forceinline__ uint4 f4_dnibbles(uint32_t fm, uint32_t fdn) {
    uint32_t db[4];
#pragma unroll
    for (int w = 0; w < 4; ++w) {
        uint32_t a8 = (fm >> (8 * w)) & 0xFFu, b8 = (fdn >> (8 * w)) & 0xFFu;
        a8 = (a8 | (a8 << 12)) & 0x000F000Fu; a8 = (a8 | (a8 << 6)) & 0x03030303u; a8 = (a8 | (a8 << 3)) & 0x11111111u;
        b8 = (b8 | (b8 << 12)) & 0x000F000Fu; b8 = (b8 | (b8 << 6)) & 0x03030303u; b8 = (b8 | (b8 << 3)) & 0x11111111u;
        db[w] = (a8 << 2) | (b8 << 3);
    }
    return make_uint4(db[0], db[1], db[2], db[3]);
}

// Profiling marks of decision thread 0 in one exchange (clock64), or unused.
struct F4ExMarks {
    long long flags0, flags7, stored0, stored7;
};

// 16-byte global -> shared copy through L2 only (cp.async.cg), and its commit-group bookkeeping.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// Wait until at most n of this thread's commit groups are pending (n folds to a constant once the caller's loop is
// unrolled; larger n waits for all).
__device__ __forceinline__ void cp_async_wait(int n) {
    switch (n) {
        case 1: asm volatile("cp.async.wait_group 1;" ::: "memory"); break;
        case 2: asm volatile("cp.async.wait_group 2;" ::: "memory"); break;
        case 3: asm volatile("cp.async.wait_group 3;" ::: "memory"); break;
        case 4: asm volatile("cp.async.wait_group 4;" ::: "memory"); break;
        case 5: asm volatile("cp.async.wait_group 5;" ::: "memory"); break;
        case 6: asm volatile("cp.async.wait_group 6;" ::: "memory"); break;
        default: asm volatile("cp.async.wait_group 0;" ::: "memory"); break;
    }
}

// Fetch one step's D (step m, parity m & 1; m = -1 is the initial state) into the ring: 8 tiles at ring positions
// q .. q+7, by the 256 decision threads: warp w copies tile rows 16w .. 16w+15, its copy instruction c covering the
// four whole 128-byte rows 16w + 4c .. 16w + 4c + 3 (lane: row + lane / 8, 16-byte chunk lane % 8), so each
// instruction touches four cache lines. Copies are asynchronous,
// one commit group per tile. Ring position t holds K chunk (t + rot) mod 8, so a CTA starts with the tile holding its
// own slice. Tile t goes out as soon as its two slices are published, and tile t - 1 is marked full right after, so
// the MMAs start on the first tile while later slices are still being published (marking tiles 0-3 full only after
// tiles 0-5 had gone out cost 6 % of the step). Tiles NS .. 7 wait for the MMAs of tiles 0 .. 7 - NS to free their
// stages; those tiles were marked full before (tile t - NS <= t - 2 is marked full before tile t is issued). A tile is marked full once its group has landed: the thread fences the
// async proxy and its warp arrives on the stage's barrier. Returns the replica's n_lin (the sum of its 64 partial
// bytes) when want_nlin, else 0. ok (warp-uniform) is false once this warp saw an error; every wait is bounded, and
// after an error the warp stops copying and arriving but still waits for the copies it has in flight.
template <int NS>
__device__ __forceinline__ int32_t f4_exchange(const F4Params& P, int g, int m, uint32_t stages_u32, uint32_t bar_full,
                                               uint32_t bar_empty, uint32_t q, int tid, int r, bool want_nlin,
                                               const uint32_t* s_flag, uint32_t tbase, int rot, bool& ok, bool prof,
                                               F4ExMarks& mk) {
    constexpr uint32_t TILE = kM * kKChunk;
    static_assert(NS >= 2 && NS <= kF4Tiles && kF4Tiles == 8, "rotation by a 3-bit mask, and two stages in flight");
    const int lane = tid & 31;
    int* err = P.err;
    const int par = m & 1;
    const uint32_t target = tbase + uint32_t(m + 2);    // the slice flags' value for step m, in the mirror's count
    const int row0 = (tid >> 5) * 16 + (lane >> 3), ch = lane & 7;    // first tile row, 16-byte chunk of this thread
    const uint8_t* src = P.dbuf + (size_t(g * 2 + par) * kM + row0) * 1024 + ch * 16;
    // 128-byte swizzle: chunk ch of row x at ch ^ (x mod 8); rows row0 + 4c have x mod 8 = (row0 mod 8) ^ 4 (c & 1)
    const uint32_t dst0 = uint32_t(row0 * 128 + ((ch ^ (row0 & 7)) << 4));
    const uint32_t dst1 = uint32_t(row0 * 128 + ((ch ^ ((row0 + 4) & 7)) << 4));
    // copy tile t into its stage once its slices are published (and, for t >= 6, its stage is free)
    auto issue = [&](int t) {
        const uint32_t qt = q + uint32_t(t), s = qt % NS, u = qt / NS;
        const int tk = (t + rot) & (kF4Tiles - 1);     // K chunk of ring position t (the CTA's own tile first)
        if (ok && u >= 1) ok = __all_sync(0xffffffffu, mbar_wait_for(bar_empty + 8 * s, (u - 1) & 1u, err, kErrEmpty, P.wait_ns));
        if (ok) {
            // both slices published: every lane acquires the poller's mirror of their flags (cta scope; the poller
            // acquired them at gpu scope)
            const uint32_t fa = smem_u32(s_flag + 2 * tk), fb = smem_u32(s_flag + 2 * tk + 1);
            const uint64_t t0 = globaltimer();
            bool seen = false;
            for (uint32_t k = 1;; ++k) {
                uint32_t va, vb;
                asm volatile("ld.acquire.cta.shared::cta.u32 %0, [%1];" : "=r"(va) : "r"(fa) : "memory");
                asm volatile("ld.acquire.cta.shared::cta.u32 %0, [%1];" : "=r"(vb) : "r"(fb) : "memory");
                if (va >= target && vb >= target) { seen = true; break; }
                if ((k & 255u) == 0 && globaltimer() - t0 > P.wait_ns) {
                    atomicCAS(err, 0, kErrFlag);
                    break;
                }
            }
            ok = __all_sync(0xffffffffu, seen);
        }
        if (prof && lane == 0) {
            if (t == 0) mk.flags0 = clock64();
            if (t == kF4Tiles - 1) mk.flags7 = clock64();
        }
        if (ok) {
            const uint32_t st = stages_u32 + s * TILE;
#pragma unroll
            for (int c = 0; c < 4; ++c)
                cp_async16(st + uint32_t(c * 512) + ((c & 1) ? dst1 : dst0), src + size_t(c) * 4096 + tk * 128);
        }
        cp_async_commit();          // one group per tile, empty when the copies were skipped
    };
    // mark tile t full once its group has landed; `later` groups were committed after it
    auto arrive = [&](int t, int later) {
        cp_async_wait(later);
        if (ok) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(bar_full + 8 * ((q + uint32_t(t)) % NS));
        }
        if (prof && lane == 0) {
            if (t == 0) mk.stored0 = clock64();
            if (t == kF4Tiles - 1) mk.stored7 = clock64();
        }
    };
    issue(0);
#pragma unroll
    for (int t = 1; t < kF4Tiles; ++t) {
        issue(t);
        arrive(t - 1, 1);
    }
    arrive(kF4Tiles - 1, 0);
    int32_t nl = 0;
    if (ok && want_nlin) {
        // every warp saw all 16 flags before its last tile
        const uint4* np = reinterpret_cast<const uint4*>(P.nlx + (size_t(g * 2 + par) * kM + r) * 128);
        uint4 nv[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) nv[i] = __ldcg(np + i);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            nl = __dp4a(int(nv[i].x), 0x01010101, nl);
            nl = __dp4a(int(nv[i].y), 0x01010101, nl);
            nl = __dp4a(int(nv[i].z), 0x01010101, nl);
            nl = __dp4a(int(nv[i].w), 0x01010101, nl);
        }
    }
    return nl;
}

template <int NS>
__global__ void __launch_bounds__(kF4Threads, 1)
    tensor_fp4_kernel(const __grid_constant__ CUtensorMap mapJ, const __grid_constant__ F4Params P) {
    constexpr int R = 8;                                    // rounds
    constexpr uint32_t TILE = kM * kKChunk;                 // 16 KB tile (128 rows x 128 bytes)
    constexpr uint32_t IDESC_F4 = (1u << 7) | (1u << 10) | (uint32_t(kF4YS >> 3) << 17) | (1u << 23) | (uint32_t(kM >> 4) << 24);

    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* jres = smem;                                   // 8 x 16 KB
    uint8_t* stages = smem + 8 * TILE;                      // NS x 16 KB
    uint64_t* bars = reinterpret_cast<uint64_t*>(stages + NS * TILE);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + f4_bars(NS));
    __shared__ volatile long long s_pub[2];      // profiling: clock64 of this CTA's flag publish, by step parity
    __shared__ uint32_t s_flag[kF4Slices];       // the poller's mirror of the slice flags: gi * (S + 2) + flag

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int cs = int(blockIdx.x % kF4Slices);
    const int gs0 = int(blockIdx.x / kF4Slices), gstride = int(gridDim.x / kF4Slices);
    const int n = P.n, S = P.S;
    int* err = P.err;
    const uint32_t bar_full = smem_u32(bars), bar_empty = smem_u32(bars + NS);
    const uint32_t bar_h = smem_u32(bars + 2 * NS), bar_j = smem_u32(bars + 2 * NS + 1);
    const uint32_t bar_fin = smem_u32(bars + 2 * NS + 2);    // MMA thread: drain before TMEM is freed

    if (tid < kF4Slices) s_flag[tid] = 0u;
    if (tid == 0) {
        for (int s = 0; s < NS; ++s) {
            mbar_init(bar_full + 8 * s, kF4DW);
            mbar_init(bar_empty + 8 * s, 1);
        }
        mbar_init(bar_h, 1);
        mbar_init(bar_j, 1);
        mbar_init(bar_fin, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == kF4MmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kF4TmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    if (warp == kF4MmaWarp && lane == 0) {
        mbar_arrive_expect_tx(bar_j, 8 * TILE);
        for (int kc = 0; kc < 8; ++kc) tma_load_2d(smem_u32(jres + kc * TILE), &mapJ, kc * kKChunk, cs * kF4YS, bar_j);
    }
    // scale factors: columns 144..255 of every lane := 0x7F7F7F7F (ue8m0 1.0); warps 0..3 cover the 128 lanes
    const uint32_t tl = uint32_t((warp & 3) * 32) << 16;
    if (warp < 4) {
        uint32_t v[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) v[e] = 0x7F7F7F7Fu;
        for (int c0 = 144; c0 < 256; c0 += 16) tmem_st16(tmem + tl + uint32_t(c0), v);
        tmem_wait_st();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();

    const int r = (warp & 3) * 32 + lane, hf = warp >> 2;
    uint32_t hph = 0u, q = 0;
    bool jready = false;
    const bool prof = P.prof != nullptr;
    long long pa = 0, pb = 0, pc = 0, pd = 0, pe = 0;   // phase cycle totals; meaning depends on the warp's role
    long long p_f0 = 0, p_f7 = 0, p_s0 = 0, p_s7 = 0;   // decision thread 0: marks after its own publish
    const long long t_loop0 = clock64();

    for (int g = gs0, gi = 0; g < P.ngroups; g += gstride, ++gi) {
        const uint32_t tbase = uint32_t(gi) * uint32_t(S + 2);   // this group's offset in the flag mirror
        if (warp < kF4DW) {
            // ---------------- decision warps ----------------
            const int chain = g * kM + r;
            const bool writer = chain < P.nchains;
            uint32_t sw[2] = {0u, 0u}, dw[2] = {0u, 0u}, vmask[2] = {0u, 0u};
            long long flips = 0;
            F4ExMarks mk{};
            const uint32_t trng = tmem + tl + uint32_t(kF4RngCol + 32 * hf);
            // initial spins from each lane's first draw per round, the state D = s0 (parity 1), the lane states and
            // the fields h = b; once per group, so not unrolled over the two quarters
#pragma unroll 1
            for (int e = 0; e < 2; ++e) {
                const int qq = 2 * hf + e;
                Xoshiro rng[4];
                uint32_t db[4] = {0u, 0u, 0u, 0u}, swq = 0u, dwq = 0u, vmq = 0u;
#pragma unroll
                for (int j = 0; j < 4; ++j) rng_seed(rng[j], P.seed, P.trial_offset + uint32_t(chain), uint32_t(16 * cs + 4 * qq + j));
#pragma unroll
                for (int k = 0; k < R; ++k)
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int col = j * R + k, i = k * 256 + 16 * cs + 4 * qq + j;
                        const uint32_t rv = rng_next(rng[j]);
                        const bool valid = i < n;
                        const uint32_t up = valid ? (rv >> 31) : 1u;
                        swq |= up << col;
                        if (valid) vmq |= 1u << col;
                        if (valid && !up) dwq |= 1u << col;
                        db[col >> 3] |= (valid ? (up ? 0x2u : 0xAu) : 0u) << (4 * (col & 7));   // e2m1 +1 / -1
                    }
                if (e == 0) { sw[0] = swq; dw[0] = dwq; vmask[0] = vmq; }
                else { sw[1] = swq; dw[1] = dwq; vmask[1] = vmq; }
                uint8_t* drow = P.dbuf + ((size_t(g) * 2 + 1) * kM + r) * 1024 + cs * 64 + qq * 16;
                *reinterpret_cast<uint4*>(drow) = make_uint4(db[0], db[1], db[2], db[3]);
                uint32_t st[16];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    st[4 * j] = rng[j].a;
                    st[4 * j + 1] = rng[j].b;
                    st[4 * j + 2] = rng[j].c;
                    st[4 * j + 3] = rng[j].d;
                }
                tmem_st16(trng + uint32_t(16 * e), st);
#pragma unroll
                for (int h2 = 0; h2 < 2; ++h2) {
#pragma unroll
                    for (int x = 0; x < 16; ++x)
                        st[x] = __float_as_uint(P.bias_perm ? float(P.bias_perm[cs * kF4YS + qq * 32 + h2 * 16 + x]) : 0.f);
                    tmem_st16(tmem + tl + uint32_t(qq * 32 + h2 * 16), st);
                }
                tmem_wait_st();
            }
            // the fields are set before any tile of this group is marked full, so before the MMA thread accumulates
            tc_fence_before();
            asm volatile("bar.sync 1, %0;" ::"r"(kF4DW * 32) : "memory");
            if (tid == 0) flag_release(P.flags + g * kF4Slices + cs, 1u);
            uint32_t pk[32];
            // the run's error word is read once per step, off the critical path (its load overlaps the draws);
            // a wait of this warp that gives up clears ok at once
            const bool eok = !err_set(err);
            f4_draw(trng, pk);
            bool ok = __all_sync(0xffffffffu, eok);
            int32_t nlin_next = f4_exchange<NS>(P, g, -1, smem_u32(stages), bar_full, bar_empty, q, tid, r, false, s_flag, tbase, cs >> 1,
                                            ok, false, mk);
            q += kF4Tiles;
            const float hclf = float(P.hclamp);
            for (int m = 0; m <= S; ++m) {
                long long t0 = prof ? clock64() : 0;
                // this step's table entries, loaded before the wait for the fields
                const int t = m < S ? m : S - 1;
                const int32_t fourT = __ldg(P.fourT + t), qv = __ldg(P.q + t), kconst = __ldg(P.kconst + t);
                const int64_t kcorr = __ldg(P.kcorr + t);
                if (ok) ok = __all_sync(0xffffffffu, mbar_wait_for(bar_h, hph & 1u, err, kErrHready, P.wait_ns));
                ++hph;
                tc_fence_after();
                if (prof) {
                    const long long t1 = clock64();
                    pa += t1 - t0;
                    t0 = t1;
                }
                const int32_t nlin_prev = nlin_next;       // n_lin of step m - 1 (0 before the first step)
                if (m >= 1 && writer && cs == 0 && hf == 0 && P.out_trace) P.out_trace[size_t(chain) * S + (m - 1)] = nlin_prev;
                if (m == S) {
                    // read-out, once per group: 16-column chunks from TMEM, not unrolled
                    long long sh = 0, bs = 0;
#pragma unroll 1
                    for (int c4 = 0; c4 < 4; ++c4) {
                        const int qq = 2 * hf + (c4 >> 1);
                        const uint32_t swq = (c4 >> 1) ? sw[1] : sw[0];
                        uint32_t hc[16];
                        tmem_ld16(tmem + tl + uint32_t(hf * 64 + 16 * c4), hc);
                        tmem_wait_ld();
#pragma unroll
                        for (int x = 0; x < 16; ++x) {
                            const int col = (c4 & 1) * 16 + x;      // column within quarter qq
                            const int j = col / R, k = col % R, i = k * 256 + 16 * cs + 4 * qq + j;
                            if (i >= n) continue;
                            const bool up = (swq >> col) & 1u;
                            const int32_t h = __float2int_rn(__uint_as_float(hc[x]));
                            sh += up ? h : -h;
                            if (P.bias_perm) {
                                const int32_t b = P.bias_perm[cs * kF4YS + qq * 32 + col];
                                bs += up ? b : -b;
                            }
                            if (writer) {
                                if (up) atomicOr(P.out_spins + size_t(chain) * 64 + (i >> 5), 1u << (i & 31));
                                if (P.out_h) P.out_h[size_t(chain) * n + i] = h;
                            }
                        }
                    }
                    if (writer) {
                        atomicAdd(P.out_sum_sh + chain, static_cast<unsigned long long>(sh));
                        atomicAdd(P.out_sum_bs + chain, static_cast<unsigned long long>(bs));
                        atomicAdd(P.out_flips + chain, static_cast<unsigned long long>(flips));
                    }
                    continue;
                }
                const int32_t twoT = fourT >> 1;
                const int32_t corr = step_corr(nlin_prev, kcorr, kconst);
                const uint32_t lw = uint32_t(2 * twoT - 1);
                const int32_t xs = qv - corr, c1 = twoT - 1, twocorr = 2 * corr;
                const int par = m & 1;
                uint4 dq[2];
                uint32_t nlb = 0u;
                uint32_t hv0[32], hv1[32];            // the two quarters' fields, loaded together
                tmem_ld32(tmem + tl + uint32_t(hf * 64), hv0);
                tmem_ld32(tmem + tl + uint32_t(hf * 64 + 32), hv1);
                tmem_wait_ld();
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const uint32_t downs = ~sw[e];    // bit set: s = -1, the field's sign flips
                    uint32_t fm, lm;                  // flip mask, linear-band mask
                    if (e == 0) {
                        if (P.hclamp > 0) f4_decide<true, 0>(pk, hv0, downs, dw[0], xs, twocorr, fourT, c1, lw, hclf, fm, lm);
                        else f4_decide<false, 0>(pk, hv0, downs, dw[0], xs, twocorr, fourT, c1, lw, hclf, fm, lm);
                    } else {
                        if (P.hclamp > 0) f4_decide<true, 1>(pk, hv1, downs, dw[1], xs, twocorr, fourT, c1, lw, hclf, fm, lm);
                        else f4_decide<false, 1>(pk, hv1, downs, dw[1], xs, twocorr, fourT, c1, lw, hclf, fm, lm);
                    }
                    fm &= vmask[e];
                    lm &= vmask[e];
                    nlb |= uint32_t(__popc(lm)) << (8 * e);
                    flips += __popc(fm);
                    dq[e] = f4_dnibbles(fm, fm & sw[e]);
                    sw[e] ^= fm;
                    dw[e] = fm;
                }
                uint8_t* drow = P.dbuf + ((size_t(g) * 2 + par) * kM + r) * 1024 + cs * 64 + hf * 32;
                reinterpret_cast<uint4*>(drow)[0] = dq[0];
                reinterpret_cast<uint4*>(drow)[1] = dq[1];
                *reinterpret_cast<uint16_t*>(P.nlx + ((size_t(g) * 2 + par) * kM + r) * 128 + cs * 4 + hf * 2) = uint16_t(nlb);
                tc_fence_before();
                if (prof) { const long long t1 = clock64(); pb += t1 - t0; t0 = t1; }
                asm volatile("bar.sync 1, %0;" ::"r"(kF4DW * 32) : "memory");
                if (tid == 0) flag_release(P.flags + g * kF4Slices + cs, uint32_t(m + 2));
                long long tpub = 0;
                if (prof) {
                    tpub = clock64();
                    pc += tpub - t0;
                    t0 = tpub;
                    if (tid == 0) s_pub[m & 1] = tpub;
                }
                // the next step's draws while the other slices publish; the run's error word is read here too
                const bool eok2 = !err_set(err);
                if (m + 1 < S) f4_draw(trng, pk);
                ok = ok && __all_sync(0xffffffffu, eok2);
                if (prof) { const long long t1 = clock64(); pd += t1 - t0; t0 = t1; }
                nlin_next = f4_exchange<NS>(P, g, m, smem_u32(stages), bar_full, bar_empty, q, tid, r, true, s_flag, tbase, cs >> 1,
                                        ok, prof, mk);
                q += kF4Tiles;
                if (prof) {
                    pe += clock64() - t0;
                    tpub = s_pub[m & 1];            // thread 0's publish: the same barrier episode for every warp
                    p_f0 += mk.flags0 - tpub;
                    p_f7 += mk.flags7 - tpub;
                    p_s0 += mk.stored0 - tpub;
                    p_s7 += mk.stored7 - tpub;
                }
            }
            tc_fence_before();
        } else if (warp == kF4MmaWarp) {
            // ---------------- MMA thread ----------------
            if (lane == 0) {
                // jready only once the J copy is seen landed: after a wait that gave up, the drain at exit waits
                // for it (a copy must not land in shared memory the CTA has released)
                if (!jready && !err_set(err)) jready = mbar_wait_for(bar_j, 0u, err, kErrJ, P.wait_ns);
                long long p_first = 0, p_last = 0, p_h = 0, tf0 = 0, tf7 = 0, pmid[5] = {0, 0, 0, 0, 0}, pti[8] = {}, ptw[8] = {};
                bool mok = true;           // false once a wait gave up or the error word was seen set
                for (int m = -1; m < S; ++m) {
                    const long long t0 = prof ? clock64() : 0;
                    mok = mok && !err_set(err);    // once per step, while the thread waits for the first tile
                    for (int t = 0; t < kF4Tiles; ++t, ++q) {
                        const int s = int(q % NS);
                        const uint32_t u = q / NS;
                        const long long w0 = prof ? clock64() : 0;
                        mok = mok && mbar_wait_for(bar_full + 8 * s, u & 1u, err, kErrFull, P.wait_ns);
                        const bool ok = mok;
                        if (prof) {
                            const long long w1 = clock64();
                            pa += w1 - w0;
                            if (t == 0) tf0 = w1;
                            if (t == kF4Tiles - 1) tf7 = w1;
                            if (t >= 2 && t <= 6 && m >= 0) pmid[t - 2] += w1 - s_pub[m & 1];
                        }
                        tc_fence_after();
                        const long long i0 = prof ? clock64() : 0;
                        if (ok) {
                            const uint32_t a0 = smem_u32(stages + size_t(s) * TILE);
                            const uint32_t b0 = smem_u32(jres + ((t + (cs >> 1)) & (kF4Tiles - 1)) * TILE);
#pragma unroll
                            for (int kk = 0; kk < kKChunk / 32; ++kk)
                                mma_mxf4(tmem, sw128_desc(a0 + 32 * kk), sw128_desc(b0 + 32 * kk), IDESC_F4,
                                         tmem + uint32_t(kF4SfCol), tmem + uint32_t(kF4SfCol + 32));
                        }
                        const long long i1 = prof ? clock64() : 0;
                        mma_commit(bar_empty + 8 * s);
                        if (prof) {
                            const long long i2 = clock64();
                            pc += i1 - i0;
                            pd += i2 - i1;
                            if (m >= 0) {
                                pti[t] += i1 - s_pub[m & 1];
                                ptw[t] += i0 - w0;
                            }
                        }
                    }
                    mma_commit(bar_h);
                    if (prof) {
                        const long long th = clock64();
                        pb += th - t0;
                        if (m >= 0) {
                            const long long pub = s_pub[m & 1];
                            p_first += tf0 - pub;
                            p_last += tf7 - pub;
                            p_h += th - pub;
                        }
                    }
                }
                if (prof) {
                    long long* dst = P.prof + size_t(blockIdx.x) * kProfSlots;
                    dst[11] += p_first;
                    dst[12] += p_last;
                    dst[14] += p_h;
                    for (int i = 0; i < 5; ++i) dst[19 + i] += pmid[i];
                    for (int i = 0; i < 8; ++i) {
                        dst[40 + i] += pti[i];
                        dst[48 + i] += ptw[i];
                    }
                }
            } else {
                q += uint32_t(S + 1) * kF4Tiles;
            }
            __syncwarp();
        } else if (warp == kF4PollWarp) {
            // ---------------- flag poller ----------------
            // lane j < 16 watches slice j's flag (values 1 .. S + 1 for steps -1 .. S - 1) with acquire loads at gpu
            // scope and releases what it newly sees to the CTA through s_flag, so the decision warps wait on shared
            // memory, not L2 (relaxed loads with a fence per new observation measured 1.4 % slower: the fence delayed
            // the next poll)
            const uint32_t* fl = P.flags + g * kF4Slices;
            uint32_t seen = 0u;
            bool pok = !err_set(err);
            for (uint32_t target = 1; pok && target <= uint32_t(S + 1); ++target) {
                const uint64_t t0 = globaltimer();
                for (uint32_t k = 1;; ++k) {
                    uint32_t v = 0u;
                    if (lane < kF4Slices)
                        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(fl + lane) : "memory");
                    const bool fresh = lane < kF4Slices && v > seen;
                    if (__any_sync(0xffffffffu, fresh)) {
                        if (fresh) {
                            asm volatile("st.release.cta.shared::cta.u32 [%0], %1;" ::"r"(smem_u32(s_flag + lane)),
                                         "r"(tbase + v)
                                         : "memory");
                            seen = v;
                        }
                    }
                    if (__all_sync(0xffffffffu, lane >= kF4Slices || seen >= target)) break;
                    if ((k & 63u) == 0) {
                        const bool late = lane == 0 && globaltimer() - t0 > P.wait_ns;
                        if (late) atomicCAS(err, 0, kErrFlag);
                        if (__shfl_sync(0xffffffffu, (late || (lane == 0 && err_set(err))) ? 1 : 0, 0)) {
                            pok = false;
                            break;
                        }
                    }
                }
            }
        }
    }
    if (warp == kF4MmaWarp && lane == 0) {
        // drain: every MMA issued has completed (and the J copy has landed) before TMEM and shared memory go away
        if (!jready) mbar_wait_for(bar_j, 0u, nullptr, 0, kWaitNs);
        mma_commit(bar_fin);
        mbar_wait_for(bar_fin, 0u, nullptr, 0, kWaitNs);
    }
    if (prof) {
        long long* dst = P.prof + size_t(blockIdx.x) * kProfSlots;
        if (tid == 0) {
            dst[0] = pa; dst[1] = pb; dst[2] = pc; dst[3] = pd; dst[4] = pe;
            dst[15] = p_f0; dst[16] = p_f7; dst[17] = p_s0; dst[18] = p_s7;
        }
        if (warp < kF4DW && lane == 0) {
            dst[24 + warp] = p_s7;
            dst[32 + warp] = p_f7;
        }
        if (warp == kF4MmaWarp && lane == 0) {
            dst[5] = pa; dst[6] = pb; dst[8] = clock64() - t_loop0; dst[9] = pc; dst[10] = pd;
        }
    }
    __syncthreads();
    if (warp == kF4MmaWarp) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kF4TmemCols) : "memory");
    }
}

// ------------------------------------------------------------------------------------------------ host side
// 2-D uint8 tensor [rows][cols] (cols contiguous), box = box_rows x 128 bytes, 128-byte swizzle.
bool make_map(CUtensorMap* map, void* base, uint64_t cols, uint64_t rows, uint32_t box_rows) {
    return make_map_2d(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, base, cols, rows, uint32_t(kKChunk), box_rows);
}

template <int R>
size_t smem_bytes_t() {
    constexpr size_t NC = 16 * R;
    return 1024 + kStages * (size_t(kM) * kKChunk + NC * kKChunk) + (2 * kStages + 1) * 8 + 16 + kM * 4;
}

template <int R>
int launch_t(const TensorParams& P, int groups, const CUtensorMap& A, const CUtensorMap& B, cudaStream_t st,
             std::string* why) {
    auto fn = tensor_kernel<R>;
    const size_t smem = smem_bytes_t<R>();
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e == cudaSuccess) e = cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) {
        if (why) *why = std::string("kernel attributes: ") + cudaGetErrorString(e);
        return -2;
    }
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = kC;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cfg.gridDim = dim3(kC * groups);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    e = cudaLaunchKernelEx(&cfg, fn, A, B, P);
    if (e != cudaSuccess) {
        if (why) *why = std::string("launch: ") + cudaGetErrorString(e);
        return -2;
    }
    return 0;
}

template <int R>
int max_clusters_t(int* out) {
    auto fn = tensor_kernel<R>;
    const size_t smem = smem_bytes_t<R>();
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e == cudaSuccess) e = cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = kC;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cfg.gridDim = dim3(kC);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = smem;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveClusters(out, fn, &cfg);
    return int(e);
}

size_t res_smem_bytes() {
    return 1024 + 16 * size_t(kResYS) * kKChunk + 2048 + size_t(kResStages) * kM * kKChunk + (2 * kResStages + 7) * 8 + 16 +
           4 * kResStages;
}

// Concurrent pair slots of the resident kernel (32 co-resident CTAs each).
int res_pair_slots(int npairs, int* out) {
    auto fn = tensor_res_kernel;
    const size_t smem = res_smem_bytes();
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    int per_sm = 0, dev = 0, sms = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kResThreads, smem);
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return int(e);
    *out = std::max(0, std::min(npairs, (per_sm * sms) / kResSlices));
    return 0;
}

}  // namespace

int tensor_geometry(int n, int nchains, TensorGeometry* g) {
    const int np = std::max(2048, ((n + 255) / 256) * 256);
    const int R = np / 256;
    if (stream_supported(n)) {
        g->cluster = 1;
        g->ctas = 128;
        g->max_active_clusters = 128;
        return 0;
    }
    if (R == 8) {
        const int npairs = ((nchains + kM - 1) / kM + 1) / 2;
        int slots = 0;
        const int rc = res_pair_slots(npairs, &slots);
        g->cluster = 1;
        g->ctas = kResSlices * slots;
        g->max_active_clusters = g->ctas;
        return rc;
    }
    g->cluster = kC;
    g->ctas = kC * ((nchains + kM - 1) / kM);
    if (R == 12) return max_clusters_t<12>(&g->max_active_clusters);
    if (R == 16) return max_clusters_t<16>(&g->max_active_clusters);
    return int(cudaErrorInvalidValue);
}

bool tensor_supported(int n, int K, int nchains) {
    (void)K;
    const int np = std::max(2048, ((n + 255) / 256) * 256);
    const int R = np / 256;
    return nchains >= 1 && (R == 8 || R == 12 || R == 16 || stream_supported(n));
}

int tensor_build_instance(const int8_t* J, int n, TensorInstance* out, std::string* why) {
    const int np = std::max(2048, ((n + 255) / 256) * 256);
    const int R = np / 256, nc = 16 * R;
    if (!(R == 8 || R == 12 || R == 16 || stream_supported(n))) {
        if (why) *why = "tensor engine supports NP in {2048, 3072, 4096} and (8192, 16384]";
        return -1;
    }
    const bool big = stream_supported(n);
    std::vector<int> p(np);
    if (big) {
        stream_permutation(np, &p);
    } else {
        for (int i = 0; i < np; ++i) {
            const int l = i % 256, k = i / 256, cc = l / 16, jl = l % 16;
            p[i] = cc * nc + jl * R + k;
        }
    }
    const int npp = big ? stream_width() : np;
    std::vector<int8_t> Jp(size_t(npp) * npp, 0);
    bool unit = true;
    int64_t rowmax = 0;
    for (int x = 0; x < n; ++x) {
        int64_t rs = 0;
        for (int y = 0; y < n; ++y) {
            const int8_t v = J[size_t(x) * n + y];
            Jp[size_t(p[y]) * npp + p[x]] = v;   // row = y (N), col = x (K)
            rs += v < 0 ? -v : v;
            unit = unit && v >= -1 && v <= 1;
        }
        rowmax = std::max(rowmax, rs);
    }
    out->n = n;
    out->np = np;
    out->npp = npp;
    out->stream = big;
    out->perm.assign(p.begin(), p.end());
    out->rowsum_max = rowmax;
    cudaError_t e = cudaMalloc(&out->d_J, Jp.size());
    if (e == cudaSuccess) e = cudaMemcpy(out->d_J, Jp.data(), Jp.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && unit && R == 8 && !big) {
        // packed e2m1, two per byte (even K index in the low nibble): +1 -> 0x2, -1 -> 0xA, 0 -> 0x0
        std::vector<uint8_t> J4(size_t(np) * np / 2, 0);
        for (size_t y = 0; y < size_t(np); ++y)
            for (size_t x = 0; x < size_t(np); ++x) {
                const int8_t v = Jp[y * np + x];
                const uint8_t code = v > 0 ? 0x2 : (v < 0 ? 0xA : 0x0);
                J4[(y * np + x) >> 1] |= uint8_t(code << (4 * (x & 1)));
            }
        e = cudaMalloc(&out->d_J4, J4.size());
        if (e == cudaSuccess) e = cudaMemcpy(out->d_J4, J4.data(), J4.size(), cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) {
        if (why) *why = std::string("upload J: ") + cudaGetErrorString(e);
        return -2;
    }
    out->bytes = Jp.size();
    return 0;
}

// Largest |h| the fp4 kernel may meet is bias_absmax + rowsum_max; it stays below 2^14, where every partial sum of
// the fp32 accumulator is an integer held exactly with 10 bits to spare.
bool tensor_fp4_eligible(const TensorInstance* ti, int64_t bias_absmax) {
    return ti->d_J4 != nullptr && ti->np == 2048 && ti->rowsum_max + bias_absmax < (int64_t(1) << 14);
}

namespace {

// Permuted bias on the device (built once per instance from the caller's device bias) and its max |b|.
int ensure_bias_perm(TensorInstance* ti, const int32_t* bias, std::string* why) {
    if (!bias || ti->d_bias_perm) return 0;
    std::vector<int32_t> b(ti->n), bp(ti->npp, 0);
    cudaError_t e = cudaMemcpy(b.data(), bias, size_t(ti->n) * 4, cudaMemcpyDeviceToHost);
    int64_t mx = 0;
    for (int i = 0; i < ti->n && e == cudaSuccess; ++i) {
        bp[ti->perm[i]] = b[i];
        mx = std::max<int64_t>(mx, b[i] < 0 ? -int64_t(b[i]) : int64_t(b[i]));
    }
    if (e == cudaSuccess) e = cudaMalloc(&ti->d_bias_perm, size_t(ti->npp) * 4);
    if (e == cudaSuccess) e = cudaMemcpy(ti->d_bias_perm, bp.data(), size_t(ti->npp) * 4, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        if (why) *why = std::string("bias: ") + cudaGetErrorString(e);
        return -2;
    }
    ti->bias_absmax = mx;
    return 0;
}

size_t f4_smem_bytes(int ns) {
    return 1024 + 8 * size_t(kM) * kKChunk + size_t(ns) * kM * kKChunk + size_t(f4_bars(ns)) * 8 + 16;
}

// The fp4 kernel's compiled ring depths; TensorRun::variant v runs kF4StageVariants[v].
constexpr int kF4StageVariants[kF4Variants] = {4, 6, 5, 3};

using F4Kernel = void (*)(const CUtensorMap, const F4Params);
F4Kernel f4_kernel(int variant) {
    switch (variant) {
        case 1: return tensor_fp4_kernel<6>;
        case 2: return tensor_fp4_kernel<5>;
        case 3: return tensor_fp4_kernel<3>;
        default: return tensor_fp4_kernel<4>;
    }
}

// Concurrent group slots of the fp4 kernel (16 co-resident CTAs each; queried with the deepest ring, one CTA per SM
// in every variant).
int f4_group_slots(int ngroups, int* out) {
    auto fn = f4_kernel(1);
    const size_t smem = f4_smem_bytes(kF4StageVariants[1]);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    int per_sm = 0, dev = 0, sms = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kF4Threads, smem);
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return int(e);
    int clusters = 0;
    {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = kF4Cluster;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        cfg.gridDim = dim3(kF4Slices);
        cfg.blockDim = dim3(kF4Threads);
        cfg.dynamicSmemBytes = smem;
        e = cudaOccupancyMaxActiveClusters(&clusters, fn, &cfg);
        if (e != cudaSuccess) return int(e);
    }
    *out = std::max(0, std::min(ngroups, std::min((per_sm * sms) / kF4Slices, clusters / (kF4Slices / kF4Cluster))));
    return 0;
}

int f4_run(TensorInstance* ti, const TensorRun& r, cudaStream_t st, std::string* why) {
    const int ngroups = (r.nchains + kM - 1) / kM;
    int slots = 0;
    int rc = f4_group_slots(ngroups, &slots);
    if (rc || slots < 1) {
        if (why) *why = "the fp4 tensor kernel cannot be co-resident on this device";
        return -2;
    }
    const size_t fbytes = ((size_t(ngroups) * kF4Slices * 4 + 255) / 256) * 256;
    const size_t dbytes = size_t(ngroups) * 2 * kM * 1024;
    const size_t nbytes = size_t(ngroups) * 2 * kM * 128;
    const size_t need = 256 + fbytes + dbytes + nbytes;
    cudaError_t e = cudaSuccess;
    if (ti->ws_bytes < need) {
        if (ti->d_ws) cudaFree(ti->d_ws);
        ti->d_ws = nullptr;
        ti->ws_bytes = 0;
        e = cudaMalloc(&ti->d_ws, need);
        if (e != cudaSuccess) {
            if (why) *why = std::string("workspace: ") + cudaGetErrorString(e);
            return -2;
        }
        ti->ws_bytes = need;
    }
    uint8_t* base = static_cast<uint8_t*>(ti->d_ws);
    int* err = reinterpret_cast<int*>(base);
    uint32_t* flags = reinterpret_cast<uint32_t*>(base + 256);
    uint8_t* dbuf = base + 256 + fbytes;
    int8_t* nlx = reinterpret_cast<int8_t*>(dbuf + dbytes);
    CUtensorMap mapJ;
    if (!make_map(&mapJ, ti->d_J4, 1024, 2048, kF4YS)) {
        if (why) *why = "cuTensorMapEncodeTiled failed";
        return -2;
    }
    e = cudaMemsetAsync(r.out_spins, 0, size_t(r.nchains) * 64 * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(r.out_sum_sh, 0, size_t(r.nchains) * 8, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(r.out_sum_bs, 0, size_t(r.nchains) * 8, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(r.out_flips, 0, size_t(r.nchains) * 8, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(base, 0, 256 + fbytes, st);     // error word + flags
    if (e != cudaSuccess) {
        if (why) *why = std::string("memset: ") + cudaGetErrorString(e);
        return -2;
    }
    F4Params P{};
    P.n = ti->n;
    P.S = r.tab.S;
    P.ngroups = ngroups;
    P.fourT = r.tab.fourT;
    P.q = r.tab.q;
    P.kcorr = r.tab.kcorr;
    P.kconst = r.tab.kconst;
    P.hclamp = r.hclamp;
    P.bias_perm = r.bias ? ti->d_bias_perm : nullptr;
    P.seed = r.seed;
    P.trial_offset = r.trial_offset;
    P.nchains = r.nchains;
    P.flags = flags;
    P.dbuf = dbuf;
    P.nlx = nlx;
    P.out_spins = r.out_spins;
    P.out_sum_sh = reinterpret_cast<unsigned long long*>(r.out_sum_sh);
    P.out_sum_bs = reinterpret_cast<unsigned long long*>(r.out_sum_bs);
    P.out_flips = reinterpret_cast<unsigned long long*>(r.out_flips);
    P.out_trace = r.out_trace;
    P.out_h = r.out_h;
    P.err = err;
    P.prof = r.prof;
    P.wait_ns = r.wait_ns;
    const int variant = (r.variant >= 0 && r.variant < kF4Variants) ? r.variant : 0;
    auto fn = f4_kernel(variant);
    const size_t smem = f4_smem_bytes(kF4StageVariants[variant]);
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    at[1].id = cudaLaunchAttributeClusterDimension;
    at[1].val.clusterDim.x = kF4Cluster;
    at[1].val.clusterDim.y = 1;
    at[1].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 2;
    cfg.gridDim = dim3(kF4Slices * slots);
    cfg.blockDim = dim3(kF4Threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    if (e == cudaSuccess) e = cudaLaunchKernelEx(&cfg, fn, mapJ, P);
    if (e != cudaSuccess) {
        if (why) *why = std::string("launch: ") + cudaGetErrorString(e);
        return -2;
    }
    ti->last_err = err;
    ti->last_kind = TENSOR_KIND_FP4;
    ti->last_ctas = kF4Slices * slots;
    ti->last_cluster = 1;
    return 0;
}

int res_run(TensorInstance* ti, const TensorRun& r, cudaStream_t st, std::string* why) {
    const int npairs = ((r.nchains + kM - 1) / kM + 1) / 2;
    const int ngroups = 2 * npairs;
    int slots = 0;
    int rc = res_pair_slots(npairs, &slots);
    if (rc || slots < 1) {
        if (why) *why = "the resident tensor kernel cannot be co-resident on this device";
        return -2;
    }
    const size_t fbytes = size_t(ngroups) * kResSlices * 4;
    const size_t dbytes = size_t(ngroups) * 2 * kM * 2048;
    const size_t nbytes = size_t(ngroups) * 2 * kM * 128;
    const size_t need = 256 + fbytes + dbytes + nbytes + 256;
    cudaError_t e = cudaSuccess;
    if (ti->ws_bytes < need) {
        if (ti->d_ws) cudaFree(ti->d_ws);
        ti->d_ws = nullptr;
        ti->ws_bytes = 0;
        e = cudaMalloc(&ti->d_ws, need);
        if (e != cudaSuccess) {
            if (why) *why = std::string("workspace: ") + cudaGetErrorString(e);
            return -2;
        }
        ti->ws_bytes = need;
    }
    uint8_t* base = static_cast<uint8_t*>(ti->d_ws);
    int* err = reinterpret_cast<int*>(base);
    uint32_t* flags = reinterpret_cast<uint32_t*>(base + 256);
    int8_t* dbuf = reinterpret_cast<int8_t*>(base + 256 + ((fbytes + 255) / 256) * 256);
    int8_t* nlx = dbuf + dbytes;
    CUtensorMap mapD, mapNL, mapJ;
    if (!make_map(&mapD, dbuf, 2048, uint64_t(ngroups) * 2 * kM, kM) ||
        !make_map(&mapNL, nlx, 128, uint64_t(ngroups) * 2 * kM, kM) || !make_map(&mapJ, ti->d_J, 2048, 2048, kResYS)) {
        if (why) *why = "cuTensorMapEncodeTiled failed";
        return -2;
    }
    e = cudaMemsetAsync(r.out_spins, 0, size_t(r.nchains) * 64 * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(r.out_sum_sh, 0, size_t(r.nchains) * 8, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(r.out_sum_bs, 0, size_t(r.nchains) * 8, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(r.out_flips, 0, size_t(r.nchains) * 8, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(base, 0, 256 + fbytes, st);     // error word + flags
    if (e != cudaSuccess) {
        if (why) *why = std::string("memset: ") + cudaGetErrorString(e);
        return -2;
    }
    ResParams P{};
    P.n = ti->n;
    P.S = r.tab.S;
    P.npairs = npairs;
    P.fourT = r.tab.fourT;
    P.q = r.tab.q;
    P.kcorr = r.tab.kcorr;
    P.kconst = r.tab.kconst;
    P.hclamp = r.hclamp;
    P.bias_perm = r.bias ? ti->d_bias_perm : nullptr;
    P.seed = r.seed;
    P.trial_offset = r.trial_offset;
    P.nchains = r.nchains;
    P.flags = flags;
    P.dbuf = dbuf;
    P.nlx = nlx;
    P.out_spins = r.out_spins;
    P.out_sum_sh = reinterpret_cast<unsigned long long*>(r.out_sum_sh);
    P.out_sum_bs = reinterpret_cast<unsigned long long*>(r.out_sum_bs);
    P.out_flips = reinterpret_cast<unsigned long long*>(r.out_flips);
    P.out_trace = r.out_trace;
    P.out_h = r.out_h;
    P.err = err;
    P.prof = r.prof;
    P.wait_ns = r.wait_ns;
    auto fn = tensor_res_kernel;
    const size_t smem = res_smem_bytes();
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cfg.gridDim = dim3(kResSlices * slots);
    cfg.blockDim = dim3(kResThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    if (e == cudaSuccess) e = cudaLaunchKernelEx(&cfg, fn, mapD, mapNL, mapJ, P);
    if (e != cudaSuccess) {
        if (why) *why = std::string("launch: ") + cudaGetErrorString(e);
        return -2;
    }
    ti->last_err = err;
    ti->last_kind = TENSOR_KIND_INT8;
    ti->last_ctas = kResSlices * slots;
    ti->last_cluster = 1;
    return 0;
}

}  // namespace

int tensor_wave_chains(int n, bool fp4, int* out) {
    const int R = std::max(2048, ((n + 255) / 256) * 256) / 256;
    constexpr int kMany = 1 << 20;   // more groups than any device holds: the query returns the device's limit
    int slots = 0, rc = 0;
    *out = 0;
    if (stream_supported(n)) {
        *out = stream_wave_chains();
        return 0;
    }
    if (R == 8 && fp4) {
        rc = f4_group_slots(kMany, &slots);        // one group of kM anneals per 16-CTA slot
        *out = slots * kM;
    } else if (R == 8) {
        rc = res_pair_slots(kMany, &slots);        // two groups per 32-CTA pair slot
        *out = 2 * slots * kM;
    } else if (R == 12 || R == 16) {
        rc = R == 12 ? max_clusters_t<12>(&slots) : max_clusters_t<16>(&slots);   // one group per cluster
        *out = slots * kM;
    } else {
        rc = int(cudaErrorInvalidValue);
    }
    return rc;
}

int tensor_run(TensorInstance* ti, const TensorRun& r, cudaStream_t st, std::string* why) {
    const int np = ti->np, R = np / 256;
    int rc0 = ensure_bias_perm(ti, r.bias, why);
    if (rc0) return rc0;
    const bool fp4 = tensor_fp4_eligible(ti, r.bias ? ti->bias_absmax : 0);
    if (r.kind == TENSOR_KIND_FP4 && !fp4) {
        if (why) *why = "the fp4 kernel needs NP = 2048, |J| <= 1 and max|b| + max_y sum_x |J_xy| < 16384";
        return -1;
    }
    if (fp4 && r.kind != TENSOR_KIND_INT8) return f4_run(ti, r, st, why);
    if (ti->stream) return stream_run(ti, r, r.bias ? ti->d_bias_perm : nullptr, st, why);
    if (R == 8) return res_run(ti, r, st, why);
    const int groups = (r.nchains + kM - 1) / kM;
    // workspace: exchange buffers, permuted bias, error word
    const size_t dbytes = size_t(groups) * 2 * kM * np;
    const size_t nlbytes = size_t(groups) * 2 * kC * kM * 4;
    cudaError_t e = cudaSuccess;
    if (ti->ws_bytes < dbytes + nlbytes + 256) {
        if (ti->d_ws) cudaFree(ti->d_ws);
        ti->d_ws = nullptr;
        ti->ws_bytes = 0;
        e = cudaMalloc(&ti->d_ws, dbytes + nlbytes + 256);
        if (e != cudaSuccess) {
            if (why) *why = std::string("workspace: ") + cudaGetErrorString(e);
            return -2;
        }
        ti->ws_bytes = dbytes + nlbytes + 256;
    }
    int8_t* dbuf = static_cast<int8_t*>(ti->d_ws);
    int32_t* nlbuf = reinterpret_cast<int32_t*>(static_cast<uint8_t*>(ti->d_ws) + dbytes);
    int* err = reinterpret_cast<int*>(static_cast<uint8_t*>(ti->d_ws) + dbytes + nlbytes);
    CUtensorMap mapA, mapB;
    if (!make_map(&mapA, dbuf, uint64_t(np), uint64_t(groups) * 2 * kM, kM) ||
        !make_map(&mapB, ti->d_J, uint64_t(np), uint64_t(np), uint32_t(16 * R))) {
        if (why) *why = "cuTensorMapEncodeTiled failed";
        return -2;
    }
    const int words = np / 32;
    e = cudaMemsetAsync(r.out_spins, 0, size_t(r.nchains) * words * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(r.out_sum_sh, 0, size_t(r.nchains) * 8, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(r.out_sum_bs, 0, size_t(r.nchains) * 8, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(r.out_flips, 0, size_t(r.nchains) * 8, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, 4, st);
    if (e != cudaSuccess) {
        if (why) *why = std::string("memset: ") + cudaGetErrorString(e);
        return -2;
    }
    TensorParams P{};
    P.n = ti->n;
    P.np = np;
    P.R = R;
    P.nc = 16 * R;
    P.S = r.tab.S;
    P.fourT = r.tab.fourT;
    P.q = r.tab.q;
    P.kcorr = r.tab.kcorr;
    P.kconst = r.tab.kconst;
    P.hclamp = r.hclamp;
    P.bias_perm = r.bias ? ti->d_bias_perm : nullptr;
    P.seed = r.seed;
    P.trial_offset = r.trial_offset;
    P.nchains = r.nchains;
    P.dbuf = dbuf;
    P.nlbuf = nlbuf;
    P.out_spins = r.out_spins;
    P.out_sum_sh = reinterpret_cast<unsigned long long*>(r.out_sum_sh);
    P.out_sum_bs = reinterpret_cast<unsigned long long*>(r.out_sum_bs);
    P.out_flips = reinterpret_cast<unsigned long long*>(r.out_flips);
    P.out_trace = r.out_trace;
    P.out_h = r.out_h;
    P.err = err;
    P.prof = r.prof;
    int rc = -1;
    if (R == 12) rc = launch_t<12>(P, groups, mapA, mapB, st, why);   // NP = 2048 runs the resident kernel above
    else if (R == 16) rc = launch_t<16>(P, groups, mapA, mapB, st, why);
    if (rc) return rc;
    ti->last_err = err;
    ti->last_kind = TENSOR_KIND_INT8;
    ti->last_ctas = kC * groups;
    ti->last_cluster = kC;
    return 0;
}

int tensor_check_error(TensorInstance* ti, cudaStream_t st, std::string* why) {
    if (!ti->last_err) return 0;
    int h = 0;
    cudaError_t e = cudaMemcpyAsync(&h, ti->last_err, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        if (why) *why = std::string("error word: ") + cudaGetErrorString(e);
        return -2;
    }
    if (h) {
        if (why) *why = "a bounded device wait expired (code " + std::to_string(h) + ")";
        return -3;
    }
    return 0;
}

void tensor_free_instance(TensorInstance* ti) {
    if (!ti) return;
    if (ti->d_J) cudaFree(ti->d_J);
    if (ti->d_ws) cudaFree(ti->d_ws);
    if (ti->d_bias_perm) cudaFree(ti->d_bias_perm);
    if (ti->d_J4) cudaFree(ti->d_J4);
    ti->d_J4 = nullptr;
    ti->d_J = nullptr;
    ti->d_ws = nullptr;
    ti->d_bias_perm = nullptr;
    ti->ws_bytes = 0;
}

}  // namespace anc
