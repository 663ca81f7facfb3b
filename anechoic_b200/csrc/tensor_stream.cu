// Batched engine for large dense instances (NP in (8192, 16384], up to 64 rounds): J is too large to keep resident
// (16384^2 int8 = 256 MB), so every step streams it from HBM once and applies it to two replica groups at a time.
//
// Layout. 128 CTAs, one per y-slice of 128 permuted columns. Slice cs owns RNG lanes 2cs and 2cs + 1, all rounds:
// slot i = k*256 + l sits at permuted column p(i) = (l / 2) * 128 + (l % 2) * 64 + k (k < R <= 64; columns with
// k >= R are padding, never decided, with zero couplings). J_perm[p(y)][p(x)] = J[x][y] (int8).
// Per step (the golden model's step, sca_ref_bias.hpp:44-68; decision as in anc_common.cuh):
//   16 decision warps: warp w decides group w / 8, replica (w % 4) * 32 + lane (its TMEM lane), RNG lane
//     2cs + (w / 4) % 2, the lane's R rounds in order (fields from TMEM, int32). It writes the replica's 64 update
//     bytes dS in {0, +-1, +-2} of its lane and its n_lin partial byte; the CTA then publishes flag[cs] = m + 2.
//   3 producer warps: chunk c of a step = J_perm rows [128 cs, +128) x columns [128 c, +128) (HBM, no dependency;
//     issued first) plus the two groups' dS tiles of slice c (L2; after slice c's flag). Two more chunks carry the
//     n_lin partials (256 bytes per replica: 2 per slice).
//   1 MMA thread: per dS chunk, 4 x 2 tcgen05.mma kind::i8 (M 128 replicas, N 128 columns, K 32) into each group's
//     int32 field accumulator; per n_lin chunk 4 x 2 i8 MMAs against a ones row into the n_lin accumulators.
// Every wait is bounded (2 s); on expiry the kernel records an error code and skips the remaining work.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "anc_ptx.cuh"
#include "anc_tensor.cuh"

namespace anc {
namespace {

using namespace ptx;

constexpr int kSM = 128;                   // replicas per group (MMA M, TMEM lanes)
constexpr int kSSlices = 128;              // y-slices (CTAs)
constexpr int kSCols = 128;                // permuted columns per slice (MMA N)
constexpr int kSNPP = kSSlices * kSCols;   // permuted width 16384
constexpr int kSDW = 16, kSPW = 3;
constexpr int kSMmaWarp = kSDW + kSPW;
constexpr int kSThreads = (kSDW + kSPW + 1) * 32;
constexpr int kSStages = 4;
constexpr uint32_t kSTile = 128 * 128;     // 16 KB
constexpr uint32_t kSStage = 3 * kSTile;   // J tile + two dS tiles
constexpr int kSChunks = kSSlices + 2;     // dS chunks + 2 n_lin chunks per step
constexpr int kErrFull = 1, kErrEmpty = 2, kErrHready = 3, kErrFlag = 4, kErrInit = 6, kErrRead = 7;

struct StreamParams {
    int n, R, S;
    const int32_t* fourT;
    const int32_t* q;
    const int64_t* kcorr;
    const int32_t* kconst;
    int32_t hclamp;
    const int32_t* bias_perm;           // [16384] or null
    uint64_t seed;
    uint32_t trial_offset;
    int nchains, npairs;
    uint32_t* flags;                    // [npairs][128] (zeroed)
    int8_t* dbuf;                       // [2 groups][2 parity][128][16384]
    int8_t* nlx;                        // [2][2][128][256]
    uint32_t* out_spins;                // [nchains][words]
    int words;                          // spin words per chain (NP / 32)
    unsigned long long* out_sum_sh;
    unsigned long long* out_sum_bs;
    unsigned long long* out_flips;
    int32_t* out_trace;
    int32_t* out_h;
    int* err;
    long long* prof;
};

__global__ void __launch_bounds__(kSThreads, 1)
    tensor_stream_kernel(const __grid_constant__ CUtensorMap mapJ, const __grid_constant__ CUtensorMap mapD,
                         const __grid_constant__ CUtensorMap mapNL, const __grid_constant__ StreamParams P) {
    constexpr uint32_t IDESC_H = (2u << 4) | (1u << 7) | (1u << 10) | (uint32_t(kSCols >> 3) << 17) | (uint32_t(kSM >> 4) << 24);
    constexpr uint32_t IDESC_NL = (2u << 4) | (1u << 7) | (1u << 10) | (uint32_t(16 >> 3) << 17) | (uint32_t(kSM >> 4) << 24);
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* stages = smem;                                 // kSStages x (J, dS0, dS1)
    uint8_t* ones = stages + kSStages * kSStage;            // 2 KB: row 0 = 128 x int8(1)
    uint64_t* bars = reinterpret_cast<uint64_t*>(ones + 2048);   // full[4], empty[4], hready, init, fields read
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kSStages + 3);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int cs = int(blockIdx.x);
    const int n = P.n, S = P.S, R = P.R;
    int* err = P.err;
    const uint32_t bar_full = smem_u32(bars), bar_empty = smem_u32(bars + kSStages);
    const uint32_t bar_h = smem_u32(bars + 2 * kSStages);
    const uint32_t bar_init = smem_u32(bars + 2 * kSStages + 1);   // decision warps: fields of a new pair set
    // decision warps: the fields of step m have been read, so step m's tiles may now be accumulated (other slices
    // can publish step m before this CTA has read the fields it decides step m from)
    const uint32_t bar_rd = smem_u32(bars + 2 * kSStages + 2);

    if (tid == 0) {
        for (int s = 0; s < kSStages; ++s) {
            mbar_init(bar_full + 8 * s, 1);
            mbar_init(bar_empty + 8 * s, 1);
        }
        mbar_init(bar_h, 1);
        mbar_init(bar_init, 1);
        mbar_init(bar_rd, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = tid; i < 2048; i += blockDim.x) ones[i] = i < 128 ? 1 : 0;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (warp == kSMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(512)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    // TMEM columns: group g fields [128 g, +128), group g n_lin accumulator [256 + 16 g, +16)

    const bool prof = P.prof != nullptr;
    long long pa = 0, pb = 0, pc = 0;
    const long long t_loop0 = clock64();
    uint32_t hph = 0u, q = 0u, rph = 0u;

    for (int pr = 0; pr < P.npairs; ++pr) {
        if (warp < kSDW) {
            // ---------------- decision warps ----------------
            const int g = warp >> 3, jl = (warp >> 2) & 1;
            const int r = (warp & 3) * 32 + lane;
            const int l = 2 * cs + jl;                       // RNG lane
            const int chain = (2 * pr + g) * kSM + r;
            const bool writer = chain < P.nchains;
            const uint32_t tl = uint32_t((warp & 3) * 32) << 16;
            const uint32_t fcol = uint32_t(128 * g + 64 * jl);   // this thread's 64 field columns
            const size_t drow0 = size_t(g * 2) * kSM + r;       // row of parity 0 in the dS buffer
            Xoshiro rng;
            rng_seed(rng, P.seed, P.trial_offset + uint32_t(chain), uint32_t(l));
            uint64_t sw = 0, dw = 0, vmask = 0;              // bit k: spin up / flipped last step / active slot
            int32_t nlin_prev = 0;
            uint32_t nlacc_prev = 0;
            long long flips = 0;
            {
                uint32_t dwords[16];
#pragma unroll
                for (int e = 0; e < 16; ++e) dwords[e] = 0u;
                for (int k = 0; k < R; ++k) {
                    const uint32_t rv = rng_next(rng);
                    const int i = k * 256 + l;
                    const bool valid = i < n;
                    const uint64_t up = valid ? (rv >> 31) : 1u;
                    sw |= up << k;
                    if (valid) vmask |= uint64_t(1) << k;
                    if (valid && !up) dw |= uint64_t(1) << k;   // s_prev = +1 initially (sca_ref_bias.hpp:29-41)
                    const uint32_t b = valid ? (up ? 0x01u : 0xFFu) : 0u;
                    dwords[k >> 2] |= b << (8 * (k & 3));
                }
                int8_t* dst = P.dbuf + ((drow0 + kSM) * kSNPP) + cs * kSCols + jl * 64;   // parity 1
#pragma unroll
                for (int e = 0; e < 4; ++e)
                    reinterpret_cast<uint4*>(dst)[e] =
                        make_uint4(dwords[4 * e], dwords[4 * e + 1], dwords[4 * e + 2], dwords[4 * e + 3]);
                P.nlx[(drow0 + kSM) * 256 + 2 * cs + jl] = 0;
                uint32_t v[16];
#pragma unroll
                for (int h4 = 0; h4 < 4; ++h4) {
#pragma unroll
                    for (int e = 0; e < 16; ++e)
                        v[e] = P.bias_perm ? uint32_t(P.bias_perm[cs * kSCols + 64 * jl + 16 * h4 + e]) : 0u;
                    tmem_st16(tmem + tl + fcol + uint32_t(16 * h4), v);
                }
                if (jl == 0) {
#pragma unroll
                    for (int e = 0; e < 16; ++e) v[e] = 0u;
                    tmem_st16(tmem + tl + uint32_t(256 + 16 * g), v);
                }
                tmem_wait_st();
            }
            writer_fence();
            tc_fence_before();
            asm volatile("bar.sync 1, %0;" ::"r"(kSDW * 32) : "memory");
            if (tid == 0) {
                // the MMA thread may accumulate into these fields only after they are set: tiles of other slices
                // can land before this CTA leaves its previous pair
                mbar_arrive(bar_init);
                asm volatile("fence.acq_rel.gpu;\n\tst.release.gpu.global.u32 [%0], %1;" ::"l"(P.flags + pr * kSSlices + cs),
                             "r"(1u)
                             : "memory");
            }
            const int32_t hcl = P.hclamp;
            for (int m = 0; m <= S; ++m) {
                long long t0 = prof ? clock64() : 0;
                const int t = m < S ? m : S - 1;
                const int32_t fourT = __ldg(P.fourT + t), qv = __ldg(P.q + t), kconst = __ldg(P.kconst + t);
                const int64_t kcorr = __ldg(P.kcorr + t);
                if (!err_set(err)) mbar_wait(bar_h, hph & 1u, err, kErrHready);
                ++hph;
                tc_fence_after();
                if (prof) { const long long t1 = clock64(); pa += t1 - t0; t0 = t1; }
                uint32_t nv;
                asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];"
                             : "=r"(nv)
                             : "r"(tmem + tl + uint32_t(256 + 16 * g)));
                tmem_wait_ld();
                const int32_t nlin = int32_t(nv - nlacc_prev);
                nlacc_prev = nv;
                if (m >= 1 && writer && cs == 0 && jl == 0 && P.out_trace) P.out_trace[size_t(chain) * S + (m - 1)] = nlin;
                nlin_prev = nlin;
                if (m == S) {
                    long long sh = 0, bs = 0;
                    for (int half = 0; half < 2; ++half) {
                        uint32_t hv[32];
                        tmem_ld32(tmem + tl + fcol + uint32_t(32 * half), hv);
                        tmem_wait_ld();
#pragma unroll
                        for (int e = 0; e < 32; ++e) {
                            const int k = 32 * half + e, i = k * 256 + l;
                            if (k >= R || i >= n) continue;
                            const bool up = (sw >> k) & 1u;
                            const int32_t h = int32_t(hv[e]);
                            sh += up ? h : -h;
                            if (P.bias_perm) {
                                const int32_t b = P.bias_perm[cs * kSCols + 64 * jl + k];
                                bs += up ? b : -b;
                            }
                            if (writer) {
                                if (up) atomicOr(P.out_spins + size_t(chain) * P.words + (i >> 5), 1u << (i & 31));
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
                const int32_t xs = qv - corr, twocorr = 2 * corr, c1 = twoT - 1;
                uint64_t fm = 0, lm = 0;
                const int par = m & 1;
                int8_t* dst = P.dbuf + ((drow0 + size_t(par) * kSM) * kSNPP) + cs * kSCols + jl * 64;
                for (int half = 0; half < 2; ++half) {
                    uint32_t hv[32];
                    tmem_ld32(tmem + tl + fcol + uint32_t(32 * half), hv);
                    tmem_wait_ld();
                    uint32_t fmh = 0, lmh = 0;
#pragma unroll
                    for (int e = 0; e < 32; ++e) {
                        const int k = 32 * half + e;
                        if (k >= R) break;
                        const uint32_t u = rng_next(rng);
                        const bool up = (sw >> k) & 1u;
                        int32_t hs = up ? int32_t(hv[e]) : -int32_t(hv[e]);
                        if (hcl > 0) hs = max(-hcl, min(hs, hcl));
                        int32_t zt = hs * 65536 + xs;
                        if ((dw >> k) & 1u) zt += twocorr;
                        const int32_t thr = __mulhi(int32_t((u & 0xffff0000u) ^ 0x80000000u), fourT);
                        if (zt < thr) fmh |= 1u << e;
                        if (uint32_t(zt + c1) < lw) lmh |= 1u << e;
                    }
                    fm |= uint64_t(fmh) << (32 * half);
                    lm |= uint64_t(lmh) << (32 * half);
                }
                fm &= vmask;
                lm &= vmask;
                flips += __popcll(fm);
                // dS bytes: flipped up -> down = -2 (0xFE), down -> up = +2 (0x02)
                uint32_t dwords[16];
#pragma unroll
                for (int e = 0; e < 16; ++e) {
                    uint32_t wv = 0u;
#pragma unroll
                    for (int b = 0; b < 4; ++b) {
                        const int k = 4 * e + b;
                        if ((fm >> k) & 1u) wv |= (((sw >> k) & 1u) ? 0xFEu : 0x02u) << (8 * b);
                    }
                    dwords[e] = wv;
                }
#pragma unroll
                for (int e = 0; e < 4; ++e)
                    reinterpret_cast<uint4*>(dst)[e] =
                        make_uint4(dwords[4 * e], dwords[4 * e + 1], dwords[4 * e + 2], dwords[4 * e + 3]);
                P.nlx[(drow0 + size_t(par) * kSM) * 256 + 2 * cs + jl] = int8_t(__popcll(lm));
                sw ^= fm;
                dw = fm;
                writer_fence();
                tc_fence_before();
                if (prof) { const long long t1 = clock64(); pb += t1 - t0; t0 = t1; }
                asm volatile("bar.sync 1, %0;" ::"r"(kSDW * 32) : "memory");
                if (tid == 0) {
                    mbar_arrive(bar_rd);
                    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(P.flags + pr * kSSlices + cs),
                                 "r"(uint32_t(m + 2))
                                 : "memory");
                }
                if (prof) pc += clock64() - t0;
            }
            tc_fence_before();
        } else if (warp < kSDW + kSPW) {
            // ---------------- producer warps ----------------
            const int pwid = warp - kSDW;
            const uint32_t* fl = P.flags + pr * kSSlices;
            for (int m = -1; m < S; ++m) {
                const int par = m & 1;
                const uint32_t target = uint32_t(m + 2);
                uint32_t ready[4] = {0u, 0u, 0u, 0u};        // slices seen at >= target, by 32-slice window
                for (int c = 0; c < kSChunks; ++c, ++q) {
                    if (int(q % kSPW) != pwid) continue;
                    if (__shfl_sync(0xffffffffu, err_set(err) ? 1 : 0, 0)) continue;
                    const int s = int(q % kSStages);
                    const uint32_t u = q / kSStages;
                    const long long w0 = prof ? clock64() : 0;
                    if (u >= 1) {
                        const int w = lane == 0 ? (mbar_wait(bar_empty + 8 * s, (u - 1) & 1u, err, kErrEmpty) ? 1 : 0) : 1;
                        if (!__shfl_sync(0xffffffffu, w, 0)) continue;
                    }
                    uint8_t* st_base = stages + size_t(s) * kSStage;
                    const bool dchunk = c < kSSlices;
                    if (lane == 0) {
                        mbar_arrive_expect_tx(bar_full + 8 * s, dchunk ? kSStage : 2 * kSTile);
                        if (dchunk) tma_load_2d(smem_u32(st_base), &mapJ, c * 128, cs * kSCols, bar_full + 8 * s);
                    }
                    // slices that must have published: c (dS chunk) or all (n_lin chunks)
                    bool ok = true;
                    for (int wdw = 0; wdw < 4 && ok; ++wdw) {
                        const uint32_t need = dchunk ? ((c >> 5) == wdw ? (1u << (c & 31)) : 0u) : 0xffffffffu;
                        if (!need || (ready[wdw] & need) == need) continue;
                        ok = false;
                        const uint64_t t0 = globaltimer();
                        for (uint32_t k = 1;; ++k) {
                            uint32_t v;
                            asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(fl + 32 * wdw + lane) : "memory");
                            ready[wdw] = __ballot_sync(0xffffffffu, v >= target);
                            if ((ready[wdw] & need) == need) { ok = true; break; }
                            if ((k & 63u) == 0 && __shfl_sync(0xffffffffu, globaltimer() - t0 > kWaitNs, 0)) {
                                if (lane == 0) atomicCAS(err, 0, kErrFlag);
                                break;
                            }
                        }
                        asm volatile("fence.acq_rel.gpu;" ::: "memory");
                        __syncwarp();
                    }
                    if (prof) pa += clock64() - w0;
                    if (lane == 0) {
                        // the stage's transaction count was posted with the J load, so the dS loads are issued even
                        // after a failed wait (the error word is set; the data is then ignored)
                        asm volatile("fence.proxy.async.global;" ::: "memory");
                        const int ay0 = (0 * 2 + par) * kSM, ay1 = (1 * 2 + par) * kSM;
                        if (dchunk) {
                            tma_load_2d(smem_u32(st_base + kSTile), &mapD, c * 128, ay0, bar_full + 8 * s);
                            tma_load_2d(smem_u32(st_base + 2 * kSTile), &mapD, c * 128, ay1, bar_full + 8 * s);
                        } else {
                            const int x = (c - kSSlices) * 128;
                            tma_load_2d(smem_u32(st_base + kSTile), &mapNL, x, ay0, bar_full + 8 * s);
                            tma_load_2d(smem_u32(st_base + 2 * kSTile), &mapNL, x, ay1, bar_full + 8 * s);
                        }
                    }
                    __syncwarp();
                }
            }
        } else if (warp == kSMmaWarp) {
            // ---------------- MMA thread ----------------
            if (lane == 0) {
                if (!err_set(err)) mbar_wait(bar_init, uint32_t(pr) & 1u, err, kErrInit);
                tc_fence_after();
                for (int m = -1; m < S; ++m) {
                    const long long t0 = prof ? clock64() : 0;
                    if (m >= 0) {
                        if (!err_set(err)) mbar_wait(bar_rd, rph & 1u, err, kErrRead);
                        ++rph;
                        tc_fence_after();
                    }
                    for (int c = 0; c < kSChunks; ++c, ++q) {
                        const int s = int(q % kSStages);
                        const uint32_t u = q / kSStages;
                        const long long w0 = prof ? clock64() : 0;
                        const bool ok = !err_set(err) && mbar_wait(bar_full + 8 * s, u & 1u, err, kErrFull);
                        if (prof) pa += clock64() - w0;
                        tc_fence_after();
                        if (ok) {
                            const uint32_t b0 = smem_u32(stages + size_t(s) * kSStage);
                            if (c < kSSlices) {
#pragma unroll
                                for (int kk = 0; kk < 4; ++kk) {
                                    const uint64_t bj = sw128_desc(b0 + 32 * kk);
                                    mma_i8(tmem, sw128_desc(b0 + kSTile + 32 * kk), bj, IDESC_H, 1u);
                                    mma_i8(tmem + 128u, sw128_desc(b0 + 2 * kSTile + 32 * kk), bj, IDESC_H, 1u);
                                }
                            } else {
                                const uint32_t o = smem_u32(ones);
#pragma unroll
                                for (int kk = 0; kk < 4; ++kk) {
                                    const uint64_t bo = sw128_desc(o + 32 * kk);
                                    mma_i8(tmem + 256u, sw128_desc(b0 + kSTile + 32 * kk), bo, IDESC_NL, 1u);
                                    mma_i8(tmem + 272u, sw128_desc(b0 + 2 * kSTile + 32 * kk), bo, IDESC_NL, 1u);
                                }
                            }
                        }
                        mma_commit(bar_empty + 8 * s);
                    }
                    mma_commit(bar_h);
                    if (prof) pb += clock64() - t0;
                }
            } else {
                q += uint32_t(S + 1) * kSChunks;
            }
            __syncwarp();
        }
    }
    if (prof) {
        long long* dst = P.prof + size_t(blockIdx.x) * kTensorProfSlots;
        if (warp == 0 && lane == 0) { dst[0] = pa; dst[1] = pb; dst[2] = pc; }
        if (warp == kSMmaWarp && lane == 0) { dst[5] = pa; dst[6] = pb; dst[8] = clock64() - t_loop0; }
        if (warp == kSDW && lane == 0) dst[7] = pa;
    }
    // on the normal path every copy has landed before the MMA thread's last wait and every MMA has completed before
    // the decision warps' last wait on bar_h; the barrier orders the TMEM dealloc after both
    __syncthreads();
    if (warp == kSMmaWarp) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
    }
}

size_t stream_smem_bytes() { return 1024 + size_t(kSStages) * kSStage + 2048 + (2 * kSStages + 3) * 8 + 16; }

}  // namespace

bool stream_supported(int n) {
    const int np = std::max(2048, ((n + 255) / 256) * 256);
    const int R = np / 256;
    return R > 32 && R <= 64;
}

void stream_permutation(int np, std::vector<int>* p) {
    p->resize(np);
    for (int i = 0; i < np; ++i) {
        const int l = i % 256, k = i / 256;
        (*p)[i] = (l / 2) * kSCols + (l % 2) * 64 + k;
    }
}

int stream_width() { return kSNPP; }

// The kernel advances one pair of replica groups at a time across all its CTAs.
int stream_wave_chains() { return 2 * kSM; }

int stream_run(TensorInstance* ti, const TensorRun& r, const int32_t* bias_perm, cudaStream_t st, std::string* why) {
    const int R = ti->np / 256;
    const int ngroups = (r.nchains + kSM - 1) / kSM;
    const int npairs = (ngroups + 1) / 2;
    int per_sm = 0, dev = 0, sms = 0;
    const size_t smem = stream_smem_bytes();
    cudaError_t e = cudaFuncSetAttribute(tensor_stream_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tensor_stream_kernel, kSThreads, smem);
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess || per_sm * sms < kSSlices) {
        if (why) *why = "the streaming tensor kernel cannot be co-resident on this device";
        return -2;
    }
    const size_t fbytes = ((size_t(npairs) * kSSlices * 4 + 255) / 256) * 256;
    const size_t dbytes = size_t(2) * 2 * kSM * kSNPP;
    const size_t nbytes = size_t(2) * 2 * kSM * 256;
    const size_t need = 256 + fbytes + dbytes + nbytes;
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
    int8_t* dbuf = reinterpret_cast<int8_t*>(base + 256 + fbytes);
    int8_t* nlx = dbuf + dbytes;
    CUtensorMap mapJ, mapD, mapNL;
    if (!make_map_2d(&mapJ, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, ti->d_J, kSNPP, kSNPP, 128, 128) ||
        !make_map_2d(&mapD, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, dbuf, kSNPP, 4 * kSM, 128, 128) ||
        !make_map_2d(&mapNL, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, nlx, 256, 4 * kSM, 128, 128)) {
        if (why) *why = "cuTensorMapEncodeTiled failed";
        return -2;
    }
    const int words = ti->np / 32;
    e = cudaMemsetAsync(r.out_spins, 0, size_t(r.nchains) * words * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(r.out_sum_sh, 0, size_t(r.nchains) * 8, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(r.out_sum_bs, 0, size_t(r.nchains) * 8, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(r.out_flips, 0, size_t(r.nchains) * 8, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(base, 0, 256 + fbytes, st);   // error word + flags
    if (e == cudaSuccess) e = cudaMemsetAsync(dbuf, 0, dbytes, st);         // padding columns stay zero
    if (e == cudaSuccess) e = cudaMemsetAsync(nlx, 0, nbytes, st);
    if (e != cudaSuccess) {
        if (why) *why = std::string("memset: ") + cudaGetErrorString(e);
        return -2;
    }
    StreamParams P{};
    P.n = ti->n;
    P.R = R;
    P.S = r.tab.S;
    P.fourT = r.tab.fourT;
    P.q = r.tab.q;
    P.kcorr = r.tab.kcorr;
    P.kconst = r.tab.kconst;
    P.hclamp = r.hclamp;
    P.bias_perm = bias_perm;
    P.seed = r.seed;
    P.trial_offset = r.trial_offset;
    P.nchains = r.nchains;
    P.npairs = npairs;
    P.flags = flags;
    P.dbuf = dbuf;
    P.nlx = nlx;
    P.out_spins = r.out_spins;
    P.words = words;
    P.out_sum_sh = reinterpret_cast<unsigned long long*>(r.out_sum_sh);
    P.out_sum_bs = reinterpret_cast<unsigned long long*>(r.out_sum_bs);
    P.out_flips = reinterpret_cast<unsigned long long*>(r.out_flips);
    P.out_trace = r.out_trace;
    P.out_h = r.out_h;
    P.err = err;
    P.prof = r.prof;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cfg.gridDim = dim3(kSSlices);
    cfg.blockDim = dim3(kSThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    e = cudaLaunchKernelEx(&cfg, tensor_stream_kernel, mapJ, mapD, mapNL, P);
    if (e != cudaSuccess) {
        if (why) *why = std::string("launch: ") + cudaGetErrorString(e);
        return -2;
    }
    ti->last_err = err;
    ti->last_kind = TENSOR_KIND_INT8;
    ti->last_ctas = kSSlices;
    ti->last_cluster = 1;
    return 0;
}

}  // namespace anc
