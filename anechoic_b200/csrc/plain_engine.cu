// Plain SCA engine kernels (see anc_plain.cuh for the algorithm and the reference lines it follows).
#include "anc_plain.cuh"

namespace anc {
namespace {

constexpr int T = kPlainThreads;
constexpr uint32_t FULL = 0xffffffffu;

// Bit-sliced counter: plane p holds bit p of 32 independent counts (one per bit position of the word).
template <int P>
struct BitCounter {
    uint32_t c[P];

    __device__ __forceinline__ void clear() {
#pragma unroll
        for (int p = 0; p < P; ++p) c[p] = 0;
    }
    // 8 words into planes 0-2 (Harley-Seal: 7 carry-save adders); returns the weight-8 carry word
    __device__ __forceinline__ uint32_t add8_low(const uint32_t (&a)[8]) {
        uint32_t t1a, t1b, t2a, t2b, t3;
        csa(c[0], t1a, c[0], a[0], a[1]);
        csa(c[0], t1b, c[0], a[2], a[3]);
        csa(c[1], t2a, c[1], t1a, t1b);
        csa(c[0], t1a, c[0], a[4], a[5]);
        csa(c[0], t1b, c[0], a[6], a[7]);
        csa(c[1], t2b, c[1], t1a, t1b);
        csa(c[2], t3, c[2], t2a, t2b);
        return t3;
    }
    // a carry word of weight 2^p0 ripples upward while any lane has one
    __device__ __forceinline__ void ripple(uint32_t t, int p0) {
#pragma unroll
        for (int p = 3; p < P; ++p) {
            if (p < p0) continue;
            if (!__any_sync(FULL, t)) break;
            const uint32_t k = c[p] & t;
            c[p] ^= t;
            t = k;
        }
    }
    // add 8 words: the weight-8 carry ripples from plane 3
    __device__ __forceinline__ void add8(const uint32_t (&a)[8]) { ripple(add8_low(a), 3); }
    // two weight-8 carry words (of two add8_low calls) into plane 3; the weight-16 carry ripples from plane 4, so
    // the vote-guarded ripple runs once per 16 words
    __device__ __forceinline__ void add_w8_pair(uint32_t x, uint32_t y) {
        uint32_t t4;
        csa(c[3], t4, c[3], x, y);
        ripple(t4, 4);
    }
    // c += other (ripple-carry over the planes; the total stays below 2^P by construction)
    __device__ __forceinline__ void add_planes(const uint32_t* o) {
        uint32_t carry = 0;
#pragma unroll
        for (int p = 0; p < P; ++p) {
            const uint32_t a = c[p], b = o[p], u = a ^ b;
            c[p] = u ^ carry;
            carry = (a & b) | (u & carry);
        }
    }
    __device__ __forceinline__ void store(uint32_t* dst) const {
#pragma unroll
        for (int p = 0; p < P; ++p) dst[p] = c[p];
    }
};

// count of slot (word wi, bit lane) from combined planes res[wi * P + p]
template <int P>
__device__ __forceinline__ int32_t extract_count(const uint32_t* res_w, int lane) {
    int32_t v = 0;
#pragma unroll
    for (int p = 0; p < P; ++p) v |= int32_t((res_w[p] >> lane) & 1u) << p;
    return v;
}

__device__ __forceinline__ uint32_t valid_mask(int w, int n) {
    const int lo = 32 * w;
    if (lo + 32 <= n) return FULL;
    if (lo >= n) return 0u;
    return (1u << (n - lo)) - 1u;
}

// Append the flagged slot i (with its new-spin sign bit `neg`) to the flip list; warp-cooperative.
__device__ __forceinline__ void append_flip(bool flag, int i, uint32_t neg, uint32_t* flist, int* counter, int lane) {
    const uint32_t b = __ballot_sync(FULL, flag);
    if (!b) return;
    int base = 0;
    if (lane == 0) base = atomicAdd(counter, __popc(b));
    base = __shfl_sync(FULL, base, 0);
    if (flag) flist[base + __popc(b & lanemask_lt())] = uint32_t(i) | (neg << 31);
}

// The flip list of a step, built after the decisions from the flip words Dw (bit set = slot flipped this step) and the
// new spin words Sw: a block-wide exclusive scan of the words' popcounts places each word's flips, in slot order, at
// its offset; entry = slot | (new spin -1) << 31. The deciding warps thus write only two words per round and take no
// shared-memory atomic. Called by every thread; returns the list's length; ends with a CTA barrier.
__device__ __forceinline__ int build_flip_list(const uint32_t* Sw, const uint32_t* Dw, int nw, uint32_t* flist,
                                               int* s_wsum) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // each thread takes cb consecutive slots: 4, 8 or 16 bits of one word while the words are few (NP <= 8192),
    // else whole words
    int cb = 32;
    if (32 * nw <= 16 * T) {
        cb = 4;
        while (cb * T < 32 * nw) cb <<= 1;
    }
    const int per = cb < 32 ? 1 : (nw + T - 1) / T;
    const int w0 = cb < 32 ? min((tid * cb) >> 5, nw) : min(tid * per, nw), w1 = min(w0 + per, nw);
    const uint32_t part = cb < 32 ? (((1u << cb) - 1u) << ((tid * cb) & 31)) : FULL;
    int c = 0;
    for (int w = w0; w < w1; ++w) c += __popc(Dw[w] & part);
    int incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) s_wsum[warp] = incl;
    __syncthreads();
    int pos = incl - c, total = 0;
#pragma unroll
    for (int j = 0; j < T / 32; ++j) {
        const int v = s_wsum[j];
        pos += j < warp ? v : 0;
        total += v;
    }
    for (int w = w0; w < w1; ++w) {
        uint32_t d = Dw[w] & part;
        const uint32_t up = Sw[w];
        while (d) {
            const int bit = __ffs(d) - 1;
            d &= d - 1;
            flist[pos++] = uint32_t(32 * w + bit) | (((up >> bit) & 1u) ? 0u : 0x80000000u);
        }
    }
    __syncthreads();
    return total;
}

__device__ __forceinline__ int64_t warp_sum64(int64_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

// Streaming layout: add counter set cc (sign/magnitude pair (b, +/-), weight +/- 2^(b-1)) of slots y < n, held in
// res[w][P], into the fields: h_y += mult * (+/-) count_y << (b - 1). Ends with a CTA barrier.
template <int P>
__device__ __forceinline__ void stream_apply(const uint32_t* res, int cc, int32_t* h, int n, int mult) {
    __syncthreads();
    const int32_t m = (cc & 1) ? -mult : mult;
    const int sh = cc >> 1;
    for (int y = threadIdx.x; y < n; y += T) h[y] += m * (extract_count<P>(res + size_t(y >> 5) * P, y & 31) << sh);
    __syncthreads();
}

// Dense field pass: bit-sliced counts of the flipped rows, combined across groups into res[cc][w][P]; with STREAM
// (K >= 2, nwj <= T) each set cc is instead combined into res[w][P] and added into h (factor mult) right away.
// DV is the compiled variant (dense_variants): whether the next 8 rows are fetched ahead (K = 1, DV = 0) and how many
// rows a batch counts (8, or 16 for K = 1, DV = 2 and K = 2, DV = 1).
template <int K, int P, bool STREAM, int DV = 0>
__device__ __forceinline__ void dense_pass(const uint32_t* __restrict__ planes, size_t plane_stride, int nwj, int nf,
                                           const uint32_t* flist, uint32_t* comb, uint32_t* res, int32_t* h, int n,
                                           int mult) {
    constexpr int NC = K <= 1 ? 1 : 2 * (K - 1);
    constexpr bool PREFETCH = K <= 1 && DV == 0;
    constexpr int RB = (K <= 1 && DV == 2) || (K == 2 && DV == 1) ? 2 : 1;
    const int tid = threadIdx.x;
    if (nwj <= T) {
        const int G = T / nwj, g = tid / nwj, w = tid - g * nwj;
        const bool active = g < G;
        BitCounter<P> cnt[NC];
#pragma unroll
        for (int cc = 0; cc < NC; ++cc) cnt[cc].clear();
        if (active && PREFETCH) {
            // one plane: the next 8 rows are fetched before the current 8 are counted, so the counting overlaps
            // the L2 latency of the fetches
            uint32_t cur[8], nxt[8];
            auto load8 = [&](int fb, uint32_t (&a)[8]) {
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int f = fb + j * G;
                    uint32_t v = 0u;
                    if (f < nf) {
                        const uint32_t e = flist[f];
                        v = __ldg(planes + size_t(e & 0x7fffffffu) * nwj + w) ^ ((e >> 31) ? FULL : 0u);
                    }
                    a[j] = v;
                }
            };
            if (g < nf) load8(g, nxt);
            for (int f0 = g; f0 < nf; f0 += 16 * G) {   // 16 rows per iteration, the second 8 possibly empty
#pragma unroll
                for (int j = 0; j < 8; ++j) cur[j] = nxt[j];
                if (f0 + 8 * G < nf) load8(f0 + 8 * G, nxt);
                const uint32_t w8a = cnt[0].add8_low(cur);
                uint32_t w8b = 0u;
                if (f0 + 8 * G < nf) {
#pragma unroll
                    for (int j = 0; j < 8; ++j) cur[j] = nxt[j];
                    if (f0 + 16 * G < nf) load8(f0 + 16 * G, nxt);
                    w8b = cnt[0].add8_low(cur);
                }
                cnt[0].add_w8_pair(w8a, w8b);
            }
        } else if (active) {
            // RB batches of 8 rows fetched together, then counted
            for (int f0 = g; f0 < nf; f0 += 8 * RB * G) {
                uint32_t a[RB][NC][8];
#pragma unroll
                for (int jj = 0; jj < 8 * RB; ++jj) {
                    const int j = jj & 7, rb = jj >> 3;
                    const int f = f0 + jj * G;
                    if (f < nf) {
                        const uint32_t e = flist[f];
                        const uint32_t neg = (e >> 31) ? FULL : 0u;
                        const uint32_t* row = planes + size_t(e & 0x7fffffffu) * nwj + w;
                        if (K <= 1) {
                            a[rb][0][j] = __ldg(row) ^ neg;
                        } else {
                            const uint32_t t = __ldg(row) ^ neg;   // 1 where s'_x * sign(J_xy) = -1
#pragma unroll
                            for (int b = 1; b < (K <= 1 ? 2 : K); ++b) {
                                const uint32_t m = __ldg(row + size_t(b) * plane_stride);
                                a[rb][2 * (b - 1)][j] = m & ~t;
                                a[rb][2 * (b - 1) + 1][j] = m & t;
                            }
                        }
                    } else {
#pragma unroll
                        for (int cc = 0; cc < NC; ++cc) a[rb][cc][j] = 0u;
                    }
                }
#pragma unroll
                for (int rb = 0; rb < RB; ++rb)
#pragma unroll
                    for (int cc = 0; cc < NC; ++cc) cnt[cc].add8(a[rb][cc]);
            }
        }
        if (G == 1) {
            if (STREAM) {
#pragma unroll
                for (int cc = 0; cc < NC; ++cc) {
                    if (active) cnt[cc].store(res + size_t(w) * P);
                    stream_apply<P>(res, cc, h, n, mult);
                }
                return;
            }
            if (active) {
#pragma unroll
                for (int cc = 0; cc < NC; ++cc) cnt[cc].store(res + (size_t(cc) * nwj + w) * P);
            }
            return;
        }
        int top = 1;
        while (top < G) top <<= 1;
#pragma unroll
        for (int cc = 0; cc < NC; ++cc) {
            if (active) cnt[cc].store(comb + (size_t(g) * nwj + w) * P);
            __syncthreads();
            for (int stride = top >> 1; stride >= 1; stride >>= 1) {
                if (active && g < stride && g + stride < G) {
                    cnt[cc].add_planes(comb + (size_t(g + stride) * nwj + w) * P);
                    if (stride > 1) cnt[cc].store(comb + (size_t(g) * nwj + w) * P);
                }
                __syncthreads();
            }
            if (STREAM) {
                if (active && g == 0) cnt[cc].store(res + size_t(w) * P);
                stream_apply<P>(res, cc, h, n, mult);
            } else if (active && g == 0) {
                cnt[cc].store(res + (size_t(cc) * nwj + w) * P);
            }
        }
    } else {
        for (int w0 = 0; w0 < nwj; w0 += T) {
            const int w = w0 + tid;
            if (w >= nwj) continue;   // nwj is a multiple of 32: whole warps skip together
            BitCounter<P> cnt[NC];
#pragma unroll
            for (int cc = 0; cc < NC; ++cc) cnt[cc].clear();
            for (int f0 = 0; f0 < nf; f0 += 8) {
                uint32_t a[NC][8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int f = f0 + j;
                    if (f < nf) {
                        const uint32_t e = flist[f];
                        const uint32_t neg = (e >> 31) ? FULL : 0u;
                        const uint32_t* row = planes + size_t(e & 0x7fffffffu) * nwj + w;
                        if (K <= 1) {
                            a[0][j] = __ldg(row) ^ neg;
                        } else {
                            const uint32_t t = __ldg(row) ^ neg;
#pragma unroll
                            for (int b = 1; b < (K <= 1 ? 2 : K); ++b) {
                                const uint32_t m = __ldg(row + size_t(b) * plane_stride);
                                a[2 * (b - 1)][j] = m & ~t;
                                a[2 * (b - 1) + 1][j] = m & t;
                            }
                        }
                    } else {
#pragma unroll
                        for (int cc = 0; cc < NC; ++cc) a[cc][j] = 0u;
                    }
                }
#pragma unroll
                for (int cc = 0; cc < NC; ++cc) cnt[cc].add8(a[cc]);
            }
#pragma unroll
            for (int cc = 0; cc < NC; ++cc) cnt[cc].store(res + (size_t(cc) * nwj + w) * P);
        }
    }
}

// Sparse field pass: h_y += m J_xy over the CSR rows x of the nf flipped slots in flist (m = mult with the sign of
// the new spin). Groups of 2^lg lanes take one row each, with lanes enough for the rows' mean degree at kSparseEdges
// edges per lane. Each group first fetches the bounds of kSparseBatch rows, then kSparseEdges edges per lane of each,
// and only then applies them, so a warp keeps 32 / 2^lg * kSparseBatch rows and kSparseEdges * kSparseBatch edge
// fetches per lane in flight where a loop over rows would keep one: the pass is bound by L2 latency, not bandwidth.
// Integer adds in any order: bit-exact. On a B200, over the 51-instance sparse batch (degrees 4 ... 48), one row per
// group with 8 edges per lane took 134 ms per launch and 4 rows x 2 edges 208 ms; a warp per row, one row at a time,
// took 684 ms.
// Sparse pass variants (rows per lane group in flight, edges fetched per lane before any is applied), chosen per
// instance at run time by the host's tuner (anc_api.cu): kSparseVariants[v] = {batch, edges}.
// log2 of the lanes per row: the power of two at or above mean degree / kSparseEdges, at most 32.
template <int kSparseEdges>
__device__ __forceinline__ int sparse_lanes_log2(int nnz, int n) {
    const int deg = (nnz + kSparseEdges * n - 1) / (kSparseEdges * max(n, 1));
    int lg = 0;
    while (lg < 5 && (1 << lg) < deg) ++lg;
    return lg;
}

// One word of edges: (y << 8) | uint8(J), or with E16 two edges y | [J = -1] << 15 (0x7fff: no edge).
template <bool E16>
__device__ __forceinline__ void sparse_apply(uint32_t v, int32_t m, int32_t* h) {
    if (E16) {
        const uint32_t lo = v & 0xffffu, hi = v >> 16;
        if ((lo & 0x7fffu) != 0x7fffu) atomicAdd(&h[lo & 0x7fffu], (lo >> 15) ? -m : m);
        if ((hi & 0x7fffu) != 0x7fffu) atomicAdd(&h[hi & 0x7fffu], (hi >> 15) ? -m : m);
    } else {
        atomicAdd(&h[v >> 8], m * int32_t(int8_t(v & 0xffu)));
    }
}

template <int kSparseBatch, int kSparseEdges, bool E16 = false>
__device__ __forceinline__ void sparse_pass(const int32_t* __restrict__ row_ptr, const uint32_t* __restrict__ adj,
                                            const uint32_t* flist, int nf, int lg, int32_t* h, int mult) {
    const int G = 1 << lg, sub = threadIdx.x & (G - 1), NG = T >> lg;
    for (int f0 = threadIdx.x >> lg; f0 < nf; f0 += NG * kSparseBatch) {
        int k0[kSparseBatch], k1[kSparseBatch];
        int32_t m[kSparseBatch];
        uint32_t a[kSparseBatch][kSparseEdges];
#pragma unroll
        for (int b = 0; b < kSparseBatch; ++b) {
            const int f = f0 + b * NG;
            k0[b] = 0;
            k1[b] = 0;
            m[b] = 0;
            if (f < nf) {
                const uint32_t e = flist[f];
                const int x = int(e & 0x7fffffffu);
                m[b] = (e >> 31) ? -mult : mult;
                k0[b] = __ldg(row_ptr + x) + sub;
                k1[b] = __ldg(row_ptr + x + 1);
            }
        }
#pragma unroll
        for (int b = 0; b < kSparseBatch; ++b)
#pragma unroll
            for (int e = 0; e < kSparseEdges; ++e) a[b][e] = k0[b] + e * G < k1[b] ? __ldg(adj + k0[b] + e * G) : 0u;
#pragma unroll
        for (int b = 0; b < kSparseBatch; ++b) {
#pragma unroll
            for (int e = 0; e < kSparseEdges; ++e)
                if (k0[b] + e * G < k1[b]) sparse_apply<E16>(a[b][e], m[b], h);
            for (int k = k0[b] + kSparseEdges * G; k < k1[b]; k += G) sparse_apply<E16>(__ldg(adj + k), m[b], h);
        }
    }
}

template <int K, int P>
__device__ __forceinline__ int32_t dense_delta(const uint32_t* res, int nwj, int wi, int lane, int nfp, bool in_f,
                                               bool s_up) {
    if (K <= 1) {
        // raw count of x in F with s'_x J_xy = +1, plus x = y when y flipped to -1 (diagonal bit reads as +1 there)
        const int32_t raw = extract_count<P>(res + size_t(wi) * P, lane);
        const int32_t pos = raw - ((in_f && !s_up) ? 1 : 0);
        return 2 * pos - nfp + (in_f ? 1 : 0);
    } else {
        int32_t v = 0;
#pragma unroll
        for (int b = 1; b < (K <= 1 ? 2 : K); ++b) {
            const int32_t pc = extract_count<P>(res + (size_t(2 * (b - 1)) * nwj + wi) * P, lane);
            const int32_t nc = extract_count<P>(res + (size_t(2 * (b - 1) + 1) * nwj + wi) * P, lane);
            v += (pc - nc) << (b - 1);
        }
        return v;
    }
}

// Adds the counts of the dense pass just completed into the fields, on every thread (slots tid, tid + T, ...):
// h_y += mult * dense_delta_y, with y's membership in the pass's F and its current spin from Dw / Sw. Running this
// right after the pass, on all 512 threads, keeps the bit-plane reads out of the deciding warps' rounds.
template <int K, int P>
__device__ __forceinline__ void apply_dense(const uint32_t* res, int nwj, const uint32_t* Sw, const uint32_t* Dw,
                                            int32_t* h, int n, int nf, bool init, int mult) {
    for (int i = threadIdx.x; i < n; i += T) {
        const int wi = i >> 5, lane = i & 31;
        const bool s_up = (Sw[wi] >> lane) & 1u, dif = (Dw[wi] >> lane) & 1u;
        h[i] += mult * dense_delta<K, P>(res, nwj, wi, lane, nf, init || dif, s_up);
    }
}

template <int K, int P, bool SPARSE, bool STREAM, int SB = 1, int SE = 8, int DV = 0>
__global__ void __launch_bounds__(T, 1) plain_kernel(const __grid_constant__ PlainLaunch L) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    __shared__ int s_item, s_nf, s_lin[8], s_wsum[T / 32];
    __shared__ long long s_red[2][16];
    int32_t* h = reinterpret_cast<int32_t*>(smem_raw);
    uint32_t* flist = reinterpret_cast<uint32_t*>(h + L.np_max);
    uint32_t* Sw = flist + L.np_max;
    uint32_t* Dw = Sw + L.nwj_max;
    uint32_t* comb = Dw + L.nwj_max;
    uint32_t* res = comb + size_t(L.nwj_max > T ? L.nwj_max : T) * P;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool decider = tid < kLanes;

    for (;;) {
        __syncthreads();
        if (tid == 0) s_item = atomicAdd(L.next_item, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= L.nitems) break;
        const int2 it = L.items ? L.items[item] : make_int2(0, item);
        const PlainJob& job = L.items ? L.jobs[it.x] : L.job0;
        const int n = job.n, np = job.np, R = np / kLanes, nw = job.nw, nwj = job.nwj, S = job.tab.S;
        const int c = it.y;
        const uint32_t* __restrict__ planes = job.planes;
        const size_t plane_stride = size_t(np) * nwj;
        const int32_t* __restrict__ fourT_t = job.tab.fourT;
        const int32_t* __restrict__ q_t = job.tab.q;
        const int64_t* __restrict__ kcorr_t = job.tab.kcorr;
        const int32_t* __restrict__ kconst_t = job.tab.kconst;
        const int32_t hclamp = job.hclamp;
        const int32_t* __restrict__ bias = job.bias;
        int32_t* trace_out = (job.trace && job.out_trace) ? job.out_trace + size_t(c) * S : nullptr;

        for (int i = tid; i < np; i += T) h[i] = (i < n && bias) ? bias[i] : 0;
        if (tid == 0) s_nf = 0;
        __syncthreads();

        // seed, initial spins (draw >> 31; padding +1), s_prev = +1 everywhere, initial flip list = all active slots
        Xoshiro rng;
        if (decider) {
            rng_seed(rng, job.seed, job.trial_offset + uint32_t(c), uint32_t(tid));
            for (int k = 0; k < R; ++k) {
                const uint32_t r = rng_next(rng);
                const int i = k * kLanes + tid;
                const bool valid = i < n;
                const uint32_t sbit = valid ? (r >> 31) : 1u;
                const uint32_t sw = __ballot_sync(FULL, sbit != 0);
                const uint32_t dw = __ballot_sync(FULL, valid && !sbit);
                if (lane == 0) { Sw[k * 8 + warp] = sw; Dw[k * 8 + warp] = dw; }
                append_flip(valid, i, sbit ^ 1u, flist, &s_nf, lane);
            }
        }
        __syncthreads();
        const int nf0 = s_nf;
        const int sparse_lg = SPARSE ? sparse_lanes_log2<SE>(__ldg(job.row_ptr + n), n) : 0;
        if (SPARSE) {
            if (job.csr16) sparse_pass<SB, SE, true>(job.row_ptr, job.adj, flist, nf0, sparse_lg, h, 1);
            else sparse_pass<SB, SE>(job.row_ptr, job.adj, flist, nf0, sparse_lg, h, 1);
        } else {
            dense_pass<K, P, STREAM, DV>(planes, plane_stride, nwj, nf0, flist, comb, res, h, n, 1);
            if (!STREAM) {
                __syncthreads();
                apply_dense<K, P>(res, nwj, Sw, Dw, h, n, nf0, true, 1);
            }
        }
        __syncthreads();

        int32_t nlin_prev = 0;
        long long flips = 0;
        for (int t = 0; t < S; ++t) {
            if (decider) {
                const int32_t fourT = __ldg(fourT_t + t), twoT = fourT >> 1, qv = __ldg(q_t + t);
                const int32_t corr = step_corr(nlin_prev, __ldg(kcorr_t + t), __ldg(kconst_t + t));
                const uint32_t lw = uint32_t(2 * twoT - 1);
                int nl = 0;
                for (int k = 0; k < R; ++k) {
                    const uint32_t u = rng_next(rng);
                    const int i = k * kLanes + tid, wi = k * 8 + warp;
                    const bool valid = i < n;
                    const uint32_t Sword = Sw[wi], Dword = Dw[wi];
                    const bool s_up = (Sword >> lane) & 1u, dif = (Dword >> lane) & 1u;
                    const int32_t hv = h[i];
                    int32_t hs = s_up ? hv : -hv;
                    if (hclamp > 0) hs = max(-hclamp, min(hs, hclamp));
                    const int32_t x = qv + (dif ? corr : -corr);      // q - (s == s_prev ? corr : -corr)
                    const int32_t zt = hs * 65536 + x;
                    const int32_t r = threshold16(u, fourT);
                    const bool fl = valid && (zt - r < 0);
                    const bool ln = valid && (uint32_t(zt + twoT - 1) < lw);
                    const uint32_t fb = __ballot_sync(FULL, fl);
                    nl += __popc(__ballot_sync(FULL, ln));
                    if (lane == 0) { Sw[wi] = Sword ^ fb; Dw[wi] = fb; }
                }
                if (lane == 0) s_lin[warp] = nl;
            }
            __syncthreads();
            const int nf = build_flip_list(Sw, Dw, nw, flist, s_wsum);
            int32_t nlin = 0;
#pragma unroll
            for (int w = 0; w < 8; ++w) nlin += s_lin[w];
            if (tid == 0) {
                flips += nf;
                if (trace_out) trace_out[t] = nlin;
            }
            nlin_prev = nlin;
            if (nf > 0) {
                if (SPARSE) {
                    if (job.csr16) sparse_pass<SB, SE, true>(job.row_ptr, job.adj, flist, nf, sparse_lg, h, 2);
                    else sparse_pass<SB, SE>(job.row_ptr, job.adj, flist, nf, sparse_lg, h, 2);
                } else {
                    dense_pass<K, P, STREAM, DV>(planes, plane_stride, nwj, nf, flist, comb, res, h, n, 2);
                    if (!STREAM) {
                        __syncthreads();
                        apply_dense<K, P>(res, nwj, Sw, Dw, h, n, nf, false, 2);
                    }
                }
            }
            __syncthreads();
        }
        // outputs
        long long sh = 0, bs = 0;
        for (int i = tid; i < n; i += T) {
            const bool up = (Sw[i >> 5] >> (i & 31)) & 1u;
            const int32_t hv = h[i];
            sh += up ? hv : -hv;
            if (bias) bs += up ? bias[i] : -bias[i];
            if (job.out_h) job.out_h[size_t(c) * n + i] = hv;
        }
        for (int w = tid; w < nw; w += T) job.out_spins[size_t(c) * nw + w] = Sw[w] & valid_mask(w, n);
        sh = warp_sum64(sh);
        bs = warp_sum64(bs);
        if (lane == 0) { s_red[0][warp] = sh; s_red[1][warp] = bs; }
        __syncthreads();
        if (tid == 0) {
            long long a = 0, b = 0;
            for (int w = 0; w < T / 32; ++w) { a += s_red[0][w]; b += s_red[1][w]; }
            job.out_sum_sh[c] = a;
            job.out_sum_bs[c] = b;
            job.out_flips[c] = flips;
        }
    }
}

// ------------------------------------------------------------------------------------------------ cluster variant
// One anneal spread over a cluster of CR = 8 or 16 CTAs (dense K = 1, NP = 2048), for the lowest latency per anneal.
// With 16 CTAs each SM holds 128 slots, half the update's work, and a warp's words interleave two rounds (below); the
// description that follows is for CR = 8.
// CTA r owns the 256 slots i = k*256 + 32r + l (round k, RNG lane 32r + l), one per thread: thread t = 32k + l keeps
// its slot's field, spin and last-flip bit in registers and a copy of lane 32r + l's xoshiro128** state, which it
// advances 8 draws per step and uses the k-th (every lane's stream is consumed in round order, as the golden model
// does). The J rows of the owned slots (by symmetry their columns, 256 x 2048 bits = 64 KB) stay in shared memory.
// Per step m (m = 0: the initial pass; m = t + 1 for step t), with p = m & 1:
//   1. every thread decides its slot; warp k's ballots give flip word wi = k*8 + r (bit l = slot k*256 + 32r + l),
//      the matching word of new spins +1 among the flipped, and the warp's counts of band slots and flips;
//   2. lanes 0 .. 7 of warp k push the warp's word pair and its packed counts to CTA `lane` with one 16-byte
//      st.async (record wi of that CTA's exchange buffer p, completing on its mbarrier p): every CTA receives
//      64 x 16 = 1024 bytes per step, and its thread 0 arrives on its own mbarrier p expecting them;
//   3. every thread makes its next draws, then waits (bounded) for mbarrier p's phase (cluster-scope acquire: the
//      remote stores are visible after it); each warp sums the 64 packed counts itself (n_lin for the next
//      correction, |F|), so no CTA barrier is needed;
//   4. every thread updates its field from all 2048 slots at once: for its row y of J (bit = [J_xy = +1]),
//        D = sum_w popc(F_w & (U_w ^ J_yw)),   h_y += 2 (|F| - 2 D)   (2 s'_x J_xy summed over the flipped x),
//      less the diagonal term when y itself flipped (J_yy = 0 is stored as a 0 bit). The initial pass uses the same
//      formula with F = the active slots, U = s0 and factor 1 (h = b + J s0).
// No step reads J from L2, no flip list is built, no counter is extracted and no barrier is crossed: the update costs
// the same whatever the flip count. Buffer p is written again at step m + 2 only by a CTA that has received every
// CTA's words of step m + 1, and a CTA sends those only after each of its warps has finished reading buffer p of step
// m (the words sent depend on the fields those reads updated); so the pushes of step m + 2 cannot overtake the reads
// of step m, nor count toward mbarrier p's phase of step m.
constexpr uint32_t kClusterTx = 64 * 16;  // exchange bytes a CTA receives per step
constexpr size_t kClusterSmem = 116 * 1024;   // above half an SM's shared memory: one CTA per SM

__device__ __forceinline__ uint32_t sm_addr(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }
__device__ __forceinline__ uint32_t cl_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cl_id() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cl_map(uint32_t local, uint32_t rank) {
    uint32_t a;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"(local), "r"(rank));
    return a;
}
__device__ __forceinline__ void cl_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
    asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ uint64_t cl_globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// remote store of one 16-byte record into another CTA's shared memory, completing on its mbarrier
__device__ __forceinline__ void st_async4(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t bar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.b32 [%0], {%1, %2, %3, %4}, [%5];"
                 ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d), "r"(bar) : "memory");
}
__device__ __forceinline__ bool cl_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for phase `parity`; false after limit_ns (0: at the first unsatisfied poll). The timer is read every
// 256 polls.
__device__ __forceinline__ bool cl_wait_for(uint32_t bar, uint32_t parity, uint64_t limit_ns) {
    if (cl_try_wait(bar, parity)) return true;
    if (limit_ns == 0) return false;
    const uint64_t t0 = cl_globaltimer();
    for (uint32_t k = 1;; ++k) {
        if (cl_try_wait(bar, parity)) return true;
        if ((k & 255u) == 0 && cl_globaltimer() - t0 > limit_ns) return false;
    }
}

// The draw of round k from this lane's stream: 8 draws per step, the k-th kept.
__device__ __forceinline__ uint32_t lane_draw(Xoshiro& rng, int k) {
    uint32_t u = 0u;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const uint32_t v = rng_next(rng);
        if (j == k) u = v;
    }
    return u;
}

// D of one slot over the 16 NB words of blocks B0 .. B0 + NB - 1 (block b: words 16b .. 16b + 15): the sum of
// popc(x_w), x_w = F_w & (U_w ^ J_yw), through a carry-save (Harley-Seal) tree -- 15 three-input adders and one
// popcount per block of 16 words, 4 more popcounts at the end, where a popcount per word took 16 per block.
template <int NB>
__device__ __forceinline__ int32_t cluster_words_d(const uint4* Jv, const uint4* FXv, int swz, int B0) {
    uint32_t ones = 0u, twos = 0u, fours = 0u, eights = 0u;
    int32_t sixteens = 0;
#pragma unroll
    for (int bb = 0; bb < NB; ++bb) {
        const int b = B0 + bb;
        uint32_t x[16];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int ch = 4 * b + q;               // 16-byte chunk of the J row: words 4ch .. 4ch+3
            const uint4 J4 = Jv[ch ^ swz], A = FXv[4 * ch], B = FXv[4 * ch + 1], C = FXv[4 * ch + 2],
                        E = FXv[4 * ch + 3];
            x[4 * q + 0] = A.x & (A.y ^ J4.x);
            x[4 * q + 1] = B.x & (B.y ^ J4.y);
            x[4 * q + 2] = C.x & (C.y ^ J4.z);
            x[4 * q + 3] = E.x & (E.y ^ J4.w);
        }
        uint32_t tA, tB, fA, fB, eA, eB, s16;
        csa(ones, tA, ones, x[0], x[1]);
        csa(ones, tB, ones, x[2], x[3]);
        csa(twos, fA, twos, tA, tB);
        csa(ones, tA, ones, x[4], x[5]);
        csa(ones, tB, ones, x[6], x[7]);
        csa(twos, fB, twos, tA, tB);
        csa(fours, eA, fours, fA, fB);
        csa(ones, tA, ones, x[8], x[9]);
        csa(ones, tB, ones, x[10], x[11]);
        csa(twos, fA, twos, tA, tB);
        csa(ones, tA, ones, x[12], x[13]);
        csa(ones, tB, ones, x[14], x[15]);
        csa(twos, fB, twos, tA, tB);
        csa(fours, eB, fours, fA, fB);
        csa(eights, s16, eights, eA, eB);
        sixteens += __popc(s16);
    }
    return 16 * sixteens + 8 * __popc(eights) + 4 * __popc(fours) + 2 * __popc(twos) + __popc(ones);
}

// Update helpers per owned slot and threads per CTA of the cluster kernel. With 16 CTAs one helper sums words
// 32 .. 63 of each slot's update (1.062 ms per 1000 steps for one anneal with two pushes per word, where three helpers
// of 16 words each took 1.092 and none 1.13; 0.994 with the packed counts summed by one warp reduction; 0.870 with one
// 16-byte push per word, 0.855 with the counts read at a 16-byte stride); with 8 CTAs the SM's ALU is already the
// bound and a helper gained nothing.
__host__ __device__ constexpr int cluster_helpers(int cr) { return cr == 16 ? 1 : 0; }
__host__ __device__ constexpr int cluster_threads(int cr) { return (2048 / cr) * (1 + cluster_helpers(cr)); }

template <int CR>
__global__ void __cluster_dims__(CR, 1, 1) __launch_bounds__(cluster_threads(CR), 1)
    plain_cluster_kernel(const __grid_constant__ PlainJob job) {
    constexpr int NWJ = 64;
    constexpr int CT = 2048 / CR;                 // owned slots (deciding threads) per CTA
    constexpr int LPC = 256 / CR;                 // RNG lanes per CTA
    constexpr int NH = cluster_helpers(CR);       // helper threads per slot, each summing part of its update
    constexpr bool HELP = NH > 0;
    constexpr int BPT = 4 / (NH + 1);             // 16-word blocks of the update per thread
    static_assert((CR == 8 || CR == 16) && (CT / 32) * CR == 64, "64 exchange words per step");
    extern __shared__ __align__(16) uint8_t smem_raw[];
    // J row of owned slot t in exchange-word order: 16 chunks of 16 bytes, chunk c at position c ^ (t & 7)
    // (conflict-free 16-byte loads)
    uint4* Jr = reinterpret_cast<uint4*>(smem_raw);                     // [CT][16]
    // [2 parities][64 words] of {flip, new spin +1, band count | flip count << 16, 0}: one 16-byte push per word
    uint4* FX = Jr + CT * 16;
    int32_t* Dh = reinterpret_cast<int32_t*>(FX + 2 * 64);               // [2][NH][CT]: helpers' partial D
    uint64_t* mbar = reinterpret_cast<uint64_t*>(Dh + 2 * NH * CT);      // [2]: exchange of each parity
    __shared__ long long s_red[2][CT / 32];
    __shared__ long long s_part[CR][3];                     // rank 0: every rank's sum of s*h, of b*s and flips

    // warp w covers rounds w * 32 / LPC ..; its lane holds round k of RNG lane l of this CTA's LPC lanes. Thread
    // st + j CT (j = 1 .. NH) is update helper j of slot st.
    const int tid = threadIdx.x, st = tid % CT, lane = st & 31, w = st >> 5, role = tid / CT;
    const bool decider = role == 0;
    const int k = w * (32 / LPC) + lane / LPC;
    const uint32_t rank = cl_rank();
    const int c = int(cl_id());                             // anneal index within the launch
    const int n = job.n, nw = job.nw, S = job.tab.S;
    const int32_t hclamp = job.hclamp;
    const int32_t* __restrict__ bias = job.bias;
    const int rlane = LPC * int(rank) + lane % LPC;         // RNG lane
    const int slot = k * kLanes + rlane;
    const bool valid = slot < n;
    const int wi_own = w * CR + int(rank);                  // this warp's exchange word

    if (tid == 0) {
        for (int q = 0; q < 2; ++q)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sm_addr(mbar + q)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // each thread of a slot loads the words of the row it sums: words 16 BPT role .. 16 BPT (role + 1) - 1
    const int wlo = 16 * BPT * role, whi = wlo + 16 * BPT;        // (role is 0 or 1 with one helper)
    if (LPC == 32) {
        // exchange word w * 8 + r is spin word w * 8 + r: the row as stored
        const uint4* row = reinterpret_cast<const uint4*>(job.planes + size_t(slot) * NWJ);
        for (int ch = wlo / 4; ch < whi / 4; ++ch) Jr[st * 16 + (ch ^ (st & 7))] = __ldg(row + ch);
    } else {
        // exchange word w * 16 + r holds the 16 lanes 16 r .. of rounds 2w (low half) and 2w + 1 (high half): halves
        // of spin words 2w * 8 + r / 2 and (2w + 1) * 8 + r / 2
        const uint32_t* row = job.planes + size_t(slot) * NWJ;
        uint32_t* Jw = reinterpret_cast<uint32_t*>(Jr + st * 16);
        for (int wi = wlo; wi < whi; ++wi) {
            const int ww = wi / CR, rr = wi % CR;
            const uint32_t A = __ldg(row + (2 * ww) * 8 + rr / 2), B = __ldg(row + (2 * ww + 1) * 8 + rr / 2);
            Jw[4 * ((wi >> 2) ^ (st & 7)) + (wi & 3)] = __byte_perm(A, B, (rr & 1) ? 0x7632 : 0x5410);
        }
    }
    // remote addresses this thread pushes to (lanes 0 .. CR - 1: CTA `lane`), word wi_own of each buffer
    const uint32_t dst_rank = uint32_t(lane % CR);
    const uint32_t dst_fx = cl_map(sm_addr(FX + wi_own), dst_rank);
    const uint32_t dst_mb = cl_map(sm_addr(mbar), dst_rank);

    Xoshiro rng;
    rng_seed(rng, job.seed, job.trial_offset + uint32_t(c), uint32_t(rlane));
    const uint32_t r0 = lane_draw(rng, k);
    bool s_up = valid ? (r0 >> 31) != 0u : true;            // padding slots: +1
    bool df = valid && !s_up;                               // s != s_prev (s_prev = +1 initially)
    int32_t h = (valid && bias) ? bias[slot] : 0;
    uint32_t u = lane_draw(rng, k);                         // step 0's draw
    int32_t nlin_prev = 0;
    long long flips = 0;
    bool ok = true;                                         // false once a wait gave up
    // the initial pass publishes F = active slots and U = s0
    bool fl = valid, up_new = s_up, ln = false;
    // this step's table entries, loaded one step ahead (off the decision's critical path)
    int32_t fourT_n = __ldg(job.tab.fourT), q_n = __ldg(job.tab.q), kconst_n = __ldg(job.tab.kconst);
    int64_t kcorr_n = __ldg(job.tab.kcorr);
    cl_sync();                                              // barriers initialised and J loaded in every CTA

    if (HELP && !decider) {
        // helper `role`: the partial D of slot st over its blocks of every step, handed over through Dh
        for (int m = 0; m <= S; ++m) {
            const int par = m & 1;
            if (ok && !cl_wait_for(sm_addr(mbar + par), uint32_t((m >> 1) & 1), job.wait_ns)) {
                ok = false;
                if (job.err) atomicCAS(job.err, 0, kClusterErrRecv);
            }
            Dh[(par * NH + role - 1) * CT + st] = cluster_words_d<BPT>(
                Jr + st * 16, FX + par * 64, st & 7, NH == 1 ? BPT : BPT * role);
            asm volatile("bar.arrive 1, %0;" ::"r"(cluster_threads(CR)) : "memory");
        }
    } else {
        for (int t = -1; t < S; ++t) {
            const int m = t + 1, par = m & 1;
            if (t >= 0) {
                const int32_t fourT = fourT_n, twoT = fourT >> 1, qv = q_n;
                const int32_t corr = step_corr(nlin_prev, kcorr_n, kconst_n);
                const uint32_t lw = uint32_t(2 * twoT - 1);
                if (t + 1 < S) {
                    fourT_n = __ldg(job.tab.fourT + t + 1);
                    q_n = __ldg(job.tab.q + t + 1);
                    kconst_n = __ldg(job.tab.kconst + t + 1);
                    kcorr_n = __ldg(job.tab.kcorr + t + 1);
                }
                int32_t hs = s_up ? h : -h;
                if (hclamp > 0) hs = max(-hclamp, min(hs, hclamp));
                const int32_t zt = hs * 65536 + (qv + (df ? corr : -corr));
                fl = valid && (zt - threshold16(u, fourT) < 0);
                ln = valid && (uint32_t(zt + twoT - 1) < lw);
                up_new = s_up != fl;
            }
            const uint32_t fw = __ballot_sync(FULL, fl), uw = __ballot_sync(FULL, fl && up_new);
            const uint32_t nlw = __ballot_sync(FULL, ln);
            if (lane < CR) {
                const uint32_t bar = dst_mb + 8u * uint32_t(par);
                st_async4(dst_fx + 16u * 64u * uint32_t(par), fw, uw,
                          uint32_t(__popc(nlw)) | (uint32_t(__popc(fw)) << 16), 0u, bar);
            }
            const uint32_t my_bar = sm_addr(mbar + par);
            if (tid == 0)
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(my_bar), "r"(kClusterTx)
                             : "memory");
            if (t >= 0) {
                if (fl) s_up = up_new;
                df = fl;
                if (t + 1 < S) u = lane_draw(rng, k);            // next step's draw, while the words travel
            }
            if (ok && !cl_wait_for(my_bar, uint32_t((m >> 1) & 1), job.wait_ns)) {
                ok = false;
                if (job.err) atomicCAS(job.err, 0, kClusterErrRecv);
            }
            // n_lin and |F| of step t: each warp sums the 64 packed counts (low half: band, high half: flips)
            // (one warp reduction instruction instead of a chain of five shuffles; records lane and lane + 32, so a
            // load's 32 fields fall on 8 banks, where records 2 lane and 2 lane + 1 fell on 4)
            const uint32_t pc = __reduce_add_sync(FULL, FX[par * 64 + lane].z + FX[par * 64 + 32 + lane].z);
            int32_t nf = int32_t(pc >> 16);
            if (t >= 0) {
                nlin_prev = int32_t(pc & 0xffffu);
                if (rank == 0 && tid == 0 && job.trace && job.out_trace) job.out_trace[size_t(c) * S + t] = nlin_prev;
                if (tid == 0) flips += nf;
            }
            // D: the 64 words at once, or the first blocks here and the rest by the helpers (handed over at barrier 1)
            const uint4* FXv = FX + par * 64;
            const uint4* Jv = Jr + st * 16;
            int32_t D;
            if (HELP) {
                D = cluster_words_d<BPT>(Jv, FXv, st & 7, 0);
                asm volatile("bar.sync 1, %0;" ::"r"(cluster_threads(CR)) : "memory");
#pragma unroll
                for (int j = 0; j < NH; ++j) D += Dh[(par * NH + j) * CT + st];
            } else {
                D = cluster_words_d<4>(Jv, FXv, st & 7, 0);
            }
            // the diagonal: if y itself is in F, its term (J_yy = 0, stored as a 0 bit) was counted as -s'_y
            if (fl) {
                nf -= 1;
                D -= up_new ? 1 : 0;
            }
            h += (t >= 0 ? 2 : 1) * (nf - 2 * D);
        }
        // outputs: spins, sum s*h, sum b*s (active slots), flips
        long long sh = 0, bs = 0;
        if (valid) {
            sh = s_up ? h : -h;
            if (bias) bs = s_up ? bias[slot] : -bias[slot];
            if (job.out_h) job.out_h[size_t(c) * n + slot] = h;
        }
        const uint32_t sword = __ballot_sync(FULL, s_up);
        if (lane == 0) {
            if (LPC == 32) {
                if (wi_own < nw) job.out_spins[size_t(c) * nw + wi_own] = sword & valid_mask(wi_own, n);
            } else {
                // the two 16-bit halves of the exchange word are half words of spin words 2w * 8 + r / 2 and
                // (2w + 1) * 8 + r / 2; every half of every spin word is written by exactly one CTA
                uint16_t* out16 = reinterpret_cast<uint16_t*>(job.out_spins + size_t(c) * nw);
                for (int hh = 0; hh < 2; ++hh) {
                    const int sw_i = (2 * w + hh) * 8 + int(rank) / 2, half = int(rank) & 1;
                    if (sw_i < nw)
                        out16[2 * sw_i + half] = uint16_t(((sword >> (16 * hh)) & 0xffffu) &
                                                          (valid_mask(sw_i, n) >> (16 * half)));
                }
            }
        }
        sh = warp_sum64(sh);
        bs = warp_sum64(bs);
        if (lane == 0) {
            s_red[0][w] = sh;
            s_red[1][w] = bs;
        }
    }
    if (!ok) {
        // a wait gave up: let pushes still in flight toward this CTA land before the cluster may exit
        const uint64_t t0 = cl_globaltimer();
        while (cl_globaltimer() - t0 < 200000ull) {
        }
    }
    __syncthreads();
    if (tid == 0) {
        long long a = 0, b = 0;
        for (int ww = 0; ww < CT / 32; ++ww) { a += s_red[0][ww]; b += s_red[1][ww]; }
        const uint32_t ad = cl_map(sm_addr(&s_part[rank][0]), 0u);
        asm volatile("st.shared::cluster.u64 [%0], %1;" ::"r"(ad), "l"(a) : "memory");
        asm volatile("st.shared::cluster.u64 [%0], %1;" ::"r"(ad + 8u), "l"(b) : "memory");
        asm volatile("st.shared::cluster.u64 [%0], %1;" ::"r"(ad + 16u), "l"(flips) : "memory");
    }
    cl_sync();
    if (rank == 0 && tid == 0) {
        long long a = 0, b = 0;
        for (int r = 0; r < CR; ++r) { a += s_part[r][0]; b += s_part[r][1]; }
        job.out_sum_sh[c] = a;
        if (job.out_sum_bs) job.out_sum_bs[c] = b;
        job.out_flips[c] = s_part[0][2];
    }
}

template <int K, int P, bool SPARSE, bool STREAM = false, int SB = 1, int SE = 8, int DV = 0>
int launch_t(const PlainLaunch& L, int grid, size_t smem, cudaStream_t st) {
    auto fn = plain_kernel<K, P, SPARSE, STREAM, SB, SE, DV>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return int(e);
    fn<<<grid, T, smem, st>>>(L);
    return int(cudaGetLastError());
}

template <int K, int P, bool SPARSE, bool STREAM = false>
int occ_t(size_t smem, int* out) {
    auto fn = plain_kernel<K, P, SPARSE, STREAM>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return int(e);
    return int(cudaOccupancyMaxActiveBlocksPerMultiprocessor(out, fn, T, smem));
}

}  // namespace

// K: 0 = sparse, 1/2/4 dense planes. P: 12 or 16 counter planes (dense only). L.stream selects the streaming layout
// (K = 2 / 4, P = 16 only: it is needed only for NP > 8192).
int plain_launch(const PlainLaunch& L, int K, int P, int grid, size_t smem, cudaStream_t st) {
    if (K == 0) {
        switch (L.sparse_variant) {
            case 1: return launch_t<1, 12, true, false, 1, 4>(L, grid, smem, st);
            case 2: return launch_t<1, 12, true, false, 2, 4>(L, grid, smem, st);
            case 3: return launch_t<1, 12, true, false, 1, 16>(L, grid, smem, st);
            default: return launch_t<1, 12, true, false, 1, 8>(L, grid, smem, st);
        }
    }
    if (L.stream) {
        if (P == 16 && K == 2) return launch_t<2, 16, false, true>(L, grid, smem, st);
        if (P == 16 && K == 4) return launch_t<4, 16, false, true>(L, grid, smem, st);
        return int(cudaErrorInvalidValue);
    }
    const int dv = L.dense_variant;
    if (P == 12) {
        if (K == 1) {
            if (dv == 1) return launch_t<1, 12, false, false, 1, 8, 1>(L, grid, smem, st);
            if (dv == 2) return launch_t<1, 12, false, false, 1, 8, 2>(L, grid, smem, st);
            return launch_t<1, 12, false>(L, grid, smem, st);
        }
        if (K == 2) {
            if (dv == 1) return launch_t<2, 12, false, false, 1, 8, 1>(L, grid, smem, st);
            return launch_t<2, 12, false>(L, grid, smem, st);
        }
        if (K == 4) return launch_t<4, 12, false>(L, grid, smem, st);
    } else if (P == 16) {
        if (K == 1) {
            if (dv == 1) return launch_t<1, 16, false, false, 1, 8, 1>(L, grid, smem, st);
            if (dv == 2) return launch_t<1, 16, false, false, 1, 8, 2>(L, grid, smem, st);
            return launch_t<1, 16, false>(L, grid, smem, st);
        }
        if (K == 2) {
            if (dv == 1) return launch_t<2, 16, false, false, 1, 8, 1>(L, grid, smem, st);
            return launch_t<2, 16, false>(L, grid, smem, st);
        }
        if (K == 4) return launch_t<4, 16, false>(L, grid, smem, st);
    }
    return int(cudaErrorInvalidValue);
}

bool plain_cluster_supported(int K, int np) { return K == 1 && np == 2048; }

namespace {
// The cluster kernel for `cr` CTAs per anneal with its attributes set (16 is a non-portable cluster size).
template <int CR>
cudaError_t cluster_prepare() {
    auto fn = plain_cluster_kernel<CR>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kClusterSmem));
    if (e == cudaSuccess && CR > 8) e = cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    return e;
}
template <int CR>
int cluster_launch_t(const PlainJob& job, cudaStream_t st) {
    cudaError_t e = cluster_prepare<CR>();
    if (e != cudaSuccess) return int(e);
    plain_cluster_kernel<CR><<<job.ntrials * CR, cluster_threads(CR), kClusterSmem, st>>>(job);
    return int(cudaGetLastError());
}
template <int CR>
int cluster_max_active_t(int* out) {
    cudaError_t e = cluster_prepare<CR>();
    if (e != cudaSuccess) return int(e);
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = CR;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cfg.gridDim = dim3(CR);
    cfg.blockDim = dim3(cluster_threads(CR));
    cfg.dynamicSmemBytes = kClusterSmem;
    return int(cudaOccupancyMaxActiveClusters(out, plain_cluster_kernel<CR>, &cfg));
}
}  // namespace

int plain_cluster_launch(const PlainJob& job, cudaStream_t st, int ctas) {
    return ctas == 16 ? cluster_launch_t<16>(job, st) : cluster_launch_t<8>(job, st);
}

int plain_cluster_max_active(int* out, int ctas) {
    return ctas == 16 ? cluster_max_active_t<16>(out) : cluster_max_active_t<8>(out);
}

int plain_max_blocks_per_sm(int K, int P, size_t smem, int* out, bool stream) {
    if (K == 0) return occ_t<1, 12, true>(smem, out);
    if (stream) {
        if (P == 16 && K == 2) return occ_t<2, 16, false, true>(smem, out);
        if (P == 16 && K == 4) return occ_t<4, 16, false, true>(smem, out);
        return int(cudaErrorInvalidValue);
    }
    if (P == 12) {
        if (K == 1) return occ_t<1, 12, false>(smem, out);
        if (K == 2) return occ_t<2, 12, false>(smem, out);
        if (K == 4) return occ_t<4, 12, false>(smem, out);
    } else if (P == 16) {
        if (K == 1) return occ_t<1, 16, false>(smem, out);
        if (K == 2) return occ_t<2, 16, false>(smem, out);
        if (K == 4) return occ_t<4, 16, false>(smem, out);
    }
    return int(cudaErrorInvalidValue);
}

}  // namespace anc
