// Mean-field relaxation kernels (see anc_meanfield.cuh for the recurrence): the J x m GEMM on tcgen05 (kind::f16,
// BF16 operands, f32 accumulation in TMEM) and the fused forward / adjoint elementwise steps.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <utility>
#include <vector>

#include "anc_meanfield.cuh"
#include "anc_ptx.cuh"

namespace anc {

struct MfContext {
    int n = 0, npad = 0;
    __nv_bfloat16* J = nullptr;       // [npad][npad] (zero padded)
    float* bias = nullptr;            // [npad]
    float* partial = nullptr;         // [npad / 256][64][npad] split-K partial products
    float* mring = nullptr;           // forward ring: 3 x [64][npad]
    __nv_bfloat16* xm = nullptr;      // [3][64][npad]: hi / mid / lo of the m operand
    __nv_bfloat16* xp = nullptr;      // [3][64][npad]: hi / mid / lo of the adjoint operand
    float* seg_m = nullptr;           // [kMfCheckpoint + 2][64][npad]: m_{t0-1} .. m_{t0+16} of a segment
    float* seg_P = nullptr;           // [kMfCheckpoint][64][npad]
    float* pbar = nullptr;            // [3][64][npad] ring of pbar_t
    float* svec = nullptr;            // [3][nch][64] ring of s_t, per 256-column chunk
    float* nbuf = nullptr;            // [S + 1][nch][64] soft counts n_t, per 256-column chunk
    float* gparts = nullptr;          // [S][4][nch][64] per-chunk schedule-gradient sums
    int nbuf_steps = 0;
    int* err = nullptr;               // device error word
    uint64_t wait_ns = ptx::kWaitNs;  // limit of each device wait before the kernel gives up (recorded in the graphs)
    CUtensorMap mapJ, mapXm[3], mapXp[3];
    // CUDA graphs of the forward and adjoint launch sequences (one step count each), captured on internal buffers:
    // the caller's inputs are copied in and the outputs copied out around each graph launch
    cudaStream_t cap = nullptr;
    cudaGraphExec_t fwd_exec = nullptr, bwd_exec = nullptr;
    int fwd_S = 0, bwd_S = 0, io_steps = 0;
    float* sched_i = nullptr;         // [4][S]
    float* m0_i = nullptr;            // [64][npad]
    float* mprev_i = nullptr;
    float* mout_i = nullptr;
    float* gm_i = nullptr;
    float* ckpt_i = nullptr;          // [ceil(S/16)][2][64][npad]
    float* gs_i = nullptr;            // [S][4][64]
};

namespace {

using namespace ptx;

// Programmatic dependent launch. Every kernel of a step sequence lets the next one in the stream launch right away
// (pdl_trigger), so that kernel's prologue -- TMEM allocation, barrier set-up, the TMA load of its J tile -- overlaps
// this kernel; it then waits for this kernel to complete, with its memory visible (pdl_wait), before reading anything
// this kernel wrote. Both are no-ops in a kernel launched without the programmatic-serialization attribute.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

constexpr int kRows = 128;                 // rows of J per CTA (MMA M)
constexpr int kRep = kMfReplicas;          // MMA N
constexpr int kKC = 256;                   // K per CTA: 4 swizzle atoms of 64 BF16
constexpr int kGemmThreads = 128;
constexpr int kElemThreads = 256;
constexpr int kErrFull = 11, kErrDone = 12;
constexpr uint32_t kATile = kRows * 128;   // 16 KB: 128 rows x 64 BF16
constexpr uint32_t kBTile = kRep * 128;    // 8 KB: 64 rows x 64 BF16

size_t gemm_smem() { return 1024 + 4 * size_t(kATile) + 12 * size_t(kBTile) + 64; }

// partial[ks][r][y] = sum_{x in [256 ks, 256 ks + 256)} J[y][x] * (X0 + X1 + X2)[r][x], X = the three BF16 terms of
// an f32 operand (24 significant bits; J is exact in BF16, so every product is exact); grid (npad / 128, npad / 256).
__global__ void __launch_bounds__(kGemmThreads, 1)
    mf_gemm_kernel(const __grid_constant__ CUtensorMap mapJ, const __grid_constant__ CUtensorMap mapXh,
                   const __grid_constant__ CUtensorMap mapXm, const __grid_constant__ CUtensorMap mapXl,
                   float* __restrict__ partial, int npad, int* err, uint64_t wait_ns) {
    // kind::f16 instruction descriptor: f32 accumulator, BF16 A and B, both K-major, N = 64, M = 128
    constexpr uint32_t IDESC =
        (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(kRep >> 3) << 17) | (uint32_t(kRows >> 4) << 24);
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sa = smem;
    uint8_t* sbh = sa + 4 * kATile;
    uint8_t* sbm = sbh + 4 * kBTile;
    uint8_t* sbl = sbm + 4 * kBTile;
    uint64_t* bars = reinterpret_cast<uint64_t*>(sbl + 4 * kBTile);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int y0 = blockIdx.x * kRows, k0 = blockIdx.y * kKC;
    const uint32_t bar_full = smem_u32(bars), bar_done = smem_u32(bars + 1);
    pdl_trigger();
    if (tid == 0) {
        mbar_init(bar_full, 1);
        mbar_init(bar_done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(512)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    if (tid == 0) {
        mbar_arrive_expect_tx(bar_full, 4 * (kATile + 3 * kBTile));
        for (int a = 0; a < 4; ++a) tma_load_2d(smem_u32(sa + a * kATile), &mapJ, k0 + 64 * a, y0, bar_full);
        // the operand terms come from the previous kernel; the partials this CTA writes are read by the previous
        // step's elementwise kernel: both only after it completed. The other threads write only after bar_done,
        // which follows this wait.
        pdl_wait();
        for (int a = 0; a < 4; ++a) {
            tma_load_2d(smem_u32(sbh + a * kBTile), &mapXh, k0 + 64 * a, 0, bar_full);
            tma_load_2d(smem_u32(sbm + a * kBTile), &mapXm, k0 + 64 * a, 0, bar_full);
            tma_load_2d(smem_u32(sbl + a * kBTile), &mapXl, k0 + 64 * a, 0, bar_full);
        }
        // a wait that gives up (after wait_ns) records the error, then waits once more, bounded by kWaitNs, for the
        // copies it issued, so that none is in flight when the CTA skips its MMAs and exits
        const bool ok = mbar_wait_for(bar_full, 0u, err, kErrFull, wait_ns);
        if (!ok) mbar_wait_for(bar_full, 0u, nullptr, 0, kWaitNs);
        tc_fence_after();
        if (ok) {
            // The tensor core's f32 accumulation truncates toward zero each time an MMA adds into an accumulator, a
            // bias of up to half an ulp of the accumulator per add. Keeping the leading-term products of each 64-wide
            // K atom in their own accumulator (columns 64a .. 64a + 63) and the small mid / lo products in a fifth
            // (columns 256 ..) keeps the accumulators small and the adds per accumulator few; the epilogue sums them
            // with round-to-nearest.
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int kk = 0; kk < 4; ++kk)
                    mma_f16(tmem + uint32_t(64 * a), sw128_desc(smem_u32(sa + a * kATile) + 32 * kk),
                            sw128_desc(smem_u32(sbh + a * kBTile) + 32 * kk), IDESC, kk != 0 ? 1u : 0u);
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int kk = 0; kk < 4; ++kk) {
                    mma_f16(tmem + 256u, sw128_desc(smem_u32(sa + a * kATile) + 32 * kk),
                            sw128_desc(smem_u32(sbm + a * kBTile) + 32 * kk), IDESC, (a | kk) != 0 ? 1u : 0u);
                    mma_f16(tmem + 256u, sw128_desc(smem_u32(sa + a * kATile) + 32 * kk),
                            sw128_desc(smem_u32(sbl + a * kBTile) + 32 * kk), IDESC, 1u);
                }
        }
        mma_commit(bar_done);
    }
    __syncwarp();
    if (!mbar_wait_for(bar_done, 0u, err, kErrDone, wait_ns)) mbar_wait_for(bar_done, 0u, nullptr, 0, kWaitNs);
    tc_fence_after();
    // warp w reads TMEM lanes 32w .. 32w + 31 = rows y0 + 32w + lane; columns = replicas
    const int y = y0 + warp * 32 + lane;
    float* dst = partial + size_t(blockIdx.y) * kRep * npad + y;
    const uint32_t tl = tmem + (uint32_t(warp * 32) << 16);
    uint32_t v[32];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        float s01[32], s23[32];
        tmem_ld32(tl + uint32_t(32 * h), v);
        tmem_wait_ld();
#pragma unroll
        for (int e = 0; e < 32; ++e) s01[e] = __uint_as_float(v[e]);
        tmem_ld32(tl + uint32_t(64 + 32 * h), v);
        tmem_wait_ld();
#pragma unroll
        for (int e = 0; e < 32; ++e) s01[e] += __uint_as_float(v[e]);
        tmem_ld32(tl + uint32_t(128 + 32 * h), v);
        tmem_wait_ld();
#pragma unroll
        for (int e = 0; e < 32; ++e) s23[e] = __uint_as_float(v[e]);
        tmem_ld32(tl + uint32_t(192 + 32 * h), v);
        tmem_wait_ld();
#pragma unroll
        for (int e = 0; e < 32; ++e) s23[e] += __uint_as_float(v[e]);
        tmem_ld32(tl + uint32_t(256 + 32 * h), v);
        tmem_wait_ld();
#pragma unroll
        for (int e = 0; e < 32; ++e) dst[size_t(32 * h + e) * npad] = (s01[e] + s23[e]) + __uint_as_float(v[e]);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
    }
}

// v = x[0] + x[1] + x[2] + O(2^-24 |v|): three BF16 terms, each rounding the remainder of the previous ones.
__device__ __forceinline__ void split_bf16(float v, __nv_bfloat16* x, size_t plane) {
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    const float r1 = v - __bfloat162float(h);
    const __nv_bfloat16 m = __float2bfloat16_rn(r1);
    x[0] = h;
    x[plane] = m;
    x[2 * plane] = __float2bfloat16_rn(r1 - __bfloat162float(m));
}

// Deterministic block sum (fixed shuffle tree, then warp 0 over the warp partials); the result is valid in warp 0.
template <int NV>
__device__ __forceinline__ void block_sum(float (&v)[NV], float* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    }
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) red[k * 32 + warp] = v[k];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            float x = lane < nw ? red[k * 32 + lane] : 0.f;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
            v[k] = x;
        }
    }
}

// Sum of replica r's per-chunk partials parts[ch][r], in chunk order (deterministic).
__device__ __forceinline__ float sum_parts(const float* __restrict__ parts, int nch, int r) {
    float v = 0.f;
    for (int ch = 0; ch < nch; ++ch) v += parts[ch * kRep + r];
    return v;
}

// Elementwise kernels run on a (replica, 256-column chunk) grid, one element per thread; per-replica sums are
// written per chunk (parts[chunk][replica]) and summed in chunk order by their readers.

// Soft count partials n[ch][r] = sum_{i in chunk, i < n} (1 - m[r,i]^2) and the BF16 terms of m.
__global__ void __launch_bounds__(kElemThreads) mf_prep_kernel(const float* __restrict__ m, int n, int npad,
                                                               float* __restrict__ nout, __nv_bfloat16* __restrict__ x) {
    __shared__ float red[32];
    pdl_trigger();
    pdl_wait();
    const int r = blockIdx.x, i = blockIdx.y * kElemThreads + threadIdx.x;
    const size_t idx = size_t(r) * npad + i;
    const float v = m[idx];
    split_bf16(v, x + idx, size_t(kRep) * npad);
    float acc[1] = {i < n ? 1.f - v * v : 0.f};
    block_sum(acc, red);
    if (threadIdx.x == 0) nout[blockIdx.y * kRep + r] = acc[0];
}

struct FwdArgs {
    const float* partial;
    int ksplit, npad, n, t;
    const float* bias;
    const float *beta, *q, *u, *w;
    const float* m_cur;
    const float* m_prev;
    const float* n_cur;      // [nch][64] partials of n_t
    float* m_next;
    __nv_bfloat16* x;        // BF16 terms of m_next [3][64][npad]
    float* n_next;           // [nch][64] partials of n_{t+1}
    float* P_out;            // [64][npad] or null
};

__global__ void __launch_bounds__(kElemThreads) mf_fwd_kernel(const FwdArgs a) {
    __shared__ float red[32];
    pdl_trigger();
    pdl_wait();
    const int r = blockIdx.x, npad = a.npad, nch = gridDim.y, i = blockIdx.y * kElemThreads + threadIdx.x;
    const float beta = a.beta[a.t], q = a.q[a.t];
    const float gamma = a.u[a.t] * sum_parts(a.n_cur, nch, r) + a.w[a.t];
    const size_t idx = size_t(r) * npad + i;
    float H = 0.f;
    for (int ks = 0; ks < a.ksplit; ++ks) H += a.partial[(size_t(ks) * kRep + r) * npad + i];
    const float P = H + a.bias[i] + q * a.m_cur[idx] - gamma * a.m_prev[idx];
    const float mn = i < a.n ? tanhf(beta * P) : 0.f;
    a.m_next[idx] = mn;
    split_bf16(mn, a.x + idx, size_t(kRep) * npad);
    if (a.P_out) a.P_out[idx] = P;
    float acc[1] = {i < a.n ? 1.f - mn * mn : 0.f};
    block_sum(acc, red);
    if (threadIdx.x == 0) a.n_next[blockIdx.y * kRep + r] = acc[0];
}

struct BwdArgs {
    const float* partial;      // J pbar_{t+1} split-K partials, or null when t = S - 1
    int ksplit, npad, n, t, S;
    const float* g_final;      // dL/dm_S (used when t = S - 1)
    const float* pbar_next;    // pbar_{t+1} or null
    const float* pbar_next2;   // pbar_{t+2} or null
    const float* s_next;       // partials of s_{t+1} [nch][64], or null
    const float* n_next2;      // partials of n_{t+2} [nch][64], or null
    const float *beta, *q, *u, *w;
    const float* m_next;       // m_{t+1}
    const float* m_cur;        // m_t
    const float* m_prev;       // m_{t-1}
    const float* P;            // P_t
    const float* n_cur;        // partials of n_t [nch][64]
    float* pbar;               // out: pbar_t
    __nv_bfloat16* x;          // out: BF16 terms of pbar_t [3][64][npad]
    float* s_out;              // out: partials of s_t [nch][64]
    float* gparts;             // out: [S][4][nch][64] partials
};

// One adjoint step t:
//   G      = dL/dm_{t+1} = J pbar_{t+1} + q_{t+1} pbar_{t+1} + 2 u_{t+1} s_{t+1} m_{t+1} - gamma_{t+2} pbar_{t+2}
//            (dL/dm_S given at t = S - 1)
//   abar_t = G (1 - m_{t+1}^2),  pbar_t = beta_t abar_t,  s_t = sum_i pbar_t m_{t-1}
//   dL/dbeta_t += sum abar_t P_t, dL/dq_t += sum pbar_t m_t, dL/du_t += -s_t n_t, dL/dw_t += -s_t
__global__ void __launch_bounds__(kElemThreads) mf_bwd_kernel(const BwdArgs a) {
    __shared__ float red[3 * 32];
    pdl_trigger();
    pdl_wait();
    const int r = blockIdx.x, npad = a.npad, t = a.t, nch = gridDim.y, ch = blockIdx.y;
    const int i = ch * kElemThreads + threadIdx.x;
    const float beta = a.beta[t];
    const bool last = t == a.S - 1;
    const float q1 = last ? 0.f : a.q[t + 1];
    const float us = last ? 0.f : 2.f * a.u[t + 1] * sum_parts(a.s_next, nch, r);
    const float g2 = a.pbar_next2 ? a.u[t + 2] * sum_parts(a.n_next2, nch, r) + a.w[t + 2] : 0.f;
    const size_t idx = size_t(r) * npad + i;
    float G;
    if (last) {
        G = a.g_final[idx];
    } else {
        float H = 0.f;
        for (int ks = 0; ks < a.ksplit; ++ks) H += a.partial[(size_t(ks) * kRep + r) * npad + i];
        G = H + q1 * a.pbar_next[idx] + us * a.m_next[idx];
        if (a.pbar_next2) G -= g2 * a.pbar_next2[idx];
    }
    const float mn = a.m_next[idx];
    const float abar = i < a.n ? G * (1.f - mn * mn) : 0.f;
    const float pb = beta * abar;
    a.pbar[idx] = pb;
    split_bf16(pb, a.x + idx, size_t(kRep) * npad);
    float acc[3] = {abar * a.P[idx], pb * a.m_cur[idx], pb * a.m_prev[idx]};   // abar P, pbar m_t, pbar m_{t-1}
    block_sum(acc, red);
    if (threadIdx.x == 0) {
        a.s_out[ch * kRep + r] = acc[2];
        float* g = a.gparts + size_t(t) * 4 * nch * kRep;
        g[(0 * nch + ch) * kRep + r] = acc[0];
        g[(1 * nch + ch) * kRep + r] = acc[1];
        g[(2 * nch + ch) * kRep + r] = -acc[2] * sum_parts(a.n_cur, nch, r);
        g[(3 * nch + ch) * kRep + r] = -acc[2];
    }
}

// gsched[t][k][r] = sum over chunks of gparts[t][k][ch][r] (chunk order); one thread per (t, k, r).
__global__ void mf_gsum_kernel(const float* __restrict__ gparts, int S, int nch, float* __restrict__ gsched) {
    pdl_trigger();
    pdl_wait();
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= S * 4 * kRep) return;
    const int r = e % kRep, tk = e / kRep;
    float v = 0.f;
    for (int ch = 0; ch < nch; ++ch) v += gparts[(size_t(tk) * nch + ch) * kRep + r];
    gsched[e] = v;
}

bool check(cudaError_t e, const char* what, std::string* why) {
    if (e == cudaSuccess) return true;
    if (why) *why = std::string(what) + ": " + cudaGetErrorString(e);
    return false;
}

// Launch with programmatic stream serialization (see pdl_trigger / pdl_wait): the kernel may start while the previous
// kernel in the stream still runs, and waits for it where it reads that kernel's outputs.
template <class... KArgs, class... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                       Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

int gemm(MfContext* c, const CUtensorMap (&mx)[3], cudaStream_t st, std::string* why) {
    const cudaError_t e = launch_pdl(mf_gemm_kernel, dim3(c->npad / kRows, c->npad / kKC), dim3(kGemmThreads),
                                     gemm_smem(), st, c->mapJ, mx[0], mx[1], mx[2], c->partial, c->npad, c->err,
                                     c->wait_ns);
    return check(e, "mean-field GEMM launch", why) ? 0 : -2;
}

float* mslot(float* base, int k, int npad) { return base + size_t(k) * kRep * npad; }

// 256-column chunks of the elementwise grid.
int nch(const MfContext* c) { return c->npad / kElemThreads; }

// Forward steps t = t0 .. t1 - 1: m_t = cur(t), m_{t-1} = prev(t); writes m_{t+1} to next(t) and P_t to pout(t)
// when that is not null. The BF16 terms of m_t must already be in c->xm.
template <class CurFn, class PrevFn, class NextFn, class PFn>
int run_steps(MfContext* c, int t0, int t1, const float* beta, const float* q, const float* u, const float* w,
              CurFn cur, PrevFn prev, NextFn next, PFn pout, cudaStream_t st, std::string* why) {
    const int npad = c->npad;
    for (int t = t0; t < t1; ++t) {
        int rc = gemm(c, c->mapXm, st, why);
        if (rc) return rc;
        FwdArgs a{};
        a.partial = c->partial;
        a.ksplit = npad / kKC;
        a.npad = npad;
        a.n = c->n;
        a.t = t;
        a.bias = c->bias;
        a.beta = beta;
        a.q = q;
        a.u = u;
        a.w = w;
        a.m_cur = cur(t);
        a.m_prev = prev(t);
        a.n_cur = c->nbuf + size_t(t) * nch(c) * kRep;
        a.m_next = next(t);
        a.x = c->xm;
        a.n_next = c->nbuf + size_t(t + 1) * nch(c) * kRep;
        a.P_out = pout(t);
        if (!check(launch_pdl(mf_fwd_kernel, dim3(kRep, nch(c)), dim3(kElemThreads), 0, st, a), "mean-field forward step",
                   why))
            return -2;
    }
    return 0;
}

int ensure_steps(MfContext* c, int S, std::string* why) {
    if (S <= c->nbuf_steps) return 0;
    for (float** p : {&c->nbuf, &c->gparts}) {
        if (*p) cudaFree(*p);
        *p = nullptr;
    }
    c->nbuf_steps = 0;
    if (!check(cudaMalloc(&c->nbuf, size_t(S + 1) * nch(c) * kRep * sizeof(float)), "cudaMalloc", why) ||
        !check(cudaMalloc(&c->gparts, size_t(S) * 4 * nch(c) * kRep * sizeof(float)), "cudaMalloc", why))
        return -2;
    c->nbuf_steps = S;
    return 0;
}

}  // namespace

int mf_npad(const MfContext* c) { return c->npad; }

int mf_create(const int8_t* J, const int32_t* bias, int n, MfContext** out, std::string* why) {
    if (!J || n < 1 || !out) {
        if (why) *why = "J, n >= 1 and an output handle are required";
        return -1;
    }
    auto* c = new MfContext();
    c->n = n;
    c->npad = ((n + 255) / 256) * 256;
    const int npad = c->npad;
    std::vector<__nv_bfloat16> Jh(size_t(npad) * npad, __float2bfloat16(0.f));
    for (int x = 0; x < n; ++x)
        for (int y = 0; y < n; ++y) Jh[size_t(y) * npad + x] = __float2bfloat16(float(J[size_t(x) * n + y]));
    std::vector<float> bh(npad, 0.f);
    if (bias)
        for (int i = 0; i < n; ++i) bh[i] = float(bias[i]);
    const size_t plane = size_t(kRep) * npad;
    bool ok = check(cudaMalloc(&c->J, Jh.size() * sizeof(__nv_bfloat16)), "cudaMalloc", why) &&
              check(cudaMemcpy(c->J, Jh.data(), Jh.size() * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice), "upload J",
                    why) &&
              check(cudaMalloc(&c->bias, npad * sizeof(float)), "cudaMalloc", why) &&
              check(cudaMemcpy(c->bias, bh.data(), npad * sizeof(float), cudaMemcpyHostToDevice), "upload bias", why) &&
              check(cudaMalloc(&c->partial, size_t(npad / kKC) * plane * sizeof(float)), "cudaMalloc", why) &&
              check(cudaMalloc(&c->mring, 3 * plane * sizeof(float)), "cudaMalloc", why) &&
              check(cudaMalloc(&c->xm, 3 * plane * sizeof(__nv_bfloat16)), "cudaMalloc", why) &&
              check(cudaMalloc(&c->xp, 3 * plane * sizeof(__nv_bfloat16)), "cudaMalloc", why) &&
              check(cudaMalloc(&c->seg_m, (kMfCheckpoint + 2) * plane * sizeof(float)), "cudaMalloc", why) &&
              check(cudaMalloc(&c->seg_P, kMfCheckpoint * plane * sizeof(float)), "cudaMalloc", why) &&
              check(cudaMalloc(&c->pbar, 3 * plane * sizeof(float)), "cudaMalloc", why) &&
              check(cudaMalloc(&c->svec, 3 * size_t(npad / kElemThreads) * kRep * sizeof(float)), "cudaMalloc", why) &&
              check(cudaMalloc(&c->err, sizeof(int)), "cudaMalloc", why) &&
              check(cudaMemset(c->err, 0, sizeof(int)), "cudaMemset", why);
    if (ok) {
        ok = make_map_2d(&c->mapJ, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, c->J, npad, npad, 64, kRows);
        for (int k = 0; k < 3 && ok; ++k)
            ok = make_map_2d(&c->mapXm[k], CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, c->xm + k * plane, npad, kRep, 64, kRep) &&
                 make_map_2d(&c->mapXp[k], CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, c->xp + k * plane, npad, kRep, 64, kRep);
        if (!ok && why) *why = "cuTensorMapEncodeTiled failed";
    }
    if (ok)
        ok = check(cudaFuncSetAttribute(mf_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(gemm_smem())),
                   "GEMM attributes", why) &&
             check(cudaStreamCreateWithFlags(&c->cap, cudaStreamNonBlocking), "capture stream", why);
    if (!ok) {
        mf_destroy(c);
        return -2;
    }
    *out = c;
    return 0;
}

namespace {

// The forward launch sequence on explicit buffers (recorded into the forward graph).
int forward_body(MfContext* c, int S, const float* beta, const float* q, const float* u, const float* w,
                 const float* m0, const float* mprev, float* ckpt, float* m_out, cudaStream_t st, std::string* why) {
    int rc = 0;
    const int npad = c->npad;
    const size_t plane = size_t(kRep) * npad;
    float* ring = c->mring;
    if (!check(cudaMemcpyAsync(mslot(ring, 0, npad), mprev, plane * 4, cudaMemcpyDeviceToDevice, st), "copy", why) ||
        !check(cudaMemcpyAsync(mslot(ring, 1, npad), m0, plane * 4, cudaMemcpyDeviceToDevice, st), "copy", why))
        return -2;
    mf_prep_kernel<<<dim3(kRep, nch(c)), kElemThreads, 0, st>>>(mslot(ring, 1, npad), c->n, npad, c->nbuf, c->xm);
    if (!check(cudaGetLastError(), "mean-field prep", why)) return -2;
    // m_t lives in ring slot (t + 1) % 3, m_{t-1} in slot t % 3
    for (int t0 = 0; t0 < S; t0 += kMfCheckpoint) {
        float* ck = ckpt + size_t(t0 / kMfCheckpoint) * 2 * plane;
        if (!check(cudaMemcpyAsync(ck, mslot(ring, t0 % 3, npad), plane * 4, cudaMemcpyDeviceToDevice, st), "ckpt",
                   why) ||
            !check(cudaMemcpyAsync(ck + plane, mslot(ring, (t0 + 1) % 3, npad), plane * 4, cudaMemcpyDeviceToDevice, st),
                   "ckpt", why))
            return -2;
        const int t1 = std::min(S, t0 + kMfCheckpoint);
        rc = run_steps(
            c, t0, t1, beta, q, u, w, [&](int t) { return mslot(ring, (t + 1) % 3, npad); },
            [&](int t) { return mslot(ring, t % 3, npad); }, [&](int t) { return mslot(ring, (t + 2) % 3, npad); },
            [](int) { return static_cast<float*>(nullptr); }, st, why);
        if (rc) return rc;
    }
    if (!check(cudaMemcpyAsync(m_out, mslot(ring, (S + 1) % 3, npad), plane * 4, cudaMemcpyDeviceToDevice, st), "copy",
               why))
        return -2;
    return 0;
}

// The adjoint launch sequence on explicit buffers (recorded into the adjoint graph).
int backward_body(MfContext* c, int S, const float* beta, const float* q, const float* u, const float* w,
                  const float* ckpt, const float* g_m, float* gsched, cudaStream_t st, std::string* why) {
    int rc = 0;
    const int npad = c->npad;
    const size_t plane = size_t(kRep) * npad;
    const int nseg = (S + kMfCheckpoint - 1) / kMfCheckpoint;
    for (int seg = nseg - 1; seg >= 0; --seg) {
        const int t0 = seg * kMfCheckpoint, t1 = std::min(S, t0 + kMfCheckpoint);
        // segment buffer slot k holds m_{t0 - 1 + k}
        const float* ck = ckpt + size_t(seg) * 2 * plane;
        if (!check(cudaMemcpyAsync(mslot(c->seg_m, 0, npad), ck, 2 * plane * 4, cudaMemcpyDeviceToDevice, st), "copy",
                   why))
            return -2;
        mf_prep_kernel<<<dim3(kRep, nch(c)), kElemThreads, 0, st>>>(mslot(c->seg_m, 1, npad), c->n, npad,
                                                                   c->nbuf + size_t(t0) * nch(c) * kRep, c->xm);
        if (!check(cudaGetLastError(), "mean-field prep", why)) return -2;
        rc = run_steps(
            c, t0, t1, beta, q, u, w, [&](int t) { return mslot(c->seg_m, t - t0 + 1, npad); },
            [&](int t) { return mslot(c->seg_m, t - t0, npad); },
            [&](int t) { return mslot(c->seg_m, t - t0 + 2, npad); },
            [&](int t) { return mslot(c->seg_P, t - t0, npad); }, st, why);
        if (rc) return rc;
        for (int t = t1 - 1; t >= t0; --t) {
            const bool last = t == S - 1;
            if (!last) {
                rc = gemm(c, c->mapXp, st, why);
                if (rc) return rc;
            }
            BwdArgs a{};
            a.partial = last ? nullptr : c->partial;
            a.ksplit = npad / kKC;
            a.npad = npad;
            a.n = c->n;
            a.t = t;
            a.S = S;
            a.g_final = g_m;
            a.pbar_next = last ? nullptr : mslot(c->pbar, (t + 1) % 3, npad);
            a.pbar_next2 = t + 2 < S ? mslot(c->pbar, (t + 2) % 3, npad) : nullptr;
            a.s_next = last ? nullptr : c->svec + size_t((t + 1) % 3) * nch(c) * kRep;
            a.n_next2 = t + 2 < S ? c->nbuf + size_t(t + 2) * nch(c) * kRep : nullptr;
            a.beta = beta;
            a.q = q;
            a.u = u;
            a.w = w;
            a.m_next = mslot(c->seg_m, t - t0 + 2, npad);
            a.m_cur = mslot(c->seg_m, t - t0 + 1, npad);
            a.m_prev = mslot(c->seg_m, t - t0, npad);
            a.P = mslot(c->seg_P, t - t0, npad);
            a.n_cur = c->nbuf + size_t(t) * nch(c) * kRep;
            a.pbar = mslot(c->pbar, t % 3, npad);
            a.x = c->xp;
            a.s_out = c->svec + size_t(t % 3) * nch(c) * kRep;
            a.gparts = c->gparts;
            if (!check(launch_pdl(mf_bwd_kernel, dim3(kRep, nch(c)), dim3(kElemThreads), 0, st, a),
                       "mean-field adjoint step", why))
                return -2;
        }
    }
    const int ne = S * 4 * kRep;
    mf_gsum_kernel<<<(ne + 255) / 256, 256, 0, st>>>(c->gparts, S, nch(c), gsched);
    if (!check(cudaGetLastError(), "mean-field gradient sum", why)) return -2;
    return 0;
}

// Internal buffers for S steps (allocated outside any capture; graphs recorded on older buffers are dropped).
int ensure_io(MfContext* c, int S, std::string* why) {
    int rc = ensure_steps(c, S, why);
    if (rc) return rc;
    if (S <= c->io_steps) return 0;
    for (float** p : {&c->sched_i, &c->m0_i, &c->mprev_i, &c->mout_i, &c->gm_i, &c->ckpt_i, &c->gs_i}) {
        if (*p) cudaFree(*p);
        *p = nullptr;
    }
    for (cudaGraphExec_t* g : {&c->fwd_exec, &c->bwd_exec}) {
        if (*g) cudaGraphExecDestroy(*g);
        *g = nullptr;
    }
    c->fwd_S = c->bwd_S = c->io_steps = 0;
    const size_t plane = size_t(kRep) * c->npad;
    const size_t nseg = (S + kMfCheckpoint - 1) / kMfCheckpoint;
    const bool ok = check(cudaMalloc(&c->sched_i, 4 * size_t(S) * 4), "cudaMalloc", why) &&
                    check(cudaMalloc(&c->m0_i, plane * 4), "cudaMalloc", why) &&
                    check(cudaMalloc(&c->mprev_i, plane * 4), "cudaMalloc", why) &&
                    check(cudaMalloc(&c->mout_i, plane * 4), "cudaMalloc", why) &&
                    check(cudaMalloc(&c->gm_i, plane * 4), "cudaMalloc", why) &&
                    check(cudaMalloc(&c->ckpt_i, nseg * 2 * plane * 4), "cudaMalloc", why) &&
                    check(cudaMalloc(&c->gs_i, size_t(S) * 4 * kRep * 4), "cudaMalloc", why);
    if (!ok) return -2;
    c->io_steps = S;
    return 0;
}

// Copy the four schedule vectors into sched_i rows [4][S].
bool copy_sched(MfContext* c, int S, const float* beta, const float* q, const float* u, const float* w, cudaStream_t st,
                std::string* why) {
    const float* v[4] = {beta, q, u, w};
    for (int k = 0; k < 4; ++k)
        if (!check(cudaMemcpyAsync(c->sched_i + size_t(k) * S, v[k], size_t(S) * 4, cudaMemcpyDeviceToDevice, st),
                   "copy schedule", why))
            return false;
    return true;
}

// Record body(cap stream) into *exec once per step count.
template <class Body>
int ensure_graph(MfContext* c, cudaGraphExec_t* exec, int* exec_S, int S, Body body, std::string* why) {
    if (*exec && *exec_S == S) return 0;
    if (*exec) cudaGraphExecDestroy(*exec);
    *exec = nullptr;
    cudaGraph_t g = nullptr;
    if (!check(cudaStreamBeginCapture(c->cap, cudaStreamCaptureModeThreadLocal), "begin capture", why)) return -2;
    const int rc = body(c->cap);
    const cudaError_t e = cudaStreamEndCapture(c->cap, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (!check(e, "end capture", why)) return -2;
    const cudaError_t ei = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    if (!check(ei, "instantiate graph", why)) return -2;
    *exec_S = S;
    return 0;
}

}  // namespace

int mf_forward(MfContext* c, int S, const float* beta, const float* q, const float* u, const float* w, const float* m0,
               const float* mprev, float* ckpt, float* m_out, cudaStream_t st, std::string* why) {
    if (!c || S < 1 || !beta || !q || !u || !w || !m0 || !mprev || !ckpt || !m_out) {
        if (why) *why = "invalid mean-field forward arguments";
        return -1;
    }
    int rc = ensure_io(c, S, why);
    if (rc) return rc;
    const size_t plane = size_t(kRep) * c->npad, nseg = (S + kMfCheckpoint - 1) / kMfCheckpoint;
    rc = ensure_graph(c, &c->fwd_exec, &c->fwd_S, S, [&](cudaStream_t cs) {
        const float* sb = c->sched_i;
        return forward_body(c, S, sb, sb + S, sb + 2 * size_t(S), sb + 3 * size_t(S), c->m0_i, c->mprev_i, c->ckpt_i,
                            c->mout_i, cs, why);
    }, why);
    if (rc) return rc;
    if (!copy_sched(c, S, beta, q, u, w, st, why) ||
        !check(cudaMemcpyAsync(c->m0_i, m0, plane * 4, cudaMemcpyDeviceToDevice, st), "copy m0", why) ||
        !check(cudaMemcpyAsync(c->mprev_i, mprev, plane * 4, cudaMemcpyDeviceToDevice, st), "copy mprev", why) ||
        !check(cudaGraphLaunch(c->fwd_exec, st), "forward graph launch", why) ||
        !check(cudaMemcpyAsync(ckpt, c->ckpt_i, nseg * 2 * plane * 4, cudaMemcpyDeviceToDevice, st), "copy ckpt", why) ||
        !check(cudaMemcpyAsync(m_out, c->mout_i, plane * 4, cudaMemcpyDeviceToDevice, st), "copy m_S", why))
        return -2;
    return 0;
}

int mf_backward(MfContext* c, int S, const float* beta, const float* q, const float* u, const float* w,
                const float* ckpt, const float* g_m, float* gsched, cudaStream_t st, std::string* why) {
    if (!c || S < 1 || !beta || !q || !u || !w || !ckpt || !g_m || !gsched) {
        if (why) *why = "invalid mean-field backward arguments";
        return -1;
    }
    int rc = ensure_io(c, S, why);
    if (rc) return rc;
    const size_t plane = size_t(kRep) * c->npad, nseg = (S + kMfCheckpoint - 1) / kMfCheckpoint;
    rc = ensure_graph(c, &c->bwd_exec, &c->bwd_S, S, [&](cudaStream_t cs) {
        const float* sb = c->sched_i;
        return backward_body(c, S, sb, sb + S, sb + 2 * size_t(S), sb + 3 * size_t(S), c->ckpt_i, c->gm_i, c->gs_i, cs,
                             why);
    }, why);
    if (rc) return rc;
    if (!copy_sched(c, S, beta, q, u, w, st, why) ||
        !check(cudaMemcpyAsync(c->ckpt_i, ckpt, nseg * 2 * plane * 4, cudaMemcpyDeviceToDevice, st), "copy ckpt", why) ||
        !check(cudaMemcpyAsync(c->gm_i, g_m, plane * 4, cudaMemcpyDeviceToDevice, st), "copy dL/dm", why) ||
        !check(cudaGraphLaunch(c->bwd_exec, st), "adjoint graph launch", why) ||
        !check(cudaMemcpyAsync(gsched, c->gs_i, size_t(S) * 4 * kRep * 4, cudaMemcpyDeviceToDevice, st), "copy grads",
               why))
        return -2;
    return 0;
}

int mf_set_wait_ns(MfContext* c, uint64_t ns) {
    if (!c) return -1;
    if (ns == c->wait_ns) return 0;
    c->wait_ns = ns;
    for (cudaGraphExec_t* g : {&c->fwd_exec, &c->bwd_exec}) {   // the limit is a kernel argument: record again
        if (*g) cudaGraphExecDestroy(*g);
        *g = nullptr;
    }
    c->fwd_S = c->bwd_S = 0;
    return 0;
}

int mf_check_error(MfContext* c, cudaStream_t st, std::string* why) {
    int h = 0;
    cudaError_t e = cudaMemcpyAsync(&h, c->err, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (!check(e, "mean-field error word", why)) return -2;
    if (h) {
        if (why) *why = "a bounded device wait expired in the mean-field GEMM (code " + std::to_string(h) + ")";
        cudaMemsetAsync(c->err, 0, 4, st);
        return -3;
    }
    return 0;
}

void mf_destroy(MfContext* c) {
    if (!c) return;
    if (c->fwd_exec) cudaGraphExecDestroy(c->fwd_exec);
    if (c->bwd_exec) cudaGraphExecDestroy(c->bwd_exec);
    if (c->cap) cudaStreamDestroy(c->cap);
    for (void* p : {static_cast<void*>(c->sched_i), static_cast<void*>(c->m0_i), static_cast<void*>(c->mprev_i),
                    static_cast<void*>(c->mout_i), static_cast<void*>(c->gm_i), static_cast<void*>(c->ckpt_i),
                    static_cast<void*>(c->gs_i)})
        if (p) cudaFree(p);
    for (void* p : {static_cast<void*>(c->J), static_cast<void*>(c->bias), static_cast<void*>(c->partial),
                    static_cast<void*>(c->mring), static_cast<void*>(c->xm), static_cast<void*>(c->xp),
                    static_cast<void*>(c->seg_m), static_cast<void*>(c->seg_P), static_cast<void*>(c->pbar),
                    static_cast<void*>(c->svec), static_cast<void*>(c->nbuf), static_cast<void*>(c->gparts),
                    static_cast<void*>(c->err)})
        if (p) cudaFree(p);
    delete c;
}

}  // namespace anc
