// C ABI of the B200 SCA engines (include/anechoic.h): instances, tables, the int32 range plan, launches and readback.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/anechoic.h"
#include "anc_meanfield.cuh"
#include "anc_plain.cuh"
#include "anc_tensor.cuh"

namespace {

thread_local std::string g_err;
thread_local double g_dev_ms = 0.0;
thread_local std::vector<double> g_prof;
thread_local int g_last_kernel = 0;
std::atomic<uint64_t> g_wait_ns{2000000000ull};   // limit of each device wait of the engines' kernels (anc_set_wait_ns)
std::mutex g_batch_tune_mu;                      // guards g_batch_tune
std::map<std::string, int> g_batch_tune;         // CSR pass variant per batch composition (anc_run_batch)
// Run-time choice among the dense kernels' compiled variants (anc_kernel_tuning), per tuning key (device, kernel,
// NP, K, replica groups): the chosen variant and each variant's probe time per step.
struct KernelTune {
    int variant = -1, nvariants = 0;
    double probe_us[4] = {0.0, 0.0, 0.0, 0.0};
};
std::mutex g_kernel_tune_mu;                     // guards g_kernel_tune
std::map<std::array<int, 5>, KernelTune> g_kernel_tune;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    return fail(ANC_ECUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define CK(call)                                                   \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call);        \
    } while (0)

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    ~DevBuf() { if (p) cudaFree(p); }
    cudaError_t ensure(size_t count) {
        if (count <= n && p) return cudaSuccess;
        if (p) { cudaFree(p); p = nullptr; n = 0; }
        cudaError_t e = cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T));
        if (e == cudaSuccess) n = count;
        return e;
    }
};

int pad_np(int n) { return std::max(2048, ((n + 255) / 256) * 256); }

// ---- ANC_ENGINE_AUTO: a cost model of one launch ----
// Device time per annealing step, in microseconds, fitted to B200 measurements: +-1 complete graphs with
// n = 500 ... 10000 and dense 2- and 4-bit instances, under schedules whose flip fractions phi (flips per spin per step)
// span 0.05 ... 0.41.
//   plain    a_K (NP / 2048)^1.5 + c_K phi n^2   a fixed part per step (decisions, n_lin, step barriers); then every
//                                               flip rewrites n fields from one row of bit planes (K planes);
//                                               a_1 = 3.4, a_2 = 5.1, a_4 = 10.2, c_1 = 5.4e-6, c_2 = 1.6e-5,
//                                               c_4 = 3.3e-5 (least squares in log time over the one-wave launches)
//   cluster  0.86 when the anneals fit one wave of 16-CTA clusters (taken as half the 8-CTA wave: 7 here), else
//            1.18 per wave of 8-CTA clusters (1-bit couplings, NP = 2048: every thread sums popcounts over all 64
//            flip words whatever flipped, so the step costs the same at any phi; measured 0.852 - 0.859 for 1 - 7
//            anneals on 16 CTAs, 1.18 - 1.19 per wave of up to 15 on 8)
//   tensor   a constant per kernel: the MMA chain and the decisions cost the same whatever flips: fp4 8.1 (8.3 with
//            more than one replica group per wave), int8 23.3 at NP = 2048, 21.7 and 28.3 at NP = 3072 and 4096,
//            streaming 99.5 (measured 99.5 at NP = 10240 and 98 at NP = 16384: bound by its step latency, not by
//            reading J)
// Each engine advances a fixed number of anneals at once (per_wave); a launch of more takes further waves.
constexpr double kPhiPrior = 0.25;   // flip fraction assumed before any run of these tables on this instance

double plain_step_us(int n, int K, double phi) {
    const double a = K == 4 ? 10.2 : K == 2 ? 5.1 : 3.4;
    const double c = K == 4 ? 3.3e-5 : K == 2 ? 1.6e-5 : 5.4e-6;
    return a * std::pow(double(pad_np(n)) / 2048.0, 1.5) + c * phi * double(n) * double(n);
}

double tensor_step_us(int n, bool fp4, int groups_per_wave) {
    const int R = pad_np(n) / 256;
    if (anc::stream_supported(n)) return 99.5;
    if (R == 8) return fp4 ? (groups_per_wave > 1 ? 8.3 : 8.1) : 23.3;
    return R == 12 ? 21.7 : 28.3;
}

// us[ANC_ENGINE_*] for nchains anneals of S steps (-1: engine unavailable, per_wave[e] == 0); returns the engine with
// the least estimate (ties: plain, then tensor, then cluster).
int estimate_engines(int n, int K, int nchains, int S, double phi, bool fp4, const int* per_wave, double* us) {
    phi = std::min(1.0, std::max(0.0, phi));
    for (int e = 0; e < 4; ++e) us[e] = -1.0;
    auto waves = [&](int e) { return double((nchains + per_wave[e] - 1) / per_wave[e]); };
    if (per_wave[ANC_ENGINE_PLAIN] > 0)
        us[ANC_ENGINE_PLAIN] = waves(ANC_ENGINE_PLAIN) * S * plain_step_us(n, K, phi);
    if (per_wave[ANC_ENGINE_TENSOR] > 0) {
        const int groups = std::min(nchains, per_wave[ANC_ENGINE_TENSOR]);
        us[ANC_ENGINE_TENSOR] = waves(ANC_ENGINE_TENSOR) * S * tensor_step_us(n, fp4, (groups + 127) / 128);
    }
    if (per_wave[ANC_ENGINE_CLUSTER] > 0)
        us[ANC_ENGINE_CLUSTER] = nchains <= per_wave[ANC_ENGINE_CLUSTER] / 2 ? S * 0.86
                                                                             : waves(ANC_ENGINE_CLUSTER) * S * 1.18;
    int best = ANC_ENGINE_PLAIN;
    for (int e : {ANC_ENGINE_PLAIN, ANC_ENGINE_TENSOR, ANC_ENGINE_CLUSTER})
        if (us[e] >= 0 && (us[best] < 0 || us[e] < us[best])) best = e;
    return best;
}

std::atomic<uint64_t> g_next_uid{1};

}  // namespace

struct anc_instance {
    int n = 0, np = 0, nw = 0, nwj = 0, K = 0;   // K = 0: sparse
    anc_instance_info info{};
    std::vector<int32_t> bias;                    // host copy (empty = none)
    DevBuf<uint32_t> planes;
    DevBuf<int32_t> row_ptr;
    DevBuf<uint32_t> adj;
    // the CSR rows with 16-bit edges, two per word (every J_xy = +-1 and n < 32767; else empty): half the fetches
    DevBuf<int32_t> row_ptr16;
    DevBuf<uint32_t> adj16;
    bool csr16 = false;
    DevBuf<int32_t> d_bias;
    std::vector<int8_t> dense;                    // host copy of dense couplings (tensor engine packs lazily)
    anc::TensorInstance tensor;                   // tensor-engine operands (built on first use)
    bool tensor_ready = false;
    int per_wave[4] = {-1, -1, -1, -1};           // anneals per wave of each engine (ANC_ENGINE_*; -1: not queried)
    int cluster16_wave = -1;                      // anneals one wave of 16-CTA clusters runs (-1: not queried)
    uint64_t uid = g_next_uid.fetch_add(1);       // identifies the instance to the tables' flip record
    // per-handle workspace for single-job launches
    DevBuf<int> counter;
    DevBuf<uint32_t> w_spins;
    DevBuf<long long> w_sh, w_bs, w_fl;
    DevBuf<int32_t> w_trace, w_h;
    DevBuf<long long> w_prof;                     // tensor-engine phase counters (opt-in)
    DevBuf<int> w_err;                            // cluster engine's error word
    bool cluster_err_pending = false;             // a cluster launch's error word is still to be read
    int prof_ctas = 0, prof_S = 0;
    // CSR pass variant chosen by the tuner (-1: not tuned yet) and its probe's device time per step of each variant
    int sparse_variant = -1;
    double sparse_probe_us[anc::kSparseVariants] = {};
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int device = 0, sms = 0;
    ~anc_instance() {
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }
};

struct anc_tables {
    int S = 0;
    // flip fraction of the last host-output run of these tables (parts per million) and the instance it ran on
    std::atomic<uint64_t> seen_uid{0};
    std::atomic<uint32_t> seen_ppm{0};
    std::vector<int32_t> fourT, q, kconst;
    std::vector<int64_t> kcorr;
    DevBuf<int32_t> d_fourT, d_q, d_kconst;
    DevBuf<int64_t> d_kcorr;
};

namespace {

void compute_info(anc_instance* I, const int32_t* row_ptr, const int32_t* col, const int8_t* val) {
    anc_instance_info& f = I->info;
    f.n = I->n;
    f.np = I->np;
    f.kbits = I->K;
    f.sparse = I->K == 0;
    int64_t sumw = 0, hmax = 0, nnz = 0;
    int32_t maxabs = 0;
    double sq = 0;
    for (int x = 0; x < I->n; ++x) {
        int64_t row = 0;
        for (int k = row_ptr[x]; k < row_ptr[x + 1]; ++k) {
            const int v = val[k];
            if (col[k] > x) sumw -= v;
            row += std::abs(v);
            maxabs = std::max(maxabs, int32_t(std::abs(v)));
            sq += double(v) * v;
            ++nnz;
        }
        hmax = std::max(hmax, row);
    }
    f.nnz = nnz;
    f.sumw = sumw;
    f.maxabs = maxabs;
    f.hmax = hmax;
    f.mean_row_sq = I->n ? sq / I->n : 0.0;
    int32_t bm = 0;
    for (int32_t b : I->bias) bm = std::max(bm, int32_t(std::abs(b)));
    f.bmax = bm;
}

int finish_common(anc_instance* I, const int32_t* bias) {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    I->device = dev;
    CK(cudaDeviceGetAttribute(&I->sms, cudaDevAttrMultiProcessorCount, dev));
    if (bias) {
        I->bias.assign(bias, bias + I->n);
        for (int32_t b : I->bias)
            if (b < -32767 || b > 32767) return fail(ANC_EINVAL, "bias outside |b| <= 32767 (B_BITS = 16)");
        CK(I->d_bias.ensure(I->n));
        CK(cudaMemcpy(I->d_bias.p, bias, sizeof(int32_t) * I->n, cudaMemcpyHostToDevice));
    }
    CK(cudaStreamCreateWithFlags(&I->stream, cudaStreamNonBlocking));
    CK(cudaEventCreate(&I->ev0));
    CK(cudaEventCreate(&I->ev1));
    CK(I->counter.ensure(1));
    return ANC_OK;
}

anc::DevTables dev_tables(anc_tables* tb) {
    anc::DevTables d;
    d.fourT = tb->d_fourT.p;
    d.q = tb->d_q.p;
    d.kcorr = tb->d_kcorr.p;
    d.kconst = tb->d_kconst.p;
    d.S = tb->S;
    return d;
}

struct Plan {
    bool plain_ok = false;
    int32_t hclamp = 0;
};

// Range plan. It accepts and refuses exactly the tables the reference's host::plan_ranges does
// (gpu/multibit_bias_20261008/src/sca_gpu_bias.cu:543-557), stated here from the decision's arithmetic:
//   z = s*h * 2^16 + (q_t -/+ corr_t) is compared with r, |r| <= 4T_t / 2, in int32.
// The part of z that is not the field is bounded over the whole schedule by
//   off = max_t ( |q_t| + |corr_t| + 4T_t ),  |corr_t| <= (n |kcorr_t|) >> 8 + |kconst_t| + 1   (n_lin <= n).
// Unclamped, |s*h| <= hmax + bmax, so the kernels may use the field as is when (hmax + bmax) 2^16 + off < 2^31 - 1.
// Otherwise they clamp s*h to +-hc with hc = floor(off / 2^16) + 1: then |hc 2^16| > off, so a clamped field decides
// z's comparison exactly as the true one would (both lie beyond every threshold), provided hc 2^16 + off still fits.
int range_plan_raw(int n, int64_t hmax, int64_t bmax, const int32_t* fourT, const int32_t* q, const int64_t* kcorr,
                   const int32_t* kconst, int S, Plan* out) {
    constexpr int64_t kInt32Top = (int64_t(1) << 31) - 1;
    constexpr int64_t kQ16 = int64_t(1) << 16;
    int64_t off = 0;
    for (int t = 0; t < S; ++t) {
        if (fourT[t] <= 0) return fail(ANC_EINVAL, "fourT must be positive (step %d)", t);
        const int64_t gain = std::llabs(kcorr[t]);
        if (gain > (int64_t(1) << 40)) return fail(ANC_EINVAL, "kcorr out of range at step %d", t);
        const int64_t corr_bound = ((int64_t(n) * gain) >> 8) + std::llabs(int64_t(kconst[t])) + 1;
        off = std::max<int64_t>(off, std::llabs(int64_t(q[t])) + corr_bound + int64_t(fourT[t]));
    }
    out->plain_ok = (hmax + bmax) * kQ16 + off < kInt32Top;
    const int64_t clamp = off / kQ16 + 1;
    if (clamp * kQ16 + off >= kInt32Top)
        return fail(ANC_EINVAL, "table range exceeds int32 kernel arithmetic even with clamping");
    out->hclamp = int32_t(clamp);
    return ANC_OK;
}

int range_plan(const anc_instance* I, const anc_tables* tb, Plan* out) {
    return range_plan_raw(I->n, I->info.hmax, I->info.bmax, tb->fourT.data(), tb->q.data(), tb->kcorr.data(),
                          tb->kconst.data(), tb->S, out);
}

int resolve_clamp(const anc_instance* I, const anc_tables* tb, const anc_run_opts* o, int32_t* hclamp) {
    Plan pl;
    int rc = range_plan(I, tb, &pl);
    if (rc) return rc;
    const int wide = o ? o->wide : -1;
    if (wide == 0 && !pl.plain_ok)
        return fail(ANC_EINVAL, "instance needs the clamped decision (|J| row sum + |b| too large for int32 decisions)");
    *hclamp = (wide == 1 || !pl.plain_ok) ? pl.hclamp : 0;
    return ANC_OK;
}

int plain_P(int np_max) { return np_max <= 2048 ? 12 : 16; }

struct OutPtrs {
    uint32_t* spins;
    long long *sh, *bs, *fl;
    int32_t *trace, *h;
};

anc::PlainJob make_job(anc_instance* I, anc_tables* tb, uint64_t seed, uint32_t off, int nchains, int32_t hclamp,
                       const OutPtrs& o) {
    anc::PlainJob j{};
    j.n = I->n;
    j.np = I->np;
    j.nw = I->nw;
    j.nwj = I->nwj;
    j.K = I->K;
    j.planes = I->planes.p;
    j.row_ptr = I->csr16 ? I->row_ptr16.p : I->row_ptr.p;
    j.adj = I->csr16 ? I->adj16.p : I->adj.p;
    j.csr16 = I->csr16 ? 1 : 0;
    j.bias = I->bias.empty() ? nullptr : I->d_bias.p;
    j.tab = dev_tables(tb);
    j.seed = seed;
    j.trial_offset = off;
    j.ntrials = nchains;
    j.trace = o.trace != nullptr;
    j.hclamp = hclamp;
    j.out_spins = o.spins;
    j.out_sum_sh = reinterpret_cast<int64_t*>(o.sh);
    j.out_sum_bs = reinterpret_cast<int64_t*>(o.bs);
    j.out_flips = reinterpret_cast<int64_t*>(o.fl);
    j.out_trace = o.trace;
    j.out_h = o.h;
    return j;
}

// Shared memory plan and co-resident CTAs per SM of the one-CTA plain engine for this instance.
int plain_residency(const anc_instance* I, int P, size_t* smem, bool* stream, int* per_sm) {
    *smem = anc::plain_smem_plan(I->np, I->K == 0 ? I->nw : I->nwj, I->K, P, stream);
    if (*smem > 227 * 1024)
        return fail(ANC_EINVAL, "instance too large for the plain engine (%zu B shared memory)", *smem);
    const int rc = anc::plain_max_blocks_per_sm(I->K, P, *smem, per_sm, *stream);
    if (rc) return cuda_fail(cudaError_t(rc), "occupancy");
    if (*per_sm < 1) return fail(ANC_EINVAL, "plain engine cannot be resident (smem %zu)", *smem);
    return ANC_OK;
}

// Launch plan of one kernel kind of a batch (the plain engine's template over K): shared memory and residency.
constexpr int kKinds[4] = {0, 1, 2, 4};     // CSR, then dense K = 1 / 2 / 4
int kind_index(int K) { return K == 0 ? 0 : K == 1 ? 1 : K == 2 ? 2 : 3; }
struct KindPlan {
    int np_max = 0, nwj_max = 0, P = 0, per_sm = 0;
    size_t smem = 0;
    bool stream = false;
};
int plan_kind(int K, int np_max, int nwj_max, int sms, KindPlan* out) {
    (void)sms;
    KindPlan p;
    p.np_max = np_max;
    p.nwj_max = nwj_max;
    p.P = plain_P(np_max);
    p.smem = anc::plain_smem_plan(np_max, nwj_max, K, p.P, &p.stream);
    if (p.smem > 227 * 1024)
        return fail(ANC_EINVAL, "batch instance too large for the plain engine (n padded to %d needs %zu B of shared "
                                "memory)", np_max, p.smem);
    const int rc = anc::plain_max_blocks_per_sm(K, p.P, p.smem, &p.per_sm, p.stream);
    if (rc) return cuda_fail(cudaError_t(rc), "occupancy");
    if (p.per_sm < 1) return fail(ANC_EINVAL, "plain engine cannot be resident (%zu B shared memory)", p.smem);
    *out = p;
    return ANC_OK;
}

int tuned_variant(anc_instance* I, int kernel, int nchains);

// One launch of the one-CTA plain engine; variant >= 0 forces the CSR pass variant (sparse instances) or the dense
// pass variant (dense instances), else the tuned one.
int launch_plain_single(anc_instance* I, const anc::PlainJob& job, cudaStream_t st, int variant = -1) {
    anc::PlainLaunch L{};
    L.job0 = job;
    L.jobs = nullptr;
    L.items = nullptr;
    L.nitems = job.ntrials;
    L.next_item = I->counter.p;
    L.np_max = I->np;
    L.nwj_max = I->K == 0 ? I->nw : I->nwj;
    const int P = plain_P(I->np);
    bool stream = false;
    size_t smem = 0;
    int per_sm = 0;
    int rc = plain_residency(I, P, &smem, &stream, &per_sm);
    if (rc) return rc;
    if (I->K == 0) {
        L.sparse_variant = variant >= 0 ? variant : std::max(0, I->sparse_variant);
    } else {
        const int nv = anc::dense_variants(I->K, stream);
        if (variant >= nv)
            return fail(ANC_EINVAL, "kernel_variant %d out of range: the plain engine has %d dense variant(s) here",
                        variant + 1, nv);
        L.dense_variant = variant >= 0 ? variant : std::min(nv - 1, tuned_variant(I, ANC_KERNEL_PLAIN, job.ntrials));
    }
    L.stream = stream ? 1 : 0;
    const int grid = std::max(1, std::min(job.ntrials, per_sm * I->sms));
    CK(cudaMemsetAsync(I->counter.p, 0, sizeof(int), st));
    rc = anc::plain_launch(L, I->K, P, grid, smem, st);
    if (rc) return cuda_fail(cudaError_t(rc), "plain engine launch");
    return ANC_OK;
}

// Whether the tensor engine would run this instance on the fp4 kernel (tensor_fp4_eligible, from the host statistics).
bool fp4_candidate(const anc_instance* I) {
    return !I->dense.empty() && I->np == 2048 && I->info.maxabs <= 1 &&
           I->info.hmax + int64_t(I->info.bmax) < (int64_t(1) << 14);
}

// Anneals per wave of each engine on this device (0: the engine cannot run the instance); queried once per instance.
const int* engine_waves(anc_instance* I) {
    if (I->per_wave[0] < 0) {
        int w[4] = {0, 0, 0, 0};
        size_t smem = 0;
        bool stream = false;
        int per_sm = 0;
        if (plain_residency(I, plain_P(I->np), &smem, &stream, &per_sm) == ANC_OK) w[ANC_ENGINE_PLAIN] = per_sm * I->sms;
        int t = 0;
        if (!I->dense.empty() && anc::tensor_supported(I->n, I->K, 1) &&
            anc::tensor_wave_chains(I->n, fp4_candidate(I), &t) == 0)
            w[ANC_ENGINE_TENSOR] = std::max(0, t);
        int c = 0;
        if (anc::plain_cluster_supported(I->K, I->np) && anc::plain_cluster_max_active(&c) == 0)
            w[ANC_ENGINE_CLUSTER] = std::max(0, c);
        cudaGetLastError();   // a failed capacity query only rules that engine out
        g_err.clear();
        std::copy(w, w + 4, I->per_wave);
    }
    return I->per_wave;
}

// Anneals one wave of 16-CTA clusters runs on this device (0 if none fits); queried once per instance.
int cluster16_wave(anc_instance* I) {
    if (I->cluster16_wave < 0) {
        int c = 0;
        if (anc::plain_cluster_max_active(&c, 16) != cudaSuccess) c = 0;
        cudaGetLastError();
        I->cluster16_wave = std::max(0, c);
    }
    return I->cluster16_wave;
}

// Tuning key of a run of nchains anneals of this instance on `kernel` (ANC_KERNEL_PLAIN for dense instances,
// ANC_KERNEL_TENSOR_FP4): device, kernel, NP, K and, for the fp4 kernel, the replica groups one wave runs at once.
std::array<int, 5> tune_key(anc_instance* I, int kernel, int nchains) {
    int groups = 0;
    if (kernel == ANC_KERNEL_TENSOR_FP4) {
        const int slots = std::max(1, engine_waves(I)[ANC_ENGINE_TENSOR] / 128);
        groups = std::max(1, std::min((nchains + 127) / 128, slots));
    }
    return {I->device, kernel, I->np, I->K, groups};
}

// The tuned variant for this key, 0 before any tuning.
int tuned_variant(anc_instance* I, int kernel, int nchains) {
    const auto key = tune_key(I, kernel, nchains);
    std::lock_guard<std::mutex> lock(g_kernel_tune_mu);
    const auto it = g_kernel_tune.find(key);
    return it == g_kernel_tune.end() ? 0 : std::max(0, it->second.variant);
}

// Flip fraction AUTO assumes: the caller's hint, else what the last host-output run of these tables on this instance
// saw, else the prior.
double flip_fraction(const anc_instance* I, const anc_tables* tb, const anc_run_opts* o) {
    if (o && o->flip_permille > 0) return o->flip_permille / 1000.0;
    if (tb->seen_uid.load(std::memory_order_relaxed) == I->uid) return tb->seen_ppm.load(std::memory_order_relaxed) * 1e-6;
    return kPhiPrior;
}

int pick_engine(anc_instance* I, anc_tables* tb, int nchains, const anc_run_opts* o, double* us = nullptr,
                double* phi_used = nullptr) {
    const int e = o ? o->engine : ANC_ENGINE_AUTO;
    if (e == ANC_ENGINE_PLAIN || e == ANC_ENGINE_TENSOR || e == ANC_ENGINE_CLUSTER) return e;
    const double phi = flip_fraction(I, tb, o);
    double est[4];
    const int best = estimate_engines(I->n, I->K, nchains, tb->S, phi, fp4_candidate(I), engine_waves(I), est);
    if (us) std::copy(est, est + 4, us);
    if (phi_used) *phi_used = phi;
    return best;
}

int ensure_tensor(anc_instance* I) {
    if (I->tensor_ready) return ANC_OK;
    if (I->dense.empty()) return fail(ANC_EINVAL, "the tensor engine needs dense couplings");
    std::string why;
    const int rc = anc::tensor_build_instance(I->dense.data(), I->n, &I->tensor, &why);
    if (rc) return fail(rc == -2 ? ANC_ECUDA : ANC_EINVAL, "tensor engine setup: %s", why.c_str());
    I->tensor_ready = true;
    return ANC_OK;
}

// Launch on device outputs; no synchronisation. S_probe > 0 runs only the first S_probe steps of the schedule (the
// run-time tuners' probes).
int run_device_impl(anc_instance* I, anc_tables* tb, uint64_t seed, uint32_t off, int nchains, const anc_run_opts* o,
                    const OutPtrs& out, cudaStream_t st, int S_probe = 0) {
    if (!I || !tb) return fail(ANC_EINVAL, "null handle");
    if (nchains < 1) return fail(ANC_EINVAL, "nchains must be >= 1");
    if (!out.spins || !out.sh || !out.fl) return fail(ANC_EINVAL, "spins, sum_sh and flips outputs are required");
    int32_t hclamp = 0;
    int rc = resolve_clamp(I, tb, o, &hclamp);
    if (rc) return rc;
    const int engine = pick_engine(I, tb, nchains, o);
    if (engine == ANC_ENGINE_TENSOR) {
        if (!anc::tensor_supported(I->n, I->K, nchains))
            return fail(ANC_EINVAL, "tensor engine does not support n=%d K=%d", I->n, I->K);
        rc = ensure_tensor(I);
        if (rc) return rc;
        const int forced = o ? o->kernel_variant : 0;
        if (forced > anc::kF4Variants)
            return fail(ANC_EINVAL, "kernel_variant %d out of range: the fp4 kernel has %d variants", forced,
                        anc::kF4Variants);
        anc::TensorRun r{};
        r.tab = dev_tables(tb);
        if (S_probe > 0) r.tab.S = std::min(r.tab.S, S_probe);
        r.variant = forced > 0 ? forced - 1 : tuned_variant(I, ANC_KERNEL_TENSOR_FP4, nchains);
        r.seed = seed;
        r.trial_offset = off;
        r.nchains = nchains;
        r.hclamp = hclamp;
        r.bias = I->bias.empty() ? nullptr : I->d_bias.p;
        r.out_spins = out.spins;
        r.out_sum_sh = reinterpret_cast<int64_t*>(out.sh);
        r.out_sum_bs = reinterpret_cast<int64_t*>(out.bs);
        r.out_flips = reinterpret_cast<int64_t*>(out.fl);
        r.out_trace = out.trace;
        r.out_h = out.h;
        r.prof = nullptr;
        r.kind = o ? o->tensor_kind : ANC_TENSOR_AUTO;
        r.wait_ns = g_wait_ns.load();
        I->prof_ctas = 0;
        if (o && o->profile) {
            anc::TensorGeometry geo;
            if (anc::tensor_geometry(I->n, nchains, &geo) != 0) return fail(ANC_ECUDA, "tensor geometry query failed");
            const int ctas = std::max(geo.ctas, 16 * ((nchains + 127) / 128));
            CK(I->w_prof.ensure(size_t(ctas) * anc::kTensorProfSlots));
            CK(cudaMemsetAsync(I->w_prof.p, 0, size_t(ctas) * anc::kTensorProfSlots * sizeof(long long), st));
            r.prof = I->w_prof.p;
            I->prof_ctas = ctas;
            I->prof_S = tb->S;
        }
        std::string why;
        rc = anc::tensor_run(&I->tensor, r, st, &why);
        if (rc == -3) return fail(ANC_ETIMEOUT, "tensor engine: %s", why.c_str());
        if (rc) return fail(rc == -2 ? ANC_ECUDA : ANC_EINVAL, "tensor engine: %s", why.c_str());
        g_last_kernel = I->tensor.last_kind == anc::TENSOR_KIND_FP4 ? ANC_KERNEL_TENSOR_FP4 : ANC_KERNEL_TENSOR_INT8;
        return ANC_OK;
    }
    anc::PlainJob job = make_job(I, tb, seed, off, nchains, hclamp, out);
    if (S_probe > 0) job.tab.S = std::min(job.tab.S, S_probe);
    if (engine == ANC_ENGINE_CLUSTER) {
        if (!anc::plain_cluster_supported(I->K, I->np))
            return fail(ANC_EINVAL, "the cluster engine needs dense 1-bit couplings with n <= 2048 (n=%d K=%d)", I->n,
                        I->K);
        const int forced = o ? o->kernel_variant : 0;
        if (forced > 2)
            return fail(ANC_EINVAL, "kernel_variant %d out of range: the cluster engine has 2 variants", forced);
        int ctas = forced == 2 ? 16 : 8;
        if (forced == 0) ctas = nchains <= cluster16_wave(I) ? 16 : 8;
        CK(I->w_err.ensure(1));
        CK(cudaMemsetAsync(I->w_err.p, 0, sizeof(int), st));
        job.err = I->w_err.p;
        // the limit, but never below 10 ms: an exchange that gave up can leave pushes in flight toward a CTA, so a
        // forced expiry (a limit of 0) is kept off this engine (a step takes about 2 us)
        job.wait_ns = std::max<uint64_t>(10000000ull, g_wait_ns.load());
        I->cluster_err_pending = true;
        rc = anc::plain_cluster_launch(job, st, ctas);
        if (rc) return cuda_fail(cudaError_t(rc), "cluster engine launch");
        g_last_kernel = ANC_KERNEL_PLAIN_CLUSTER;
        return ANC_OK;
    }
    if (I->K == 0 && o && o->kernel_variant > 0) {
        // CSR edge format: 1 = 32-bit edges, 2 = 16-bit edges (unit weights and n < 32767 only)
        if (o->kernel_variant > 2 || (o->kernel_variant == 2 && !I->csr16))
            return fail(ANC_EINVAL, "kernel_variant %d: CSR instances take 1 (32-bit edges) or, with unit weights "
                                    "and n < 32767, 2 (16-bit edges)", o->kernel_variant);
        if (o->kernel_variant == 1) {
            job.row_ptr = I->row_ptr.p;
            job.adj = I->adj.p;
            job.csr16 = 0;
        }
    }
    const int forced = o ? (I->K == 0 ? o->sparse_variant : o->kernel_variant) : 0;
    rc = launch_plain_single(I, job, st, forced > 0 ? forced - 1 : -1);
    if (rc == ANC_OK) g_last_kernel = ANC_KERNEL_PLAIN;
    return rc;
}

// Run-time tuner of the CSR pass (the plain engine on sparse instances): on the first synchronous run of an
// instance, each compiled variant (kSparseVariantShape: rows in flight per lane group x edges per lane) runs the
// first min(S, 64) steps of min(nchains, one wave) anneals of that run -- twice, the second launch timed with CUDA
// events -- and the fastest is kept for every later launch of the instance (device, batch and graph-captured
// launches included). Every variant computes the same fields; only the time differs. The probes write into the
// handle's own workspaces, never into the caller's outputs.
int tune_sparse(anc_instance* I, anc_tables* tb, uint64_t seed, uint32_t off, int nchains, const anc_run_opts* o) {
    if (I->K != 0 || I->sparse_variant >= 0) return ANC_OK;
    int32_t hclamp = 0;
    int rc = resolve_clamp(I, tb, o, &hclamp);
    if (rc) return rc;
    const int P = plain_P(I->np);
    bool stream = false;
    size_t smem = 0;
    int per_sm = 0;
    rc = plain_residency(I, P, &smem, &stream, &per_sm);
    if (rc) return rc;
    const int np = std::max(1, std::min(nchains, per_sm * I->sms));
    const int Sp = std::min(tb->S, 64);
    CK(I->w_spins.ensure(size_t(I->nw) * np));
    CK(I->w_sh.ensure(np));
    CK(I->w_bs.ensure(np));
    CK(I->w_fl.ensure(np));
    OutPtrs out{I->w_spins.p, I->w_sh.p, I->w_bs.p, I->w_fl.p, nullptr, nullptr};
    anc::PlainJob job = make_job(I, tb, seed, off, np, hclamp, out);
    job.tab.S = Sp;
    cudaStream_t st = I->stream;
    int best = 0;
    for (int v = 0; v < anc::kSparseVariants; ++v) {
        float ms = 0.f;
        for (int rep = 0; rep < 2; ++rep) {
            CK(cudaEventRecord(I->ev0, st));
            rc = launch_plain_single(I, job, st, v);
            if (rc) return rc;
            CK(cudaEventRecord(I->ev1, st));
            CK(cudaEventSynchronize(I->ev1));
            CK(cudaEventElapsedTime(&ms, I->ev0, I->ev1));
        }
        I->sparse_probe_us[v] = 1000.0 * double(ms) / Sp;
        if (I->sparse_probe_us[v] < I->sparse_probe_us[best]) best = v;
    }
    I->sparse_variant = best;
    return ANC_OK;
}

// Run-time tuner of the dense kernels' compiled variants (anc_kernel_tuning): when a run would use the plain engine
// on a dense instance or the fp4 kernel, and that run's tuning key (tune_key) has not been tuned in this process, each
// variant runs the first min(S, 256) steps of the run's anneals (one wave of the plain engine; every replica group of
// one fp4 wave) three times; its probe time is the least of the last two launches (CUDA events). Variant 0, the one
// measured fastest on a B200 when the variants were compiled, is kept unless another probes more than 1 % faster:
// the variants differ by a few percent, and a 64-step probe of one launch picked the wrong one in a third of the
// recorded fp4 cases. The probes write into the handle's workspaces `out`, never into the caller's outputs; every
// variant computes the same bits.
int tune_kernel(anc_instance* I, anc_tables* tb, uint64_t seed, uint32_t off, int nchains, const anc_run_opts* o,
                const OutPtrs& out) {
    if (o && o->kernel_variant > 0) return ANC_OK;
    const int engine = pick_engine(I, tb, nchains, o);
    int kernel = 0, nv = 1, nprobe = nchains;
    if (engine == ANC_ENGINE_PLAIN && I->K != 0) {
        size_t smem = 0;
        bool stream = false;
        int per_sm = 0;
        const int rc = plain_residency(I, plain_P(I->np), &smem, &stream, &per_sm);
        if (rc) return rc;
        kernel = ANC_KERNEL_PLAIN;
        nv = anc::dense_variants(I->K, stream);
        nprobe = std::min(nchains, per_sm * I->sms);
    } else if (engine == ANC_ENGINE_TENSOR && fp4_candidate(I) && anc::tensor_supported(I->n, I->K, nchains) &&
               !(o && o->tensor_kind == ANC_TENSOR_INT8)) {
        kernel = ANC_KERNEL_TENSOR_FP4;
        nv = anc::kF4Variants;
        nprobe = std::min(nchains, std::max(128, engine_waves(I)[ANC_ENGINE_TENSOR]));
    }
    if (nv < 2) return ANC_OK;
    const auto key = tune_key(I, kernel, nchains);
    {
        std::lock_guard<std::mutex> lock(g_kernel_tune_mu);
        if (g_kernel_tune.count(key)) return ANC_OK;
    }
    anc_run_opts po{};
    if (o) po = *o;
    else po.wide = -1;     // the defaults of a call without options: clamp only where the range plan needs it
    po.engine = engine;
    po.profile = 0;
    if (kernel == ANC_KERNEL_TENSOR_FP4) po.tensor_kind = ANC_TENSOR_FP4;
    const int Sp = std::min(tb->S, 256);
    OutPtrs pout = out;
    pout.trace = nullptr;
    pout.h = nullptr;
    cudaStream_t st = I->stream;
    KernelTune rec;
    rec.nvariants = nv;
    for (int v = 0; v < nv; ++v) {
        po.kernel_variant = v + 1;
        float ms = 0.f, best_ms = 0.f;
        for (int rep = 0; rep < 3; ++rep) {
            CK(cudaEventRecord(I->ev0, st));
            int rc = run_device_impl(I, tb, seed, off, nprobe, &po, pout, st, Sp);
            if (rc) return rc;
            CK(cudaEventRecord(I->ev1, st));
            CK(cudaEventSynchronize(I->ev1));
            CK(cudaEventElapsedTime(&ms, I->ev0, I->ev1));
            if (I->tensor_ready && I->tensor.last_err) {
                std::string why;
                rc = anc::tensor_check_error(&I->tensor, st, &why);
                I->tensor.last_err = nullptr;
                if (rc == -3) return fail(ANC_ETIMEOUT, "tensor engine (tuning probe): %s", why.c_str());
                if (rc) return fail(ANC_ECUDA, "tensor engine (tuning probe): %s", why.c_str());
            }
            if (rep == 1 || (rep > 1 && ms < best_ms)) best_ms = ms;
        }
        rec.probe_us[v] = 1000.0 * double(best_ms) / Sp;
    }
    rec.variant = 0;
    for (int v = 1; v < nv; ++v)
        if (rec.probe_us[v] < 0.99 * rec.probe_us[0] && rec.probe_us[v] < rec.probe_us[rec.variant]) rec.variant = v;
    std::lock_guard<std::mutex> lock(g_kernel_tune_mu);
    g_kernel_tune.emplace(key, rec);
    return ANC_OK;
}

int run_host_impl(anc_instance* I, anc_tables* tb, uint64_t seed, uint32_t off, int nchains, const anc_run_opts* o,
                  uint64_t* spins, int64_t* sum_sh, int64_t* sum_bs, int64_t* flips, int32_t* trace,
                  int32_t* fields) {
    if (!I || !tb) return fail(ANC_EINVAL, "null handle");
    if (nchains < 1) return fail(ANC_EINVAL, "nchains must be >= 1");
    if (!spins || !sum_sh) return fail(ANC_EINVAL, "spins and sum_sh outputs are required");
    const size_t nw = size_t(I->nw);
    CK(I->w_spins.ensure(nw * nchains));
    CK(I->w_sh.ensure(nchains));
    CK(I->w_bs.ensure(nchains));
    CK(I->w_fl.ensure(nchains));
    if (trace) CK(I->w_trace.ensure(size_t(nchains) * tb->S));
    if (fields) CK(I->w_h.ensure(size_t(nchains) * I->n));
    OutPtrs out{I->w_spins.p, I->w_sh.p, I->w_bs.p, I->w_fl.p, trace ? I->w_trace.p : nullptr,
                fields ? I->w_h.p : nullptr};
    cudaStream_t st = I->stream;
    if (I->K == 0 && !(o && o->sparse_variant > 0)) {
        const int trc = tune_sparse(I, tb, seed, off, nchains, o);
        if (trc) return trc;
    }
    if (I->K != 0) {
        const int trc = tune_kernel(I, tb, seed, off, nchains, o, out);
        if (trc) return trc;
    }
    CK(cudaEventRecord(I->ev0, st));
    int rc = run_device_impl(I, tb, seed, off, nchains, o, out, st);
    if (rc) return rc;
    CK(cudaEventRecord(I->ev1, st));
    CK(cudaMemcpyAsync(spins, I->w_spins.p, nw * nchains * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(sum_sh, I->w_sh.p, size_t(nchains) * 8, cudaMemcpyDeviceToHost, st));
    if (sum_bs) CK(cudaMemcpyAsync(sum_bs, I->w_bs.p, size_t(nchains) * 8, cudaMemcpyDeviceToHost, st));
    if (flips) CK(cudaMemcpyAsync(flips, I->w_fl.p, size_t(nchains) * 8, cudaMemcpyDeviceToHost, st));
    if (trace) CK(cudaMemcpyAsync(trace, I->w_trace.p, size_t(nchains) * tb->S * 4, cudaMemcpyDeviceToHost, st));
    if (fields) CK(cudaMemcpyAsync(fields, I->w_h.p, size_t(nchains) * I->n * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (I->cluster_err_pending) {
        int e = 0;
        CK(cudaMemcpy(&e, I->w_err.p, sizeof(int), cudaMemcpyDeviceToHost));
        I->cluster_err_pending = false;
        if (e) return fail(ANC_ETIMEOUT, "cluster engine: a step's exchange did not arrive within the wait limit (%llu ns)",
                           static_cast<unsigned long long>(g_wait_ns.load()));
    }
    if (I->tensor_ready && I->tensor.last_err) {
        std::string why;
        rc = anc::tensor_check_error(&I->tensor, st, &why);
        I->tensor.last_err = nullptr;
        if (rc == -3) return fail(ANC_ETIMEOUT, "tensor engine: %s", why.c_str());
        if (rc) return fail(ANC_ECUDA, "tensor engine: %s", why.c_str());
    }
    // the flip fraction this run saw, for AUTO's next choice on these tables and this instance
    if (flips && I->n > 0) {
        double total = 0;
        for (int c = 0; c < nchains; ++c) total += double(flips[c]);
        const double phi = total / (double(nchains) * I->n * tb->S);
        tb->seen_ppm.store(uint32_t(std::min(1.0, std::max(0.0, phi)) * 1e6 + 0.5), std::memory_order_relaxed);
        tb->seen_uid.store(I->uid, std::memory_order_relaxed);
    }
    if (I->prof_ctas > 0) {
        const size_t ns = anc::kTensorProfSlots;
        std::vector<long long> h(size_t(I->prof_ctas) * ns);
        CK(cudaMemcpy(h.data(), I->w_prof.p, h.size() * sizeof(long long), cudaMemcpyDeviceToHost));
        g_prof.assign(22 + (ns - 19), 0.0);
        int slot_of[anc::kTensorProfSlots] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21};
        for (size_t s = 19; s < ns; ++s) slot_of[s] = int(22 + s - 19);                  // slot -> output
        for (size_t s = 0; s < ns; ++s) {
            double acc = 0;
            for (int b = 0; b < I->prof_ctas; ++b) acc += double(h[size_t(b) * ns + s]);
            g_prof[slot_of[s]] = acc / I->prof_ctas / std::max(1, I->prof_S);
        }
        anc::TensorGeometry geo;
        anc::tensor_geometry(I->n, nchains, &geo);
        g_prof[9] = I->tensor.last_ctas;
        g_prof[10] = I->tensor.last_cluster;
        g_prof[11] = geo.max_active_clusters;
        I->prof_ctas = 0;
    }
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, I->ev0, I->ev1));
    g_dev_ms = ms;
    return ANC_OK;
}

}  // namespace

extern "C" {

const char* anc_last_error(void) { return g_err.c_str(); }

// ---- mean-field relaxation ----
struct anc_meanfield {
    anc::MfContext* ctx = nullptr;
};

int anc_mf_create(const int8_t* J, int n, const int32_t* bias, anc_meanfield** out) {
    if (!J || n < 1 || !out) return fail(ANC_EINVAL, "anc_mf_create: J, n >= 1 and out are required");
    std::string why;
    anc::MfContext* c = nullptr;
    const int rc = anc::mf_create(J, bias, n, &c, &why);
    if (rc) return fail(rc == -2 ? ANC_ECUDA : ANC_EINVAL, "mean-field setup: %s", why.c_str());
    *out = new anc_meanfield{c};
    return ANC_OK;
}

int anc_mf_npad(const anc_meanfield* mf) { return mf && mf->ctx ? anc::mf_npad(mf->ctx) : 0; }

int anc_mf_forward(anc_meanfield* mf, int S, const float* sched, const float* m0, const float* mprev, float* ckpt,
                   float* m_out, void* stream) {
    if (!mf || !mf->ctx || S < 1 || !sched) return fail(ANC_EINVAL, "anc_mf_forward: invalid arguments");
    std::string why;
    const int rc = anc::mf_forward(mf->ctx, S, sched, sched + S, sched + 2 * size_t(S), sched + 3 * size_t(S), m0,
                                   mprev, ckpt, m_out, static_cast<cudaStream_t>(stream), &why);
    if (rc) return fail(rc == -2 ? ANC_ECUDA : ANC_EINVAL, "mean-field forward: %s", why.c_str());
    return ANC_OK;
}

int anc_mf_backward(anc_meanfield* mf, int S, const float* sched, const float* ckpt, const float* g_m, float* gsched,
                    void* stream) {
    if (!mf || !mf->ctx || S < 1 || !sched) return fail(ANC_EINVAL, "anc_mf_backward: invalid arguments");
    std::string why;
    const int rc = anc::mf_backward(mf->ctx, S, sched, sched + S, sched + 2 * size_t(S), sched + 3 * size_t(S), ckpt,
                                    g_m, gsched, static_cast<cudaStream_t>(stream), &why);
    if (rc) return fail(rc == -2 ? ANC_ECUDA : ANC_EINVAL, "mean-field adjoint: %s", why.c_str());
    return ANC_OK;
}

int anc_mf_check(anc_meanfield* mf, void* stream) {
    if (!mf || !mf->ctx) return fail(ANC_EINVAL, "anc_mf_check: null handle");
    std::string why;
    const int rc = anc::mf_check_error(mf->ctx, static_cast<cudaStream_t>(stream), &why);
    if (rc == -3) return fail(ANC_ETIMEOUT, "%s", why.c_str());
    if (rc) return fail(ANC_ECUDA, "%s", why.c_str());
    return ANC_OK;
}

int anc_mf_set_wait_ns(anc_meanfield* mf, uint64_t ns) {
    if (!mf || !mf->ctx) return fail(ANC_EINVAL, "anc_mf_set_wait_ns: null handle");
    anc::mf_set_wait_ns(mf->ctx, ns);
    return ANC_OK;
}

void anc_mf_destroy(anc_meanfield* mf) {
    if (!mf) return;
    anc::mf_destroy(mf->ctx);
    delete mf;
}

int anc_last_profile(double* out, int max) {
    const int k = std::min<int>(max, int(g_prof.size()));
    for (int i = 0; i < k; ++i) out[i] = g_prof[i];
    return k;
}
const char* anc_version(void) { return "anechoic-b200 0.1 (sm_100a)"; }
double anc_last_device_ms(void) { return g_dev_ms; }
int anc_sparse_tuning(const anc_instance* I, int* variant, double* probe_us) {
    if (!I) return fail(ANC_EINVAL, "null handle");
    if (variant) *variant = I->K == 0 ? I->sparse_variant : -1;
    if (probe_us)
        for (int v = 0; v < anc::kSparseVariants; ++v) probe_us[v] = I->sparse_probe_us[v];
    return ANC_OK;
}
int anc_kernel_tuning(const anc_instance* Ic, int kernel, int nchains, int* variant, int* nvariants,
                      double* probe_us) {
    if (!Ic) return fail(ANC_EINVAL, "null handle");
    anc_instance* I = const_cast<anc_instance*>(Ic);    // the key may query (and cache) the engines' wave sizes
    int nv = 1;
    if (kernel == ANC_KERNEL_PLAIN) {
        if (I->K == 0) return fail(ANC_EINVAL, "CSR instances are tuned by the CSR-pass tuner (anc_sparse_tuning)");
        size_t smem = 0;
        bool stream = false;
        int per_sm = 0;
        const int rc = plain_residency(I, plain_P(I->np), &smem, &stream, &per_sm);
        if (rc) return rc;
        nv = anc::dense_variants(I->K, stream);
    } else if (kernel == ANC_KERNEL_TENSOR_FP4) {
        nv = anc::kF4Variants;
    } else {
        return fail(ANC_EINVAL, "kernel %d has no compiled variants to tune", kernel);
    }
    if (nchains < 1) return fail(ANC_EINVAL, "nchains must be >= 1");
    const auto key = tune_key(I, kernel, nchains);
    KernelTune rec;
    {
        std::lock_guard<std::mutex> lock(g_kernel_tune_mu);
        const auto it = g_kernel_tune.find(key);
        if (it != g_kernel_tune.end()) rec = it->second;
    }
    if (variant) *variant = rec.variant;
    if (nvariants) *nvariants = nv;
    if (probe_us)
        for (int v = 0; v < 4; ++v) probe_us[v] = rec.probe_us[v];
    return ANC_OK;
}
int anc_set_wait_ns(uint64_t ns) {
    g_wait_ns.store(ns);
    return ANC_OK;
}
uint64_t anc_get_wait_ns(void) { return g_wait_ns.load(); }
int anc_last_kernel(void) { return g_last_kernel; }
int anc_np(int n) { return pad_np(n); }
int anc_spin_words(int n) { return pad_np(n) / 64; }

int anc_instance_create(const int8_t* J, int n, int kbits, const int32_t* bias, anc_instance** out) {
    if (!out) return fail(ANC_EINVAL, "out is null");
    *out = nullptr;
    if (!J || n < 1 || n > 65536) return fail(ANC_EINVAL, "need J and 1 <= n <= 65536");
    std::unique_ptr<anc_instance> I(new anc_instance());
    I->n = n;
    I->np = pad_np(n);
    I->nw = I->np / 32;
    I->nwj = ((I->nw + 31) / 32) * 32;
    // validate and derive statistics (via CSR of the nonzeros)
    std::vector<int32_t> rp(size_t(n) + 1, 0), col;
    std::vector<int8_t> val;
    bool pm1 = true;
    int maxabs = 0;
    for (int x = 0; x < n; ++x) {
        const int8_t* row = J + size_t(x) * n;
        if (row[x] != 0) return fail(ANC_EINVAL, "nonzero diagonal coupling at %d", x);
        for (int y = 0; y < n; ++y) {
            const int v = row[y];
            if (v != J[size_t(y) * n + x]) return fail(ANC_EINVAL, "J not symmetric at (%d, %d)", x, y);
            if (y != x && v != 1 && v != -1) pm1 = false;
            if (v) { col.push_back(y); val.push_back(int8_t(v)); maxabs = std::max(maxabs, std::abs(v)); }
        }
        rp[x + 1] = int32_t(col.size());
    }
    int K = kbits;
    if (K == 0) K = pm1 ? 1 : (maxabs <= 1 ? 2 : (maxabs <= 7 ? 4 : 8));
    if (K == 1 && !pm1) return fail(ANC_EINVAL, "kbits = 1 needs a +-1 complete graph");
    if (K != 1 && K != 2 && K != 4) return fail(ANC_EINVAL, "kbits must be 1, 2 or 4 (|J| <= 7)");
    if (maxabs > (1 << (K - 1)) - 1 && K != 1) return fail(ANC_EINVAL, "|J| = %d exceeds 2^(K-1)-1 for K=%d", maxabs, K);
    I->K = K;
    if (bias) I->bias.assign(bias, bias + n);
    compute_info(I.get(), rp.data(), col.data(), val.data());
    // bit planes: [Kp][np][nwj]; K = 1: bit = [J = +1]; K >= 2: plane 0 = [J < 0], plane b = bit b-1 of |J|
    const int Kp = K;
    const size_t plane_words = size_t(I->np) * I->nwj;
    std::vector<uint32_t> P(plane_words * Kp, 0u);
    for (int x = 0; x < n; ++x) {
        const int8_t* row = J + size_t(x) * n;
        for (int y = 0; y < n; ++y) {
            const int v = row[y];
            if (!v) continue;
            const size_t wd = size_t(x) * I->nwj + (y >> 5);
            const uint32_t bit = 1u << (y & 31);
            if (K == 1) {
                if (v > 0) P[wd] |= bit;
            } else {
                if (v < 0) P[wd] |= bit;
                const int a = std::abs(v);
                for (int b = 1; b < K; ++b)
                    if ((a >> (b - 1)) & 1) P[size_t(b) * plane_words + wd] |= bit;
            }
        }
    }
    I->dense.assign(J, J + size_t(n) * n);
    int rc = finish_common(I.get(), bias);
    if (rc) return rc;
    cudaError_t e = I->planes.ensure(P.size());
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(planes)");
    e = cudaMemcpy(I->planes.p, P.data(), P.size() * 4, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy(planes)");
    *out = I.release();
    return ANC_OK;
}

int anc_instance_create_csr(int n, const int32_t* row_ptr, const int32_t* col, const int8_t* val, const int32_t* bias,
                            anc_instance** out) {
    if (!out) return fail(ANC_EINVAL, "out is null");
    *out = nullptr;
    if (!row_ptr || n < 1 || n > (1 << 24)) return fail(ANC_EINVAL, "need row_ptr and 1 <= n < 2^24");
    if (row_ptr[0] != 0) return fail(ANC_EINVAL, "row_ptr[0] must be 0");
    for (int x = 0; x < n; ++x)
        if (row_ptr[x + 1] < row_ptr[x]) return fail(ANC_EINVAL, "row_ptr not monotone at %d", x);
    const int64_t nnz = row_ptr[n];
    if (nnz > 0 && (!col || !val)) return fail(ANC_EINVAL, "col and val required");
    std::vector<std::pair<int64_t, int8_t>> keys, keysT;
    keys.reserve(nnz);
    keysT.reserve(nnz);
    std::vector<uint32_t> adj(nnz);
    for (int x = 0; x < n; ++x)
        for (int k = row_ptr[x]; k < row_ptr[x + 1]; ++k) {
            const int y = col[k];
            if (y < 0 || y >= n) return fail(ANC_EINVAL, "column index out of range in row %d", x);
            if (y == x) return fail(ANC_EINVAL, "nonzero diagonal coupling at %d", x);
            if (val[k] == 0) return fail(ANC_EINVAL, "explicit zero coupling in row %d", x);
            if (val[k] == -128) return fail(ANC_EINVAL, "coupling -128 not supported");
            keys.push_back({int64_t(x) * n + y, val[k]});
            keysT.push_back({int64_t(y) * n + x, val[k]});
            adj[k] = (uint32_t(y) << 8) | uint8_t(val[k]);
        }
    std::sort(keys.begin(), keys.end());
    std::sort(keysT.begin(), keysT.end());
    if (keys != keysT) return fail(ANC_EINVAL, "J not symmetric (or duplicate entries)");
    for (size_t i = 1; i < keys.size(); ++i)
        if (keys[i].first == keys[i - 1].first) return fail(ANC_EINVAL, "duplicate coupling");
    std::unique_ptr<anc_instance> I(new anc_instance());
    I->n = n;
    I->np = pad_np(n);
    I->nw = I->np / 32;
    I->nwj = ((I->nw + 31) / 32) * 32;
    I->K = 0;
    if (bias) I->bias.assign(bias, bias + n);
    compute_info(I.get(), row_ptr, col, val);
    int rc = finish_common(I.get(), bias);
    if (rc) return rc;
    cudaError_t e = I->row_ptr.ensure(size_t(n) + 1);
    if (e == cudaSuccess) e = cudaMemcpy(I->row_ptr.p, row_ptr, (size_t(n) + 1) * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = I->adj.ensure(std::max<int64_t>(nnz, 1));
    if (e == cudaSuccess && nnz) e = cudaMemcpy(I->adj.p, adj.data(), size_t(nnz) * 4, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "upload CSR");
    // unit weights and n < 32767: the same rows with 16-bit edges y | [J = -1] << 15, two per word, each row padded
    // to a whole word with the skip edge 0x7fff; the CSR pass then fetches half the words
    bool unit = n < 0x7fff;
    for (int64_t k = 0; unit && k < nnz; ++k) unit = val[k] == 1 || val[k] == -1;
    if (unit) {
        std::vector<int32_t> rp16(size_t(n) + 1, 0);
        for (int x = 0; x < n; ++x) rp16[x + 1] = rp16[x] + (row_ptr[x + 1] - row_ptr[x] + 1) / 2;
        std::vector<uint32_t> a16(std::max<int32_t>(rp16[n], 1), 0x7fff7fffu);
        for (int x = 0; x < n; ++x)
            for (int k = row_ptr[x]; k < row_ptr[x + 1]; ++k) {
                const int i = k - row_ptr[x];
                const uint32_t ed = uint32_t(col[k]) | (val[k] < 0 ? 0x8000u : 0u);
                uint32_t& wd = a16[size_t(rp16[x]) + i / 2];
                wd = (i & 1) ? ((wd & 0xffffu) | (ed << 16)) : ((wd & 0xffff0000u) | ed);
            }
        e = I->row_ptr16.ensure(size_t(n) + 1);
        if (e == cudaSuccess) e = cudaMemcpy(I->row_ptr16.p, rp16.data(), (size_t(n) + 1) * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = I->adj16.ensure(a16.size());
        if (e == cudaSuccess) e = cudaMemcpy(I->adj16.p, a16.data(), a16.size() * 4, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return cuda_fail(e, "upload 16-bit CSR");
        I->csr16 = true;
    }
    *out = I.release();
    return ANC_OK;
}

int anc_instance_get_info(const anc_instance* I, anc_instance_info* info) {
    if (!I || !info) return fail(ANC_EINVAL, "null argument");
    *info = I->info;
    return ANC_OK;
}

void anc_instance_destroy(anc_instance* I) {
    if (I) anc::tensor_free_instance(&I->tensor);
    delete I;
}

int anc_tables_create(const int32_t* fourT, const int32_t* q, const int64_t* kcorr, const int32_t* kconst, int S,
                      anc_tables** out) {
    if (!out) return fail(ANC_EINVAL, "out is null");
    *out = nullptr;
    if (S < 1 || S > (1 << 20) || !fourT || !q || !kcorr || !kconst) return fail(ANC_EINVAL, "need 1 <= S and all arrays");
    for (int t = 0; t < S; ++t)
        if (fourT[t] <= 0) return fail(ANC_EINVAL, "fourT must be positive (step %d)", t);
    std::unique_ptr<anc_tables> tb(new anc_tables());
    tb->S = S;
    tb->fourT.assign(fourT, fourT + S);
    tb->q.assign(q, q + S);
    tb->kcorr.assign(kcorr, kcorr + S);
    tb->kconst.assign(kconst, kconst + S);
    cudaError_t e = tb->d_fourT.ensure(S);
    if (e == cudaSuccess) e = tb->d_q.ensure(S);
    if (e == cudaSuccess) e = tb->d_kconst.ensure(S);
    if (e == cudaSuccess) e = tb->d_kcorr.ensure(S);
    if (e == cudaSuccess) e = cudaMemcpy(tb->d_fourT.p, fourT, size_t(S) * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(tb->d_q.p, q, size_t(S) * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(tb->d_kconst.p, kconst, size_t(S) * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(tb->d_kcorr.p, kcorr, size_t(S) * 8, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "upload tables");
    *out = tb.release();
    return ANC_OK;
}

// v80host::geom / build_tables (tables.hpp:14-40) and mb::tables (mb_common.hpp:132-154): the same double-precision
// formula and rounding (std::pow, std::llround), so the tables are bit-identical to the reference's.
int anc_tables_from_schedule(int S, double t0, double t1, double q, double lam, double jv, double kappa, int ramp,
                             double scale, anc_tables** out) {
    if (S < 1) return fail(ANC_EINVAL, "steps must be >= 1");
    std::vector<int32_t> f(S), qq(S), kc(S);
    std::vector<int64_t> kr(S);
    const int rc = anc_schedule_tables(S, t0, t1, q, lam, jv, kappa, ramp, scale, f.data(), qq.data(), kr.data(),
                                       kc.data());
    if (rc) return rc;
    return anc_tables_create(f.data(), qq.data(), kr.data(), kc.data(), S, out);
}

int anc_plan_ranges(int n, int64_t hmax, int64_t bmax, const int32_t* fourT, const int32_t* q, const int64_t* kcorr,
                    const int32_t* kconst, int S, int* plain_ok, int32_t* hclamp) {
    if (n < 1 || S < 1 || !fourT || !q || !kcorr || !kconst) return fail(ANC_EINVAL, "bad arguments");
    Plan pl;
    const int rc = range_plan_raw(n, hmax, bmax, fourT, q, kcorr, kconst, S, &pl);
    if (rc) return rc;
    if (plain_ok) *plain_ok = pl.plain_ok;
    if (hclamp) *hclamp = pl.hclamp;
    return ANC_OK;
}

int anc_schedule_tables(int S, double t0, double t1, double q, double lam, double jv, double kappa, int ramp,
                        double scale, int32_t* fourT, int32_t* q_out, int64_t* kcorr, int32_t* kconst) {
    if (S < 1 || !fourT || !q_out || !kcorr || !kconst) return fail(ANC_EINVAL, "bad arguments");
    if (!(t0 > 0) || !(t1 > 0)) return fail(ANC_EINVAL, "temperatures must be positive");
    std::vector<double> T(S), L(S, lam);
    for (int t = 0; t < S; ++t) T[t] = t0 * std::pow(t1 / t0, double(t) / std::max(1, S - 1));
    if (ramp)
        for (int t = 0; t < S; ++t)
            if (t >= 0.7 * S) L[t] = lam * (S - 1 - t) / std::max(1.0, S - 1 - 0.7 * S);
    if (scale != 1.0)
        for (double& l : L) l *= scale;
    for (int t = 0; t < S; ++t) {
        const double f = 4.0 * T[t] * 65536.0;
        if (!(f >= 1.0 && f < 2147483647.0)) return fail(ANC_EINVAL, "4T out of the Q16.16 range at step %d", t);
        fourT[t] = int32_t(std::llround(f));
        q_out[t] = int32_t(std::llround(q * 65536.0));
        kcorr[t] = t == 0 ? 0 : int64_t(std::llround(L[t] / (2.0 * T[t - 1]) * 16777216.0));
        kconst[t] = t == 0 ? 0 : int32_t(std::llround(-jv * 65536.0));
    }
    if (kappa > 0)
        for (int t = 1; t < S; ++t) {
            const double rf = (ramp && t >= 0.7 * S) ? (S - 1 - t) / std::max(1.0, S - 1 - 0.7 * S) : 1.0;
            const double k = scale != 1.0 ? kappa * scale : kappa;
            kconst[t] = int32_t(std::llround(k * T[t - 1] * rf * 65536.0));
            kcorr[t] = 0;
        }
    return ANC_OK;
}

int anc_tables_steps(const anc_tables* tb) { return tb ? tb->S : 0; }

int anc_tables_read(const anc_tables* tb, int32_t* fourT, int32_t* q, int64_t* kcorr, int32_t* kconst) {
    if (!tb) return fail(ANC_EINVAL, "null handle");
    if (fourT) std::memcpy(fourT, tb->fourT.data(), size_t(tb->S) * 4);
    if (q) std::memcpy(q, tb->q.data(), size_t(tb->S) * 4);
    if (kcorr) std::memcpy(kcorr, tb->kcorr.data(), size_t(tb->S) * 8);
    if (kconst) std::memcpy(kconst, tb->kconst.data(), size_t(tb->S) * 4);
    return ANC_OK;
}

void anc_tables_destroy(anc_tables* tb) { delete tb; }

int anc_range_plan(const anc_instance* I, const anc_tables* tb, int* plain_ok, int32_t* hclamp) {
    if (!I || !tb) return fail(ANC_EINVAL, "null handle");
    Plan pl;
    const int rc = range_plan(I, tb, &pl);
    if (rc) return rc;
    if (plain_ok) *plain_ok = pl.plain_ok;
    if (hclamp) *hclamp = pl.hclamp;
    return ANC_OK;
}

int anc_auto_estimate(int n, int kbits, int nchains, int S, double phi, int fp4, const int* per_wave, double* us) {
    if (n < 1 || nchains < 1 || S < 1 || !per_wave || !us || !(kbits == 0 || kbits == 1 || kbits == 2 || kbits == 4))
        return fail(ANC_EINVAL, "anc_auto_estimate: n, nchains, S >= 1, kbits in {0, 1, 2, 4}, per_wave and us");
    int w[4];
    for (int e = 0; e < 4; ++e) w[e] = std::max(0, per_wave[e]);
    if (w[ANC_ENGINE_PLAIN] + w[ANC_ENGINE_TENSOR] + w[ANC_ENGINE_CLUSTER] == 0)
        return fail(ANC_EINVAL, "anc_auto_estimate: no engine available");
    return estimate_engines(n, kbits, nchains, S, phi, fp4 != 0, w, us);
}

int anc_auto_choice(anc_instance* I, anc_tables* tb, int nchains, const anc_run_opts* o, double* us, int* per_wave,
                    double* phi) {
    if (!I || !tb || nchains < 1) return fail(ANC_EINVAL, "anc_auto_choice: handles and nchains >= 1 required");
    anc_run_opts a = o ? *o : anc_run_opts{};
    a.engine = ANC_ENGINE_AUTO;
    double est[4], f = 0;
    const int e = pick_engine(I, tb, nchains, &a, est, &f);
    if (us) std::copy(est, est + 4, us);
    if (per_wave) std::copy(I->per_wave, I->per_wave + 4, per_wave);
    if (phi) *phi = f;
    return e;
}

int anc_run(anc_instance* I, anc_tables* tb, uint64_t seed, uint32_t off, int nchains, const anc_run_opts* o,
            uint64_t* spins, int64_t* sum_sh, int64_t* sum_bs, int64_t* flips, int32_t* trace) {
    return run_host_impl(I, tb, seed, off, nchains, o, spins, sum_sh, sum_bs, flips, trace, nullptr);
}

int anc_run_fields(anc_instance* I, anc_tables* tb, uint64_t seed, uint32_t off, int nchains, const anc_run_opts* o,
                   uint64_t* spins, int64_t* sum_sh, int64_t* sum_bs, int64_t* flips, int32_t* trace,
                   int32_t* fields) {
    if (!fields) return fail(ANC_EINVAL, "fields output required");
    return run_host_impl(I, tb, seed, off, nchains, o, spins, sum_sh, sum_bs, flips, trace, fields);
}

int anc_run_device(anc_instance* I, anc_tables* tb, uint64_t seed, uint32_t off, int nchains, const anc_run_opts* o,
                   uint64_t* d_spins, int64_t* d_sum_sh, int64_t* d_sum_bs, int64_t* d_flips, int32_t* d_trace,
                   void* stream) {
    OutPtrs out{reinterpret_cast<uint32_t*>(d_spins), reinterpret_cast<long long*>(d_sum_sh),
                reinterpret_cast<long long*>(d_sum_bs), reinterpret_cast<long long*>(d_flips), d_trace, nullptr};
    if (!d_sum_bs) return fail(ANC_EINVAL, "sum_bs output required on the device path");
    return run_device_impl(I, tb, seed, off, nchains, o, out, reinterpret_cast<cudaStream_t>(stream));
}

int anc_run_batch(int njobs, const anc_job* jobs, const anc_run_opts* o) {
    if (njobs < 1 || !jobs) return fail(ANC_EINVAL, "need jobs");
    // group by kernel kind (sparse / dense K); each group is one persistent launch with a cost-ordered work queue
    struct Prepared {
        int idx;
        int32_t hclamp;
    };
    std::vector<Prepared> prep;
    for (int k = 0; k < njobs; ++k) {
        const anc_job& j = jobs[k];
        if (!j.inst || !j.tb || j.nchains < 1 || !j.spins || !j.sum_sh)
            return fail(ANC_EINVAL, "job %d: need inst, tb, nchains >= 1, spins, sum_sh", k);
        int32_t hc = 0;
        const int rc = resolve_clamp(j.inst, j.tb, o, &hc);
        if (rc) return rc;
        prep.push_back({k, hc});
    }
    int dev = 0, sms = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    // every kind's launch plan (shared memory, residency) is checked before anything is allocated or enqueued, so a
    // refused batch leaves the caller's buffers and the device untouched
    KindPlan plans[4];
    {
        int np_k[4] = {0, 0, 0, 0}, nwj_k[4] = {0, 0, 0, 0};
        for (int k = 0; k < njobs; ++k) {
            const int ki = kind_index(jobs[k].inst->K);
            np_k[ki] = std::max(np_k[ki], jobs[k].inst->np);
            nwj_k[ki] = std::max(nwj_k[ki], jobs[k].inst->K == 0 ? jobs[k].inst->nw : jobs[k].inst->nwj);
        }
        for (int ki = 0; ki < 4; ++ki) {
            if (!np_k[ki]) continue;
            const int rc = plan_kind(kKinds[ki], np_k[ki], nwj_k[ki], sms, &plans[ki]);
            if (rc) return rc;
        }
    }
    cudaStream_t st = nullptr;
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    std::unique_ptr<CUstream_st, void (*)(cudaStream_t)> st_guard(st, [](cudaStream_t s) { cudaStreamDestroy(s); });
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    std::unique_ptr<CUevent_st, void (*)(cudaEvent_t)> g0(e0, [](cudaEvent_t e) { cudaEventDestroy(e); });
    std::unique_ptr<CUevent_st, void (*)(cudaEvent_t)> g1(e1, [](cudaEvent_t e) { cudaEventDestroy(e); });
    // per-job device outputs
    struct JobBufs {
        DevBuf<uint32_t> spins;
        DevBuf<long long> sh, bs, fl;
        DevBuf<int32_t> trace;
    };
    std::vector<std::unique_ptr<JobBufs>> bufs(njobs);
    std::vector<anc::PlainJob> pj(njobs);
    for (const Prepared& p : prep) {
        const anc_job& j = jobs[p.idx];
        bufs[p.idx].reset(new JobBufs());
        JobBufs& b = *bufs[p.idx];
        CK(b.spins.ensure(size_t(j.inst->nw) * j.nchains));
        CK(b.sh.ensure(j.nchains));
        CK(b.bs.ensure(j.nchains));
        CK(b.fl.ensure(j.nchains));
        if (j.trace) CK(b.trace.ensure(size_t(j.nchains) * j.tb->S));
        OutPtrs out{b.spins.p, b.sh.p, b.bs.p, b.fl.p, j.trace ? b.trace.p : nullptr, nullptr};
        pj[p.idx] = make_job(j.inst, j.tb, j.seed, j.trial_offset, j.nchains, p.hclamp, out);
    }
    DevBuf<anc::PlainJob> d_jobs;
    CK(d_jobs.ensure(njobs));
    CK(cudaMemcpy(d_jobs.p, pj.data(), sizeof(anc::PlainJob) * njobs, cudaMemcpyHostToDevice));
    DevBuf<int> counters;
    CK(counters.ensure(4));
    std::vector<DevBuf<int2>> d_items(4);
    // from here on work is enqueued: a failure waits for the stream before the buffers above are freed
    auto drain = [&](int rc) {
        cudaStreamSynchronize(st);
        return rc;
    };
    // work items per kind: a longest-processing-time-first queue, cost ~ np * S per anneal (dense np^2 * S)
    int nitems[4] = {0, 0, 0, 0};
    for (int ki = 0; ki < 4; ++ki) {
        const int K = kKinds[ki];
        std::vector<std::pair<double, int2>> items;
        for (int k = 0; k < njobs; ++k) {
            if (jobs[k].inst->K != K) continue;
            const double cost = double(jobs[k].inst->np) * jobs[k].tb->S * (K == 0 ? 1.0 : double(jobs[k].inst->np));
            for (int c = 0; c < jobs[k].nchains; ++c) items.push_back({cost, make_int2(k, c)});
        }
        if (items.empty()) continue;
        std::stable_sort(items.begin(), items.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
        std::vector<int2> it(items.size());
        for (size_t i = 0; i < items.size(); ++i) it[i] = items[i].second;
        cudaError_t e = d_items[ki].ensure(it.size());
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_items[ki].p, it.data(), it.size() * sizeof(int2), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return drain(cuda_fail(e, "work items"));
        nitems[ki] = int(it.size());
    }
    auto launch_kind = [&](int ki, const anc::PlainJob* djobs, int variant) -> int {
        const KindPlan& kp = plans[ki];
        anc::PlainLaunch L{};
        L.sparse_variant = variant;
        L.jobs = djobs;
        L.items = d_items[ki].p;
        L.nitems = nitems[ki];
        L.next_item = counters.p + ki;
        L.np_max = kp.np_max;
        L.nwj_max = kp.nwj_max;
        L.stream = kp.stream ? 1 : 0;
        const int grid = std::max(1, std::min(L.nitems, kp.per_sm * sms));
        cudaError_t e = cudaMemsetAsync(counters.p + ki, 0, sizeof(int), st);
        if (e != cudaSuccess) return cuda_fail(e, "memset");
        const int rc = anc::plain_launch(L, kKinds[ki], kp.P, grid, kp.smem, st);
        return rc ? cuda_fail(cudaError_t(rc), "plain engine launch") : ANC_OK;
    };
    // the CSR pass variant of the sparse launch: forced by the options, else tuned on this batch as a whole (each
    // variant runs the first min(S, 64) steps of every sparse job, twice, the second timed) and kept for batches of
    // the same instances and anneal counts
    int sparse_variant = (o && o->sparse_variant > 0) ? o->sparse_variant - 1 : -1;
    if (nitems[0] > 0 && sparse_variant < 0) {
        std::string key = std::to_string(dev);
        for (int k = 0; k < njobs; ++k)
            if (jobs[k].inst->K == 0)
                key += ":" + std::to_string(jobs[k].inst->uid) + "x" + std::to_string(jobs[k].nchains) + "s" +
                       std::to_string(std::min(jobs[k].tb->S, 64));
        {
            std::lock_guard<std::mutex> lock(g_batch_tune_mu);
            auto it = g_batch_tune.find(key);
            if (it != g_batch_tune.end()) sparse_variant = it->second;
        }
        if (sparse_variant < 0) {
            std::vector<anc::PlainJob> probe = pj;
            for (int k = 0; k < njobs; ++k) probe[k].tab.S = std::min(probe[k].tab.S, 64);
            DevBuf<anc::PlainJob> d_probe;
            CK(d_probe.ensure(njobs));
            CK(cudaMemcpy(d_probe.p, probe.data(), sizeof(anc::PlainJob) * njobs, cudaMemcpyHostToDevice));
            float best = 0.f;
            for (int v = 0; v < anc::kSparseVariants; ++v) {
                float ms = 0.f;
                for (int rep = 0; rep < 2; ++rep) {
                    CK(cudaEventRecord(e0, st));
                    const int rc = launch_kind(0, d_probe.p, v);
                    if (rc) return drain(rc);
                    CK(cudaEventRecord(e1, st));
                    CK(cudaEventSynchronize(e1));
                    CK(cudaEventElapsedTime(&ms, e0, e1));
                }
                if (sparse_variant < 0 || ms < best) { best = ms; sparse_variant = v; }
            }
            std::lock_guard<std::mutex> lock(g_batch_tune_mu);
            g_batch_tune[key] = sparse_variant;
        }
    }
    if (cudaEventRecord(e0, st) != cudaSuccess) return drain(cuda_fail(cudaGetLastError(), "event"));
    for (int ki = 0; ki < 4; ++ki) {
        if (!nitems[ki]) continue;
        const int rc = launch_kind(ki, d_jobs.p, ki == 0 ? std::max(0, sparse_variant) : 0);
        if (rc) return drain(rc);
    }
    if (cudaEventRecord(e1, st) != cudaSuccess) return drain(cuda_fail(cudaGetLastError(), "event"));
    for (const Prepared& p : prep) {
        const anc_job& j = jobs[p.idx];
        JobBufs& b = *bufs[p.idx];
        cudaError_t e = cudaMemcpyAsync(j.spins, b.spins.p, size_t(j.inst->nw) * j.nchains * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(j.sum_sh, b.sh.p, size_t(j.nchains) * 8, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess && j.sum_bs) e = cudaMemcpyAsync(j.sum_bs, b.bs.p, size_t(j.nchains) * 8, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess && j.flips) e = cudaMemcpyAsync(j.flips, b.fl.p, size_t(j.nchains) * 8, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess && j.trace)
            e = cudaMemcpyAsync(j.trace, b.trace.p, size_t(j.nchains) * j.tb->S * 4, cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) return drain(cuda_fail(e, "result copy"));
    }
    CK(cudaStreamSynchronize(st));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    g_dev_ms = ms;
    return ANC_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------------------------------
// Allocation-free batch entry point (anc_run_batch_noalloc). Its scratch lives in one file-scope device array, and
// the job table reaches it as the parameter block of a setup kernel, so no call here allocates or leaves a pointer to
// host memory in the stream: a CUDA graph that captured a call replays it as it was.
namespace {

constexpr int kNaMaxJobs = ANC_NOALLOC_MAX_JOBS;
constexpr int kNaMaxAnneals = ANC_NOALLOC_MAX_ANNEALS;
constexpr size_t kNaJobsOff = 256;   // [0, 256): four work-queue counters (one per kernel kind)
constexpr size_t kNaItemsOff = kNaJobsOff + ((size_t(kNaMaxJobs) * sizeof(anc::PlainJob) + 255) / 256) * 256;
constexpr size_t kNaBytes = kNaItemsOff + size_t(kNaMaxAnneals) * sizeof(int2);
static_assert(kNaBytes <= ANC_NOALLOC_SCRATCH_BYTES, "scratch larger than the size the header states");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

std::mutex g_na_mu;                       // guards the address table
void* g_na_addr[256] = {};                // device address of g_noalloc_scratch, per device ordinal

// One call's job table, passed by value to na_setup_kernel (sm_70+ kernels take parameter blocks up to 32764 bytes).
// Jobs are ordered by kernel kind; job k owns work items [first[k], first[k + 1]).
struct NaSetup {
    int njobs, nitems;
    int first[kNaMaxJobs + 1];
    anc::PlainJob jobs[kNaMaxJobs];
};
static_assert(sizeof(NaSetup) <= 32764, "job table exceeds the kernel parameter limit");

// Writes the job table into the scratch array and expands it into (job, anneal) work items.
__global__ void na_setup_kernel(const __grid_constant__ NaSetup s, anc::PlainJob* jobs, int2* items) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < s.njobs) jobs[t] = s.jobs[t];
    for (int i = t; i < s.nitems; i += gridDim.x * blockDim.x) {
        int lo = 0, hi = s.njobs - 1;   // the last job with first[k] <= i
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (s.first[mid] <= i) lo = mid; else hi = mid - 1;
        }
        items[i] = make_int2(lo, i - s.first[lo]);
    }
}

}  // namespace

extern "C" int anc_run_batch_noalloc(int njobs, const anc_device_job* jobs, void* stream) {
    if (njobs < 1 || !jobs) return fail(ANC_EINVAL, "need 1 <= njobs and a job array");
    if (njobs > kNaMaxJobs) return fail(ANC_EINVAL, "at most %d jobs per allocation-free call (got %d)", kNaMaxJobs, njobs);
    long long total = 0;
    for (int k = 0; k < njobs; ++k) {
        const anc_device_job& j = jobs[k];
        if (j.n < 1 || j.n > 65536) return fail(ANC_EINVAL, "job %d: n must be in 1..65536", k);
        if (!(j.kbits == 0 || j.kbits == 1 || j.kbits == 2 || j.kbits == 4))
            return fail(ANC_EINVAL, "job %d: kbits must be 0 (CSR), 1, 2 or 4", k);
        if (j.kbits ? !j.planes : (!j.row_ptr || !j.adj)) return fail(ANC_EINVAL, "job %d: coupling pointers missing", k);
        if (!j.fourT || !j.q || !j.kcorr || !j.kconst || j.S < 1) return fail(ANC_EINVAL, "job %d: tables missing", k);
        if (!j.spins || !j.sum_sh || !j.sum_bs || !j.flips) return fail(ANC_EINVAL, "job %d: outputs missing", k);
        if (j.nchains < 1 || j.hclamp < 0) return fail(ANC_EINVAL, "job %d: need nchains >= 1 and hclamp >= 0", k);
        total += j.nchains;
    }
    if (total > kNaMaxAnneals)
        return fail(ANC_EINVAL, "at most %d anneals per allocation-free call (got %lld)", kNaMaxAnneals, total);
    std::lock_guard<std::mutex> lock(g_na_mu);
    int dev = 0, sms = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 256) return fail(ANC_EINVAL, "device ordinal out of range");
    if (!g_na_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_na_addr[dev] = p;
    }
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    uint8_t* base = static_cast<uint8_t*>(g_na_addr[dev]);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    static thread_local NaSetup setup;   // 12 KB: kept off the stack
    NaSetup& S = setup;
    S.njobs = njobs;
    int kind_first[5] = {0, 0, 0, 0, 0}, kind_np[4] = {0, 0, 0, 0}, kind_nwj[4] = {0, 0, 0, 0};
    int slot = 0, items = 0;
    for (int ki = 0; ki < 4; ++ki) {
        kind_first[ki] = items;
        for (int k = 0; k < njobs; ++k) {
            const anc_device_job& j = jobs[k];
            if (j.kbits != kKinds[ki]) continue;
            anc::PlainJob& p = S.jobs[slot];
            p = anc::PlainJob{};
            p.n = j.n;
            p.np = pad_np(j.n);
            p.nw = p.np / 32;
            p.nwj = ((p.nw + 31) / 32) * 32;
            p.K = j.kbits;
            p.planes = j.planes;
            p.row_ptr = j.row_ptr;
            p.adj = j.adj;
            p.bias = j.bias;
            p.tab.fourT = j.fourT;
            p.tab.q = j.q;
            p.tab.kcorr = j.kcorr;
            p.tab.kconst = j.kconst;
            p.tab.S = j.S;
            p.seed = j.seed;
            p.trial_offset = j.trial_offset;
            p.ntrials = j.nchains;
            p.trace = j.trace != nullptr;
            p.hclamp = j.hclamp;
            p.out_spins = reinterpret_cast<uint32_t*>(j.spins);
            p.out_sum_sh = j.sum_sh;
            p.out_sum_bs = j.sum_bs;
            p.out_flips = j.flips;
            p.out_trace = j.trace;
            p.out_h = nullptr;
            kind_np[ki] = std::max(kind_np[ki], p.np);
            kind_nwj[ki] = std::max(kind_nwj[ki], p.K == 0 ? p.nw : p.nwj);
            S.first[slot++] = items;
            items += j.nchains;
        }
    }
    kind_first[4] = items;
    S.first[njobs] = items;
    S.nitems = items;
    // every kind's launch plan is checked before anything is enqueued: a refused call touches neither the scratch
    // array nor the caller's buffers
    KindPlan plans[4];
    for (int ki = 0; ki < 4; ++ki) {
        if (kind_first[ki + 1] == kind_first[ki]) continue;
        const int rc = plan_kind(kKinds[ki], kind_np[ki], kind_nwj[ki], sms, &plans[ki]);
        if (rc) return rc;
    }
    auto* d_jobs = reinterpret_cast<anc::PlainJob*>(base + kNaJobsOff);
    auto* d_items = reinterpret_cast<int2*>(base + kNaItemsOff);
    na_setup_kernel<<<(items + 255) / 256, 256, 0, st>>>(S, d_jobs, d_items);
    CK(cudaGetLastError());
    CK(cudaMemsetAsync(base, 0, 256, st));   // the counters must start at zero on every call
    for (int ki = 0; ki < 4; ++ki) {
        const int K = kKinds[ki];
        const int cnt = kind_first[ki + 1] - kind_first[ki], item_off = kind_first[ki];
        if (!cnt) continue;
        const KindPlan& kp = plans[ki];
        anc::PlainLaunch L{};
        L.jobs = d_jobs;
        L.items = d_items + item_off;
        L.nitems = cnt;
        L.next_item = reinterpret_cast<int*>(base) + ki;
        L.np_max = kp.np_max;
        L.nwj_max = kp.nwj_max;
        L.stream = kp.stream ? 1 : 0;
        const int rc = anc::plain_launch(L, K, kp.P, std::max(1, std::min(cnt, kp.per_sm * sms)), kp.smem, st);
        if (rc) return cuda_fail(cudaError_t(rc), "plain engine launch");
    }
    return ANC_OK;
}
