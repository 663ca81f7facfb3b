/* anechoic-b200: C ABI of the B200 SCA (stochastic cellular automata) annealing engines.
 *
 * The reference has no library API: its drop-in surface is the CLI pair sca_gpu / sca_gpu_bias, their output files,
 * and the golden model's header functions. Each entry point below names the reference interface it replaces
 * (paths relative to the reference project root).
 *
 * Conventions
 *   - Plain C types only; the caller owns every host buffer. Handles own their device memory and free it in destroy.
 *   - Every function returns an int status (ANC_OK = 0 or a negative ANC_E* code); anc_last_error() returns the
 *     message of the calling thread's last failure. No C++ exception crosses the ABI.
 *   - Spin vectors are uint64 words, bit i of word i/64 set iff s_i = +1 (active spins only), anc_spin_words(n)
 *     words per anneal: the layout of the reference's PREFIX.spins.bin records (32 words for n <= 2048).
 *   - Calls on one handle must be serialised by the caller. Synchronous calls return after the results are on the
 *     host. One process drives one GPU (the current CUDA device when the handle is created).
 */
#ifndef ANECHOIC_H
#define ANECHOIC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define ANC_API __attribute__((visibility("default")))
#else
#define ANC_API
#endif

#define ANC_OK 0
#define ANC_EINVAL (-1)    /* invalid argument, or the int32 range plan refused the tables (reference: FAIL + exit 1) */
#define ANC_ECUDA (-2)     /* CUDA runtime error */
#define ANC_ETIMEOUT (-3)  /* a bounded device-side wait gave up (the kernel returned an error status) */
#define ANC_EMISMATCH (-4) /* internal consistency check failed (reference: cut mismatch, exit 2) */

#define ANC_ENGINE_AUTO 0   /* pick per launch: the engine with the least estimated device time (anc_auto_estimate) */
#define ANC_ENGINE_PLAIN 1  /* bit-column engine: one CTA per anneal, bit-packed couplings, flipped columns only */
#define ANC_ENGINE_TENSOR 2 /* batched engine: replicas sharing J, tcgen05 int8 J * dS update */
#define ANC_ENGINE_CLUSTER 3 /* bit-column engine with each anneal spread over a cluster of 8 CTAs (dense K = 1,
                               n <= 2048): the lowest latency per anneal. The reference's engine keeps one anneal on
                               an 8-CTA cluster too (gpu/onsager_v2_20261007/src/sca_gpu.cu:223-295) */

#define ANC_TENSOR_AUTO 0   /* fp4 when exact for the instance (NP = 2048, |J| <= 1, small fields), else int8 */
#define ANC_TENSOR_INT8 1   /* tcgen05.mma kind::i8, int32 accumulation (any K) */
#define ANC_TENSOR_FP4 2    /* tcgen05.mma kind::mxf4 on packed e2m1 with unit block scales, fp32 accumulation;
                              exact because J in {-1,0,1}, dS in {0,+-1,+-2} and |h| < 2^14 (EINVAL otherwise) */

typedef struct anc_instance anc_instance;
typedef struct anc_tables anc_tables;

/* Instance statistics (jmat::finish, gpu/multibit_bias_20261008/src/jmat.hpp:21-40). */
typedef struct {
    int n;            /* active spins */
    int np;           /* padded spins: max(2048, ceil(n/256)*256); 256 RNG lanes x np/256 rounds */
    int kbits;        /* bits per coupling of the packed planes (1 = +-1 complete graph; 2, 4; 0 = CSR) */
    int sparse;       /* 1 if couplings are held as CSR rows */
    int64_t nnz;      /* nonzero couplings (both triangles) */
    int64_t sumw;     /* sum_{i<j} w_ij, w = -J: cut = (sumw + sum_sh / 2) / 2 */
    int32_t maxabs;   /* max |J| */
    int64_t hmax;     /* max_y sum_x |J_xy| */
    int32_t bmax;     /* max |b| */
    double mean_row_sq; /* mean_i sum_j J_ij^2 */
} anc_instance_info;

/* Replaces sca::load_graph / jmat::load + jmat::load_bias (sca_ref.hpp:31-49, jmat.hpp:115-120,164-178) as the way
 * couplings reach the engine. J_dense: n*n int8 row-major, symmetric, zero diagonal. kbits: 0 = smallest fitting
 * (1 for a +-1 complete graph, else 2/4), or 1/2/4 explicitly. bias: n int32 (|b| <= 32767) or NULL. */
ANC_API int anc_instance_create(const int8_t* J_dense, int n, int kbits, const int32_t* bias, anc_instance** out);

/* Sparse couplings as CSR rows: row_ptr[n+1], col[nnz], val[nnz] (every nonzero of row x; each pair in both rows). */
ANC_API int anc_instance_create_csr(int n, const int32_t* row_ptr, const int32_t* col, const int8_t* val, const int32_t* bias,
                            anc_instance** out);

ANC_API int anc_instance_get_info(const anc_instance* inst, anc_instance_info* info);
ANC_API void anc_instance_destroy(anc_instance* inst);

/* Replaces sca::make_tables / v80host::build_tables (sca_ref.hpp:51-68, tables.hpp:24-40): explicit per-step tables.
 * fourT: Q16.16 of 4T_t (> 0); q: Q16.16; kcorr: Q8.24 of lambda_t / (2 T_{t-1}); kconst: Q16.16. */
ANC_API int anc_tables_create(const int32_t* fourT, const int32_t* q, const int64_t* kcorr, const int32_t* kconst, int S,
                      anc_tables** out);

/* Schedule -> tables, bit-identical to v80host::build_tables (scale == 1) and mb::tables (mb_common.hpp:141-154):
 * T_t = t0 (t1/t0)^(t/(S-1)); lam > 0 counted Onsager (with optional ramp); kappa > 0 temperature-scaled (TEC-T);
 * jv != 0 TEC; all zero = no correction. */
ANC_API int anc_tables_from_schedule(int S, double t0, double t1, double q, double lam, double jv, double kappa, int ramp,
                             double scale, anc_tables** out);
ANC_API int anc_tables_steps(const anc_tables* tb);
ANC_API int anc_tables_read(const anc_tables* tb, int32_t* fourT, int32_t* q, int64_t* kcorr, int32_t* kconst);
ANC_API void anc_tables_destroy(anc_tables* tb);

/* Range plan (host::check_ranges / host::plan_ranges, gpu/onsager_v2_20261007/src/sca_gpu.cu:519-528,
 * gpu/multibit_bias_20261008/src/sca_gpu_bias.cu:536-557): plain_ok = 1 if s*h*65536 + q -/+ corr fits int32
 * unclamped; hclamp = clamp bound used otherwise (exact). ANC_EINVAL if even the clamped form overflows. */
ANC_API int anc_range_plan(const anc_instance* inst, const anc_tables* tb, int* plain_ok, int32_t* hclamp);

/* Host-only forms of the two functions above (no CUDA call; usable without a GPU).
 * anc_schedule_tables fills caller arrays of S entries exactly as anc_tables_from_schedule would upload them.
 * anc_plan_ranges takes n, hmax = max_y sum_x |J_xy| and bmax = max |b| (see anc_instance_info). */
ANC_API int anc_schedule_tables(int S, double t0, double t1, double q, double lam, double jv, double kappa, int ramp,
                                double scale, int32_t* fourT, int32_t* q_out, int64_t* kcorr, int32_t* kconst);
ANC_API int anc_plan_ranges(int n, int64_t hmax, int64_t bmax, const int32_t* fourT, const int32_t* q,
                            const int64_t* kcorr, const int32_t* kconst, int S, int* plain_ok, int32_t* hclamp);

/* Words per spin vector: anc_np(n) / 64. */
ANC_API int anc_spin_words(int n);
ANC_API int anc_np(int n);

typedef struct {
    int engine;      /* ANC_ENGINE_* */
    int wide;        /* -1 auto (clamp only if the plan needs it), 0 never (EINVAL if needed), 1 always */
    int threads;     /* host threads for rescoring; 0 = default */
    int profile;     /* 1: record per-phase cycle counters of the tensor engine (anc_last_profile) */
    int tensor_kind; /* ANC_TENSOR_*: operand format of the tensor engine's field update */
    int flip_permille; /* AUTO's flip fraction (flips per spin per step) x 1000; 0 = the fraction the last anc_run /
                          anc_run_fields of these tables on this instance saw, else 0.25 */
    int sparse_variant; /* CSR instances on the plain engine: 0 = the variant the run-time tuner chose for the instance
                           (anc_sparse_tuning), v + 1 = force variant v (0 .. 3) */
    int kernel_variant; /* dense instances on the plain engine and the tensor engine's fp4 kernel: 0 = the variant the
                           run-time tuner chose (anc_kernel_tuning; the default variant before any tuning), v + 1 =
                           force variant v. Cluster engine: 0 = 16 CTAs per anneal when the anneals fit one wave of
                           16-CTA clusters, else 8; 1 = 8 CTAs; 2 = 16 CTAs. CSR instances on the plain engine: the
                           edge format -- 0 = 16-bit edges (two per fetched word) when every weight is +-1 and
                           n < 32767, else 32-bit; 1 = 32-bit; 2 = 16-bit (EINVAL when not eligible) */
} anc_run_opts;

/* No counterpart in the reference (its kernel geometry is fixed per build by flags, sca_gpu_bias.cu:637-644). The
 * run-time tuner of the plain engine's CSR pass: on an instance's first synchronous run (anc_run / anc_run_fields /
 * anc_run_batch) each compiled variant -- lane groups x edges fetched per lane before any is applied: {1, 8},
 * {1, 4}, {2, 4}, {1, 16} -- runs the first min(S, 64) steps of up to one wave of that run's anneals into the handle's
 * own workspaces (twice; the second launch is timed), and the fastest is used for every later launch of the
 * instance. Writes the chosen variant (-1 = not tuned yet, or not a CSR instance) and probe_us[4], each variant's
 * probe time per step in microseconds (may be NULL). */
ANC_API int anc_sparse_tuning(const anc_instance* inst, int* variant, double* probe_us);

/* No counterpart in the reference (its tile shapes and depths are fixed per build by flags, sca_gpu_bias.cu:637-644).
 * The run-time tuner of the dense kernels' compiled variants:
 *   ANC_KERNEL_PLAIN (dense instances): rows of bit planes a thread counts per batch -- K = 1: 0 = 8 rows with the
 *     next 8 fetched ahead, 1 = 8 rows, 2 = 16 rows; K = 2: 0 = 8 rows, 1 = 16 rows; K = 4 and NP > 8192: one variant;
 *   ANC_KERNEL_TENSOR_FP4: the depth of the shared-memory ring of dS tiles -- 0 = 4 stages, 1 = 6, 2 = 5, 3 = 3.
 * The first synchronous run (anc_run / anc_run_fields) that uses one of these kernels for a (device, kernel, NP, K,
 * replica groups) key not yet tuned runs each variant on the first min(S, 256) steps of that run's anneals (one wave
 * of the plain engine, every replica group of the fp4 kernel) into the handle's own workspaces -- three times, the
 * least of the last two launches timed -- and keeps variant 0 unless another probes more than 1 % faster, in which
 * case the fastest, for every later launch with that key in the process (device and
 * graph-captured launches included; anc_run_batch and anc_run_batch_noalloc use variant 0). For the key a run of
 * nchains anneals of this instance on `kernel` would use, writes the chosen variant (-1 = not tuned yet), the number
 * of compiled variants and probe_us[4], each variant's probe time per step in microseconds (may be NULL). */
ANC_API int anc_kernel_tuning(const anc_instance* inst, int kernel, int nchains, int* variant, int* nvariants,
                              double* probe_us);

/* No counterpart in the reference (its CLI has one engine). The cost model behind ANC_ENGINE_AUTO, host-only: the
 * estimated device time in microseconds of nchains anneals of S steps on each engine, for n spins with kbits-bit dense
 * couplings (0 = sparse rows), flip fraction phi (mean flips per spin per step), fp4 = whether the tensor engine would
 * run its fp4 kernel, and per_wave[e] = the anneals engine e advances at once on the device (0 = unavailable; index
 * ANC_ENGINE_*, entry 0 unused). Writes us[ANC_ENGINE_PLAIN / _TENSOR / _CLUSTER] (-1 = unavailable) and returns the
 * engine with the least estimate. Per-step costs are fitted to B200 measurements (anc_api.cu). */
ANC_API int anc_auto_estimate(int n, int kbits, int nchains, int S, double phi, int fp4, const int* per_wave,
                              double* us);

/* The engine AUTO would pick for anc_run(inst, tb, ..., nchains, opts), with the inputs it used: us[4] as above,
 * per_wave[4] queried on the current device, phi the flip fraction assumed. Any output may be NULL. */
ANC_API int anc_auto_choice(anc_instance* inst, anc_tables* tb, int nchains, const anc_run_opts* opts, double* us,
                            int* per_wave, double* phi);

/* Phase profile of the calling thread's last synchronous tensor-engine run with opts.profile = 1 (the counterpart
 * of the reference's SCA_PROFILE build, sca_gpu.cu:163-168): out[0..8] = mean SM cycles per step of
 *   0 wait for fields, 1 TMEM load + decide + update store, 2 n_lin publish, 3 cluster barrier, 4 n_lin read,
 *   5 MMA waiting for TMA, 6 MMA phase (barrier to last commit), 7 TMA waiting for free stages, 8 whole step;
 * out[9] = CTAs, out[10] = CTAs per cluster, out[11] = co-resident clusters, out[12] = MMA issue, out[13] = MMA
 * commits (cycles per step); fp4 kernel, cycles after the CTA's own publish: out[14] first update tile in shared
 * memory, out[15] last update tile, out[16] n_lin tile, out[17] fields-ready commit, out[18] / out[19] flags of
 * update tile 0 / 7 seen, out[20] / out[21] TMA of tile 0 / 7 issued (slot 3 there is the flag publish alone and
 * slot 4 the fields-ready wake-up after the own publish). Returns the count written (<= max). */
ANC_API int anc_last_profile(double* out, int max);

/* Replaces one launch + readback of sca_gpu / sca_gpu_bias (sca_gpu.cu:699-713, sca_gpu_bias.cu:716-733) and
 * sca::run_trial / run_trial_bias per chain: nchains anneals with trial ids trial_offset + c.
 * Outputs (host, caller-owned, may be NULL unless noted):
 *   spins   [nchains][anc_spin_words(n)] (required)
 *   sum_sh  [nchains]  sum_i s_i h_i over active spins with the biased fields (required)
 *   sum_bs  [nchains]  sum_i b_i s_i
 *   flips   [nchains]  total flips
 *   trace   [nchains][S] n_lin per step (the reference's PREFIX.trace.bin layout)
 * opts may be NULL (auto engine, auto wide). */
ANC_API int anc_run(anc_instance* inst, anc_tables* tb, uint64_t seed, uint32_t trial_offset, int nchains,
            const anc_run_opts* opts, uint64_t* spins, int64_t* sum_sh, int64_t* sum_bs, int64_t* flips,
            int32_t* trace);

/* As anc_run, also returning the final fields h [nchains][n] (for --check-fields, jmat.hpp:153-161). */
ANC_API int anc_run_fields(anc_instance* inst, anc_tables* tb, uint64_t seed, uint32_t trial_offset, int nchains,
                   const anc_run_opts* opts, uint64_t* spins, int64_t* sum_sh, int64_t* sum_bs, int64_t* flips,
                   int32_t* trace, int32_t* fields);

/* Device-resident variant (no host copies, no synchronisation; graph-capturable once the handle has run once):
 * outputs are DEVICE pointers laid out as in anc_run; trace may be NULL; stream is a cudaStream_t (NULL = default). */
ANC_API int anc_run_device(anc_instance* inst, anc_tables* tb, uint64_t seed, uint32_t trial_offset, int nchains,
                   const anc_run_opts* opts, uint64_t* d_spins, int64_t* d_sum_sh, int64_t* d_sum_bs,
                   int64_t* d_flips, int32_t* d_trace, void* stream);

/* Many instances / schedules in ONE persistent launch (work queue, uneven sizes). */
typedef struct {
    anc_instance* inst;
    anc_tables* tb;
    uint64_t seed;
    uint32_t trial_offset;
    int nchains;
    uint64_t* spins;   /* host outputs as in anc_run */
    int64_t* sum_sh;
    int64_t* sum_bs;
    int64_t* flips;
    int32_t* trace;
} anc_job;

/* Replaces running sca_gpu_bias once per instance (run_gsel.sh / run_bias.sh loops). */
ANC_API int anc_run_batch(int njobs, const anc_job* jobs, const anc_run_opts* opts);

/* No counterpart in the reference. Allocation-free batch run of the plain engine, for callers that cannot call
 * cudaMalloc: applications that own every byte of device memory through their own pool or allocator (a serving
 * runtime or framework caching allocator that has reserved the GPU), and callers with a fixed device-memory budget
 * that must not grow. All inputs and outputs are DEVICE memory owned by the caller; the call allocates nothing
 * (no cudaMalloc, no cudaFree, no allocating library routine). Its scratch -- job descriptors, the work-item queue
 * and its counters -- is one file-scope device array of ANC_NOALLOC_SCRATCH_BYTES that every GPU loading the library
 * holds until exit. The first call on a device does a one-time set-up with that device current: it looks the array
 * up (cudaGetSymbolAddress), queries occupancy, and may load the kernels; make that first call before any stream
 * capture on the device. Limits: at most ANC_NOALLOC_MAX_JOBS jobs and ANC_NOALLOC_MAX_ANNEALS anneals (sum of
 * nchains) per call; larger requests return ANC_EINVAL. Every call reuses the same array and resets its counters:
 * calls that overlap on the GPU (different streams, or several host threads) race; calls in order on one stream do
 * not. A call whose jobs cannot run (sizes, a kind the plain engine cannot hold) returns ANC_EINVAL before it
 * enqueues anything. The job table travels as a kernel parameter block, so the call leaves no reference to host
 * memory in the stream.
 * Job layout:
 *   kbits 1/2/4: planes = [kbits][NP][NWJ] uint32 with NP = anc_np(n), NWJ = ceil(NP/32) rounded up to a multiple of
 *   32; word x*NWJ + y/32, bit y%32 of plane p describes J_xy: kbits 1 -> [J_xy = +1] (a +-1 complete graph);
 *   kbits 2/4 -> plane 0 = [J_xy < 0], plane b = bit b-1 of |J_xy|. kbits 0: CSR row_ptr[n+1] and
 *   adj[k] = (y << 8) | (uint8)J_xy for every nonzero of row x.
 *   hclamp: 0 when anc_plan_ranges reports plain_ok, else its hclamp. This call does not re-check it (the tables are
 *   in device memory): an hclamp of 0 where the plan needs the clamp lets the int32 decision overflow silently and
 *   gives wrong results. Outputs as anc_run_device. */
#define ANC_NOALLOC_MAX_JOBS 64
#define ANC_NOALLOC_MAX_ANNEALS 16384
#define ANC_NOALLOC_SCRATCH_BYTES (144 * 1024) /* upper bound of the device scratch array (139 KB used) */
typedef struct {
    int n;
    int kbits;
    const uint32_t* planes;
    const int32_t* row_ptr;
    const uint32_t* adj;
    const int32_t* bias;      /* n entries or NULL */
    const int32_t* fourT;     /* tables, S entries each */
    const int32_t* q;
    const int64_t* kcorr;
    const int32_t* kconst;
    int S;
    int32_t hclamp;
    uint64_t seed;
    uint32_t trial_offset;
    int nchains;
    uint64_t* spins;          /* [nchains][anc_spin_words(n)] */
    int64_t* sum_sh;          /* [nchains] */
    int64_t* sum_bs;          /* [nchains] */
    int64_t* flips;           /* [nchains] */
    int32_t* trace;           /* [nchains][S] or NULL */
} anc_device_job;
ANC_API int anc_run_batch_noalloc(int njobs, const anc_device_job* jobs, void* stream);

/* ---------------------------------------------------------------------------------------------------------------
 * Differentiable mean-field relaxation (new; the reference has no differentiable path). Soft surrogate of the
 * corrected dynamics, per replica r and step t = 0 .. S-1:
 *   P_t = J m_t + b + q_t m_t - gamma_t m_{t-1},  gamma_t[r] = u_t sum_i (1 - m_t[r,i]^2) + w_t,  m_{t+1} = tanh(beta_t P_t)
 * with beta_t = 1/(2 T_t), u_t = lambda_t / (2 T_{t-1}) (counted Onsager gain), w_t the constant correction
 * (kappa T_{t-1} temperature-scaled, -jv constant): the tanh form of the reference's effective process
 * (research/dmft_sca_20261004/dmft_torch.py:38-57) and the soft version of sca_ref.hpp:118-131.
 * J in BF16 (exact for the integer couplings), f32 magnetisations and accumulation (tcgen05 kind::f16 GEMM with m
 * split into three BF16 terms), checkpoints every 16 steps in the adjoint. All pointers below are DEVICE pointers;
 * calls are asynchronous on `stream` (NULL = default); anc_mf_check synchronises and reports a device wait timeout.
 *   sched:  [4][S] f32 rows beta, q, u, w
 *   m0, mprev, m_out: [64][npad] f32 (rows = replicas; unused rows and columns i >= n stay zero)
 *   ckpt:   [ceil(S/16)][2][64][npad] f32 (written by forward, read by backward)
 *   g_m:    dL/dm_S [64][npad];  gsched: [S][4][64] per-replica partials of dL/d(beta, q, u, w)_t
 * --------------------------------------------------------------------------------------------------------------- */
typedef struct anc_meanfield anc_meanfield;
ANC_API int anc_mf_create(const int8_t* J, int n, const int32_t* bias, anc_meanfield** out);
ANC_API int anc_mf_npad(const anc_meanfield* mf);
ANC_API int anc_mf_forward(anc_meanfield* mf, int S, const float* sched, const float* m0, const float* mprev,
                           float* ckpt, float* m_out, void* stream);
ANC_API int anc_mf_backward(anc_meanfield* mf, int S, const float* sched, const float* ckpt, const float* g_m,
                            float* gsched, void* stream);
ANC_API int anc_mf_check(anc_meanfield* mf, void* stream);
/* Limit (ns, default 2e9) of each device wait of this context's kernels. A wait that reaches it makes the kernel
 * record an error, let its own copies and MMAs finish, skip the rest of its work and return; anc_mf_check then
 * returns ANC_ETIMEOUT and clears the error, and the context stays usable. */
ANC_API int anc_mf_set_wait_ns(anc_meanfield* mf, uint64_t ns);
ANC_API void anc_mf_destroy(anc_meanfield* mf);

/* No counterpart in the reference, whose spins on its exchange mbarriers have no bound
 * (gpu/onsager_v2_20261007/src/sca_gpu.cu:249). Limit (ns, default 2e9) of each device-side wait of the tensor engine's
 * kernels launched after this call, process-wide. A wait that reaches it makes the kernel record an error, stop
 * issuing work, wait (with its own fixed bound) for the copies and MMAs it has in flight, and return; the call
 * returns ANC_ETIMEOUT, the results are not valid, and the context and handles stay usable. 0 gives up at the first
 * unsatisfied poll (for tests of that path). The cluster engine's exchange waits use the same limit with a floor of
 * 10 ms. anc_get_wait_ns returns the current limit. */
ANC_API int anc_set_wait_ns(uint64_t ns);
ANC_API uint64_t anc_get_wait_ns(void);

/* Last device time of a synchronous run on this thread (ms, CUDA events around the launch). */
ANC_API double anc_last_device_ms(void);

/* Kernel used by this thread's last anc_run / anc_run_fields / anc_run_device: ANC_KERNEL_* (0 if none yet). */
#define ANC_KERNEL_PLAIN 1        /* bit-column engine */
#define ANC_KERNEL_TENSOR_INT8 2  /* tcgen05 kind::i8 engine */
#define ANC_KERNEL_TENSOR_FP4 3   /* tcgen05 kind::mxf4 engine */
#define ANC_KERNEL_PLAIN_CLUSTER 4 /* bit-column engine, one anneal per 8-CTA cluster */
ANC_API int anc_last_kernel(void);

/* Message of the calling thread's last failure ("" if none). */
ANC_API const char* anc_last_error(void);

/* Library version string. */
ANC_API const char* anc_version(void);

#ifdef __cplusplus
}
#endif
#endif /* ANECHOIC_H */
