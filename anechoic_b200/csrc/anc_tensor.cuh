// Batched SCA engine for replicas sharing J (tcgen05 int8 J * dS update); host-facing interface.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "anc_common.cuh"

namespace anc {

struct TensorInstance {
    int n = 0, np = 0;
    int npp = 0;                 // permuted width of J_perm (np, or 16384 for the streaming kernel)
    bool stream = false;         // 32 < NP/256 <= 64: J streamed from HBM (tensor_stream.cu)
    std::vector<int> perm;       // slot i -> permuted index (CTA-contiguous slot slices)
    int8_t* d_J = nullptr;       // J_perm [np][np] int8 (row = y, contiguous x)
    size_t bytes = 0;
    void* d_ws = nullptr;        // exchange buffers + error word
    size_t ws_bytes = 0;
    int32_t* d_bias_perm = nullptr;
    int64_t bias_absmax = 0;     // max |b_i| (set with d_bias_perm)
    uint8_t* d_J4 = nullptr;     // J_perm as packed e2m1 [2048][1024] when NP = 2048 and every |J_xy| <= 1, else null
    int64_t rowsum_max = 0;      // max_y sum_x |J_xy|
    int* last_err = nullptr;     // error word of the last launch
    int last_kind = 0;           // kernel of the last launch: TENSOR_KIND_INT8 or TENSOR_KIND_FP4
    int last_ctas = 0, last_cluster = 0;
};

// Slots per CTA of the opt-in phase profile (clock64 totals, see tensor_engine.cu).
constexpr int kTensorProfSlots = 56;

// Operand format of the field update: int8 (any |J| <= 127) or packed fp4 e2m1 (|J| <= 1, NP = 2048).
constexpr int TENSOR_KIND_AUTO = 0, TENSOR_KIND_INT8 = 1, TENSOR_KIND_FP4 = 2;

struct TensorRun {
    DevTables tab;
    uint64_t seed;
    uint32_t trial_offset;
    int nchains;
    int32_t hclamp;
    const int32_t* bias;
    uint32_t* out_spins;
    int64_t* out_sum_sh;
    int64_t* out_sum_bs;
    int64_t* out_flips;
    int32_t* out_trace;
    int32_t* out_h;
    long long* prof;          // device [grid][16] phase cycle totals, or null (profiling off)
    int kind;                 // TENSOR_KIND_*
    uint64_t wait_ns;         // limit of each device wait of the launch (0: give up at the first unsatisfied poll)
    int variant;              // compiled variant of the fp4 kernel (kF4Variants; 0 = the 4-stage ring)
};

// Compiled variants of the fp4 kernel: the depth of its shared-memory ring of dS tiles (variant 0 .. 3: 4, 6, 5 or 3
// stages of 16 KB; 4 measured fastest on a B200 at 1 and 8 replica groups, so it is the default before tuning).
constexpr int kF4Variants = 4;

// Launch geometry of a run: CTAs in the grid, CTAs per cluster, and how many clusters can be co-resident.
struct TensorGeometry {
    int ctas = 0, cluster = 0, max_active_clusters = 0;
};
int tensor_geometry(int n, int nchains, TensorGeometry* g);

bool tensor_supported(int n, int K, int nchains);
// Anneals one launch of the tensor kernel that runs this instance advances together (more anneals take further waves
// of replica groups inside the launch): fp4 is whether the fp4 kernel would run it.
int tensor_wave_chains(int n, bool fp4, int* out);
int tensor_build_instance(const int8_t* J, int n, TensorInstance* out, std::string* why);
int tensor_run(TensorInstance* ti, const TensorRun& r, cudaStream_t st, std::string* why);
// Whether the fp4 kernel can run this instance with this bias bound exactly (the fields stay far inside the range
// where fp32 accumulation of integers is exact).
bool tensor_fp4_eligible(const TensorInstance* ti, int64_t bias_absmax);
// Streaming kernel for NP in (8192, 16384] (tensor_stream.cu): support test, slot permutation, permuted width, launch.
bool stream_supported(int n);
void stream_permutation(int np, std::vector<int>* p);
int stream_width();
int stream_wave_chains();
int stream_run(TensorInstance* ti, const TensorRun& r, const int32_t* bias_perm, cudaStream_t st, std::string* why);
// After the stream has reached the launch: -3 if a bounded device wait expired, 0 otherwise.
int tensor_check_error(TensorInstance* ti, cudaStream_t st, std::string* why);
void tensor_free_instance(TensorInstance* ti);

}  // namespace anc
