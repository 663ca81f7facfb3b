// Batched SCA engine for replicas sharing J (tcgen05 int8 J * dS update); host-facing interface.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "anc_common.cuh"

namespace anc {

struct TensorInstance {
    int n = 0, np = 0;
    std::vector<int> perm;       // slot i -> permuted index (CTA-contiguous slot slices)
    int8_t* d_J = nullptr;       // J_perm [np][np] int8 (row = y, contiguous x)
    size_t bytes = 0;
    void* d_ws = nullptr;        // exchange buffers + error word
    size_t ws_bytes = 0;
    int32_t* d_bias_perm = nullptr;
    int* last_err = nullptr;     // error word of the last launch
};

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
};

// Launch geometry of a run: CTAs in the grid, CTAs per cluster, and how many clusters can be co-resident.
struct TensorGeometry {
    int ctas = 0, cluster = 0, max_active_clusters = 0;
};
int tensor_geometry(int n, int nchains, TensorGeometry* g);

bool tensor_supported(int n, int K, int nchains);
bool tensor_prefer(int n, int K, int nchains, int S);
int tensor_build_instance(const int8_t* J, int n, TensorInstance* out, std::string* why);
int tensor_run(TensorInstance* ti, const TensorRun& r, cudaStream_t st, std::string* why);
// After the stream has reached the launch: -3 if a bounded device wait expired, 0 otherwise.
int tensor_check_error(TensorInstance* ti, cudaStream_t st, std::string* why);
void tensor_free_instance(TensorInstance* ti);

}  // namespace anc
