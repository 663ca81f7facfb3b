// Differentiable mean-field relaxation of the corrected SCA dynamics (soft surrogate of the exact integer engine).
//
// Forward, per replica r and step t = 0 .. S-1 (m_t in [-1, 1]^n, f32):
//   P_t = J m_t + b + q_t m_t - gamma_t m_{t-1},   gamma_t[r] = u_t * n_t[r] + w_t,   n_t[r] = sum_i (1 - m_t[r,i]^2)
//   m_{t+1} = tanh(beta_t P_t)
// beta_t = 1 / (2 T_t); u_t = lambda_t / (2 T_{t-1}) is the counted (Onsager) gain and w_t the constant correction
// (kappa T_{t-1}: temperature-scaled; -jv: constant). This is the tanh form of the effective process in
// research/dmft_sca_20261004/dmft_torch.py:38-57, and the soft version of the golden model's decision
// (sca_ref.hpp:118-131: flip probability (1 - clamp(s g / 2T)) / 2 with g = h + q s - corr s_prev, and n_lin -> the
// expected number of slots inside the linear band).
//
// J is held in BF16 (exact for |J| <= 256); J m is a tcgen05 kind::f16 GEMM (M 128 rows of J, N 64 replicas,
// K split over CTAs) with m given as three BF16 terms (24 significant bits, so every product is the f32 product),
// f32 accumulation, and the split-K partials summed in a fixed order by the elementwise kernels (deterministic).
//
// The adjoint runs the recurrence backwards from dL/dm_S with activation checkpoints every 16 steps (each segment
// recomputed once) and returns per-step sums dL/dbeta_t, dL/dq_t, dL/du_t, dL/dw_t (one value per replica, summed
// by the caller).
#pragma once
#include <cstdint>
#include <string>

#include <cuda_runtime.h>

namespace anc {

constexpr int kMfReplicas = 64;   // replica rows of every m buffer (MMA N); unused rows carry zero gradients
constexpr int kMfCheckpoint = 16;

struct MfContext;

// J: host int8 [n][n] (symmetric), bias: host int32 [n] or null. npad = ceil(n / 256) * 256.
int mf_create(const int8_t* J, const int32_t* bias, int n, MfContext** out, std::string* why);
int mf_npad(const MfContext* c);
// Device buffers: sched = 4 arrays [S] (beta, q, u, w); m0, mprev: [64][npad]; ckpt: [ceil(S/16)][2][64][npad];
// m_out: [64][npad].
int mf_forward(MfContext* c, int S, const float* beta, const float* q, const float* u, const float* w, const float* m0,
               const float* mprev, float* ckpt, float* m_out, cudaStream_t st, std::string* why);
// g_m: dL/dm_S [64][npad]; gsched: [S][4][64] per-replica partial sums (beta, q, u, w).
int mf_backward(MfContext* c, int S, const float* beta, const float* q, const float* u, const float* w,
                const float* ckpt, const float* g_m, float* gsched, cudaStream_t st, std::string* why);
// Limit of each device wait (default 2 s); a wait that reaches it makes the kernel record an error, let its own
// copies and MMAs finish, skip the rest of its work and return.
int mf_set_wait_ns(MfContext* c, uint64_t ns);
// -3 if a bounded device wait expired during the last call on this context, 0 otherwise (synchronises st).
int mf_check_error(MfContext* c, cudaStream_t st, std::string* why);
void mf_destroy(MfContext* c);

}  // namespace anc
