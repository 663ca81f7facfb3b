// Device-side pieces shared by the SCA engines: the reference's random stream and fixed-point decision arithmetic.
//
// Random stream: xoshiro128** per (trial, RNG lane), seeded by splitmix64(seed ^ trial << 20 ^ lane << 48 ^ 0x5CA0F00D)
// with an all-zero guard -- the stream of sca::Rng (reference gpu/onsager_v2_20261007/src/sca_ref.hpp:70-91). Spin slot
// i = k * 256 + l is decided by lane l in round k; every lane draws once per round, padding slots included.
//
// Decision (sca_ref.hpp:118-131): corr = ((n_lin_prev * kcorr_t) >> 8) + kconst_t;
//   z = s*h*65536 + q_t - (s == s_prev ? corr : -corr);  r = ((u16 - 32768) * fourT_t) >> 16 (floor);
//   flip iff z < r;  n_lin counts -2T < z < 2T with 2T = fourT >> 1.
// The engines evaluate z in int32 with hs = s*h (clamped to +-hclamp when the host range plan asks for it); the host
// proves |hs| * 65536 + |q -/+ corr| + fourT < 2^31 for every step before launching.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace anc {

constexpr int kLanes = 256;

struct DevTables {
    const int32_t* fourT;
    const int32_t* q;
    const int64_t* kcorr;
    const int32_t* kconst;
    int S;
};

struct Xoshiro {
    uint32_t a, b, c, d;
};

__device__ __forceinline__ uint64_t splitmix64(uint64_t& x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ void rng_seed(Xoshiro& r, uint64_t seed, uint32_t trial, uint32_t lane) {
    uint64_t x = seed ^ (uint64_t(trial) << 20) ^ (uint64_t(lane) << 48) ^ 0x5CA0F00Dull;
    const uint64_t u = splitmix64(x), v = splitmix64(x);
    r.a = uint32_t(u);
    r.b = uint32_t(u >> 32);
    r.c = uint32_t(v);
    r.d = uint32_t(v >> 32);
    if (!(r.a | r.b | r.c | r.d)) r.a = 1;
}

__device__ __forceinline__ uint32_t rng_next(Xoshiro& r) {
    const uint32_t m = r.b * 5u;
    const uint32_t out = __funnelshift_l(m, m, 7) * 9u;
    const uint32_t t = r.b << 9;
    r.c ^= r.a;
    r.d ^= r.b;
    r.b ^= r.c;
    r.a ^= r.d;
    r.c ^= t;
    r.d = __funnelshift_l(r.d, r.d, 11);
    return out;
}

// r = floor((u16 - 32768) * fourT / 65536) for u16 = draw >> 16; |r| <= 2T fits int32.
__device__ __forceinline__ int32_t threshold16(uint32_t draw, int32_t fourT) {
    const int32_t a = int32_t(draw >> 16) - 32768;
    return int32_t((int64_t(a) * int64_t(fourT)) >> 16);
}

// corr_t in int64 then narrowed (the host range plan bounds it).
__device__ __forceinline__ int32_t step_corr(int32_t nlin_prev, int64_t kcorr, int32_t kconst) {
    return int32_t(((int64_t(nlin_prev) * kcorr) >> 8) + int64_t(kconst));
}

// Carry-save adder: three words in, sum and carry words out (each a single LOP3).
__device__ __forceinline__ void csa(uint32_t& sum, uint32_t& carry, uint32_t a, uint32_t b, uint32_t c) {
    const uint32_t u = a ^ b;
    sum = u ^ c;
    carry = (a & b) | (u & c);
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

}  // namespace anc
