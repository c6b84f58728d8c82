// Counter-based random streams for the level sampler on sm_100a.
//
// Threefry2x64-20 (Random123/threefry.h:86-93 rotation constants, :171 parity constant,
// :190-286 rounds and key injections), bit-identical to the reference's r123::Threefry2x64, and
// the two ways the sampler addresses it:
//
//  * CORE layout — the reference CPU build's random_state (par_omp.hpp:72-121): key = (seed,
//    core), counter (b, 0) for the b-th block, 64-bit words consumed v[1] then v[0], so stream
//    word w is block(w >> 1).v[1 - (w & 1)].  A normal pair consumes two consecutive words; the
//    first word drawn is Box-Muller's u1 (radius) and the second its u0 (angle), the order g++
//    gives boxmuller(rand(), rand()) (par_omp.hpp:83).  Because every word has an address, the 32
//    lanes of a warp skip ahead to their own slice of a phase instead of drawing sequentially.
//  * OUTER layout — one key per outer sample (seed, level << 56 | outer index) and one counter
//    namespace per phase (counter = (block, phase tag)); each block gives four 32-bit words
//    [lo(v0), hi(v0), lo(v1), hi(v1)]; normal k of a phase comes from the pair of words
//    (2(k>>1), 2(k>>1)+1), uniform k from word k.  Independent of scheduling, so any thread may
//    evaluate any inner sample.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace nmlmc {

struct TfKey {
    uint64_t k0, k1, k2;   // k2 = parity ^ k0 ^ k1
};

__host__ __device__ __forceinline__ TfKey tf_key(uint64_t k0, uint64_t k1) {
    return TfKey{k0, k1, 0x1BD11BDAA9FC1A22ull ^ k0 ^ k1};
}

#ifdef __CUDACC__
template <int R>
__device__ __forceinline__ uint64_t rotl64c(uint64_t x) {
    uint32_t lo = (uint32_t)x, hi = (uint32_t)(x >> 32);
    if (R >= 32) { uint32_t t = lo; lo = hi; hi = t; }
    constexpr int r = R & 31;
    if (r == 0) return ((uint64_t)hi << 32) | lo;
    uint32_t nhi = __funnelshift_l(lo, hi, r);
    uint32_t nlo = __funnelshift_l(hi, lo, r);
    return ((uint64_t)nhi << 32) | nlo;
}

#define NMLMC_TF_ROUND(R)          \
    x0 += x1;                      \
    x1 = rotl64c<R>(x1);           \
    x1 ^= x0;

// One Threefry2x64-20 block: out = F(ctr = (c0, c1), key).
__device__ __forceinline__ void threefry2x64(uint64_t c0, uint64_t c1, const TfKey& k,
                                             uint64_t& o0, uint64_t& o1) {
    uint64_t x0 = c0 + k.k0, x1 = c1 + k.k1;
    NMLMC_TF_ROUND(16) NMLMC_TF_ROUND(42) NMLMC_TF_ROUND(12) NMLMC_TF_ROUND(31)
    x0 += k.k1; x1 += k.k2 + 1;
    NMLMC_TF_ROUND(16) NMLMC_TF_ROUND(32) NMLMC_TF_ROUND(24) NMLMC_TF_ROUND(21)
    x0 += k.k2; x1 += k.k0 + 2;
    NMLMC_TF_ROUND(16) NMLMC_TF_ROUND(42) NMLMC_TF_ROUND(12) NMLMC_TF_ROUND(31)
    x0 += k.k0; x1 += k.k1 + 3;
    NMLMC_TF_ROUND(16) NMLMC_TF_ROUND(32) NMLMC_TF_ROUND(24) NMLMC_TF_ROUND(21)
    x0 += k.k1; x1 += k.k2 + 4;
    NMLMC_TF_ROUND(16) NMLMC_TF_ROUND(42) NMLMC_TF_ROUND(12) NMLMC_TF_ROUND(31)
    x0 += k.k2; x1 += k.k0 + 5;
    o0 = x0;
    o1 = x1;
}
#undef NMLMC_TF_ROUND

// ---- uniform conversions (Random123/uniform.hpp:144-180), rounding made explicit ------------
// u01<double>(uint64): in * 2^-64 + 2^-65 (the product is exact; one rounding in the add).
__device__ __forceinline__ double u01_d(uint64_t in) {
    return __dadd_rn(__dmul_rn(__ull2double_rn(in), 0x1p-64), 0x1p-65);
}
// u01<float>(uint64): (float)in * 2^-64 + 2^-65 in float.
__device__ __forceinline__ float u01_f(uint64_t in) {
    return __fadd_rn(__fmul_rn(__ull2float_rn(in), 0x1p-64f), 0x1p-65f);
}
// uneg11<double>(uint64): (int64)in * 2^-63 + 2^-64.
__device__ __forceinline__ double uneg11_d(uint64_t in) {
    return __dadd_rn(__dmul_rn(__ll2double_rn((long long)in), 0x1p-63), 0x1p-64);
}

// r123::boxmuller(uint64 u0, uint64 u1) in double with the CPU sincospi(x) = sincos(PI * x)
// (Random123/boxmuller.hpp:96-104, 128-137).
__device__ __forceinline__ void boxmuller64(uint64_t u0, uint64_t u1, double& x, double& y) {
    const double PI = 3.1415926535897932;
    double s, c;
    sincos(__dmul_rn(PI, uneg11_d(u0)), &s, &c);
    double r = sqrt(__dmul_rn(-2.0, log(u01_d(u1))));
    x = __dmul_rn(s, r);
    y = __dmul_rn(c, r);
}

// OUTER layout Box-Muller on two 32-bit words.
// Double: angle a = (int32)u0 * 2^-31 + 2^-32, radius sqrt(-2 log(u1 * 2^-32 + 2^-33)) — the same
// expressions as the CPU oracle.
__device__ __forceinline__ void boxmuller32_d(uint32_t u0, uint32_t u1, double& x, double& y) {
    const double PI = 3.1415926535897932;
    double a = __dadd_rn(__dmul_rn((double)(int32_t)u0, 0x1p-31), 0x1p-32);
    double u = __dadd_rn(__dmul_rn((double)u1, 0x1p-32), 0x1p-33);
    double s, c;
    sincos(__dmul_rn(PI, a), &s, &c);
    double r = sqrt(__dmul_rn(-2.0, log(u)));
    x = __dmul_rn(s, r);
    y = __dmul_rn(c, r);
}

// FP32 fast Box-Muller on the SFU: MUFU sin/cos of the angle pi*a (absolute error <= 2^-21.4 on
// [-pi, pi]; pi*a formed in one FMA from the word), MUFU lg2 for the log and MUFU rsqrt for the
// root.  Near u = 1 the MUFU log's absolute error (2^-22) would dominate the small radius, so
// there t = -2 ln(1 - q) is summed from its series in the exact complement
// q = 1 - u = (~u1 + 1/2) 2^-32: t = q (2 + q (1 + 2q/3)), whose truncation (q^4 / 2) is below
// 2^-20 of t for q < 1/64.  |z - z_double| <= 4e-6 over the whole range (checked against
// boxmuller32_d in the tests).
__device__ __forceinline__ void boxmuller32_f(uint32_t u0, uint32_t u1, float& x, float& y) {
    const float PI = 3.14159265358979f;
    const float th = fmaf((float)(int32_t)u0, PI * 0x1p-31f, PI * 0x1p-32f);
    const float u = fmaf((float)u1, 0x1p-32f, 0x1p-33f);
    const float q = fmaf((float)(~u1), 0x1p-32f, 0x1p-33f);
    float s, c;
    __sincosf(th, &s, &c);
    const float t_log = (-2.0f * 0.69314718055994531f) * __log2f(u);
    const float t_ser = q * fmaf(q, fmaf(q, 0.66666667f, 1.0f), 2.0f);
    const float t = (q < 0.015625f) ? t_ser : t_log;   // -2 ln u > 0: t_ser >= 2q >= 2^-32, t_log > 0.03
    const float r = t * rsqrtf(t);
    x = s * r;
    y = c * r;
}

// ---- OUTER layout addressing --------------------------------------------------------------
__device__ __forceinline__ uint64_t outer_stream_id(uint32_t ell, uint64_t idx) {
    return ((uint64_t)ell << 56) | (idx & ((1ull << 56) - 1));
}
#endif  // __CUDACC__

// Phase tags of the OUTER layout (counter word 1).
enum : uint32_t {
    PH_OUTER = 0,          // outer draws
    PH_FINE = 1,           // fine pilot k       -> 1 + k
    PH_COARSE = 64,        // coarse pilot k     -> 64 + k
    PH_FINAL = 128,        // final phi (antithetic groups, fine-only, non-antithetic fine)
    PH_FINAL_C = 129,      // non-antithetic coarse phi
    PH_ADJOINT = 200,      // inner paths of the path-simulated loss (option index in bits 32..63)
};

}  // namespace nmlmc
