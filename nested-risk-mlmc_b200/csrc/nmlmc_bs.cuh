// FP32 Black-Scholes on the SFU for the batched portfolio path.
//
// The loss of option i at the outer sample Y (option_diff_from_blackscholes and the delta control
// variate of sample_inner_bs, portfolio_sampler.cpp:186-210, 453-468) is regrouped so that all
// per-option constants are folded on the host (in double, then rounded once):
//
//   m d1 = (ln R + c1) * (m inv_s),   m d2 = m d1 - m s,   m = +1 call / -1 put
//   V  = m (R Phi(m d1) - K e^{-r(T-tau)} Phi(m d2))          (BS at tau, remaining time T - tau)
//   loss_i = w V0 - w e^{-r tau} V  +  cv (R - S0)            (cv = w Delta_BS(S0, T) when the
//                                                             delta control variate is on)
// with c1 = -ln K + (r + sigma^2/2)(T - tau), s = sigma sqrt(T - tau), inv_s = 1/s.  The record
// stores the signed m inv_s and m s (the sign flip is exact, so m d1 and m d2 round exactly as
// d1 and d2 would), wR = -w e^{-r tau} m, wK = w e^{-r tau} m K e^{-r(T - tau)},
// wV0 = w V0 - cv S0 (the control variate's constant folded in) and cv, so one inner sample needs
// no per-stock data but R and ln R of its stock at this outer sample.
//
// Phi(x) = erfc(-x/sqrt 2) / 2 with the rational-Chebyshev erfc of Numerical Recipes in C
// (2nd ed., §6.2, "erfcc": fractional error below 1.2e-7 for all arguments), its exponential and
// reciprocal on MUFU (ex2.approx, rcp.approx).  Measured against double erfc over |x| <= 10 the
// composite Phi has absolute error <= 2.1e-7 and, where Phi >= 1e-20, relative error <= 5e-6: in
// the far tail the FP32 rounding of the exponent (up to ~72 in base 2) dominates, not the erfc fit
// (tests/test_gpu_portfolio.py, bounds 2.5e-7 and 1e-5).
// The loss of one option is then within
// 1e-6 * (|wV0| + |wR R| + |wK| + |cv| (R + S0)) of the double-precision value.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace nmlmc {

// Packed option record of the FP32 path: 32 bytes, read with one 256-bit load.
struct __align__(32) FastOption {
    float c1, inv_s, s, wR;    // inv_s and s carry the call/put sign m
    float wK, wV0, cv;
    uint32_t stock;            // stock index
};
static_assert(sizeof(FastOption) == 32, "FastOption layout");

// Alias column of the FP32 path's importance sub-sampling (portfolios of at most 256 stocks and
// fewer than 2^24 options): option j's sampler record without s, which the kernel recomputes as
// 1 / inv_s, and column j of the alias table in the freed words — the coin threshold and the
// alias index, packed with the stock index (link = alias << 8 | stock).  A draw reads column j;
// only a coin at or above the threshold reads the alias column, so most inner samples need one
// 32-byte gather instead of an alias entry and then a record.
struct __align__(32) FastColumn {
    float c1, inv_s, wR, wK;
    float wV0, cv;
    uint32_t thr, link;
};
static_assert(sizeof(FastColumn) == 32, "FastColumn layout");
constexpr uint32_t kColumnMaxStocks = 256;
constexpr uint32_t kColumnMaxOptions = 1u << 24;

#ifdef __CUDACC__
// 1 / x from the SFU alone (PTX rcp.approx: relative error below 2^-23, normal x).
__device__ __forceinline__ float rcp_sfu(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// 2^x on the SFU (PTX ex2.approx; results below 2^-126 flush to zero).
__device__ __forceinline__ float ex2_sfu(float x) {
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Phi(x) for any x from h = Phi(-|x|) = erfc(z) / 2, z = |x| / sqrt 2, with the Numerical Recipes
// "erfcc" form erfc(z) = t exp(-z^2 + P(t)), t = 1 / (1 + z / 2).  The coefficients below are
// erfcc's times log2(e), the constant term also less 1 (the half), so that
// h = t 2^(P2(t) - |x|^2 log2(e) / 2) takes one SFU exponential and no further products.
__device__ __forceinline__ float norm_cdf_fast(float x) {
    const float a = fabsf(x);
    const float t = rcp_sfu(fmaf(a, 0.35355339f, 1.0f));    // 1 / (1 + |x| / (2 sqrt 2))
    float p = fmaf(t, 0.24651730f, -1.18611491f);
    p = fmaf(t, p, 2.14747453f);
    p = fmaf(t, p, -1.63775313f);
    p = fmaf(t, p, 0.40232158f);
    p = fmaf(t, p, -0.26875687f);
    p = fmaf(t, p, 0.13963005f);
    p = fmaf(t, p, 0.53970063f);
    p = fmaf(t, p, 1.44272923f);
    p = fmaf(t, p, -2.82574821f);
    const float h = t * ex2_sfu(fmaf(-a, a * 0.72134751f, p));
    return x >= 0.f ? 1.0f - h : h;
}

// loss_i(R) of one option (see the header comment); lnR = ln R of its stock at this outer sample.
__device__ __forceinline__ float option_loss_fast(const FastOption& o, float R, float lnR) {
    const float d1 = (lnR + o.c1) * o.inv_s;           // m d1
    const float d2 = d1 - o.s;                         // m d2
    const float n1 = norm_cdf_fast(d1), n2 = norm_cdf_fast(d2);
    const float v = fmaf(o.wR * R, n1, fmaf(o.wK, n2, o.wV0));
    return fmaf(o.cv, R, v);
}

// The same loss from an alias column: m d1 as above, m s = 1 / (m inv_s) from the SFU estimate
// (within one ulp of the record's m s, the only difference from option_loss_fast; one ulp of s
// moves Phi(d2) by less than 2e-8).
__device__ __forceinline__ float column_loss_fast(const FastColumn& c, float R, float lnR) {
    const float d1 = (lnR + c.c1) * c.inv_s;
    const float d2 = d1 - rcp_sfu(c.inv_s);
    const float n1 = norm_cdf_fast(d1), n2 = norm_cdf_fast(d2);
    const float v = fmaf(c.wR * R, n1, fmaf(c.wK, n2, c.wV0));
    return fmaf(c.cv, R, v);
}
#endif

}  // namespace nmlmc
