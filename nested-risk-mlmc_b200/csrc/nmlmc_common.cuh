// Shared device-side definitions of the level sampler: exactly-rounded arithmetic helpers,
// the parameter blocks handed to the kernels, trace records and the per-level adaptive
// count parameters.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "nmlmc_bs.cuh"
#include "nmlmc_rng.cuh"

namespace nmlmc {

// Per-outer-sample record (same layout as the CPU oracle's o_trace_rec).
struct TraceRec {
    uint64_t count_f, count_c;
    double phi_f, phi_c;
    double mean_big, min_abs_small;
    uint32_t core, pilots;
};
static_assert(sizeof(TraceRec) == 56, "trace record layout");

// Adaptive inner-count parameters of one level (get_samples_count ctor,
// nested_sampler.hpp:225-239), evaluated on the host with the same libm calls as the
// reference so tmp is bit-identical.
struct CountParams {
    uint64_t max_count, base_count;
    double tmp;          // real_t value widened
};

// Sampler kinds: the reference's model, the X = Y + Z model, the portfolio, a caller-written
// SAMPLER class (include/nmlmc_sampler.cuh), and — on the batched layout only — the portfolio
// with path-simulated (Exact / Unbiased) options, a kernel instantiation of its own so that the
// Black-Scholes-only kernels carry none of the path code.
enum Kind : int { KIND_REF_MODEL = 0, KIND_SHIFT_MODEL = 1, KIND_PORTFOLIO = 2, KIND_USER = 3, KIND_PF_PATHS = 4 };
__host__ __device__ constexpr bool is_portfolio_kind(int kind) {
    return kind == KIND_PORTFOLIO || kind == KIND_PF_PATHS;
}
enum Sub : int { SUB_NONE = 0, SUB_RANDOM = 1, SUB_UNIFORM = -1 };

enum Method : int { METHOD_BS = 0, METHOD_EXACT = 1, METHOD_UNBIASED = 2 };

// Time steps one path-simulated inner sample may take (h0 beta^L of the Unbiased method); a
// draw above it stops the call with NMLMC_ERR_LIMIT instead of running unbounded.
constexpr uint64_t kMaxPathSteps = 1ull << 24;

// Option table in HBM, structure of arrays.  Options are grouped by compute method
// (portfolio::data::options[3], portfolio_sampler.cpp:62-92): method m occupies
// [m_off[m], m_off[m] + m_n[m]) and its CDF restarts at 0.
template <class RT>
struct OptionTable {
    const RT* strike;
    const RT* maturity;
    const RT* start;       // V0 (portfolio_comp_params)
    const RT* w;
    const RT* prob;
    const RT* W_est;
    const RT* cdf;         // per-method CDF of prob (portfolio_update_data)
    const uint32_t* stock_ind;
    const int8_t* type;    // +1 call, -1 put
    // stocks
    const RT* S0;
    const RT* mu;
    const RT* sigma;
    const RT* delta_coalesce;
    const struct FastOption* fast;   // FP32 path: packed records (nmlmc_bs.cuh), else nullptr
    const struct FastOption* fast_s; // the same records scaled by 1 / (sampling probability)
    const uint2* alias;              // OUTER Subsampling::Random: alias table {threshold, alias}
    const struct FastColumn* fast_col; // FP32 path, Subsampling::Random: records fused with the
                                       // alias table (nmlmc_bs.cuh), or nullptr
    const RT* phat;                  // sampling probability of each option under the alias table
    uint32_t P, Q;
    RT r, rho, s1_rho2, max_loss, tau, stau, prob_norm, compute_prob0, inv_count_prob;
    int subsample, use_delta_cv, discount;
    // compute methods and the path-simulated inner values (portfolio_sampler.cpp:74-87)
    uint32_t m_off[3], m_n[3];
    RT compute_prob[3];
    int mixed;                       // an Exact or Unbiased option is present
    uint32_t dt_h0inv, dt_beta;
    RT dt_prob_expo;
    int use_coarse_delta_cv, use_antithetic_risk, use_milstein;
};

template <class RT>
struct ModelParams {
    RT stau, s1tau, max_loss;
};

#ifdef __CUDACC__
// ---- exactly rounded arithmetic (no FMA contraction), overloaded on float / double ---------
__device__ __forceinline__ float xadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float xsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float xmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float xdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double xdiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float xsqrt(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ double xsqrt(double a) { return __dsqrt_rn(a); }
__device__ __forceinline__ float xlog(float a) { return logf(a); }
__device__ __forceinline__ double xlog(double a) { return log(a); }
__device__ __forceinline__ float xexp(float a) { return expf(a); }
__device__ __forceinline__ double xexp(double a) { return exp(a); }
__device__ __forceinline__ float xerfc(float a) { return erfcf(a); }
__device__ __forceinline__ double xerfc(double a) { return erfc(a); }
__device__ __forceinline__ float xceil(float a) { return ceilf(a); }
__device__ __forceinline__ double xceil(double a) { return ceil(a); }
template <class RT> __device__ __forceinline__ RT to_rt(double v);
template <> __device__ __forceinline__ float to_rt<float>(double v) { return __double2float_rn(v); }
template <> __device__ __forceinline__ double to_rt<double>(double v) { return v; }
// powf of the reference evaluated as a correctly rounded double pow narrowed to real_t.
__device__ __forceinline__ float xpow(float a, float b) { return __double2float_rn(pow((double)a, (double)b)); }
__device__ __forceinline__ double xpow(double a, double b) { return pow(a, b); }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
    return v;
}
__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v) {
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
    return v;
}

// ---- Black-Scholes in the reference's real_t evaluation order (portfolio_sampler.cpp) -------
template <class RT>
__device__ __forceinline__ RT norm_cdf_ref(RT x) {                 // common.hpp:201-202
    const RT SQRT_2 = (RT)1.414213562373095;
    return to_rt<RT>(__dmul_rn(0.5, (double)xerfc(xdiv(-x, SQRT_2))));
}

template <class RT>
__device__ __forceinline__ RT simulate_stock_ref(RT S0, RT mu, RT sigma, RT t, RT dW) {  // :136-138
    double e = __dadd_rn((double)xmul(sigma, dW),
                         __dmul_rn(__dsub_rn((double)mu, __dmul_rn(__dmul_rn(0.5, (double)sigma), (double)sigma)),
                                   (double)t));
    return to_rt<RT>(__dmul_rn((double)S0, exp(e)));
}

template <class RT>
__device__ __forceinline__ RT bs_d1_ref(RT S0, RT strike, RT r, RT t, RT sigma) {
    RT v1 = xlog(xdiv(S0, strike));
    RT v2 = to_rt<RT>(__dmul_rn(__dadd_rn((double)r, __ddiv_rn((double)xmul(sigma, sigma), 2.0)), (double)t));
    RT v3 = xmul(sigma, xsqrt(t));
    return xdiv(xadd(v1, v2), v3);
}

template <class RT>
__device__ __forceinline__ RT calc_bs_ref(int type, RT S0, RT strike, RT r, RT t, RT sigma) {  // :140-150
    RT d1 = bs_d1_ref(S0, strike, r, t, sigma);
    RT d2 = xsub(d1, xmul(sigma, xsqrt(t)));
    RT mod = (RT)type;
    RT a = xmul(xmul(mod, S0), norm_cdf_ref(xmul(mod, d1)));
    RT b = xmul(xmul(xmul(mod, strike), xexp(xmul(-r, t))), norm_cdf_ref(xmul(mod, d2)));
    return xsub(a, b);
}

template <class RT>
__device__ __forceinline__ RT calc_delta_ref(int type, RT S0, RT strike, RT r, RT t, RT sigma) {  // :152-160
    RT d1 = bs_d1_ref(S0, strike, r, t, sigma);
    return xsub(norm_cdf_ref(d1), (RT)(type == -1 ? 1 : 0));
}
#endif  // __CUDACC__

}  // namespace nmlmc
