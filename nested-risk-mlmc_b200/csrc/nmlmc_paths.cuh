// Path-simulated inner values of the portfolio sampler (portfolio_sampler.cpp:212-225, 470-604;
// gbm_approx.hpp:18-57) in the reference's real_t / double evaluation order, shared by both stream
// layouts: Rs is R_tau of the option's stock at this outer sample, and NZ supplies the inner
// sample's normals in draw order (nz.next()) — the reference's
// CORE streams (nmlmc_core.cu) or an inner sample's own OUTER counter namespace
// (nmlmc_outer_impl.cuh).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "nmlmc_common.cuh"

namespace nmlmc {

template <class RT>
__device__ __forceinline__ RT opt_diff_stock(const OptionTable<RT>& ot, uint32_t j, RT S0_T, RT St_T) {
    // option_diff_from_stock (portfolio_sampler.cpp:212-219)
    const RT mod = (RT)ot.type[j], K = ot.strike[j];
    const RT a = xmul(mod, xsub(S0_T, K)), b = xmul(mod, xsub(St_T, K));
    const RT start = a > (RT)0 ? a : (RT)0, finish = b > (RT)0 ? b : (RT)0;
    return xmul(xmul(ot.w[j], xexp(xmul(-ot.r, ot.maturity[j]))), xsub(start, finish));
}

template <class RT>
__device__ __forceinline__ RT opt_derv_stock(const OptionTable<RT>& ot, uint32_t j, RT St_T, RT S0) {
    // option_derv_from_stock (portfolio_sampler.cpp:221-225)
    const RT df = (RT)((ot.type[j] == 1 ? 1 : 0) - (St_T < ot.strike[j] ? 1 : 0));
    return xmul(xmul(xmul(ot.w[j], xdiv(St_T, S0)), xexp(xmul(-ot.r, ot.maturity[j]))), df);
}

// simulate_stock_dt<with_coarse> (gbm_approx.hpp:18-57) on the three paths S[0..3) of
// sample_inner_approx, plus (with_coarse) the coupled coarse paths S[3..6) stepping every
// coarse_step fine steps on the summed increments.  States in double, increments in real_t.
template <class RT, class NZ>
__device__ void stock_dt(NZ& nz, double* S, uint64_t N, RT mu, RT sigma, RT t, bool milstein,
                         bool with_coarse, uint32_t coarse_step) {
    const RT dt = xdiv(t, (RT)N);
    const RT sqrt_dt = xsqrt(dt);
    const RT dt_c = xdiv(t, (RT)(N / coarse_step));
    const double hs2 = __dmul_rn(0.5, (double)xmul(sigma, sigma));
    const RT mudt = xmul(mu, dt), mudt_c = xmul(mu, dt_c);
    RT dW_c = (RT)0;
    for (uint64_t n = 0; n < N; n++) {
        const RT dW = xmul(sqrt_dt, nz.next());
        const RT m = milstein ? to_rt<RT>(__dmul_rn(hs2, (double)xsub(xmul(dW, dW), dt))) : (RT)0;
        const double inc = (double)xadd(xadd(mudt, xmul(sigma, dW)), m);
#pragma unroll
        for (int i = 0; i < 3; i++) S[i] = __dadd_rn(S[i], __dmul_rn(S[i], inc));
        if (with_coarse) {
            dW_c = xadd(dW_c, dW);
            if ((n + 1) % coarse_step == 0) {
                const RT mc = milstein ? to_rt<RT>(__dmul_rn(hs2, (double)xsub(xmul(dW_c, dW_c), dt_c))) : (RT)0;
                const double incc = (double)xadd(xadd(mudt_c, xmul(sigma, dW_c)), mc);
#pragma unroll
                for (int i = 3; i < 6; i++) S[i] = __dadd_rn(S[i], __dmul_rn(S[i], incc));
                dW_c = (RT)0;
            }
        }
    }
}

// sample_inner_exact (portfolio_sampler.cpp:470-519): exact GBM from tau to maturity for the
// antithetic pair started at S0 and for the path started at R_tau.
template <class RT, class NZ>
__device__ RT inner_exact(const OptionTable<RT>& ot, RT Rs, uint32_t j, NZ& nz, double& work) {
    const bool anti = ot.use_antithetic_risk != 0;
    work += (double)ot.W_est[j];
    const uint32_t s = ot.stock_ind[j];
    const RT S0 = ot.S0[s], sg = ot.sigma[s], r = ot.r, tau = ot.tau;
    const RT Tr = xsub(ot.maturity[j], tau);
    const RT dW_0_tau = xmul(ot.stau, nz.next());
    const RT dW_tau_T = xmul(xsqrt(Tr), nz.next());
    const RT S0_t_1 = simulate_stock_ref<RT>(S0, r, sg, tau, dW_0_tau);
    const RT S0_T_1 = simulate_stock_ref<RT>(S0_t_1, r, sg, Tr, dW_tau_T);
    RT S0_T_2 = (RT)0;
    if (anti) {
        const RT S0_t_2 = simulate_stock_ref<RT>(S0, r, sg, tau, -dW_0_tau);
        S0_T_2 = simulate_stock_ref<RT>(S0_t_2, r, sg, Tr, dW_tau_T);
    }
    const RT St_T = simulate_stock_ref<RT>(Rs, r, sg, Tr, dW_tau_T);
    const RT v1 = opt_diff_stock(ot, j, S0_T_1, St_T);
    const RT v2 = anti ? opt_diff_stock(ot, j, S0_T_2, St_T) : v1;
    RT d1 = (RT)0, d2 = (RT)0;
    if (ot.use_delta_cv) {
        const RT diff = xsub(Rs, S0);
        d1 = xmul(diff, opt_derv_stock(ot, j, S0_T_1, S0));
        d2 = anti ? xmul(diff, opt_derv_stock(ot, j, S0_T_2, S0)) : d1;
    }
    return to_rt<RT>(__dmul_rn(0.5, (double)xadd(xadd(xadd(v1, v2), d1), d2)));
}

// sample_inner_approx (portfolio_sampler.cpp:539-604): fine level L with N = h0 beta^L steps
// and, for L > 0, the coupled coarse level; payoff differences of the antithetic pair.
template <class RT, class NZ>
__device__ RT inner_approx(const OptionTable<RT>& ot, RT Rs, uint32_t j, NZ& nz, double& work,
                           uint32_t L, uint64_t N_l) {
    const uint32_t s = ot.stock_ind[j];
    const RT S0 = ot.S0[s], sg = ot.sigma[s], r = ot.r, tau = ot.tau;
    const RT dW = xmul(ot.stau, nz.next());
    const RT S0_t_1 = simulate_stock_ref<RT>(S0, r, sg, tau, dW);
    const RT S0_t_2 = simulate_stock_ref<RT>(S0, r, sg, tau, -dW);
    const uint64_t N = (uint64_t)ot.dt_h0inv * N_l;
    work += (double)xmul((RT)N_l, ot.W_est[j]);
    double S[6] = {(double)S0_t_1, (double)Rs, (double)S0_t_2, (double)S0_t_1, (double)Rs, (double)S0_t_2};
    const RT Tr = xsub(ot.maturity[j], tau);
    if (L) {
        stock_dt<RT, NZ>(nz, S, N, r, sg, Tr, ot.use_milstein != 0, true, ot.dt_beta);
        work += (double)xmul((RT)(N_l / ot.dt_beta), ot.W_est[j]);
    } else {
        stock_dt<RT, NZ>(nz, S, N, r, sg, Tr, ot.use_milstein != 0, false, 2);
    }
    const bool anti = ot.use_antithetic_risk != 0;
    const RT m = anti ? (RT)0.5 : (RT)1;
    const RT diff = xsub(Rs, S0);
    const bool do_d_f = ot.use_delta_cv && (ot.use_coarse_delta_cv || L == 0);
    const bool do_d_c = ot.use_delta_cv && ot.use_coarse_delta_cv;
    RT vf = 0, vc = 0, vdf = 0, vdc = 0;
    for (int i = 0; i < (anti ? 2 : 1); i++) {
        const int ic = 2 * i;
        vf = xadd(vf, xmul(m, opt_diff_stock(ot, j, to_rt<RT>(S[ic]), to_rt<RT>(S[1]))));
        if (do_d_f) vdf = xadd(vdf, xmul(m, opt_derv_stock(ot, j, to_rt<RT>(S[ic]), S0)));
        if (L == 0) continue;
        vc = xadd(vc, xmul(m, opt_diff_stock(ot, j, to_rt<RT>(S[ic + 3]), to_rt<RT>(S[4]))));
        if (do_d_c) vdc = xadd(vdc, xmul(m, opt_derv_stock(ot, j, to_rt<RT>(S[ic + 3]), S0)));
    }
    return xadd(xsub(vf, vc), xmul(diff, xsub(vdf, vdc)));
}

// Level of sample_inner_unbiased (portfolio_sampler.cpp:521-537) from its randu_sync value u:
// L = floor(log u / (log beta * e)), P(L) proportional to beta^(e L).  Returns false (and
// n_steps = 0) when h0 beta^L exceeds NMLMC_MAX_PATH_STEPS.
template <class RT>
__device__ __forceinline__ bool unbiased_level(const OptionTable<RT>& ot, RT u, uint32_t& L, uint64_t& N_l) {
    const RT e = ot.dt_prob_expo, x = (RT)ot.dt_beta;
    const RT q = xdiv(xlog(u), xmul(xlog(x), e));
    const RT fl = sizeof(RT) == 4 ? (RT)floorf((float)q) : (RT)floor((double)q);
    L = (uint32_t)fl;
    N_l = 1;
    for (uint32_t i = 0; i < L; i++) {
        N_l *= ot.dt_beta;
        if (N_l * ot.dt_h0inv > kMaxPathSteps) return false;
    }
    return N_l * ot.dt_h0inv <= kMaxPathSteps;
}

template <class RT, class NZ>
__device__ __forceinline__ RT inner_unbiased(const OptionTable<RT>& ot, RT Rs, uint32_t j, NZ& nz,
                                             double& work, uint32_t L, uint64_t N_l) {
    const RT ret = inner_approx<RT, NZ>(ot, Rs, j, nz, work, L, N_l);
    const RT e = ot.dt_prob_expo, x = (RT)ot.dt_beta;
    const RT Lp = to_rt<RT>(__ddiv_rn((double)xpow(x, xmul(-e, (RT)L)), __dsub_rn(1.0, (double)xpow(x, e))));
    return xmul(ret, Lp);
}

// ---- FP32 versions for the batched fast path -------------------------------------------------
// The same estimators with float arithmetic and SFU exponentials (__expf, exp2f), the path states
// still in double (the reference keeps them in sum_t: float states drift over long paths,
// portfolio_sampler.cpp:559-560), the discount e^{-r T} computed once per sample, and the
// Unbiased level's weight beta^{-e L} / (1 - beta^e) without a double pow.  The level L itself is
// computed in double as on the FP64 path, so both precisions step the same number of steps.

// simulate_stock_dt<with_coarse> (gbm_approx.hpp:18-57) in float increments.
template <class NZ>
__device__ void stock_dt_fast(NZ& nz, double* S, uint64_t N, float mu, float sigma, float t, bool milstein,
                              bool with_coarse, uint32_t coarse_step) {
    const float dt = t / (float)N;
    const float sqrt_dt = sqrtf(dt);
    const float dt_c = dt * (float)coarse_step;
    const float hs2 = milstein ? 0.5f * sigma * sigma : 0.f;
    float dW_c = 0.f;
    for (uint64_t n = 0; n < N; n++) {
        const float dW = sqrt_dt * nz.next();
        const double inc = (double)fmaf(hs2, fmaf(dW, dW, -dt), fmaf(sigma, dW, mu * dt));
#pragma unroll
        for (int i = 0; i < 3; i++) S[i] = fma(S[i], inc, S[i]);
        if (with_coarse) {
            dW_c += dW;
            if ((n + 1) % coarse_step == 0) {
                const double incc = (double)fmaf(hs2, fmaf(dW_c, dW_c, -dt_c), fmaf(sigma, dW_c, mu * dt_c));
#pragma unroll
                for (int i = 3; i < 6; i++) S[i] = fma(S[i], incc, S[i]);
                dW_c = 0.f;
            }
        }
    }
}

// w e^{-r T} (max(m (S0_T - K), 0) - max(m (St_T - K), 0)) (option_diff_from_stock, 212-219)
__device__ __forceinline__ float opt_diff_stock_fast(float wdisc, float m, float K, float S0_T, float St_T) {
    return wdisc * (fmaxf(m * (S0_T - K), 0.f) - fmaxf(m * (St_T - K), 0.f));
}
// w (St_T / S0) e^{-r T} (1{call} - 1{St_T < K}) (option_derv_from_stock, 221-225)
__device__ __forceinline__ float opt_derv_stock_fast(float wdisc, bool call, float K, float St_T, float S0) {
    return wdisc * (St_T / S0) * (float)((call ? 1 : 0) - (St_T < K ? 1 : 0));
}

template <class NZ>
__device__ float inner_exact_fast(const OptionTable<float>& ot, float Rs, uint32_t j, NZ& nz, double& work) {
    const bool anti = ot.use_antithetic_risk != 0;
    work += (double)ot.W_est[j];
    const uint32_t s = ot.stock_ind[j];
    const float S0 = ot.S0[s], sg = ot.sigma[s], r = ot.r, tau = ot.tau, T = ot.maturity[j], K = ot.strike[j];
    const float m = (float)ot.type[j], Tr = T - tau, wdisc = ot.w[j] * __expf(-r * T);
    const float mu_t = (r - 0.5f * sg * sg) * tau, mu_T = (r - 0.5f * sg * sg) * Tr;
    const float dW_0_tau = ot.stau * nz.next();
    const float dW_tau_T = sqrtf(Tr) * nz.next();
    const float gT = __expf(fmaf(sg, dW_tau_T, mu_T));
    const float S0_T_1 = S0 * __expf(fmaf(sg, dW_0_tau, mu_t)) * gT;
    const float S0_T_2 = anti ? S0 * __expf(fmaf(-sg, dW_0_tau, mu_t)) * gT : 0.f;
    const float St_T = Rs * gT;
    const float v1 = opt_diff_stock_fast(wdisc, m, K, S0_T_1, St_T);
    const float v2 = anti ? opt_diff_stock_fast(wdisc, m, K, S0_T_2, St_T) : v1;
    float d1 = 0.f, d2 = 0.f;
    if (ot.use_delta_cv) {
        const float diff = Rs - S0;
        d1 = diff * opt_derv_stock_fast(wdisc, m > 0.f, K, S0_T_1, S0);
        d2 = anti ? diff * opt_derv_stock_fast(wdisc, m > 0.f, K, S0_T_2, S0) : d1;
    }
    return 0.5f * (v1 + v2 + d1 + d2);
}

template <class NZ>
__device__ float inner_approx_fast(const OptionTable<float>& ot, float Rs, uint32_t j, NZ& nz, double& work,
                                   uint32_t L, uint64_t N_l) {
    const uint32_t s = ot.stock_ind[j];
    const float S0 = ot.S0[s], sg = ot.sigma[s], r = ot.r, tau = ot.tau, T = ot.maturity[j], K = ot.strike[j];
    const float m = (float)ot.type[j], wdisc = ot.w[j] * __expf(-r * T);
    const float mu_t = (r - 0.5f * sg * sg) * tau;
    const float dW = ot.stau * nz.next();
    const float S0_t_1 = S0 * __expf(fmaf(sg, dW, mu_t));
    const float S0_t_2 = S0 * __expf(fmaf(-sg, dW, mu_t));
    const uint64_t N = (uint64_t)ot.dt_h0inv * N_l;
    const float West = ot.W_est[j];
    work += (double)((float)N_l * West);
    double S[6] = {(double)S0_t_1, (double)Rs, (double)S0_t_2, (double)S0_t_1, (double)Rs, (double)S0_t_2};
    const float Tr = T - tau;
    if (L) {
        stock_dt_fast<NZ>(nz, S, N, r, sg, Tr, ot.use_milstein != 0, true, ot.dt_beta);
        work += (double)((float)(N_l / ot.dt_beta) * West);
    } else {
        stock_dt_fast<NZ>(nz, S, N, r, sg, Tr, ot.use_milstein != 0, false, 2);
    }
    const bool anti = ot.use_antithetic_risk != 0;
    const float half = anti ? 0.5f : 1.f;
    const float diff = Rs - S0;
    const bool do_d_f = ot.use_delta_cv && (ot.use_coarse_delta_cv || L == 0);
    const bool do_d_c = ot.use_delta_cv && ot.use_coarse_delta_cv;
    float vf = 0.f, vc = 0.f, vdf = 0.f, vdc = 0.f;
#pragma unroll
    for (int i = 0; i < 2; i++) {
        if (i == 1 && !anti) break;
        const int ic = 2 * i;
        vf += half * opt_diff_stock_fast(wdisc, m, K, (float)S[ic], (float)S[1]);
        if (do_d_f) vdf += half * opt_derv_stock_fast(wdisc, m > 0.f, K, (float)S[ic], S0);
        if (L == 0) continue;
        vc += half * opt_diff_stock_fast(wdisc, m, K, (float)S[ic + 3], (float)S[4]);
        if (do_d_c) vdc += half * opt_derv_stock_fast(wdisc, m > 0.f, K, (float)S[ic + 3], S0);
    }
    return (vf - vc) + diff * (vdf - vdc);
}

// sample_inner_unbiased (521-537): ret * beta^{-e L} / (1 - beta^e), the weight in float
template <class NZ>
__device__ __forceinline__ float inner_unbiased_fast(const OptionTable<float>& ot, float Rs, uint32_t j, NZ& nz,
                                                     double& work, uint32_t L, uint64_t N_l) {
    const float ret = inner_approx_fast<NZ>(ot, Rs, j, nz, work, L, N_l);
    const float e = ot.dt_prob_expo, lb = __log2f((float)ot.dt_beta);
    return ret * (exp2f(-e * lb * (float)L) / (1.0f - exp2f(e * lb)));
}

}  // namespace nmlmc
