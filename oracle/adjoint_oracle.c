/* CPU oracle of the path-simulated portfolio loss — TEST INFRASTRUCTURE ONLY.
 *
 * Restates, in double and one sample at a time, the estimator the GPU library's adjoint module
 * computes (see the header of nested-risk-mlmc_b200/csrc/nmlmc_adjoint.cu for its definition):
 * the outer draw of portfolio_sampler.cpp:293-311 on the OUTER stream layout, antithetic
 * Milstein / Euler inner paths (gbm_approx.hpp:18-57 with risk-neutral drift) on 2^ell steps
 * from tau to each option's maturity, and the loss L = sum_i w_i (V_i(0) - e^{-r tau} C_i).
 * Gradients are checked against central differences of this function with common random
 * numbers (the same seed for both sides).  Parity of the path recursion is pinned to the
 * reference through the golden cases of the Exact / Unbiased methods (same gbm_approx step);
 * this batched estimator itself has no reference counterpart.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#include "nmlmc_oracle.h"

#define PH_OUTER_TAG 0u
#define PH_ADJOINT_TAG 200u

/* Box-Muller on two 32-bit words in double (the OUTER layout's normal pair). */
static void bm32d(uint32_t u0, uint32_t u1, double *x, double *y) {
    const double PI = 3.1415926535897932;
    double a = (double)(int32_t)u0 * 0x1p-31 + 0x1p-32;
    double u = (double)u1 * 0x1p-32 + 0x1p-33;
    double s = sin(PI * a), c = cos(PI * a);
    double r = sqrt(-2.0 * log(u));
    *x = s * r;
    *y = c * r;
}

static void normals4(uint64_t c0, uint64_t c1, const uint64_t key[2], double z[4]) {
    uint64_t ctr[2] = {c0, c1}, v[2];
    o_threefry2x64(ctr, key, v);
    bm32d((uint32_t)v[0], (uint32_t)(v[0] >> 32), &z[0], &z[1]);
    bm32d((uint32_t)v[1], (uint32_t)(v[1] >> 32), &z[2], &z[3]);
}

static double norm_cdf(double x) { return 0.5 * erfc(-x / sqrt(2.0)); }

static double bs_price(int type, double S0, double K, double r, double T, double sg) {
    double d1 = (log(S0 / K) + (r + 0.5 * sg * sg) * T) / (sg * sqrt(T));
    double d2 = d1 - sg * sqrt(T);
    return type * S0 * norm_cdf(type * d1) - type * K * exp(-r * T) * norm_cdf(type * d2);
}

/* L[p * M + m] for every portfolio of the batch. */
void o_adj_loss(uint32_t n, const uint32_t *stock_off, const uint32_t *option_off, const double *S0,
                const double *mu, const double *sigma, const double *strike, const double *maturity,
                const double *w, const uint32_t *stock_ind, const int32_t *type, double r, double rho,
                double tau, uint32_t ell, uint32_t pairs, uint64_t M, uint64_t seed, int milstein,
                double *L) {
    const double stau = sqrt(tau), s1_rho2 = sqrt(1 - rho * rho), disc_tau = exp(-r * tau);
    const uint32_t steps = 1u << ell;
    for (uint32_t p = 0; p < n; p++) {
        const uint32_t s0 = stock_off[p], Q = stock_off[p + 1] - s0;
        const uint32_t o0 = option_off[p], P = option_off[p + 1] - o0;
        double *R = (double *)malloc(Q * sizeof(double));
        for (uint64_t m = 0; m < M; m++) {
            const uint64_t key[2] = {seed, ((uint64_t)ell << 56) | ((uint64_t)p << 32) | (m & 0xffffffffull)};
            /* outer draw: normal 0 systemic, 1 + j per stock (a single stock takes normal 0) */
            const uint32_t nnorm = Q == 1 ? 1 : Q + 1;
            double dW_sys = 0, z[4];
            for (uint32_t k = 0; k < nnorm; k++) {
                if ((k & 3) == 0) normals4(k >> 2, PH_OUTER_TAG, key, z);
                if (k == 0) {
                    dW_sys = stau * z[0];
                    if (Q > 1) continue;
                }
                const uint32_t j = Q == 1 ? 0 : k - 1;
                const double W = Q == 1 ? dW_sys : rho * dW_sys + s1_rho2 * (stau * z[k & 3]);
                const double sg = sigma[s0 + j];
                R[j] = S0[s0 + j] * exp(sg * W + (mu[s0 + j] - 0.5 * sg * sg) * tau);
            }
            double Lm = 0;
            for (uint32_t il = 0; il < P; il++) {
                const uint32_t i = o0 + il, s = stock_ind[i];
                const double K = strike[i], T = maturity[i], sg = sigma[s0 + s], ty = (double)type[i];
                const double Tr = T - tau, h = Tr / (double)steps, sh = sqrt(h);
                const uint64_t c1 = ((uint64_t)il << 32) | PH_ADJOINT_TAG;
                double C = 0;
                uint64_t q = 0;
                for (uint32_t nn = 0; nn < pairs; nn++) {
                    double Sp = R[s], Sm = R[s];
                    for (uint32_t k = 0; k < steps; k++, q++) {
                        if ((q & 3) == 0) normals4(q >> 2, c1, key, z);
                        const double dW = sh * z[q & 3];
                        const double corr = milstein ? 0.5 * sg * sg * (dW * dW - h) : 0.0;
                        Sp *= 1 + r * h + sg * dW + corr;
                        Sm *= 1 + r * h - sg * dW + corr;
                    }
                    const double xp = ty * (Sp - K), xm = ty * (Sm - K);
                    C += 0.5 * ((xp > 0 ? xp : 0) + (xm > 0 ? xm : 0));
                }
                C *= exp(-r * Tr) / (double)pairs;
                const double V0 = bs_price(type[i], S0[s0 + s], K, r, T, sg);
                Lm += w[i] * (V0 - disc_tau * C);
            }
            L[(size_t)p * M + m] = Lm;
        }
        free(R);
    }
}
