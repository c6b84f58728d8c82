// Path-simulated portfolio loss with its adjoint, for a batch of portfolios in one launch.
//
// Per portfolio p and outer sample m (stream key (seed, ell<<56 | p<<32 | m), so a single
// portfolio at p = 0 draws exactly the outer samples of the OUTER layout):
//   R_tau,j  = S0_j exp(sigma_j W_j + (mu_j - sigma_j^2/2) tau),  W_j = rho W_sys + sqrt(1-rho^2) W_ind,j
//              (portfolio_sampler.cpp:293-311, normal 0 systemic, 1 + j per stock)
//   C_i(m)   = e^{-r (T_i - tau)} (1/N) sum_n (pay(S+_n) + pay(S-_n)) / 2, S+- an antithetic pair of
//              Milstein paths (gbm_approx.hpp:18-57, risk-neutral drift r) on 2^ell steps from
//              (tau, R_tau,s(i)) to T_i; pay(S) = max(type (S - K_i), 0)
//   L_m      = sum_i w_i (V_i(0) - e^{-r tau} C_i(m))
// Pass 1 sums L_m over the options; the weight kernel forms E[L], the sigmoid-smoothed
// P_delta = E[s((L - K)/delta)], the plain exceedance frequency and the adjoint weights
// dF/dL_m (1/M for E[L], s'(x)/(delta M) for P_delta); pass 2 recomputes every inner draw from
// the counter RNG (nothing is stored between the passes), carries dS/dsigma along each path
// (one scalar parameter per path, so the tangent costs what a reverse sweep would and needs no
// tape) and pulls the weights back to every option position w_i and stock volatility sigma_j.
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

#include "nmlmc_common.cuh"
#include "nmlmc_internal.h"

namespace nmlmc {

namespace {

constexpr int kAdjThreads = 128;

__device__ __forceinline__ uint64_t adj_stream_id(uint32_t ell, uint32_t p, uint64_t m) {
    return ((uint64_t)ell << 56) | ((uint64_t)p << 32) | (m & 0xffffffffull);
}

// Four normals of one Threefry block: Box-Muller on the words (v0 lo, v0 hi) and (v1 lo, v1 hi);
// SFU Box-Muller for float, the double one for double.
template <class RT>
__device__ __forceinline__ void normals4(uint64_t v0, uint64_t v1, RT* z) {
    if constexpr (sizeof(RT) == 4) {
        boxmuller32_f((uint32_t)v0, (uint32_t)(v0 >> 32), z[0], z[1]);
        boxmuller32_f((uint32_t)v1, (uint32_t)(v1 >> 32), z[2], z[3]);
    } else {
        boxmuller32_d((uint32_t)v0, (uint32_t)(v0 >> 32), z[0], z[1]);
        boxmuller32_d((uint32_t)v1, (uint32_t)(v1 >> 32), z[2], z[3]);
    }
}

template <class RT>
__device__ __forceinline__ RT rexp(RT x) {
    if constexpr (sizeof(RT) == 4) return expf(x); else return exp(x);
}

// ---- outer draws: R_tau and dR_tau/dsigma per (portfolio, outer sample, stock) ----------------
template <class RT>
__global__ void __launch_bounds__(256) k_adj_outer(AdjLaunch<RT> A) {
    const uint64_t total = (uint64_t)A.n * A.M;
    for (uint64_t id = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; id < total;
         id += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t p = (uint32_t)(id / A.M);
        const uint64_t m = id % A.M;
        const TfKey key = tf_key(A.seed, adj_stream_id(A.ell, p, m));
        const uint32_t s0 = A.stock_off[p], Q = A.stock_off[p + 1] - s0;
        RT* Rrow = A.R + (size_t)s0 * A.M + (size_t)m * Q;
        RT* Drow = A.dR + (size_t)s0 * A.M + (size_t)m * Q;
        const uint32_t nnorm = Q == 1 ? 1 : Q + 1;
        RT dW_sys = 0;
        for (uint32_t b = 0; 4 * b < nnorm; b++) {
            uint64_t v0, v1;
            threefry2x64(b, PH_OUTER, key, v0, v1);
            RT z[4];
            normals4<RT>(v0, v1, z);
            for (uint32_t q = 0; q < 4; q++) {
                const uint32_t k = 4 * b + q;
                if (k >= nnorm) break;
                if (k == 0) {
                    dW_sys = A.stau * z[0];
                    if (Q > 1) continue;
                }
                const uint32_t j = Q == 1 ? 0 : k - 1;
                const RT W = Q == 1 ? dW_sys : A.rho * dW_sys + A.s1_rho2 * (A.stau * z[q]);
                const RT sg = A.sigma[s0 + j];
                const RT R = A.S0[s0 + j] * rexp<RT>(sg * W + (A.mu[s0 + j] - (RT)0.5 * sg * sg) * A.tau);
                Rrow[j] = R;
                Drow[j] = R * (W - sg * A.tau);
            }
        }
    }
}

// ---- inner paths: pass 1 (GRAD = false) sums L_m, pass 2 (GRAD = true) pulls back dF/dL_m ----
template <class RT, bool GRAD>
__global__ void __launch_bounds__(kAdjThreads) k_adj_paths(AdjLaunch<RT> A) {
    extern __shared__ double adj_sh[];                  // [kMaxTile][warps] | 2 * Qmax (GRAD)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int warps = kAdjThreads / 32;
    // portfolio of this option chunk
    const uint32_t chunk = blockIdx.x;
    uint32_t p = 0;
    while (p + 1 < A.n && A.chunk_off[p + 1] <= chunk) p++;
    const uint32_t o0 = A.option_off[p], P = A.option_off[p + 1] - o0;
    const uint32_t s0 = A.stock_off[p], Q = A.stock_off[p + 1] - s0;
    const uint32_t il = (chunk - A.chunk_off[p]) * kAdjThreads + threadIdx.x;
    const bool valid = il < P;
    const uint32_t i = o0 + (valid ? il : 0);
    const uint64_t m0 = (uint64_t)blockIdx.y * A.tile;
    const uint64_t m1 = m0 + A.tile < A.M ? m0 + A.tile : A.M;

    double* gs_sh = adj_sh;                              // GRAD: [2][Q]
    if (GRAD) {
        for (uint32_t t = threadIdx.x; t < 2 * Q; t += blockDim.x) gs_sh[t] = 0;
        __syncthreads();
    }

    const uint32_t s = A.stock_ind[i];
    const RT K = A.strike[i], T = A.maturity[i], w = A.w[i];
    const RT type = (RT)A.type[i];
    const RT sg = A.sigma[s0 + s];
    const uint32_t steps = 1u << A.ell;
    const RT Tr = T - A.tau;
    const RT h = Tr / (RT)steps;
    const RT sh = sqrt(h);
    const RT rh1 = (RT)1 + A.r * h;
    const RT hs2 = (RT)0.5 * sg * sg;
    const RT disc_in = rexp<RT>(-A.r * Tr);
    const RT V0 = A.V0[i], vega = A.vega[i];
    const RT invN = (RT)1 / (RT)A.pairs;
    const uint64_t ctr1 = ((uint64_t)il << 32) | PH_ADJOINT;

    double gwE = 0, gwP = 0, gsE = 0, gsP = 0;
    for (uint64_t m = m0; m < m1; m++) {
        const TfKey key = tf_key(A.seed, adj_stream_id(A.ell, p, m));
        const size_t ridx = (size_t)s0 * A.M + (size_t)m * Q + s;
        const RT Rt = A.R[ridx];
        const RT Dt = GRAD ? A.dR[ridx] : (RT)0;
        RT Csum = 0, dCsum = 0;
        uint64_t q = 0;                                  // normal index of the (i, m) stream
        RT z[4];
        for (uint32_t n = 0; n < A.pairs; n++) {
            RT Sp = Rt, Sm = Rt, Dp = Dt, Dm = Dt;
            for (uint32_t k = 0; k < steps; k++, q++) {
                if ((q & 3) == 0) {
                    uint64_t v0, v1;
                    threefry2x64(q >> 2, ctr1, key, v0, v1);
                    normals4<RT>(v0, v1, z);
                }
                const uint32_t e = (uint32_t)(q & 3);       // select, not a dynamic index
                const RT zq = e == 0 ? z[0] : (e == 1 ? z[1] : (e == 2 ? z[2] : z[3]));
                const RT dW = sh * zq;
                const RT corr = A.milstein ? hs2 * (dW * dW - h) : (RT)0;
                const RT gp = rh1 + sg * dW + corr, gm = rh1 - sg * dW + corr;
                if (GRAD) {
                    const RT dc = A.milstein ? sg * (dW * dW - h) : (RT)0;
                    Dp = Dp * gp + Sp * (dW + dc);
                    Dm = Dm * gm + Sm * (dc - dW);
                }
                Sp *= gp;
                Sm *= gm;
            }
            const RT xp = type * (Sp - K), xm = type * (Sm - K);
            Csum += (RT)0.5 * ((xp > 0 ? xp : (RT)0) + (xm > 0 ? xm : (RT)0));
            if (GRAD) dCsum += (RT)0.5 * ((xp > 0 ? type * Dp : (RT)0) + (xm > 0 ? type * Dm : (RT)0));
        }
        const RT C = disc_in * Csum * invN;
        const RT dl_dw = V0 - A.disc_tau * C;
        if (!GRAD) {
            double v = valid ? (double)(w * dl_dw) : 0.0;
            v = warp_sum(v);
            if (lane == 0) adj_sh[(m - m0) * warps + warp] = v;
        } else if (valid) {
            const double wE = A.wE[p], wP = A.omega[(size_t)p * A.M + m];
            const RT dl_ds = w * (vega - A.disc_tau * disc_in * dCsum * invN);
            gwE += wE * (double)dl_dw;
            gwP += wP * (double)dl_dw;
            gsE += wE * (double)dl_ds;
            gsP += wP * (double)dl_ds;
        }
    }
    if (!GRAD) {
        __syncthreads();
        for (uint64_t t = threadIdx.x; t < m1 - m0; t += blockDim.x) {
            double v = 0;
            for (int k = 0; k < warps; k++) v += adj_sh[t * warps + k];
            atomicAdd(&A.L[(size_t)p * A.M + m0 + t], v);
        }
        return;
    }
    if (valid) {
        atomicAdd(&A.gw_E[i], gwE);
        atomicAdd(&A.gw_P[i], gwP);
        atomicAdd(&gs_sh[s], gsE);
        atomicAdd(&gs_sh[Q + s], gsP);
    }
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < Q; t += blockDim.x) {
        if (gs_sh[t] != 0) atomicAdd(&A.gs_E[s0 + t], gs_sh[t]);
        if (gs_sh[Q + t] != 0) atomicAdd(&A.gs_P[s0 + t], gs_sh[Q + t]);
    }
}

// ---- estimates and adjoint weights per portfolio (one block per portfolio) -------------------
template <class RT>
__global__ void __launch_bounds__(256) k_adj_weights(AdjLaunch<RT> A) {
    const uint32_t p = blockIdx.x;
    const double K = A.K[p], delta = A.delta[p];
    const double invM = 1.0 / (double)A.M;
    double sL = 0, sS = 0, sH = 0;
    for (uint64_t m = threadIdx.x; m < A.M; m += blockDim.x) {
        const double L = A.L[(size_t)p * A.M + m];
        const double x = (L - K) / delta;
        const double sgm = 1.0 / (1.0 + exp(-x));
        A.omega[(size_t)p * A.M + m] = sgm * (1.0 - sgm) / delta * invM;
        sL += L;
        sS += sgm;
        sH += L > K ? 1.0 : 0.0;
    }
    __shared__ double red[3][8];
    sL = warp_sum(sL);
    sS = warp_sum(sS);
    sH = warp_sum(sH);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { red[0][warp] = sL; red[1][warp] = sS; red[2][warp] = sH; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = 0, c = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) { a += red[0][k]; b += red[1][k]; c += red[2][k]; }
        A.est[3 * p + 0] = a * invM;
        A.est[3 * p + 1] = b * invM;
        A.est[3 * p + 2] = c * invM;
        A.wE[p] = invM;
    }
}

template <class RT>
cudaError_t launch_adjoint_t(const AdjLaunch<RT>& A, bool grad, cudaStream_t stream) {
    if (A.tile == 0 || A.tile > kAdjMaxTile) return cudaErrorInvalidValue;
    const uint32_t warps = kAdjThreads / 32;
    const uint32_t ob = (uint32_t)(((uint64_t)A.n * A.M + 255) / 256);
    k_adj_outer<RT><<<ob < 148 * 8 ? ob : 148 * 8, 256, 0, stream>>>(A);
    const dim3 grid(A.n_chunks, (uint32_t)((A.M + A.tile - 1) / A.tile));
    k_adj_paths<RT, false><<<grid, kAdjThreads, (size_t)A.tile * warps * sizeof(double), stream>>>(A);
    k_adj_weights<RT><<<A.n, 256, 0, stream>>>(A);
    count_launch(3);
    if (grad) {
        const size_t sh = (size_t)2 * A.q_max * sizeof(double);
        if (sh > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(k_adj_paths<RT, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
            if (e != cudaSuccess) return e;
        }
        k_adj_paths<RT, true><<<grid, kAdjThreads, sh, stream>>>(A);
        count_launch(1);
    }
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_adjoint(const AdjLaunch<float>& A, bool grad, cudaStream_t stream) {
    return launch_adjoint_t<float>(A, grad, stream);
}
cudaError_t launch_adjoint(const AdjLaunch<double>& A, bool grad, cudaStream_t stream) {
    return launch_adjoint_t<double>(A, grad, stream);
}

}  // namespace nmlmc
