// OUTER-layout (batched) level sampler: the precision/kind dispatch of a level call, the
// full-portfolio loss sweep, device timestamps, launch counting and the utility kernels.  The
// kernels and the launch sequence of a level are in nmlmc_outer_impl.cuh; their instantiations per
// sampler kind are compiled from nmlmc_outer_kind.cu.
#include <atomic>

#include "nmlmc_outer_impl.cuh"

namespace nmlmc {

// Device timestamp (%globaltimer, nanoseconds): marks level boundaries inside a CUDA graph,
// where event-record nodes carry no elapsed time.
__global__ void k_stamp(uint64_t* slot) {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    *slot = t;
}

cudaError_t launch_stamp(uint64_t* slot, cudaStream_t stream) {
    k_stamp<<<1, 1, 0, stream>>>(slot);
    count_launch();
    return cudaGetLastError();
}

// ---- host orchestration ----------------------------------------------------------------------
static std::atomic<uint64_t> g_launches{0};
void count_launch(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
uint64_t launches_total() { return g_launches.load(std::memory_order_relaxed); }

cudaError_t outer_level_begin(OuterBuffers& B, cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(B.level_acc, 0, 16 * sizeof(double), stream);
    if (e != cudaSuccess) return e;
    return cudaMemsetAsync(B.block_sums, 0, (size_t)B.grid * 16 * sizeof(double), stream);
}

// Level sequences instantiated per kind in nmlmc_outer_kind.cu.
#define NMLMC_SLT(RT, KIND, PREC) \
    extern template cudaError_t sample_level_t<RT, KIND, PREC>(const OuterLevel<RT>&, OuterBuffers&, TraceRec*, cudaStream_t);
NMLMC_SLT(float, KIND_REF_MODEL, PREC_FP32) NMLMC_SLT(float, KIND_SHIFT_MODEL, PREC_FP32) NMLMC_SLT(float, KIND_PORTFOLIO, PREC_FP32)
NMLMC_SLT(float, KIND_REF_MODEL, PREC_REF32) NMLMC_SLT(float, KIND_SHIFT_MODEL, PREC_REF32) NMLMC_SLT(float, KIND_PORTFOLIO, PREC_REF32)
NMLMC_SLT(double, KIND_REF_MODEL, PREC_FP64) NMLMC_SLT(double, KIND_SHIFT_MODEL, PREC_FP64) NMLMC_SLT(double, KIND_PORTFOLIO, PREC_FP64)
NMLMC_SLT(float, KIND_PF_PATHS, PREC_FP32) NMLMC_SLT(float, KIND_PF_PATHS, PREC_REF32) NMLMC_SLT(double, KIND_PF_PATHS, PREC_FP64)
#undef NMLMC_SLT

template <class RT>
cudaError_t outer_sample_level(const OuterLevel<RT>& L, int kind, int prec, OuterBuffers& B,
                               TraceRec* trace, cudaStream_t stream) {
    if (prec == PREC_FP64) {
        if constexpr (sizeof(RT) == 8) {
            if (kind == KIND_REF_MODEL) return sample_level_t<RT, KIND_REF_MODEL, PREC_FP64>(L, B, trace, stream);
            if (kind == KIND_SHIFT_MODEL) return sample_level_t<RT, KIND_SHIFT_MODEL, PREC_FP64>(L, B, trace, stream);
            if (L.ot.mixed) return sample_level_t<RT, KIND_PF_PATHS, PREC_FP64>(L, B, trace, stream);
            return sample_level_t<RT, KIND_PORTFOLIO, PREC_FP64>(L, B, trace, stream);
        }
        return cudaErrorInvalidValue;
    }
    if constexpr (sizeof(RT) == 4) {
        if (prec == PREC_FP32) {
            if (kind == KIND_REF_MODEL) return sample_level_t<RT, KIND_REF_MODEL, PREC_FP32>(L, B, trace, stream);
            if (kind == KIND_SHIFT_MODEL) return sample_level_t<RT, KIND_SHIFT_MODEL, PREC_FP32>(L, B, trace, stream);
            if (L.ot.mixed) return sample_level_t<RT, KIND_PF_PATHS, PREC_FP32>(L, B, trace, stream);
            return sample_level_t<RT, KIND_PORTFOLIO, PREC_FP32>(L, B, trace, stream);
        }
        if (kind == KIND_REF_MODEL) return sample_level_t<RT, KIND_REF_MODEL, PREC_REF32>(L, B, trace, stream);
        if (kind == KIND_SHIFT_MODEL) return sample_level_t<RT, KIND_SHIFT_MODEL, PREC_REF32>(L, B, trace, stream);
        if (L.ot.mixed) return sample_level_t<RT, KIND_PF_PATHS, PREC_REF32>(L, B, trace, stream);
        return sample_level_t<RT, KIND_PORTFOLIO, PREC_REF32>(L, B, trace, stream);
    }
    return cudaErrorInvalidValue;
}

template cudaError_t outer_sample_level<float>(const OuterLevel<float>&, int, int, OuterBuffers&, TraceRec*, cudaStream_t);
template cudaError_t outer_sample_level<double>(const OuterLevel<double>&, int, int, OuterBuffers&, TraceRec*, cudaStream_t);

// ---- full portfolio loss sweep ---------------------------------------------------------------
// L(Y) over every option: init_inner_sampler without sub-sampling and sample_inner_all_options
// (portfolio_sampler.cpp:312-324, 336-344), one warp per outer sample, for the K quantile.
template <class RT, int PREC>
__global__ void k_full_loss(DevLevel<RT> D, uint32_t nb, double* loss) {
    // one warp per outer sample: lanes stride the option table, double accumulation
    const int lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    const OptionTable<RT>& ot = D.L.ot;
    for (uint32_t i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < nb; i += warps) {
        constexpr uint32_t RS = RStride<PREC>::v;
        const RT* Rrow = reinterpret_cast<const RT*>(D.B.Rt) + (size_t)i * ot.Q * RS;
        double s = 0;
        for (uint32_t j = lane; j < ot.P; j += 32) {
            uint32_t st = ot.stock_ind[j];
            RT bs = calc_bs_ref<RT>(ot.type[j], Rrow[st * RS], ot.strike[j], ot.r, xsub(ot.maturity[j], ot.tau), ot.sigma[st]);
            RT finish = ot.discount ? xmul(xexp(xmul(-ot.r, ot.tau)), bs) : bs;
            s += (double)xmul(ot.w[j], xsub(ot.start[j], finish));
        }
        s = warp_sum(s);
        if (lane == 0) loss[i] = s;
    }
}

// FP32 sweep of the packed option table: a CTA takes a tile of kLossTile outer samples (their
// R and ln R rows in shared memory) and streams the table once per tile, so every 32-byte
// record fetched from L2/HBM feeds kLossTile Black-Scholes evaluations.  Per-thread partial sums
// are float (each thread adds P/256 options), combined in double across the CTA.
constexpr int kLossTile = 32;

__global__ void __launch_bounds__(kTile) k_full_loss_fast(DevLevel<float> D, uint32_t nb, double* loss) {
    extern __shared__ float sm_rows[];   // R[kLossTile][Q], lnR[kLossTile][Q]
    __shared__ double red[kWarps][kLossTile];
    const OptionTable<float>& ot = D.L.ot;
    const uint32_t Q = ot.Q, P = ot.P;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    float* sR = sm_rows;
    float* slnR = sm_rows + (size_t)kLossTile * Q;
    const float2* Rt = reinterpret_cast<const float2*>(D.B.Rt);     // (R, ln R) per stock
    const uint32_t ntiles = (nb + kLossTile - 1) / kLossTile;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint32_t o0 = tile * kLossTile;
        const uint32_t n_here = (nb - o0) < (uint32_t)kLossTile ? (nb - o0) : (uint32_t)kLossTile;
        for (uint32_t k = t; k < (uint32_t)kLossTile * Q; k += blockDim.x) {
            const uint32_t o = k / Q;
            const float2 R = o < n_here ? Rt[(size_t)(o0 + o) * Q + (k - o * Q)] : make_float2(1.0f, 0.0f);
            sR[k] = R.x;
            slnR[k] = R.y;
        }
        __syncthreads();
        float acc[kLossTile];
#pragma unroll
        for (int o = 0; o < kLossTile; o++) acc[o] = 0.f;
        for (uint32_t j = t; j < P; j += blockDim.x) {
            const FastOption op = ot.fast[j];     // full-loss records: no control variate
            const uint32_t st = op.stock;
#pragma unroll
            for (int o = 0; o < kLossTile; o++) acc[o] += option_loss_fast(op, sR[o * Q + st], slnR[o * Q + st]);
        }
#pragma unroll
        for (int o = 0; o < kLossTile; o++) {
            double v = (double)acc[o];
            for (int m = 16; m > 0; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
            if (lane == 0) red[warp][o] = v;
        }
        __syncthreads();
        if (t < (int)n_here) {
            double s = 0;
            for (int w = 0; w < kWarps; w++) s += red[w][t];
            loss[o0 + t] = s;
        }
        __syncthreads();
    }
}

template <class RT>
cudaError_t outer_full_loss(const OuterLevel<RT>& L, int prec, OuterBuffers& B, double* d_loss,
                            cudaStream_t stream) {
    DevLevel<RT> D;
    D.L = L;
    D.B = B;
    for (uint64_t done = 0; done < L.M;) {
        const uint64_t nb = (L.M - done) < B.cap ? (L.M - done) : B.cap;
        D.L.first_index = L.first_index + done;
        int og = (int)((nb + kTile - 1) / kTile);
        if (og > B.grid) og = B.grid;
        if (og < 1) og = 1;
        if (prec == PREC_FP64) {
            if constexpr (sizeof(RT) == 8) {
                k_outer<RT, KIND_PORTFOLIO, PREC_FP64><<<og, kTile, 0, stream>>>(D, (uint32_t)nb);
                k_full_loss<RT, PREC_FP64><<<B.grid, kTile, 0, stream>>>(D, (uint32_t)nb, d_loss + done);
            }
        } else {
            if constexpr (sizeof(RT) == 4) {
                if (prec == PREC_FP32 && L.ot.fast) {
                    k_outer<RT, KIND_PORTFOLIO, PREC_FP32><<<og, kTile, 0, stream>>>(D, (uint32_t)nb);
                    const size_t smem = (size_t)2 * kLossTile * L.ot.Q * sizeof(float);
                    if (smem > 200 * 1024) return cudaErrorInvalidValue;   // Q above 800 stocks
                    if (smem > 48 * 1024) {
                        cudaError_t ea = cudaFuncSetAttribute(k_full_loss_fast, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
                        if (ea != cudaSuccess) return ea;
                    }
                    const int lg = (int)((nb + kLossTile - 1) / kLossTile) < B.grid ? (int)((nb + kLossTile - 1) / kLossTile) : B.grid;
                    k_full_loss_fast<<<lg, kTile, smem, stream>>>(D, (uint32_t)nb, d_loss + done);
                    count_launch(2);
                } else if (prec == PREC_FP32) {
                    k_outer<RT, KIND_PORTFOLIO, PREC_FP32><<<og, kTile, 0, stream>>>(D, (uint32_t)nb);
                    k_full_loss<RT, PREC_FP32><<<B.grid, kTile, 0, stream>>>(D, (uint32_t)nb, d_loss + done);
                } else {
                    k_outer<RT, KIND_PORTFOLIO, PREC_REF32><<<og, kTile, 0, stream>>>(D, (uint32_t)nb);
                    k_full_loss<RT, PREC_REF32><<<B.grid, kTile, 0, stream>>>(D, (uint32_t)nb, d_loss + done);
                }
            }
        }
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        done += nb;
    }
    return cudaSuccess;
}

template cudaError_t outer_full_loss<float>(const OuterLevel<float>&, int, OuterBuffers&, double*, cudaStream_t);
template cudaError_t outer_full_loss<double>(const OuterLevel<double>&, int, OuterBuffers&, double*, cudaStream_t);

}  // namespace nmlmc

// ---- utility kernels: raw Threefry blocks and OUTER-layout normals ---------------------------
namespace nmlmc {

__global__ void k_threefry_blocks(const uint64_t* ctr, const uint64_t* key, uint64_t* out, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t o0, o1;
        threefry2x64(ctr[2 * i], ctr[2 * i + 1], tf_key(key[2 * i], key[2 * i + 1]), o0, o1);
        out[2 * i] = o0;
        out[2 * i + 1] = o1;
    }
}

template <int PREC>
__global__ void k_outer_normals(uint64_t seed, uint64_t stream, uint32_t tag, uint64_t n, double* out) {
    const TfKey key = tf_key(seed, stream);
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
        if (PREC == PREC_FP32) out[k] = (double)outer_normal_at<PREC_FP32, float>(key, tag, k);
        else out[k] = outer_normal_at<PREC_FP64, double>(key, tag, k);
    }
}

cudaError_t launch_threefry_blocks(const uint64_t* ctr, const uint64_t* key, uint64_t* out, uint64_t n,
                                   cudaStream_t s) {
    k_threefry_blocks<<<256, 256, 0, s>>>(ctr, key, out, n);
    return cudaGetLastError();
}

// Phi(x) of the FP32 Black-Scholes path (norm_cdf_fast, nmlmc_bs.cuh) on n points.
__global__ void k_norm_cdf_fast(const float* x, float* out, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = norm_cdf_fast(x[i]);
}

cudaError_t launch_norm_cdf_fast(const float* x, float* out, uint64_t n, cudaStream_t s) {
    k_norm_cdf_fast<<<256, 256, 0, s>>>(x, out, n);
    return cudaGetLastError();
}

cudaError_t launch_outer_normals(int prec, uint64_t seed, uint64_t stream, uint32_t tag, uint64_t n,
                                 double* out, cudaStream_t s) {
    if (prec == PREC_FP32) k_outer_normals<PREC_FP32><<<256, 256, 0, s>>>(seed, stream, tag, n, out);
    else k_outer_normals<PREC_FP64><<<256, 256, 0, s>>>(seed, stream, tag, n, out);
    return cudaGetLastError();
}

}  // namespace nmlmc
