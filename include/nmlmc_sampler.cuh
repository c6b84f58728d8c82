// nmlmc_sampler.cuh — the reference's SAMPLER extension interface on the batched B200 path.
//
// In the reference a new nested problem is a new SAMPLER class: it derives from
// inner_sampler_base (nested_sampler.hpp:36-85), which hands it the random draws, and provides
// sample_outer, copy_outer, init_inner_sampler, sample_inner and add_phi (model_sampler.cpp:42-92,
// portfolio_sampler.cpp:227-334); sample<SAMPLER>(ell, ...) (nested_sampler.hpp:646-694) runs the
// nested level sampler over it.  This header keeps that interface and runs such a class on the
// library's batched level sampler (breadth-first adaptive pilots, work-queue phase kernel, the same
// code as the built-in kinds; csrc/nmlmc_outer_impl.cuh) for the caller's own sm_100a build:
//
//   nvcc -gencode arch=compute_100a,code=sm_100a -std=c++17 --expt-relaxed-constexpr
//        -I include -I nested-risk-mlmc_b200/csrc  <the caller's .cu file>
//
// A SAMPLER here:
//   * derives from nmlmc::inner_sampler_base<real_t> (real_t = float: the FP32 path with SFU
//     Box-Muller, Kahan FP32 inner sums and FP64 moments; double: the FP64 path);
//   * declares static constexpr uint32_t normals_per_inner and uniforms_per_inner: the most
//     randn() and randu() calls one sample_inner makes.  Every inner sample has its own slice of
//     its phase's draws (the OUTER layout addresses each inner sample, so any thread may evaluate
//     it); this is the one addition to the reference's concept;
//   * has the reference's members, all __device__: a constructor taking the workspace pointer,
//     static GetWorkspaceSize(data) (host), sample_outer(ell, work), copy_outer(rhs),
//     init_inner_sampler(count, work) -> start, sample_inner(i, count, work) -> value,
//     static add_phi(mean, coeff, phi*);
//   * is trivially copyable: the batched path stores one object per outer sample (its outer
//     state) and copies it into every thread that evaluates that sample's inner samples.
//
// Differences from the reference's engine, all imposed by batching: init_inner_sampler is called
// once per outer sample, after sample_outer, with the level's base count, and its start value is
// used for every inner estimate of that sample (the reference assumes start independent of the
// count too, nested_sampler.hpp:213); the workspace (GetWorkspaceSize bytes) is one block per outer
// sample that sample_outer may write and inner sampling may only read; sample_inner's `count` is
// the inner count of the phase being evaluated; add_phi's phi has one entry (phi_size 1).
//
// Streams (OUTER layout): outer sample m of level ell has the Threefry2x64-20 key
// (seed, ell << 56 | m).  randn_sync()/randu_sync() (sample_outer) draw normal / uniform k of
// the outer phase (counter word 1 = 0); randn()/randu() of inner sample i draw normal
// i * normals_per_inner + j / uniform i * uniforms_per_inner + j of the phase being evaluated
// (pilot round or final).  Normal k is component k & 1 of the Box-Muller pair made of 32-bit words
// 2(k >> 1) and 2(k >> 1) + 1 of the phase (four words per block: lo(v0), hi(v0), lo(v1), hi(v1)),
// exactly as the built-in model kinds draw them; uniforms come from a separate counter
// namespace (counter word 1 = phase tag + 2^32), word k giving u = (w + 1/2) 2^-32.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <type_traits>

#include <cuda_runtime.h>

#include "nmlmc.h"
#include "nmlmc_outer_impl.cuh"

namespace nmlmc {

constexpr uint64_t kUniformNamespace = 1ull << 32;

// inner_sampler_base (nested_sampler.hpp:36-85) on the OUTER layout.
template <class RT>
class inner_sampler_base {
    static_assert(std::is_same<RT, float>::value || std::is_same<RT, double>::value, "real_t is float or double");
    static constexpr int kPrec = sizeof(RT) == 4 ? PREC_FP32 : PREC_FP64;

public:
    using real_type = RT;

    __device__ RT randn_sync() { return nm_normal(PH_OUTER, nm_sync_n_++); }
    __device__ RT randu_sync() { return nm_uniform(PH_OUTER, nm_sync_u_++); }
    __device__ RT randn() { return nm_normal(nm_tag_, nm_n_++); }
    __device__ RT randu() { return nm_uniform(nm_tag_, nm_u_++); }

    // Set by the batched kernels before sample_outer / before each sample_inner.
    __device__ void nm_begin_outer(const TfKey& key) {
        nm_key_ = key;
        nm_sync_n_ = nm_sync_u_ = 0;
        nm_blk_tag_ = ~0ull;
    }
    template <class S>
    __device__ void nm_begin_inner_of(const TfKey& key, uint64_t tag, uint64_t i) {
        nm_key_ = key;
        nm_tag_ = tag;
        nm_n_ = i * S::normals_per_inner;
        nm_u_ = i * S::uniforms_per_inner;
    }

private:
    TfKey nm_key_{};
    uint64_t nm_tag_ = 0, nm_n_ = 0, nm_u_ = 0, nm_sync_n_ = 0, nm_sync_u_ = 0;
    uint64_t nm_blk_ = 0, nm_blk_tag_ = ~0ull, nm_v0_ = 0, nm_v1_ = 0;   // last Threefry block

    __device__ void nm_block(uint64_t tag, uint64_t blk) {
        if (blk != nm_blk_ || tag != nm_blk_tag_) {
            threefry2x64(blk, tag, nm_key_, nm_v0_, nm_v1_);
            nm_blk_ = blk;
            nm_blk_tag_ = tag;
        }
    }
    __device__ RT nm_normal(uint64_t tag, uint64_t k) {
        nm_block(tag, k >> 2);
        const uint64_t e = ((k >> 1) & 1) ? nm_v1_ : nm_v0_;
        RT x, y;
        bm_pair<kPrec, RT>((uint32_t)e, (uint32_t)(e >> 32), x, y);
        return (k & 1) ? y : x;
    }
    __device__ RT nm_uniform(uint64_t tag, uint64_t k) {
        nm_block(tag + kUniformNamespace, k >> 2);
        const uint64_t e = ((k >> 1) & 1) ? nm_v1_ : nm_v0_;
        return u01_word<kPrec, RT>((k & 1) ? (uint32_t)(e >> 32) : (uint32_t)e);
    }
};

// The batched level sampler over a caller's SAMPLER class: device buffers for `batch` outer
// samples per launch sequence (larger calls run in batches, with the same results), one CUDA
// stream.  Calls are synchronous, like the reference's sample<SAMPLER>.
template <class SAMPLER>
class batched_sampler {
    using RT = typename SAMPLER::real_type;
    static constexpr int kPrec = sizeof(RT) == 4 ? PREC_FP32 : PREC_FP64;
    static_assert(std::is_base_of<inner_sampler_base<RT>, SAMPLER>::value,
                  "a SAMPLER derives from nmlmc::inner_sampler_base<real_t>");
    static_assert(std::is_trivially_copyable<SAMPLER>::value, "a SAMPLER is trivially copyable");
    static_assert(SAMPLER::normals_per_inner + SAMPLER::uniforms_per_inner > 0,
                  "a SAMPLER declares normals_per_inner and uniforms_per_inner");

public:
    batched_sampler() = default;
    batched_sampler(const batched_sampler&) = delete;
    batched_sampler& operator=(const batched_sampler&) = delete;
    ~batched_sampler() { release(); }

    // N0, beta, adaptive_r, antithetic as nested_sampler_params (nested_sampler.hpp:14-34; the
    // batched path needs the antithetic estimator and N0 a power-of-two multiple of its chunk),
    // adaptive_incl_r2 admits r = 2; seed: the streams' key; workspace_bytes:
    // SAMPLER::GetWorkspaceSize(data).  Returns an NMLMC_* status.
    int init(uint32_t N0, uint32_t beta, double adaptive_r, bool antithetic, bool adaptive_incl_r2,
             uint64_t seed, uint32_t workspace_bytes, uint64_t batch = 1u << 18, cudaStream_t stream = nullptr) {
        release();
        const uint32_t chunk = N0 >= 32 ? 32 : N0;
        if (N0 == 0 || beta < 2 || (beta & (beta - 1)) || !antithetic || chunk < 4 || (chunk & (chunk - 1)) ||
            N0 % chunk || batch == 0 || batch > (1ull << 31))
            return NMLMC_ERR_ARG;
        N0_ = N0; beta_ = beta; r_ = adaptive_r; incl_r2_ = adaptive_incl_r2; seed_ = seed; chunk_ = chunk;
        stream_ = stream;
        int dev = 0, sms = 148;
        if (cudaGetDevice(&dev) != cudaSuccess) return NMLMC_ERR_CUDA;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        B_ = OuterBuffers{};
        B_.cap = batch;
        B_.grid = 4 * sms;
        B_.state_bytes = (uint32_t)((sizeof(SAMPLER) + 15) & ~(size_t)15);
        B_.ws_bytes = (workspace_bytes + 15u) & ~15u;
        bool ok = alloc(&B_.Yv, batch * sizeof(double)) && alloc(&B_.cnt_f, batch * 4) && alloc(&B_.cnt_c, batch * 4) &&
                  alloc(&B_.lists, 4 * batch * 4) && alloc(&B_.class_items, batch * 4) &&
                  alloc(&B_.counters, 256 * 4) && alloc(&B_.block_sums, (size_t)B_.grid * 16 * sizeof(double)) &&
                  alloc(&B_.level_acc, 16 * sizeof(double)) && alloc(&B_.user_state, batch * B_.state_bytes) &&
                  (B_.ws_bytes == 0 || alloc(&B_.user_ws, batch * B_.ws_bytes));
        if (!ok) {
            release();
            return NMLMC_ERR_NOMEM;
        }
        if (cudaMemset(B_.counters, 0, 256 * 4) != cudaSuccess) return NMLMC_ERR_CUDA;
        memset(next_, 0, sizeof next_);
        ready_ = true;
        return NMLMC_OK;
    }

    // sample<SAMPLER>(ell, override_dyn_inner, &M, fsums, diffsums, &total_work, inner_stats)
    // (nested_sampler.hpp:646-694): M outer samples of level ell (the next unused outer indices of
    // the level), the fine-only estimate at ell = 0.  inner_stats: inner samples, outer samples,
    // outer samples at the maximum count, at the base count, 0, 0.
    int sample(uint32_t ell, uint64_t M, double fsums[4], double diffsums[4], double* total_work,
               uint64_t inner_stats[6]) {
        if (!ready_) return NMLMC_ERR_STATE;
        if (ell >= NMLMC_MAX_LEVELS || (double)N0_ * pow((double)beta_, (double)ell) > 4.0e9) return NMLMC_ERR_ARG;
        OuterLevel<RT> L{};
        L.ell = ell;
        L.M = M;
        L.first_index = next_[ell];
        L.seed = seed_;
        L.fine_only = ell == 0;
        L.antithetic = true;
        L.N0 = N0_;
        L.chunk = chunk_;
        L.variant = 0;
        L.adaptive_r = (RT)r_;
        L.cf = counts(ell);
        L.cc = counts(ell == 0 ? 0 : ell - 1);
        const bool adapt = adaptive();
        L.adaptive_f = adapt && L.cf.max_count > 2 * L.cf.base_count;
        L.adaptive_c = !L.fine_only && adapt && L.cc.max_count > 2 * L.cc.base_count;
        cudaError_t e = outer_level_begin(B_, stream_);
        if (e == cudaSuccess && M) e = sample_level_t<RT, KIND_USER, kPrec, SAMPLER>(L, B_, nullptr, stream_);
        double acc[16];
        if (e == cudaSuccess) e = cudaMemcpyAsync(acc, B_.level_acc, sizeof acc, cudaMemcpyDeviceToHost, stream_);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
        if (e != cudaSuccess) return NMLMC_ERR_CUDA;
        for (int j = 0; j < 4; j++) {
            fsums[j] = acc[j];
            if (diffsums) diffsums[j] = acc[4 + j];
        }
        *total_work = acc[8];
        const uint64_t st[6] = {(uint64_t)acc[9], M, (uint64_t)acc[10], (uint64_t)acc[11], 0, 0};
        if (inner_stats) memcpy(inner_stats, st, sizeof st);
        next_[ell] += M;
        return NMLMC_OK;
    }

    void release() {
        void* ptrs[] = {B_.Yv, B_.cnt_f, B_.cnt_c, B_.lists, B_.class_items, B_.counters, B_.block_sums,
                        B_.level_acc, B_.user_state, B_.user_ws};
        for (void* p : ptrs)
            if (p) cudaFree(p);
        B_ = OuterBuffers{};
        ready_ = false;
    }

private:
    OuterBuffers B_{};
    cudaStream_t stream_ = nullptr;
    uint32_t N0_ = 0, beta_ = 2, chunk_ = 32;
    double r_ = 0;
    bool incl_r2_ = false, ready_ = false;
    uint64_t seed_ = 0;
    uint64_t next_[NMLMC_MAX_LEVELS] = {};

    template <class T>
    static bool alloc(T** p, size_t bytes) {
        return cudaMalloc(reinterpret_cast<void**>(p), bytes) == cudaSuccess;
    }
    // nested_sampler_params::adaptive() (nested_sampler.hpp:33) in real_t, r = 2 admitted on request
    bool adaptive() const {
        const RT r = (RT)r_;
        return r > 1 && (incl_r2_ ? r <= 2 : r < 2);
    }
    static uint64_t upow(uint64_t x, uint32_t n) {
        uint64_t v = 1;
        while (n--) v *= x;
        return v;
    }
    // get_samples_count's constructor (nested_sampler.hpp:225-239), evaluated as the library does
    CountParams counts(uint32_t l) const {
        CountParams p;
        p.max_count = (uint64_t)N0_ * upow(beta_, l);
        if (adaptive()) {
            p.base_count = (uint64_t)N0_ * upow(beta_ >> 1, l);
            if (kPrec == PREC_FP64)
                p.tmp = (double)p.max_count * pow(9.0 / (double)p.max_count, r_ / 2);
            else
                p.tmp = (double)((float)p.max_count * powf(9.f / (float)p.max_count, (float)r_ / 2));
        } else {
            p.base_count = p.max_count;
            p.tmp = 0;
        }
        return p;
    }
};

// The reference's process-wide call shape for one SAMPLER class: init_samplers<SAMPLER>(params,
// seed, workspace) (after init_nestedmc_sampler and init_samplers, nested_sampler.hpp:618-644),
// sample<SAMPLER>(...) and cleanup_samplers<SAMPLER>().
template <class SAMPLER>
batched_sampler<SAMPLER>& samplers_of() {
    static batched_sampler<SAMPLER> s;
    return s;
}

template <class SAMPLER>
int init_samplers(const nested_sampler_params& p, uint64_t seed, uint32_t workspace_size,
                  bool adaptive_incl_r2 = false) {
    return samplers_of<SAMPLER>().init(p.N0, p.beta, (double)p.adaptive_r, p.antithetic, adaptive_incl_r2, seed,
                                       workspace_size);
}

template <class SAMPLER>
int sample(uint32_t ell, uint64_t /*override_dyn_inner*/, uint64_t* M, double* out_fsums, double* out_diffsums,
           double* out_total_work, uint64_t* out_inner_stats) {
    return samplers_of<SAMPLER>().sample(ell, *M, out_fsums, out_diffsums, out_total_work, out_inner_stats);
}

template <class SAMPLER>
void cleanup_samplers() {
    samplers_of<SAMPLER>().release();
}

}  // namespace nmlmc
