// The X = Y + Z model of the benchmark written as a caller's SAMPLER class (the reference's
// interface: inner_sampler_base, sample_outer, copy_outer, init_inner_sampler, sample_inner,
// add_phi; model_sampler.cpp:42-92) and run through include/nmlmc_sampler.cuh on the batched path.
// tests/test_gpu_sampler_api.py compares it with the library's built-in KIND_SHIFT_MODEL on the
// same streams (bit-exact).  Built by __graft_entry__.build() into tests/abi/_build/.
#include "nmlmc_sampler.cuh"

namespace {

__constant__ double g_K;        // the threshold K (model::data::max_loss)

template <class RT>
struct shift_sampler : nmlmc::inner_sampler_base<RT> {
    static constexpr uint32_t normals_per_inner = 1, uniforms_per_inner = 0;
    RT Y;

    static uint32_t GetWorkspaceSize(double) { return 0; }
    __device__ explicit shift_sampler(void*) : Y(0) {}
    __device__ void sample_outer(uint64_t, double&) { Y = this->randn_sync(); }       // Y ~ N(0, 1)
    __device__ void copy_outer(const shift_sampler& o) { Y = o.Y; }
    __device__ RT init_inner_sampler(uint64_t&, double&) { return (RT)-g_K; }
    __device__ RT sample_inner(uint64_t, uint64_t, double& work) {                    // X = Y + Z
        work += 1;
        return Y + this->randn();
    }
    __device__ static void add_phi(RT mean, RT coeff, RT* phi) { *phi += coeff * (RT)(mean >= (RT)0); }
};

template <class RT>
int init(uint32_t N0, uint32_t beta, float r, uint64_t seed, double K) {
    if (cudaMemcpyToSymbol(g_K, &K, sizeof K) != cudaSuccess) return NMLMC_ERR_CUDA;
    nested_sampler_params p{N0, beta, true, 4, 4, r};
    return nmlmc::init_samplers<shift_sampler<RT>>(p, seed, shift_sampler<RT>::GetWorkspaceSize(K));
}

}  // namespace

extern "C" int user_shift_init(int32_t fp64, uint32_t N0, uint32_t beta, float r, uint64_t seed, double K) {
    return fp64 ? init<double>(N0, beta, r, seed, K) : init<float>(N0, beta, r, seed, K);
}

extern "C" int user_shift_sample(int32_t fp64, uint32_t ell, uint64_t M, double* fsums, double* diffsums,
                                 double* work, uint64_t* stats) {
    return fp64 ? nmlmc::sample<shift_sampler<double>>(ell, 0, &M, fsums, diffsums, work, stats)
                : nmlmc::sample<shift_sampler<float>>(ell, 0, &M, fsums, diffsums, work, stats);
}

extern "C" void user_shift_cleanup(void) {
    nmlmc::cleanup_samplers<shift_sampler<float>>();
    nmlmc::cleanup_samplers<shift_sampler<double>>();
}
