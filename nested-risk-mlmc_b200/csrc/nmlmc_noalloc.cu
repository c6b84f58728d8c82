// Allocation-free entry point: one level call of the model problem on the batched (OUTER
// layout) path, with every piece of scratch it needs carved out of one file-scope device array.
//
// Who needs it: callers that may not allocate device memory themselves — code that runs while
// a framework owns the device memory pool (a cudaMalloc behind its back fragments the pool or
// blocks on its allocator), latency-critical code for which cudaMalloc's implicit device-wide
// synchronisation is not acceptable, and hosts that cap device memory and reserve it up front.  They pass
// scalars in and a device buffer for the result out; nothing is allocated per call.
//
// The array below is reserved in every process that loads this library, on every GPU it touches,
// until the process exits (NMLMC_NOALLOC_SCRATCH_BYTES, 3 MiB).  All calls share it: a call
// clears the counters and partial sums it relies on before use, and two calls whose work
// overlaps on the GPU (different streams, or different host threads on one device) race on it.
// The first call on a device looks up the array's device address and keeps it for the life of
// the process: a device reset (cudaDeviceReset) or a destroyed primary context after that first
// call is not supported.  Failures are reported like every other entry point's, through the
// return value and nmlmc_last_error().
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/nmlmc.h"
#include "nmlmc_internal.h"

using namespace nmlmc;

static constexpr size_t kScratchBytes = NMLMC_NOALLOC_SCRATCH_BYTES;
static constexpr uint64_t kMaxOuter = NMLMC_NOALLOC_MAX_OUTER;
static constexpr int kMaxGrid = 1024;   // CTAs whose partial sums fit the reserved slice

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

struct DeviceScratch {
    bool ready = false;
    unsigned char* base = nullptr;   // device address of g_noalloc_scratch on this device
    int grid = 0;
};

constexpr int kMaxDevices = 64;
DeviceScratch g_scratch[kMaxDevices];
std::mutex g_scratch_mu;

inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Carves the batch buffers of one level call out of the scratch array.
bool carve(unsigned char* base, int grid, OuterBuffers& B) {
    size_t off = 0;
    auto take = [&](size_t bytes) {
        unsigned char* p = base + off;
        off += align256(bytes);
        return p;
    };
    B = OuterBuffers{};
    B.cap = kMaxOuter;
    B.Q = 0;
    B.Yv = take(kMaxOuter * sizeof(double));
    B.Rt = nullptr;                                          // models only: no R_tau rows
    B.cnt_f = reinterpret_cast<uint32_t*>(take(kMaxOuter * sizeof(uint32_t)));
    B.cnt_c = reinterpret_cast<uint32_t*>(take(kMaxOuter * sizeof(uint32_t)));
    B.lists = reinterpret_cast<uint32_t*>(take(4 * kMaxOuter * sizeof(uint32_t)));
    B.class_items = reinterpret_cast<uint32_t*>(take(kMaxOuter * sizeof(uint32_t)));
    B.counters = reinterpret_cast<uint32_t*>(take(256 * sizeof(uint32_t)));
    B.block_sums = reinterpret_cast<double*>(take((size_t)kMaxGrid * 16 * sizeof(double)));
    B.level_acc = reinterpret_cast<double*>(take(16 * sizeof(double)));
    B.grid = grid;
    B.prof_mark = nullptr;
    B.prof_user = nullptr;
    return off <= kScratchBytes;
}

// Once per device, with that device current: the device address of the scratch array.
int setup_device(int dev, DeviceScratch*& out) {
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    DeviceScratch& s = g_scratch[dev];
    if (!s.ready) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            fprintf(stderr, "nmlmc: cudaGetSymbolAddress(noalloc scratch) failed: %s\n", cudaGetErrorString(e));
            return NMLMC_ERR_CUDA;
        }
        int sms = 148;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) sms = 148;
        s.base = static_cast<unsigned char*>(p);
        s.grid = sms * 4 < kMaxGrid ? sms * 4 : kMaxGrid;
        s.ready = true;
    }
    out = &s;
    return NMLMC_OK;
}

uint64_t upow(uint64_t x, uint32_t n) {
    uint64_t r = 1;
    while (n--) r *= x;
    return r;
}

}  // namespace

extern "C" int nmlmc_sample_level_noalloc(int32_t kind, double tau, double max_loss, uint32_t N0,
                                          uint32_t beta, double adaptive_r, int32_t adaptive_incl_r2,
                                          int32_t precision, uint64_t seed, uint32_t ell,
                                          uint64_t first_index, uint64_t M, double* d_out,
                                          void* stream) {
    if (kind != NMLMC_MODEL_REFERENCE && kind != NMLMC_MODEL_SHIFT) return set_last_error(NMLMC_ERR_ARG);
    if (precision != NMLMC_PREC_FP32 && precision != NMLMC_PREC_FP64) return set_last_error(NMLMC_ERR_ARG);
    // the model checks of nmlmc_set_model: finite inputs, and the reference model's sqrt(tau),
    // sqrt(1 - tau) (model_sampler.cpp:21-39) need 0 <= tau <= 1
    if (!std::isfinite(tau) || !std::isfinite(max_loss) || !std::isfinite(adaptive_r)) return set_last_error(NMLMC_ERR_ARG);
    if (kind == NMLMC_MODEL_REFERENCE && !(tau >= 0 && tau <= 1)) return set_last_error(NMLMC_ERR_ARG);
    if (M > kMaxOuter) {
        fprintf(stderr, "nmlmc_sample_level_noalloc: M = %llu exceeds the scratch limit of %llu outer samples\n",
                (unsigned long long)M, (unsigned long long)kMaxOuter);
        return set_last_error(NMLMC_ERR_ARG);
    }
    if (!d_out || N0 == 0 || beta < 2 || (beta & (beta - 1)) || ell >= NMLMC_MAX_LEVELS) return set_last_error(NMLMC_ERR_ARG);
    const uint32_t chunk = N0 >= 32 ? 32 : N0;
    if ((N0 % chunk) != 0 || (chunk & (chunk - 1)) != 0 || chunk < 4) return set_last_error(NMLMC_ERR_ARG);
    // the level's largest inner count N0 beta^ell, in double like nmlmc_sample (an integer power
    // would wrap around for large beta and ell), checked before any count is formed
    if ((double)N0 * pow((double)beta, (double)ell) > 4.0e9) return set_last_error(NMLMC_ERR_ARG);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return set_last_error(NMLMC_ERR_CUDA);
    DeviceScratch* ds = nullptr;
    int rc = setup_device(dev, ds);
    if (rc) return set_last_error(rc);
    OuterBuffers B;
    if (!carve(ds->base, ds->grid, B)) return set_last_error(NMLMC_ERR_NOMEM);
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // get_samples_count parameters of the fine and coarse levels (nested_sampler.hpp:225-239)
    auto params = [&](uint32_t l) {
        CountParams p;
        p.max_count = (uint64_t)N0 * upow(beta, l);
        const bool f64 = precision == NMLMC_PREC_FP64;
        const double r = f64 ? adaptive_r : (double)(float)adaptive_r;
        const bool adaptive = r > 1 && (adaptive_incl_r2 ? r <= 2 : r < 2);
        if (adaptive) {
            p.base_count = (uint64_t)N0 * upow(beta >> 1, l);
            p.tmp = f64 ? (double)p.max_count * pow(9.0 / (double)p.max_count, r / 2)
                        : (double)((float)p.max_count * powf(9.f / (float)p.max_count, (float)r / 2));
        } else {
            p.base_count = p.max_count;
            p.tmp = 0;
        }
        return p;
    };
    const CountParams cf = params(ell), cc = params(ell == 0 ? 0 : ell - 1);
    const bool adaptive = cf.base_count != cf.max_count;

    // clear what the kernels accumulate into (the array keeps the previous call's contents)
    cudaError_t e = cudaMemsetAsync(B.counters, 0, 256 * sizeof(uint32_t), st);
    if (e == cudaSuccess) e = outer_level_begin(B, st);
    if (e == cudaSuccess && M) {
        if (precision == NMLMC_PREC_FP32) {
            OuterLevel<float> L{};
            L.ell = ell; L.M = M; L.first_index = first_index; L.seed = seed;
            L.fine_only = ell == 0; L.antithetic = true; L.N0 = N0; L.chunk = chunk;
            L.adaptive_r = (float)adaptive_r; L.cf = cf; L.cc = cc;
            L.adaptive_f = adaptive && cf.max_count > 2 * cf.base_count;
            L.adaptive_c = !L.fine_only && adaptive && cc.max_count > 2 * cc.base_count;
            const float t = (float)tau;
            L.mp.stau = sqrtf(t); L.mp.s1tau = sqrtf(1.0f - t); L.mp.max_loss = (float)max_loss;
            e = outer_sample_level<float>(L, kind, PREC_FP32, B, nullptr, st);
        } else {
            OuterLevel<double> L{};
            L.ell = ell; L.M = M; L.first_index = first_index; L.seed = seed;
            L.fine_only = ell == 0; L.antithetic = true; L.N0 = N0; L.chunk = chunk;
            L.adaptive_r = adaptive_r; L.cf = cf; L.cc = cc;
            L.adaptive_f = adaptive && cf.max_count > 2 * cf.base_count;
            L.adaptive_c = !L.fine_only && adaptive && cc.max_count > 2 * cc.base_count;
            L.mp.stau = sqrt(tau); L.mp.s1tau = sqrt(1.0 - tau); L.mp.max_loss = max_loss;
            e = outer_sample_level<double>(L, kind, PREC_FP64, B, nullptr, st);
        }
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_out, B.level_acc, 16 * sizeof(double), cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) {
        fprintf(stderr, "nmlmc_sample_level_noalloc: %s\n", cudaGetErrorString(e));
        return set_last_error(NMLMC_ERR_CUDA);
    }
    return set_last_error(NMLMC_OK);
}
