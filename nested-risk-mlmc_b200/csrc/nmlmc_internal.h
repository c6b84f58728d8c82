// Host/device interface between the C-ABI layer (nmlmc_api.cu) and the kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "nmlmc_common.cuh"

namespace nmlmc {

// One random_state of the CORE layout: 64-bit word position and the cached second normal.
struct CoreStream {
    uint64_t wpos;
    uint32_t saved, pad;
    double sval;
};
static_assert(sizeof(CoreStream) == 24, "CoreStream layout");

template <class RT>
struct CoreLaunch {
    uint32_t cores, ell;
    uint64_t M;
    uint64_t seed;
    bool fine_only, antithetic;
    double adaptive_r;
    CountParams cf, cc;
    ModelParams<RT> mp;
    OptionTable<RT> ot;
};

cudaError_t launch_core(const CoreLaunch<float>& L, int kind, CoreStream* states, double* part_sums,
                        uint64_t* part_stats, double* out_sums, uint64_t* out_stats, TraceRec* trace,
                        cudaStream_t stream);
cudaError_t launch_core(const CoreLaunch<double>& L, int kind, CoreStream* states, double* part_sums,
                        uint64_t* part_stats, double* out_sums, uint64_t* out_stats, TraceRec* trace,
                        cudaStream_t stream);

// ---- OUTER layout (batched) ----------------------------------------------------------------
enum Prec : int { PREC_REF32 = 0, PREC_FP64 = 1, PREC_FP32 = 2 };

// Per-level launch description of the batched path.
template <class RT>
struct OuterLevel {
    uint32_t ell;
    uint64_t M;             // outer samples of this call
    uint64_t first_index;   // stream index of the first outer sample (OUTER layout key)
    uint64_t seed;
    bool fine_only, antithetic, adaptive_f, adaptive_c;
    uint32_t N0, chunk;     // chunk = inner samples per thread (power of two dividing all counts)
    uint32_t variant;       // phase-kernel register/occupancy variant (FP32 path: 0, 1, 2)
    RT adaptive_r;
    CountParams cf, cc;
    ModelParams<RT> mp;
    OptionTable<RT> ot;
};

// Device work buffers of the batched path, sized for `cap` outer samples per batch.
struct OuterBuffers {
    uint64_t cap;
    uint32_t Q;
    void* Yv;                // RT[cap]       model Y / portfolio constant
    void* Rt;                // cap * Q slots of 8 bytes: portfolio R_tau rows (RT R, or the
                             // float pair (R, ln R) on the FP32 path)
    uint32_t* cnt_f;         // final fine count / chunk size (0 = undecided)
    uint32_t* cnt_c;
    uint32_t* lists;         // 4 * cap: fine/coarse round lists, ping-pong
    uint32_t* class_items;   // cap: items sorted by final class
    uint32_t* counters;      // device counters (see nmlmc_outer.cu)
    double* block_sums;      // per-CTA partial moments [grid][16]
    double* level_acc;       // accumulated level result [16]
    int grid;
    // KIND_USER only (caller-written SAMPLER classes): the SAMPLER object of every outer sample
    // (its outer state, state_bytes each) and its workspace (ws_bytes each)
    void* user_state;
    void* user_ws;
    uint32_t state_bytes, ws_bytes;
    // optional CUDA-event timing of the phase kernel: called around each k_phase launch
    void (*prof_mark)(void* user, int end, cudaStream_t stream);
    void* prof_user;
};

// Device counter slot (OuterBuffers::counters) that the batched kernels set when a
// path-simulated inner sample would exceed kMaxPathSteps (the call then fails with
// NMLMC_ERR_LIMIT); the host clears it.
constexpr uint32_t kCounterPathLimit = 240;

// Records a failed status for nmlmc_last_error() (this thread) and returns it.
int set_last_error(int e);

// Kernel launches issued by the library (incremented at every launch site).
void count_launch(uint64_t n = 1);
uint64_t launches_total();

template <class RT>
cudaError_t outer_sample_level(const OuterLevel<RT>& L, int kind, int prec, OuterBuffers& B,
                               TraceRec* trace, cudaStream_t stream);
cudaError_t outer_level_begin(OuterBuffers& B, cudaStream_t stream);
cudaError_t launch_stamp(uint64_t* slot, cudaStream_t stream);   // %globaltimer -> *slot

// Portfolio loss sweep L(Y) over all options (K-quantile precompute).
template <class RT>
cudaError_t outer_full_loss(const OuterLevel<RT>& L, int prec, OuterBuffers& B, double* d_loss,
                            cudaStream_t stream);

// ---- path-simulated loss and its adjoint (nmlmc_adjoint.cu) --------------------------------
constexpr uint32_t kAdjMaxTile = 64;     // outer samples per CTA of the path kernels

template <class RT>
struct AdjLaunch {
    uint32_t n, n_chunks, q_max;          // portfolios, option chunks of 128, max stocks per portfolio
    uint32_t ell, pairs, tile;            // 2^ell steps, antithetic pairs, outer samples per CTA
    uint64_t M, seed;
    int milstein;
    RT r, rho, s1_rho2, tau, stau, disc_tau;
    const uint32_t *stock_off, *option_off, *chunk_off;   // [n + 1]
    const RT *S0, *mu, *sigma;                             // [stocks]
    const RT *strike, *maturity, *w, *V0, *vega;           // [options]
    const uint32_t* stock_ind;                             // [options], within the portfolio
    const int8_t* type;
    const double *K, *delta;                               // [n]
    RT *R, *dR;                                            // [stocks * M], row (p, m) of Q_p values
    double *L, *omega, *est, *wE;                          // [n * M], [n * M], [3 n], [n]
    double *gw_E, *gw_P, *gs_E, *gs_P;                     // [options], [stocks]
};
cudaError_t launch_adjoint(const AdjLaunch<float>& A, bool grad, cudaStream_t stream);
cudaError_t launch_adjoint(const AdjLaunch<double>& A, bool grad, cudaStream_t stream);

cudaError_t launch_threefry_blocks(const uint64_t* ctr, const uint64_t* key, uint64_t* out, uint64_t n,
                                   cudaStream_t s);
cudaError_t launch_norm_cdf_fast(const float* x, float* out, uint64_t n, cudaStream_t s);
cudaError_t launch_outer_normals(int prec, uint64_t seed, uint64_t stream, uint32_t tag, uint64_t n,
                                 double* out, cudaStream_t s);

}  // namespace nmlmc
