/* nmlmc — B200-native nested MLMC level sampler: the C ABI.
 *
 * Two layers:
 *
 *  1. Drop-in entry points with the names, argument meaning and struct layouts of the
 *     reference's extern "C" surface (haji-ali/nested-risk-mlmc; "meant to be used in python",
 *     common.hpp:34-36), operating on one process-wide sampler as the reference does.  The
 *     structs mirror the reference's default build (real_t = float).  Where the reference
 *     exit()s on a CUDA error (par_nvcc.hpp:46-54) these record the error, print it to stderr
 *     and return; nmlmc_last_error() reports it.
 *
 *  2. The native API (nmlmc_*): explicit context, int status returns, double-precision inputs,
 *     precision / stream-layout selection, batched multi-level sampling and the host MLMC driver.
 *
 * Plain C: no torch or CUDA types appear in any signature.
 */
#ifndef NMLMC_H
#define NMLMC_H

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------------ */
enum {
    NMLMC_OK = 0,
    NMLMC_ERR_ARG = 1,        /* invalid argument (also: unsupported configuration)       */
    NMLMC_ERR_CUDA = 2,       /* a CUDA runtime call failed                                */
    NMLMC_ERR_STATE = 3,      /* call out of order (no model / portfolio set, no context),
                                 a level sampler that failed, or sampler-state / checkpoint
                                 I/O that failed                                           */
    NMLMC_ERR_NOMEM = 4,      /* device or host allocation failed                          */
    NMLMC_ERR_TIMEOUT = 5,    /* a bounded device wait gave up                             */
    NMLMC_ERR_LIMIT = 6       /* a path-simulated inner sample drew a level whose step count
                                 h0 beta^L exceeds NMLMC_MAX_PATH_STEPS (the call stops)   */
};

/* Time steps one Unbiased-method inner sample may take (P(L) ~ beta^(e L): at h0 = 8,
 * beta = 4, e = -1.5 a draw above the limit has probability about 1e-10). */
#define NMLMC_MAX_PATH_STEPS (1ull << 24)

enum { NMLMC_PREC_REF32 = 0, NMLMC_PREC_FP64 = 1, NMLMC_PREC_FP32 = 2 };
enum { NMLMC_STREAMS_CORE = 0, NMLMC_STREAMS_OUTER = 1 };
enum { NMLMC_MODEL_REFERENCE = 0, NMLMC_MODEL_SHIFT = 1 };
enum { NMLMC_SUB_NONE = 0, NMLMC_SUB_RANDOM = 1, NMLMC_SUB_UNIFORM = -1 };

/* ================================================================================================
 * 1. Reference-compatible surface
 * ============================================================================================== */

/* nested_sampler_params (nested_sampler.hpp:14-34), real_t = float. */
typedef struct nested_sampler_params {
    uint32_t N0;
    uint32_t beta;
    bool antithetic;
    uint32_t fine_moments;
    uint32_t diff_moments;
    float adaptive_r;
} nested_sampler_params;

/* sample_output (common.hpp:37-55): the caller owns fsums / diffsums (phi_size x moments). */
typedef struct sample_output {
    uint64_t M;
    double* fsums;
    double* diffsums;
    double total_work;
    uint64_t inner_stats[6];
} sample_output;

/* model::data (model_sampler.cpp:21-39). */
typedef struct model_data {
    float stau;       /* sqrt(tau)   */
    float s1tau;      /* sqrt(1-tau) */
    float max_loss;
    int32_t phi_type; /* 0 Indicator (the only phi on this path) */
} model_data;

/* portfolio::option_params / stock_params / data (portfolio_sampler.cpp:42-92). */
typedef struct option_params {
    float strike, maturity, start, w, delta_est;
    uint32_t stock_ind;
    int32_t type;     /* +1 call, -1 put */
    float prob;
    float W_est;
} option_params;

typedef struct stock_params { float S0, mu, sigma; } stock_params;
typedef struct { option_params* data; size_t size; } nmlmc_options_span;
typedef struct { stock_params* data; size_t size; } nmlmc_stocks_span;

typedef struct portfolio_data {
    nmlmc_options_span options[3];   /* ComputeMethod::BS, Exact, Unbiased                      */
    nmlmc_stocks_span stocks;
    float r, rho, s1_rho2;
    float max_loss;
    float tau;
    uint32_t dt_h0inv;
    uint32_t dt_beta;
    float dt_prob_expo;
    int32_t phi_type;
    uint32_t _phi_size;
    int32_t subsample;               /* NMLMC_SUB_*                                             */
    bool use_delta_cv;
    bool use_coarse_delta_cv;
    bool use_antithetic_risk;
    bool use_milstein;
} portfolio_data;

/* init_nestedmc_sampler / cleanup_nestedmc_sampler (common.cpp:20-31). `cores` is the number
 * of virtual cores: core c draws from the Threefry streams keyed (seed, c) and takes OpenMP's
 * static share of each call's outer samples, so cores = OMP_NUM_THREADS reproduces the
 * reference CPU build's draws. */
void init_nestedmc_sampler(uint32_t cores, const nested_sampler_params* params);
void cleanup_nestedmc_sampler(void);

/* model_update_data / model_init / model_sample (model_sampler.cpp:94-114). */
void model_update_data(const model_data* data);
void model_init(const model_data* data, uint64_t seed);
void model_sample(uint32_t ell, uint64_t M, sample_output* out);

/* portfolio_update_data / portfolio_init / portfolio_sample / portfolio_cleanup /
 * portfolio_comp_params (portfolio_sampler.cpp:618-756).  options[0..2] hold the BS, Exact and
 * Unbiased options (portfolio_sampler.cpp:17-22); Exact / Unbiased options are sampled on the
 * CORE streams (the reference-surface default). */
void portfolio_update_data(const portfolio_data* data);
void portfolio_init(const portfolio_data* data, uint64_t seed);
void portfolio_sample(uint32_t ell, uint64_t override_dyn_inner, uint64_t M, sample_output* out);
void portfolio_cleanup(void);
void portfolio_comp_params(portfolio_data* data);
/* portfolio_gen_data / portfolio_free_data (portfolio_sampler.cpp:784-912): the reference demo
 * main's portfolio, with the reference's values for the same arguments.  Q stocks, P >= 2Q
 * options; options[m] gets floor(probs[m] * P) of them (m = BS, Exact, Unbiased; the three
 * must add up to P), delta-hedged per stock, weights normalised to sum 1, prob = |w| (1 with
 * uniform_prob), each method sorted by decreasing prob.  uniform_weights starts every weight at
 * 1.  The arrays belong to the library until portfolio_free_data; invalid arguments return a
 * zeroed portfolio_data and set nmlmc_last_error(). */
portfolio_data portfolio_gen_data(uint32_t P, uint32_t Q, uint64_t seed, double* probs,
                                  bool uniform_weights, bool uniform_prob);
void portfolio_free_data(portfolio_data* data);

/* norm_cdf_inv (common.cpp:53-86). */
float norm_cdf_inv(float p);

/* Status of the last reference-surface call (or allocation-free level call), and the precision
 * used by the reference surface (NMLMC_PREC_REF32 unless nmlmc_default_set_precision changes it). */
int nmlmc_last_error(void);
int nmlmc_default_set_precision(int32_t precision, int32_t streams);

/* ================================================================================================
 * 2. Native API
 * ============================================================================================== */
typedef struct nmlmc_ctx nmlmc_ctx;

typedef struct nmlmc_config {
    uint32_t cores;            /* virtual cores of the CORE layout (0 -> 2048)                  */
    uint32_t N0;               /* inner samples at level 0                                      */
    uint32_t beta;             /* inner refinement factor (power of two)                         */
    double adaptive_r;         /* adaptive exponent r; adaptive iff 1 < r < 2 (or <= 2, below)   */
    int32_t antithetic;        /* antithetic coarse estimator                                   */
    int32_t adaptive_incl_r2;  /* 1: treat r = 2 as adaptive (the 3-sigma doubling rule)         */
    int32_t precision;         /* NMLMC_PREC_*                                                   */
    int32_t streams;           /* NMLMC_STREAMS_*                                                */
    uint64_t seed;
    uint64_t batch;            /* OUTER layout: outer samples per batch (0: grows with the calls
                                  up to 1<<24; portfolios: at most 1 GiB of R_tau rows)        */
} nmlmc_config;

typedef struct nmlmc_level_result {
    double fsums[4];           /* sum of phi_f^k, k = 1..4                                      */
    double diffsums[4];        /* sum of (phi_f - phi_c)^k (zero at level 0)                    */
    double total_work;
    uint64_t M;
    uint64_t inner_stats[6];   /* inner samples, decisions, hit max, hit base, #randu, #randn */
    double seconds;            /* device time of the level: CUDA events around a single call;
                                  inside a round's graph, %globaltimer stamps at its boundaries */
} nmlmc_level_result;

typedef struct nmlmc_portfolio {
    uint32_t Q, P;                        /* stocks, options                                 */
    const double *S0, *mu, *sigma;        /* [Q]                                             */
    const double *strike, *maturity, *w;  /* [P]                                             */
    const double* prob;                   /* [P], positive, non-increasing; NULL = all 1     */
    const uint32_t* stock_ind;            /* [P]                                             */
    const int32_t* type;                  /* [P] +1 call / -1 put                            */
    double r, rho, max_loss, tau;
    int32_t subsample;                    /* NMLMC_SUB_*                                     */
    int32_t use_delta_cv;
    int32_t discount;                     /* 1: finish value discounted by exp(-r tau)       */
} nmlmc_portfolio;

/* Seeded synthetic portfolio: Q stocks with spot S0, drift mu and sigma ~ U[sigma_lo, sigma_hi];
 * P options, each on a uniformly chosen stock, a call with probability call_fraction, strike ~
 * U[strike_lo, strike_hi] * S0, maturity ~ U[maturity_lo, maturity_hi], position ~ N(0, 1).
 * Every field comes from a counter-based Threefry2x64-20 stream keyed by the seed, so the
 * portfolio depends only on (spec, seed).  No counterpart in the reference (whose demo generator,
 * portfolio_gen_data, builds a different portfolio).  Arrays are caller-owned ([Q] and [P]). */
typedef struct nmlmc_portfolio_spec {
    uint32_t Q, P;
    double S0, r, mu;
    double sigma_lo, sigma_hi;
    double strike_lo, strike_hi;
    double maturity_lo, maturity_hi;
    double call_fraction;
} nmlmc_portfolio_spec;
int nmlmc_portfolio_generate(const nmlmc_portfolio_spec* spec, uint64_t seed, double* S0,
                             double* mu, double* sigma, double* strike, double* maturity,
                             double* w, uint32_t* stock_ind, int32_t* type);

/* Per-outer-sample record written by nmlmc_sample when a trace buffer is armed. */
typedef struct nmlmc_trace_rec {
    uint64_t count_f, count_c;
    double phi_f, phi_c;
    double mean_big, min_abs_small;
    uint32_t core, pilots;
} nmlmc_trace_rec;

const char* nmlmc_error_string(int status);
int nmlmc_version(void);

/* A context replaces the reference's process-wide sampler state (g_p_nestedmc_data and the
 * __constant__ parameters, common.cpp:15-31): create / destroy ~ init_nestedmc_sampler /
 * cleanup_nestedmc_sampler, configure ~ nested_sampler_params (nested_sampler.hpp:14-34) plus
 * the precision and stream layout. */
int nmlmc_create(nmlmc_ctx** out, int device);
int nmlmc_destroy(nmlmc_ctx* ctx);
int nmlmc_configure(nmlmc_ctx* ctx, const nmlmc_config* cfg);
/* model_init (model_sampler.cpp:99-104) with the model's data (model_sampler.cpp:21-39).
 * kind NMLMC_MODEL_REFERENCE: model::sampler with tau, max_loss;
 * kind NMLMC_MODEL_SHIFT: Y ~ N(0,1), inner X = Y + Z, threshold K = max_loss. */
int nmlmc_set_model(nmlmc_ctx* ctx, int32_t kind, double tau, double max_loss);
/* portfolio_comp_params + portfolio_init (portfolio_sampler.cpp:618-756) from structure-of-arrays
 * doubles; out_start / out_delta_est receive the options' start values and delta estimates. */
int nmlmc_set_portfolio(nmlmc_ctx* ctx, const nmlmc_portfolio* pf, double* out_start,
                        double* out_delta_est);
/* Path-simulated inner values (portfolio_sampler.cpp:74-87, 470-604; gbm_approx.hpp:18-57):
 * method[j] = 0 BS, 1 Exact (exact GBM from tau to maturity), 2 Unbiased (randomised
 * Milstein / Euler level L, P(L) proportional to dt_beta^(dt_prob_expo L), h0 dt_beta^L steps).
 * Options are grouped by method in the caller's order; prob must be non-increasing within each
 * method.  Sampling with Exact / Unbiased options needs the CORE stream layout. */
typedef struct nmlmc_path_methods {
    const int32_t* method;                /* [P]                                             */
    uint32_t dt_h0inv, dt_beta;           /* h0 = 1 / dt_h0inv steps at L = 0; beta >= 2     */
    double dt_prob_expo;                  /* < 0                                             */
    int32_t use_coarse_delta_cv, use_antithetic_risk, use_milstein;
} nmlmc_path_methods;
int nmlmc_set_portfolio_methods(nmlmc_ctx* ctx, const nmlmc_portfolio* pf, const nmlmc_path_methods* pm,
                                double* out_start, double* out_delta_est);
/* ---- path-simulated loss and its adjoint (no counterpart in the reference) --------------------
 * A batch of n portfolios evaluated in one launch.  Portfolio p owns stocks
 * [stock_off[p], stock_off[p+1]) and options [option_off[p], option_off[p+1]); stock_ind is the
 * stock's index within its portfolio.  For outer sample m of portfolio p (OUTER-layout key
 * (seed, ell<<56 | p<<32 | m): at p = 0 the outer draws of nmlmc_portfolio_full_loss):
 *   L_m = sum_i w_i (V_i(0) - e^{-r tau} C_i(m)),
 *   C_i(m) = e^{-r (T_i - tau)} (1/N) sum_n (pay(S+_n) + pay(S-_n)) / 2,
 * S+-_n an antithetic pair of Milstein (or Euler) paths on 2^ell steps from (tau, R_tau) to T_i
 * under the risk-neutral drift, N = inner_pairs.  Estimates per portfolio: E[L], the smoothed
 * exceedance P_delta = E[1 / (1 + exp(-(L - K) / delta))] with delta = delta_rel |K| (delta_rel
 * when K = 0), and the plain frequency of L > K.  Gradients (pathwise, inner draws recomputed from
 * the counter RNG): dE[L]/dw_i, dP_delta/dw_i, dE[L]/dsigma_j, dP_delta/dsigma_j. */
typedef struct nmlmc_portfolio_batch {
    uint32_t n;
    const uint32_t *stock_off, *option_off;        /* [n + 1]                                  */
    const double *S0, *mu, *sigma;                 /* [stock_off[n]]                           */
    const double *strike, *maturity, *w;           /* [option_off[n]]; maturity > tau          */
    const uint32_t* stock_ind;                     /* [option_off[n]]                          */
    const int32_t* type;                           /* [option_off[n]] +1 call / -1 put          */
    const double* K;                               /* [n] loss thresholds                      */
    double r, rho, tau;
} nmlmc_portfolio_batch;
typedef struct nmlmc_adjoint_config {
    uint32_t ell;            /* 2^ell time steps from tau to maturity (ell <= 16)               */
    uint32_t inner_pairs;    /* antithetic path pairs per option and outer sample               */
    uint64_t M;              /* outer samples per portfolio (< 2^32)                            */
    double delta_rel;        /* sigmoid width relative to |K|                                   */
    int32_t precision;       /* NMLMC_PREC_FP32 (FP32 paths, FP64 sums) or NMLMC_PREC_FP64      */
    int32_t milstein;        /* 1 Milstein, 0 Euler-Maruyama                                    */
    uint64_t seed;
} nmlmc_adjoint_config;
typedef struct nmlmc_adjoint_result {
    double EL, P_smooth, P_hard;
} nmlmc_adjoint_result;
/* res [n] required; gradients [options] / [stocks] and loss [n * M] may be NULL (all four
 * gradient pointers NULL: the loss pass only).  seconds: device time of the kernels (may be NULL). */
int nmlmc_path_adjoint(nmlmc_ctx* ctx, const nmlmc_portfolio_batch* batch, const nmlmc_adjoint_config* cfg,
                       nmlmc_adjoint_result* res, double* grad_w_EL, double* grad_w_P,
                       double* grad_sigma_EL, double* grad_sigma_P, double* loss, double* seconds);
/* Restart every stream, as init_samplers does (nested_sampler.hpp:618-643; CORE:
 * random_state(seed, core) from counter 0; OUTER: outer indices from 0). */
int nmlmc_reset_streams(nmlmc_ctx* ctx);
/* One level: M outer samples at level ell (sample<SAMPLER>, nested_sampler.hpp:646-694). */
int nmlmc_sample(nmlmc_ctx* ctx, uint32_t ell, uint64_t M, nmlmc_level_result* out);
/* Several levels in one submission.  OUTER layout: the levels' launch sequences are captured
 * into one CUDA graph (kept and updated in place while the topology repeats), each level summing
 * into its own slot, one device->host copy and one synchronisation for the round; levels run one
 * after another inside the graph.  Up to 64 levels; with tracing or phase profiling armed, or on
 * the CORE layout, the levels run as consecutive nmlmc_sample calls. */
int nmlmc_sample_levels(nmlmc_ctx* ctx, uint32_t n, const uint32_t* ells, const uint64_t* Ms,
                        nmlmc_level_result* outs);
/* ---- phase-kernel autotuner (batched FP32 path) ----------------------------------------------
 * No counterpart in the reference (its CUDA build has one fixed launch shape).  The phase kernel
 * of the OUTER layout has three register/occupancy variants (0: up to 255 registers per thread,
 * 1: three resident CTAs of 256 threads per SM guaranteed, 2: four), for portfolios a fourth (3: two
 * CTAs per SM, with the next inner samples' table gathers issued before the current ones are
 * evaluated; other kinds run variant 0 for it) and a chunk length (inner
 * samples per thread; power of two in [4, 64] dividing N0; a level's items of n inner samples
 * take n / chunk threads, so it also sets the outer samples per warp).  With autotuning on, the
 * first nmlmc_sample / nmlmc_sample_levels call of a level with enough work times the
 * candidates on a probe of the level's own parameters whose outer stream indices start at 2^55
 * (no result changes) and keeps the fastest for that level in the context.  Mode 1 (the
 * default) tunes the variant only; the variants give identical results.  Mode 2 also tries half
 * and double the chunk length; another chunk length regroups the FP32 compensated inner sums
 * (last-bit differences of inner means), so pin the configuration to make such runs reproducible
 * across processes.  Changing the model, portfolio or configuration drops the tuned (not the
 * pinned) choices.  Tuning applies to NMLMC_PREC_FP32 only. */
typedef struct nmlmc_phase_config {
    uint32_t variant;          /* 0, 1, 2, 3 (above)                                             */
    uint32_t chunk;            /* inner samples per thread                                       */
    int32_t state;             /* get: 0 default, 1 autotuned, 2 pinned                          */
    double probe_ms;           /* get: device time of the tuned choice on its probe              */
} nmlmc_phase_config;
int nmlmc_set_autotune(nmlmc_ctx* ctx, int32_t mode);   /* 0 off, 1 variants (default), 2 + chunk */
int nmlmc_get_phase_config(nmlmc_ctx* ctx, uint32_t ell, nmlmc_phase_config* out);
/* Pins level ell's configuration (cfg == NULL unpins it: default, tunable again). */
int nmlmc_set_phase_config(nmlmc_ctx* ctx, uint32_t ell, const nmlmc_phase_config* cfg);
/* Tunes level ell now, variant and chunk length, on a probe of about 20 ms of device time (at
 * most one batch of outer samples; the batch buffers grow to M first) — replaces a tuned or
 * pinned choice. */
int nmlmc_autotune_level(nmlmc_ctx* ctx, uint32_t ell, uint64_t M);

/* Fault injection for tests (no counterpart in the reference): after `after` more successful
 * device allocations by the library, the next one fails as if the device were out of memory;
 * -1 switches it off.  The failing call returns NMLMC_ERR_NOMEM and the context stays usable. */
int nmlmc_inject_alloc_failure(int32_t after);

/* CUDA graphs of nmlmc_sample_levels: instantiated, updated in place, launched. */
int nmlmc_graph_stats(nmlmc_ctx* ctx, uint64_t* instantiations, uint64_t* updates, uint64_t* launches);
/* Arms a host buffer of `cap` records for the next nmlmc_sample call (M <= cap). */
int nmlmc_set_trace(nmlmc_ctx* ctx, nmlmc_trace_rec* host_buf, uint64_t cap);
/* Full portfolio loss L(Y) for outer samples [first, first + n) of level `ell` (OUTER layout
 * streams): sum_i w_i (V_i(0) - disc V_i(tau, S_tau)). */
int nmlmc_portfolio_full_loss(nmlmc_ctx* ctx, uint32_t ell, uint64_t first, uint64_t n,
                              double* host_loss);

/* Sharding over ranks (OUTER layout): each nmlmc_sample(ell, M) call then evaluates only this
 * rank's contiguous share of the call's M outer samples (ranks below M mod world take
 * floor(M / world) + 1 of them, the others floor(M / world)), with the stream indices a single
 * device would give them; the caller sums the ranks' level results (an all-reduce of
 * 16 doubles) and gets the single-device result.  world = 1 restores the default. */
int nmlmc_set_shard(nmlmc_ctx* ctx, uint32_t rank, uint32_t world);
/* CUDA-event timing of the phase kernel (the dominant kernel): 1 enables; the totals since
 * enabling are read with nmlmc_phase_kernel_time. */
int nmlmc_set_profiling(nmlmc_ctx* ctx, int32_t on);
int nmlmc_phase_kernel_time(nmlmc_ctx* ctx, uint64_t* launches, double* seconds);
/* Number of kernels this library has launched since it was loaded. */
uint64_t nmlmc_kernel_launches(void);

/* Threefry2x64-20 blocks computed on the GPU: out[2i..2i+1] = F(ctr[2i..2i+1], key[2i..2i+1])
 * (host buffers).  Bit-identical to Random123's r123::Threefry2x64. */
int nmlmc_threefry_blocks(const uint64_t* ctr, const uint64_t* key, uint64_t* out, uint64_t n);
/* Normals k = 0..n-1 of one OUTER-layout phase (key (seed, stream), counter namespace `tag`)
 * computed on the GPU at `precision` (NMLMC_PREC_FP64 or NMLMC_PREC_FP32), widened to double. */
int nmlmc_outer_normals(int32_t precision, uint64_t seed, uint64_t stream, uint32_t tag, uint64_t n,
                        double* out);
/* Phi(x) of the FP32 Black-Scholes path (rational erfc on the SFU) at n points (host buffers). */
int nmlmc_norm_cdf_fast(const float* x, float* out, uint64_t n);

/* ---- allocation-free level call ------------------------------------------------------------
 * No counterpart in the reference.  For callers that may not allocate device memory: code that
 * runs while a framework owns the device memory pool, latency-critical code that cannot afford
 * cudaMalloc's implicit device-wide synchronisation, hosts that reserve all device memory up
 * front.  One level call of the model problem
 * (kind NMLMC_MODEL_REFERENCE or NMLMC_MODEL_SHIFT; the OUTER stream layout, precision
 * NMLMC_PREC_FP32 or NMLMC_PREC_FP64, antithetic) over outer samples [first_index,
 * first_index + M) of level `ell`, on `stream` (a cudaStream_t; NULL = the default stream) of the
 * current device.  It allocates nothing: all scratch lives in one file-scope device array of
 * NMLMC_NOALLOC_SCRATCH_BYTES that every process loading this library reserves on each GPU it
 * uses until exit, which limits a call to M <= NMLMC_NOALLOC_MAX_OUTER (larger M is rejected
 * with NMLMC_ERR_ARG).  The first call on a device looks the array's device address up
 * (cudaGetSymbolAddress), so make that first call before any stream capture; that address is
 * kept for the life of the process, so a device reset (cudaDeviceReset, or a destroyed primary
 * context) after the first call is not supported.  Calls share the array — each clears what it
 * accumulates into, but calls that overlap on the GPU race.  Failures return a status and set
 * nmlmc_last_error(), with the input checks of nmlmc_set_model and nmlmc_sample.
 * d_out (device memory, 16 doubles) receives: sums of phi_f^k (k = 1..4), sums of
 * (phi_f - phi_c)^k, work, inner samples, outer samples that hit the maximum count, outer
 * samples that stayed at the base count, and 4 zeros.  The copy into d_out is ordered on
 * `stream`; synchronize the stream before reading it. */
#define NMLMC_NOALLOC_MAX_OUTER 65536u
#define NMLMC_NOALLOC_SCRATCH_BYTES (3u << 20)
int nmlmc_sample_level_noalloc(int32_t kind, double tau, double max_loss, uint32_t N0,
                               uint32_t beta, double adaptive_r, int32_t adaptive_incl_r2,
                               int32_t precision, uint64_t seed, uint32_t ell,
                               uint64_t first_index, uint64_t M, double* d_out, void* stream);

/* ---- host continuation-MLMC driver (mlmc_t::run, mlmc.hpp:290-337) ------------------------- */
typedef struct nmlmc_mlmc_input {
    double targetTOL;              /* 1e-3 */
    double startTOL;               /* 0.5  */
    double theta;                  /* 0.5  */
    double starting_level_coeff;   /* 1.5  */
    double Ca;                     /* 3    */
    uint64_t M0;                   /* 100  */
    int32_t verbose;               /* print the reference's "# Sampling" lines and tables */
    uint32_t max_levels;           /* the run stops with NMLMC_ERR_ARG when it would need
                                      more levels (0: NMLMC_MAX_LEVELS = 64)               */
    int32_t batched;               /* 1: one nmlmc_sample_levels submission per round      */
    uint32_t max_iterations;       /* stop after this many completed TOL iterations (0: run
                                      to targetTOL); with a checkpoint, resume later        */
} nmlmc_mlmc_input;

#define NMLMC_MAX_LEVELS 64
typedef struct nmlmc_mlmc_output {
    uint32_t nlevels, starting_level;
    double bias_est, stat_error, TOL, Eg;
    double total_work, total_time;          /* total_time: wall seconds of the run          */
    uint64_t calls;                          /* sample_level invocations                     */
    uint64_t level_M[NMLMC_MAX_LEVELS];
    double level_fsums[NMLMC_MAX_LEVELS][4];
    double level_diffsums[NMLMC_MAX_LEVELS][4];
    double level_work[NMLMC_MAX_LEVELS];
    double level_time[NMLMC_MAX_LEVELS];
    uint32_t iterations_done;               /* TOL iterations completed, resumed ones included */
    uint32_t complete;                      /* 1: targetTOL reached; 0: stopped by max_iterations */
} nmlmc_mlmc_output;

typedef void (*nmlmc_sample_level_fn)(void* user, uint32_t ell, uint64_t M,
                                      nmlmc_level_result* out);
typedef void (*nmlmc_sample_levels_fn)(void* user, uint32_t n, const uint32_t* ells,
                                       const uint64_t* Ms, nmlmc_level_result* outs);

nmlmc_mlmc_input nmlmc_mlmc_default_input(void);
/* The runs below return NMLMC_ERR_ARG before any sample call unless targetTOL and startTOL are
 * finite with 0 < targetTOL <= startTOL, 0 < theta < 1, Ca > 0 and M0 >= 1 (other values ask for a
 * loop that does not end or has no samples).  During a run, a level result with a non-finite sum
 * or work (or M = 0) stops it with NMLMC_ERR_STATE; a level that would need 2^62 or more samples,
 * or a level beyond max_levels, stops it with NMLMC_ERR_ARG. */
/* Runs the continuation MLMC with the GPU sampler of `ctx`.  `table` (may be NULL) receives the
 * final to_string() table of the reference's mlmc_output_t. */
int nmlmc_mlmc_run(nmlmc_ctx* ctx, const nmlmc_mlmc_input* in, nmlmc_mlmc_output* out,
                   char* table, size_t table_cap);
/* Same driver over caller-provided level samplers (levels_fn may be NULL). */
int nmlmc_mlmc_run_cb(const nmlmc_mlmc_input* in, nmlmc_sample_level_fn level_fn,
                      nmlmc_sample_levels_fn levels_fn, void* user, nmlmc_mlmc_output* out,
                      char* table, size_t table_cap);

/* ---- checkpoint / resume of the driver ----------------------------------------------------
 * No counterpart in the reference (its mlmc_t::run keeps the state in memory only).  After
 * every completed TOL iteration the driver writes `path` (atomically: a temporary file renamed
 * over it): the input parameters, the iteration state (next iteration, TOL, starting level,
 * calls) and every level's FP64 sums (M, sum phi_f^k, sum dphi^k, work, time), followed by the
 * sampler's state (`save`; for nmlmc_mlmc_run_ckpt the context's stream positions).  With
 * `resume` set and `path` present, a run whose input parameters (targetTOL, startTOL, theta,
 * starting_level_coeff, Ca, M0) equal the saved ones continues at the saved iteration with the
 * saved sums and sampler state, and ends exactly as the uninterrupted run would (on the FP32
 * batched path: with autotuning in mode 0 or 1, or chunk lengths pinned, since a fresh context
 * tunes again and another chunk length regroups the FP32 inner sums); otherwise it
 * warm-starts: the saved level sums seed a run of the new parameters from its first iteration.
 * The file is little-endian: "NMLMCCK1", u32 version = 1, u32 header bytes, then the fields in
 * the order above (nmlmc/checkpoint.py reads it). */
/* save(user, NULL, 0) returns the bytes needed, save(user, buf, cap) writes them and returns
 * the count; (size_t)-1 reports a failure (the run stops with NMLMC_ERR_STATE).  load returns
 * NMLMC_OK or an error status. */
typedef size_t (*nmlmc_state_save_fn)(void* user, void* buf, size_t cap);
typedef int (*nmlmc_state_load_fn)(void* user, const void* buf, size_t size);
typedef struct nmlmc_checkpoint_io {
    const char* path;              /* NULL: no checkpoint                                   */
    int32_t resume;                /* 1: start from `path` when it exists                    */
    nmlmc_state_save_fn save;      /* optional sampler state stored in the checkpoint        */
    nmlmc_state_load_fn load;
} nmlmc_checkpoint_io;
int nmlmc_mlmc_run_cb_ckpt(const nmlmc_mlmc_input* in, nmlmc_sample_level_fn level_fn,
                           nmlmc_sample_levels_fn levels_fn, void* user, const nmlmc_checkpoint_io* io,
                           nmlmc_mlmc_output* out, char* table, size_t table_cap);
/* The GPU driver with checkpoints: the sampler state saved is the context's (below). */
int nmlmc_mlmc_run_ckpt(nmlmc_ctx* ctx, const nmlmc_mlmc_input* in, const char* path, int32_t resume,
                        nmlmc_mlmc_output* out, char* table, size_t table_cap);

/* Sampler state of a context: its configuration (checked on restore), the OUTER layout's next
 * outer-sample index per level and, on the CORE layout, every virtual core's two stream states.
 * nmlmc_get_sampler_state writes at most `cap` bytes and reports the size needed in *size
 * (buf may be NULL to query it). */
int nmlmc_get_sampler_state(nmlmc_ctx* ctx, void* buf, size_t cap, size_t* size);
int nmlmc_set_sampler_state(nmlmc_ctx* ctx, const void* buf, size_t size);

#ifdef __cplusplus
}
#endif
#endif /* NMLMC_H */
