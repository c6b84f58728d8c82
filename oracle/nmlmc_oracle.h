/* CPU oracle for the nested MLMC level sampler — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's level-sampler algorithm (haji-ali/nested-risk-mlmc),
 * used by tests/, by __graft_entry__.smoke() and by bench.py's cpu_baseline leg as the checker.
 * The product never links or loads this library.
 *
 * Parity: pinned against the unmodified reference compiled here (oracle/_ref, built by
 * oracle/Makefile from the reference sources) through the golden fixtures under tests/golden/
 * (tests/golden/make_golden.py).  Every function cites the reference file:line it follows.
 *
 * Two random-stream layouts are restated:
 *   O_STREAMS_CORE  — the reference CPU build: virtual core c owns random_state(seed, c) for both
 *                     its sync and inner streams (nested_sampler.hpp:634-642), outer samples are
 *                     split over cores by OpenMP's static schedule (nested_sampler.hpp:417) and
 *                     the streams persist across sample() calls.
 *   O_STREAMS_OUTER — the order-independent layout used by the batched GPU path: one
 *                     Threefry2x64-20 key per outer sample, one counter namespace per phase,
 *                     32-bit words.  Not a reference layout (the reference has no such mode); it
 *                     is restated here so the GPU path has a CPU checker on the same streams.
 */
#ifndef NMLMC_ORACLE_H
#define NMLMC_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { O_PREC_REF32 = 0, O_PREC_FP64 = 1 };          /* real_t = float / double            */
enum { O_STREAMS_CORE = 0, O_STREAMS_OUTER = 1 };
enum { O_MODEL_REFERENCE = 0, O_MODEL_SHIFT = 1 };   /* model::sampler / X = Y + Z model  */
enum { O_SUB_NONE = 0, O_SUB_RANDOM = 1, O_SUB_UNIFORM = -1 };

/* Per-outer-sample record (identical layout in the GPU library's trace buffer). */
typedef struct {
    uint64_t count_f, count_c;   /* final inner counts (count_c = 0 when fine only)          */
    double phi_f, phi_c;         /* phi of the fine / coarse inner estimate                  */
    double mean_big;             /* inner mean whose phi is the bigger-count term            */
    double min_abs_small;        /* min |inner mean| over the small groups (inf: none)       */
    uint32_t core, pilots;       /* virtual core (CORE layout) / pilot rounds taken          */
} o_trace_rec;

/* Event log in the format of oracle/ref_harness.cpp: 'O' outer, 'I' init_inner(count),
 * 'P' add_phi(mean, coeff). */
typedef struct { char *kinds; double *values, *aux; uint64_t cap, n; } o_events;

void o_threefry2x64(const uint64_t ctr[2], const uint64_t key[2], uint64_t out[2]);
void o_threefry_batch(const uint64_t *ctr, const uint64_t *key, uint64_t *out, uint64_t n);
void o_stream_draws(int prec, uint64_t seed, uint64_t core, const char *ops, uint64_t n,
                    double *out_real, uint64_t *out_u64);
void o_boxmuller(const uint64_t *u0, const uint64_t *u1, double *x, double *y, uint64_t n);

typedef struct o_ctx o_ctx;
/* adaptive_incl_r2: 0 = the reference predicate 1 < r < 2 (nested_sampler.hpp:33),
 * 1 = 1 < r <= 2 (the r = 2 rule "double while |mean-K| < 3 sigma/sqrt(N)"). */
o_ctx *o_create(int prec, int streams, uint32_t cores, uint32_t N0, uint32_t beta,
                double adaptive_r, int antithetic, int adaptive_incl_r2, uint64_t seed);
void o_destroy(o_ctx *);
/* OUTER layout sharding: each o_sample(ell, M) evaluates the rank's static share of the M outer
 * samples with their single-device stream indices (the semantics of nmlmc_set_shard). */
void o_set_shard(o_ctx *, uint32_t rank, uint32_t world);
/* With buf set, every o_sample call writes buf[m] for its outer sample m: the smallest
 * |ln(new_count / cur)| over that sample's adaptive decisions (get_samples_count's test
 * new_count <= cur, nested_sampler.hpp:262-266), +inf if it took none.  Test instrumentation:
 * how far an FP64 decision was from flipping. */
void o_set_margins(o_ctx *, double *buf);
void o_set_model(o_ctx *, int kind, double tau, double max_loss);
/* Portfolio of BS options (ComputeMethod::BS only).  start/delta_est are computed as
 * portfolio_comp_params does (portfolio_sampler.cpp:687-700) and returned. */
int o_set_portfolio(o_ctx *, uint32_t Q, const double *S0, const double *mu, const double *sigma,
                    uint32_t P, const double *strike, const double *maturity, const double *w,
                    const uint32_t *stock_ind, const int32_t *type, const double *prob,
                    double r, double rho, double max_loss, double tau, int subsample,
                    int use_delta_cv, int discount, double *out_start, double *out_delta_est);
/* Mixed compute methods (portfolio_sampler.cpp:17-22): method[j] = 0 BS, 1 Exact, 2 Unbiased.
 * Options are grouped by method in the order given (prob non-increasing within a method), as
 * portfolio::data.options[3] holds them.  CORE layout only. */
int o_set_portfolio_methods(o_ctx *, uint32_t Q, const double *S0, const double *mu,
                            const double *sigma, uint32_t P, const double *strike,
                            const double *maturity, const double *w, const uint32_t *stock_ind,
                            const int32_t *type, const double *prob, const int32_t *method,
                            double r, double rho, double max_loss, double tau, int subsample,
                            int use_delta_cv, int use_coarse_delta_cv, int use_antithetic_risk,
                            int use_milstein, uint32_t dt_h0inv, uint32_t dt_beta,
                            double dt_prob_expo);
/* Alias table of the OUTER layout's importance sub-sampling (see nmlmc_oracle.c). */
void o_build_alias(uint32_t P, const double *p, uint32_t *thr, uint32_t *alias, double *phat);
/* One sample(ell, M) call (nested_sampler.hpp:646-694).  trace (M records) and events may be
 * NULL.  Returns 0, or -1 if the events buffer is too small. */
int o_sample(o_ctx *, uint32_t ell, uint64_t M, double fsums[4], double diffsums[4],
             double *work, uint64_t stats[6], o_trace_rec *trace, o_events *events);
/* Full portfolio loss L(Y) = sum_i w_i (V_i(0) - disc*V_i(tau, S_tau)) for the outer samples
 * [first, first+n) of level `ell` on the OUTER layout (the K-quantile sweep). */
void o_portfolio_full_loss(o_ctx *, uint32_t ell, uint64_t first, uint64_t n, double *loss);

double o_norm_cdf_inv(double p, int prec);    /* common.cpp:53-86 */

/* Path-simulated portfolio loss of a batch of portfolios (adjoint_oracle.c): L[p * M + m]. */
void o_adj_loss(uint32_t n, const uint32_t *stock_off, const uint32_t *option_off, const double *S0,
                const double *mu, const double *sigma, const double *strike, const double *maturity,
                const double *w, const uint32_t *stock_ind, const int32_t *type, double r, double rho,
                double tau, uint32_t ell, uint32_t pairs, uint64_t M, uint64_t seed, int milstein,
                double *L);

#ifdef __cplusplus
}
#endif
#endif
