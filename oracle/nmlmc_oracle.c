/* CPU oracle for the nested MLMC level sampler — TEST INFRASTRUCTURE ONLY (see nmlmc_oracle.h).
 *
 * Plain C restatement of the reference's level sampler.  Only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline leg load it, as the checker.  Compiled with -ffp-contract=off on
 * x86-64 (SSE arithmetic, FLT_EVAL_METHOD 0) so every float/double operation rounds exactly as
 * the reference's g++ -O3 build does; the mixed float/double expression types of the reference
 * are reproduced operation by operation.
 *
 * The precision-dependent body lives in nmlmc_oracle_body.inc and is instantiated twice:
 * R = float  (the reference's default build, real_t = float)   -> suffix _f32
 * R = double (the reference's -DREAL_DOUBLE build)               -> suffix _f64
 */
#define _GNU_SOURCE
#include "nmlmc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------------------------ */
/* Threefry2x64-20 (Random123/threefry.h:86-93 rotation constants, :171 key-schedule parity,
 * :190-286 rounds and key injections; the Threefish-based counter RNG of Salmon et al., SC'11). */
static inline uint64_t rotl64(uint64_t x, unsigned r) { return (x << r) | (x >> (64 - r)); }

void o_threefry2x64(const uint64_t ctr[2], const uint64_t key[2], uint64_t out[2]) {
    static const unsigned R[8] = {16, 42, 12, 31, 16, 32, 24, 21};
    uint64_t ks[3];
    ks[0] = key[0];
    ks[1] = key[1];
    ks[2] = 0x1BD11BDAA9FC1A22ull ^ key[0] ^ key[1];
    uint64_t x0 = ctr[0] + ks[0], x1 = ctr[1] + ks[1];
    for (unsigned r = 0; r < 20; r++) {
        x0 += x1;
        x1 = rotl64(x1, R[r & 7]);
        x1 ^= x0;
        if ((r & 3) == 3) {          /* key injection s = r/4 + 1 after every fourth round */
            unsigned s = (r >> 2) + 1;
            x0 += ks[s % 3];
            x1 += ks[(s + 1) % 3] + s;
        }
    }
    out[0] = x0;
    out[1] = x1;
}

void o_threefry_batch(const uint64_t *ctr, const uint64_t *key, uint64_t *out, uint64_t n) {
    for (uint64_t i = 0; i < n; i++) o_threefry2x64(ctr + 2 * i, key + 2 * i, out + 2 * i);
}

/* r123::u01<double>(uint64) and r123::uneg11<double>(uint64) (Random123/uniform.hpp:144-180):
 * factor = 2^-64 (resp. 2^-63 for the signed cast), plus half a factor. */
static inline double u01_d64(uint64_t in) { return (double)in * 0x1p-64 + 0x1p-65; }
static inline float u01_f64in(uint64_t in) { return (float)in * 0x1p-64f + 0x1p-65f; }
static inline double uneg11_d64(uint64_t in) { return (double)(int64_t)in * 0x1p-63 + 0x1p-64; }

/* r123::boxmuller(uint64_t u0, uint64_t u1) (Random123/boxmuller.hpp:128-137) with the CPU
 * sincospi(x) = sincos(PI*x) (boxmuller.hpp:96-104). */
static inline void bm64(uint64_t u0, uint64_t u1, double *x, double *y) {
    const double PI = 3.1415926535897932;
    double s, c;
    sincos(PI * uneg11_d64(u0), &s, &c);
    double r = sqrt(-2. * log(u01_d64(u1)));
    *x = s * r;
    *y = c * r;
}

void o_boxmuller(const uint64_t *u0, const uint64_t *u1, double *x, double *y, uint64_t n) {
    for (uint64_t i = 0; i < n; i++) bm64(u0[i], u1[i], x + i, y + i);
}

/* OUTER layout, 32-bit words: u01 of a 32-bit word (exact in double) and the signed variant. */
static inline double u01_w32(uint32_t w) { return (double)w * 0x1p-32 + 0x1p-33; }
static inline float u01_w32f(uint32_t w) { return (float)w * 0x1p-32f + 0x1p-33f; }
static inline double uneg11_w32(uint32_t w) { return (double)(int32_t)w * 0x1p-31 + 0x1p-32; }
static inline void bm32(uint32_t u0, uint32_t u1, double *x, double *y) {
    const double PI = 3.1415926535897932;
    double s, c;
    sincos(PI * uneg11_w32(u0), &s, &c);
    double r = sqrt(-2. * log(u01_w32(u1)));
    *x = s * r;
    *y = c * r;
}

/* ------------------------------------------------------------------------------------------ */
/* random_state of the CPU build (par_omp.hpp:72-121): key = (seed, core), counter from {0,0},
 * a two-word cache consumed v[1] then v[0], and a cached second normal. */
typedef struct {
    uint64_t key[2], ctr[2], cur[2];
    int cached, saved;
    double saved_val;           /* real_t value widened */
} o_rs;

static void rs_seed(o_rs *s, uint64_t seed, uint64_t core) {        /* par_omp.hpp:101-108 */
    s->key[0] = seed; s->key[1] = core;
    s->ctr[0] = s->ctr[1] = 0;
    s->cached = 0; s->saved = 0; s->saved_val = 0;
}
static uint64_t rs_rand(o_rs *s) {                                     /* par_omp.hpp:92-99 */
    if (s->cached <= 0) {
        o_threefry2x64(s->ctr, s->key, s->cur);
        if (++s->ctr[0] == 0) ++s->ctr[1];                             /* array.h:133 incr */
        s->cached = 2;
    }
    return s->cur[--s->cached];
}

/* ------------------------------------------------------------------------------------------ */
/* Portfolio option record (portfolio_sampler.cpp:42-52) and stock (53-55), widened to double
 * storage; values are rounded to real_t at set-up. */
typedef struct {
    double strike, maturity, start, w, delta_est, prob, W_est;
    uint32_t stock_ind;
    int type;                   /* +1 call, -1 put (OptionType) */
} o_opt;

struct o_ctx {
    int prec, streams;
    uint32_t cores, N0, beta;
    double adaptive_r;
    int antithetic, adaptive_incl_r2;
    uint64_t seed;
    /* model */
    int kind;                   /* 0 reference model, 1 shift model, 2 portfolio */
    double stau, s1tau, max_loss;
    /* portfolio (portfolio::data / data_ex, portfolio_sampler.cpp:62-132) */
    uint32_t Q, P;
    double *S0, *mu, *sigma, *cdf, *delta_coalesce;
    o_opt *opt;
    double r, rho, s1_rho2, tau, prob_norm, compute_prob0;
    int subsample, use_delta_cv, discount;
    /* compute methods (ComputeMethod BS / Exact / Unbiased): options are grouped by method,
     * method m occupying [m_off[m], m_off[m] + m_n[m]); compute_prob[m] = sum of its probs */
    uint32_t m_off[3], m_n[3];
    double compute_prob[3];
    int mixed;                  /* more than the BS method present */
    int use_coarse_delta_cv, use_antithetic_risk, use_milstein;
    uint32_t dt_h0inv, dt_beta;
    double dt_prob_expo;
    /* OUTER layout, Subsampling::Random: alias table of the exact masses (o_build_alias) */
    uint32_t *alias_thr, *alias_idx;
    double *phat;
    /* CORE layout: persistent per-core streams */
    o_rs *rs_sync, *rs_inner;
    /* OUTER layout: next outer index per level, shard */
    uint64_t next_outer[64];
    uint32_t shard_rank, shard_world;
    /* optional per-outer-sample record of the adaptive decisions' distance from their threshold */
    double *margins;
};

void o_set_shard(o_ctx *c, uint32_t rank, uint32_t world) {
    c->shard_rank = rank;
    c->shard_world = world ? world : 1;
}

void o_set_margins(o_ctx *c, double *buf) { c->margins = buf; }

o_ctx *o_create(int prec, int streams, uint32_t cores, uint32_t N0, uint32_t beta,
                double adaptive_r, int antithetic, int adaptive_incl_r2, uint64_t seed) {
    o_ctx *c = (o_ctx *)calloc(1, sizeof(o_ctx));
    c->prec = prec; c->streams = streams; c->cores = cores ? cores : 1;
    c->N0 = N0; c->beta = beta; c->adaptive_r = adaptive_r;
    c->antithetic = antithetic; c->adaptive_incl_r2 = adaptive_incl_r2; c->seed = seed;
    c->rs_sync = (o_rs *)calloc(c->cores, sizeof(o_rs));
    c->rs_inner = (o_rs *)calloc(c->cores, sizeof(o_rs));
    /* init_samplers, CPU branch (nested_sampler.hpp:634-642): both streams keyed (seed, core). */
    for (uint32_t i = 0; i < c->cores; i++) {
        rs_seed(&c->rs_sync[i], seed, i);
        rs_seed(&c->rs_inner[i], seed, i);
    }
    return c;
}

static void free_portfolio(o_ctx *c) {
    free(c->S0); free(c->mu); free(c->sigma); free(c->cdf); free(c->delta_coalesce); free(c->opt);
    free(c->alias_thr); free(c->alias_idx); free(c->phat);
    c->S0 = c->mu = c->sigma = c->cdf = c->delta_coalesce = NULL; c->opt = NULL;
    c->alias_thr = c->alias_idx = NULL; c->phat = NULL;
}

/* Alias table of the OUTER layout's importance sub-sampling (the batched path's own addressing;
 * the reference draws with rand_int_cdf, common.hpp:160-176, which the CORE layout keeps).
 * Walker's method in Vose's construction on integers: masses W_j = round(p_j / sum p * P 2^32),
 * the rounding residue to the largest, sum exactly P 2^32; column j keeps thr_j of its own mass
 * and hands the rest to alias_j; full columns keep thr = 2^32 - 1 and alias themselves.  Option j
 * is drawn with probability exactly phat_j = W_j / (P 2^32). */
void o_build_alias(uint32_t P, const double *p, uint32_t *thr, uint32_t *alias, double *phat) {
    double S = 0;
    for (uint32_t j = 0; j < P; j++) S += p[j];
    const uint64_t unit = 1ull << 32, total = (uint64_t)P << 32;
    uint64_t *W = (uint64_t *)malloc(P * sizeof(uint64_t));
    uint32_t *small = (uint32_t *)malloc(P * sizeof(uint32_t)), *large = (uint32_t *)malloc(P * sizeof(uint32_t));
    uint64_t sum = 0;
    uint32_t jmax = 0, ns = 0, nl = 0;
    for (uint32_t j = 0; j < P; j++) {
        W[j] = (uint64_t)llround(p[j] / S * (double)total);
        sum += W[j];
        if (W[j] > W[jmax]) jmax = j;
    }
    if (sum > total) W[jmax] -= sum - total; else W[jmax] += total - sum;
    for (uint32_t j = 0; j < P; j++) {
        phat[j] = (double)W[j] / (double)total;
        thr[j] = 0xffffffffu;
        alias[j] = j;
        if (W[j] < unit) small[ns++] = j; else large[nl++] = j;
    }
    while (ns > 0 && nl > 0) {
        const uint32_t sj = small[--ns], lj = large[nl - 1];
        thr[sj] = (uint32_t)W[sj];
        alias[sj] = lj;
        W[lj] -= unit - W[sj];
        if (W[lj] < unit) {
            nl--;
            small[ns++] = lj;
        }
    }
    for (uint32_t q = 0; q < ns; q++) thr[small[q]] = W[small[q]] < 0xffffffffull ? (uint32_t)W[small[q]] : 0xffffffffu;
    free(W); free(small); free(large);
}

void o_destroy(o_ctx *c) {
    if (!c) return;
    free_portfolio(c);
    free(c->rs_sync); free(c->rs_inner);
    free(c);
}

/* ------------------------------------------------------------------------------------------ */
/* uint_pow for the powers of two used here (common.hpp:146-157), with clog2(1) = 0: the
 * semantics of the reference's CUDA build (__clzll(0) = 64).  The reference CPU build's default
 * x86-64 code evaluates __builtin_clzl(0) (undefined) and gets clog2(1) = 1 instead. */
static uint64_t uint_pow_u64(uint64_t x, uint64_t n) {
    uint64_t r = 1;
    while (n--) r *= x;
    return r;
}

/* Per-outer-sample stream cursor.  CORE layout: points at the core's persistent random_state
 * pair.  OUTER layout: key (seed, level<<56 | outer index), counter (block, phase tag). */
typedef struct {
    o_ctx *ctx;
    o_rs *sync, *inner;         /* CORE */
    uint64_t key[2];            /* OUTER */
    uint64_t tag;
    uint64_t nword, nnorm;      /* OUTER: next word / next normal of the current phase */
    int draw_kind;              /* OUTER: 0 none yet, 1 normals, 2 uniforms (a phase is one kind) */
    uint64_t randu_count, randn_count;
    uint64_t ninner;            /* OUTER: inner samples drawn in the current phase */
    /* OUTER, path-simulated inner sample: its own counter namespace for normals (pns) and
     * uniforms (pns | O_PATH_UNIFORM), next normal / uniform */
    int path;
    uint64_t pns, pn, pu;
} o_cursor;

/* Counter namespaces of a path-simulated inner sample on the OUTER layout: inner sample i of the
 * phase with tag t draws its normals from counter word 1 = t | (i + 1) << 16 and its uniforms
 * from t | (i + 1) << 16 | 2^15. */
#define O_PATH_UNIFORM (1ull << 15)
static uint64_t path_ns(uint64_t tag, uint64_t i) { return tag | ((i + 1) << 16); }

enum { PH_OUTER = 0, PH_FINE = 1, PH_COARSE = 64, PH_FINAL = 128, PH_FINAL_C = 129 };

static void cur_phase(o_cursor *k, uint64_t tag) {
    k->tag = tag; k->nword = 0; k->nnorm = 0; k->draw_kind = 0; k->ninner = 0; k->path = 0;
}

/* word j of counter namespace ns of the current OUTER key */
static uint32_t ns_word(const o_cursor *k, uint64_t ns, uint64_t j) {
    uint64_t ctr[2] = {j >> 2, ns}, v[2];
    o_threefry2x64(ctr, k->key, v);
    uint64_t e = v[(j >> 1) & 1];
    return (j & 1) ? (uint32_t)(e >> 32) : (uint32_t)e;
}

static uint32_t outer_word(const o_cursor *k, uint64_t j) {
    uint64_t ctr[2] = {j >> 2, k->tag}, v[2];
    o_threefry2x64(ctr, k->key, v);
    uint64_t e = v[(j >> 1) & 1];
    return (j & 1) ? (uint32_t)(e >> 32) : (uint32_t)e;
}

/* 64-bit value #j of the current OUTER phase: element j & 1 of block j >> 1 (portfolio draws) */
static uint64_t outer_u64(const o_cursor *k, uint64_t j) {
    uint64_t ctr[2] = {j >> 1, k->tag}, v[2];
    o_threefry2x64(ctr, k->key, v);
    return v[j & 1];
}

/* normal #k of the current OUTER phase: pair k>>1 from words (2p, 2p+1) */
static double outer_normal(o_cursor *k) {
    uint64_t idx = k->nnorm++;
    uint64_t p = idx >> 1;
    double x, y;
    bm32(outer_word(k, 2 * p), outer_word(k, 2 * p + 1), &x, &y);
    return (idx & 1) ? y : x;
}

#define R float
#define SFX(name) name##_f32
#define IS_F32 1
#include "nmlmc_oracle_body.inc"
#undef R
#undef SFX
#undef IS_F32

#define R double
#define SFX(name) name##_f64
#define IS_F32 0
#include "nmlmc_oracle_body.inc"
#undef R
#undef SFX
#undef IS_F32

void o_stream_draws(int prec, uint64_t seed, uint64_t core, const char *ops, uint64_t n,
                    double *out_real, uint64_t *out_u64) {
    if (prec == O_PREC_REF32) stream_draws_f32(seed, core, ops, n, out_real, out_u64);
    else stream_draws_f64(seed, core, ops, n, out_real, out_u64);
}

void o_set_model(o_ctx *c, int kind, double tau, double max_loss) {
    if (c->prec == O_PREC_REF32) set_model_f32(c, kind, tau, max_loss);
    else set_model_f64(c, kind, tau, max_loss);
}

int o_set_portfolio(o_ctx *c, uint32_t Q, const double *S0, const double *mu, const double *sigma,
                    uint32_t P, const double *strike, const double *maturity, const double *w,
                    const uint32_t *stock_ind, const int32_t *type, const double *prob,
                    double r, double rho, double max_loss, double tau, int subsample,
                    int use_delta_cv, int discount, double *out_start, double *out_delta_est) {
    if (c->prec == O_PREC_REF32)
        return set_portfolio_f32(c, Q, S0, mu, sigma, P, strike, maturity, w, stock_ind, type, prob,
                                 r, rho, max_loss, tau, subsample, use_delta_cv, discount, out_start,
                                 out_delta_est);
    return set_portfolio_f64(c, Q, S0, mu, sigma, P, strike, maturity, w, stock_ind, type, prob,
                             r, rho, max_loss, tau, subsample, use_delta_cv, discount, out_start,
                             out_delta_est);
}

int o_sample(o_ctx *c, uint32_t ell, uint64_t M, double fsums[4], double diffsums[4], double *work,
             uint64_t stats[6], o_trace_rec *trace, o_events *events) {
    if (c->prec == O_PREC_REF32) return sample_f32(c, ell, M, fsums, diffsums, work, stats, trace, events);
    return sample_f64(c, ell, M, fsums, diffsums, work, stats, trace, events);
}

void o_portfolio_full_loss(o_ctx *c, uint32_t ell, uint64_t first, uint64_t n, double *loss) {
    if (c->prec == O_PREC_REF32) full_loss_f32(c, ell, first, n, loss);
    else full_loss_f64(c, ell, first, n, loss);
}

double o_norm_cdf_inv(double p, int prec) {
    return prec == O_PREC_REF32 ? (double)norm_cdf_inv_f32((float)p) : norm_cdf_inv_f64(p);
}

int o_set_portfolio_methods(o_ctx *c, uint32_t Q, const double *S0, const double *mu,
                            const double *sigma, uint32_t P, const double *strike,
                            const double *maturity, const double *w, const uint32_t *stock_ind,
                            const int32_t *type, const double *prob, const int32_t *method,
                            double r, double rho, double max_loss, double tau, int subsample,
                            int use_delta_cv, int use_coarse_delta_cv, int use_antithetic_risk,
                            int use_milstein, uint32_t dt_h0inv, uint32_t dt_beta,
                            double dt_prob_expo) {
    if (c->prec == O_PREC_REF32)
        return set_portfolio_m_f32(c, Q, S0, mu, sigma, P, strike, maturity, w, stock_ind, type, prob,
                                   method, r, rho, max_loss, tau, subsample, use_delta_cv, 1,
                                   use_coarse_delta_cv, use_antithetic_risk, use_milstein, dt_h0inv,
                                   dt_beta, dt_prob_expo, NULL, NULL);
    return set_portfolio_m_f64(c, Q, S0, mu, sigma, P, strike, maturity, w, stock_ind, type, prob,
                               method, r, rho, max_loss, tau, subsample, use_delta_cv, 1,
                               use_coarse_delta_cv, use_antithetic_risk, use_milstein, dt_h0inv,
                               dt_beta, dt_prob_expo, NULL, NULL);
}
