// C ABI of the level sampler: contexts, the reference-named surface and host-side set-up.
#include <algorithm>
#include <cmath>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <stdexcept>
#include <vector>

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include "../../include/nmlmc.h"
#include "nmlmc_internal.h"

using namespace nmlmc;

// ---------------------------------------------------------------------------------------------
// Host-side portfolio arithmetic in real_t, in the reference's evaluation order
// (portfolio_sampler.cpp:140-160, common.hpp:201-202); compiled without FP contraction.
namespace {

template <class RT> RT h_erfc(RT x);
template <> float h_erfc<float>(float x) { return erfcf(x); }
template <> double h_erfc<double>(double x) { return erfc(x); }
template <class RT> RT h_log(RT x);
template <> float h_log<float>(float x) { return logf(x); }
template <> double h_log<double>(double x) { return log(x); }
template <class RT> RT h_exp(RT x);
template <> float h_exp<float>(float x) { return expf(x); }
template <> double h_exp<double>(double x) { return exp(x); }
template <class RT> RT h_sqrt(RT x);
template <> float h_sqrt<float>(float x) { return sqrtf(x); }
template <> double h_sqrt<double>(double x) { return sqrt(x); }

template <class RT>
RT h_norm_cdf(RT x) {
    const RT SQRT_2 = (RT)1.414213562373095;
    return (RT)(0.5 * (double)h_erfc<RT>(-x / SQRT_2));
}

template <class RT>
RT h_d1(RT S0, RT strike, RT r, RT t, RT sigma) {
    RT v1 = h_log<RT>(S0 / strike);
    RT v2 = (RT)(((double)r + (double)(sigma * sigma) / 2.0) * (double)t);
    RT v3 = sigma * h_sqrt<RT>(t);
    return (v1 + v2) / v3;
}

template <class RT>
RT h_calc_bs(int type, RT S0, RT strike, RT r, RT t, RT sigma) {
    RT d1 = h_d1<RT>(S0, strike, r, t, sigma);
    RT d2 = d1 - sigma * h_sqrt<RT>(t);
    RT mod = (RT)type;
    return mod * S0 * h_norm_cdf<RT>(mod * d1) - mod * strike * h_exp<RT>(-r * t) * h_norm_cdf<RT>(mod * d2);
}

template <class RT>
RT h_calc_delta(int type, RT S0, RT strike, RT r, RT t, RT sigma) {
    return h_norm_cdf<RT>(h_d1<RT>(S0, strike, r, t, sigma)) - (RT)(type == -1 ? 1 : 0);
}

template <class RT>
RT h_norm_cdf_inv(RT p) {
    // Acklam's rational approximation with the coefficient values the reference truncates them
    // to (common.cpp:53-86).
    const RT a[] = {-39.696830f, 220.946098f, -275.928510f, 138.357751f, -30.664798f, 2.506628f};
    const RT b[] = {-54.476098f, 161.585836f, -155.698979f, 66.801311f, -13.280681f};
    const RT c[] = {-0.007784894002f, -0.32239645f, -2.400758f, -2.549732f, 4.374664f, 2.938163f};
    const RT d[] = {0.007784695709f, 0.32246712f, 2.445134f, 3.754408f};
    const RT plow = 0.02425f, phigh = 1 - plow;
    if (p < plow) {
        RT q = h_sqrt<RT>(-2 * h_log<RT>(p));
        return (((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
               ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1);
    }
    if (phigh < p) {
        RT q = h_sqrt<RT>(-2 * h_log<RT>(1 - p));
        return -(((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
               ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1);
    }
    RT q = p - 0.5f, r = q * q;
    return (((((a[0] * r + a[1]) * r + a[2]) * r + a[3]) * r + a[4]) * r + a[5]) * q /
           (((((b[0] * r + b[1]) * r + b[2]) * r + b[3]) * r + b[4]) * r + 1);
}

// Levels one nmlmc_sample_levels submission may hold (accumulator slots of the OUTER buffers).
constexpr uint32_t kMaxSubmit = 64;

// Portfolio as handed to the sampler, kept on the host in double (the values are the real_t
// ones when the context computes in float).
struct HostPortfolio {
    uint32_t Q = 0, P = 0;
    std::vector<double> S0, mu, sigma;
    std::vector<double> strike, maturity, w, prob, W_est, start, delta_est;
    std::vector<uint32_t> stock_ind;
    std::vector<int8_t> type;
    double r = 0, rho = 0, s1_rho2 = 1, max_loss = 0, tau = 0;
    int subsample = SUB_UNIFORM, use_delta_cv = 0, discount = 1;
    bool s1_rho2_given = false;
    bool own_params = false;   // start / delta_est computed here (native API), per precision
    // compute methods: options are stored grouped by method (BS, Exact, Unbiased) in the order
    // given; m_n counts them, order[k] is the caller's index of stored option k
    uint32_t m_n[3] = {0, 0, 0};
    std::vector<uint32_t> order;
    uint32_t dt_h0inv = 8, dt_beta = 4;
    double dt_prob_expo = -1.5;
    int use_coarse_delta_cv = 0, use_antithetic_risk = 1, use_milstein = 1;
    bool mixed() const { return m_n[1] + m_n[2] > 0; }
};

template <class RT>
struct DevPortfolio {
    RT *strike = nullptr, *maturity = nullptr, *start = nullptr, *w = nullptr, *prob = nullptr,
       *W_est = nullptr, *cdf = nullptr, *S0 = nullptr, *mu = nullptr, *sigma = nullptr,
       *delta_coalesce = nullptr;
    uint32_t* stock_ind = nullptr;
    int8_t* type = nullptr;
    FastOption* fast = nullptr;       // packed records of the FP32 path
    FastOption* fast_s = nullptr;     // the same, scaled by 1 / sampling probability
    FastColumn* fast_col = nullptr;   // sampler records fused with the alias table
    uint2* alias = nullptr;           // alias table (OUTER, Subsampling::Random)
    RT* phat = nullptr;
    OptionTable<RT> table{};
};

}  // namespace

// An executable graph of one submission topology: the levels of the round and their batch
// counts (the launch sequence of a level follows from its level and batch count).
struct GraphSlot {
    std::vector<uint64_t> key;
    cudaGraphExec_t exec = nullptr;
    uint64_t last_use = 0;
};
constexpr size_t kGraphCache = 16;

// Phase-kernel configuration of one level: register/occupancy variant and chunk length.
struct PhaseChoice {
    int32_t state = 0;        // 0 default, 1 tuned, 2 pinned by the caller
    uint32_t variant = 0, chunk = 0;
    double probe_ms = 0;      // device time of the chosen configuration on the tuning probe
};

struct nmlmc_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    nmlmc_config cfg{};
    bool configured = false;
    // model / portfolio
    int kind = -1;
    double tau = 0, max_loss = 0, stau = 0, s1tau = 0;
    bool stau_given = false;
    HostPortfolio pf;
    int pf_prec = -1;                 // precision the device portfolio was built for
    DevPortfolio<float> dpf32;
    DevPortfolio<double> dpf64;
    // CORE layout
    CoreStream* d_states = nullptr;
    double* d_part_sums = nullptr;
    uint64_t* d_part_stats = nullptr;
    double* d_out_sums = nullptr;     // [10]
    uint64_t* d_out_stats = nullptr;  // [6]
    uint32_t states_cores = 0;
    // OUTER layout
    OuterBuffers ob{};
    bool ob_alloc = false;
    uint64_t next_outer[NMLMC_MAX_LEVELS] = {};
    // pinned staging
    double* h_pin = nullptr;          // 32 doubles
    // one-submission level rounds (nmlmc_sample_levels on the OUTER layout)
    double* h_lev = nullptr;          // pinned [kMaxSubmit][16] sums, then [kMaxSubmit][2] stamps
    uint64_t* d_stamps = nullptr;     // device [kMaxSubmit][2] level begin / end (ns)
    std::vector<GraphSlot> graphs;    // executable graphs of recent submissions, by topology
    uint64_t graph_clock = 0;
    uint64_t graph_instantiations = 0, graph_updates = 0, graph_launches = 0;
    // trace
    nmlmc_trace_rec* trace_host = nullptr;
    uint64_t trace_cap = 0;
    TraceRec* d_trace = nullptr;
    uint64_t d_trace_cap = 0;
    // sharding over ranks (OUTER layout)
    uint32_t shard_rank = 0, shard_world = 1;
    // phase-kernel configuration per level on the batched FP32 path (autotuned or pinned)
    int32_t autotune = 1;             // 0 off, 1 variants, 2 variants and chunk length
    bool batch_default = true;        // cfg.batch was 0: the library chose the batch size
    PhaseChoice phase[NMLMC_MAX_LEVELS];
    // phase-kernel timing
    bool prof = false;
    std::vector<cudaEvent_t> pev;
    size_t pn = 0;
    uint64_t prof_launches = 0;
    double prof_seconds = 0;
};

namespace {

thread_local int g_tls_error = NMLMC_OK;

// NVTX range for profilers (nsys, ncu --nvtx): header-only NVTX v3, inert unless a tool attaches.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// Device allocations of the library go through dev_malloc so that tests can make one of them fail
// (nmlmc_inject_alloc_failure): -1 = off, k >= 0 = k more allocations succeed, then one fails.
std::atomic<int64_t> g_fail_alloc{-1};

template <class T>
cudaError_t dev_malloc(T** p, size_t bytes) {
    const int64_t k = g_fail_alloc.load();
    if (k == 0) {
        g_fail_alloc.store(-1);
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    if (k > 0) g_fail_alloc.store(k - 1);
    return cudaMalloc(p, bytes);
}

int set_err(int e) {
    g_tls_error = e;
    return e;
}

// Host containers sized by the caller's input can throw; no exception may cross the C ABI.
template <class F>
int host_guard(F&& f) {
    try {
        return f();
    } catch (const std::bad_alloc&) {
        return set_err(NMLMC_ERR_NOMEM);
    } catch (const std::length_error&) {
        return set_err(NMLMC_ERR_ARG);
    }
}

int cuda_status(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return NMLMC_OK;
    fprintf(stderr, "nmlmc: %s: %s\n", what, cudaGetErrorString(e));
    return set_err(NMLMC_ERR_CUDA);
}

#define NM_CUDA(call, what)                                  \
    do {                                                     \
        int _s = cuda_status((call), what);                  \
        if (_s != NMLMC_OK) return _s;                       \
    } while (0)

template <class T>
void dfree(T*& p) {
    if (p) cudaFree(p);
    p = nullptr;
}

template <class RT>
void free_dev_portfolio(DevPortfolio<RT>& d) {
    dfree(d.strike); dfree(d.maturity); dfree(d.start); dfree(d.w); dfree(d.prob); dfree(d.W_est);
    dfree(d.cdf); dfree(d.S0); dfree(d.mu); dfree(d.sigma); dfree(d.delta_coalesce);
    dfree(d.stock_ind); dfree(d.type); dfree(d.fast); dfree(d.fast_s); dfree(d.fast_col); dfree(d.alias); dfree(d.phat);
    d.table = OptionTable<RT>{};
}

template <class T>
int upload(T*& d, const std::vector<T>& h) {
    dfree(d);
    size_t n = h.size() ? h.size() : 1;
    if (dev_malloc(&d, n * sizeof(T)) != cudaSuccess) return set_err(NMLMC_ERR_NOMEM);
    if (!h.empty()) NM_CUDA(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
    return NMLMC_OK;
}

template <class RT>
std::vector<RT> narrow(const std::vector<double>& v) {
    std::vector<RT> o(v.size());
    for (size_t i = 0; i < v.size(); i++) o[i] = (RT)v[i];
    return o;
}

// start / delta_est of every option (portfolio_comp_params, portfolio_sampler.cpp:687-700).
template <class RT>
void comp_params(HostPortfolio& h) {
    for (uint32_t j = 0; j < h.P; j++) {
        const uint32_t s = h.stock_ind[j];
        h.start[j] = (double)h_calc_bs<RT>(h.type[j], (RT)h.S0[s], (RT)h.strike[j], (RT)h.r, (RT)h.maturity[j], (RT)h.sigma[s]);
        h.delta_est[j] = (double)h_calc_delta<RT>(h.type[j], (RT)h.S0[s], (RT)h.strike[j], (RT)h.r, (RT)h.maturity[j], (RT)h.sigma[s]);
    }
}

// Alias table of the OUTER layout's importance sub-sampling (Walker's method in Vose's
// construction, on integers).  The masses W_j = round(p_j / sum p * P 2^32), with the rounding
// residue given to the largest, sum exactly to P 2^32; column j keeps threshold thr_j < 2^32 of
// its own mass and hands the rest to alias_j.  One 64-bit draw v picks column floor(v P / 2^64)
// and the coin (v P mod 2^64) >> 32, so option j is drawn with probability exactly
// phat_j = W_j / (P 2^32), the weight the estimator divides by.  Full columns carry
// thr = 2^32 - 1 and alias = themselves.
void build_alias(uint32_t P, const std::vector<double>& p, std::vector<uint2>& tab, std::vector<double>& phat) {
    double S = 0;
    for (uint32_t j = 0; j < P; j++) S += p[j];
    const uint64_t unit = 1ull << 32, total = (uint64_t)P << 32;
    std::vector<uint64_t> W(P);
    uint64_t sum = 0;
    uint32_t jmax = 0;
    for (uint32_t j = 0; j < P; j++) {
        W[j] = (uint64_t)llround(p[j] / S * (double)total);
        sum += W[j];
        if (W[j] > W[jmax]) jmax = j;
    }
    if (sum > total) W[jmax] -= sum - total; else W[jmax] += total - sum;
    phat.resize(P);
    for (uint32_t j = 0; j < P; j++) phat[j] = (double)W[j] / (double)total;
    tab.assign(P, uint2{0xffffffffu, 0});
    std::vector<uint32_t> small, large;
    for (uint32_t j = 0; j < P; j++) {
        tab[j].y = j;
        (W[j] < unit ? small : large).push_back(j);
    }
    while (!small.empty() && !large.empty()) {
        const uint32_t sj = small.back(), lj = large.back();
        small.pop_back();
        tab[sj].x = (uint32_t)W[sj];
        tab[sj].y = lj;
        W[lj] -= unit - W[sj];
        if (W[lj] < unit) {
            large.pop_back();
            small.push_back(lj);
        }
    }
    for (uint32_t j : small) tab[j].x = (uint32_t)std::min<uint64_t>(W[j], 0xffffffffull);   // == unit: exact sums
}

// portfolio_comp_params + portfolio_update_data (portfolio_sampler.cpp:631-700) in real_t.
template <class RT>
int build_dev_portfolio(nmlmc_ctx* c, DevPortfolio<RT>& d) {
    HostPortfolio& h = c->pf;
    free_dev_portfolio(d);
    if (h.own_params) comp_params<RT>(h);
    const uint32_t P = h.P, Q = h.Q;
    std::vector<RT> S0 = narrow<RT>(h.S0), mu = narrow<RT>(h.mu), sg = narrow<RT>(h.sigma);
    std::vector<RT> K = narrow<RT>(h.strike), T = narrow<RT>(h.maturity), w = narrow<RT>(h.w);
    std::vector<RT> prob = narrow<RT>(h.prob), West = narrow<RT>(h.W_est);
    std::vector<RT> start(P), cdf(P), delta(Q, (RT)0);
    RT prob_norm = 0, acc = 0, cprob[3] = {0, 0, 0};
    uint32_t m_off[3] = {0, h.m_n[0], h.m_n[0] + h.m_n[1]};
    for (uint32_t j = 0; j < P; j++) {
        const uint32_t s = h.stock_ind[j];
        const uint32_t m = j < m_off[1] ? 0 : (j < m_off[2] ? 1 : 2);
        if (j == m_off[m]) acc = 0;                      // the CDF restarts for every method
        RT st = (RT)h.start[j], de = (RT)h.delta_est[j];
        start[j] = st;
        cdf[j] = acc;
        acc += prob[j];
        delta[s] += w[j] * de;
        prob_norm += prob[j];
        cprob[m] += prob[j];
    }
    int rc;
    if ((rc = upload(d.strike, K)) || (rc = upload(d.maturity, T)) || (rc = upload(d.start, start)) ||
        (rc = upload(d.w, w)) || (rc = upload(d.prob, prob)) || (rc = upload(d.W_est, West)) ||
        (rc = upload(d.cdf, cdf)) || (rc = upload(d.S0, S0)) || (rc = upload(d.mu, mu)) ||
        (rc = upload(d.sigma, sg)) || (rc = upload(d.delta_coalesce, delta)) ||
        (rc = upload(d.stock_ind, h.stock_ind)) || (rc = upload(d.type, h.type)))
        return rc;
    OptionTable<RT>& t = d.table;
    t.strike = d.strike; t.maturity = d.maturity; t.start = d.start; t.w = d.w; t.prob = d.prob;
    t.W_est = d.W_est; t.cdf = d.cdf; t.stock_ind = d.stock_ind; t.type = d.type; t.S0 = d.S0;
    t.mu = d.mu; t.sigma = d.sigma; t.delta_coalesce = d.delta_coalesce;
    t.P = P; t.Q = Q;
    t.r = (RT)h.r; t.rho = (RT)h.rho;
    t.s1_rho2 = h.s1_rho2_given ? (RT)h.s1_rho2 : h_sqrt<RT>(1 - (RT)h.rho * (RT)h.rho);
    t.max_loss = (RT)h.max_loss; t.tau = (RT)h.tau;
    t.stau = h_sqrt<RT>((RT)h.tau);                      // data_ex ctor, portfolio_sampler.cpp:97-98
    t.prob_norm = prob_norm; t.compute_prob0 = cprob[0];
    t.inv_count_prob = (RT)(1. / (double)P);              // portfolio_sampler.cpp:360
    t.subsample = h.subsample; t.use_delta_cv = h.use_delta_cv; t.discount = h.discount;
    for (int m = 0; m < 3; m++) { t.m_off[m] = m_off[m]; t.m_n[m] = h.m_n[m]; t.compute_prob[m] = cprob[m]; }
    t.mixed = h.mixed() ? 1 : 0;
    t.dt_h0inv = h.dt_h0inv; t.dt_beta = h.dt_beta; t.dt_prob_expo = (RT)h.dt_prob_expo;
    t.use_coarse_delta_cv = h.use_coarse_delta_cv; t.use_antithetic_risk = h.use_antithetic_risk;
    t.use_milstein = h.use_milstein;
    t.fast = nullptr;
    t.fast_s = nullptr;
    t.fast_col = nullptr;
    t.alias = nullptr;
    t.phat = nullptr;
    std::vector<double> phat;
    std::vector<uint2> tab;
    if (h.subsample == SUB_RANDOM) {             // the OUTER layout's draw (all methods)
        std::vector<double> pr(P);
        for (uint32_t j = 0; j < P; j++) pr[j] = (double)prob[j];
        build_alias(P, pr, tab, phat);
        std::vector<RT> ph(P);
        for (uint32_t j = 0; j < P; j++) ph[j] = (RT)phat[j];
        if ((rc = upload(d.alias, tab)) || (rc = upload(d.phat, ph))) return rc;
        t.alias = d.alias;
        t.phat = d.phat;
    }
    if constexpr (sizeof(RT) == 4) {
        // packed FP32 records (nmlmc_bs.cuh): per-option constants folded in double, rounded once;
        // only for unit work estimates (every option of the BS method costs one evaluation)
        bool unit = true;
        for (uint32_t j = 0; j < P; j++) unit = unit && h.W_est[j] == 1.0;
        if (unit && !h.mixed()) {
            // Record of option j with its weights scaled by sc and, with cv_on, the delta control
            // variate: cv = sc w Delta_BS(S0, T) and its constant -cv S0 folded into wV0.
            auto record = [&](uint32_t j, double sc, bool cv_on) {
                const uint32_t s = h.stock_ind[j];
                const double sg = h.sigma[s], K = h.strike[j], T = h.maturity[j], Tr = T - h.tau;
                const double m = h.type[j] > 0 ? 1.0 : -1.0;
                const double sd = sg * sqrt(Tr);
                const double V0 = h_calc_bs<double>(h.type[j], h.S0[s], K, h.r, T, sg);
                const double disc = h.discount ? exp(-h.r * h.tau) : 1.0;
                const double cv = cv_on ? sc * h.w[j] * h_calc_delta<double>(h.type[j], h.S0[s], K, h.r, T, sg) : 0.0;
                FastOption o;
                o.c1 = (float)(-log(K) + (h.r + 0.5 * sg * sg) * Tr);
                o.inv_s = (float)(m / sd);
                o.s = (float)(m * sd);
                o.wR = (float)(-sc * h.w[j] * disc * m);
                o.wK = (float)(sc * h.w[j] * disc * m * K * exp(-h.r * Tr));
                o.wV0 = (float)(sc * h.w[j] * V0 - cv * h.S0[s]);
                o.cv = (float)cv;
                o.stock = s;
                return o;
            };
            // full-loss records: the loss L(Y) itself, no control variate
            std::vector<FastOption> fo(P);
            for (uint32_t j = 0; j < P; j++) fo[j] = record(j, 1.0, false);
            if ((rc = upload(d.fast, fo))) return rc;
            t.fast = d.fast;
            if (h.subsample != SUB_NONE) {
                // sampler records: the inner value X = loss_j / phat_j folded into the weights
                for (uint32_t j = 0; j < P; j++) {
                    const double sc = h.subsample == SUB_UNIFORM ? (double)P : (phat[j] > 0 ? 1.0 / phat[j] : 0.0);
                    fo[j] = record(j, sc, h.use_delta_cv != 0);
                }
                if ((rc = upload(d.fast_s, fo))) return rc;
                t.fast_s = d.fast_s;
                if (h.subsample == SUB_RANDOM && Q <= kColumnMaxStocks && P < kColumnMaxOptions) {
                    std::vector<FastColumn> col(P);
                    for (uint32_t j = 0; j < P; j++) {
                        const FastOption& o = fo[j];
                        col[j] = FastColumn{o.c1, o.inv_s, o.wR, o.wK, o.wV0, o.cv, tab[j].x, (tab[j].y << 8) | o.stock};
                    }
                    if ((rc = upload(d.fast_col, col))) return rc;
                    t.fast_col = d.fast_col;
                }
            }
        }
    }
    return NMLMC_OK;
}

int ensure_portfolio(nmlmc_ctx* c) {
    if (c->kind != KIND_PORTFOLIO) return NMLMC_OK;
    const int want = c->cfg.precision == NMLMC_PREC_FP64 ? 1 : 0;
    if (c->pf_prec == want) return NMLMC_OK;
    int rc = want ? build_dev_portfolio<double>(c, c->dpf64) : build_dev_portfolio<float>(c, c->dpf32);
    if (rc == NMLMC_OK) c->pf_prec = want;
    return rc;
}

bool is_adaptive(const nmlmc_config& cfg, double r) {
    if (cfg.precision == NMLMC_PREC_FP64) return r > 1 && (cfg.adaptive_incl_r2 ? r <= 2 : r < 2);
    float rf = (float)r;
    return rf > 1 && (cfg.adaptive_incl_r2 ? rf <= 2 : rf < 2);
}

uint64_t upow(uint64_t x, uint32_t n) {
    uint64_t r = 1;
    while (n--) r *= x;
    return r;
}

// get_samples_count ctor (nested_sampler.hpp:225-239) with the host libm, in real_t.
CountParams count_params(const nmlmc_config& cfg, uint32_t ell) {
    CountParams p;
    p.max_count = (uint64_t)cfg.N0 * upow(cfg.beta, ell);
    if (is_adaptive(cfg, cfg.adaptive_r)) {
        p.base_count = (uint64_t)cfg.N0 * upow(cfg.beta >> 1, ell);
        if (cfg.precision == NMLMC_PREC_FP64)
            p.tmp = (double)p.max_count * pow(9.0 / (double)p.max_count, cfg.adaptive_r / 2);
        else
            p.tmp = (double)((float)p.max_count * powf(9.f / (float)p.max_count, (float)cfg.adaptive_r / 2));
    } else {
        p.base_count = p.max_count;
        p.tmp = 0;
    }
    return p;
}

int alloc_core(nmlmc_ctx* c) {
    const uint32_t cores = c->cfg.cores;
    if (c->states_cores == cores && c->d_states) return NMLMC_OK;
    dfree(c->d_states); dfree(c->d_part_sums); dfree(c->d_part_stats);
    c->states_cores = 0;
    if (dev_malloc(&c->d_states, (size_t)cores * 2 * sizeof(CoreStream)) != cudaSuccess ||
        dev_malloc(&c->d_part_sums, (size_t)cores * 10 * sizeof(double)) != cudaSuccess ||
        dev_malloc(&c->d_part_stats, (size_t)cores * 6 * sizeof(uint64_t)) != cudaSuccess) {
        dfree(c->d_states); dfree(c->d_part_sums); dfree(c->d_part_stats);
        return set_err(NMLMC_ERR_NOMEM);
    }
    c->states_cores = cores;
    return NMLMC_OK;
}

void free_outer(nmlmc_ctx* c) {
    OuterBuffers& B = c->ob;
    if (c->ob_alloc) {
        cudaFree(B.Yv); cudaFree(B.Rt); cudaFree(B.cnt_f); cudaFree(B.cnt_c);
        cudaFree(B.lists); cudaFree(B.class_items); cudaFree(B.counters); cudaFree(B.block_sums);
        cudaFree(B.level_acc);
    }
    B.Yv = B.Rt = nullptr;
    B.cnt_f = B.cnt_c = B.lists = B.class_items = B.counters = nullptr;
    B.block_sums = B.level_acc = nullptr;
    B.cap = 0;
    c->ob_alloc = false;
}

void drop_graphs(nmlmc_ctx* c) {
    for (GraphSlot& g : c->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    c->graphs.clear();
}

// Batch buffers for calls of up to `want` outer samples per rank.  An explicit cfg.batch is the
// batch size; the default grows on demand in powers of two from 2^16 up to the default maximum
// (2^24 outer samples, portfolios at most 1 GiB of R_tau rows), so small users stay small.
int alloc_outer(nmlmc_ctx* c, uint64_t want) {
    const uint32_t Q = c->kind == KIND_PORTFOLIO ? c->pf.Q : 0;
    uint64_t cap = c->cfg.batch;
    if (c->batch_default) {
        uint64_t cap_max = cap;
        if (Q) {
            const uint64_t lim = (1ull << 30) / ((uint64_t)Q * sizeof(double));
            const uint64_t lo = 1ull << 16;
            if (cap_max > lim) cap_max = lim > lo ? lim : lo;
        }
        cap = 1ull << 16;
        while (cap < want && cap < cap_max) cap <<= 1;
        if (cap > cap_max) cap = cap_max;
        if (c->ob_alloc && c->ob.cap >= cap && c->ob.Q >= Q) return NMLMC_OK;
        if (c->ob_alloc && c->ob.cap > cap) cap = c->ob.cap;      // never shrink
    } else if (c->ob_alloc && c->ob.cap == cap && c->ob.Q >= Q) {
        return NMLMC_OK;
    }
    OuterBuffers& B = c->ob;
    drop_graphs(c);                       // their nodes hold the old buffers
    free_outer(c);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    B.cap = cap;
    B.Q = Q;
    B.grid = sms * 4;            // partial-sum slots; the phase kernel runs its resident CTAs (<= grid)
    bool ok = dev_malloc(&B.Yv, cap * sizeof(double)) == cudaSuccess &&
              dev_malloc(&B.Rt, (Q ? cap * Q : 1) * sizeof(double)) == cudaSuccess &&
              dev_malloc(&B.cnt_f, cap * sizeof(uint32_t)) == cudaSuccess &&
              dev_malloc(&B.cnt_c, cap * sizeof(uint32_t)) == cudaSuccess &&
              dev_malloc(&B.lists, 4 * cap * sizeof(uint32_t)) == cudaSuccess &&
              dev_malloc(&B.class_items, cap * sizeof(uint32_t)) == cudaSuccess &&
              dev_malloc(&B.counters, 256 * sizeof(uint32_t)) == cudaSuccess &&
              dev_malloc(&B.block_sums, (size_t)B.grid * 16 * sizeof(double)) == cudaSuccess &&
              dev_malloc(&B.level_acc, kMaxSubmit * 16 * sizeof(double)) == cudaSuccess;
    c->ob_alloc = true;                   // free_outer releases a partial set too
    if (!ok) {
        free_outer(c);
        return set_err(NMLMC_ERR_NOMEM);
    }
    cudaMemset(B.counters, 0, 256 * sizeof(uint32_t));
    return NMLMC_OK;
}

template <class RT>
ModelParams<RT> model_params(const nmlmc_ctx* c) {
    ModelParams<RT> mp;
    if (c->stau_given) {
        mp.stau = (RT)c->stau;
        mp.s1tau = (RT)c->s1tau;
    } else {
        RT t = (RT)c->tau;                       // model::data ctor (model_sampler.cpp:24-29)
        mp.stau = h_sqrt<RT>(t);
        mp.s1tau = h_sqrt<RT>((RT)1 - t);
    }
    mp.max_loss = (RT)c->max_loss;
    return mp;
}

int ensure_trace(nmlmc_ctx* c, uint64_t M) {
    if (!c->trace_host) return NMLMC_OK;
    if (M > c->trace_cap) return set_err(NMLMC_ERR_ARG);
    if (c->d_trace_cap < M) {
        dfree(c->d_trace);
        if (dev_malloc(&c->d_trace, M * sizeof(TraceRec)) != cudaSuccess) return set_err(NMLMC_ERR_NOMEM);
        c->d_trace_cap = M;
    }
    return NMLMC_OK;
}

template <class RT>
int sample_core(nmlmc_ctx* c, uint32_t ell, uint64_t M, nmlmc_level_result* out) {
    CoreLaunch<RT> L{};
    L.cores = c->cfg.cores;
    L.ell = ell;
    L.M = M;
    L.seed = c->cfg.seed;
    L.fine_only = ell == 0;
    L.antithetic = c->cfg.antithetic != 0;
    L.adaptive_r = c->cfg.precision == NMLMC_PREC_FP64 ? c->cfg.adaptive_r : (double)(float)c->cfg.adaptive_r;
    L.cf = count_params(c->cfg, ell);
    L.cc = count_params(c->cfg, ell == 0 ? 0 : ell - 1);
    L.mp = model_params<RT>(c);
    if (c->kind == KIND_PORTFOLIO) {
        if constexpr (sizeof(RT) == 4) L.ot = c->dpf32.table; else L.ot = c->dpf64.table;
    }
    TraceRec* tr = c->trace_host ? c->d_trace : nullptr;
    NM_CUDA(cudaEventRecord(c->ev0, c->stream), "event");
    NM_CUDA(launch_core(L, c->kind, c->d_states, c->d_part_sums, c->d_part_stats, c->d_out_sums,
                        c->d_out_stats, tr, c->stream), "core level kernel");
    NM_CUDA(cudaEventRecord(c->ev1, c->stream), "event");
    NM_CUDA(cudaMemcpyAsync(c->h_pin, c->d_out_sums, 10 * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "d2h");
    NM_CUDA(cudaMemcpyAsync(c->h_pin + 16, c->d_out_stats, 6 * sizeof(uint64_t), cudaMemcpyDeviceToHost, c->stream), "d2h");
    if (tr) NM_CUDA(cudaMemcpyAsync(c->trace_host, tr, M * sizeof(TraceRec), cudaMemcpyDeviceToHost, c->stream), "d2h");
    NM_CUDA(cudaStreamSynchronize(c->stream), "sync");
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    for (int j = 0; j < 4; j++) { out->fsums[j] = c->h_pin[j]; out->diffsums[j] = c->h_pin[4 + j]; }
    out->total_work = c->h_pin[8];
    out->M = M;
    memcpy(out->inner_stats, c->h_pin + 16, 6 * sizeof(uint64_t));
    out->seconds = ms * 1e-3;
    c->trace_host = nullptr;
    if (c->h_pin[9] != 0) return set_err(NMLMC_ERR_LIMIT);   // a sample exceeded kMaxPathSteps
    return NMLMC_OK;
}

void prof_mark(void* user, int end, cudaStream_t stream) {
    nmlmc_ctx* c = static_cast<nmlmc_ctx*>(user);
    const size_t idx = 2 * c->pn + (end ? 1 : 0);
    while (c->pev.size() <= idx) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return;
        c->pev.push_back(e);
    }
    cudaEventRecord(c->pev[idx], stream);
    if (end) c->pn++;
}

void prof_collect(nmlmc_ctx* c) {
    for (size_t i = 0; i < c->pn; i++) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, c->pev[2 * i], c->pev[2 * i + 1]) == cudaSuccess) c->prof_seconds += ms * 1e-3;
    }
    c->prof_launches += c->pn;
    c->pn = 0;
}

void fill_outer_result(const nmlmc_ctx* c, const double* a, uint64_t M, double seconds, nmlmc_level_result* out) {
    for (int j = 0; j < 4; j++) { out->fsums[j] = a[j]; out->diffsums[j] = a[4 + j]; }
    out->total_work = a[8];
    out->M = M;
    const uint64_t inner = (uint64_t)a[9];
    out->inner_stats[0] = inner;
    out->inner_stats[1] = M;
    out->inner_stats[2] = (uint64_t)a[10];
    out->inner_stats[3] = (uint64_t)a[11];
    if (c->kind == KIND_PORTFOLIO) {
        out->inner_stats[4] = inner;
        out->inner_stats[5] = M * (c->pf.Q == 1 ? 1 : (uint64_t)c->pf.Q + 1);
    } else {
        out->inner_stats[4] = 0;
        out->inner_stats[5] = M + inner * (c->kind == KIND_REF_MODEL ? 2 : 1);
    }
    out->seconds = seconds;
}

// Default phase configuration: up to 255 registers for the models (their inner loop is ALU-bound
// and gains nothing from more warps), four CTAs per SM for the FP32 portfolio (its option-table
// gathers need the warps to hide L2 latency), chunks of min(N0, 32) inner samples.
// Defaults of the FP32 path, measured per level of the benchmark runs: the portfolio kernel at
// 64 registers (variant 2: four CTAs per SM keep more table gathers in flight), the model kinds at
// 80 (variant 1: fastest or within 0.3 % of it at every level of the adaptive model problem, 3-7 %
// ahead of variant 0).
PhaseChoice default_phase(const nmlmc_ctx* c) {
    PhaseChoice p;
    p.variant = c->cfg.precision != NMLMC_PREC_FP32 ? 0u : c->kind == KIND_PORTFOLIO ? 2u : 1u;
    p.chunk = c->cfg.N0 >= 32 ? 32u : c->cfg.N0;
    return p;
}

bool valid_chunk(const nmlmc_config& k, uint32_t ch);

// The level's tuned or pinned choice; a pinned chunk that no longer divides N0 falls back to the
// default.
PhaseChoice phase_choice(const nmlmc_ctx* c, uint32_t ell) {
    const PhaseChoice& p = c->phase[ell];
    return (p.state && valid_chunk(c->cfg, p.chunk)) ? p : default_phase(c);
}

void reset_phase(nmlmc_ctx* c) {
    for (auto& p : c->phase) {
        if (p.state != 2) p = PhaseChoice{};
    }
}

bool valid_chunk(const nmlmc_config& k, uint32_t ch) {
    return ch >= 4 && ch <= 64 && (ch & (ch - 1)) == 0 && (k.N0 % ch) == 0;
}

template <class RT>
OuterLevel<RT> outer_level_params(const nmlmc_ctx* c, uint32_t ell, uint64_t M, uint64_t first_index) {
    OuterLevel<RT> L{};
    L.ell = ell;
    L.M = M;
    L.first_index = first_index;
    L.seed = c->cfg.seed;
    L.fine_only = ell == 0;
    L.antithetic = c->cfg.antithetic != 0;
    L.N0 = c->cfg.N0;
    const PhaseChoice pc = phase_choice(c, ell);
    L.chunk = pc.chunk;
    L.variant = pc.variant;
    L.adaptive_r = (RT)c->cfg.adaptive_r;
    L.cf = count_params(c->cfg, ell);
    L.cc = count_params(c->cfg, ell == 0 ? 0 : ell - 1);
    const bool adapt = is_adaptive(c->cfg, c->cfg.adaptive_r);
    L.adaptive_f = adapt && L.cf.max_count > 2 * L.cf.base_count;
    L.adaptive_c = !L.fine_only && adapt && L.cc.max_count > 2 * L.cc.base_count;
    L.mp = model_params<RT>(c);
    if (c->kind == KIND_PORTFOLIO) {
        if constexpr (sizeof(RT) == 4) L.ot = c->dpf32.table; else L.ot = c->dpf64.table;
    }
    return L;
}

// ---- phase-kernel autotuner (batched FP32 path) ---------------------------------------------
// The first call of a level that carries enough work to time (>= 4096 outer samples and ~8e6
// inner samples in one batch) times candidate configurations on a probe — the level's own
// parameters on about 20 ms of work (probe_size), from outer samples whose
// stream indices start at 2^55, far from any real index, so the probe changes no result — and
// keeps the fastest for the level:
//   1. the register/occupancy variants 0, 1, 2 (and 3 for the portfolio) at the default chunk
//      length, another than the
//      default taken only if > 3 % faster;
//   2. (mode 2, or an explicit nmlmc_autotune_level) half and double the chunk length at the
//      best variant, taken only if > 3 % faster.
// The variants compute identically, so mode 1 never changes a result; the chunk length changes
// the grouping of the FP32 compensated inner sums (last-bit differences of inner means).
// Pinned levels are not tuned.
constexpr uint64_t kProbeIndex = 1ull << 55;
constexpr double kProbeMs = 20.0;       // device time of one tuning probe

template <class RT>
cudaError_t time_phase_config(nmlmc_ctx* c, uint32_t ell, uint64_t Mp, const PhaseChoice& pc, double& ms_out) {
    OuterLevel<RT> L = outer_level_params<RT>(c, ell, Mp, kProbeIndex);
    L.chunk = pc.chunk;
    L.variant = pc.variant;
    OuterBuffers B = c->ob;
    B.prof_mark = nullptr;
    cudaError_t e = cudaSuccess;
    float ms = 0;
    for (int rep = 0; rep < 2 && e == cudaSuccess; rep++) {       // the first run warms up
        e = cudaEventRecord(c->ev0, c->stream);
        if (e == cudaSuccess) e = outer_level_begin(B, c->stream);
        if (e == cudaSuccess) e = outer_sample_level<RT>(L, c->kind, c->cfg.precision, B, nullptr, c->stream);
        if (e == cudaSuccess) e = cudaEventRecord(c->ev1, c->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(c->ev1);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    }
    ms_out = ms;
    return e;
}

// Probe size, measured: starting from 4096 outer samples, the default configuration is timed on
// growing probes (at most 8x per step, launch overheads make small probes look cheap) until one
// takes kProbeMs of device time or the probe fills one batch.  The probe is not bounded by the
// call's M (its outer samples are not the call's): probes shorter than kProbeMs mis-ranked the
// variants of the large-portfolio levels and kept the default on the model levels whose first
// tuned call was small.  The work per outer sample ranges from the base count to the maximum count
// of the level, too wide to predict from the configuration.
template <class RT>
cudaError_t probe_size(nmlmc_ctx* c, uint32_t ell, uint64_t& Mp) {
    const uint64_t lim = c->ob.cap;
    Mp = lim < 4096 ? lim : 4096;
    for (;;) {
        double ms = 0;
        cudaError_t e = time_phase_config<RT>(c, ell, Mp, default_phase(c), ms);
        if (e != cudaSuccess) return e;
        if (ms >= kProbeMs || Mp >= lim) return cudaSuccess;
        double grow = ms > 0 ? kProbeMs / ms : 8.0;
        if (grow > 8.0) grow = 8.0;
        if (grow < 2.0) grow = 2.0;
        const double next = (double)Mp * grow;
        Mp = next >= (double)lim ? lim : (uint64_t)next;
    }
}

template <class RT>
int tune_level(nmlmc_ctx* c, uint32_t ell, bool chunks) {
    NvtxRange nv("nmlmc autotune level");
    uint64_t Mp = 0;
    NM_CUDA(probe_size<RT>(c, ell, Mp), "autotune probe size");
    // the default stays unless another candidate is more than 3 % faster on the probe (near-ties
    // on a short probe are noise)
    PhaseChoice best = default_phase(c);
    best.state = 1;
    double best_ms;
    NM_CUDA(time_phase_config<RT>(c, ell, Mp, best, best_ms), "autotune probe");
    const uint32_t v0 = best.variant;
    const uint32_t n_var = c->kind == KIND_PORTFOLIO ? 4u : 3u;   // variant 3: portfolio only
    for (uint32_t v = 0; v < n_var; v++) {
        if (v == v0) continue;
        PhaseChoice pc = best;
        pc.variant = v;
        double ms;
        NM_CUDA(time_phase_config<RT>(c, ell, Mp, pc, ms), "autotune probe");
        if (ms < 0.97 * best_ms) { best_ms = ms; best.variant = v; }
    }
    const uint32_t c0 = best.chunk;
    for (uint32_t ch : {c0 / 2, c0 * 2}) {
        if (!chunks || !valid_chunk(c->cfg, ch)) continue;
        PhaseChoice pc = best;
        pc.chunk = ch;
        double ms;
        NM_CUDA(time_phase_config<RT>(c, ell, Mp, pc, ms), "autotune probe");
        if (ms < 0.97 * best_ms) { best_ms = ms; best.chunk = ch; }
    }
    best.probe_ms = best_ms;
    c->phase[ell] = best;
    return NMLMC_OK;
}

// Tunes `ell` if autotuning is on, the level is still on its default configuration and this
// call (M outer samples on this rank) is large enough to time.
template <class RT>
int ensure_tuned(nmlmc_ctx* c, uint32_t ell, uint64_t M) {
    if (!c->autotune || c->cfg.precision != NMLMC_PREC_FP32 || c->phase[ell].state != 0) return NMLMC_OK;
    if (c->kind == KIND_PORTFOLIO && c->pf.mixed()) return NMLMC_OK;   // path methods: one variant
    const uint64_t Mp = M < c->ob.cap ? M : c->ob.cap;
    const CountParams cf = count_params(c->cfg, ell);
    if (Mp < 4096 || (double)Mp * (double)cf.base_count * (double)(ell + 1) < 8.0e6) return NMLMC_OK;
    return tune_level<RT>(c, ell, c->autotune == 2);
}

template <class RT>
int sample_outer(nmlmc_ctx* c, uint32_t ell, uint64_t Mtotal, nmlmc_level_result* out) {
    // this rank's static share of the call's outer samples (all of them when world = 1)
    const uint64_t q = Mtotal / c->shard_world, rem = Mtotal % c->shard_world;
    const uint64_t lo = q * c->shard_rank + (c->shard_rank < rem ? c->shard_rank : rem);
    const uint64_t M = q + (c->shard_rank < rem ? 1 : 0);
    char label[64];
    snprintf(label, sizeof label, "nmlmc level %u M %llu", ell, (unsigned long long)Mtotal);
    NvtxRange nv(label);
    int rc = ensure_tuned<RT>(c, ell, M);
    if (rc) return rc;
    OuterLevel<RT> L = outer_level_params<RT>(c, ell, M, c->next_outer[ell] + lo);
    TraceRec* tr = c->trace_host ? c->d_trace : nullptr;
    c->ob.prof_mark = c->prof ? prof_mark : nullptr;
    c->ob.prof_user = c;
    NM_CUDA(cudaEventRecord(c->ev0, c->stream), "event");
    NM_CUDA(outer_level_begin(c->ob, c->stream), "level begin");
    if (M) NM_CUDA(outer_sample_level<RT>(L, c->kind, c->cfg.precision, c->ob, tr, c->stream), "outer level kernels");
    NM_CUDA(cudaEventRecord(c->ev1, c->stream), "event");
    NM_CUDA(cudaMemcpyAsync(c->h_pin, c->ob.level_acc, 16 * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "d2h");
    if (tr && M) NM_CUDA(cudaMemcpyAsync(c->trace_host, tr, M * sizeof(TraceRec), cudaMemcpyDeviceToHost, c->stream), "d2h");
    uint32_t path_limit = 0;
    const bool paths = c->kind == KIND_PORTFOLIO && c->pf.mixed();
    if (paths)
        NM_CUDA(cudaMemcpyAsync(&path_limit, c->ob.counters + kCounterPathLimit, sizeof path_limit,
                                cudaMemcpyDeviceToHost, c->stream), "d2h");
    NM_CUDA(cudaStreamSynchronize(c->stream), "sync");
    if (path_limit) {                            // a sample exceeded kMaxPathSteps
        NM_CUDA(cudaMemset(c->ob.counters + kCounterPathLimit, 0, sizeof path_limit), "memset");
        return set_err(NMLMC_ERR_LIMIT);
    }
    if (c->prof) prof_collect(c);
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    fill_outer_result(c, c->h_pin, M, ms * 1e-3, out);
    c->next_outer[ell] += Mtotal;
    c->trace_host = nullptr;
    return NMLMC_OK;
}

// This rank's share [lo, lo + M) of a call's Mtotal outer samples.
void shard_range(const nmlmc_ctx* c, uint64_t Mtotal, uint64_t& lo, uint64_t& M) {
    const uint64_t q = Mtotal / c->shard_world, rem = Mtotal % c->shard_world;
    lo = q * c->shard_rank + (c->shard_rank < rem ? c->shard_rank : rem);
    M = q + (c->shard_rank < rem ? 1 : 0);
}

// All levels of one MLMC round in one submission: the level sequences are captured from the
// stream into a CUDA graph (no host round trip inside: device counters size every phase), each
// level accumulating into its own slot; one copy of the slots and one synchronisation per round.
// The executable graph is kept and updated in place (cudaGraphExecUpdate) while later rounds
// have the same topology (the same levels and batch counts), re-instantiated otherwise.
template <class RT>
int sample_outer_levels(nmlmc_ctx* c, uint32_t n, const uint32_t* ells, const uint64_t* Mtot,
                        nmlmc_level_result* outs) {
    NvtxRange nv("nmlmc round submission");
    uint64_t next[NMLMC_MAX_LEVELS];
    memcpy(next, c->next_outer, sizeof(next));
    std::vector<uint64_t> Ms(n);
    for (uint32_t i = 0; i < n; i++) {             // tuning probes run before the capture
        uint64_t lo, M;
        shard_range(c, Mtot[i], lo, M);
        int rc = ensure_tuned<RT>(c, ells[i], M);
        if (rc) return rc;
    }
    NM_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    cudaError_t err = cudaSuccess;
    for (uint32_t i = 0; i < n && err == cudaSuccess; i++) {
        const uint32_t ell = ells[i];
        uint64_t lo, M;
        shard_range(c, Mtot[i], lo, M);
        Ms[i] = M;
        OuterLevel<RT> L = outer_level_params<RT>(c, ell, M, next[ell] + lo);
        next[ell] += Mtot[i];
        OuterBuffers B = c->ob;
        B.level_acc = c->ob.level_acc + 16 * (size_t)i;
        B.prof_mark = nullptr;
        err = launch_stamp(c->d_stamps + 2 * i, c->stream);
        if (err == cudaSuccess) err = outer_level_begin(B, c->stream);
        if (err == cudaSuccess && M) err = outer_sample_level<RT>(L, c->kind, c->cfg.precision, B, nullptr, c->stream);
        if (err == cudaSuccess) err = launch_stamp(c->d_stamps + 2 * i + 1, c->stream);
    }
    uint64_t* h_st = reinterpret_cast<uint64_t*>(c->h_lev + kMaxSubmit * 16);
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(c->h_lev, c->ob.level_acc, (size_t)n * 16 * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(h_st, c->d_stamps, (size_t)n * 2 * sizeof(uint64_t), cudaMemcpyDeviceToHost, c->stream);
    cudaGraph_t graph = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(c->stream, &graph);
    if (err == cudaSuccess) err = e2;
    if (err != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return cuda_status(err, "capture level round");
    }
    // the executable graph of this topology, if a recent round had it: update it in place
    std::vector<uint64_t> key;
    for (uint32_t i = 0; i < n; i++) {
        key.push_back(ells[i]);
        key.push_back((Ms[i] + c->ob.cap - 1) / c->ob.cap);
    }
    GraphSlot* slot = nullptr;
    for (GraphSlot& g : c->graphs)
        if (g.key == key) slot = &g;
    if (slot && slot->exec) {
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(slot->exec, graph, &info) == cudaSuccess) {
            c->graph_updates++;
        } else {
            cudaGetLastError();
            cudaGraphExecDestroy(slot->exec);
            slot->exec = nullptr;
        }
    }
    if (!slot || !slot->exec) {
        cudaGraphExec_t exec = nullptr;
        err = cudaGraphInstantiate(&exec, graph, 0);
        if (err != cudaSuccess) {
            cudaGraphDestroy(graph);
            return cuda_status(err, "instantiate level round");
        }
        c->graph_instantiations++;
        if (!slot) {
            if (c->graphs.size() >= kGraphCache) {        // evict the least recently used
                size_t lru = 0;
                for (size_t j = 1; j < c->graphs.size(); j++)
                    if (c->graphs[j].last_use < c->graphs[lru].last_use) lru = j;
                if (c->graphs[lru].exec) cudaGraphExecDestroy(c->graphs[lru].exec);
                c->graphs.erase(c->graphs.begin() + lru);
            }
            c->graphs.push_back(GraphSlot{key, nullptr, 0});
            slot = &c->graphs.back();
        }
        slot->exec = exec;
    }
    slot->last_use = ++c->graph_clock;
    cudaGraphDestroy(graph);
    NM_CUDA(cudaGraphLaunch(slot->exec, c->stream), "graph launch");
    c->graph_launches++;
    NM_CUDA(cudaStreamSynchronize(c->stream), "sync");
    for (uint32_t i = 0; i < n; i++) {
        const double sec = (double)(h_st[2 * i + 1] - h_st[2 * i]) * 1e-9;
        fill_outer_result(c, c->h_lev + 16 * (size_t)i, Ms[i], sec, &outs[i]);
        c->next_outer[ells[i]] += Mtot[i];
    }
    return NMLMC_OK;
}

}  // namespace

// ============================================================================================
extern "C" {

const char* nmlmc_error_string(int s) {
    switch (s) {
    case NMLMC_OK: return "ok";
    case NMLMC_ERR_ARG: return "invalid argument";
    case NMLMC_ERR_CUDA: return "CUDA error";
    case NMLMC_ERR_STATE: return "call out of order, failed level sampler or state / checkpoint I/O";
    case NMLMC_ERR_NOMEM: return "out of memory";
    case NMLMC_ERR_TIMEOUT: return "bounded device wait gave up";
    case NMLMC_ERR_LIMIT: return "a path-simulated inner sample exceeded NMLMC_MAX_PATH_STEPS";
    default: return "unknown status";
    }
}

int nmlmc_version(void) { return 1; }

int nmlmc_create(nmlmc_ctx** out, int device) {
    if (!out) return set_err(NMLMC_ERR_ARG);
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        fprintf(stderr, "nmlmc: no CUDA device available\n");
        return set_err(NMLMC_ERR_CUDA);
    }
    if (device < 0 || device >= n) return set_err(NMLMC_ERR_ARG);
    NM_CUDA(cudaSetDevice(device), "cudaSetDevice");
    nmlmc_ctx* c = new (std::nothrow) nmlmc_ctx();
    if (!c) return set_err(NMLMC_ERR_NOMEM);
    c->device = device;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
        cudaMallocHost(&c->h_pin, 64 * sizeof(double)) != cudaSuccess ||
        dev_malloc(&c->d_out_sums, 16 * sizeof(double)) != cudaSuccess ||
        dev_malloc(&c->d_out_stats, 8 * sizeof(uint64_t)) != cudaSuccess) {
        nmlmc_destroy(c);
        return set_err(NMLMC_ERR_CUDA);
    }
    *out = c;
    return NMLMC_OK;
}

int nmlmc_destroy(nmlmc_ctx* c) {
    if (!c) return NMLMC_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    free_dev_portfolio(c->dpf32);
    free_dev_portfolio(c->dpf64);
    dfree(c->d_states); dfree(c->d_part_sums); dfree(c->d_part_stats);
    dfree(c->d_out_sums); dfree(c->d_out_stats); dfree(c->d_trace);
    free_outer(c);
    for (cudaEvent_t e : c->pev) cudaEventDestroy(e);
    dfree(c->d_stamps);
    drop_graphs(c);
    if (c->h_lev) cudaFreeHost(c->h_lev);
    if (c->h_pin) cudaFreeHost(c->h_pin);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return NMLMC_OK;
}

int nmlmc_configure(nmlmc_ctx* c, const nmlmc_config* cfg) {
    if (!c || !cfg) return set_err(NMLMC_ERR_ARG);
    nmlmc_config k = *cfg;
    c->batch_default = k.batch == 0;
    if (k.cores == 0) k.cores = 2048;
    if (k.batch == 0) k.batch = 1u << 24;
    // beta: a power of two >= 2 (the adaptive base count N0 * (beta/2)^ell is 0 for beta = 1)
    if (k.N0 == 0 || k.beta < 2 || (k.beta & (k.beta - 1)) != 0) return set_err(NMLMC_ERR_ARG);
    if (k.precision < NMLMC_PREC_REF32 || k.precision > NMLMC_PREC_FP32) return set_err(NMLMC_ERR_ARG);
    if (k.streams != NMLMC_STREAMS_CORE && k.streams != NMLMC_STREAMS_OUTER) return set_err(NMLMC_ERR_ARG);
    if (k.streams == NMLMC_STREAMS_CORE && k.precision == NMLMC_PREC_FP32) return set_err(NMLMC_ERR_ARG);
    if (k.streams == NMLMC_STREAMS_OUTER) {
        // chunks of min(N0, 32) samples must tile every count N0 * 2^k; the breadth-first path
        // implements the antithetic estimator
        const uint32_t ch = k.N0 >= 32 ? 32 : k.N0;
        if ((k.N0 % ch) != 0 || (ch & (ch - 1)) != 0 || ch < 4 || !k.antithetic) return set_err(NMLMC_ERR_ARG);
        if (k.batch > (1ull << 31)) return set_err(NMLMC_ERR_ARG);
    }
    cudaSetDevice(c->device);
    const bool prec_changed = c->cfg.precision != k.precision;
    // a new seed keeps the tuned phase configurations; any other change drops them
    const nmlmc_config& a = c->cfg;
    const bool retune = !c->configured || a.cores != k.cores || a.N0 != k.N0 || a.beta != k.beta ||
                        a.adaptive_r != k.adaptive_r || a.antithetic != k.antithetic ||
                        a.adaptive_incl_r2 != k.adaptive_incl_r2 || a.precision != k.precision ||
                        a.streams != k.streams || a.batch != k.batch;
    c->cfg = k;
    c->configured = true;
    if (prec_changed) c->pf_prec = -1;
    if (retune) reset_phase(c);
    return nmlmc_reset_streams(c);
}

int nmlmc_reset_streams(nmlmc_ctx* c) {
    if (!c || !c->configured) return set_err(NMLMC_ERR_STATE);
    cudaSetDevice(c->device);
    memset(c->next_outer, 0, sizeof(c->next_outer));
    if (c->cfg.streams == NMLMC_STREAMS_CORE) {
        int rc = alloc_core(c);
        if (rc) return rc;
        // init_samplers: both random_state(seed, core) from counter {0,0}, no cached normal
        NM_CUDA(cudaMemset(c->d_states, 0, (size_t)c->cfg.cores * 2 * sizeof(CoreStream)), "reset streams");
    }
    return NMLMC_OK;
}

int nmlmc_set_model(nmlmc_ctx* c, int32_t kind, double tau, double max_loss) {
    if (!c) return set_err(NMLMC_ERR_ARG);
    if (kind != NMLMC_MODEL_REFERENCE && kind != NMLMC_MODEL_SHIFT) return set_err(NMLMC_ERR_ARG);
    // finite inputs; the reference model needs sqrt(tau) and sqrt(1 - tau) (model_sampler.cpp:21-39)
    if (!std::isfinite(tau) || !std::isfinite(max_loss)) return set_err(NMLMC_ERR_ARG);
    if (kind == NMLMC_MODEL_REFERENCE && !(tau >= 0 && tau <= 1)) return set_err(NMLMC_ERR_ARG);
    c->kind = kind;
    c->tau = tau;
    c->max_loss = max_loss;
    c->stau_given = false;
    reset_phase(c);
    return NMLMC_OK;
}

static int set_portfolio_impl(nmlmc_ctx* c, const nmlmc_portfolio* p, const nmlmc_path_methods* pm,
                              double* out_start, double* out_delta) {
    if (!c || !p || !c->configured) return set_err(!c || !p ? NMLMC_ERR_ARG : NMLMC_ERR_STATE);
    if (p->Q == 0 || p->P == 0 || !p->S0 || !p->mu || !p->sigma || !p->strike || !p->maturity || !p->w ||
        !p->stock_ind || !p->type)
        return set_err(NMLMC_ERR_ARG);
    if (p->subsample != NMLMC_SUB_NONE && p->subsample != NMLMC_SUB_RANDOM && p->subsample != NMLMC_SUB_UNIFORM)
        return set_err(NMLMC_ERR_ARG);
    // finite inputs, positive prices and volatilities (a NaN would turn into phi = 0 silently)
    if (!std::isfinite(p->r) || !std::isfinite(p->rho) || !std::isfinite(p->max_loss) || !std::isfinite(p->tau))
        return set_err(NMLMC_ERR_ARG);
    for (uint32_t s = 0; s < p->Q; s++)
        if (!(p->S0[s] > 0) || !std::isfinite(p->S0[s]) || !std::isfinite(p->mu[s]) || !(p->sigma[s] > 0) ||
            !std::isfinite(p->sigma[s]))
            return set_err(NMLMC_ERR_ARG);
    for (uint32_t j = 0; j < p->P; j++)
        if (!(p->strike[j] > 0) || !std::isfinite(p->strike[j]) || !std::isfinite(p->maturity[j]) ||
            !std::isfinite(p->w[j]) || (p->prob && !std::isfinite(p->prob[j])))
            return set_err(NMLMC_ERR_ARG);
    const int32_t* method = pm ? pm->method : nullptr;
    if (pm && (pm->dt_h0inv == 0 || pm->dt_beta < 2 || !(pm->dt_prob_expo < 0)))
        return set_err(NMLMC_ERR_ARG);                     // portfolio_sampler.cpp:525
    HostPortfolio& h = c->pf;
    h = HostPortfolio{};
    h.Q = p->Q;
    h.P = p->P;
    h.S0.assign(p->S0, p->S0 + p->Q);
    h.mu.assign(p->mu, p->mu + p->Q);
    h.sigma.assign(p->sigma, p->sigma + p->Q);
    // stored order: grouped by compute method, the caller's order within a method
    for (int m = 0; m < 3; m++)
        for (uint32_t j = 0; j < p->P; j++) {
            const int32_t mj = method ? method[j] : 0;
            if (mj < 0 || mj > 2) return set_err(NMLMC_ERR_ARG);
            if (mj == m) { h.order.push_back(j); h.m_n[m]++; }
        }
    const bool f32 = c->cfg.precision != NMLMC_PREC_FP64;
    double prev = INFINITY;
    h.type.resize(p->P);
    for (uint32_t k = 0; k < p->P; k++) {
        const uint32_t j = h.order[k];
        if (k == h.m_n[0] || k == h.m_n[0] + h.m_n[1]) prev = INFINITY;
        if (p->stock_ind[j] >= p->Q || (p->type[j] != 1 && p->type[j] != -1)) return set_err(NMLMC_ERR_ARG);
        const double pj = p->prob ? p->prob[j] : 1.0;
        const double pr = f32 ? (double)(float)pj : pj;
        if (!(pr > 0) || !(prev >= pr)) return set_err(NMLMC_ERR_ARG);   // portfolio_sampler.cpp:654
        prev = pr;
        h.strike.push_back(p->strike[j]);
        h.maturity.push_back(p->maturity[j]);
        h.w.push_back(p->w[j]);
        h.prob.push_back(pj);
        h.stock_ind.push_back(p->stock_ind[j]);
        h.type[k] = (int8_t)p->type[j];
    }
    h.W_est.assign(p->P, 1.0);
    h.start.assign(p->P, 0.0);
    h.delta_est.assign(p->P, 0.0);
    h.r = p->r; h.rho = p->rho; h.max_loss = p->max_loss; h.tau = p->tau;
    h.subsample = p->subsample; h.use_delta_cv = p->use_delta_cv; h.discount = p->discount;
    if (pm) {
        h.dt_h0inv = pm->dt_h0inv; h.dt_beta = pm->dt_beta; h.dt_prob_expo = pm->dt_prob_expo;
        h.use_coarse_delta_cv = pm->use_coarse_delta_cv != 0;
        h.use_antithetic_risk = pm->use_antithetic_risk != 0;
        h.use_milstein = pm->use_milstein != 0;
    }
    h.own_params = true;
    if (f32) comp_params<float>(h); else comp_params<double>(h);
    for (uint32_t k = 0; k < p->P; k++) {
        if (out_start) out_start[h.order[k]] = h.start[k];
        if (out_delta) out_delta[h.order[k]] = h.delta_est[k];
    }
    c->kind = KIND_PORTFOLIO;
    c->pf_prec = -1;
    reset_phase(c);
    cudaSetDevice(c->device);
    return ensure_portfolio(c);
}

int nmlmc_set_portfolio(nmlmc_ctx* c, const nmlmc_portfolio* p, double* out_start, double* out_delta) {
    return host_guard([&] { return set_portfolio_impl(c, p, nullptr, out_start, out_delta); });
}

int nmlmc_set_portfolio_methods(nmlmc_ctx* c, const nmlmc_portfolio* p, const nmlmc_path_methods* pm,
                                double* out_start, double* out_delta) {
    if (!pm) return set_err(NMLMC_ERR_ARG);
    return host_guard([&] { return set_portfolio_impl(c, p, pm, out_start, out_delta); });
}

// ---- path-simulated loss and its adjoint -------------------------------------------------------
}  // extern "C"

namespace {

struct DevAlloc {                       // device buffers of one nmlmc_path_adjoint call
    std::vector<void*> ptrs;
    ~DevAlloc() { for (void* p : ptrs) cudaFree(p); }
    template <class T>
    T* get(size_t n) {
        void* p = nullptr;
        if (dev_malloc(&p, (n ? n : 1) * sizeof(T)) != cudaSuccess) return nullptr;
        ptrs.push_back(p);
        return static_cast<T*>(p);
    }
    template <class T>
    T* put(const std::vector<T>& h) {
        T* d = get<T>(h.size());
        if (d && !h.empty() && cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
            return nullptr;
        return d;
    }
};

template <class RT>
int path_adjoint_t(nmlmc_ctx* c, const nmlmc_portfolio_batch* b, const nmlmc_adjoint_config* a,
                   nmlmc_adjoint_result* res, double* gwE, double* gwP, double* gsE, double* gsP,
                   double* loss, double* seconds) {
    const uint32_t n = b->n, NS = b->stock_off[n], NO = b->option_off[n];
    const bool grad = gwE || gwP || gsE || gsP;
    DevAlloc D;
    AdjLaunch<RT> A{};
    A.n = n; A.ell = a->ell; A.pairs = a->inner_pairs; A.M = a->M; A.seed = a->seed;
    A.milstein = a->milstein ? 1 : 0;
    A.tile = 0;
    A.r = (RT)b->r; A.rho = (RT)b->rho; A.tau = (RT)b->tau;
    A.s1_rho2 = (RT)sqrt(1 - b->rho * b->rho); A.stau = (RT)sqrt(b->tau); A.disc_tau = (RT)exp(-b->r * b->tau);
    std::vector<uint32_t> so(b->stock_off, b->stock_off + n + 1), oo(b->option_off, b->option_off + n + 1);
    std::vector<uint32_t> co(n + 1, 0);
    uint32_t qmax = 0;
    for (uint32_t p = 0; p < n; p++) {
        co[p + 1] = co[p] + (oo[p + 1] - oo[p] + 127) / 128;
        qmax = std::max(qmax, so[p + 1] - so[p]);
    }
    A.n_chunks = co[n];
    A.q_max = qmax;
    // outer samples per CTA: at most kAdjMaxTile, and small enough for about 32 CTAs of four
    // warps per SM (two waves at full occupancy) when the option chunks alone are too few
    {
        const uint64_t want = 148ull * 32;
        const uint64_t rows = (want + A.n_chunks - 1) / A.n_chunks;
        const uint64_t t = (a->M + rows - 1) / rows;
        A.tile = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>({kAdjMaxTile, a->M, t}));
    }
    std::vector<RT> S0(NS), mu(NS), sg(NS), K(NO), T(NO), w(NO), V0(NO), vega(NO);
    std::vector<int8_t> ty(NO);
    std::vector<uint32_t> si(b->stock_ind, b->stock_ind + NO);
    for (uint32_t j = 0; j < NS; j++) { S0[j] = (RT)b->S0[j]; mu[j] = (RT)b->mu[j]; sg[j] = (RT)b->sigma[j]; }
    for (uint32_t p = 0; p < n; p++)
        for (uint32_t i = oo[p]; i < oo[p + 1]; i++) {
            const uint32_t s = so[p] + si[i];
            const double Sd = b->S0[s], sd = b->sigma[s], Kd = b->strike[i], Td = b->maturity[i];
            K[i] = (RT)Kd; T[i] = (RT)Td; w[i] = (RT)b->w[i]; ty[i] = (int8_t)b->type[i];
            V0[i] = (RT)h_calc_bs<double>(b->type[i], Sd, Kd, b->r, Td, sd);
            const double d1 = h_d1<double>(Sd, Kd, b->r, Td, sd);
            vega[i] = (RT)(Sd * exp(-0.5 * d1 * d1) * 0.39894228040143268 * sqrt(Td));   // S0 phi(d1) sqrt(T)
        }
    std::vector<double> Kp(n), dl(n);
    for (uint32_t p = 0; p < n; p++) {
        Kp[p] = b->K[p];
        dl[p] = b->K[p] != 0 ? a->delta_rel * fabs(b->K[p]) : a->delta_rel;
    }
    A.stock_off = D.put(so); A.option_off = D.put(oo); A.chunk_off = D.put(co);
    A.S0 = D.put(S0); A.mu = D.put(mu); A.sigma = D.put(sg);
    A.strike = D.put(K); A.maturity = D.put(T); A.w = D.put(w); A.V0 = D.put(V0); A.vega = D.put(vega);
    A.stock_ind = D.put(si); A.type = D.put(ty); A.K = D.put(Kp); A.delta = D.put(dl);
    A.R = D.get<RT>((size_t)NS * a->M); A.dR = D.get<RT>((size_t)NS * a->M);
    A.L = D.get<double>((size_t)n * a->M); A.omega = D.get<double>((size_t)n * a->M);
    A.est = D.get<double>(3 * n); A.wE = D.get<double>(n);
    A.gw_E = D.get<double>(NO); A.gw_P = D.get<double>(NO); A.gs_E = D.get<double>(NS); A.gs_P = D.get<double>(NS);
    if (!A.stock_off || !A.option_off || !A.chunk_off || !A.S0 || !A.mu || !A.sigma || !A.strike || !A.maturity ||
        !A.w || !A.V0 || !A.vega || !A.stock_ind || !A.type || !A.K || !A.delta || !A.R || !A.dR || !A.L ||
        !A.omega || !A.est || !A.wE || !A.gw_E || !A.gw_P || !A.gs_E || !A.gs_P)
        return set_err(NMLMC_ERR_NOMEM);
    NM_CUDA(cudaMemsetAsync(A.L, 0, (size_t)n * a->M * sizeof(double), c->stream), "memset");
    NM_CUDA(cudaMemsetAsync(A.gw_E, 0, NO * sizeof(double), c->stream), "memset");
    NM_CUDA(cudaMemsetAsync(A.gw_P, 0, NO * sizeof(double), c->stream), "memset");
    NM_CUDA(cudaMemsetAsync(A.gs_E, 0, NS * sizeof(double), c->stream), "memset");
    NM_CUDA(cudaMemsetAsync(A.gs_P, 0, NS * sizeof(double), c->stream), "memset");
    NM_CUDA(cudaEventRecord(c->ev0, c->stream), "event");
    NM_CUDA(launch_adjoint(A, grad, c->stream), "adjoint kernels");
    NM_CUDA(cudaEventRecord(c->ev1, c->stream), "event");
    std::vector<double> est(3 * n);
    NM_CUDA(cudaMemcpyAsync(est.data(), A.est, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "d2h");
    if (loss) NM_CUDA(cudaMemcpyAsync(loss, A.L, (size_t)n * a->M * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "d2h");
    if (gwE) NM_CUDA(cudaMemcpyAsync(gwE, A.gw_E, NO * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "d2h");
    if (gwP) NM_CUDA(cudaMemcpyAsync(gwP, A.gw_P, NO * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "d2h");
    if (gsE) NM_CUDA(cudaMemcpyAsync(gsE, A.gs_E, NS * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "d2h");
    if (gsP) NM_CUDA(cudaMemcpyAsync(gsP, A.gs_P, NS * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "d2h");
    NM_CUDA(cudaStreamSynchronize(c->stream), "sync");
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    if (seconds) *seconds = ms * 1e-3;
    for (uint32_t p = 0; p < n; p++) res[p] = nmlmc_adjoint_result{est[3 * p], est[3 * p + 1], est[3 * p + 2]};
    return NMLMC_OK;
}

}  // namespace

extern "C" {

int nmlmc_path_adjoint(nmlmc_ctx* c, const nmlmc_portfolio_batch* b, const nmlmc_adjoint_config* a,
                       nmlmc_adjoint_result* res, double* gwE, double* gwP, double* gsE, double* gsP,
                       double* loss, double* seconds) {
    if (!c || !b || !a || !res || b->n == 0 || b->n >= (1u << 24) || !b->stock_off || !b->option_off ||
        !b->S0 || !b->mu || !b->sigma || !b->strike || !b->maturity || !b->w || !b->stock_ind || !b->type || !b->K)
        return set_err(NMLMC_ERR_ARG);
    if (a->ell > 16 || a->inner_pairs == 0 || a->M == 0 || a->M >= (1ull << 32) || !(a->delta_rel > 0) ||
        (a->precision != NMLMC_PREC_FP32 && a->precision != NMLMC_PREC_FP64) || !(b->tau > 0) ||
        !(fabs(b->rho) < 1))
        return set_err(NMLMC_ERR_ARG);
    for (uint32_t p = 0; p < b->n; p++) {
        const uint32_t Q = b->stock_off[p + 1] - b->stock_off[p], P = b->option_off[p + 1] - b->option_off[p];
        if (b->stock_off[p + 1] <= b->stock_off[p] || b->option_off[p + 1] <= b->option_off[p]) return set_err(NMLMC_ERR_ARG);
        for (uint32_t i = b->option_off[p]; i < b->option_off[p + 1]; i++)
            if (b->stock_ind[i] >= Q || (b->type[i] != 1 && b->type[i] != -1) || !(b->maturity[i] > b->tau))
                return set_err(NMLMC_ERR_ARG);
        (void)P;
    }
    if (b->stock_off[0] != 0 || b->option_off[0] != 0) return set_err(NMLMC_ERR_ARG);
    cudaSetDevice(c->device);
    return host_guard([&] {
        return a->precision == NMLMC_PREC_FP64 ? path_adjoint_t<double>(c, b, a, res, gwE, gwP, gsE, gsP, loss, seconds)
                                               : path_adjoint_t<float>(c, b, a, res, gwE, gwP, gsE, gsP, loss, seconds);
    });
}

int nmlmc_set_trace(nmlmc_ctx* c, nmlmc_trace_rec* host_buf, uint64_t cap) {
    if (!c) return set_err(NMLMC_ERR_ARG);
    c->trace_host = host_buf;
    c->trace_cap = host_buf ? cap : 0;
    return NMLMC_OK;
}

int nmlmc_sample(nmlmc_ctx* c, uint32_t ell, uint64_t M, nmlmc_level_result* out) {
    if (!c || !out) return set_err(NMLMC_ERR_ARG);
    if (!c->configured || c->kind < 0) return set_err(NMLMC_ERR_STATE);
    if (ell >= NMLMC_MAX_LEVELS) return set_err(NMLMC_ERR_ARG);
    memset(out, 0, sizeof(*out));
    out->M = M;
    const nmlmc_config& k = c->cfg;
    // counts must fit the 32-bit per-item counters of the batched path
    if ((double)k.N0 * pow((double)k.beta, (double)ell) > 4.0e9) return set_err(NMLMC_ERR_ARG);
    // the batched (OUTER) layout draws one option per inner sample: no Subsampling::None there
    if (c->kind == KIND_PORTFOLIO && k.streams == NMLMC_STREAMS_OUTER && c->pf.subsample == SUB_NONE)
        return set_err(NMLMC_ERR_ARG);
    if (M == 0) return NMLMC_OK;
    cudaSetDevice(c->device);
    int rc = ensure_portfolio(c);
    if (rc) return rc;
    if ((rc = ensure_trace(c, M))) return rc;
    const bool f64 = k.precision == NMLMC_PREC_FP64;
    if (k.streams == NMLMC_STREAMS_CORE) {
        if ((rc = alloc_core(c))) return rc;
        return f64 ? sample_core<double>(c, ell, M, out) : sample_core<float>(c, ell, M, out);
    }
    if ((rc = alloc_outer(c, (M + c->shard_world - 1) / c->shard_world))) return rc;
    return f64 ? sample_outer<double>(c, ell, M, out) : sample_outer<float>(c, ell, M, out);
}

int nmlmc_sample_levels(nmlmc_ctx* c, uint32_t n, const uint32_t* ells, const uint64_t* Ms,
                        nmlmc_level_result* outs) {
    if (!c || (n && (!ells || !Ms || !outs))) return set_err(NMLMC_ERR_ARG);
    if (!c->configured || c->kind < 0) return set_err(NMLMC_ERR_STATE);
    const nmlmc_config& k = c->cfg;
    if (c->kind == KIND_PORTFOLIO && k.streams == NMLMC_STREAMS_OUTER && c->pf.subsample == SUB_NONE)
        return set_err(NMLMC_ERR_ARG);          // as nmlmc_sample: no Subsampling::None on the batched layout
    bool one_submission = n > 0 && n <= kMaxSubmit && k.streams == NMLMC_STREAMS_OUTER && !c->prof &&
                          !c->trace_host && !(c->kind == KIND_PORTFOLIO && c->pf.mixed());
    for (uint32_t i = 0; i < n && one_submission; i++) {
        if (ells[i] >= NMLMC_MAX_LEVELS || (double)k.N0 * pow((double)k.beta, (double)ells[i]) > 4.0e9)
            return set_err(NMLMC_ERR_ARG);
    }
    if (one_submission) {
        cudaSetDevice(c->device);
        uint64_t want = 0;
        for (uint32_t i = 0; i < n; i++) {
            const uint64_t m = (Ms[i] + c->shard_world - 1) / c->shard_world;
            if (m > want) want = m;
        }
        int rc = ensure_portfolio(c);
        if (rc || (rc = alloc_outer(c, want))) return rc;
        if (!c->h_lev && cudaMallocHost(&c->h_lev, kMaxSubmit * 18 * sizeof(double)) != cudaSuccess)
            return set_err(NMLMC_ERR_NOMEM);
        if (!c->d_stamps && dev_malloc(&c->d_stamps, kMaxSubmit * 2 * sizeof(uint64_t)) != cudaSuccess)
            return set_err(NMLMC_ERR_NOMEM);
        for (uint32_t i = 0; i < n; i++) memset(&outs[i], 0, sizeof(outs[i]));
        return k.precision == NMLMC_PREC_FP64 ? sample_outer_levels<double>(c, n, ells, Ms, outs)
                                              : sample_outer_levels<float>(c, n, ells, Ms, outs);
    }
    for (uint32_t i = 0; i < n; i++) {
        int rc = nmlmc_sample(c, ells[i], Ms[i], &outs[i]);
        if (rc) return rc;
    }
    return NMLMC_OK;
}

// ---- sampler state (checkpoints of the MLMC driver) --------------------------------------------
// Blob: SamplerStateHeader, then (CORE layout) cores x 2 CoreStream records as on the device.
namespace {
struct SamplerStateHeader {
    char magic[8];
    uint32_t streams, cores;
    uint64_t seed;
    uint32_t N0, beta;
    double adaptive_r;
    int32_t precision, antithetic;
    uint32_t shard_rank, shard_world;
    uint64_t next_outer[NMLMC_MAX_LEVELS];
    uint64_t core_bytes;
};
constexpr char kStateMagic[8] = {'N', 'M', 'L', 'M', 'C', 'S', 'S', '1'};
}  // namespace

int nmlmc_get_sampler_state(nmlmc_ctx* c, void* buf, size_t cap, size_t* size) {
    if (!c || !size) return set_err(NMLMC_ERR_ARG);
    if (!c->configured) return set_err(NMLMC_ERR_STATE);
    const bool core = c->cfg.streams == NMLMC_STREAMS_CORE;
    const uint64_t core_bytes = core ? (uint64_t)c->cfg.cores * 2 * sizeof(CoreStream) : 0;
    *size = sizeof(SamplerStateHeader) + core_bytes;
    if (!buf) return NMLMC_OK;
    if (cap < *size) return set_err(NMLMC_ERR_ARG);
    SamplerStateHeader h;
    memset(&h, 0, sizeof h);
    memcpy(h.magic, kStateMagic, 8);
    h.streams = (uint32_t)c->cfg.streams;
    h.cores = c->cfg.cores;
    h.seed = c->cfg.seed;
    h.N0 = c->cfg.N0;
    h.beta = c->cfg.beta;
    h.adaptive_r = c->cfg.adaptive_r;
    h.precision = c->cfg.precision;
    h.antithetic = c->cfg.antithetic;
    h.shard_rank = c->shard_rank;
    h.shard_world = c->shard_world;
    memcpy(h.next_outer, c->next_outer, sizeof(h.next_outer));
    h.core_bytes = core_bytes;
    memcpy(buf, &h, sizeof h);
    if (core_bytes) {
        cudaSetDevice(c->device);
        int rc = alloc_core(c);
        if (rc) return rc;
        NM_CUDA(cudaStreamSynchronize(c->stream), "sync");
        NM_CUDA(cudaMemcpy(static_cast<char*>(buf) + sizeof h, c->d_states, core_bytes, cudaMemcpyDeviceToHost),
                "sampler state d2h");
    }
    return NMLMC_OK;
}

int nmlmc_set_sampler_state(nmlmc_ctx* c, const void* buf, size_t size) {
    if (!c || !buf || size < sizeof(SamplerStateHeader)) return set_err(NMLMC_ERR_ARG);
    if (!c->configured) return set_err(NMLMC_ERR_STATE);
    SamplerStateHeader h;
    memcpy(&h, buf, sizeof h);
    if (memcmp(h.magic, kStateMagic, 8) != 0) return set_err(NMLMC_ERR_ARG);
    // the state belongs to the same streams: layout, cores, seed, counts and precision
    if (h.streams != (uint32_t)c->cfg.streams || h.cores != c->cfg.cores || h.seed != c->cfg.seed ||
        h.N0 != c->cfg.N0 || h.beta != c->cfg.beta || h.adaptive_r != c->cfg.adaptive_r ||
        h.precision != c->cfg.precision || h.antithetic != c->cfg.antithetic ||
        h.shard_rank != c->shard_rank || h.shard_world != c->shard_world)
        return set_err(NMLMC_ERR_ARG);
    const uint64_t core_bytes = c->cfg.streams == NMLMC_STREAMS_CORE ? (uint64_t)c->cfg.cores * 2 * sizeof(CoreStream) : 0;
    if (h.core_bytes != core_bytes || size != sizeof h + core_bytes) return set_err(NMLMC_ERR_ARG);
    memcpy(c->next_outer, h.next_outer, sizeof(c->next_outer));
    if (core_bytes) {
        cudaSetDevice(c->device);
        int rc = alloc_core(c);
        if (rc) return rc;
        NM_CUDA(cudaStreamSynchronize(c->stream), "sync");
        NM_CUDA(cudaMemcpy(c->d_states, static_cast<const char*>(buf) + sizeof h, core_bytes, cudaMemcpyHostToDevice),
                "sampler state h2d");
    }
    return NMLMC_OK;
}

int nmlmc_set_shard(nmlmc_ctx* c, uint32_t rank, uint32_t world) {
    if (!c || world == 0 || rank >= world) return set_err(NMLMC_ERR_ARG);
    if (world > 1 && c->cfg.streams != NMLMC_STREAMS_OUTER) return set_err(NMLMC_ERR_ARG);
    c->shard_rank = rank;
    c->shard_world = world;
    return NMLMC_OK;
}

int nmlmc_set_profiling(nmlmc_ctx* c, int32_t on) {
    if (!c) return set_err(NMLMC_ERR_ARG);
    c->prof = on != 0;
    c->prof_launches = 0;
    c->prof_seconds = 0;
    c->pn = 0;
    return NMLMC_OK;
}

int nmlmc_phase_kernel_time(nmlmc_ctx* c, uint64_t* launches, double* seconds) {
    if (!c || !launches || !seconds) return set_err(NMLMC_ERR_ARG);
    *launches = c->prof_launches;
    *seconds = c->prof_seconds;
    return NMLMC_OK;
}

uint64_t nmlmc_kernel_launches(void) { return launches_total(); }

int nmlmc_set_autotune(nmlmc_ctx* c, int32_t mode) {
    if (!c || mode < 0 || mode > 2) return set_err(NMLMC_ERR_ARG);
    c->autotune = mode;
    return NMLMC_OK;
}

int nmlmc_get_phase_config(nmlmc_ctx* c, uint32_t ell, nmlmc_phase_config* out) {
    if (!c || !out || ell >= NMLMC_MAX_LEVELS) return set_err(NMLMC_ERR_ARG);
    if (!c->configured) return set_err(NMLMC_ERR_STATE);
    const PhaseChoice p = phase_choice(c, ell);
    out->variant = p.variant;
    out->chunk = p.chunk;
    out->state = c->phase[ell].state;
    out->probe_ms = p.probe_ms;
    return NMLMC_OK;
}

int nmlmc_set_phase_config(nmlmc_ctx* c, uint32_t ell, const nmlmc_phase_config* cfg) {
    if (!c || ell >= NMLMC_MAX_LEVELS) return set_err(NMLMC_ERR_ARG);
    if (!c->configured) return set_err(NMLMC_ERR_STATE);
    if (!cfg) {                                   // unpin: back to the default, tunable again
        c->phase[ell] = PhaseChoice{};
        return NMLMC_OK;
    }
    if (cfg->variant > 3 || !valid_chunk(c->cfg, cfg->chunk)) return set_err(NMLMC_ERR_ARG);
    PhaseChoice p;
    p.state = 2;
    p.variant = cfg->variant;
    p.chunk = cfg->chunk;
    c->phase[ell] = p;
    return NMLMC_OK;
}

int nmlmc_autotune_level(nmlmc_ctx* c, uint32_t ell, uint64_t M) {
    if (!c || ell >= NMLMC_MAX_LEVELS || M == 0) return set_err(NMLMC_ERR_ARG);
    if (!c->configured || c->kind < 0) return set_err(NMLMC_ERR_STATE);
    if (c->cfg.streams != NMLMC_STREAMS_OUTER || c->cfg.precision != NMLMC_PREC_FP32) return set_err(NMLMC_ERR_ARG);
    if ((double)c->cfg.N0 * pow((double)c->cfg.beta, (double)ell) > 4.0e9) return set_err(NMLMC_ERR_ARG);
    cudaSetDevice(c->device);
    int rc = ensure_portfolio(c);
    if (rc || (rc = alloc_outer(c, M))) return rc;
    if (c->kind == KIND_PORTFOLIO && c->pf.mixed()) return set_err(NMLMC_ERR_ARG);
    return tune_level<float>(c, ell, true);
}

int nmlmc_inject_alloc_failure(int32_t after) {
    if (after < -1) return set_err(NMLMC_ERR_ARG);
    g_fail_alloc.store(after);
    return NMLMC_OK;
}

int nmlmc_graph_stats(nmlmc_ctx* c, uint64_t* instantiations, uint64_t* updates, uint64_t* launches) {
    if (!c || !instantiations || !updates || !launches) return set_err(NMLMC_ERR_ARG);
    *instantiations = c->graph_instantiations;
    *updates = c->graph_updates;
    *launches = c->graph_launches;
    return NMLMC_OK;
}

int nmlmc_portfolio_full_loss(nmlmc_ctx* c, uint32_t ell, uint64_t first, uint64_t n, double* host_loss) {
    if (!c || !host_loss) return set_err(NMLMC_ERR_ARG);
    if (!c->configured || c->kind != KIND_PORTFOLIO) return set_err(NMLMC_ERR_STATE);
    if (n == 0) return NMLMC_OK;
    cudaSetDevice(c->device);
    int rc = ensure_portfolio(c);
    if (rc || (rc = alloc_outer(c, n))) return rc;
    double* d_loss = nullptr;
    if (dev_malloc(&d_loss, n * sizeof(double)) != cudaSuccess) return set_err(NMLMC_ERR_NOMEM);
    cudaError_t e;
    if (c->cfg.precision == NMLMC_PREC_FP64) {
        OuterLevel<double> L{};
        L.ell = ell; L.M = n; L.first_index = first; L.seed = c->cfg.seed; L.ot = c->dpf64.table;
        e = outer_full_loss<double>(L, c->cfg.precision, c->ob, d_loss, c->stream);
    } else {
        OuterLevel<float> L{};
        L.ell = ell; L.M = n; L.first_index = first; L.seed = c->cfg.seed; L.ot = c->dpf32.table;
        e = outer_full_loss<float>(L, c->cfg.precision, c->ob, d_loss, c->stream);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(host_loss, d_loss, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(d_loss);
    return cuda_status(e, "full loss");
}

int nmlmc_threefry_blocks(const uint64_t* ctr, const uint64_t* key, uint64_t* out, uint64_t n) {
    if (!ctr || !key || !out) return set_err(NMLMC_ERR_ARG);
    if (n == 0) return NMLMC_OK;
    uint64_t* d = nullptr;
    if (dev_malloc(&d, 6 * n * sizeof(uint64_t)) != cudaSuccess) return set_err(NMLMC_ERR_NOMEM);
    cudaError_t e = cudaMemcpy(d, ctr, 2 * n * sizeof(uint64_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d + 2 * n, key, 2 * n * sizeof(uint64_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = launch_threefry_blocks(d, d + 2 * n, d + 4 * n, n, 0);
    if (e == cudaSuccess) e = cudaMemcpy(out, d + 4 * n, 2 * n * sizeof(uint64_t), cudaMemcpyDeviceToHost);
    cudaFree(d);
    return cuda_status(e, "threefry blocks");
}

int nmlmc_outer_normals(int32_t precision, uint64_t seed, uint64_t stream, uint32_t tag, uint64_t n,
                        double* out) {
    if (!out || (precision != NMLMC_PREC_FP32 && precision != NMLMC_PREC_FP64)) return set_err(NMLMC_ERR_ARG);
    if (n == 0) return NMLMC_OK;
    double* d = nullptr;
    if (dev_malloc(&d, n * sizeof(double)) != cudaSuccess) return set_err(NMLMC_ERR_NOMEM);
    cudaError_t e = launch_outer_normals(precision, seed, stream, tag, n, d, 0);
    if (e == cudaSuccess) e = cudaMemcpy(out, d, n * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d);
    return cuda_status(e, "outer normals");
}

int nmlmc_norm_cdf_fast(const float* x, float* out, uint64_t n) {
    if (!x || !out) return set_err(NMLMC_ERR_ARG);
    if (n == 0) return NMLMC_OK;
    float* d = nullptr;
    if (dev_malloc(&d, 2 * n * sizeof(float)) != cudaSuccess) return set_err(NMLMC_ERR_NOMEM);
    cudaError_t e = cudaMemcpy(d, x, n * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = launch_norm_cdf_fast(d, d + n, n, 0);
    if (e == cudaSuccess) e = cudaMemcpy(out, d + n, n * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(d);
    return cuda_status(e, "norm_cdf_fast");
}

// ---- reference-named surface (one process-wide sampler, like g_p_nestedmc_data) --------------
static nmlmc_ctx* g_ctx = nullptr;
static int32_t g_default_prec = NMLMC_PREC_REF32, g_default_streams = NMLMC_STREAMS_CORE;
static int g_last = NMLMC_OK;
static std::mutex g_mu;
// moments the caller's sample_output arrays hold (nested_sampler_params fine/diff_moments):
// the reference copies exactly that many sums back (nested_sampler.hpp:571)
static uint32_t g_fine_moments = 4, g_diff_moments = 4;

static void ref_fail(int rc, const char* fn) {
    g_last = rc;
    if (rc != NMLMC_OK) fprintf(stderr, "nmlmc: %s failed: %s\n", fn, nmlmc_error_string(rc));
}

int nmlmc_last_error(void) { return g_last; }

}  // extern "C"

// The status that nmlmc_last_error() reports, for entry points outside this file.
int nmlmc::set_last_error(int e) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_last = e;
    return set_err(e);
}

extern "C" {

// Records the status of a reference-named call implemented in another translation unit
// (portfolio_gen_data / portfolio_free_data in nmlmc_portfolio.cpp).  Not part of the ABI.
__attribute__((visibility("hidden"))) void nmlmc_ref_status(int rc, const char* fn) {
    std::lock_guard<std::mutex> lk(g_mu);
    ref_fail(rc, fn);
}

int nmlmc_default_set_precision(int32_t precision, int32_t streams) {
    if (precision < NMLMC_PREC_REF32 || precision > NMLMC_PREC_FP32) return NMLMC_ERR_ARG;
    if (streams != NMLMC_STREAMS_CORE && streams != NMLMC_STREAMS_OUTER) return NMLMC_ERR_ARG;
    g_default_prec = precision;
    g_default_streams = streams;
    return NMLMC_OK;
}

void init_nestedmc_sampler(uint32_t cores, const nested_sampler_params* params) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!params) return ref_fail(NMLMC_ERR_ARG, "init_nestedmc_sampler");
    if (params->fine_moments > 4 || params->diff_moments > 4)   // c_max_moments (nested_sampler.hpp:5)
        return ref_fail(NMLMC_ERR_ARG, "init_nestedmc_sampler");
    if (!g_ctx) {
        int rc = nmlmc_create(&g_ctx, 0);
        if (rc) return ref_fail(rc, "init_nestedmc_sampler");
    }
    g_fine_moments = params->fine_moments;
    g_diff_moments = params->diff_moments;
    nmlmc_config k{};
    k.cores = cores;
    k.N0 = params->N0;
    k.beta = params->beta;
    k.adaptive_r = (double)params->adaptive_r;
    k.antithetic = params->antithetic ? 1 : 0;
    k.precision = g_default_prec;
    k.streams = g_default_streams;
    k.seed = 0;
    ref_fail(nmlmc_configure(g_ctx, &k), "init_nestedmc_sampler");
}

void cleanup_nestedmc_sampler(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    nmlmc_destroy(g_ctx);
    g_ctx = nullptr;
    g_last = NMLMC_OK;
}

void model_update_data(const model_data* d) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_ctx || !d) return ref_fail(!d ? NMLMC_ERR_ARG : NMLMC_ERR_STATE, "model_update_data");
    g_ctx->kind = KIND_REF_MODEL;
    g_ctx->stau = d->stau;
    g_ctx->s1tau = d->s1tau;
    g_ctx->max_loss = d->max_loss;
    g_ctx->stau_given = true;
    g_last = NMLMC_OK;
}

void model_init(const model_data* d, uint64_t seed) {
    model_update_data(d);
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_last) return;
    g_ctx->cfg.seed = seed;
    ref_fail(nmlmc_reset_streams(g_ctx), "model_init");
}

static void fill_sample_output(const nmlmc_level_result& r, sample_output* out) {
    out->M = r.M;
    if (out->fsums) for (uint32_t j = 0; j < g_fine_moments; j++) out->fsums[j] = r.fsums[j];
    if (out->diffsums) for (uint32_t j = 0; j < g_diff_moments; j++) out->diffsums[j] = r.diffsums[j];
    out->total_work = r.total_work;
    memcpy(out->inner_stats, r.inner_stats, sizeof(out->inner_stats));
}

void model_sample(uint32_t ell, uint64_t M, sample_output* out) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_ctx || !out) return ref_fail(!out ? NMLMC_ERR_ARG : NMLMC_ERR_STATE, "model_sample");
    if (g_ctx->kind != KIND_REF_MODEL) return ref_fail(NMLMC_ERR_STATE, "model_sample");
    nmlmc_level_result r;
    int rc = nmlmc_sample(g_ctx, ell, M, &r);
    if (rc) return ref_fail(rc, "model_sample");
    fill_sample_output(r, out);
    g_last = NMLMC_OK;
}

static int portfolio_from_ref(const portfolio_data* d) {
    if (d->phi_type != 0) return NMLMC_ERR_ARG;                          // Indicator only
    const nmlmc_stocks_span& s = d->stocks;
    size_t P = 0;
    for (int m = 0; m < 3; m++) {
        if (d->options[m].size && !d->options[m].data) return NMLMC_ERR_ARG;
        P += d->options[m].size;
    }
    if (!P || !s.size || !s.data) return NMLMC_ERR_ARG;
    if (d->options[1].size + d->options[2].size &&
        (d->dt_h0inv == 0 || d->dt_beta < 2 || !(d->dt_prob_expo < 0)))
        return NMLMC_ERR_ARG;                                            // portfolio_sampler.cpp:525
    HostPortfolio& h = g_ctx->pf;
    h = HostPortfolio{};
    h.Q = (uint32_t)s.size;
    h.P = (uint32_t)P;
    for (size_t i = 0; i < s.size; i++) {
        h.S0.push_back(s.data[i].S0); h.mu.push_back(s.data[i].mu); h.sigma.push_back(s.data[i].sigma);
    }
    // options[m] in order, as portfolio_update_data stores them (portfolio_sampler.cpp:647-668)
    for (int m = 0; m < 3; m++) {
        const nmlmc_options_span& o = d->options[m];
        float prev = INFINITY;
        for (size_t j = 0; j < o.size; j++) {
            const option_params& op = o.data[j];
            if (op.stock_ind >= s.size || !(op.prob > 0) || !(prev >= op.prob)) return NMLMC_ERR_ARG;
            prev = op.prob;
            h.strike.push_back(op.strike); h.maturity.push_back(op.maturity); h.w.push_back(op.w);
            h.prob.push_back(op.prob); h.W_est.push_back(op.W_est); h.start.push_back(op.start);
            h.delta_est.push_back(op.delta_est); h.stock_ind.push_back(op.stock_ind);
            h.type.push_back((int8_t)(op.type > 0 ? 1 : -1));
            h.order.push_back((uint32_t)h.order.size());
        }
        h.m_n[m] = (uint32_t)o.size;
    }
    h.r = d->r; h.rho = d->rho; h.s1_rho2 = d->s1_rho2; h.s1_rho2_given = true;
    h.max_loss = d->max_loss; h.tau = d->tau;
    h.subsample = d->subsample; h.use_delta_cv = d->use_delta_cv ? 1 : 0; h.discount = 1;
    h.dt_h0inv = d->dt_h0inv; h.dt_beta = d->dt_beta; h.dt_prob_expo = d->dt_prob_expo;
    h.use_coarse_delta_cv = d->use_coarse_delta_cv ? 1 : 0;
    h.use_antithetic_risk = d->use_antithetic_risk ? 1 : 0;
    h.use_milstein = d->use_milstein ? 1 : 0;
    g_ctx->kind = KIND_PORTFOLIO;
    g_ctx->pf_prec = -1;
    return ensure_portfolio(g_ctx);
}

void portfolio_update_data(const portfolio_data* d) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_ctx || !d) return ref_fail(!d ? NMLMC_ERR_ARG : NMLMC_ERR_STATE, "portfolio_update_data");
    ref_fail(host_guard([&] { return portfolio_from_ref(d); }), "portfolio_update_data");
}

void portfolio_init(const portfolio_data* d, uint64_t seed) {
    portfolio_update_data(d);
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_last) return;
    g_ctx->cfg.seed = seed;
    ref_fail(nmlmc_reset_streams(g_ctx), "portfolio_init");
}

void portfolio_sample(uint32_t ell, uint64_t override_dyn_inner, uint64_t M, sample_output* out) {
    (void)override_dyn_inner;   // child-grid width of the reference's CUDA build; no counterpart
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_ctx || !out) return ref_fail(!out ? NMLMC_ERR_ARG : NMLMC_ERR_STATE, "portfolio_sample");
    if (g_ctx->kind != KIND_PORTFOLIO) return ref_fail(NMLMC_ERR_STATE, "portfolio_sample");
    nmlmc_level_result r;
    int rc = nmlmc_sample(g_ctx, ell, M, &r);
    if (rc) return ref_fail(rc, "portfolio_sample");
    fill_sample_output(r, out);
    g_last = NMLMC_OK;
}

void portfolio_cleanup(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_ctx) return;
    free_dev_portfolio(g_ctx->dpf32);
    free_dev_portfolio(g_ctx->dpf64);
    g_ctx->pf = HostPortfolio{};
    g_ctx->pf_prec = -1;
    if (g_ctx->kind == KIND_PORTFOLIO) g_ctx->kind = -1;
}

void portfolio_comp_params(portfolio_data* d) {
    if (!d) { g_last = NMLMC_ERR_ARG; return; }
    for (int m = 0; m < 3; m++) {
        for (size_t j = 0; j < d->options[m].size; j++) {
            option_params& op = d->options[m].data[j];
            const stock_params& s = d->stocks.data[op.stock_ind];
            int type = op.type > 0 ? 1 : -1;
            op.start = h_calc_bs<float>(type, s.S0, op.strike, d->r, op.maturity, s.sigma);
            op.delta_est = h_calc_delta<float>(type, s.S0, op.strike, d->r, op.maturity, s.sigma);
        }
    }
    g_last = NMLMC_OK;
}

float norm_cdf_inv(float p) { return h_norm_cdf_inv<float>(p); }

}  // extern "C"
