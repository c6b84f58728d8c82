// Test-infrastructure harness around the UNMODIFIED reference sources.
//
// This translation unit is compiled by oracle/Makefile with the reference tree on the include
// path; it includes the reference's own common.cpp, model_sampler.cpp and portfolio_sampler.cpp
// exactly as they lie and adds a flat extern "C" surface that the test suite (ctypes) and the
// fixture generator (tests/golden/make_golden.py) call.  It is a checker only: nothing in the
// product links or loads it.
//
// What it adds on top of the reference:
//   * ref_threefry / ref_stream_draws: raw Threefry2x64-20 blocks and random_state draws
//     (Random123/threefry.h:190-286, par_omp.hpp:72-121).
//   * shift_model::sampler: the X = Y + Z model (Y ~ N(0,1), inner X = Y + Z, start = -K),
//     plugged into the reference engine through the same SAMPLER concept as model::sampler
//     (model_sampler.cpp:42-92).  The reference has no such model; the engine that drives it
//     (nested_sampler.hpp:369-485, 646-694) is the reference's own.
//   * traced<S>: a SAMPLER wrapper whose hooks log, per outer sample, the inner counts handed to
//     init_inner_sampler and the inner means handed to add_phi, so per-outer-sample parity can
//     be checked against the reference's own kernel_sample loop.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>
#include <omp.h>
#include <cstddef>
#include <string>

#include "common.cpp"
#include "model_sampler.cpp"
#include "portfolio_sampler.cpp"

// ---------------------------------------------------------------------------------------------
// Per-thread event log used by traced<S>.
//   kind 'O' : sample_outer (start of an outer sample)
//   kind 'I' : init_inner_sampler(count)      value = count
//   kind 'P' : add_phi(mean, coeff)           value = mean, aux = coeff
struct ref_event { char kind; double value; double aux; };
static std::vector<std::vector<ref_event>> g_events;
static bool g_trace_on = false;

static inline void log_event(char k, double v, double a) {
    if (!g_trace_on) return;
    g_events[omp_get_thread_num()].push_back(ref_event{k, v, a});
}

template <class BASE>
class traced : public BASE {
public:
    PAR_DEVICE traced(void* w) : BASE(w) {}
    PAR_DEVICE void sample_outer(uint64_t ell, work_t& w) { log_event('O', 0, 0); BASE::sample_outer(ell, w); }
    PAR_DEVICE real_t init_inner_sampler(uint64_t& count, work_t& w) {
        log_event('I', (double)count, 0);
        return BASE::init_inner_sampler(count, w);
    }
    static PAR_DEVICE void add_phi(real_t avg, real_t coeff, real_t* phi) {
        log_event('P', (double)avg, (double)coeff);
        BASE::add_phi(avg, coeff, phi);
    }
};

// ---------------------------------------------------------------------------------------------
// The X = Y + Z model of the nested-risk problem P(E[X|Y] > K).
namespace shift_model {
    struct data { real_t K; };
    static data g_data;

    class sampler : public inner_sampler_base {
        real_t Y;
    public:
        static uint32_t GetWorkspaceSize(const data&) { return 0; }
        sampler(void*) : Y(NAN) {}
        void sample_outer(uint64_t, work_t&) { Y = randn_sync(); }
        void copy_outer(const sampler& rhs) { Y = rhs.Y; }
        real_t init_inner_sampler(uint64_t&, work_t&) { return -g_data.K; }
        real_t sample_inner(uint64_t, uint64_t, work_t& total_work) {
            total_work++;
            return Y + randn();
        }
        static void add_phi(real_t inner_avg, real_t coeff, real_t* phi) {
            *phi += coeff * (inner_avg >= 0.f);
        }
    };
}

extern "C" {

int ref_real_size() { return (int)sizeof(real_t); }

// out[2*i], out[2*i+1] = Threefry2x64-20(ctr_i, key_i)
void ref_threefry(const uint64_t* ctr, const uint64_t* key, uint64_t* out, uint64_t n) {
    r123::Threefry2x64 rng;
    for (uint64_t i = 0; i < n; i++) {
        r123::Threefry2x64::ctr_type c = {{ctr[2 * i], ctr[2 * i + 1]}};
        r123::Threefry2x64::key_type k = {{key[2 * i], key[2 * i + 1]}};
        r123::Threefry2x64::ctr_type r = rng(c, k);
        out[2 * i] = r.v[0];
        out[2 * i + 1] = r.v[1];
    }
}

// Replays a script of draws on one random_state(seed, core).  ops[i] = 'r' (raw rand(), the
// 64-bit word is stored bitwise in out_u64[i]), 'u' (randu), 'n' (randn); out_real[i] holds the
// real_t result widened to double.
void ref_stream_draws(uint64_t seed, uint64_t core, const char* ops, uint64_t n,
                      double* out_real, uint64_t* out_u64) {
    random_state st(seed, core);
    for (uint64_t i = 0; i < n; i++) {
        out_u64[i] = 0;
        out_real[i] = 0;
        switch (ops[i]) {
        case 'r': out_u64[i] = st.rand(); break;
        case 'u': out_real[i] = (double)st.randu(); break;
        case 'n': out_real[i] = (double)st.randn(); break;
        default: break;
        }
    }
}

// r123::boxmuller(u0, u1) in double (Random123/boxmuller.hpp:128-137).
void ref_boxmuller(const uint64_t* u0, const uint64_t* u1, double* x, double* y, uint64_t n) {
    for (uint64_t i = 0; i < n; i++) {
        r123::double2 d = r123::boxmuller(u0[i], u1[i]);
        x[i] = d.x;
        y[i] = d.y;
    }
}

void ref_set_threads(int t) { omp_set_num_threads(t); }

// init_nestedmc_sampler with fine/diff moments = 4 (the mains' mlmc_real::moments).
void ref_nested_init(uint32_t cores, uint32_t N0, uint32_t beta, double adaptive_r, int antithetic) {
    if (g_p_nestedmc_data) cleanup_nestedmc_sampler();
    nested_sampler_params p(4, 4, N0, beta, (real_t)adaptive_r, antithetic != 0);
    init_nestedmc_sampler(cores, &p);
    g_events.assign(cores, {});
}

void ref_cleanup() {
    if (g_p_nestedmc_data) cleanup_nestedmc_sampler();
}

// kind 0: reference model::sampler (tau, max_loss); kind 1: X = Y + Z model (K = max_loss).
static int g_model_kind = 0;
void ref_model_init(int kind, double tau, double max_loss, uint64_t seed, int traced_run) {
    g_model_kind = kind * 2 + (traced_run ? 1 : 0);
    if (kind == 0) {
        model::data d(model::PhiType::Indicator, (real_t)tau, (real_t)max_loss);
        model::model_update_data(&d);
        if (traced_run) init_samplers<traced<model::sampler>>(seed, 0);
        else init_samplers<model::sampler>(seed, 0);
    } else {
        shift_model::g_data.K = (real_t)max_loss;
        PAR_SET_CONST(gc_phi_size, 1u);
        if (traced_run) init_samplers<traced<shift_model::sampler>>(seed, 0);
        else init_samplers<shift_model::sampler>(seed, 0);
    }
}

static void run_sample(int which, uint32_t ell, uint64_t M, sample_output* out) {
    out->M = M;
    switch (which) {
    case 0: sample<model::sampler>(ell, 0, &out->M, out->fsums, out->diffsums, &out->total_work, out->inner_stats); break;
    case 1: sample<traced<model::sampler>>(ell, 0, &out->M, out->fsums, out->diffsums, &out->total_work, out->inner_stats); break;
    case 2: sample<shift_model::sampler>(ell, 0, &out->M, out->fsums, out->diffsums, &out->total_work, out->inner_stats); break;
    case 3: sample<traced<shift_model::sampler>>(ell, 0, &out->M, out->fsums, out->diffsums, &out->total_work, out->inner_stats); break;
    case 4: sample<portfolio::sampler>(ell, 0, &out->M, out->fsums, out->diffsums, &out->total_work, out->inner_stats); break;
    case 5: sample<traced<portfolio::sampler>>(ell, 0, &out->M, out->fsums, out->diffsums, &out->total_work, out->inner_stats); break;
    }
}

static void copy_out(const sample_output& o, double* fsums, double* diffsums, double* work, uint64_t* stats) {
    for (int i = 0; i < 4; i++) { fsums[i] = o.fsums[i]; diffsums[i] = o.diffsums[i]; }
    *work = o.total_work;
    for (int i = 0; i < c_inner_stats_count; i++) stats[i] = o.inner_stats[i];
}

// Flattens the per-thread event logs (thread 0 first: the static schedule gives thread t a
// contiguous block of outer samples, so this is outer-sample order).  Returns the event count
// written, or -(needed) if cap is too small.
static int64_t flush_events(char* kinds, double* values, double* aux, uint64_t cap) {
    uint64_t n = 0;
    for (auto& v : g_events) n += v.size();
    if (n > cap) { for (auto& v : g_events) v.clear(); return -(int64_t)n; }
    uint64_t k = 0;
    for (auto& v : g_events) {
        for (auto& e : v) { kinds[k] = e.kind; values[k] = e.value; aux[k] = e.aux; k++; }
        v.clear();
    }
    return (int64_t)n;
}

// One sample(ell, M) call; if the model was initialised with traced_run, the event log of the
// call is written to kinds/values/aux (cap entries).
int64_t ref_model_sample(uint32_t ell, uint64_t M, double* fsums, double* diffsums, double* work,
                         uint64_t* stats, char* kinds, double* values, double* aux, uint64_t cap) {
    sample_output out(4, 4, 1);
    g_trace_on = (g_model_kind & 1) != 0;
    run_sample(g_model_kind, ell, M, &out);
    g_trace_on = false;
    copy_out(out, fsums, diffsums, work, stats);
    if (g_model_kind & 1) return flush_events(kinds, values, aux, cap);
    return 0;
}

// Portfolio set-up from flat arrays.  Options are all ComputeMethod::BS (the only method on
// the measured path); prob must be > 0 and non-increasing (portfolio_sampler.cpp:654).
// subsample: 0 None, 1 Random (CDF), -1 Random_Uniform.  Fills start/delta_est through the
// reference's own portfolio_comp_params.
static portfolio::data g_pdata;
static std::vector<portfolio::option_params> g_opts;
static std::vector<portfolio::stock_params> g_stocks;
static bool g_port_traced = false;

static std::vector<portfolio::option_params> g_opts_m[3];

// Mixed compute methods: method[j] in {0 BS, 1 Exact, 2 Unbiased}; options keep their order
// within a method (prob must be non-increasing within each method).  dt_* and the flags are the
// portfolio::data fields of the path-simulated methods (portfolio_sampler.cpp:74-87).
void ref_portfolio_init_methods(uint32_t Q, const double* S0, const double* mu, const double* sigma,
                                uint32_t P, const double* strike, const double* maturity,
                                const double* w, const uint32_t* stock_ind, const int32_t* type,
                                const double* prob, const int32_t* method, double r, double rho,
                                double max_loss, double tau, int subsample, int use_delta_cv,
                                int use_coarse_delta_cv, int use_antithetic_risk, int use_milstein,
                                uint32_t dt_h0inv, uint32_t dt_beta, double dt_prob_expo,
                                uint64_t seed, int traced_run) {
    g_stocks.resize(Q);
    for (uint32_t i = 0; i < Q; i++) {
        g_stocks[i].S0 = (real_t)S0[i]; g_stocks[i].mu = (real_t)mu[i]; g_stocks[i].sigma = (real_t)sigma[i];
    }
    for (int m = 0; m < 3; m++) g_opts_m[m].clear();
    for (uint32_t j = 0; j < P; j++) {
        portfolio::option_params o;
        o.strike = (real_t)strike[j]; o.maturity = (real_t)maturity[j]; o.w = (real_t)w[j];
        o.stock_ind = stock_ind[j];
        o.type = type[j] > 0 ? portfolio::OptionType::Call : portfolio::OptionType::Put;
        o.prob = (prob_t)prob[j]; o.W_est = 1; o.start = 0; o.delta_est = 0;
        g_opts_m[method[j]].push_back(o);
    }
    portfolio::data& d = g_pdata;
    for (int m = 0; m < 3; m++)
        d.options[m] = portfolio::options_array::create(g_opts_m[m].empty() ? nullptr : g_opts_m[m].data(),
                                                        g_opts_m[m].size());
    d.stocks = portfolio::stocks_array::create(g_stocks.data(), Q);
    d.r = (real_t)r; d.rho = (real_t)rho; d.s1_rho2 = std::sqrt(1 - POW2(d.rho));
    d.max_loss = (real_t)max_loss; d.tau = (real_t)tau;
    d.dt_h0inv = dt_h0inv; d.dt_beta = dt_beta; d.dt_prob_expo = (real_t)dt_prob_expo;
    d.phi_type = portfolio::PhiType::Indicator; d._phi_size = 1;
    d.subsample = (portfolio::Subsampling)subsample;
    d.use_delta_cv = use_delta_cv != 0; d.use_coarse_delta_cv = use_coarse_delta_cv != 0;
    d.use_antithetic_risk = use_antithetic_risk != 0; d.use_milstein = use_milstein != 0;
    portfolio::portfolio_comp_params(&d);
    portfolio::portfolio_update_data(&d);
    g_port_traced = traced_run != 0;
    if (g_port_traced)
        init_samplers<traced<portfolio::sampler>>(seed, portfolio::sampler::GetWorkspaceSize(d));
    else
        init_samplers<portfolio::sampler>(seed, portfolio::sampler::GetWorkspaceSize(d));
}

void ref_portfolio_init(uint32_t Q, const double* S0, const double* mu, const double* sigma,
                        uint32_t P, const double* strike, const double* maturity, const double* w,
                        const uint32_t* stock_ind, const int32_t* type, const double* prob,
                        double r, double rho, double max_loss, double tau, int subsample,
                        int use_delta_cv, uint64_t seed, int traced_run,
                        double* out_start, double* out_delta_est) {
    g_stocks.resize(Q);
    for (uint32_t i = 0; i < Q; i++) {
        g_stocks[i].S0 = (real_t)S0[i]; g_stocks[i].mu = (real_t)mu[i]; g_stocks[i].sigma = (real_t)sigma[i];
    }
    g_opts.resize(P);
    for (uint32_t j = 0; j < P; j++) {
        auto& o = g_opts[j];
        o.strike = (real_t)strike[j]; o.maturity = (real_t)maturity[j]; o.w = (real_t)w[j];
        o.stock_ind = stock_ind[j];
        o.type = type[j] > 0 ? portfolio::OptionType::Call : portfolio::OptionType::Put;
        o.prob = (prob_t)prob[j]; o.W_est = 1; o.start = 0; o.delta_est = 0;
    }
    portfolio::data& d = g_pdata;
    d.options[0] = portfolio::options_array::create(g_opts.data(), P);
    d.options[1] = portfolio::options_array::create(nullptr, 0);
    d.options[2] = portfolio::options_array::create(nullptr, 0);
    d.stocks = portfolio::stocks_array::create(g_stocks.data(), Q);
    d.r = (real_t)r; d.rho = (real_t)rho; d.s1_rho2 = std::sqrt(1 - POW2(d.rho));
    d.max_loss = (real_t)max_loss; d.tau = (real_t)tau;
    d.dt_h0inv = 8; d.dt_beta = 4; d.dt_prob_expo = -1.5;
    d.phi_type = portfolio::PhiType::Indicator; d._phi_size = 1;
    d.subsample = (portfolio::Subsampling)subsample;
    d.use_delta_cv = use_delta_cv != 0; d.use_coarse_delta_cv = false;
    d.use_antithetic_risk = true; d.use_milstein = true;
    portfolio::portfolio_comp_params(&d);
    for (uint32_t j = 0; j < P; j++) { out_start[j] = g_opts[j].start; out_delta_est[j] = g_opts[j].delta_est; }
    portfolio::portfolio_update_data(&d);
    g_port_traced = traced_run != 0;
    if (g_port_traced)
        init_samplers<traced<portfolio::sampler>>(seed, portfolio::sampler::GetWorkspaceSize(d));
    else
        init_samplers<portfolio::sampler>(seed, portfolio::sampler::GetWorkspaceSize(d));
}

int64_t ref_portfolio_sample(uint32_t ell, uint64_t M, double* fsums, double* diffsums, double* work,
                             uint64_t* stats, char* kinds, double* values, double* aux, uint64_t cap) {
    sample_output out(4, 4, 1);
    g_trace_on = g_port_traced;
    run_sample(g_port_traced ? 5 : 4, ell, M, &out);
    g_trace_on = false;
    copy_out(out, fsums, diffsums, work, stats);
    if (g_port_traced) return flush_events(kinds, values, aux, cap);
    return 0;
}

void ref_portfolio_cleanup() { portfolio::portfolio_cleanup(); }

// Black-Scholes price / delta exactly as the reference evaluates them (real_t arithmetic).
void ref_bs(int type, const double* S, const double* K, double r, const double* t,
            const double* sigma, double* price, double* delta, uint64_t n) {
    auto ty = type > 0 ? portfolio::OptionType::Call : portfolio::OptionType::Put;
    for (uint64_t i = 0; i < n; i++) {
        price[i] = portfolio::calc_option_blackscholes(ty, (real_t)S[i], (real_t)K[i], (real_t)r, (real_t)t[i], (real_t)sigma[i]);
        delta[i] = portfolio::calc_delta_blackscholes(ty, (real_t)S[i], (real_t)K[i], (real_t)r, (real_t)t[i], (real_t)sigma[i]);
    }
}

// gbm_approx.hpp:18-57 on one path set (size paths, fine + coarse when with_coarse); draws come
// from random_state(seed, core).randn().  S has 2*size entries when with_coarse.  Returns W_T.
double ref_simulate_stock_dt(int with_coarse, uint64_t seed, uint64_t core, double* S, uint64_t N,
                             double mu, double sigma, double t, uint32_t size, int milstein,
                             uint32_t coarse_step) {
    random_state st(seed, core);
    auto rn = [&st]() { return st.randn(); };
    std::vector<sum_t> s(S, S + (with_coarse ? 2 * size : size));
    real_t W;
    if (with_coarse)
        W = simulate_stock_dt<true>(rn, s.data(), N, (real_t)mu, (real_t)sigma, (real_t)t, size, milstein != 0, coarse_step);
    else
        W = simulate_stock_dt<false>(rn, s.data(), N, (real_t)mu, (real_t)sigma, (real_t)t, size, milstein != 0, coarse_step);
    for (size_t i = 0; i < s.size(); i++) S[i] = s[i];
    return W;
}

// norm_cdf_inv (common.cpp:53-86).
double ref_norm_cdf_inv(double p) { return (double)norm_cdf_inv((real_t)p); }

// ---------------------------------------------------------------------------------------------
// mlmc_t::run (mlmc.hpp:290-337) driven by a deterministic synthetic level sampler, to pin the
// host continuation-MLMC driver.  Each sample_level(ell, M) call returns sums of a synthetic
// level with mean a*2^(-alpha*ell), variance v*2^(-beta*ell) and work w*2^(gamma*ell) built
// from a splitmix64 stream (no reference randomness involved).  The call sequence (ell, M) and
// the final levels are written out.
static uint64_t sm_state;
static double sm_next() {
    uint64_t z = (sm_state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

int64_t ref_mlmc_synthetic(double targetTOL, uint64_t M0, double a, double alpha, double v,
                           double beta, double w, double gamma, uint64_t seed,
                           uint32_t* call_ell, uint64_t* call_M, uint64_t cap,
                           double* out_levels /* [ell][4 fine,4 diff, work, M] */, uint32_t lvl_cap,
                           uint32_t* out_nlevels, double* out_misc /* starting_level,bias,stat,TOL */,
                           char* table, uint64_t table_cap) {
    sm_state = seed;
    uint64_t ncalls = 0;
    mlmc_t<double, 4>::mlmc_input_t in;
    in.targetTOL = targetTOL;
    in.M0 = M0;
    in.verbose = false;
    in.sample_level = [&](uint32_t ell, uint64_t M) {
        if (ncalls < cap) { call_ell[ncalls] = ell; call_M[ncalls] = M; }
        ncalls++;
        mlmc_t<double, 4>::mc_diff_output_t o;
        double mf = a * std::pow(2.0, -alpha * ell) + 0.1;
        double md = ell == 0 ? 0 : a * std::pow(2.0, -alpha * ell);
        double sd_f = std::sqrt(v), sd_d = std::sqrt(v * std::pow(2.0, -beta * ell));
        // sums of M synthetic draws: uniform noise with the requested sd, so all moments are finite
        const uint64_t n = M < 64 ? M : 64;   // stratified: 64 representative draws scaled
        for (uint64_t i = 0; i < n; i++) {
            double u = (sm_next() - 0.5) * std::sqrt(12.0);
            double f = mf + sd_f * u, d = md + sd_d * u;
            double pf = 1, pd = 1;
            for (int j = 0; j < 4; j++) {
                pf *= f; pd *= d;
                o.sums_fine[j] += pf * ((double)M / n);
                o.sums_diff[j] += ell == 0 ? 0 : pd * ((double)M / n);
            }
        }
        o.M = M;
        o.work = w * std::pow(2.0, gamma * ell) * M;
        o.time = 0;
        return o;
    };
    auto out = mlmc_t<double, 4>::run(in);
    *out_nlevels = (uint32_t)out.levels.size();
    for (uint32_t l = 0; l < out.levels.size() && l < lvl_cap; l++) {
        double* p = out_levels + l * 10;
        for (int j = 0; j < 4; j++) { p[j] = out.levels[l].sums_fine[j]; p[4 + j] = out.levels[l].sums_diff[j]; }
        p[8] = out.levels[l].work; p[9] = (double)out.levels[l].M;
    }
    out_misc[0] = out.starting_level; out_misc[1] = out.bias_est; out_misc[2] = out.stat_error; out_misc[3] = out.TOL;
    if (table && table_cap) {
        std::string str = out.to_string();
        size_t n = str.size() < table_cap - 1 ? str.size() : table_cap - 1;
        memcpy(table, str.data(), n);
        table[n] = 0;
    }
    return (int64_t)ncalls;
}

// sizeof / offsetof of the reference structs that cross its C ABI.
void ref_abi_sizes(uint64_t* out) {
    out[0] = sizeof(nested_sampler_params);
    out[1] = sizeof(sample_output);
    out[2] = sizeof(model::data);
    out[3] = sizeof(portfolio::data);
    out[4] = sizeof(portfolio::option_params);
    out[5] = sizeof(portfolio::stock_params);
    out[6] = offsetof(nested_sampler_params, adaptive_r);
    out[7] = offsetof(sample_output, inner_stats);
    out[8] = offsetof(portfolio::data, subsample);
    out[9] = offsetof(portfolio::data, use_milstein);
    out[10] = offsetof(portfolio::option_params, W_est);
    out[11] = offsetof(model::data, phi_type);
}

}  // extern "C"
