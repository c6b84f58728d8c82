// Seeded synthetic option portfolios (host, C++).
//
// The benchmark portfolios are specified by distributions (stocks: sigma ~ U[lo, hi]; options:
// uniformly chosen stock, call with a given probability, strike ~ U[lo, hi] * S0, maturity ~
// U[lo, hi], position ~ N(0, 1)).  Every random field is drawn from a counter-based Threefry2x64-20
// stream — value(field f, index i) = Threefry(ctr = (i, f), key = (seed, 'PORTGEN')) — so a
// portfolio is a pure function of (spec, seed), independent of platform, thread count and
// generation order.
//
// The reference's own demo generator, portfolio_gen_data / portfolio_free_data
// (portfolio_sampler.cpp:784-912), is part of its extern "C" surface and is provided below with
// the same outputs (same seeds, same libstdc++ random engines and distributions, same delta hedge,
// normalisation and per-method sort), so the reference's portfolio main runs unchanged against
// this library.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <memory>
#include <new>
#include <random>
#include <stdexcept>
#include <vector>

#include "../../include/nmlmc.h"

extern "C" void nmlmc_ref_status(int rc, const char* fn);   // nmlmc_api.cu

namespace {

inline uint64_t rotl(uint64_t x, unsigned r) { return (x << r) | (x >> (64 - r)); }

// Threefry2x64-20 (Random123/threefry.h:86-93, 171, 190-286), host copy of the device function.
void threefry(uint64_t c0, uint64_t c1, uint64_t k0, uint64_t k1, uint64_t& o0, uint64_t& o1) {
    static const unsigned R[8] = {16, 42, 12, 31, 16, 32, 24, 21};
    const uint64_t ks[3] = {k0, k1, 0x1BD11BDAA9FC1A22ull ^ k0 ^ k1};
    uint64_t x0 = c0 + ks[0], x1 = c1 + ks[1];
    for (unsigned r = 0; r < 20; r++) {
        x0 += x1;
        x1 = rotl(x1, R[r & 7]);
        x1 ^= x0;
        if ((r & 3) == 3) {
            const unsigned s = (r >> 2) + 1;
            x0 += ks[s % 3];
            x1 += ks[(s + 1) % 3] + s;
        }
    }
    o0 = x0;
    o1 = x1;
}

constexpr uint64_t kGenKey = 0x4e454754524f50ull;   // "PORTGEN"

enum Field : uint64_t { F_SIGMA = 1, F_ASSET = 2, F_TYPE = 3, F_STRIKE = 4, F_MATURITY = 5, F_WEIGHT = 6 };

struct Gen {
    uint64_t seed;
    uint64_t raw(Field f, uint64_t i, int which = 0) const {
        uint64_t a, b;
        threefry(i, f, seed, kGenKey, a, b);
        return which ? b : a;
    }
    double u01(Field f, uint64_t i) const {          // (0, 1), 53 bits
        return ((double)(raw(f, i) >> 11) + 0.5) * 0x1p-53;
    }
    double normal(Field f, uint64_t i) const {       // Box-Muller on the block's two words
        uint64_t a, b;
        threefry(i, f, seed, kGenKey, a, b);
        const double u1 = ((double)(a >> 11) + 0.5) * 0x1p-53, u2 = ((double)(b >> 11) + 0.5) * 0x1p-53;
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * 3.141592653589793 * u2);
    }
};

}  // namespace

extern "C" int nmlmc_portfolio_generate(const nmlmc_portfolio_spec* sp, uint64_t seed, double* S0,
                                        double* mu, double* sigma, double* strike, double* maturity,
                                        double* w, uint32_t* stock_ind, int32_t* type) {
    if (!sp || !S0 || !mu || !sigma || !strike || !maturity || !w || !stock_ind || !type) return NMLMC_ERR_ARG;
    if (sp->Q == 0 || sp->P == 0 || !(sp->sigma_hi >= sp->sigma_lo) || !(sp->strike_hi >= sp->strike_lo) ||
        !(sp->maturity_hi >= sp->maturity_lo) || !(sp->call_fraction >= 0 && sp->call_fraction <= 1))
        return NMLMC_ERR_ARG;
    const Gen g{seed};
    for (uint32_t j = 0; j < sp->Q; j++) {
        S0[j] = sp->S0;
        mu[j] = sp->mu;
        sigma[j] = sp->sigma_lo + (sp->sigma_hi - sp->sigma_lo) * g.u01(F_SIGMA, j);
    }
    for (uint32_t i = 0; i < sp->P; i++) {
        const unsigned __int128 prod = (unsigned __int128)g.raw(F_ASSET, i) * sp->Q;
        stock_ind[i] = (uint32_t)(prod >> 64);                       // exact uniform index
        type[i] = g.u01(F_TYPE, i) < sp->call_fraction ? 1 : -1;
        strike[i] = sp->S0 * (sp->strike_lo + (sp->strike_hi - sp->strike_lo) * g.u01(F_STRIKE, i));
        maturity[i] = sp->maturity_lo + (sp->maturity_hi - sp->maturity_lo) * g.u01(F_MATURITY, i);
        w[i] = g.normal(F_WEIGHT, i);
    }
    return NMLMC_OK;
}

// ---- the reference's demo generator (portfolio_sampler.cpp:784-912) -------------------------
//
// Steps that decide the values, in the reference's order:
//  * one std::mt19937 seeded with `seed`; every field is drawn from a fresh copy of that seeded
//    engine (the reference hands the engine to std::bind by value, so each field restarts from
//    the same state): S0 ~ U(90, 110), sigma ~ U(0.01, 0.4), mu ~ U(0.03, 0.3), type ~ U{0, 1},
//    stock ~ U{0, Q-1}, maturity ~ U(1, 5), strike ~ U(80, 120), weight ~ N(0, 1), all real_t =
//    float;
//  * options i < Q and Q + i are a call and a put on stock i (so P >= 2Q);
//  * options[m] takes the next floor(probs[m] * P) options (m = BS, Exact, Unbiased), which must
//    add up to P;
//  * start / delta_est from portfolio_comp_params; the calls' weights on each stock are scaled
//    by -(sum of put delta * w) / (sum of call delta * w) (a delta hedge, sums in double), then
//    every weight is divided by the sum of all weights;
//  * prob = |w| / sqrt(W_est) (or 1 with uniform_prob), W_est = 1, and each method's options are
//    sorted by decreasing prob with std::sort.
// Two reference behaviours are not carried over: with uniform_weights the reference leaves every
// weight at 0 (so the normalisation divides 0 by 0) where its caller documents weights of 1, and
// the reference's W_est update of the Unbiased options changes a copy (so W_est stays 1, as here).
static portfolio_data gen_data(uint32_t P, uint32_t Q, uint64_t seed, const double* probs,
                               bool uniform_weights, bool uniform_prob) {
    portfolio_data d{};
    if (!probs || Q == 0 || (uint64_t)P < 2ull * Q) {
        nmlmc_ref_status(NMLMC_ERR_ARG, "portfolio_gen_data");
        return d;
    }
    uint32_t count[3];
    uint64_t total = 0;
    for (int m = 0; m < 3; m++) {
        if (!(probs[m] >= 0)) {
            nmlmc_ref_status(NMLMC_ERR_ARG, "portfolio_gen_data");
            return d;
        }
        count[m] = (uint32_t)(probs[m] * P);
        total += count[m];
    }
    if (total != P) {                         // the reference asserts this
        nmlmc_ref_status(NMLMC_ERR_ARG, "portfolio_gen_data");
        return d;
    }
    d.r = 0.05f;
    d.rho = 0.2f;
    d.s1_rho2 = std::sqrt(1 - d.rho * d.rho);
    d.max_loss = 0.7f;
    d.tau = 0.02f;
    d.dt_h0inv = 8;
    d.dt_beta = 4;
    d.dt_prob_expo = -1.5f;
    d.phi_type = 0;                           // Indicator
    d._phi_size = 1;
    d.subsample = NMLMC_SUB_NONE;
    d.use_delta_cv = true;
    d.use_coarse_delta_cv = false;
    d.use_antithetic_risk = true;
    d.use_milstein = true;

    const std::mt19937 engine(seed);
    auto draw = [&engine](auto& out, auto dist) {
        std::mt19937 g = engine;              // each field from the seeded state
        for (auto& x : out) x = dist(g);
    };
    using uni = std::uniform_real_distribution<float>;
    using unii = std::uniform_int_distribution<uint32_t>;
    std::vector<float> S0(Q), sigma(Q), mu(Q), maturity(P, 1.f), strike(P), weight(P, 1.f);
    std::vector<uint32_t> type(P), stock(P);
    draw(S0, uni(90, 110));
    draw(sigma, uni(0.01, 0.4));
    draw(mu, uni(0.03, 0.3));
    draw(type, unii(0, 1));
    draw(stock, unii(0, Q - 1));
    draw(maturity, uni(1, 5));
    draw(strike, uni(80, 120));
    if (!uniform_weights) draw(weight, std::normal_distribution<float>(0, 1));

    std::unique_ptr<option_params[]> ops_owner(new option_params[P]());
    std::unique_ptr<stock_params[]> stocks_owner(new stock_params[Q]());
    option_params* ops = ops_owner.get();
    stock_params* stocks = stocks_owner.get();
    for (uint32_t i = 0; i < Q; i++) {
        type[i] = 0;
        type[Q + i] = 1;
        stock[i] = stock[Q + i] = i;
        stocks[i].S0 = S0[i];
        stocks[i].mu = mu[i];
        stocks[i].sigma = sigma[i];
    }
    for (uint32_t i = 0; i < P; i++) {
        ops[i].w = weight[i];
        ops[i].strike = strike[i];
        ops[i].type = type[i] ? -1 : 1;       // 1: put, 0: call
        ops[i].maturity = maturity[i];
        ops[i].stock_ind = stock[i];
        ops[i].prob = -1;
        ops[i].W_est = 1;
    }
    d.stocks.data = stocks;
    d.stocks.size = Q;
    uint32_t off = 0;
    for (int m = 0; m < 3; m++) {
        d.options[m].data = ops + off;
        d.options[m].size = count[m];
        off += count[m];
    }
    portfolio_comp_params(&d);

    std::vector<double> call_dw(Q, 0.0), put_dw(Q, 0.0);
    for (int m = 0; m < 3; m++)
        for (size_t j = 0; j < d.options[m].size; j++) {
            const option_params& op = d.options[m].data[j];
            const double dw = op.delta_est * op.w;
            (op.type > 0 ? call_dw : put_dw)[op.stock_ind] += dw;
        }
    double wsum = 0;
    for (int m = 0; m < 3; m++)
        for (size_t j = 0; j < d.options[m].size; j++) {
            option_params& op = d.options[m].data[j];
            if (op.type > 0) op.w *= -put_dw[op.stock_ind] / call_dw[op.stock_ind];
            wsum += op.w;
        }
    for (int m = 0; m < 3; m++) {
        option_params* b = d.options[m].data;
        for (size_t j = 0; j < d.options[m].size; j++) {
            b[j].w /= wsum;
            b[j].prob = uniform_prob ? 1.f : std::abs(b[j].w) / std::sqrt(b[j].W_est);
        }
        std::sort(b, b + d.options[m].size,
                  [](const option_params& x, const option_params& y) { return x.prob > y.prob; });
    }
    ops_owner.release();                     // now owned by d (portfolio_free_data)
    stocks_owner.release();
    nmlmc_ref_status(NMLMC_OK, "portfolio_gen_data");
    return d;
}

// No exception may cross the C ABI: a failed host allocation returns the zeroed portfolio_data.
extern "C" portfolio_data portfolio_gen_data(uint32_t P, uint32_t Q, uint64_t seed, double* probs,
                                             bool uniform_weights, bool uniform_prob) {
    try {
        return gen_data(P, Q, seed, probs, uniform_weights, uniform_prob);
    } catch (const std::bad_alloc&) {
        nmlmc_ref_status(NMLMC_ERR_NOMEM, "portfolio_gen_data");
    } catch (const std::length_error&) {
        nmlmc_ref_status(NMLMC_ERR_ARG, "portfolio_gen_data");
    }
    return portfolio_data{};
}

// Frees what portfolio_gen_data allocated (portfolio_sampler.cpp:906-912): the stock array and
// the option array, which starts at options[0].
extern "C" void portfolio_free_data(portfolio_data* d) {
    if (!d) {
        nmlmc_ref_status(NMLMC_ERR_ARG, "portfolio_free_data");
        return;
    }
    delete[] d->stocks.data;
    delete[] d->options[0].data;
    d->stocks.data = nullptr;
    d->stocks.size = 0;
    for (int m = 0; m < 3; m++) {
        d->options[m].data = nullptr;
        d->options[m].size = 0;
    }
    nmlmc_ref_status(NMLMC_OK, "portfolio_free_data");
}
