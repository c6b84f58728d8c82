// Seeded synthetic option portfolios (host, C++).
//
// The benchmark portfolios are specified by distributions (stocks: sigma ~ U[lo, hi]; options:
// uniformly chosen stock, call with a given probability, strike ~ U[lo, hi] * S0, maturity ~
// U[lo, hi], position ~ N(0, 1)).  Every random field is drawn from a counter-based Threefry2x64-20
// stream — value(field f, index i) = Threefry(ctr = (i, f), key = (seed, 'PORTGEN')) — so a
// portfolio is a pure function of (spec, seed), independent of platform, thread count and
// generation order.  The reference's own generator (portfolio_gen_data, portfolio_sampler.cpp:
// 784-904, mt19937 with a delta hedge and renormalised weights) builds a different, smaller
// portfolio for its demo main and is not reproduced.
#include <cmath>
#include <cstdint>

#include "../../include/nmlmc.h"

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
