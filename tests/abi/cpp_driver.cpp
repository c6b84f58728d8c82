// The C++ entry points of include/nmlmc.hpp, used as the reference's C++ callers use mlmc.hpp and
// sample<SAMPLER> (compiled and run by tests/test_abi.py; no device needed):
//  1. nmlmc::mlmc_real::run over a std::function level sampler takes exactly the decisions and
//     prints exactly the table of the C driver (nmlmc_mlmc_run_cb) over the same sampler;
//  2. an exception thrown by the level sampler leaves run() as that exception;
//  3. sample<model::sampler> before model_init records an error instead of exiting;
//  4. the reference's model:: / portfolio:: names and constructors compile and behave.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>

#include "nmlmc.hpp"

namespace {

// Synthetic level sampler: level ell has fine mean 0.3 + 2^-ell, difference mean 2^-ell and
// difference variance 2^-2ell; samples are normals from a splitmix64 stream per (ell, call).
struct Synthetic {
    uint64_t calls = 0;
    int throw_at = -1;
    static uint64_t mix(uint64_t& s) {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    static double normal(uint64_t& s) {
        const double u1 = std::ldexp((mix(s) >> 11) + 0.5, -53), u2 = std::ldexp((mix(s) >> 11) + 0.5, -53);
        return std::sqrt(-2 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
    void level(uint32_t ell, uint64_t M, double* f, double* d, double& work) {
        if ((int)calls == throw_at) throw std::domain_error("synthetic sampler failure");
        uint64_t s = (uint64_t)ell << 40 | calls++;
        const double h = std::ldexp(1.0, -(int)ell);
        for (int j = 0; j < 4; j++) f[j] = d[j] = 0;
        for (uint64_t m = 0; m < M; m++) {
            const double z = normal(s), y = 0.3 + h + 0.5 * z;
            const double x = ell == 0 ? 0 : h + h * normal(s);
            double pf = 1, pd = 1;
            for (int j = 0; j < 4; j++) {
                pf *= y;
                pd *= x;
                f[j] += pf;
                d[j] += pd;
            }
        }
        work = (double)M * std::ldexp(1.0, (int)ell);
    }
};

void c_level(void* user, uint32_t ell, uint64_t M, nmlmc_level_result* out) {
    std::memset(out, 0, sizeof *out);
    static_cast<Synthetic*>(user)->level(ell, M, out->fsums, out->diffsums, out->total_work);
    out->M = M;
}

}  // namespace

int main() {
    int bad = 0;
    const double tol = 2e-3;
    // 1. the C++ driver interface against the C one
    Synthetic a, b;
    nmlmc::mlmc_real::mlmc_input_t in;
    in.targetTOL = tol;
    in.M0 = 200;
    in.verbose = false;
    in.sample_level = [&a](uint32_t ell, uint64_t M) {
        nmlmc::mlmc_real::mc_diff_output_t o;
        a.level(ell, M, o.sums_fine, o.sums_diff, o.work);
        o.M = M;
        return o;
    };
    const nmlmc::mlmc_real::mlmc_output_t r = nmlmc::mlmc_real::run(in);
    nmlmc_mlmc_input ci = nmlmc_mlmc_default_input();
    ci.targetTOL = tol;
    ci.M0 = 200;
    ci.verbose = 0;
    nmlmc_mlmc_output co;
    static char table[1 << 16];
    if (nmlmc_mlmc_run_cb(&ci, c_level, nullptr, &b, &co, table, sizeof table) != NMLMC_OK) bad++;
    if (r.levels.size() != co.nlevels || r.calls != co.calls || r.Eg != co.Eg) bad++;
    for (size_t l = 0; l < r.levels.size() && l < co.nlevels; l++)
        if (r.levels[l].M != co.level_M[l] || r.levels[l].sums_fine[1] != co.level_fsums[l][1]) bad++;
    if (r.to_string() != table || r.to_string().empty()) bad++;
    printf("levels %zu calls %llu Eg %.6f stat_error %.3g bias %.3g\n", r.levels.size(),
           (unsigned long long)r.calls, r.Eg, r.stat_error, r.bias_est);
    // 2. the sampler's exception comes out of run()
    Synthetic c;
    c.throw_at = 3;
    in.sample_level = [&c](uint32_t ell, uint64_t M) {
        nmlmc::mlmc_real::mc_diff_output_t o;
        c.level(ell, M, o.sums_fine, o.sums_diff, o.work);
        o.M = M;
        return o;
    };
    bool thrown = false;
    try {
        nmlmc::mlmc_real::run(in);
    } catch (const std::domain_error&) {
        thrown = true;
    }
    if (!thrown) bad++;
    // 3. sample<SAMPLER> before init: an error status, not an exit
    uint64_t M = 10, stats[6] = {0};
    double f[4], d[4], w = 0;
    sample<model::sampler>(2, 0, &M, f, d, &w, stats);
    if (nmlmc_last_error() == NMLMC_OK) bad++;
    sample<portfolio::sampler>(2, 0, &M, f, d, &w, stats);
    if (nmlmc_last_error() == NMLMC_OK) bad++;
    // 4. the reference's names: model::data and its constructor, model::model_sample on an owning
    //    sample_output, the params constructor's argument order, portfolio::portfolio_gen_data
    static_assert(sizeof(model::data) == sizeof(model_data), "model::data keeps model_data's layout");
    const model::data md(model::PhiType::Indicator, 0.02f, 0.1f);
    if (md.stau != std::sqrt(0.02f) || md.s1tau != std::sqrt(1 - 0.02f) || md.max_loss != 0.1f ||
        md.phi_type != 0 || md.phi_size() != 1)
        bad++;
    nmlmc::level_output out(4, 4, 1);
    model::model_sample(2, 10, out);                       // before model_init: an error status
    if (nmlmc_last_error() == NMLMC_OK || out->fsums == nullptr || out->diffsums == nullptr) bad++;
    const nested_sampler_params p = nmlmc::make_nested_sampler_params(4, 2, 32, 4, 1.5f, true);
    if (p.fine_moments != 4 || p.diff_moments != 2 || p.N0 != 32 || p.beta != 4 || !p.antithetic ||
        p.adaptive_r != 1.5f)
        bad++;
    double probs[3] = {0.5, 0.25, 0.25};
    portfolio::data pd = portfolio::portfolio_gen_data(40, 4, 9, probs, false, false);
    const int32_t t0 = pd.options[0].size ? pd.options[0].data[0].type : 0;
    if (nmlmc_last_error() != NMLMC_OK || pd.options[0].size != 20 || pd.options[1].size != 10 ||
        pd.stocks.size != 4 ||
        (t0 != static_cast<int32_t>(portfolio::OptionType::Call) &&
         t0 != static_cast<int32_t>(portfolio::OptionType::Put)))
        bad++;
    portfolio::portfolio_free_data(&pd);
    printf("ok-checks %d\n", bad);
    return bad != 0;
}
