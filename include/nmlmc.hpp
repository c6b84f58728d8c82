/* nmlmc.hpp — the reference's C++ entry points, over the C ABI of nmlmc.h (header-only, C++11 or
 * later; the reference builds with C++14).
 *
 *  sample<SAMPLER>(ell, override_dyn_inner, &M, fsums, diffsums, &total_work, inner_stats)
 *      The level call of nested_sampler.hpp:646-694 for SAMPLER = model::sampler or
 *      portfolio::sampler, on the process-wide sampler that init_nestedmc_sampler and
 *      model_init / portfolio_init set up.  Fine sums only when ell == 0 or diffsums is NULL.
 *      The caller's arrays hold the fine / diff moments given to init_nestedmc_sampler.  Errors
 *      are recorded in nmlmc_last_error() and printed (the reference exit()s).  A SAMPLER type
 *      selects one of the library's kernels; the samplers' device code lives in the library.
 *
 *  model:: / portfolio:: names of the reference (model::data with its constructor, PhiType,
 *      ComputeMethod, OptionType, Subsampling, the entry points as model::model_init, ...) and
 *      nmlmc::make_nested_sampler_params / nmlmc::level_output for the two C structs whose
 *      reference constructors a C header cannot carry (nested_sampler_params, sample_output).
 *
 *  nmlmc::mlmc_t<T, S>::run(mlmc_input_t&)
 *      The continuation-MLMC driver of mlmc.hpp:207-337 with its std::function level callback
 *      (mlmc_input_t::fn_sample_level_t, mlmc.hpp:224).  The loop is the library's C++ driver
 *      (nmlmc_mlmc_run_cb), which keeps the level sums in FP64: T must be double and S = 4
 *      moments.  `nmlmc::mlmc_real` is mlmc_t<double, 4>.  The default bias estimate of the
 *      reference (default_bias_estimate, mlmc.hpp:207-214) is built in; mlmc_input_t has no
 *      est_bias hook.  A failing run throws: the callback's own exception if it threw, else
 *      std::runtime_error with the library's status text.
 */
#ifndef NMLMC_HPP
#define NMLMC_HPP

#include <cmath>
#include <cstdint>
#include <cstring>
#include <exception>
#include <functional>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "nmlmc.h"

namespace model {
enum class PhiType { Indicator = 0, Max = 1 };     /* model_sampler.cpp:16-19 (Indicator only here) */

/* model::data (model_sampler.cpp:21-39): the same fields and layout as model_data. */
struct data : ::model_data {
    data() : ::model_data() {}
    data(PhiType phi, float tau, float loss) : ::model_data() {
        stau = std::sqrt(tau);
        s1tau = std::sqrt(1 - tau);
        max_loss = loss;
        phi_type = static_cast<int32_t>(phi);
    }
    uint32_t phi_size() const { return 1; }
};
using ::model_update_data;
using ::model_init;
using ::model_sample;

struct sampler {               /* model::sampler (model_sampler.cpp:42-92) */
    static void sample_level(uint32_t ell, uint64_t, sample_output* out) {
        model_sample(ell, out->M, out);
    }
};
}  // namespace model

namespace portfolio {
enum class ComputeMethod { BS = 0, Exact = 1, Unbiased = 2 };        /* portfolio_sampler.cpp:17-22 */
enum class OptionType { Call = 1, Put = -1 };                       /* :24-27 */
enum class Subsampling { None = 0, Random = 1, Random_Uniform = -1 };  /* :36-40 */
typedef ::portfolio_data data;
typedef ::option_params option_params;
typedef ::stock_params stock_params;
using ::portfolio_update_data;
using ::portfolio_init;
using ::portfolio_sample;
using ::portfolio_cleanup;
using ::portfolio_comp_params;
using ::portfolio_gen_data;
using ::portfolio_free_data;

struct sampler {               /* portfolio::sampler (portfolio_sampler.cpp:227-606) */
    static void sample_level(uint32_t ell, uint64_t override_dyn_inner, sample_output* out) {
        portfolio_sample(ell, override_dyn_inner, out->M, out);
    }
};
}  // namespace portfolio

namespace nmlmc {
/* nested_sampler_params(fine_moments, diff_moments, N0, beta, adaptive_r, antithetic), the
 * reference's constructor argument order (nested_sampler.hpp:16-26). */
inline nested_sampler_params make_nested_sampler_params(uint32_t fine_moments, uint32_t diff_moments,
                                                        uint32_t N0, uint32_t beta, float adaptive_r,
                                                        bool antithetic) {
    nested_sampler_params p;
    p.N0 = N0;
    p.beta = beta;
    p.antithetic = antithetic;
    p.fine_moments = fine_moments;
    p.diff_moments = diff_moments;
    p.adaptive_r = adaptive_r;
    return p;
}

/* A sample_output that owns its sums, as the reference's sample_output(fsize, dsize, phi_size)
 * does (common.hpp:37-55); converts to the sample_output* the C entry points take. */
class level_output {
  public:
    explicit level_output(uint32_t fsize, uint32_t dsize = 0, uint32_t phi_size = 1)
        : f_(static_cast<size_t>(fsize) * phi_size, 0.0), d_(static_cast<size_t>(dsize) * phi_size, 0.0) {
        std::memset(&o_, 0, sizeof o_);
        o_.fsums = f_.empty() ? nullptr : f_.data();
        o_.diffsums = d_.empty() ? nullptr : d_.data();
    }
    level_output(const level_output&) = delete;
    level_output& operator=(const level_output&) = delete;
    operator sample_output*() { return &o_; }
    sample_output* operator->() { return &o_; }
    const sample_output* operator->() const { return &o_; }

  private:
    std::vector<double> f_, d_;
    sample_output o_;
};
}  // namespace nmlmc

template <class SAMPLER>
inline void sample(uint32_t ell, uint64_t override_dyn_inner, uint64_t* M, double* out_fsums,
                   double* out_diffsums, double* out_total_work, uint64_t* out_inner_stats) {
    sample_output o;
    std::memset(&o, 0, sizeof o);
    o.M = M ? *M : 0;
    o.fsums = out_fsums;
    o.diffsums = out_diffsums;              /* zeros at level 0, as the reference copies back */
    SAMPLER::sample_level(ell, override_dyn_inner, &o);
    if (nmlmc_last_error() != NMLMC_OK) return;
    if (M) *M = o.M;
    if (out_total_work) *out_total_work = o.total_work;
    if (out_inner_stats) std::memcpy(out_inner_stats, o.inner_stats, sizeof o.inner_stats);
}

namespace nmlmc {

template <class T = double, int S = 4>
struct mlmc_t {
    static_assert(std::is_same<T, double>::value && S == 4,
                  "the library's driver keeps 4 moments of FP64 level sums");
    static const uint32_t moments = S;

    /* mc_diff_output_t (mlmc.hpp:21-85): one level's sums */
    struct mc_diff_output_t {
        T sums_fine[S]{};
        T sums_diff[S]{};
        double work{0};
        double time{0};
        uint64_t M{0};
        T dEl() const { return sums_diff[0] * (1. / M); }
        T fEl() const { return sums_fine[0] * (1. / M); }
        double Wl() const { return work / M; }
        T dVl() const { return sums_diff[1] * (1. / M) - dEl() * dEl(); }
        T fVl() const { return sums_fine[1] * (1. / M) - fEl() * fEl(); }
    };

    /* mlmc_output_t (mlmc.hpp:87-205): the levels and the run's estimates */
    struct mlmc_output_t {
        std::vector<mc_diff_output_t> levels;
        uint32_t starting_level{0};
        double bias_est{0}, stat_error{0}, TOL{0};
        double Eg{0};                       /* the MLMC estimate                          */
        double total_work{0}, total_time{0};
        uint64_t calls{0};                  /* sample_level invocations                   */
        std::string table;                  /* to_string(): the reference's table text    */
        uint32_t L() const { return (uint32_t)levels.size() - starting_level - 1; }
        std::string to_string() const { return table; }
    };

    /* mlmc_input_t (mlmc.hpp:216-238) */
    struct mlmc_input_t {
        typedef std::function<mc_diff_output_t(uint32_t ell, uint64_t M)> fn_sample_level_t;
        fn_sample_level_t sample_level;
        double targetTOL{1e-3};
        double startTOL{0.5};
        double theta{0.5};
        double starting_level_coeff{1.5};
        double Ca{3};
        bool verbose{true};
        uint64_t M0{100};
    };

    static mlmc_output_t run(mlmc_input_t& in) {
        if (!in.sample_level) throw std::invalid_argument("mlmc_input_t::sample_level is empty");
        nmlmc_mlmc_input c = nmlmc_mlmc_default_input();
        c.targetTOL = in.targetTOL;
        c.startTOL = in.startTOL;
        c.theta = in.theta;
        c.starting_level_coeff = in.starting_level_coeff;
        c.Ca = in.Ca;
        c.M0 = in.M0;
        c.verbose = in.verbose ? 1 : 0;
        struct Call {
            mlmc_input_t* in;
            std::exception_ptr error;
        } call{&in, nullptr};
        nmlmc_sample_level_fn level = [](void* user, uint32_t ell, uint64_t M, nmlmc_level_result* out) {
            Call* k = static_cast<Call*>(user);
            std::memset(out, 0, sizeof *out);
            if (k->error) return;
            try {
                const mc_diff_output_t r = k->in->sample_level(ell, M);
                for (int j = 0; j < S; j++) {
                    out->fsums[j] = r.sums_fine[j];
                    out->diffsums[j] = r.sums_diff[j];
                }
                out->total_work = r.work;
                out->seconds = r.time;
                out->M = r.M;
            } catch (...) {                 /* M stays 0: the driver stops */
                k->error = std::current_exception();
            }
        };
        nmlmc_mlmc_output o;
        std::vector<char> table(1 << 16, '\0');
        const int rc = nmlmc_mlmc_run_cb(&c, level, nullptr, &call, &o, table.data(), table.size());
        if (call.error) std::rethrow_exception(call.error);
        if (rc != NMLMC_OK) throw std::runtime_error(std::string("nmlmc_mlmc_run_cb: ") + nmlmc_error_string(rc));
        mlmc_output_t out;
        out.levels.resize(o.nlevels);
        for (uint32_t l = 0; l < o.nlevels; l++) {
            mc_diff_output_t& v = out.levels[l];
            for (int j = 0; j < S; j++) {
                v.sums_fine[j] = o.level_fsums[l][j];
                v.sums_diff[j] = o.level_diffsums[l][j];
            }
            v.work = o.level_work[l];
            v.time = o.level_time[l];
            v.M = o.level_M[l];
        }
        out.starting_level = o.starting_level;
        out.bias_est = o.bias_est;
        out.stat_error = o.stat_error;
        out.TOL = o.TOL;
        out.Eg = o.Eg;
        out.total_work = o.total_work;
        out.total_time = o.total_time;
        out.calls = o.calls;
        out.table = table.data();
        return out;
    }
};

typedef mlmc_t<double, 4> mlmc_real;

}  // namespace nmlmc

#endif /* NMLMC_HPP */
