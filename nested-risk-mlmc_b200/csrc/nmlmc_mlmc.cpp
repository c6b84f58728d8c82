// Host continuation-MLMC driver over the level sampler (C++).
//
// The same algorithm and decisions as the reference's mlmc_t<real, 4>::run (mlmc.hpp:290-337):
// a TOL sequence from startTOL halving in sqrt(2) steps down to targetTOL, the adaptive
// starting level (better_starting_level, 241-262), the optimal per-level sample counts
// (get_optimal_Ml, 265-288), the statistical-error / bias split with theta and Ca, and a new
// level whenever the bias estimate (default_bias_estimate, 207-214) is too large.  The level
// estimators (mc_diff_output_t, 21-85) and the final report (mlmc_output_t::to_string with
// table_t, 106-183 and table_output.hpp) keep the reference's arithmetic and text layout, so
// runs can be compared and parsed the same way.
//
// With `batched`, the missing samples of all levels in one round are requested in a single
// submission (nmlmc_sample_levels) instead of one synchronous call per level; on the OUTER
// stream layout the results are identical because every outer sample owns its stream.
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <functional>
#include <iomanip>
#include <iostream>
#include <limits>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/nmlmc.h"

namespace {

inline double sq(double x) { return x * x; }

// mc_diff_output_t<double, 4> (mlmc.hpp:21-85)
struct Level {
    double f[4] = {0, 0, 0, 0}, d[4] = {0, 0, 0, 0};
    double work = 0, time = 0;
    uint64_t M = 0;
    double dEl() const { return d[0] * (1. / M); }
    double fEl() const { return f[0] * (1. / M); }
    double Wl() const { return work / M; }
    double dVl() const { return d[1] * (1. / M) - sq(dEl()); }
    double fVl() const { return f[1] * (1. / M) - sq(fEl()); }
    // fourth central moment as the reference forms it: the cross terms use the fine sums for
    // both the fine and the difference estimator (mlmc.hpp:78-84)
    double mu4(const double* s) const {
        double t = s[3] * (1. / M);
        t += (s[0] * (1. / M)) * (f[2] * (1. / M)) * (-4.);
        t += sq(s[0] * (1. / M)) * (f[1] * (1. / M)) * (6);
        t += sq(sq(s[0] * (1. / M))) * (-3.);
        return t;
    }
    double dKl() const { return mu4(d) / sq(dVl()); }
    double fKl() const { return mu4(f) / sq(fVl()); }
    Level& operator+=(const Level& o) {
        for (int s = 0; s < 4; s++) { f[s] += o.f[s]; d[s] += o.d[s]; }
        work += o.work;
        time += o.time;
        M += o.M;
        return *this;
    }
};

struct Output {
    std::vector<Level> levels;
    uint32_t starting_level = 0;
    double bias_est = std::nan(""), stat_error = std::nan(""), TOL = std::nan("");
    double total_variance() const {
        uint32_t l = starting_level;
        double t = levels[l].fVl() / levels[l].M;
        for (l = starting_level + 1; l < levels.size(); l++) t += levels[l].dVl() / levels[l].M;
        return t;
    }
};

// ---- text table in the layout of the reference's table_t (table_output.hpp:38-112) ----------
struct Column {
    std::string header;
    size_t min_len;
    std::function<void(std::stringstream&, uint32_t)> value;   // row i
};

void centered(std::ostream& s, const std::string& str) {
    std::streamsize w = s.width();
    if (w > (std::streamsize)str.size()) {
        std::streamsize left = (w + (std::streamsize)str.size()) / 2;
        s.width(left);
        s << str;
        s.width(w - left);
        s << "";
    } else {
        s << str;
    }
}

void render_table(std::stringstream& s, uint32_t nrows, std::vector<Column>& cols) {
    const uint32_t rows = nrows + 1;
    auto cell = [&](Column& c, std::stringstream& o, uint32_t i) {
        if (i == 0) centered(o, c.header);
        else c.value(o, i - 1);
    };
    for (auto& c : cols) {
        for (uint32_t i = 0; i < rows; i++) {
            std::stringstream tmp;
            tmp.copyfmt(s);
            tmp << std::setw(0);
            cell(c, tmp, i);
            c.min_len = std::max(tmp.str().size(), c.min_len);
        }
    }
    for (uint32_t i = 0; i < rows; i++) {
        const bool line = (i == 0 || i == rows - 1);
        s << "| ";
        for (auto& c : cols) {
            s << std::setw((int)c.min_len);
            cell(c, s, i);
            s << " | ";
        }
        s << std::endl;
        if (line) {
            s << "+" << std::setfill('-');
            for (auto& c : cols) s << std::setw((int)(3 + c.min_len)) << "+";
            s << std::setfill(' ') << std::endl;
        }
    }
}

std::string to_string(const Output& out) {
    using namespace std;
    stringstream str;
    double dwork = 0, dtime = 0;
    for (uint32_t l = 0; l < out.starting_level; l++) { dwork += out.levels[l].work; dtime += out.levels[l].time; }
    double ttime = dtime, twork = dwork;
    for (uint32_t l = out.starting_level; l < out.levels.size(); l++) { twork += out.levels[l].work; ttime += out.levels[l].time; }
    double Eg = out.levels[out.starting_level].fEl();
    for (uint32_t l = out.starting_level + 1; l < out.levels.size(); l++) Eg += out.levels[l].dEl();
    str << "TOL: " << out.TOL << std::endl;
    str << "RMS: " << std::sqrt(sq(out.bias_est) + sq(out.stat_error)) << " (" << out.bias_est << ", "
        << out.stat_error << ") " << std::endl;
    str << "Eg: " << Eg << " --- [" << Eg - out.TOL << "," << Eg + out.TOL << "]" << std::endl;
    str << "Discarded Work: " << dwork << std::endl;
    str << "Discarded Time: " << dtime << std::endl;
    str << "Total Work: " << twork << std::endl;
    str << "Total Time: " << ttime << std::endl;
    str << std::scientific << setprecision(4);
    const std::vector<Level>& L = out.levels;
    const uint32_t sl = out.starting_level;
    std::vector<Column> cols;
    cols.push_back({"ell", 3, [&](stringstream& o, uint32_t i) {
                        if (i < sl) o << "*" + std::to_string(i); else o << i; }});
    cols.push_back({"dEl", 10, [&](stringstream& o, uint32_t i) { o << L[i].dEl(); }});
    cols.push_back({"fEl", 10, [&](stringstream& o, uint32_t i) { o << L[i].fEl(); }});
    cols.push_back({"dVl", 10, [&](stringstream& o, uint32_t i) { o << L[i].dVl(); }});
    cols.push_back({"fVl", 10, [&](stringstream& o, uint32_t i) { o << L[i].fVl(); }});
    cols.push_back({"dKl", 10, [&](stringstream& o, uint32_t i) { o << L[i].dKl(); }});
    cols.push_back({"fKl", 10, [&](stringstream& o, uint32_t i) { o << L[i].fKl(); }});
    cols.push_back({"Wl", 10, [&](stringstream& o, uint32_t i) { o << L[i].Wl(); }});
    cols.push_back({"M", 5, [&](stringstream& o, uint32_t i) { o << L[i].M; }});
    cols.push_back({"Time", 10, [&](stringstream& o, uint32_t i) { o << L[i].time / L[i].M; }});
    render_table(str, (uint32_t)L.size(), cols);
    return str.str();
}

double default_bias_estimate(const Output& out, double rate = 0.5) {   // mlmc.hpp:207-214
    if (out.levels.size() > 2) {
        double b0 = std::abs(out.levels[out.levels.size() - 1].dEl());
        double b1 = std::abs(out.levels[out.levels.size() - 2].dEl()) * rate;
        return b0 > b1 ? b0 : b1;
    }
    return std::numeric_limits<double>::infinity();
}

uint32_t better_starting_level(const Output& out, double coeff) {      // mlmc.hpp:241-262
    uint32_t l0 = out.starting_level;
    while (true) {
        bool change = false;
        double lhs = std::sqrt(out.levels[l0].fVl() * out.levels[l0].Wl());
        for (uint32_t lp = l0 + 1; lp < out.levels.size(); lp++) {
            lhs += std::sqrt(out.levels[lp].dVl() * out.levels[lp].Wl());
            double rhs = std::sqrt(out.levels[lp].fVl() * out.levels[lp].Wl());
            if (lhs / rhs > coeff) { change = true; break; }
        }
        if (!change) break;
        l0 += 1;
    }
    return l0;
}

void optimal_Ml(double tol2, uint64_t M0, const Output& out, std::vector<uint64_t>& Ml) {  // 265-288
    uint32_t l = out.starting_level;
    Ml.resize(out.levels.size());
    std::fill(Ml.begin(), Ml.begin() + l, 0);
    double lambda = out.levels[l].M == 0 ? 0 : std::sqrt(out.levels[l].Wl() * out.levels[l].fVl());
    for (l = out.starting_level + 1; l < out.levels.size(); l++)
        lambda += out.levels[l].M == 0 ? 0 : std::sqrt(out.levels[l].Wl() * out.levels[l].dVl());
    lambda /= tol2;
    l = out.starting_level;
    Ml[l] = (out.levels[l].M == 0) ? M0
                                   : static_cast<uint64_t>(std::ceil(lambda * std::sqrt(out.levels[l].fVl() / out.levels[l].Wl())));
    for (l = out.starting_level + 1; l < out.levels.size(); l++)
        Ml[l] = (out.levels[l].M == 0) ? M0
                                       : static_cast<uint64_t>(std::ceil(lambda * std::sqrt(out.levels[l].dVl() / out.levels[l].Wl())));
}

Level from_result(const nmlmc_level_result& r) {
    Level o;
    for (int j = 0; j < 4; j++) { o.f[j] = r.fsums[j]; o.d[j] = r.diffsums[j]; }
    o.work = r.total_work;
    o.time = r.seconds;
    o.M = r.M;
    return o;
}

int run(const nmlmc_mlmc_input& in, nmlmc_sample_level_fn level_fn, nmlmc_sample_levels_fn levels_fn,
        void* user, nmlmc_mlmc_output* res, char* table, size_t table_cap) {
    const auto t0 = std::chrono::steady_clock::now();
    Output out;
    const double sqrt_2_inv = 1. / std::sqrt(2);
    uint32_t total_itrs = static_cast<uint32_t>(-(std::log2(in.targetTOL) - std::log2(in.startTOL)));
    out.TOL = in.targetTOL * (1 << total_itrs);
    total_itrs *= 2;
    out.levels.resize(1);
    std::vector<uint64_t> Ml(out.levels.size());
    uint64_t calls = 0;
    for (uint32_t itr = 0; itr <= total_itrs; itr++) {
        out.starting_level = better_starting_level(out, in.starting_level_coeff);
        while (true) {
            optimal_Ml(in.theta * sq(out.TOL) / in.Ca, in.M0, out, Ml);
            std::vector<uint32_t> ells;
            std::vector<uint64_t> Ms;
            for (uint32_t l = 0; l < out.levels.size(); l++) {
                if (out.levels[l].M < Ml[l]) {
                    ells.push_back(l);
                    Ms.push_back(Ml[l] - out.levels[l].M);
                }
            }
            if (in.batched && levels_fn && !ells.empty()) {
                if (in.verbose)
                    for (size_t i = 0; i < ells.size(); i++)
                        std::cout << "# Sampling " << Ms[i] << " of " << ells[i] << std::endl;
                std::vector<nmlmc_level_result> rs(ells.size());
                levels_fn(user, (uint32_t)ells.size(), ells.data(), Ms.data(), rs.data());
                calls += ells.size();
                for (size_t i = 0; i < ells.size(); i++) {
                    if (rs[i].M != Ms[i]) return NMLMC_ERR_STATE;
                    out.levels[ells[i]] += from_result(rs[i]);
                }
            } else {
                for (uint32_t l = 0; l < out.levels.size(); l++) {
                    while (out.levels[l].M < Ml[l]) {
                        uint64_t M = Ml[l] - out.levels[l].M;
                        if (in.verbose) std::cout << "# Sampling " << M << " of " << l << std::endl;
                        nmlmc_level_result r;
                        memset(&r, 0, sizeof r);
                        level_fn(user, l, M, &r);
                        calls++;
                        if (r.M == 0) return NMLMC_ERR_STATE;   // the sampler failed
                        out.levels[l] += from_result(r);
                    }
                }
            }
            out.stat_error = std::sqrt(in.Ca * out.total_variance());
            if (sq(out.stat_error) >= in.theta * sq(out.TOL)) continue;
            out.bias_est = default_bias_estimate(out);
            if (sq(out.bias_est) >= (1 - in.theta) * sq(out.TOL)) {
                if (in.max_levels && out.levels.size() >= in.max_levels) return NMLMC_ERR_ARG;
                out.levels.resize(out.levels.size() + 1);
                continue;
            }
            if (in.verbose) std::cout << to_string(out);
            break;
        }
        out.TOL *= sqrt_2_inv;
    }
    const double total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (in.verbose) std::cout << "# Total time taken: " << total << " seconds." << std::endl;
    if (res) {
        memset(res, 0, sizeof(*res));
        res->nlevels = (uint32_t)out.levels.size();
        res->starting_level = out.starting_level;
        res->bias_est = out.bias_est;
        res->stat_error = out.stat_error;
        res->TOL = out.TOL;
        double Eg = out.levels[out.starting_level].fEl();
        for (uint32_t l = out.starting_level + 1; l < out.levels.size(); l++) Eg += out.levels[l].dEl();
        res->Eg = Eg;
        res->total_time = total;
        res->calls = calls;
        for (uint32_t l = 0; l < out.levels.size() && l < NMLMC_MAX_LEVELS; l++) {
            res->level_M[l] = out.levels[l].M;
            for (int j = 0; j < 4; j++) { res->level_fsums[l][j] = out.levels[l].f[j]; res->level_diffsums[l][j] = out.levels[l].d[j]; }
            res->level_work[l] = out.levels[l].work;
            res->level_time[l] = out.levels[l].time;
            res->total_work += out.levels[l].work;
        }
    }
    if (table && table_cap) {
        std::string s = to_string(out);
        size_t n = s.size() < table_cap - 1 ? s.size() : table_cap - 1;
        memcpy(table, s.data(), n);
        table[n] = 0;
    }
    return NMLMC_OK;
}

// GPU sampler callbacks
struct GpuUser {
    nmlmc_ctx* ctx;
    int status;
};
void gpu_level(void* u, uint32_t ell, uint64_t M, nmlmc_level_result* out) {
    GpuUser* g = static_cast<GpuUser*>(u);
    int rc = nmlmc_sample(g->ctx, ell, M, out);
    if (rc) { g->status = rc; out->M = 0; }
}
void gpu_levels(void* u, uint32_t n, const uint32_t* ells, const uint64_t* Ms, nmlmc_level_result* outs) {
    GpuUser* g = static_cast<GpuUser*>(u);
    int rc = nmlmc_sample_levels(g->ctx, n, ells, Ms, outs);
    if (rc) { g->status = rc; for (uint32_t i = 0; i < n; i++) outs[i].M = 0; }
}

}  // namespace

extern "C" {

nmlmc_mlmc_input nmlmc_mlmc_default_input(void) {
    nmlmc_mlmc_input in;
    in.targetTOL = 1e-3;                 // mlmc_input_t defaults (mlmc.hpp:230-238)
    in.startTOL = 0.5;
    in.theta = 0.5;
    in.starting_level_coeff = 1.5;
    in.Ca = 3;
    in.M0 = 100;
    in.verbose = 1;
    in.max_levels = 0;
    in.batched = 0;
    return in;
}

int nmlmc_mlmc_run_cb(const nmlmc_mlmc_input* in, nmlmc_sample_level_fn level_fn,
                      nmlmc_sample_levels_fn levels_fn, void* user, nmlmc_mlmc_output* out,
                      char* table, size_t table_cap) {
    if (!in || !level_fn || !(in->targetTOL > 0) || !(in->startTOL >= in->targetTOL)) return NMLMC_ERR_ARG;
    return run(*in, level_fn, levels_fn, user, out, table, table_cap);
}

int nmlmc_mlmc_run(nmlmc_ctx* ctx, const nmlmc_mlmc_input* in, nmlmc_mlmc_output* out, char* table,
                   size_t table_cap) {
    if (!ctx || !in) return NMLMC_ERR_ARG;
    GpuUser u{ctx, NMLMC_OK};
    int rc = nmlmc_mlmc_run_cb(in, gpu_level, gpu_levels, &u, out, table, table_cap);
    return u.status ? u.status : rc;
}

}  // extern "C"
