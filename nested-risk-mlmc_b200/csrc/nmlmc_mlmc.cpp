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
//
// Checkpoints (no counterpart in the reference): after every completed TOL iteration the state
// of the loop — the level sums in FP64, the iteration, TOL and starting level — and the
// sampler's stream state are written to a file; a run resumed from it with the same parameters
// continues at that iteration and ends exactly as the uninterrupted run.
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <functional>
#include <iomanip>
#include <iostream>
#include <limits>
#include <new>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/nmlmc.h"

namespace {

inline double sq(double x) { return x * x; }

// Profiler range (NVTX v3, header-only; inert unless a tool such as nsys attaches).
struct NvtxScope {
    explicit NvtxScope(const char* name) { nvtxRangePushA(name); }
    ~NvtxScope() { nvtxRangePop(); }
    NvtxScope(const NvtxScope&) = delete;
    NvtxScope& operator=(const NvtxScope&) = delete;
};

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

// A level's sample count from the optimal-allocation formula.  A variance that rounds below zero
// makes the formula NaN (the reference then converts NaN to an integer, which C++ leaves
// undefined): it counts as no further samples.  A count at or beyond 2^62 cannot be a run that
// ends and is reported as kCountOverflow.
constexpr uint64_t kCountOverflow = ~0ull;
uint64_t to_count(double x) {
    if (!(x > 0)) return 0;
    const double c = std::ceil(x);
    return c >= 0x1p62 ? kCountOverflow : static_cast<uint64_t>(c);
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
    Ml[l] = (out.levels[l].M == 0) ? M0 : to_count(lambda * std::sqrt(out.levels[l].fVl() / out.levels[l].Wl()));
    for (l = out.starting_level + 1; l < out.levels.size(); l++)
        Ml[l] = (out.levels[l].M == 0) ? M0 : to_count(lambda * std::sqrt(out.levels[l].dVl() / out.levels[l].Wl()));
}

// A sampler's level result the driver can use: finite sums and a finite, non-negative work.
bool usable(const nmlmc_level_result& r) {
    bool ok = std::isfinite(r.total_work) && r.total_work >= 0;
    for (int j = 0; j < 4; j++) ok = ok && std::isfinite(r.fsums[j]) && std::isfinite(r.diffsums[j]);
    return ok;
}

Level from_result(const nmlmc_level_result& r) {
    Level o;
    for (int j = 0; j < 4; j++) { o.f[j] = r.fsums[j]; o.d[j] = r.diffsums[j]; }
    o.work = r.total_work;
    o.time = r.seconds;
    o.M = r.M;
    return o;
}

// ---- checkpoints ---------------------------------------------------------------------------
// Little-endian file: "NMLMCCK1", u32 version, u32 bytes of the fixed part (up to the levels),
// the input parameters (targetTOL, startTOL, theta, starting_level_coeff, Ca: f64; M0: u64), the
// iteration state (next iteration, total iterations, levels, starting level: u32; calls: u64;
// TOL, bias_est, stat_error, elapsed seconds: f64), per level M (u64), the 4 + 4 FP64 sums, work
// and time (f64), then the sampler state (u64 size + bytes).
constexpr char kCkptMagic[8] = {'N', 'M', 'L', 'M', 'C', 'C', 'K', '1'};
constexpr size_t kStateError = (size_t)-1;     // a state hook's failure (nmlmc_state_save_fn)
constexpr uint32_t kCkptVersion = 1;

struct Checkpoint {
    double targetTOL = 0, startTOL = 0, theta = 0, coeff = 0, Ca = 0;
    uint64_t M0 = 0;
    uint32_t itr_next = 0, total_itrs = 0, starting_level = 0;
    uint64_t calls = 0;
    double TOL = 0, bias_est = 0, stat_error = 0, elapsed = 0;
    std::vector<Level> levels;
    std::string sampler;
};

template <class T>
void put(std::string& b, const T& v) { b.append(reinterpret_cast<const char*>(&v), sizeof(T)); }

template <class T>
bool get(const std::string& b, size_t& o, T& v) {
    if (o + sizeof(T) > b.size()) return false;
    memcpy(&v, b.data() + o, sizeof(T));
    o += sizeof(T);
    return true;
}

int write_checkpoint(const char* path, const Checkpoint& k) {
    std::string b;
    b.append(kCkptMagic, 8);
    put(b, kCkptVersion);
    const uint32_t fixed = 8 + 4 + 4 + 5 * 8 + 8 + 4 * 4 + 8 + 4 * 8;
    put(b, fixed);
    put(b, k.targetTOL); put(b, k.startTOL); put(b, k.theta); put(b, k.coeff); put(b, k.Ca); put(b, k.M0);
    put(b, k.itr_next); put(b, k.total_itrs); put(b, (uint32_t)k.levels.size()); put(b, k.starting_level);
    put(b, k.calls); put(b, k.TOL); put(b, k.bias_est); put(b, k.stat_error); put(b, k.elapsed);
    for (const Level& l : k.levels) {
        put(b, l.M);
        for (int j = 0; j < 4; j++) put(b, l.f[j]);
        for (int j = 0; j < 4; j++) put(b, l.d[j]);
        put(b, l.work);
        put(b, l.time);
    }
    put(b, (uint64_t)k.sampler.size());
    b += k.sampler;
    const std::string tmp = std::string(path) + ".tmp";
    FILE* fp = fopen(tmp.c_str(), "wb");
    if (!fp) return NMLMC_ERR_STATE;
    const bool ok = fwrite(b.data(), 1, b.size(), fp) == b.size();
    if (fclose(fp) != 0 || !ok || rename(tmp.c_str(), path) != 0) {
        remove(tmp.c_str());
        return NMLMC_ERR_STATE;
    }
    return NMLMC_OK;
}

constexpr int kNoCheckpoint = -1;

// kNoCheckpoint: no file at `path`; NMLMC_ERR_ARG: not a readable checkpoint.
int read_checkpoint(const char* path, Checkpoint& k) {
    FILE* fp = fopen(path, "rb");
    if (!fp) return kNoCheckpoint;
    std::string b;
    char chunk[1 << 16];
    size_t n;
    while ((n = fread(chunk, 1, sizeof chunk, fp)) > 0) b.append(chunk, n);
    fclose(fp);
    size_t o = 8;
    uint32_t version = 0, fixed = 0, nlev = 0;
    if (b.size() < 8 || memcmp(b.data(), kCkptMagic, 8) != 0) return NMLMC_ERR_ARG;
    if (!get(b, o, version) || version != kCkptVersion || !get(b, o, fixed)) return NMLMC_ERR_ARG;
    bool ok = get(b, o, k.targetTOL) && get(b, o, k.startTOL) && get(b, o, k.theta) && get(b, o, k.coeff) &&
              get(b, o, k.Ca) && get(b, o, k.M0) && get(b, o, k.itr_next) && get(b, o, k.total_itrs) &&
              get(b, o, nlev) && get(b, o, k.starting_level) && get(b, o, k.calls) && get(b, o, k.TOL) &&
              get(b, o, k.bias_est) && get(b, o, k.stat_error) && get(b, o, k.elapsed);
    if (!ok || o != fixed || nlev == 0 || nlev > NMLMC_MAX_LEVELS || k.starting_level >= nlev) return NMLMC_ERR_ARG;
    k.levels.resize(nlev);
    for (Level& l : k.levels) {
        ok = ok && get(b, o, l.M);
        for (int j = 0; j < 4; j++) ok = ok && get(b, o, l.f[j]);
        for (int j = 0; j < 4; j++) ok = ok && get(b, o, l.d[j]);
        ok = ok && get(b, o, l.work) && get(b, o, l.time);
    }
    uint64_t ns = 0;
    if (!ok || !get(b, o, ns) || o + ns != b.size()) return NMLMC_ERR_ARG;
    // a damaged file whose layout still parses: non-finite level sums or a bad TOL would turn
    // into NaN sample counts
    if (!std::isfinite(k.TOL) || !(k.TOL > 0)) return NMLMC_ERR_ARG;
    for (const Level& l : k.levels) {
        bool fin = std::isfinite(l.work) && l.work >= 0 && std::isfinite(l.time);
        for (int j = 0; j < 4; j++) fin = fin && std::isfinite(l.f[j]) && std::isfinite(l.d[j]);
        if (!fin) return NMLMC_ERR_ARG;
    }
    k.sampler.assign(b.data() + o, ns);
    return NMLMC_OK;
}

bool same_inputs(const Checkpoint& k, const nmlmc_mlmc_input& in) {
    return k.targetTOL == in.targetTOL && k.startTOL == in.startTOL && k.theta == in.theta &&
           k.coeff == in.starting_level_coeff && k.Ca == in.Ca && k.M0 == in.M0;
}

int run(const nmlmc_mlmc_input& in, nmlmc_sample_level_fn level_fn, nmlmc_sample_levels_fn levels_fn,
        void* user, const nmlmc_checkpoint_io* io, nmlmc_mlmc_output* res, char* table, size_t table_cap) {
    const auto t0 = std::chrono::steady_clock::now();
    Output out;
    const double sqrt_2_inv = 1. / std::sqrt(2);
    uint32_t total_itrs = static_cast<uint32_t>(-(std::log2(in.targetTOL) - std::log2(in.startTOL)));
    // targetTOL 2^k as the reference's targetTOL * (1 << k), which is undefined from k = 31 on
    // (startTOL / targetTOL >= 2^31); ldexp gives the same value below that and the right one above
    out.TOL = std::ldexp(in.targetTOL, (int)total_itrs);
    total_itrs *= 2;
    out.levels.resize(1);
    std::vector<uint64_t> Ml(out.levels.size());
    uint64_t calls = 0;
    uint32_t itr0 = 0;
    double elapsed0 = 0;
    const bool ckpt = io && io->path;
    if (ckpt && io->resume) {
        Checkpoint k;
        const int rc = read_checkpoint(io->path, k);
        if (rc == NMLMC_ERR_ARG) return rc;
        if (rc == NMLMC_OK) {
            // the saved level sums come from the sampler's streams up to the saved positions: both
            // an exact resume and a warm start continue from there
            if (!k.sampler.empty()) {
                if (!io->load || io->load(user, k.sampler.data(), k.sampler.size()) != NMLMC_OK) return NMLMC_ERR_STATE;
            }
            out.levels = k.levels;
            out.starting_level = k.starting_level;
            if (same_inputs(k, in) && k.total_itrs == total_itrs) {   // continue the same run
                itr0 = k.itr_next;
                out.TOL = k.TOL;
                out.bias_est = k.bias_est;
                out.stat_error = k.stat_error;
                calls = k.calls;
                elapsed0 = k.elapsed;
            }
        }
    }
    auto save = [&](uint32_t itr_next) -> int {
        Checkpoint k;
        k.targetTOL = in.targetTOL; k.startTOL = in.startTOL; k.theta = in.theta;
        k.coeff = in.starting_level_coeff; k.Ca = in.Ca; k.M0 = in.M0;
        k.itr_next = itr_next; k.total_itrs = total_itrs; k.starting_level = out.starting_level;
        k.calls = calls; k.TOL = out.TOL; k.bias_est = out.bias_est; k.stat_error = out.stat_error;
        k.elapsed = elapsed0 + std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        k.levels = out.levels;
        if (io->save) {
            const size_t need = io->save(user, nullptr, 0);
            if (need == kStateError) return NMLMC_ERR_STATE;
            k.sampler.resize(need);
            if (need && io->save(user, &k.sampler[0], need) != need) return NMLMC_ERR_STATE;
        }
        return write_checkpoint(io->path, k);
    };
    uint32_t done_here = 0;
    bool complete = true;
    uint32_t itr_end = itr0;
    for (uint32_t itr = itr0; itr <= total_itrs; itr++) {
        char label[48];
        snprintf(label, sizeof label, "nmlmc TOL iteration %u", itr);
        const NvtxScope nv(label);
        out.starting_level = better_starting_level(out, in.starting_level_coeff);
        while (true) {
            optimal_Ml(in.theta * sq(out.TOL) / in.Ca, in.M0, out, Ml);
            for (uint64_t m : Ml)
                if (m == kCountOverflow) return NMLMC_ERR_ARG;        // no run of this size ends
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
                    if (rs[i].M != Ms[i] || !usable(rs[i])) return NMLMC_ERR_STATE;
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
                        if (r.M == 0 || !usable(r)) return NMLMC_ERR_STATE;   // the sampler failed
                        out.levels[l] += from_result(r);
                    }
                }
            }
            out.stat_error = std::sqrt(in.Ca * out.total_variance());
            if (sq(out.stat_error) >= in.theta * sq(out.TOL)) continue;
            out.bias_est = default_bias_estimate(out);
            if (sq(out.bias_est) >= (1 - in.theta) * sq(out.TOL)) {
                // a bias that does not decay would add levels for good: the level arrays of the
                // output and of checkpoints hold NMLMC_MAX_LEVELS
                if ((in.max_levels && out.levels.size() >= in.max_levels) || out.levels.size() >= NMLMC_MAX_LEVELS)
                    return NMLMC_ERR_ARG;
                out.levels.resize(out.levels.size() + 1);
                continue;
            }
            if (in.verbose) std::cout << to_string(out);
            break;
        }
        out.TOL *= sqrt_2_inv;
        itr_end = itr + 1;
        if (ckpt) {
            const int rc = save(itr + 1);
            if (rc) return rc;
        }
        if (in.max_iterations && ++done_here >= in.max_iterations && itr < total_itrs) {
            complete = false;
            break;
        }
    }
    const double total = elapsed0 + std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
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
        res->iterations_done = itr_end;
        res->complete = complete ? 1u : 0u;
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

size_t gpu_save_state(void* u, void* buf, size_t cap) {
    GpuUser* g = static_cast<GpuUser*>(u);
    size_t need = 0;
    if (nmlmc_get_sampler_state(g->ctx, nullptr, 0, &need) != NMLMC_OK) return kStateError;
    if (!buf) return need;
    if (cap < need || nmlmc_get_sampler_state(g->ctx, buf, cap, &need) != NMLMC_OK) return kStateError;
    return need;
}
int gpu_load_state(void* u, const void* buf, size_t size) {
    GpuUser* g = static_cast<GpuUser*>(u);
    return nmlmc_set_sampler_state(g->ctx, buf, size);
}

}  // namespace

// Inputs the loop can finish with: tolerances finite and positive, the error split theta strictly
// inside (0, 1) (theta = 0 asks for a zero statistical error, theta = 1 for a zero bias: either
// runs for good), Ca > 0 and at least one sample per new level.
static bool valid_input(const nmlmc_mlmc_input& in) {
    return std::isfinite(in.targetTOL) && in.targetTOL > 0 && std::isfinite(in.startTOL) &&
           in.startTOL >= in.targetTOL && in.theta > 0 && in.theta < 1 && std::isfinite(in.Ca) &&
           in.Ca > 0 && std::isfinite(in.starting_level_coeff) && in.M0 >= 1;
}

// No exception may cross the C ABI: a host allocation that fails inside the driver (levels,
// report text, checkpoint buffers) becomes NMLMC_ERR_NOMEM.
static int guarded_run(const nmlmc_mlmc_input& in, nmlmc_sample_level_fn level_fn,
                       nmlmc_sample_levels_fn levels_fn, void* user, const nmlmc_checkpoint_io* io,
                       nmlmc_mlmc_output* out, char* table, size_t table_cap) {
    try {
        return run(in, level_fn, levels_fn, user, io, out, table, table_cap);
    } catch (const std::bad_alloc&) {
        return NMLMC_ERR_NOMEM;
    } catch (const std::length_error&) {
        return NMLMC_ERR_ARG;
    }
}

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
    in.max_iterations = 0;
    return in;
}

int nmlmc_mlmc_run_cb(const nmlmc_mlmc_input* in, nmlmc_sample_level_fn level_fn,
                      nmlmc_sample_levels_fn levels_fn, void* user, nmlmc_mlmc_output* out,
                      char* table, size_t table_cap) {
    if (!in || !level_fn || !valid_input(*in)) return NMLMC_ERR_ARG;
    return guarded_run(*in, level_fn, levels_fn, user, nullptr, out, table, table_cap);
}

int nmlmc_mlmc_run_cb_ckpt(const nmlmc_mlmc_input* in, nmlmc_sample_level_fn level_fn,
                           nmlmc_sample_levels_fn levels_fn, void* user, const nmlmc_checkpoint_io* io,
                           nmlmc_mlmc_output* out, char* table, size_t table_cap) {
    if (!in || !level_fn || !valid_input(*in)) return NMLMC_ERR_ARG;
    return guarded_run(*in, level_fn, levels_fn, user, io, out, table, table_cap);
}

int nmlmc_mlmc_run(nmlmc_ctx* ctx, const nmlmc_mlmc_input* in, nmlmc_mlmc_output* out, char* table,
                   size_t table_cap) {
    if (!ctx || !in) return NMLMC_ERR_ARG;
    GpuUser u{ctx, NMLMC_OK};
    int rc = nmlmc_mlmc_run_cb(in, gpu_level, gpu_levels, &u, out, table, table_cap);
    return u.status ? u.status : rc;
}

int nmlmc_mlmc_run_ckpt(nmlmc_ctx* ctx, const nmlmc_mlmc_input* in, const char* path, int32_t resume,
                        nmlmc_mlmc_output* out, char* table, size_t table_cap) {
    if (!ctx || !in || !path) return NMLMC_ERR_ARG;
    GpuUser u{ctx, NMLMC_OK};
    nmlmc_checkpoint_io io{path, resume, gpu_save_state, gpu_load_state};
    int rc = nmlmc_mlmc_run_cb_ckpt(in, gpu_level, gpu_levels, &u, &io, out, table, table_cap);
    return u.status ? u.status : rc;
}

}  // extern "C"
