// CORE-layout level sampler: the reference's stream semantics on the GPU.
//
// One warp per virtual core.  Core c owns the random_state pair (seed, c) of the reference's CPU
// build (nested_sampler.hpp:634-642), takes the outer samples OpenMP's static schedule gives
// thread c (nested_sampler.hpp:417) and its streams persist across sample() calls.  Within an
// inner phase the 32 lanes split the phase's samples into contiguous slices and skip ahead to
// their first draw (every draw of the stream has an address), then a warp butterfly reduces the
// double sums — so the per-outer-sample counts and phi values equal the reference's.
//
// Follows kernel_sample (nested_sampler.hpp:369-485), inner_sampler (102-275),
// model::sampler (model_sampler.cpp:42-92) and the BS path of portfolio::sampler
// (portfolio_sampler.cpp:293-468).  RT = float reproduces the default build (real_t = float,
// double Box-Muller and sums), RT = double the -DREAL_DOUBLE build.
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

#include "nmlmc_common.cuh"
#include "nmlmc_internal.h"
#include "nmlmc_paths.cuh"

namespace nmlmc {

// ---- stream reads on the CORE layout ------------------------------------------------------
__device__ __forceinline__ uint64_t core_word(const TfKey& k, uint64_t w) {
    uint64_t v0, v1;
    threefry2x64(w >> 1, 0, k, v0, v1);
    return (w & 1) ? v0 : v1;
}

// words w (drawn first: Box-Muller u1) and w + 1 (drawn second: u0)
__device__ __forceinline__ void core_word_pair(const TfKey& k, uint64_t w, uint64_t& first,
                                               uint64_t& second) {
    uint64_t v0, v1;
    threefry2x64(w >> 1, 0, k, v0, v1);
    if ((w & 1) == 0) {
        first = v1;
        second = v0;
    } else {
        first = v0;
        uint64_t n0, n1;
        threefry2x64((w >> 1) + 1, 0, k, n0, n1);
        second = n1;
    }
}

template <class RT>
__device__ __forceinline__ void core_pair(const TfKey& k, uint64_t w, RT& x, RT& y) {
    uint64_t first, second;
    core_word_pair(k, w, first, second);
    double dx, dy;
    boxmuller64(second, first, dx, dy);
    x = to_rt<RT>(dx);
    y = to_rt<RT>(dy);
}

// Normals of one phase of a CORE stream, addressed by their index in the phase.
template <class RT>
struct PhaseNormals {
    TfKey key;
    uint64_t wpos0;
    bool saved0;
    RT sval0;
    uint64_t cached;
    RT cx, cy;
    __device__ __forceinline__ void init(const TfKey& k, const CoreStream& s) {
        key = k;
        wpos0 = s.wpos;
        saved0 = s.saved != 0;
        sval0 = (RT)s.sval;
        cached = ~0ull;
    }
    __device__ __forceinline__ RT get(uint64_t i) {
        if (saved0) {
            if (i == 0) return sval0;
            i -= 1;
        }
        uint64_t p = i >> 1;
        if (p != cached) {
            core_pair<RT>(key, wpos0 + 2 * p, cx, cy);
            cached = p;
        }
        return (i & 1) ? cy : cx;
    }
};

// Advances a CORE stream past n normals drawn in one phase (warp-uniform).
template <class RT>
__device__ __forceinline__ void advance_normals(CoreStream& s, const TfKey& k, uint64_t n) {
    if (n == 0) return;
    uint64_t fresh = n - (s.saved ? 1 : 0);
    uint64_t pairs = (fresh + 1) / 2;
    if (fresh & 1) {
        RT x, y;
        core_pair<RT>(k, s.wpos + 2 * (pairs - 1), x, y);
        s.saved = 1;
        s.sval = (double)y;
    } else {
        s.saved = 0;
    }
    s.wpos += 2 * pairs;
}

// ---- samplers -----------------------------------------------------------------------------
template <class RT, int KIND>
struct CoreCtx {
    ModelParams<RT> mp;
    OptionTable<RT> ot;
    TfKey key;                  // (seed, core): both streams (nested_sampler.hpp:640-641)
    CoreStream sync, inner;     // warp-uniform copies
    RT* Rt;                     // portfolio: per-warp R_tau in shared memory
    RT Y, constant;
    int err;                    // a path-simulated sample exceeded kMaxPathSteps
};

template <class RT>
__device__ __forceinline__ RT portfolio_bs_value(const OptionTable<RT>& ot, const RT* Rt, uint32_t j,
                                                 double& work) {
    // sample_inner_bs (portfolio_sampler.cpp:453-468) -> option_diff_from_blackscholes (186-200)
    work += (double)ot.W_est[j];
    uint32_t s = ot.stock_ind[j];
    int type = ot.type[j];
    RT sigma = ot.sigma[s];
    RT bs = calc_bs_ref<RT>(type, Rt[s], ot.strike[j], ot.r, xsub(ot.maturity[j], ot.tau), sigma);
    RT finish = ot.discount ? xmul(xexp(xmul(-ot.r, ot.tau)), bs) : bs;
    RT val = xmul(ot.w[j], xsub(ot.start[j], finish));
    RT cv = (RT)0;
    if (ot.use_delta_cv) {
        RT derv = xmul(ot.w[j], calc_delta_ref<RT>(type, ot.S0[s], ot.strike[j], ot.r, ot.maturity[j], sigma));
        cv = xmul(xsub(Rt[s], ot.S0[s]), derv);
    }
    return xadd(val, cv);
}

template <class RT>
__device__ __forceinline__ RT u01_rt(uint64_t w) {
    if constexpr (sizeof(RT) == 4) return u01_f(w); else return u01_d(w);
}

// ---- path-simulated inner values (portfolio_sampler.cpp:212-225, 470-604; gbm_approx.hpp) ----

// Normals of one inner sample, drawn in order from the inner CORE stream: a pending second
// normal of an earlier pair when `have`, then fresh pairs from word position w.
template <class RT>
struct SeqNormals {
    TfKey key;
    uint64_t w;
    bool have;
    RT y;
    __device__ __forceinline__ RT next() {
        if (have) {
            have = false;
            return y;
        }
        RT x;
        core_pair<RT>(key, w, x, y);
        w += 2;
        have = true;
        return x;
    }
};


// rand_int_pdf over compute_prob (common.hpp:178-195), as sample_inner_random_option_ind
// picks the compute method (portfolio_sampler.cpp:350-352).
template <class RT>
__device__ __forceinline__ uint32_t pick_method(const OptionTable<RT>& ot, RT uc) {
    const RT u = xmul(uc, ot.prob_norm);
    RT p = 0;
    uint32_t ret = 0;
    for (uint32_t i = 0; i < 3; i++) {
        const RT cpi = ot.compute_prob[i];
        if (cpi <= (RT)0) continue;
        p = xadd(p, cpi);
        ret = i;
        if (u <= p) break;
    }
    return ret;
}

// Option within method m from the inner randu (portfolio_sampler.cpp:353-369): uniform
// ceil(u n) - 1 with prob 1 / options_count, or rand_int_cdf on the method's CDF.
template <class RT>
__device__ __forceinline__ uint32_t pick_option(const OptionTable<RT>& ot, uint32_t m, RT u, RT& prob) {
    const uint32_t nm = ot.m_n[m], off = ot.m_off[m];
    if (ot.subsample == SUB_UNIFORM) {
        prob = ot.inv_count_prob;
        return off + (uint32_t)(xceil(xmul(u, (RT)nm)) - (RT)1);
    }
    const RT uu = xmul(u, ot.compute_prob[m]);
    uint32_t pos0 = 0, pos1 = nm;
    if (nm > 1) {
        const uint32_t steps = 32 - __clz(nm - 1);
        for (uint32_t t = 0; t < steps; t++) {
            const uint32_t mid = (pos0 + pos1) / 2;
            if (mid > 0 && uu < ot.cdf[off + mid]) pos1 = mid; else pos0 = mid;
        }
    }
    prob = xdiv(ot.prob[off + pos0], ot.prob_norm);
    return off + pos0;
}

__device__ __forceinline__ uint32_t nth_set_bit(uint32_t m, uint32_t n) {   // 32 when absent
    for (uint32_t i = 0; i < n && m; i++) m &= m - 1;
    return m ? (uint32_t)(__ffs(m) - 1) : 32u;
}

// init_inner_sampler: start value (model: -max_loss; portfolio: Y.constant, plus the full
// deterministic BS sum when Subsampling::None).  Warp-cooperative, result in every lane.
template <class RT, int KIND>
__device__ RT core_init_inner(CoreCtx<RT, KIND>& c, double& work, int lane) {
    if (KIND != KIND_PORTFOLIO) return -c.mp.max_loss;
    if (c.ot.subsample != SUB_NONE) return c.constant;
    double det = 0, w = 0;
    for (uint32_t j = lane; j < c.ot.m_n[METHOD_BS]; j += 32) det += (double)portfolio_bs_value<RT>(c.ot, c.Rt, j, w);
    det = warp_sum(det);
    work += warp_sum(w);             // warp total, identical in every lane
    return xadd(to_rt<RT>(det), c.constant);
}

// Inner phase of a portfolio with Exact / Unbiased options on the CORE streams.  A sample draws
// a variable number of words: on the sync stream the method word (sub-sampled modes) and one
// level word per Unbiased evaluation; on the inner stream the option-index word (sub-sampled
// modes) and the normals of its paths.  Windows of up to 32 samples, one per lane: the sync
// words of a window are parsed first (a word is a method word unless the previous method word
// chose Unbiased), the normal counts are prefix-summed over the lanes, and every lane then
// addresses its own words directly — a normal pair's words sit after the index words of the
// samples up to the one that drew it — so the draws equal the reference's sequential ones.
template <class RT>
__device__ void core_phase_paths(CoreCtx<RT, KIND_PORTFOLIO>& c, uint64_t count, bool want_s2, double& a1,
                                 double& a2, double& w, uint64_t& nu, uint64_t& nn, int lane, bool& err) {
    const OptionTable<RT>& ot = c.ot;
    const bool none = ot.subsample == SUB_NONE;
    const uint64_t r_in = none ? 0 : 1;                 // inner-stream index words per sample
    const uint32_t n_exact = ot.m_n[METHOD_EXACT], n_unb = ot.m_n[METHOD_UNBIASED];
    uint64_t done = 0;
    while (done < count) {
        const uint64_t rem = count - done;
        uint32_t nsamp;
        uint64_t sync_used;
        uint32_t my_m = METHOD_BS;
        uint64_t my_lword = 0;                          // sub-sampled: the Unbiased level word
        uint64_t n_norm = 0;                            // normals this lane's sample draws
        bool ok = true;
        if (!none) {
            const uint64_t sw = core_word(c.key, c.sync.wpos + (uint64_t)lane);
            const uint32_t mth = pick_method<RT>(ot, u01_rt<RT>(sw));
            const uint32_t U = __ballot_sync(0xffffffffu, mth == METHOD_UNBIASED);
            uint32_t mask = 0, pos = 0;
            nsamp = 0;
            while (pos < 32 && nsamp < rem) {
                mask |= 1u << pos;
                nsamp++;
                pos += 1 + ((U >> pos) & 1u);
            }
            sync_used = pos;
            const uint32_t q = nth_set_bit(mask, (uint32_t)lane);
            const uint32_t qm = __shfl_sync(0xffffffffu, mth, q & 31);
            uint64_t lw = __shfl_sync(0xffffffffu, (unsigned long long)sw, (q + 1) & 31);
            if ((uint32_t)lane < nsamp) {
                my_m = qm;
                if (my_m == METHOD_UNBIASED) {
                    if (q + 1 >= 32) lw = core_word(c.key, c.sync.wpos + q + 1);
                    my_lword = lw;
                    uint32_t L;
                    uint64_t N_l;
                    ok = unbiased_level<RT>(ot, u01_rt<RT>(lw), L, N_l);
                    n_norm = ok ? 1 + (uint64_t)ot.dt_h0inv * N_l : 0;
                } else if (my_m == METHOD_EXACT) {
                    n_norm = 2;
                }
            }
        } else {
            // sample_inner_all_options (portfolio_sampler.cpp:336-344): every Exact option, then
            // every Unbiased one, each of the latter with its own level word
            nsamp = (uint32_t)(rem < 32 ? rem : 32);
            sync_used = (uint64_t)nsamp * n_unb;
            if ((uint32_t)lane < nsamp) {
                n_norm = 2ull * n_exact;
                const uint64_t w0 = c.sync.wpos + (uint64_t)lane * n_unb;
                for (uint32_t k = 0; k < n_unb && ok; k++) {
                    uint32_t L;
                    uint64_t N_l;
                    ok = unbiased_level<RT>(ot, u01_rt<RT>(core_word(c.key, w0 + k)), L, N_l);
                    n_norm += ok ? 1 + (uint64_t)ot.dt_h0inv * N_l : 0;
                }
            }
        }
        if (!ok) err = true;
        // exclusive prefix of the normal counts over the lanes
        uint64_t incl = n_norm;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint64_t t = __shfl_up_sync(0xffffffffu, (unsigned long long)incl, d);
            if (lane >= d) incl += t;
        }
        const uint64_t C = incl - n_norm;
        const uint64_t C_tot = __shfl_sync(0xffffffffu, (unsigned long long)incl, 31);
        const uint32_t nz_mask = __ballot_sync(0xffffffffu, n_norm > 0);
        const uint64_t wpos_w = c.inner.wpos;
        const uint64_t s0 = c.inner.saved ? 1 : 0;
        // pairs drawn for the first C normals of the window: ceil((C - s0) / 2)
        const uint64_t pairs_before = (C + 1 - s0) >> 1;
        if ((uint32_t)lane < nsamp && ok) {
            SeqNormals<RT> nz;
            nz.key = c.key;
            nz.w = wpos_w + r_in * ((uint64_t)lane + 1) + 2 * pairs_before;
            nz.have = ((s0 ^ (C & 1)) != 0);
            nz.y = (RT)0;
            if (nz.have && n_norm > 0) {
                if (C == 0) {
                    nz.y = (RT)c.inner.sval;
                } else {
                    // the pending normal is the second one of the pair the last earlier lane
                    // with normals drew
                    const uint32_t prior = nz_mask & ((1u << lane) - 1u);
                    const uint32_t l = 31 - __clz(prior);
                    RT x;
                    core_pair<RT>(c.key, wpos_w + r_in * ((uint64_t)l + 1) + 2 * (pairs_before - 1), x, nz.y);
                }
            }
            double wk = 0;
            RT v;
            RT prob = (RT)1;
            if (!none) {
                const uint64_t iw = core_word(c.key, wpos_w + (uint64_t)lane + 2 * pairs_before);
                const uint32_t j = pick_option<RT>(ot, my_m, u01_rt<RT>(iw), prob);
                if (my_m == METHOD_BS) {
                    v = portfolio_bs_value<RT>(ot, c.Rt, j, wk);
                } else if (my_m == METHOD_EXACT) {
                    v = inner_exact<RT, SeqNormals<RT>>(ot, c.Rt[ot.stock_ind[j]], j, nz, wk);
                } else {
                    uint32_t L;
                    uint64_t N_l;
                    unbiased_level<RT>(ot, u01_rt<RT>(my_lword), L, N_l);
                    v = inner_unbiased<RT, SeqNormals<RT>>(ot, c.Rt[ot.stock_ind[j]], j, nz, wk, L, N_l);
                }
                v = xdiv(v, prob);
            } else {
                double acc = 0;
                const uint32_t oe = ot.m_off[METHOD_EXACT], ou = ot.m_off[METHOD_UNBIASED];
                for (uint32_t k = 0; k < n_exact; k++) acc += (double)inner_exact<RT, SeqNormals<RT>>(ot, c.Rt[ot.stock_ind[oe + k]], oe + k, nz, wk);
                const uint64_t w0 = c.sync.wpos + (uint64_t)lane * n_unb;
                for (uint32_t k = 0; k < n_unb; k++) {
                    uint32_t L;
                    uint64_t N_l;
                    unbiased_level<RT>(ot, u01_rt<RT>(core_word(c.key, w0 + k)), L, N_l);
                    acc += (double)inner_unbiased<RT, SeqNormals<RT>>(ot, c.Rt[ot.stock_ind[ou + k]], ou + k, nz, wk, L, N_l);
                }
                v = to_rt<RT>(acc);
            }
            w += wk;
            a1 += (double)v;
            if (want_s2) a2 += (double)xmul(v, v);
        }
        __syncwarp();
        // stream states after the window
        const uint64_t pairs_tot = (C_tot + 1 - s0) >> 1;
        const uint64_t s_end = s0 ^ (C_tot & 1);
        if (C_tot > 0 && s_end) {
            const uint32_t l_last = 31 - __clz(nz_mask);
            RT x, y;
            core_pair<RT>(c.key, wpos_w + r_in * ((uint64_t)l_last + 1) + 2 * (pairs_tot - 1), x, y);
            c.inner.sval = (double)y;
        }
        c.inner.saved = (uint32_t)s_end;
        c.inner.wpos = wpos_w + r_in * nsamp + 2 * pairs_tot;
        c.sync.wpos += sync_used;
        nu += sync_used + r_in * nsamp;
        nn += C_tot;
        done += nsamp;
    }
}

// The inner phase: `count` inner samples split over the lanes; returns warp totals of s1 (and
// s2 when want_s2) in every lane; advances the streams.  Sums are double like sum_t
// (nested_sampler.hpp:131-161); d*d is formed in real_t as the reference does.
template <class RT, int KIND>
__device__ void core_phase(CoreCtx<RT, KIND>& c, uint64_t count, bool want_s2, double& s1, double& s2,
                           double& work, uint64_t& nrandu, uint64_t& nrandn, int lane) {
    const uint64_t lo = (uint64_t)lane * count / 32, hi = (uint64_t)(lane + 1) * count / 32;
    double a1 = 0, a2 = 0, w = 0;
    if (KIND == KIND_REF_MODEL || KIND == KIND_SHIFT_MODEL) {
        PhaseNormals<RT> pn;
        pn.init(c.key, c.inner);
        for (uint64_t i = lo; i < hi; i++) {
            RT d;
            if (KIND == KIND_REF_MODEL) {       // model_sampler.cpp:62-76
                RT X = pn.get(2 * i), Y2 = pn.get(2 * i + 1);
                RT a = xadd(xmul(c.mp.stau, c.Y), xmul(c.mp.s1tau, X));
                RT b = xadd(xmul(c.mp.stau, Y2), xmul(c.mp.s1tau, X));
                d = xsub(xmul(a, a), xmul(b, b));
            } else {                            // X = Y + Z
                d = xadd(c.Y, pn.get(i));
            }
            w += 1.0;
            a1 += (double)d;
            if (want_s2) a2 += (double)xmul(d, d);
        }
        const uint64_t per = (KIND == KIND_REF_MODEL) ? 2 : 1;
        __syncwarp();
        advance_normals<RT>(c.inner, c.key, per * count);
        nrandn += per * count;
    } else if (c.ot.mixed) {
        if constexpr (KIND == KIND_PORTFOLIO) {
            bool err = false;
            core_phase_paths<RT>(c, count, want_s2, a1, a2, w, nrandu, nrandn, lane, err);
            if (__any_sync(0xffffffffu, err)) c.err = 1;
        }
    } else if (c.ot.subsample != SUB_NONE) {
        // sample_inner_random_option(_ind) (portfolio_sampler.cpp:346-380): one randu_sync for
        // the method (rand_int_pdf over compute_prob) and one randu for the option index.
        uint64_t cached_blk_s = ~0ull, cached_blk_i = ~0ull;
        uint64_t sv0 = 0, sv1 = 0, iv0 = 0, iv1 = 0;
        for (uint64_t i = lo; i < hi; i++) {
            uint64_t ws = c.sync.wpos + i, wi = c.inner.wpos + i;
            if ((ws >> 1) != cached_blk_s) { threefry2x64(ws >> 1, 0, c.key, sv0, sv1); cached_blk_s = ws >> 1; }
            if ((wi >> 1) != cached_blk_i) { threefry2x64(wi >> 1, 0, c.key, iv0, iv1); cached_blk_i = wi >> 1; }
            uint64_t wsync = (ws & 1) ? sv0 : sv1, winner = (wi & 1) ? iv0 : iv1;
            RT uc = sizeof(RT) == 4 ? (RT)u01_f(wsync) : (RT)u01_d(wsync);
            (void)uc;   // a single compute method carries probability: rand_int_pdf returns it
            RT u = sizeof(RT) == 4 ? (RT)u01_f(winner) : (RT)u01_d(winner);
            uint32_t idx;
            RT prob;
            if (c.ot.subsample == SUB_UNIFORM) {
                idx = (uint32_t)(xceil(xmul(u, (RT)c.ot.P)) - (RT)1);
                prob = c.ot.inv_count_prob;
            } else {
                RT uu = xmul(u, c.ot.compute_prob0);
                // rand_int_cdf (common.hpp:160-176)
                uint32_t pos0 = 0, pos1 = c.ot.P;
                if (c.ot.P > 1) {
                    uint32_t steps = 32 - __clz(c.ot.P - 1);
                    for (uint32_t s = 0; s < steps; s++) {
                        uint32_t mid = (pos0 + pos1) / 2;
                        if (mid > 0 && uu < c.ot.cdf[mid]) pos1 = mid; else pos0 = mid;
                    }
                }
                idx = pos0;
                prob = xdiv(c.ot.prob[idx], c.ot.prob_norm);
            }
            RT v = portfolio_bs_value<RT>(c.ot, c.Rt, idx, w);
            RT d = xdiv(v, prob);
            a1 += (double)d;
            if (want_s2) a2 += (double)xmul(d, d);
        }
        c.sync.wpos += count;
        c.inner.wpos += count;
        nrandu += 2 * count;
    } else {
        // Subsampling::None with BS options only: sample_inner_all_options covers the other
        // compute methods, none here, so every inner sample is 0.
    }
    s1 = warp_sum(a1);
    if (want_s2) s2 = warp_sum(a2);
    work += warp_sum(w);
}

template <class RT, int KIND>
__device__ void core_sample_outer(CoreCtx<RT, KIND>& c, uint64_t& nrandn, int lane) {
    __syncwarp();
    if (KIND != KIND_PORTFOLIO) {                     // model_sampler.cpp:53-55
        PhaseNormals<RT> pn;
        pn.init(c.key, c.sync);
        c.Y = pn.get(0);
        __syncwarp();
        advance_normals<RT>(c.sync, c.key, 1);
        nrandn += 1;
        return;
    }
    // portfolio_sampler.cpp:293-311: dW_sys then one normal per stock
    const OptionTable<RT>& ot = c.ot;
    PhaseNormals<RT> pn;
    pn.init(c.key, c.sync);
    RT dW_sys = xmul(ot.stau, pn.get(0));
    if (ot.Q == 1) {
        if (lane == 0) c.Rt[0] = simulate_stock_ref<RT>(ot.S0[0], ot.mu[0], ot.sigma[0], ot.tau, dW_sys);
    } else {
        for (uint32_t i = lane; i < ot.Q; i += 32) {
            RT dW_ind = xmul(ot.stau, pn.get(1 + i));
            RT W = xadd(xmul(ot.rho, dW_sys), xmul(ot.s1_rho2, dW_ind));
            c.Rt[i] = simulate_stock_ref<RT>(ot.S0[i], ot.mu[i], ot.sigma[i], ot.tau, W);
        }
    }
    __syncwarp();
    uint64_t n = (ot.Q == 1) ? 1 : (uint64_t)ot.Q + 1;
    advance_normals<RT>(c.sync, c.key, n);
    nrandn += n;
    // compute_delta_cv (606-614): sequential real_t sum, as the reference accumulates it
    RT cv = (RT)0;
    if (ot.use_delta_cv)
        for (uint32_t i = 0; i < ot.Q; i++) cv = xadd(cv, xmul(xsub(c.Rt[i], ot.S0[i]), ot.delta_coalesce[i]));
    c.constant = xsub(-ot.max_loss, cv);
}

template <class RT>
__device__ __forceinline__ void add_phi_ref(RT mean, RT coeff, RT& phi) {   // model_sampler.cpp:77-86
    phi = xadd(phi, xmul(coeff, (RT)(mean >= (RT)0 ? 1 : 0)));
}

// get_samples_count<WITH_STATS>::operator() (nested_sampler.hpp:240-273)
template <class RT, int KIND>
__device__ uint64_t core_count(CoreCtx<RT, KIND>& c, const CountParams& cp, RT r, bool with_stats,
                               uint64_t* st, double& work, uint64_t& nu, uint64_t& nn,
                               uint32_t& pilots, int lane) {
    uint64_t cur = cp.base_count;
    const RT tmp = (RT)cp.tmp;
    for (;;) {
        if (cp.max_count <= 2 * cur) { cur = cp.max_count; break; }
        st[0] += cur;
        pilots++;
        // sample_inner_delta2 (120-129)
        RT start = core_init_inner<RT, KIND>(c, work, lane);
        double s1 = 0, s2 = 0;
        core_phase<RT, KIND>(c, cur, true, s1, s2, work, nu, nn, lane);
        RT out_var = to_rt<RT>(__dsub_rn(__ddiv_rn(s2, (double)(cur - 1)),
                                         __ddiv_rn(__dmul_rn(s1, s1), (double)(cur * (cur - 1)))));
        RT dist = xadd(start, to_rt<RT>(__ddiv_rn(s1, (double)cur)));
        RT delta2 = xdiv(xmul(dist, dist), out_var);
        RT newc = xmul(xpow(delta2, xdiv(-r, (RT)2)), tmp);
        if (newc <= (RT)cur) break;
        cur *= 2;
    }
    if (with_stats) {
        st[1] += 1;
        st[2] += (cur == cp.max_count);
        st[3] += (cur == cp.base_count);
    }
    return cur;
}

template <class RT, int KIND>
__global__ void __launch_bounds__(256) core_level_kernel(CoreLaunch<RT> L, CoreStream* states,
                                                         double* out_sums, uint64_t* out_stats,
                                                         TraceRec* trace) {
    extern __shared__ unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const uint32_t warp_in_block = threadIdx.x >> 5;
    const uint32_t core = blockIdx.x * (blockDim.x >> 5) + warp_in_block;
    if (core >= L.cores) return;

    CoreCtx<RT, KIND> c;
    c.mp = L.mp;
    c.ot = L.ot;
    c.key = tf_key(L.seed, core);
    c.sync = states[2 * core];
    c.inner = states[2 * core + 1];
    c.Rt = reinterpret_cast<RT*>(smem_raw) + (size_t)warp_in_block * (L.ot.Q ? L.ot.Q : 1);
    c.Y = 0;
    c.constant = 0;
    c.err = 0;

    const uint64_t q = L.M / L.cores, rem = L.M % L.cores;
    const uint64_t mcount = q + (core < rem ? 1 : 0);
    const uint64_t mfirst = q * core + (core < rem ? core : rem);
    const bool fine_only = L.fine_only;
    const RT r = (RT)L.adaptive_r;

    double f_sums[4] = {0, 0, 0, 0}, d_sums[4] = {0, 0, 0, 0}, work = 0;
    uint64_t st[6] = {0, 0, 0, 0, 0, 0};
    uint64_t nu = 0, nn = 0;

    for (uint64_t mm = 0; mm < mcount; mm++) {
        TraceRec tr;
        tr.core = core;
        tr.pilots = 0;
        tr.min_abs_small = INFINITY;
        tr.mean_big = 0;
        core_sample_outer<RT, KIND>(c, nn, lane);
        uint64_t cf = core_count<RT, KIND>(c, L.cf, r, true, st, work, nu, nn, tr.pilots, lane);
        uint64_t cc = 0;
        RT f_phi = (RT)0, c_phi = (RT)0;
        if (fine_only) {
            st[0] += cf;
            RT start = core_init_inner<RT, KIND>(c, work, lane);   // sample_inner_mean (112-119)
            double s1 = 0, s2 = 0;
            core_phase<RT, KIND>(c, cf, false, s1, s2, work, nu, nn, lane);
            RT mean = to_rt<RT>(__dadd_rn((double)start, __ddiv_rn(s1, (double)cf)));
            add_phi_ref<RT>(mean, (RT)1, f_phi);
            tr.mean_big = (double)mean;
        } else {
            cc = core_count<RT, KIND>(c, L.cc, r, false, st, work, nu, nn, tr.pilots, lane);
            if (L.antithetic) {
                // sample_phi_antithetic (171-216)
                uint64_t cbig, csmall;
                RT *obig, *osmall;
                if (cf > cc) { obig = &f_phi; osmall = &c_phi; cbig = cf; csmall = cc; }
                else { obig = &c_phi; osmall = &f_phi; cbig = cc; csmall = cf; }
                uint64_t groups = cbig / csmall;
                RT coeff = xdiv((RT)1, (RT)groups);
                RT start_small = 0;
                double s1_big = 0, min_abs = INFINITY;
                for (uint64_t g = 0; g < groups; g++) {
                    start_small = core_init_inner<RT, KIND>(c, work, lane);
                    double s1 = 0, s2 = 0;
                    core_phase<RT, KIND>(c, csmall, false, s1, s2, work, nu, nn, lane);
                    RT ms = to_rt<RT>(__dadd_rn((double)start_small, __ddiv_rn(s1, (double)csmall)));
                    add_phi_ref<RT>(ms, coeff, *osmall);
                    min_abs = fmin(min_abs, fabs((double)ms));
                    s1_big = __dadd_rn(s1_big, s1);
                }
                RT mb = to_rt<RT>(__dadd_rn((double)start_small, __ddiv_rn(s1_big, (double)cbig)));
                add_phi_ref<RT>(mb, (RT)1, *obig);
                st[0] += cbig;
                tr.mean_big = (double)mb;
                tr.min_abs_small = min_abs;
            } else {
                st[0] += cf + cc;
                RT s0 = core_init_inner<RT, KIND>(c, work, lane);
                double s1 = 0, s2 = 0;
                core_phase<RT, KIND>(c, cf, false, s1, s2, work, nu, nn, lane);
                RT mf = to_rt<RT>(__dadd_rn((double)s0, __ddiv_rn(s1, (double)cf)));
                add_phi_ref<RT>(mf, (RT)1, f_phi);
                s0 = core_init_inner<RT, KIND>(c, work, lane);
                core_phase<RT, KIND>(c, cc, false, s1, s2, work, nu, nn, lane);
                RT mc = to_rt<RT>(__dadd_rn((double)s0, __ddiv_rn(s1, (double)cc)));
                add_phi_ref<RT>(mc, (RT)1, c_phi);
                tr.mean_big = (double)mf;
                tr.min_abs_small = fabs((double)mc);
            }
        }
        // add_moments (87-100)
        RT p = (RT)1;
        for (int j = 0; j < 4; j++) { p = xmul(p, f_phi); f_sums[j] += (double)p; }
        if (!fine_only) {
            RT dphi = xsub(f_phi, c_phi);
            p = (RT)1;
            for (int j = 0; j < 4; j++) { p = xmul(p, dphi); d_sums[j] += (double)p; }
        }
        if (trace && lane == 0) {
            tr.count_f = cf;
            tr.count_c = cc;
            tr.phi_f = (double)f_phi;
            tr.phi_c = (double)c_phi;
            trace[mfirst + mm] = tr;
        }
    }
    if (lane == 0) {
        states[2 * core] = c.sync;
        states[2 * core + 1] = c.inner;
        double* o = out_sums + (size_t)core * 10;
        for (int j = 0; j < 4; j++) { o[j] = f_sums[j]; o[4 + j] = d_sums[j]; }
        o[8] = work;
        o[9] = c.err ? 1.0 : 0.0;
        uint64_t* s = out_stats + (size_t)core * 6;
        for (int j = 0; j < 4; j++) s[j] = st[j];
        s[4] = nu;
        s[5] = nn;
    }
}

// Sums the per-core partials in core order (one block).
__global__ void core_reduce_kernel(uint32_t cores, const double* in_sums, const uint64_t* in_stats,
                                   double* out_sums, uint64_t* out_stats) {
    __shared__ double sd[256][10];
    __shared__ uint64_t su[256][6];
    const uint32_t t = threadIdx.x;
    double a[10] = {0};
    uint64_t b[6] = {0};
    for (uint32_t c = t; c < cores; c += blockDim.x) {
        for (int j = 0; j < 10; j++) a[j] += in_sums[(size_t)c * 10 + j];
        for (int j = 0; j < 6; j++) b[j] += in_stats[(size_t)c * 6 + j];
    }
    for (int j = 0; j < 10; j++) sd[t][j] = a[j];
    for (int j = 0; j < 6; j++) su[t][j] = b[j];
    __syncthreads();
    for (uint32_t s = blockDim.x / 2; s > 0; s >>= 1) {
        if (t < s) {
            for (int j = 0; j < 10; j++) sd[t][j] += sd[t + s][j];
            for (int j = 0; j < 6; j++) su[t][j] += su[t + s][j];
        }
        __syncthreads();
    }
    if (t == 0) {
        for (int j = 0; j < 10; j++) out_sums[j] = sd[0][j];
        for (int j = 0; j < 6; j++) out_stats[j] = su[0][j];
    }
}

template <class RT>
static cudaError_t launch_core_t(const CoreLaunch<RT>& L, int kind, CoreStream* states, double* part_sums,
                                 uint64_t* part_stats, double* out_sums, uint64_t* out_stats,
                                 TraceRec* trace, cudaStream_t stream) {
    const int threads = 256, warps = threads / 32;
    const uint32_t blocks = (L.cores + warps - 1) / warps;
    size_t smem = (kind == KIND_PORTFOLIO) ? (size_t)warps * (L.ot.Q ? L.ot.Q : 1) * sizeof(RT) : 0;
    if (kind == KIND_REF_MODEL)
        core_level_kernel<RT, KIND_REF_MODEL><<<blocks, threads, smem, stream>>>(L, states, part_sums, part_stats, trace);
    else if (kind == KIND_SHIFT_MODEL)
        core_level_kernel<RT, KIND_SHIFT_MODEL><<<blocks, threads, smem, stream>>>(L, states, part_sums, part_stats, trace);
    else {
        if (smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(core_level_kernel<RT, KIND_PORTFOLIO>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
        }
        core_level_kernel<RT, KIND_PORTFOLIO><<<blocks, threads, smem, stream>>>(L, states, part_sums, part_stats, trace);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    core_reduce_kernel<<<1, 256, 0, stream>>>(L.cores, part_sums, part_stats, out_sums, out_stats);
    count_launch(2);
    return cudaGetLastError();
}

cudaError_t launch_core(const CoreLaunch<float>& L, int kind, CoreStream* states, double* part_sums,
                        uint64_t* part_stats, double* out_sums, uint64_t* out_stats, TraceRec* trace,
                        cudaStream_t stream) {
    return launch_core_t<float>(L, kind, states, part_sums, part_stats, out_sums, out_stats, trace, stream);
}
cudaError_t launch_core(const CoreLaunch<double>& L, int kind, CoreStream* states, double* part_sums,
                        uint64_t* part_stats, double* out_sums, uint64_t* out_stats, TraceRec* trace,
                        cudaStream_t stream) {
    return launch_core_t<double>(L, kind, states, part_sums, part_stats, out_sums, out_stats, trace, stream);
}

}  // namespace nmlmc
