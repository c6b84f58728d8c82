#pragma once
// OUTER-layout (batched) level sampler: kernels and the per-level launch sequence.
//
// Included by nmlmc_outer.cu (dispatch, full-loss sweep, utilities) and by nmlmc_outer_kind.cu,
// which is compiled once per sampler kind (NMLMC_OUTER_KIND) so the kernel instantiations build
// in parallel.
//
// The reference walks each outer sample depth-first: pilots of doubling size until the
// adaptive rule stops (get_samples_count, nested_sampler.hpp:240-273), then the antithetic
// fine/coarse estimate (sample_phi_antithetic, 171-216).  Adaptive counts differ by up to 2^ell
// between outer samples, so a warp per outer sample leaves most of the GPU idle behind the few
// samples that refine to the maximum.  Here every outer sample has its own counter-based
// stream (key = (seed, level<<56 | index), counter = (block, phase tag)), which makes each
// inner sample addressable, and a level call runs breadth-first:
//
//   k_outer      one thread per outer sample: outer draws (Y, or R_tau row + constant)
//   k_phase      pilot round r: every outer sample still refining, fine and coarse, as
//                uniform-size segments; one thread per chunk of inner samples, block-segmented
//                reduction, the adaptive decision fused in (survivors appended to the next
//                round's list)
//   k_classify   bucket outer samples by their final count (a power of two)
//   k_phase      final: antithetic groups and the big-count mean, phi, 4 moments into per-CTA
//                partial sums (fixed order, no atomics on the sums)
//   k_reduce     per-CTA partials -> the level's sums
//
// Every thread does the same unit of work (one chunk), so the device stays full whatever the
// spread of inner counts.  An item with more chunks than a CTA has threads is walked tile by
// tile by one CTA.
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

#include "nmlmc_common.cuh"
#include "nmlmc_internal.h"
#include "nmlmc_paths.cuh"

namespace nmlmc {

constexpr int kTile = 256;           // threads per CTA = chunks per tile
constexpr int kWarps = kTile / 32;
constexpr int kMaxSegs = 40;

// device counter slots (uint32 each)
enum : int {
    CNT_LIST = 0,        // [4]: fine list size (ping-pong slots 0/1), coarse list size (2/3)
    CNT_CLASS = 8,       // [64]: outer samples per final class
    CNT_FILL = 72,       // [64]: scatter fill per class
    CNT_TOTAL = 144,
    CNT_QUEUE = 192,     // [kMaxSegs]: tile tickets of the phase kernel's work queue, per segment
    CNT_ERR = kCounterPathLimit   // set when a path-simulated inner sample exceeds kMaxPathSteps
};
static_assert(CNT_QUEUE + kMaxSegs <= CNT_ERR && CNT_ERR < 256, "counter slots");

// ---- accumulators -------------------------------------------------------------------------
// FP32: compensated pair (hi + lo) — Kahan accumulation inside a thread (of pairs of consecutive
// inner values where the kind draws them together), TwoSum merging across threads.  FP64 and
// REF32: double, the reference's sum_t, one value at a time in the reference's order.
template <int PREC> struct Acc;

template <> struct Acc<PREC_FP32> {
    float hi, lo;
    __device__ __forceinline__ void zero() { hi = 0.f; lo = 0.f; }
    __device__ __forceinline__ void add(float v) {
        float y = __fadd_rn(v, lo);
        float t = __fadd_rn(hi, y);
        lo = __fsub_rn(y, __fsub_rn(t, hi));
        hi = t;
    }
    __device__ __forceinline__ void merge(const Acc& o) {
        float s = __fadd_rn(hi, o.hi);
        float bp = __fsub_rn(s, hi);
        float e = __fadd_rn(__fsub_rn(hi, __fsub_rn(s, bp)), __fsub_rn(o.hi, bp));
        hi = s;
        lo = __fadd_rn(__fadd_rn(lo, o.lo), e);
    }
    __device__ __forceinline__ Acc shfl_xor(int m) const {
        Acc r;
        r.hi = __shfl_xor_sync(0xffffffffu, hi, m);
        r.lo = __shfl_xor_sync(0xffffffffu, lo, m);
        return r;
    }
    __device__ __forceinline__ float value() const { return __fadd_rn(hi, lo); }
    // plain addition: the pilots' sum of squares, which only feeds the variance estimate of the
    // adaptive rule (sums of 4-64 squares per thread of values centred on the threshold)
    __device__ __forceinline__ void add_sq(float v) { hi = fmaf(v, v, hi); }
    // the pilots' sum of squares across lanes: a plain sum, like add_sq (its lo stays zero)
    __device__ __forceinline__ void sq_merge_xor(int m) { hi = __fadd_rn(hi, __shfl_xor_sync(0xffffffffu, hi, m)); }
    // two consecutive inner values: their plain sum (one rounding of a value bounded by the two
    // summands), then the compensated step
    __device__ __forceinline__ void add2(float v0, float v1) { add(__fadd_rn(v0, v1)); }
};

template <> struct Acc<PREC_FP64> {
    double v;
    __device__ __forceinline__ void zero() { v = 0; }
    __device__ __forceinline__ void sq_merge_xor(int m) { v = __dadd_rn(v, __shfl_xor_sync(0xffffffffu, v, m)); }
    __device__ __forceinline__ void add(double x) { v = __dadd_rn(v, x); }
    __device__ __forceinline__ void add2(double x0, double x1) { add(x0); add(x1); }
    __device__ __forceinline__ void add_sq(double x) { v = __dadd_rn(v, __dmul_rn(x, x)); }
    __device__ __forceinline__ void merge(const Acc& o) { v = __dadd_rn(v, o.v); }
    __device__ __forceinline__ Acc shfl_xor(int m) const { Acc r; r.v = __shfl_xor_sync(0xffffffffu, v, m); return r; }
    __device__ __forceinline__ double value() const { return v; }
};
template <> struct Acc<PREC_REF32> {
    double v;
    __device__ __forceinline__ void zero() { v = 0; }
    __device__ __forceinline__ void sq_merge_xor(int m) { v = __dadd_rn(v, __shfl_xor_sync(0xffffffffu, v, m)); }
    __device__ __forceinline__ void add(double x) { v = __dadd_rn(v, x); }
    __device__ __forceinline__ void add2(double x0, double x1) { add(x0); add(x1); }
    __device__ __forceinline__ void add_sq(double x) { v = __dadd_rn(v, __dmul_rn(x, x)); }
    __device__ __forceinline__ void merge(const Acc& o) { v = __dadd_rn(v, o.v); }
    __device__ __forceinline__ Acc shfl_xor(int m) const { Acc r; r.v = __shfl_xor_sync(0xffffffffu, v, m); return r; }
    __device__ __forceinline__ double value() const { return v; }
};

template <class RT>
struct DevLevel {
    OuterLevel<RT> L;
    OuterBuffers B;
};

// s / count; a power-of-two count multiplies by its exact reciprocal, which gives the same
// correctly rounded quotient without the division sequence.
__device__ __forceinline__ float div_count(float s, uint64_t count) {
    if ((count & (count - 1)) == 0) return __fmul_rn(s, __int_as_float((127 - (63 - __clzll((long long)count))) << 23));
    return __fdiv_rn(s, (float)count);
}
__device__ __forceinline__ double div_count(double s, uint64_t count) {
    if ((count & (count - 1)) == 0)
        return __dmul_rn(s, __longlong_as_double((long long)(1023 - (63 - __clzll((long long)count))) << 52));
    return __ddiv_rn(s, (double)count);
}

// inner mean start + s1 / count (sample_inner_mean, nested_sampler.hpp:112-119)
template <class RT, int PREC>
__device__ __forceinline__ RT inner_mean(RT start, const Acc<PREC>& s1, uint64_t count) {
    if (PREC == PREC_FP32) return __fadd_rn((float)start, div_count((float)s1.value(), count));
    return to_rt<RT>(__dadd_rn((double)start, div_count((double)s1.value(), count)));
}

// Box-Muller pair from two OUTER words at the context precision.
template <int PREC, class RT>
__device__ __forceinline__ void bm_pair(uint32_t u0, uint32_t u1, RT& x, RT& y) {
    if (PREC == PREC_FP32) {
        float fx, fy;
        boxmuller32_f(u0, u1, fx, fy);
        x = (RT)fx;
        y = (RT)fy;
    } else {
        double dx, dy;
        boxmuller32_d(u0, u1, dx, dy);
        x = to_rt<RT>(dx);
        y = to_rt<RT>(dy);
    }
}

template <int PREC, class RT>
__device__ __forceinline__ RT u01_word(uint32_t w) {
    if (PREC == PREC_FP64) return (RT)__dadd_rn(__dmul_rn((double)w, 0x1p-32), 0x1p-33);
    return (RT)__fadd_rn(__fmul_rn(__uint2float_rn(w), 0x1p-32f), 0x1p-33f);
}

// normal k of an OUTER phase (used for the outer draws)
template <int PREC, class RT>
__device__ __forceinline__ RT outer_normal_at(const TfKey& key, uint32_t tag, uint64_t k) {
    uint64_t v0, v1;
    threefry2x64(k >> 2, tag, key, v0, v1);
    uint64_t e = ((k >> 1) & 1) ? v1 : v0;
    RT x, y;
    bm_pair<PREC, RT>((uint32_t)e, (uint32_t)(e >> 32), x, y);
    return (k & 1) ? y : x;
}

// ---- path-simulated inner values on the OUTER layout ----------------------------------------
// An Exact or Unbiased option (portfolio_sampler.cpp:470-604) drawn by inner sample i of the phase
// with tag t takes its draws from its own counter namespaces, so every inner sample stays
// addressable whatever the number of draws it makes: normals from counter word 1 =
// t | (i + 1) << 16 (normal k = component k & 1 of the Box-Muller pair of words 2(k >> 1),
// 2(k >> 1) + 1), uniforms (the Unbiased level) from t | (i + 1) << 16 | 2^15, word k.
constexpr uint64_t kPathUniform = 1ull << 15;
__device__ __forceinline__ uint64_t path_ns(uint32_t tag, uint64_t i) { return (uint64_t)tag | ((i + 1) << 16); }

template <class RT, int PREC>
struct OuterPathNormals {
    TfKey key;
    uint64_t ns;
    uint64_t p;          // next pair
    bool have;
    RT y;
    uint64_t v1;         // the block's second value (pairs 2b + 1)
    // positions the stream at normal k (the next next() returns normal k)
    __device__ __forceinline__ void seek(uint64_t k) {
        p = k >> 1;
        have = false;
        if (p & 1) {                                 // next() takes pair p from the cached v1
            uint64_t e0;
            threefry2x64(p >> 1, ns, key, e0, v1);
        }
        if (k & 1) (void)next();                     // normal k is the second of pair p
    }
    __device__ __forceinline__ RT next() {
        if (have) {
            have = false;
            return y;
        }
        uint64_t e;
        if (p & 1) {
            e = v1;                                  // the block was drawn with pair p - 1
        } else {
            threefry2x64(p >> 1, ns, key, e, v1);
        }
        RT x;
        bm_pair<PREC, RT>((uint32_t)e, (uint32_t)(e >> 32), x, y);
        p++;
        have = true;
        return x;
    }
};

// ---- portfolio inner value (BS path of portfolio::sampler) ----------------------------------
// sample_inner_bs with option_diff_from_blackscholes and the delta CV (portfolio_sampler.cpp:
// 453-468, 186-200, 202-210) in the reference's arithmetic (REF32 / FP64 tables).
// R_tau rows of the batched path: per outer sample and stock, R alone (the reference-arithmetic
// precisions) or the pair (R, ln R) on the FP32 path, whose Black-Scholes needs ln R and takes it
// from the row instead of a logarithm per inner sample.
template <int PREC> struct RStride { static constexpr uint32_t v = PREC == PREC_FP32 ? 2 : 1; };

template <class RT, uint32_t RS>
__device__ __forceinline__ RT pf_value(const OptionTable<RT>& ot, const RT* Rrow, uint32_t j) {
    uint32_t s = ot.stock_ind[j];
    int type = ot.type[j];
    RT sigma = ot.sigma[s];
    const RT R = Rrow[s * RS];
    RT bs = calc_bs_ref<RT>(type, R, ot.strike[j], ot.r, xsub(ot.maturity[j], ot.tau), sigma);
    RT finish = ot.discount ? xmul(xexp(xmul(-ot.r, ot.tau)), bs) : bs;
    RT val = xmul(ot.w[j], xsub(ot.start[j], finish));
    if (ot.use_delta_cv) {
        RT derv = xmul(ot.w[j], calc_delta_ref<RT>(type, ot.S0[s], ot.strike[j], ot.r, ot.maturity[j], sigma));
        val = xadd(val, xmul(xsub(R, ot.S0[s]), derv));
    }
    return val;
}

// Option index of one inner sample from one 64-bit value of the OUTER layout (the draw of
// sample_inner_random_option_ind, 346-370, with its own addressing): column j = floor(v P / 2^64),
// exact in every precision.  Uniform sub-sampling takes j (prob 1 / P); importance sub-sampling
// (Subsampling::Random) flips the column's alias coin (v P mod 2^64) >> 32 — O(1) instead of the
// reference's CDF binary search, the distribution of the table's exact masses phat.
// j and the coin from two 32 x 32 -> 64-bit products (P < 2^32): v P = 2^32 (v_hi P + (v_lo P >> 32))
// + (v_lo P mod 2^32), and the bracket stays below 2^64.
__device__ __forceinline__ void draw_column(uint64_t v, uint32_t P, uint32_t& j, uint32_t& coin) {
    const uint64_t lo = (uint64_t)(uint32_t)v * P;
    const uint64_t hi = (uint64_t)(uint32_t)(v >> 32) * P + (lo >> 32);
    j = (uint32_t)(hi >> 32);
    coin = (uint32_t)hi;
}

__device__ __forceinline__ uint32_t pf_index(const uint2* alias, uint32_t P, uint64_t v) {
    uint32_t j, coin;
    draw_column(v, P, j, coin);
    if (!alias) return j;
    const uint2 e = alias[j];
    return coin < e.x ? j : e.y;
}

// The sub-sampled option index and its sampling probability (sample_inner_random_option_ind,
// portfolio_sampler.cpp:346-370, on the OUTER layout's draws).
template <class RT>
__device__ __forceinline__ uint32_t pf_pick(const OptionTable<RT>& ot, uint64_t v, RT& prob) {
    const uint32_t j = pf_index(ot.subsample == SUB_UNIFORM ? nullptr : ot.alias, ot.P, v);
    prob = ot.subsample == SUB_UNIFORM ? ot.inv_count_prob : ot.phat[j];
    return j;
}

// Table gathers of the FP32 portfolio path.  Every inner sample reads a random entry of the
// option tables (alias entry, record or alias column; L2-resident, 8 to 32 bytes each), so a warp
// load touches ~32 cache lines and the L1's tag stage, about one line per clock per SM, is the
// path's throughput limit.  The gathers are single requests per lane (a record or column in one
// 256-bit load, ld.global.v8 on sm_100) that bypass L1 allocation (L1::no_allocate).
__device__ __forceinline__ uint2 load_alias(const uint2* p) {
    uint2 e;
    asm("ld.global.nc.L1::no_allocate.v2.u32 {%0,%1}, [%2];" : "=r"(e.x), "=r"(e.y) : "l"(p));
    return e;
}
__device__ __forceinline__ FastOption load_record(const FastOption* p) {
    FastOption o;
    float st;
    asm("ld.global.nc.L1::no_allocate.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=f"(o.c1), "=f"(o.inv_s), "=f"(o.s), "=f"(o.wR), "=f"(o.wK), "=f"(o.wV0), "=f"(o.cv), "=f"(st)
        : "l"(p));
    o.stock = __float_as_uint(st);
    return o;
}
// The same record through L1: uniform draws from a table of at most kL1TableBytes (1 MB), which
// stays largely resident in the SMs' L1 (7 % faster on the 10^4-option portfolio than L2 reads).
__device__ __forceinline__ FastOption load_record_l1(const FastOption* p) {
    FastOption o;
    float st;
    asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=f"(o.c1), "=f"(o.inv_s), "=f"(o.s), "=f"(o.wR), "=f"(o.wK), "=f"(o.wV0), "=f"(o.cv), "=f"(st)
        : "l"(p));
    o.stock = __float_as_uint(st);
    return o;
}
__device__ __forceinline__ FastColumn load_column(const FastColumn* p) {
    FastColumn c;
    float thr, link;
    asm("ld.global.nc.L1::no_allocate.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=f"(c.c1), "=f"(c.inv_s), "=f"(c.wR), "=f"(c.wK), "=f"(c.wV0), "=f"(c.cv), "=f"(thr), "=f"(link)
        : "l"(p));
    c.thr = __float_as_uint(thr);
    c.link = __float_as_uint(link);
    return c;
}

// How the FP32 portfolio path draws an option: uniformly (records), from the alias table
// (alias entry, then record) or from the alias columns (column, and the alias column when the coin
// says so).
// PF_COLUMN_PIPE: the alias columns with the next four samples' gathers issued before the current
// four are evaluated (the 128-register variant).
enum PfMode : int { PF_UNIFORM = 0, PF_ALIAS = 1, PF_COLUMN = 2, PF_COLUMN_PIPE = 3, PF_UNIFORM_L1 = 4 };
constexpr uint64_t kL1TableBytes = 1ull << 20;   // uniform draws from tables up to 1 MB read through L1

// Loss of the option drawn by the 64-bit value v: column j = floor(v P / 2^64), alias coin
// (v P mod 2^64) >> 32, the option kept when coin < threshold and its alias otherwise (the same
// option in every mode); Rrow holds (R, ln R) per stock of this outer sample.
template <int MODE>
__device__ __forceinline__ float pf_sample_loss(uint64_t v, const OptionTable<float>& ot, const float2* Rrow) {
    uint32_t j, coin;
    draw_column(v, ot.P, j, coin);
    if (MODE == PF_COLUMN) {
        FastColumn c = load_column(ot.fast_col + j);
        if (coin >= c.thr) c = load_column(ot.fast_col + (c.link >> 8));
        const float2 r = Rrow[c.link & 0xffu];
        return column_loss_fast(c, r.x, r.y);
    }
    uint32_t i = j;
    if (MODE == PF_ALIAS) {
        const uint2 e = load_alias(ot.alias + j);
        i = coin < e.x ? j : e.y;
    }
    const FastOption o = MODE == PF_UNIFORM_L1 ? load_record_l1(ot.fast_s + i) : load_record(ot.fast_s + i);
    const float2 r = Rrow[o.stock];
    return option_loss_fast(o, r.x, r.y);
}

// Four samples of the alias-column path: the Threefry blocks blk, blk + 1 and the four column
// gathers they select (issued together, not waited for).
__device__ __forceinline__ void column_issue(const TfKey& key, uint32_t tag, uint64_t blk, const OptionTable<float>& ot,
                                             FastColumn (&c)[4], uint32_t (&coin)[4]) {
    uint64_t v[4];
    threefry2x64(blk, tag, key, v[0], v[1]);
    threefry2x64(blk + 1, tag, key, v[2], v[3]);
#pragma unroll
    for (int q = 0; q < 4; q++) {
        uint32_t j;
        draw_column(v[q], ot.P, j, coin[q]);
        c[q] = load_column(ot.fast_col + j);
    }
}

// The rest of those four samples: the alias-column gathers of the draws whose coin asks for them,
// then the four losses, added to the sums in sample order (pairs into the compensated sum).
template <int PREC, bool S2>
__device__ __forceinline__ void column_finish(FastColumn (&c)[4], const uint32_t (&coin)[4], const OptionTable<float>& ot,
                                              const float2* Rrow, float shift, Acc<PREC>& a1, Acc<PREC>& a2) {
#pragma unroll
    for (int q = 0; q < 4; q++)
        if (coin[q] >= c[q].thr) c[q] = load_column(ot.fast_col + (c[q].link >> 8));
    float x[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const float2 r = Rrow[c[q].link & 0xffu];
        x[q] = column_loss_fast(c[q], r.x, r.y);
        if (S2) { x[q] += shift; a2.add_sq(x[q]); }
    }
    a1.add2(x[0], x[1]);
    a1.add2(x[2], x[3]);
}

// C inner samples of the FP32 portfolio path from Threefry blocks b0, b0 + 1, ... (two samples per
// block, one 64-bit value each, added to the compensated sum as a pair).  Pilots (S2) accumulate
// the losses shifted by `shift`.  With alias columns the loop takes two blocks (four samples) at a
// time and issues their four column gathers together, then the alias-column gathers of the draws
// that need them, so a thread has four samples' L2 round trips in flight at once (4 % faster than
// two at a time, spills included).  PF_COLUMN_PIPE keeps two such groups, A and B: B's blocks and
// column gathers are issued before A's alias gathers and losses, so B's round trip runs while A is
// evaluated.  Every mode adds the samples to the sums in the same order.
template <int PREC, uint32_t C, bool S2, int MODE>
__device__ __forceinline__ void pf_chunk_fast(const TfKey& key, uint32_t tag, uint64_t b0,
                                              const OptionTable<float>& ot, const float2* Rrow, float shift,
                                              Acc<PREC>& a1, Acc<PREC>& a2) {
    if constexpr (MODE == PF_COLUMN) {
#pragma unroll 1
        for (uint32_t b = 0; b < C / 2; b += 2) {
            FastColumn c[4];
            uint32_t coin[4];
            column_issue(key, tag, b0 + b, ot, c, coin);
            column_finish<PREC, S2>(c, coin, ot, Rrow, shift, a1, a2);
        }
    } else if constexpr (MODE == PF_COLUMN_PIPE) {
        constexpr uint32_t G = C / 4;           // groups of four samples
        FastColumn ca[4], cb[4];
        uint32_t ka[4], kb[4];
        column_issue(key, tag, b0, ot, ca, ka);
#pragma unroll 1
        for (uint32_t g = 0; g < G; g += 2) {
            if (g + 1 < G) column_issue(key, tag, b0 + 2 * (g + 1), ot, cb, kb);
            column_finish<PREC, S2>(ca, ka, ot, Rrow, shift, a1, a2);
            if (g + 1 < G) {
                if (g + 2 < G) column_issue(key, tag, b0 + 2 * (g + 2), ot, ca, ka);
                column_finish<PREC, S2>(cb, kb, ot, Rrow, shift, a1, a2);
            }
        }
    } else {
#pragma unroll 2
        for (uint32_t b = 0; b < C / 2; b++) {
            uint64_t v[2];
            threefry2x64(b0 + b, tag, key, v[0], v[1]);
            float x[2];
#pragma unroll
            for (int q = 0; q < 2; q++) {
                x[q] = pf_sample_loss<MODE>(v[q], ot, Rrow);
                if (S2) { x[q] += shift; a2.add_sq(x[q]); }
            }
            a1.add2(x[0], x[1]);
        }
    }
}

// R_tau rows staged in shared memory: segments whose tiles hold at most kRowItems outer samples
// (every segment with 32 or more chunks per outer sample, where nearly all inner samples of a
// level are) read R and ln R from shared memory, which takes the per-sample row lookups off the L1
// tag stage.  kMaxStagedStocks bounds the dynamic shared memory (kRowItems x Q float2 = 16 KB).
constexpr uint32_t kRowItems = 8;
constexpr uint32_t kMaxStagedStocks = 256;
constexpr size_t kRowSmemBytes = (size_t)kRowItems * kMaxStagedStocks * sizeof(float2);

// Copies the rows of the outer samples lin0 .. lin0 + n - 1 of a segment into dst (n rows of Q).
__device__ __forceinline__ void stage_rows(const float2* Rt, uint32_t Q, const uint32_t* list, uint64_t lin0,
                                           uint32_t n, uint32_t n_items, float2* dst) {
    for (uint32_t k = threadIdx.x; k < n * Q; k += blockDim.x) {
        const uint32_t r = k / Q, q = k - r * Q;
        const uint64_t lin = lin0 + r;
        if (lin < n_items) {
            const uint32_t item = list ? list[lin] : (uint32_t)lin;
            dst[k] = Rt[(size_t)item * Q + q];
        }
    }
}

// ---- sampler kinds -------------------------------------------------------------------------
// KIND_USER runs a caller-written SAMPLER class (the reference's SAMPLER concept, nested_sampler.hpp:
// 36-85 and model_sampler.cpp:42-92, on the OUTER streams; include/nmlmc_sampler.cuh): its
// sample_outer, init_inner_sampler, sample_inner and add_phi replace the built-in kinds' code, and
// the batched machinery below is the same.  S is that class (NoSampler for the built-in kinds).
struct NoSampler {};

// The phi contribution coeff * phi(mean) of one inner mean (add_phi): the Indicator phi of the
// built-in kinds (model_sampler.cpp:77-86), or the SAMPLER's own add_phi.
template <int KIND, class S, class RT>
__device__ __forceinline__ float phi_of(RT mean, float coeff) {
    if constexpr (KIND == KIND_USER) {
        RT p = 0;
        S::add_phi(mean, (RT)coeff, &p);
        return (float)p;
    } else {
        return mean >= (RT)0 ? coeff : 0.f;
    }
}

// SAMPLER objects of KIND_USER: the one of outer sample `item` (its outer state, stored by
// k_outer) and its workspace (OuterBuffers::user_ws, ws_bytes per outer sample).
template <class S>
__device__ __forceinline__ const S* user_state(const OuterBuffers& B, uint32_t item) {
    return reinterpret_cast<const S*>(static_cast<const unsigned char*>(B.user_state) + (size_t)item * B.state_bytes);
}
__device__ __forceinline__ void* user_ws(const OuterBuffers& B, uint32_t item) {
    return B.ws_bytes ? static_cast<unsigned char*>(B.user_ws) + (size_t)item * B.ws_bytes : nullptr;
}

// ---- one chunk: inner samples [s0, s0 + C) of phase `tag` of outer sample `item` ----------
// The chunk's share of sample_inner's sums (nested_sampler.hpp:131-161; model::sampler::
// sample_inner, model_sampler.cpp:66-79, or the portfolio's inner value above).
// C (inner samples per chunk) is a compile-time constant so the independent Threefry blocks of a
// chunk can be interleaved (two at a time) for instruction-level parallelism.
// ---- path-simulated portfolio, FP32 -------------------------------------------------------
// Steps N_l = beta^L of an Unbiased level (false when h0 N_l exceeds kMaxPathSteps).
__device__ __forceinline__ bool level_steps(const OptionTable<float>& ot, uint32_t Lv, uint64_t& N_l) {
    N_l = 1;
    bool ok = true;
    for (uint32_t i = 0; i < Lv && ok; i++) {
        N_l *= ot.dt_beta;
        ok = N_l * ot.dt_h0inv <= kMaxPathSteps;
    }
    return ok && N_l * ot.dt_h0inv <= kMaxPathSteps;
}

// The Unbiased level of the inner sample with path namespace ns, drawn in double as the FP64 path
// draws it (sample_inner_unbiased, portfolio_sampler.cpp:521-537), and its steps.
__device__ __forceinline__ bool level_fp32(const OptionTable<float>& ot, const TfKey& key, uint64_t ns,
                                           uint32_t& Lv, uint64_t& N_l) {
    uint64_t u0, u1;
    threefry2x64(0, ns | kPathUniform, key, u0, u1);
    const double u = __dadd_rn(__dmul_rn((double)(uint32_t)u0, 0x1p-32), 0x1p-33);
    const double qL = log(u) / (log((double)ot.dt_beta) * (double)ot.dt_prob_expo);
    Lv = (uint32_t)floor(qL);
    return level_steps(ot, Lv, N_l);
}

// Inner samples of a chunk of at most kPathSortChunk per thread are evaluated in the order of
// their cost class (0 Black-Scholes, 1 Exact, 2 + L for an Unbiased option at level L <= 12, 15
// beyond), each thread its own order: the Unbiased level makes a sample's cost vary by powers of
// beta, and in sample order every step of a warp waits for the longest path among its 32 lanes
// (about 8x the mean at beta = 2, P(L) ~ 2^(-1.5 L)).  A first pass draws every sample's option
// and level and keeps the option index and class in shared memory (5 bytes per sample and
// thread); the second evaluates them cheapest class first.  The sums receive the same values in
// another order.
constexpr uint32_t kPathSortChunk = 32;
constexpr size_t kPathSortSmemBytes = (size_t)kPathSortChunk * kTile * (sizeof(uint32_t) + 1);

// Unbiased samples at levels >= kCoopLevel (and those whose level is recomputed) are evaluated by
// the whole warp, one at a time: the fine and coarse paths of the Milstein / Euler scheme are
// products of per-step growth factors S_N = S_0 prod (1 + inc_n), so each lane multiplies the
// factors of a contiguous range of coarse steps (drawing its normals at their stream positions)
// and a butterfly product combines the lanes.  The same values as the sequential stepper up to
// the order of the double products.  Rare (0.55 % of the samples at beta = 2, P(L) ~ 2^(-1.5 L)),
// these samples carried about a fifth of the steps and, evaluated by one lane, kept the other 31
// lanes of the warp and the other warps of the CTA waiting at the tile's barrier.
constexpr uint32_t kCoopLevel = 5;

// loss * weight of an Unbiased sample (inner_unbiased_fast) evaluated by all 32 lanes of the warp;
// every lane returns the value, `work` is the owner's to add.
__device__ __forceinline__ float inner_unbiased_coop(const OptionTable<float>& ot, float Rs, uint32_t j,
                                                     const TfKey& key, uint64_t ns, uint32_t L, uint64_t N_l,
                                                     uint32_t lane) {
    const uint32_t s = ot.stock_ind[j];
    const float S0 = ot.S0[s], sg = ot.sigma[s], r = ot.r, tau = ot.tau, T = ot.maturity[j], K = ot.strike[j];
    const float m = (float)ot.type[j], wdisc = ot.w[j] * __expf(-r * T);
    const float mu_t = (r - 0.5f * sg * sg) * tau;
    OuterPathNormals<float, PREC_FP32> nz{key, ns, 0, false, 0.f, 0};
    const float dW0 = ot.stau * nz.next();
    const float S0_t_1 = S0 * __expf(fmaf(sg, dW0, mu_t));
    const float S0_t_2 = S0 * __expf(fmaf(-sg, dW0, mu_t));
    const uint64_t N = (uint64_t)ot.dt_h0inv * N_l;
    const uint32_t cs = ot.dt_beta;                          // fine steps per coarse step (L > 0)
    const uint64_t Nc = N / cs;
    const float Tr = T - tau;
    const float dt = Tr / (float)N, sqrt_dt = sqrtf(dt), dt_c = dt * (float)cs;
    const float hs2 = ot.use_milstein ? 0.5f * sg * sg : 0.f;
    // this lane's coarse steps [c0, c1): fine steps c0 cs .. c1 cs - 1, normals 1 + n
    const uint64_t c0 = Nc * lane / 32, c1 = Nc * (lane + 1) / 32;
    double Ff = 1.0, Fc = 1.0;
    if (c1 > c0) {
        nz.seek(1 + c0 * cs);
        for (uint64_t c = c0; c < c1; c++) {
            float dW_c = 0.f;
            for (uint32_t i = 0; i < cs; i++) {
                const float dW = sqrt_dt * nz.next();
                const double inc = (double)fmaf(hs2, fmaf(dW, dW, -dt), fmaf(sg, dW, r * dt));
                Ff = fma(Ff, inc, Ff);
                dW_c += dW;
            }
            const double incc = (double)fmaf(hs2, fmaf(dW_c, dW_c, -dt_c), fmaf(sg, dW_c, r * dt_c));
            Fc = fma(Fc, incc, Fc);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        Ff *= __shfl_xor_sync(0xffffffffu, Ff, o);
        Fc *= __shfl_xor_sync(0xffffffffu, Fc, o);
    }
    const double S[6] = {(double)S0_t_1 * Ff, (double)Rs * Ff, (double)S0_t_2 * Ff,
                         (double)S0_t_1 * Fc, (double)Rs * Fc, (double)S0_t_2 * Fc};
    const bool anti = ot.use_antithetic_risk != 0;
    const float half = anti ? 0.5f : 1.f;
    const float diff = Rs - S0;
    const bool do_d_f = ot.use_delta_cv && ot.use_coarse_delta_cv;   // L > 0
    const bool do_d_c = ot.use_delta_cv && ot.use_coarse_delta_cv;
    float vf = 0.f, vc = 0.f, vdf = 0.f, vdc = 0.f;
#pragma unroll
    for (int i = 0; i < 2; i++) {
        if (i == 1 && !anti) break;
        const int ic = 2 * i;
        vf += half * opt_diff_stock_fast(wdisc, m, K, (float)S[ic], (float)S[1]);
        if (do_d_f) vdf += half * opt_derv_stock_fast(wdisc, m > 0.f, K, (float)S[ic], S0);
        vc += half * opt_diff_stock_fast(wdisc, m, K, (float)S[ic + 3], (float)S[4]);
        if (do_d_c) vdc += half * opt_derv_stock_fast(wdisc, m > 0.f, K, (float)S[ic + 3], S0);
    }
    const float ret = (vf - vc) + diff * (vdf - vdc);
    const float e = ot.dt_prob_expo, lb = __log2f((float)ot.dt_beta);
    return ret * (exp2f(-e * lb * (float)L) / (1.0f - exp2f(e * lb)));
}

// `own`: this lane evaluates a chunk (lanes past the end of a segment's last tile take part in
// the warp's cooperative samples only).  All 32 lanes of the warp call it together.
template <uint32_t C, bool S2, int PREC>
__device__ __forceinline__ void pf_paths_sorted(const DevLevel<float>& D, const TfKey& key, uint32_t tag, uint64_t s0,
                                                const float* Rrow, float shift, Acc<PREC>& a1, Acc<PREC>& a2,
                                                double& work, bool own) {
    static_assert(C <= kPathSortChunk, "sorted path chunk");
    extern __shared__ float2 k_phase_rows[];     // the phase kernel's dynamic shared memory
    const OptionTable<float>& ot = D.L.ot;
    uint32_t* jbuf = reinterpret_cast<uint32_t*>(k_phase_rows) + threadIdx.x;                 // [q * kTile]
    uint8_t* cbuf = reinterpret_cast<uint8_t*>(reinterpret_cast<uint32_t*>(k_phase_rows) + kPathSortChunk * kTile) +
                    threadIdx.x;
    // pass 1: option, class; the samples of classes {0, 1, 2}, 3, 4, 5, 6 (levels 1-4) as bit
    // sets, and those the warp evaluates together (levels >= kCoopLevel, class 15)
    static_assert(kCoopLevel >= 1 && kCoopLevel <= 5, "class sets");
    uint32_t m0 = 0, m1 = 0, m2 = 0, m3 = 0, m4 = 0, m5 = 0;
#pragma unroll 1
    for (uint32_t b = 0; b < (own ? C / 2 : 0u); b++) {
        uint64_t v[2];
        threefry2x64((s0 >> 1) + b, tag, key, v[0], v[1]);
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const uint32_t q = 2 * b + h;
            float prob;
            const uint32_t j = pf_pick<float>(ot, v[h], prob);
            uint32_t c = 0;
            if (j >= ot.m_off[1]) {
                if (j < ot.m_off[2]) {
                    c = 1;
                } else {
                    uint32_t Lv;
                    uint64_t N_l;
                    const bool ok = level_fp32(ot, key, path_ns(tag, s0 + q), Lv, N_l);
                    c = (ok && Lv <= 12) ? 2 + Lv : 15u;
                }
            }
            jbuf[q * kTile] = j;
            cbuf[q * kTile] = (uint8_t)c;
            const uint32_t bit = 1u << q;
            if (c >= 2 + kCoopLevel) m5 |= bit;
            else if (c <= 2) m0 |= bit;
            else if (c == 3) m1 |= bit;
            else if (c == 4) m2 |= bit;
            else if (c == 5) m3 |= bit;
            else if (c == 6) m4 |= bit;
            else m5 |= bit;
        }
    }
    // pass 2: cheapest class first, sample order within a set; each lane its own samples
#pragma unroll 1
    for (;;) {
        const bool has = (m0 | m1 | m2 | m3 | m4) != 0;
        if (!__any_sync(0xffffffffu, has)) break;
        if (!has) continue;
        uint32_t q;
        if (m0) { q = __ffs(m0) - 1; m0 &= m0 - 1; }
        else if (m1) { q = __ffs(m1) - 1; m1 &= m1 - 1; }
        else if (m2) { q = __ffs(m2) - 1; m2 &= m2 - 1; }
        else if (m3) { q = __ffs(m3) - 1; m3 &= m3 - 1; }
        else { q = __ffs(m4) - 1; m4 &= m4 - 1; }
        const uint32_t j = jbuf[q * kTile];
        const uint32_t c = cbuf[q * kTile];
        const float prob = ot.subsample == SUB_UNIFORM ? ot.inv_count_prob : ot.phat[j];
        float val;
        if (c == 0) {
            val = pf_value<float, 2>(ot, Rrow, j);
            work += (double)ot.W_est[j];
        } else {
            const uint64_t ns = path_ns(tag, s0 + q);
            OuterPathNormals<float, PREC_FP32> nz{key, ns, 0, false, 0.f, 0};
            const float Rs = Rrow[ot.stock_ind[j] * 2];
            if (c == 1) {
                val = inner_exact_fast(ot, Rs, j, nz, work);
            } else {
                uint32_t Lv;
                uint64_t N_l;
                bool ok;
                if (c < 15) { Lv = c - 2; ok = level_steps(ot, Lv, N_l); }
                else ok = level_fp32(ot, key, ns, Lv, N_l);
                if (ok) {
                    val = inner_unbiased_fast(ot, Rs, j, nz, work, Lv, N_l);
                } else {                         // beyond kMaxPathSteps: the call fails
                    atomicOr(D.B.counters + CNT_ERR, 1u);
                    val = 0.f;
                }
            }
        }
        float d = __fdiv_rn(val, prob);
        if (S2) d = __fadd_rn(d, shift);
        a1.add(d);
        if (S2) a2.add_sq(d);
    }
    // pass 3: the deep samples of all lanes, one at a time by the whole warp (its owner first by
    // lane, then in sample order); the lanes read each other's pass-1 entries after the warp
    // barrier orders them
    __syncwarp();
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t* jcol = reinterpret_cast<const uint32_t*>(k_phase_rows) + (threadIdx.x & ~31u);
    const uint8_t* ccol = reinterpret_cast<const uint8_t*>(reinterpret_cast<const uint32_t*>(k_phase_rows) +
                                                           kPathSortChunk * kTile) + (threadIdx.x & ~31u);
#pragma unroll 1
    for (;;) {
        const unsigned pend = __ballot_sync(0xffffffffu, m5 != 0);
        if (!pend) break;
        const uint32_t src = __ffs(pend) - 1;
        uint32_t myq = 0;
        if (lane == src) { myq = __ffs(m5) - 1; m5 &= m5 - 1; }
        const uint32_t q = __shfl_sync(0xffffffffu, myq, src);
        const uint32_t j = jcol[q * kTile + src];
        const uint32_t c = ccol[q * kTile + src];
        const TfKey skey{__shfl_sync(0xffffffffu, key.k0, src), __shfl_sync(0xffffffffu, key.k1, src),
                         __shfl_sync(0xffffffffu, key.k2, src)};
        const uint64_t ns = path_ns(tag, __shfl_sync(0xffffffffu, s0, src) + q);
        const float Rs = __shfl_sync(0xffffffffu, lane == src ? Rrow[ot.stock_ind[j] * 2] : 0.f, src);
        uint32_t Lv;
        uint64_t N_l;
        bool ok;
        if (c < 15) { Lv = c - 2; ok = level_steps(ot, Lv, N_l); }
        else ok = level_fp32(ot, skey, ns, Lv, N_l);
        float val = 0.f;
        if (ok) val = inner_unbiased_coop(ot, Rs, j, skey, ns, Lv, N_l, lane);
        if (lane == src) {
            if (ok) {
                const float West = ot.W_est[j];
                work += (double)((float)N_l * West);
                work += (double)((float)(N_l / ot.dt_beta) * West);
            } else {                                     // beyond kMaxPathSteps: the call fails
                atomicOr(D.B.counters + CNT_ERR, 1u);
            }
            const float prob = ot.subsample == SUB_UNIFORM ? ot.inv_count_prob : ot.phat[j];
            float d = __fdiv_rn(val, prob);
            if (S2) d = __fadd_rn(d, shift);
            a1.add(d);
            if (S2) a2.add_sq(d);
        }
    }
}

template <class RT, int KIND, int PREC, uint32_t C, bool S2, class S, bool PIPE>
__device__ __forceinline__ void eval_chunk_c(const DevLevel<RT>& D, uint32_t item, uint32_t tag,
                                             uint64_t s0, uint64_t count, float shift, const float2* srow,
                                             Acc<PREC>& a1, Acc<PREC>& a2, double& work, bool own) {
    if (!own && !(KIND == KIND_PF_PATHS && PREC == PREC_FP32 && C <= kPathSortChunk)) return;
    const OuterLevel<RT>& L = D.L;
    const TfKey key = tf_key(L.seed, outer_stream_id(L.ell, L.first_index + item));
    const RT* Yv = reinterpret_cast<const RT*>(D.B.Yv);
    if constexpr (KIND == KIND_USER) {           // the caller's SAMPLER (sample_inner)
        S smp(user_ws(D.B, item));
        smp.copy_outer(*user_state<S>(D.B, item));
        double w = 0;
        for (uint32_t q = 0; q < C; q += 2) {
            RT d[2];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                smp.template nm_begin_inner_of<S>(key, tag, s0 + q + h);
                d[h] = smp.sample_inner(s0 + q + h, count, w);
                if (PREC == PREC_FP32 && S2) d[h] = (RT)((float)d[h] + shift);
                if (S2) { if (PREC == PREC_FP32) a2.add_sq(d[h]); else a2.add(d[h] * d[h]); }
            }
            a1.add2(d[0], d[1]);
        }
        work += w;
    } else if (KIND == KIND_SHIFT_MODEL) {       // X = Y + Z: one normal per inner sample
        const RT Y = Yv[item];
#pragma unroll 2
        for (uint32_t b = 0; b < C / 4; b++) {
            uint64_t v0, v1;
            threefry2x64((s0 >> 2) + b, tag, key, v0, v1);
            RT z[4];
            bm_pair<PREC, RT>((uint32_t)v0, (uint32_t)(v0 >> 32), z[0], z[1]);
            bm_pair<PREC, RT>((uint32_t)v1, (uint32_t)(v1 >> 32), z[2], z[3]);
#pragma unroll
            for (int q = 0; q < 4; q++) {
                RT d = (PREC == PREC_FP32) ? (RT)(Y + z[q]) : xadd(Y, z[q]);
                if (PREC == PREC_FP32 && S2) d = (RT)((float)d + shift);
                z[q] = d;
                if (S2) { if (PREC == PREC_FP32) a2.add_sq(d); else a2.add(xmul(d, d)); }
            }
            a1.add2(z[0], z[1]);
            a1.add2(z[2], z[3]);
        }
        work += (double)C;
    } else if (KIND == KIND_REF_MODEL) {         // model_sampler.cpp:62-76: two normals
        const RT Y = Yv[item];
        const RT st = L.mp.stau, s1t = L.mp.s1tau;
#pragma unroll 2
        for (uint32_t b = 0; b < C / 2; b++) {   // one block = two inner samples
            uint64_t v0, v1;
            threefry2x64((s0 >> 1) + b, tag, key, v0, v1);
            RT X[2], Y2[2];
            bm_pair<PREC, RT>((uint32_t)v0, (uint32_t)(v0 >> 32), X[0], Y2[0]);
            bm_pair<PREC, RT>((uint32_t)v1, (uint32_t)(v1 >> 32), X[1], Y2[1]);
#pragma unroll
            for (int q = 0; q < 2; q++) {
                RT a = xadd(xmul(st, Y), xmul(s1t, X[q]));
                RT c = xadd(xmul(st, Y2[q]), xmul(s1t, X[q]));
                RT d = xsub(xmul(a, a), xmul(c, c));
                if (PREC == PREC_FP32 && S2) d = (RT)((float)d + shift);
                X[q] = d;
                if (S2) { if (PREC == PREC_FP32) a2.add_sq(d); else a2.add(xmul(d, d)); }
            }
            a1.add2(X[0], X[1]);
        }
        work += (double)C;
    } else if (KIND == KIND_PORTFOLIO && PREC == PREC_FP32 && L.ot.fast_s) {
        // portfolio, FP32: packed records scaled by 1 / (sampling probability), the SFU
        // Black-Scholes (nmlmc_bs.cuh); X = loss_j / phat_j.  srow: the outer sample's R_tau row
        // staged in shared memory, else read from the batch buffer.
        if constexpr (sizeof(RT) == 4) {
            const OptionTable<float>& ot = L.ot;
            const float2* grow = reinterpret_cast<const float2*>(D.B.Rt) + (size_t)item * ot.Q;
            const uint64_t b0 = s0 >> 1;
            if (ot.fast_col) {
                constexpr int CM = PIPE ? PF_COLUMN_PIPE : PF_COLUMN;
                if (srow) pf_chunk_fast<PREC, C, S2, CM>(key, tag, b0, ot, srow, shift, a1, a2);
                else pf_chunk_fast<PREC, C, S2, CM>(key, tag, b0, ot, grow, shift, a1, a2);
            } else if (ot.subsample == SUB_UNIFORM && (uint64_t)ot.P * sizeof(FastOption) <= kL1TableBytes) {
                if (srow) pf_chunk_fast<PREC, C, S2, PF_UNIFORM_L1>(key, tag, b0, ot, srow, shift, a1, a2);
                else pf_chunk_fast<PREC, C, S2, PF_UNIFORM_L1>(key, tag, b0, ot, grow, shift, a1, a2);
            } else if (ot.subsample == SUB_UNIFORM) {
                if (srow) pf_chunk_fast<PREC, C, S2, PF_UNIFORM>(key, tag, b0, ot, srow, shift, a1, a2);
                else pf_chunk_fast<PREC, C, S2, PF_UNIFORM>(key, tag, b0, ot, grow, shift, a1, a2);
            } else {
                if (srow) pf_chunk_fast<PREC, C, S2, PF_ALIAS>(key, tag, b0, ot, srow, shift, a1, a2);
                else pf_chunk_fast<PREC, C, S2, PF_ALIAS>(key, tag, b0, ot, grow, shift, a1, a2);
            }
        }
        work += (double)C;
    } else if constexpr (KIND == KIND_PF_PATHS && PREC == PREC_FP32 && C <= kPathSortChunk) {
        if constexpr (sizeof(RT) == 4) {
            const float* Rrow = reinterpret_cast<const float*>(D.B.Rt) + (size_t)item * L.ot.Q * 2;
            pf_paths_sorted<C, S2, PREC>(D, key, tag, s0, Rrow, shift, a1, a2, work, own);
        }
    } else {                                     // portfolio: one 64-bit value per inner sample
        const OptionTable<RT>& ot = L.ot;
        constexpr uint32_t RS = RStride<PREC>::v;
        const RT* Rrow = reinterpret_cast<const RT*>(D.B.Rt) + (size_t)item * ot.Q * RS;
#pragma unroll 2
        for (uint32_t b = 0; b < C / 2; b++) {
            uint64_t v[2];
            threefry2x64((s0 >> 1) + b, tag, key, v[0], v[1]);
#pragma unroll
            for (int q = 0; q < 2; q++) {
                RT prob;
                uint32_t j = pf_pick<RT>(ot, v[q], prob);
                RT val;
                if (KIND == KIND_PF_PATHS && j >= ot.m_off[1]) {
                    // Exact / Unbiased option (sample_inner_option, portfolio_sampler.cpp:382-396)
                    const uint64_t ns = path_ns(tag, s0 + 2 * b + q);
                    OuterPathNormals<RT, PREC> nz{key, ns, 0, false, (RT)0, 0};
                    const RT Rs = Rrow[ot.stock_ind[j] * RS];
                    if (j < ot.m_off[2]) {
                        if constexpr (PREC == PREC_FP32) val = inner_exact_fast(ot, Rs, j, nz, work);
                        else val = inner_exact<RT>(ot, Rs, j, nz, work);
                    } else {
                        uint64_t u0, u1;
                        threefry2x64(0, ns | kPathUniform, key, u0, u1);
                        uint32_t Lv;
                        uint64_t N_l;
                        bool ok;
                        if constexpr (PREC == PREC_FP32) {
                            ok = level_fp32(ot, key, ns, Lv, N_l);
                        } else {
                            ok = unbiased_level<RT>(ot, u01_word<PREC, RT>((uint32_t)u0), Lv, N_l);
                        }
                        if (ok) {
                            if constexpr (PREC == PREC_FP32) val = inner_unbiased_fast(ot, Rs, j, nz, work, Lv, N_l);
                            else val = inner_unbiased<RT>(ot, Rs, j, nz, work, Lv, N_l);
                        } else {                 // beyond kMaxPathSteps: the call fails
                            atomicOr(D.B.counters + CNT_ERR, 1u);
                            val = (RT)0;
                        }
                    }
                } else {
                    val = pf_value<RT, RS>(ot, Rrow, j);
                    work += (double)ot.W_est[j];
                }
                RT d = xdiv(val, prob);
                if (PREC == PREC_FP32 && S2) d = (RT)((float)d + shift);
                a1.add(d);
                if (S2) { if (PREC == PREC_FP32) a2.add_sq(d); else a2.add(xmul(d, d)); }
            }
        }
    }
}

template <class RT, int KIND, int PREC, bool S2, class S, bool PIPE>
__device__ __forceinline__ void eval_chunk_s(const DevLevel<RT>& D, uint32_t item, uint32_t tag,
                                             uint64_t s0, uint64_t count, uint32_t C, float shift,
                                             const float2* srow, Acc<PREC>& a1, Acc<PREC>& a2, double& work,
                                             bool own) {
    switch (C) {
    case 64: eval_chunk_c<RT, KIND, PREC, 64, S2, S, PIPE>(D, item, tag, s0, count, shift, srow, a1, a2, work, own); break;
    case 32: eval_chunk_c<RT, KIND, PREC, 32, S2, S, PIPE>(D, item, tag, s0, count, shift, srow, a1, a2, work, own); break;
    case 16: eval_chunk_c<RT, KIND, PREC, 16, S2, S, PIPE>(D, item, tag, s0, count, shift, srow, a1, a2, work, own); break;
    case 8: eval_chunk_c<RT, KIND, PREC, 8, S2, S, PIPE>(D, item, tag, s0, count, shift, srow, a1, a2, work, own); break;
    default: eval_chunk_c<RT, KIND, PREC, 4, S2, S, PIPE>(D, item, tag, s0, count, shift, srow, a1, a2, work, own); break;
    }
}

// want_s2 (pilots: the sum of squares for the variance) is resolved once per chunk, so the
// inner loop carries no per-sample test.  `count`: the segment's inner count per outer sample (the
// SAMPLER's sample_inner argument).  On the FP32 path a pilot accumulates the inner values
// shifted by the outer sample's start value (d + start, whose mean is the distance from the
// threshold that the adaptive rule compares with the spread), so the one-pass variance
// s2 - s1^2 / n does not cancel where the decision is close; the final phase accumulates d.
// `srow`: the outer sample's R_tau row in shared memory, or nullptr (FP32 portfolio path).
// PIPE: the pipelined alias-column loop (the 128-register variant of the phase kernel).
// own: this thread's chunk is real (false for threads past the end of a segment's last tile,
// which take part only in the warp-cooperative samples of the FP32 path-simulated kernel).
template <class RT, int KIND, int PREC, class S, bool PIPE>
__device__ __forceinline__ void eval_chunk(const DevLevel<RT>& D, uint32_t item, uint32_t tag,
                                           uint64_t s0, uint64_t count, uint32_t C, bool want_s2, RT start,
                                           const float2* srow, Acc<PREC>& a1, Acc<PREC>& a2, double& work,
                                           bool own = true) {
    if (want_s2) eval_chunk_s<RT, KIND, PREC, true, S, PIPE>(D, item, tag, s0, count, C, (float)start, srow, a1, a2, work, own);
    else eval_chunk_s<RT, KIND, PREC, false, S, PIPE>(D, item, tag, s0, count, C, 0.f, srow, a1, a2, work, own);
}

// ---- segments of uniform chunk count ------------------------------------------------------
struct Seg {
    const uint32_t* list;    // item ids; nullptr: identity 0..n-1
    uint32_t n_slot;         // counter slot with the item count (list != nullptr)
    uint32_t n_host;         // item count (list == nullptr)
    uint32_t nch_log2;       // chunks per item = 1 << nch_log2
    uint32_t tag;            // OUTER phase tag
    uint32_t mode;           // 0 fine pilot, 1 coarse pilot, 2 final
    uint32_t class_k;        // final: class index (list offset = items of lower classes)
    uint32_t next_slot;      // pilots: counter slot of the next round's list
    uint32_t* next_list;
    uint64_t count;          // inner samples per item in this segment
};

struct SegSet {
    int n;
    Seg s[kMaxSegs];
};

// Adaptive decision after a pilot of `cur` samples (get_samples_count, 240-273, with
// sample_inner_delta2, 120-129).  Writes the final count of a decided item; returns true when
// the item goes on to the next pilot round.
template <class RT, int PREC>
__device__ __forceinline__ bool pilot_decide(const DevLevel<RT>& D, const Seg& g, uint32_t item, RT start,
                                             const Acc<PREC>& a1, const Acc<PREC>& a2) {
    const OuterLevel<RT>& L = D.L;
    const CountParams& cp = (g.mode == 0) ? L.cf : L.cc;
    const uint64_t cur = g.count;
    bool done;
    if (PREC == PREC_FP32) {
        // the sums are of d + start (eval_chunk): their mean is the distance start + mean(d);
        // num = (n - 1) var, delta2 = dist^2 (n - 1) / num
        const float s1 = (float)a1.value(), s2 = (float)a2.value(), n = (float)cur;
        const float dist = div_count(s1, cur);
        const float num = __fsub_rn(s2, __fmul_rn(s1, dist));
        if (L.adaptive_r == (RT)2) {
            const float delta2 = __fdiv_rn(__fmul_rn(dist, dist), __fdiv_rn(num, n - 1.0f));
            done = __fdiv_rn((float)cp.tmp, delta2) <= n;
        } else {
            // newc = tmp delta2^(-r/2) <= cur compared in base-2 logarithms on the SFU: no pow and
            // no division (a decision moves only within ~1e-5 relative of its threshold).  The
            // degenerate sums decide as the power form does: delta2 = 0 (dist = 0) continues,
            // delta2 = inf (num = 0) stops, a negative or 0/0 delta2 (NaN) continues.
            const float l2d = fmaf(2.0f, __log2f(fabsf(dist)), __log2f(n - 1.0f) - __log2f(num));
            done = fmaf(-0.5f * (float)L.adaptive_r, l2d, __log2f((float)cp.tmp)) <= __log2f(n);
        }
    } else {
        double s1 = (double)a1.value(), s2 = (double)a2.value();
        RT out_var = to_rt<RT>(__dsub_rn(__ddiv_rn(s2, (double)(cur - 1)),
                                         __ddiv_rn(__dmul_rn(s1, s1), (double)(cur * (cur - 1)))));
        RT dist = xadd(start, to_rt<RT>(div_count(s1, cur)));
        RT delta2 = xdiv(xmul(dist, dist), out_var);
        RT newc;
        if (L.adaptive_r == (RT)2) newc = xdiv((RT)cp.tmp, delta2);
        else newc = xmul(xpow(delta2, xdiv(-L.adaptive_r, (RT)2)), (RT)cp.tmp);
        done = newc <= (RT)cur;
    }
    uint32_t* cnt = (g.mode == 0) ? D.B.cnt_f : D.B.cnt_c;
    if (done) { cnt[item] = (uint32_t)cur; return false; }
    const uint64_t nxt = cur * 2;
    if (cp.max_count <= 2 * nxt) { cnt[item] = (uint32_t)cp.max_count; return false; }
    return true;
}

// Appends the warp's surviving items to the next round's list: one atomic per warp (all 32
// lanes call it).
__device__ __forceinline__ void warp_append(bool surv, uint32_t item, uint32_t* count, uint32_t* list, int lane) {
    const unsigned bal = __ballot_sync(0xffffffffu, surv);
    if (!bal) return;
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(count, (uint32_t)__popc(bal));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (surv) list[base + __popc(bal & ((1u << lane) - 1u))] = item;
}

// Pilot rounds an item went through on one side, recovered from its final count: a count below
// the maximum was fixed by the pilot of that size (rounds 0..r), the maximum is reached after
// every round of the side (get_samples_count, 240-273).
__device__ __forceinline__ uint32_t pilots_taken(uint32_t cnt, const CountParams& cp, bool adaptive) {
    if (!adaptive) return 0;
    uint32_t r = 0;
    if (cnt == (uint32_t)cp.max_count) {
        for (uint64_t c = cp.base_count; cp.max_count > 2 * c; c *= 2) r++;
        return r;
    }
    for (uint64_t c = cp.base_count; c < cnt; c *= 2) r++;
    return r + 1;
}

// Per-item completion of the final phase (sample_phi_antithetic, nested_sampler.hpp:171-216, and
// add_moments, 87-100): phi_f, phi_c; their moments go into this thread's
// moment slots mom[q * kTile] (q = 0..3 phi_f^k, 4..7 (phi_f - phi_c)^k; a zero phi adds
// nothing and touches no slot), the counts of items that hit the maximum / stayed at the base
// count, and the trace record.
template <class RT, int KIND, class S>
__device__ __forceinline__ void final_item(const DevLevel<RT>& D, uint32_t item, RT mean_big, RT phi_small,
                                           bool fine_big, double* mom, uint32_t& n_max, uint32_t& n_base,
                                           TraceRec* trace) {
    RT phi_big = (RT)phi_of<KIND, S, RT>(mean_big, 1.f);
    RT f_phi, c_phi;
    if (D.L.fine_only) { f_phi = phi_big; c_phi = 0; }
    else if (fine_big) { f_phi = phi_big; c_phi = phi_small; }
    else { f_phi = phi_small; c_phi = phi_big; }
    if (f_phi != (RT)0) {
        RT p = 1;
#pragma unroll
        for (int q = 0; q < 4; q++) { p = xmul(p, f_phi); mom[q * kTile] += (double)p; }
    }
    if (!D.L.fine_only) {
        const RT dphi = xsub(f_phi, c_phi);
        if (dphi != (RT)0) {
            RT p = 1;
#pragma unroll
            for (int q = 0; q < 4; q++) { p = xmul(p, dphi); mom[(4 + q) * kTile] += (double)p; }
        }
    }
    const uint32_t cf = D.B.cnt_f[item];
    n_max += (cf == (uint32_t)D.L.cf.max_count) ? 1u : 0u;
    n_base += (cf == (uint32_t)D.L.cf.base_count) ? 1u : 0u;
    if (trace) {
        TraceRec tr;
        tr.count_f = cf;
        tr.count_c = D.L.fine_only ? 0 : D.B.cnt_c[item];
        tr.phi_f = (double)f_phi;
        tr.phi_c = (double)c_phi;
        tr.mean_big = (double)mean_big;
        tr.min_abs_small = INFINITY;
        tr.core = 0;
        tr.pilots = pilots_taken(cf, D.L.cf, D.L.adaptive_f) +
                    (D.L.fine_only ? 0u : pilots_taken((uint32_t)tr.count_c, D.L.cc, D.L.adaptive_c));
        trace[item] = tr;
    }
}

// Block partial sums (OuterBuffers::block_sums layout): [0..3] phi_f moments, [4..7] difference
// moments, [8] work, [9] inner samples, [10] hit the maximum count, [11] stayed at the base count.
// The batched form of kernel_sample's per-outer-sample loop (nested_sampler.hpp:369-485): pilot
// and final phases of many outer samples drained from device work queues.
// MINB = CTAs per SM the register allocation must allow (1: up to 255 registers per thread,
// 2: 128 with the pipelined alias-column loop, 3: 80, 4: 64) — the register/occupancy variants the
// autotuner chooses between.  The variants run the same arithmetic in the same order, so their
// results are identical.
template <class RT, int KIND, int PREC, int MINB, class S = NoSampler>
__global__ void __launch_bounds__(kTile, MINB) k_phase(DevLevel<RT> D, SegSet SS, TraceRec* trace) {
    __shared__ Acc<PREC> sm_a1[kWarps];
    __shared__ Acc<PREC> sm_a2[kWarps];
    __shared__ float sm_ind[kWarps];
    __shared__ double sm_mom[8 * kTile];        // per-thread moment slots [q][thread]
    __shared__ double sm_acc[kWarps][16];
    __shared__ uint32_t sm_ticket;
    extern __shared__ float2 k_phase_rows[];             // staged R_tau rows (FP32 portfolio path)
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    // R_tau rows of the FP32 portfolio path can be staged (kRowItems rows of Q stocks)
    const uint32_t Qs = D.L.ot.Q;
    const float2* Rt2 = reinterpret_cast<const float2*>(D.B.Rt);
    const bool can_stage = KIND == KIND_PORTFOLIO && PREC == PREC_FP32 && D.L.ot.fast_s != nullptr &&
                           Qs <= kMaxStagedStocks;
    const uint32_t C = D.L.chunk;
    uint32_t* counters = D.B.counters;
    double wsum = 0;                                     // work of this thread's chunks
    uint32_t n_max = 0, n_base = 0;
    double* mom = sm_mom + t;
#pragma unroll
    for (int q = 0; q < 8; q++) mom[q * kTile] = 0;
    if (lane < 16) sm_acc[warp][lane] = 0;
    __syncthreads();
    const RT* Yv = reinterpret_cast<const RT*>(D.B.Yv);

    for (int si = 0; si < SS.n; si++) {
        const Seg g = SS.s[si];
        const uint32_t* list = g.list;
        uint32_t n_items = g.list ? counters[g.n_slot] : g.n_host;
        if (g.mode == 2 && g.list) {
            uint32_t off = 0;
            for (uint32_t k = 0; k < g.class_k; k++) off += counters[CNT_CLASS + k];
            list += off;
        }
        if (n_items == 0) continue;
        const uint32_t nch = 1u << g.nch_log2;
        const bool pilot = g.mode != 2;
        if (blockIdx.x == 0 && t == 0) sm_acc[0][9] += (double)n_items * (double)g.count;

        // The grid is persistent (the CTAs resident at once) and claims the segment's tiles from a
        // device work queue: one ticket per tile, so no CTA waits for a second wave and uneven
        // tiles balance themselves.  The next ticket is claimed while the current tile is
        // evaluated.  Which CTA evaluates a tile does not change any result.
        uint32_t* queue = counters + CNT_QUEUE + si;
        if (t == 0) sm_ticket = atomicAdd(queue, 1u);
        __syncthreads();
        uint64_t ticket = sm_ticket;
        if (nch <= (uint32_t)kTile) {
            // ---- a tile holds kTile / nch whole items ----
            const uint32_t per_tile = kTile / nch;
            const uint64_t tiles = ((uint64_t)n_items + per_tile - 1) / per_tile;
            const bool stage = can_stage && per_tile <= kRowItems;
            for (;;) {
                __syncthreads();                         // every thread has read the ticket
                if (ticket >= tiles) break;
                uint32_t next = 0;
                if (t == 0) next = atomicAdd(queue, 1u);
                if (stage) {                             // the tile's rows (the previous tile is done)
                    stage_rows(Rt2, Qs, list, ticket * per_tile, per_tile, n_items, k_phase_rows);
                    __syncthreads();
                }
                const float2* srow = stage ? k_phase_rows + (size_t)(t >> g.nch_log2) * Qs : nullptr;
                const uint64_t lin = ticket * per_tile + (t >> g.nch_log2);
                const uint32_t j = t & (nch - 1);
                const bool valid = lin < n_items;
                const uint32_t item = valid ? (list ? list[lin] : (uint32_t)lin) : 0;
                uint32_t gs = nch;
                uint64_t csmall = g.count;
                bool fine_big = true;
                if (!pilot && valid && !D.L.fine_only) {
                    uint32_t cf = D.B.cnt_f[item], cc = D.B.cnt_c[item];
                    csmall = cf < cc ? cf : cc;
                    fine_big = cf > cc;
                    gs = (uint32_t)(csmall / C);
                }
                const RT start = valid ? ((KIND == KIND_USER || D.L.ot.P) ? Yv[item] : -D.L.mp.max_loss) : (RT)0;
                Acc<PREC> a1, a2;
                a1.zero();
                a2.zero();
                // the FP32 path-simulated kernel evaluates deep samples warp-wide: all lanes call
                constexpr bool kCoopKind = KIND == KIND_PF_PATHS && PREC == PREC_FP32;
                if (valid || (kCoopKind && C <= kPathSortChunk))
                    eval_chunk<RT, KIND, PREC, S, MINB == 2>(D, item, g.tag, (uint64_t)j * C, g.count, C, pilot, start,
                                                             srow, a1, a2, wsum, valid);
                const float coeff = (float)gs / (float)nch;     // 1 / groups (a power of two)
                float ind = 0.f;
                if (!pilot && gs == 1) ind = phi_of<KIND, S, RT>(inner_mean<RT, PREC>(start, a1, csmall), coeff);
                const uint32_t wl = nch < 32 ? nch : 32;
                for (uint32_t m = 1; m < wl; m <<= 1) {
                    a1.merge(a1.shfl_xor(m));
                    if (pilot) a2.sq_merge_xor(m);
                    else {
                        ind += __shfl_xor_sync(0xffffffffu, ind, m);
                        if (2 * m == gs) ind = phi_of<KIND, S, RT>(inner_mean<RT, PREC>(start, a1, csmall), coeff);
                    }
                }
                const bool leader = (j == 0) && valid;
                if (nch > 32) {
                    if (lane == 0) { sm_a1[warp] = a1; sm_a2[warp] = a2; sm_ind[warp] = ind; }
                    __syncthreads();
                    if (leader) {
                        const uint32_t nw = nch / 32;
                        Acc<PREC> t1, t2;
                        t1.zero();
                        t2.zero();
                        float ti = 0.f;
                        if (!pilot && gs > 32) {
                            const uint32_t gw = gs / 32;
                            for (uint32_t gq = 0; gq < nw / gw; gq++) {
                                Acc<PREC> gsum;
                                gsum.zero();
                                for (uint32_t q = 0; q < gw; q++) gsum.merge(sm_a1[warp + gq * gw + q]);
                                ti += phi_of<KIND, S, RT>(inner_mean<RT, PREC>(start, gsum, csmall), coeff);
                                t1.merge(gsum);
                            }
                        } else {
                            for (uint32_t q = 0; q < nw; q++) {
                                t1.merge(sm_a1[warp + q]);
                                if (pilot) t2.merge(sm_a2[warp + q]);
                                ti += sm_ind[warp + q];
                            }
                        }
                        a1 = t1;
                        a2 = t2;
                        ind = ti;
                    }
                    __syncthreads();
                }
                if (pilot) {
                    const bool surv = leader && pilot_decide<RT, PREC>(D, g, item, start, a1, a2);
                    warp_append(surv, item, counters + g.next_slot, g.next_list, lane);
                } else if (leader) {
                    final_item<RT, KIND, S>(D, item, inner_mean<RT, PREC>(start, a1, g.count), (RT)ind, fine_big, mom,
                                   n_max, n_base, trace);
                }
                if (t == 0) sm_ticket = next;
                __syncthreads();
                ticket = sm_ticket;
            }
        } else {
            // ---- one CTA walks an item tile by tile ----
            const uint32_t tiles_per_item = nch / kTile;
            for (;;) {
                __syncthreads();                         // every thread has read the ticket
                if (ticket >= n_items) break;
                uint32_t next = 0;
                if (t == 0) next = atomicAdd(queue, 1u);
                const uint32_t item = list ? list[ticket] : (uint32_t)ticket;
                if (can_stage) {                         // this item's row (the previous item is done)
                    stage_rows(Rt2, Qs, nullptr, item, 1, item + 1, k_phase_rows);
                    __syncthreads();
                }
                const float2* srow = can_stage ? k_phase_rows : nullptr;
                uint32_t gs = nch;
                uint64_t csmall = g.count;
                bool fine_big = true;
                if (!pilot && !D.L.fine_only) {
                    uint32_t cf = D.B.cnt_f[item], cc = D.B.cnt_c[item];
                    csmall = cf < cc ? cf : cc;
                    fine_big = cf > cc;
                    gs = (uint32_t)(csmall / C);
                }
                const RT start = (KIND == KIND_USER || D.L.ot.P) ? Yv[item] : -D.L.mp.max_loss;
                const float coeff = (float)gs / (float)nch;
                Acc<PREC> tot1, tot2, gacc;
                tot1.zero();
                tot2.zero();
                gacc.zero();
                float tind = 0.f;
                for (uint32_t tl = 0; tl < tiles_per_item; tl++) {
                    const uint32_t j = tl * kTile + t;
                    Acc<PREC> a1, a2;
                    a1.zero();
                    a2.zero();
                    eval_chunk<RT, KIND, PREC, S, MINB == 2>(D, item, g.tag, (uint64_t)j * C, g.count, C, pilot, start, srow, a1, a2, wsum);
                    float ind = 0.f;
                    if (!pilot && gs == 1) ind = phi_of<KIND, S, RT>(inner_mean<RT, PREC>(start, a1, csmall), coeff);
                    for (uint32_t m = 1; m < 32; m <<= 1) {
                        a1.merge(a1.shfl_xor(m));
                        if (pilot) a2.sq_merge_xor(m);
                        else {
                            ind += __shfl_xor_sync(0xffffffffu, ind, m);
                            if (2 * m == gs) ind = phi_of<KIND, S, RT>(inner_mean<RT, PREC>(start, a1, csmall), coeff);
                        }
                    }
                    if (lane == 0) { sm_a1[warp] = a1; sm_a2[warp] = a2; sm_ind[warp] = ind; }
                    __syncthreads();
                    if (t == 0) {
                        if (!pilot && gs > 32 && gs < (uint32_t)kTile) {
                            const uint32_t gw = gs / 32;
                            for (uint32_t gq = 0; gq < (uint32_t)kWarps / gw; gq++) {
                                Acc<PREC> gsum;
                                gsum.zero();
                                for (uint32_t q = 0; q < gw; q++) gsum.merge(sm_a1[gq * gw + q]);
                                tind += phi_of<KIND, S, RT>(inner_mean<RT, PREC>(start, gsum, csmall), coeff);
                                tot1.merge(gsum);
                            }
                        } else {
                            Acc<PREC> t1;
                            t1.zero();
                            for (int q = 0; q < kWarps; q++) {
                                t1.merge(sm_a1[q]);
                                if (pilot) tot2.merge(sm_a2[q]);
                                if (!pilot && gs <= 32) tind += sm_ind[q];
                            }
                            tot1.merge(t1);
                            if (!pilot && gs >= (uint32_t)kTile) {
                                gacc.merge(t1);
                                if ((((uint64_t)tl + 1) * kTile) % gs == 0) {
                                    tind += phi_of<KIND, S, RT>(inner_mean<RT, PREC>(start, gacc, csmall), coeff);
                                    gacc.zero();
                                }
                            }
                        }
                    }
                    __syncthreads();
                }
                if (t == 0) {
                    if (pilot) {
                        if (pilot_decide<RT, PREC>(D, g, item, start, tot1, tot2))
                            g.next_list[atomicAdd(&counters[g.next_slot], 1u)] = item;
                    } else {
                        final_item<RT, KIND, S>(D, item, inner_mean<RT, PREC>(start, tot1, g.count), (RT)tind, fine_big, mom,
                                       n_max, n_base, trace);
                    }
                    sm_ticket = next;
                }
                __syncthreads();
                ticket = sm_ticket;
            }
        }
    }
    // this thread's work, moments and counts -> per-warp sums -> this CTA's partial-sum slot
    for (int m = 16; m > 0; m >>= 1) {
        wsum += __shfl_down_sync(0xffffffffu, wsum, m);
        n_max += __shfl_down_sync(0xffffffffu, n_max, m);
        n_base += __shfl_down_sync(0xffffffffu, n_base, m);
    }
    double mv[8];
#pragma unroll
    for (int q = 0; q < 8; q++) {
        mv[q] = mom[q * kTile];
        for (int m = 16; m > 0; m >>= 1) mv[q] += __shfl_down_sync(0xffffffffu, mv[q], m);
    }
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < 8; q++) sm_acc[warp][q] += mv[q];
        sm_acc[warp][8] += wsum;
        sm_acc[warp][10] += (double)n_max;
        sm_acc[warp][11] += (double)n_base;
    }
    __syncthreads();
    if (t < 16) {
        double v = 0;
        for (int w = 0; w < kWarps; w++) v += sm_acc[w][t];
        D.B.block_sums[(size_t)blockIdx.x * 16 + t] += v;
    }
}

// ---- outer draws ---------------------------------------------------------------------------
// sample_outer of the model (Y = randn_sync, model_sampler.cpp:57-59) or of the portfolio (the
// stocks at tau and the delta-CV constant, portfolio_sampler.cpp:293-311, 606-614) per outer
// sample, from the OUTER layout's phase-0 draws.
template <class RT, int KIND, int PREC, class S = NoSampler>
__global__ void __launch_bounds__(kTile) k_outer(DevLevel<RT> D, uint32_t nb) {
    const OuterLevel<RT>& L = D.L;
    RT* Yv = reinterpret_cast<RT*>(D.B.Yv);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x) {
        const TfKey key = tf_key(L.seed, outer_stream_id(L.ell, L.first_index + i));
        D.B.cnt_f[i] = L.adaptive_f ? 0u : (uint32_t)L.cf.max_count;
        D.B.cnt_c[i] = L.adaptive_c ? 0u : (uint32_t)L.cc.max_count;
        if constexpr (KIND == KIND_USER) {
            // the caller's SAMPLER: sample_outer from the outer stream, then the start value of its
            // inner estimates (init_inner_sampler, called once per outer sample: the batched path
            // needs a start that does not depend on the count); the object keeps the outer state
            S smp(user_ws(D.B, i));
            smp.nm_begin_outer(key);
            double w = 0;
            smp.sample_outer(L.ell, w);
            uint64_t cnt = L.cf.base_count;
            Yv[i] = smp.init_inner_sampler(cnt, w);
            *const_cast<S*>(user_state<S>(D.B, i)) = smp;
        } else if (!is_portfolio_kind(KIND)) {
            Yv[i] = outer_normal_at<PREC, RT>(key, PH_OUTER, 0);
        } else {
            // portfolio_sampler.cpp:293-311 on the OUTER layout: normal 0 systemic, 1 + s per stock
            const OptionTable<RT>& ot = L.ot;
            constexpr uint32_t RS = RStride<PREC>::v;
            RT* Rrow = reinterpret_cast<RT*>(D.B.Rt) + (size_t)i * ot.Q * RS;
            RT dW_sys = 0, cv = (RT)0;
            const uint32_t nnorm = ot.Q == 1 ? 1 : ot.Q + 1;
            for (uint32_t b = 0; 4 * b < nnorm; b++) {          // four normals per block
                uint64_t v0, v1;
                threefry2x64(b, PH_OUTER, key, v0, v1);
                RT z[4];
                bm_pair<PREC, RT>((uint32_t)v0, (uint32_t)(v0 >> 32), z[0], z[1]);
                bm_pair<PREC, RT>((uint32_t)v1, (uint32_t)(v1 >> 32), z[2], z[3]);
                for (uint32_t q = 0; q < 4; q++) {
                    const uint32_t k = 4 * b + q;
                    if (k >= nnorm) break;
                    if (k == 0) { dW_sys = xmul(ot.stau, z[0]); if (ot.Q > 1) continue; }
                    const uint32_t s = ot.Q == 1 ? 0 : k - 1;
                    RT W = ot.Q == 1 ? dW_sys : xadd(xmul(ot.rho, dW_sys), xmul(ot.s1_rho2, xmul(ot.stau, z[q])));
                    RT R;
                    if (PREC == PREC_FP32) {     // GBM at tau in float (expf) and its logarithm
                        const float sg = (float)ot.sigma[s], S0 = (float)ot.S0[s];
                        const float e = sg * (float)W + ((float)ot.mu[s] - 0.5f * sg * sg) * (float)ot.tau;
                        R = (RT)(S0 * expf(e));
                        Rrow[s * RS + 1] = (RT)(logf(S0) + e);
                    } else {
                        R = simulate_stock_ref<RT>(ot.S0[s], ot.mu[s], ot.sigma[s], ot.tau, W);
                    }
                    Rrow[s * RS] = R;
                    if (ot.use_delta_cv) cv = xadd(cv, xmul(xsub(R, ot.S0[s]), ot.delta_coalesce[s]));
                }
            }
            Yv[i] = xsub(-ot.max_loss, cv);
        }
    }
}

// ---- bucket outer samples by final count (count_big = max(cnt_f, cnt_c)) ------------------
// Pass 0 counts the outer samples of each class, pass 1 scatters their indices into class order.
// Each CTA histograms a tile in shared memory first, so the global counters see one atomic per
// class per tile instead of one per outer sample.
template <class RT>
__global__ void k_classify(DevLevel<RT> D, uint32_t nb, int pass) {
    uint32_t* counters = D.B.counters;
    const uint32_t C = D.L.chunk;
    __shared__ uint32_t offs[64], hist[64], base[64];
    if (pass == 1 && threadIdx.x == 0) {
        uint32_t a = 0;
        for (int k = 0; k < 64; k++) { offs[k] = a; a += counters[CNT_CLASS + k]; }
    }
    for (uint32_t t0 = blockIdx.x * blockDim.x; t0 < nb; t0 += gridDim.x * blockDim.x) {
        if (threadIdx.x < 64) hist[threadIdx.x] = 0;
        __syncthreads();
        const uint32_t i = t0 + threadIdx.x;
        const bool valid = i < nb;
        uint32_t k = 0, rank = 0;
        if (valid) {
            uint32_t cf = D.B.cnt_f[i], cc = D.L.fine_only ? 0u : D.B.cnt_c[i];
            uint32_t q = (cf > cc ? cf : cc) / C;
            k = q ? 31 - __clz(q) : 0;
            rank = atomicAdd(&hist[k], 1u);
        }
        __syncthreads();
        if (threadIdx.x < 64 && hist[threadIdx.x]) {
            if (pass == 0) atomicAdd(&counters[CNT_CLASS + threadIdx.x], hist[threadIdx.x]);
            else base[threadIdx.x] = atomicAdd(&counters[CNT_FILL + threadIdx.x], hist[threadIdx.x]);
        }
        __syncthreads();
        if (pass == 1 && valid) D.B.class_items[offs[k] + base[k] + rank] = i;
        __syncthreads();
    }
}

// Per-CTA partials -> the level's 16 sums, one CTA of 256 threads: thread t adds sum q = t % 16 of
// CTA slots t / 16, t / 16 + 16, ... (consecutive threads read consecutive doubles), then thread q
// adds its 16 group sums in a fixed order.  Launch with 256 threads.
static __global__ void __launch_bounds__(256) k_reduce_blocks(const double* block_sums, int grid, double* level_acc) {
    __shared__ double sm[16][17];
    const int t = threadIdx.x, q = t & 15, g = t >> 4;
    double v = 0;
    for (int b = g; b < grid; b += 16) v += block_sums[(size_t)b * 16 + q];
    sm[g][q] = v;
    __syncthreads();
    if (t < 16) {
        double s = 0;
        for (int k = 0; k < 16; k++) s += sm[k][t];
        level_acc[t] += s;
    }
}

// Persistent grid of the phase kernel: the CTAs that are resident at once (occupancy x SMs),
// at most the grid the partial-sum buffer was sized for.
// Dynamic shared memory of a phase-kernel instantiation: the staged R_tau rows of the FP32
// portfolio path (set as the kernel's maximum once, before the occupancy query and the first
// launch).
template <int KIND, int PREC>
constexpr size_t phase_dyn_smem() {
    return PREC != PREC_FP32 ? 0 : KIND == KIND_PORTFOLIO ? kRowSmemBytes : KIND == KIND_PF_PATHS ? kPathSortSmemBytes : 0;
}

template <class RT, int KIND, int PREC, int MINB, class S = NoSampler>
static int phase_grid(int cap) {
    static int g = 0;
    if (g == 0) {
        int dev = 0, sms = 148, per_sm = 0;
        constexpr size_t dyn = phase_dyn_smem<KIND, PREC>();
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (dyn) cudaFuncSetAttribute(k_phase<RT, KIND, PREC, MINB, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_phase<RT, KIND, PREC, MINB, S>, kTile, dyn) != cudaSuccess ||
            per_sm < 1)
            per_sm = 1;
        g = per_sm * sms;
    }
    return g < cap ? g : cap;
}

template <class RT, int KIND, int PREC, int MINB, class S = NoSampler>
static void launch_phase_v(const DevLevel<RT>& D, const SegSet& SS, TraceRec* trace, cudaStream_t stream) {
    cudaMemsetAsync(D.B.counters + CNT_QUEUE, 0, kMaxSegs * sizeof(uint32_t), stream);
    if (D.B.prof_mark) D.B.prof_mark(D.B.prof_user, 0, stream);
    const int grid = phase_grid<RT, KIND, PREC, MINB, S>(D.B.grid);
    k_phase<RT, KIND, PREC, MINB, S><<<grid, kTile, phase_dyn_smem<KIND, PREC>(), stream>>>(D, SS, trace);
    if (D.B.prof_mark) D.B.prof_mark(D.B.prof_user, 1, stream);
    count_launch();
}

// The FP32 path has three register/occupancy variants (OuterLevel::variant 0, 1, 2 -> 1, 3, 4
// resident CTAs per SM guaranteed), and the portfolio a fourth (3 -> 2 CTAs per SM, 128 registers,
// the pipelined alias-column loop; other kinds run variant 0 for it); the parity precisions run
// variant 0, the FP32 kernel of path-simulated portfolios two CTAs per SM (128 registers: the
// class-ordered loop spills at 80, and runs 7 % faster at two CTAs without spills than at three
// with them; the FP64 path states and exponentials leave one CTA per SM at the compiler's choice).
template <class RT, int KIND, int PREC, class S = NoSampler>
static void launch_phase(const DevLevel<RT>& D, const SegSet& SS, TraceRec* trace, cudaStream_t stream) {
    if constexpr (PREC == PREC_FP32 && KIND != KIND_USER && KIND != KIND_PF_PATHS) {
        if (D.L.variant == 1) return launch_phase_v<RT, KIND, PREC, 3>(D, SS, trace, stream);
        if (D.L.variant == 2) return launch_phase_v<RT, KIND, PREC, 4>(D, SS, trace, stream);
        if constexpr (KIND == KIND_PORTFOLIO)
            if (D.L.variant == 3) return launch_phase_v<RT, KIND, PREC, 2>(D, SS, trace, stream);
    }
    launch_phase_v<RT, KIND, PREC, (KIND == KIND_PF_PATHS && PREC == PREC_FP32) ? 2 : 1, S>(D, SS, trace, stream);
}

static inline uint32_t ilog2_u64(uint64_t v) {
    uint32_t r = 0;
    while ((1ull << (r + 1)) <= v) r++;
    return r;
}

template <class RT, int KIND, int PREC, class S = NoSampler>
static cudaError_t run_batch(DevLevel<RT>& D, uint32_t nb, TraceRec* trace, cudaStream_t stream) {
    const OuterLevel<RT>& L = D.L;
    OuterBuffers& B = D.B;
    const uint32_t C = L.chunk;
    const int grid = B.grid;
    cudaError_t e;
    int og = (int)((nb + kTile - 1) / kTile);
    if (og > grid) og = grid;
    if (og < 1) og = 1;
    k_outer<RT, KIND, PREC, S><<<og, kTile, 0, stream>>>(D, nb);
    count_launch();
    if ((e = cudaGetLastError()) != cudaSuccess) return e;

    if (L.adaptive_f || L.adaptive_c) {
        uint32_t rounds_f = 0, rounds_c = 0;
        if (L.adaptive_f) for (uint64_t c = L.cf.base_count; L.cf.max_count > 2 * c; c *= 2) rounds_f++;
        if (L.adaptive_c) for (uint64_t c = L.cc.base_count; L.cc.max_count > 2 * c; c *= 2) rounds_c++;
        const uint32_t rounds = rounds_f > rounds_c ? rounds_f : rounds_c;
        uint32_t* listF[2] = {B.lists, B.lists + B.cap};
        uint32_t* listC[2] = {B.lists + 2 * B.cap, B.lists + 3 * B.cap};
        for (uint32_t r = 0; r < rounds; r++) {
            const int cur = r & 1, nxt = cur ^ 1;
            e = cudaMemsetAsync(B.counters + CNT_LIST + nxt, 0, sizeof(uint32_t), stream);
            if (e == cudaSuccess) e = cudaMemsetAsync(B.counters + CNT_LIST + 2 + nxt, 0, sizeof(uint32_t), stream);
            if (e != cudaSuccess) return e;
            SegSet SS;
            SS.n = 0;
            for (int which = 0; which < 2; which++) {
                const bool fine = which == 0;
                if (fine ? (r >= rounds_f) : (r >= rounds_c)) continue;
                const CountParams& cp = fine ? L.cf : L.cc;
                Seg& g = SS.s[SS.n++];
                g.list = (r == 0) ? nullptr : (fine ? listF[cur] : listC[cur]);
                g.n_slot = CNT_LIST + (fine ? 0 : 2) + cur;
                g.n_host = nb;
                g.count = cp.base_count << r;
                g.nch_log2 = ilog2_u64(g.count / C);
                g.tag = (fine ? PH_FINE : PH_COARSE) + r;
                g.mode = fine ? 0 : 1;
                g.class_k = 0;
                g.next_slot = CNT_LIST + (fine ? 0 : 2) + nxt;
                g.next_list = fine ? listF[nxt] : listC[nxt];
            }
            if (SS.n == 0) continue;
            launch_phase<RT, KIND, PREC, S>(D, SS, nullptr, stream);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
        e = cudaMemsetAsync(B.counters + CNT_CLASS, 0, 128 * sizeof(uint32_t), stream);
        if (e != cudaSuccess) return e;
        k_classify<RT><<<og, kTile, 0, stream>>>(D, nb, 0);
        k_classify<RT><<<og, kTile, 0, stream>>>(D, nb, 1);
        count_launch(2);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        const uint64_t maxc = L.cf.max_count > L.cc.max_count ? L.cf.max_count : L.cc.max_count;
        const uint32_t kmax = ilog2_u64(maxc / C);
        SegSet SS;
        SS.n = 0;
        for (uint32_t k = 0; k <= kmax && SS.n < kMaxSegs; k++) {
            Seg& g = SS.s[SS.n++];
            g.list = B.class_items;
            g.n_slot = CNT_CLASS + k;
            g.n_host = 0;
            g.count = (uint64_t)C << k;
            g.nch_log2 = k;
            g.tag = PH_FINAL;
            g.mode = 2;
            g.class_k = k;
            g.next_slot = 0;
            g.next_list = nullptr;
        }
        launch_phase<RT, KIND, PREC, S>(D, SS, trace, stream);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    } else {
        const uint64_t cbig = (L.fine_only || L.cf.max_count >= L.cc.max_count) ? L.cf.max_count : L.cc.max_count;
        SegSet SS;
        SS.n = 1;
        Seg& g = SS.s[0];
        g.list = nullptr;
        g.n_slot = 0;
        g.n_host = nb;
        g.count = cbig;
        g.nch_log2 = ilog2_u64(cbig / C);
        g.tag = PH_FINAL;
        g.mode = 2;
        g.class_k = 0;
        g.next_slot = 0;
        g.next_list = nullptr;
        launch_phase<RT, KIND, PREC, S>(D, SS, trace, stream);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template <class RT, int KIND, int PREC, class S = NoSampler>
cudaError_t sample_level_t(const OuterLevel<RT>& L, OuterBuffers& B, TraceRec* trace,
                                  cudaStream_t stream) {
    DevLevel<RT> D;
    D.L = L;
    D.B = B;
    for (uint64_t done = 0; done < L.M;) {
        const uint64_t nb = (L.M - done) < B.cap ? (L.M - done) : B.cap;
        D.L.first_index = L.first_index + done;
        cudaError_t e = run_batch<RT, KIND, PREC, S>(D, (uint32_t)nb, trace ? trace + done : nullptr, stream);
        if (e != cudaSuccess) return e;
        done += nb;
    }
    k_reduce_blocks<<<1, 256, 0, stream>>>(B.block_sums, B.grid, B.level_acc);
    count_launch();
    return cudaGetLastError();
}

}  // namespace nmlmc
