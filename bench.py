"""Benchmark: time-to-eps of the nested-MLMC estimate of P(L > K) on B200.

Default workload (the large-portfolio configuration): d = 200 GBM stocks (S0 = 100, r = mu = 0.05,
sigma ~ U[0.1, 0.4], tau = 1/52), P = 1e6 European options (seeded generator, seed 1: uniform
stock, 50/50 call/put, strike ~ U[0.8, 1.2] S0, maturity ~ U[0.25, 2], position ~ N(0, 1)), loss
L(Y) = sum_i w_i (V_i(0) - V_i(tau, S(tau))) with Black-Scholes values, K = the 99 % quantile of L
over 1e5 full evaluations.  P(L > K) ~ 0.01 by continuation MLMC to RMSE eps = 1e-4 with the
reference's default importance sub-sampling (prob ~ |w_i|), the delta control variate, adaptive
inner sampling (N0 = 64, beta = 2, r = 1.5) and the antithetic estimator.  A step is one complete
MLMC run (host driver + level sampler) to eps; synthetic inputs (seeded generator, no dataset).

Our arm: the batched FP32 sampler (OUTER streams, SFU Black-Scholes, Kahan FP32 inner sums, FP64
moments), all levels of an MLMC round in one submission (one CUDA graph per round).  `value` is the
device time of the run's levels (%globaltimer stamps at the level boundaries inside each round's
graph); `e2e` is the wall time of the same step through the C ABI from host buffers: the upload of
the portfolio tables (set_portfolio: option records, alias table) and the whole run (host driver
decisions, graph updates and launches, the device->host copy of every level result).  Reported
beside it on the same GPU: the plain FP64 drop-in (the reference's stream layout, 2048 virtual
cores, one synchronous call per level; timed per level on bounded samples and scaled by the level
counts of the run, with a full measured run at eps = 1e-3 as its calibration), the per-level
FP32 error against the all-FP64 sampler on the same streams, the phase kernel's roofline, the
K-quantile sweep; and the reference's own CPU sampler (oracle/_ref, OpenMP on all host threads),
timed the same way with a full measured CPU run at a looser eps as its calibration.

Multi-GPU (torchrun): every rank samples its share of each level call and the level results are
all-reduced (16 doubles per level), so the estimate equals the single-GPU one and total work is
fixed (strong scaling).

--case c1 is the adaptive model problem (Y ~ N(0,1), X = Y + Z, K = 1, exact 1 - Phi(1)) to
eps = 1e-4; the other cases are profiling cases of single kernels.

--impl reference times the reference's own CPU implementation (oracle/_ref: the reference sources
compiled here, OpenMP on all host threads; the C restatement if absent) on bounded per-level
samples and multiplies its per-outer-sample cost by the level sample counts the MLMC run needs at
eps (bench_schedule.json, recorded from the GPU run).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "nested-risk-mlmc_b200")
SCHEDULE = os.path.join(ROOT, "bench_schedule.json")

EPS = 1e-4
METRIC = "time-to-ε (s) for MLMC P(loss>K) at ε=1e-4, batched FP32 vs plain FP64, 1 B200"
ADAPTIVE_R = 1.5
# The large-portfolio configuration; the same dict is the `config` of both arms' lines.
C3_CONFIG = dict(workload="large portfolio: d=200 GBM stocks, P=1e6 European options, P(L>K) with "
                          "K the 99% loss quantile of 1e5 full evaluations",
                 stocks=200, options=1_000_000, generator_seed=1, tau="1/52", r=0.05, rho=0.0,
                 sub_sampling="importance, prob ~ |w_i|", delta_cv=True, N0=64, beta=2,
                 adaptive_r=ADAPTIVE_R, antithetic=True, moments=4, eps=EPS, M0=1024,
                 deviations=("r=1.5 (the reference's default exponent); the host driver adds levels "
                             "until its bias test passes (to level 15, from starting level 11) where "
                             "the configuration text names levels 0-10; the FP32 option table is one "
                             "packed 32-byte record per option plus an 8-byte alias entry (40 MB) "
                             "instead of the 21-byte structure of arrays; the loss carries no "
                             "e^{-r tau} discount (the configuration's L(Y))"),
                 l2_flush="not flushed: inputs (40 MB of option and alias tables) stay L2-resident "
                          "by design; every inner draw is computed from a counter")
C1_WORKLOAD = dict(workload="model problem X=Y+Z, K=1, adaptive inner sampling, levels to eps",
                   N0=32, beta=2, adaptive_r=ADAPTIVE_R, antithetic=True, moments=4, eps=EPS, M0=1024,
                   adaptive_rule_note=("r=1.5, the reference's default exponent; the r=2 rule (double "
                                       "while |mean-K| < 3 sigma/sqrt(N)) keeps a fixed 3-sigma stopping "
                                       "confidence at every level and its bias levels off at 3.7e-4 > eps"),
                   l2_flush="not needed: no input data; every inner draw is computed from a counter")
# Algorithmic lane operations per inner sample of the X = Y + Z model on the FP32 path:
#   Threefry2x64-20 block = 140 INT32 ops (20 rounds x (64-bit add 2 + rotate 2 + xor 2) less
#   two 32-bit rotations, 6 key injections x 4) shared by 4 normals -> 35;
#   Box-Muller pair ~ 22 FP32/ALU + 4 SFU ops shared by 2 normals -> 13;
#   X = Y + Z (1) and a Kahan update of the inner sum (4) -> 5.
OPS_PER_INNER = 35 + 13 + 5
# Algorithmic lane operations per inner sample of the large portfolio on the FP32 path:
#   half a Threefry2x64-20 block (70); the option draw: column floor(vP/2^64), coin, alias
#   compare and select (5); the Black-Scholes loss: ln R (2), call/put sign (1), d1 and d2 (3),
#   two Phi = rational erfc (|x| scale 2, reciprocal 1, 10 FMA, exponential 2, product and
#   half 2, reflection 2: 19 each), the position-weighted value (4), delta control variate (2);
#   Kahan update (4).
C3_OPS_PER_INNER = 70 + 5 + (2 + 1 + 3 + 2 * 19 + 4 + 2) + 4


def exact_p():
    return 0.5 * math.erfc(1 / math.sqrt(2))


# ---------------------------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms in the background."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return dict(sm_mhz=None, sm_max_mhz=None, reasons=["nvidia-smi unavailable"])
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        text = self.f.read()
        os.unlink(self.f.name)
        return parse_clock_samples(text)


def parse_clock_samples(text: str) -> dict:
    """Median SM clock, maximum SM clock and the throttle reasons seen in nvidia-smi CSV rows of
    ClockSampler.FIELDS (index, clocks.sm, clocks.max.sm, power.draw, active mask, then the four
    reasons as Active / Not Active)."""
    sm, smax, reasons = [], None, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for line in text.strip().splitlines():
        r = [x.strip() for x in line.split(",")]
        try:
            sm.append(float(r[1]))
            smax = float(r[2])
        except (ValueError, IndexError):
            continue
        for name, v in zip(names, r[5:9]):
            if v.lower().startswith("active"):
                reasons.add(name)
    return dict(sm_mhz=statistics.median(sm) if sm else None, sm_max_mhz=smax,
                reasons=sorted(reasons), samples=len(sm))


# ---------------------------------------------------------------------------------------------
def ddp_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def make_sampler(nm, device, precision, streams, seed, cores=2048):
    s = nm.Sampler(device, cores=cores, N0=32, beta=2, adaptive_r=ADAPTIVE_R,
                   precision=precision, streams=streams, seed=seed)
    s.set_model(nm.MODEL_SHIFT, 0.0, 1.0)
    if precision == nm.PREC_FP32:
        s.set_autotune(2)       # per level: register/occupancy variant and chunk length (warm-up tunes)
    return s


def phase_choices(s, nlevels):
    """The per-level phase-kernel configuration: [variant, chunk, tuned or pinned?]."""
    out = {}
    for ell in range(nlevels):
        p = s.phase_config(ell)
        out[str(ell)] = [p["variant"], p["chunk"], bool(p["state"] in (1, 2))]
    return out


def run_once(nm, s, batched, dist=None, eps=EPS, M0=1024):
    """One MLMC run to eps. Returns (result dict, wall seconds)."""
    if dist is None:
        t0 = time.perf_counter()
        out = s.mlmc_run(targetTOL=eps, M0=M0, batched=batched)
        return out, time.perf_counter() - t0
    from nmlmc.distributed import sharded_mlmc_run
    _, dev = dist
    t0 = time.perf_counter()
    out = sharded_mlmc_run(s, device=dev, targetTOL=eps, M0=M0, batched=batched)
    return out, time.perf_counter() - t0


def per_level_error(nm, device, nlevels, M=1 << 16):
    """Each level's FP32 estimate against the all-FP64 one on the same OUTER streams (M outer
    samples): mean of phi_f and of phi_f - phi_c, the outer samples whose phi differs, and the
    largest |inner mean - K| among them (the FP32 flip bound is 2e-5)."""
    import numpy as np
    out = []
    for ell in range(nlevels):
        a = make_sampler(nm, device, nm.PREC_FP32, nm.STREAMS_OUTER, seed=11)
        b = make_sampler(nm, device, nm.PREC_FP64, nm.STREAMS_OUTER, seed=11)
        a.set_autotune(0)
        ra, rb = a.sample(ell, M, trace=True), b.sample(ell, M, trace=True)
        ta, tb = ra["trace"], rb["trace"]
        flip = (ta["phi_f"] != tb["phi_f"]) | (ta["phi_c"] != tb["phi_c"])
        out.append({"level": ell, "M": M,
                    "fEl_fp32_minus_fp64": (ra["fsums"][0] - rb["fsums"][0]) / M,
                    "dEl_fp32_minus_fp64": (ra["diffsums"][0] - rb["diffsums"][0]) / M,
                    "phi_flips": int(flip.sum()),
                    "max_abs_mean_at_flip": (max(abs(float(x)) for x in np.minimum(
                        np.abs(tb["mean_big"][flip]), tb["min_abs_small"][flip])) if flip.any() else None)})
    return out


# ---------------------------------------------------------------------------------------------
def level_costs(sample, levels, Ms, budget_s, m0):
    """Seconds per outer sample of `sample(ell, m)` at each level: calls of m0, 2 m0, ... outer
    samples until a call takes a quarter of the level's share of the budget (or reaches M)."""
    per_level = budget_s / max(1, len(levels))
    cost, details = {}, []
    for ell, M in zip(levels, Ms):
        if M == 0:
            continue
        m = min(m0, M)
        while True:
            t0 = time.perf_counter()
            sample(ell, m)
            dt = time.perf_counter() - t0
            if dt >= per_level / 4 or m >= M:
                break
            m = min(M, m * max(2, int(per_level / 4 / max(dt, 1e-4))))
        cost[ell] = dt / m
        details.append(f"l{ell}:{m}")
    return cost, details


def cpu_reference_time(schedule: dict, budget_s: float = 20.0, threads: int | None = None):
    """The reference's CPU level sampler of the model problem on bounded per-level samples;
    returns the time-to-eps it implies for `schedule` (outer samples per level at eps) and a
    description."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    threads = threads or os.cpu_count() or 1
    levels = [int(l) for l in schedule["levels"]]
    Ms = [int(m) for m in schedule["M"]]
    if O.ref_available("f32_lzcnt"):
        kind = "reference"
        ref = O.Reference("f32_lzcnt")
        ref.init(threads, 32, 2, ADAPTIVE_R, True)
        ref.model_init(1, 0.0, 1.0, 0, traced=False)
        sample = ref.sample
        cores = threads
    else:
        kind = "port"
        s = O.Sampler(O.PREC_REF32, O.STREAMS_CORE, 1, 32, 2, ADAPTIVE_R, True, False, 0)
        s.set_model(O.MODEL_SHIFT, 0.0, 1.0)
        sample = s.sample
        cores = 1
    cost, details = level_costs(sample, levels, Ms, budget_s, 64 * cores)
    total = sum(cost[l] * M for l, M in zip(levels, Ms) if M)
    desc = (f"reference level sampler ({'oracle/_ref, real_t=float' if kind == 'reference' else 'C port'}"
            f", {cores} threads) timed on bounded samples per level [{', '.join(details)} outer samples], "
            f"cost per outer sample x the level counts of the eps={EPS:g} run; extrapolated")
    return total, kind, cores, desc


def c3_cpu_reference(pfw, K, threads=None):
    """The reference's CPU level sampler of the large portfolio (oracle/_ref: the reference's
    portfolio_sample with Subsampling::Random, prob ~ |w|, the delta control variate, N0 = 64,
    beta = 2, r = 1.5, OpenMP on `threads`), or the C restatement on one thread when the
    reference is not built.  Returns (sample(ell, M), kind, cores, reinit(seed))."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    threads = threads or os.cpu_count() or 1
    if O.ref_available("f32_lzcnt"):
        ref = O.Reference("f32_lzcnt")

        def reinit(seed):
            ref.init(threads, 64, 2, ADAPTIVE_R, True)
            ref.portfolio_init(pfw, r=0.05, rho=0.0, max_loss=K, tau=1 / 52, subsample=O.SUB_RANDOM,
                               use_delta_cv=True, seed=seed, traced=False)
        reinit(0)
        return ref.sample, "reference", threads, reinit
    s = O.Sampler(O.PREC_REF32, O.STREAMS_CORE, 1, 64, 2, ADAPTIVE_R, True, False, 0)

    def reinit_port(seed):
        s.set_portfolio(pfw, r=0.05, rho=0.0, max_loss=K, tau=1 / 52, subsample=O.SUB_RANDOM,
                        use_delta_cv=True, discount=False)
    reinit_port(0)
    return s.sample, "port", 1, reinit_port


def c3_cpu_baseline(nm, pfw, K, schedule: dict, budget_s: float, calibrate_s: float = 0.0,
                    threads=None) -> dict:
    """The reference CPU sampler's time-to-eps for the large portfolio: its cost per outer sample
    on every level (bounded samples) times the level counts of the GPU run at eps (`schedule`);
    with `calibrate_s` > 0 also one complete CPU run of the host driver at the loosest eps in
    (1e-2, 5e-3, 2.5e-3, ...) that is expected to finish within calibrate_s, measured, beside the
    same extrapolation from that run's own level counts."""
    sample, kind, cores, reinit = c3_cpu_reference(pfw, K, threads)
    levels = [int(l) for l in schedule["levels"]]
    Ms = [int(m) for m in schedule["M"]]
    cost, details = level_costs(sample, levels, Ms, budget_s, cores)
    total = sum(cost[l] * M for l, M in zip(levels, Ms) if M)
    out = {"value": total, "unit": "s", "cores": cores, "kind": kind,
           "sample": (f"reference level sampler ({'oracle/_ref, real_t=float' if kind == 'reference' else 'C port'}, "
                      f"{cores} threads) timed on bounded samples per level [{', '.join(details)} outer samples], "
                      f"cost per outer sample x the level counts of the GPU run at eps={schedule['eps']:g}; "
                      f"extrapolated (the reference's loss keeps its e^(-r tau) discount: same cost)")}
    if calibrate_s > 0:
        def level(ell, M):
            r = sample(ell, M)
            return dict(fsums=r["fsums"], diffsums=r["diffsums"], work=r["work"])
        eps_c, last = 1e-2, None
        while True:
            reinit(7)
            t0 = time.perf_counter()
            run = nm.mlmc_run_cb(level, targetTOL=eps_c, M0=1024)
            wall = time.perf_counter() - t0
            last = (eps_c, wall, run)
            if wall * 4 > calibrate_s or eps_c < 1e-3:     # the next halving of eps costs ~4x
                break
            eps_c /= 2
        eps_c, wall, run = last
        lm = [int(x) for x in run["level_M"]]
        miss = [l for l, M in enumerate(lm) if M and l not in cost]
        if miss:
            more, _ = level_costs(sample, miss, [lm[l] for l in miss], budget_s / 4, cores)
            cost.update(more)
        ext = sum(cost[l] * M for l, M in enumerate(lm) if M)
        out["calibration"] = {"eps": eps_c, "measured_s": wall, "extrapolated_s": ext,
                              "extrapolated_over_measured": ext / wall, "levels": len(lm),
                              "level_M": lm, "Eg": float(run["Eg"]),
                              "note": "one complete run of the host driver over the reference's CPU "
                                      "sampler, and the per-level extrapolation from its level counts"}
    return out


def read_schedule(case: str) -> dict | None:
    if not os.path.exists(SCHEDULE):
        return None
    with open(SCHEDULE) as f:
        d = json.load(f)
    return d.get(case)


def reference_arm(args):
    world, rank, _ = ddp_env()
    if rank != 0:
        return
    case = "c1" if args.case == "c1" else "c3"
    schedule = read_schedule(case)
    if schedule is None:
        print(json.dumps({"impl": "reference", "unavailable": f"bench_schedule.json has no {case} schedule"}))
        return
    times = []
    t_all0 = time.perf_counter()
    per_step = max(5.0, args.ref_budget * 3 / max(1, args.steps))
    if case == "c1":
        kind = cores = desc = None
        for _ in range(args.steps):
            v, kind, cores, desc = cpu_reference_time(schedule, budget_s=per_step)
            times.append(v)
        value = statistics.median(times)
        cpu = {"value": value, "unit": "s", "cores": cores, "kind": kind, "sample": desc}
        config = C1_WORKLOAD
    else:
        sys.path.insert(0, PKG)
        import nmlmc as nm
        pfw = c3_portfolio(nm)
        K = float(schedule["K"])
        cpu = None
        for k in range(args.steps):
            c = c3_cpu_baseline(nm, pfw, K, schedule, budget_s=per_step,
                                calibrate_s=(args.ref_budget if k == 0 else 0.0))
            times.append(c["value"])
            cpu = cpu or c
        value = statistics.median(times)
        cpu = dict(cpu, value=value)
        config = C3_CONFIG
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": value * 1e3,
            "higher_is_better": False, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": config, "cpu_baseline": cpu,
            "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "measure_wall_s": time.perf_counter() - t_all0}
    print(json.dumps(line))


def small_case():
    """Fixed level calls of the FP32 sampler (the profiling case): level 0 with 2^24 outer samples
    (fine only, 32 inner samples each) and level 8 with 2^16 (adaptive pilots and the antithetic
    final phase), on the default register variant without tuning probes, so the first phase-kernel
    launch is level 0's first pilot round.  Device memory: the batch buffers, grown to 2^24 outer
    samples (~600 MB)."""
    sys.path.insert(0, PKG)
    import nmlmc as nm
    s = make_sampler(nm, 0, nm.PREC_FP32, nm.STREAMS_OUTER, seed=0)
    s.set_autotune(0)
    for ell, M in ((0, 1 << 24), (8, 1 << 16), (0, 1 << 24), (8, 1 << 16)):
        r = s.sample(ell, M)
        print(f"level {ell} M {M}: {r['seconds'] * 1e3:.3f} ms, {r['stats'][0] / r['seconds']:.3e} inner/s")


# The reference's own model main (model_sampler.cpp:120-147): reference model with tau = 0.02 and
# max_loss = tau (Phi^-1(eta/2)^2 - 1), eta = 0.025 (the exact answer), N0 = 32, beta = 4,
# r = 1.5, antithetic, TOL = 1e-3, M0 = 1024.
REF_MAIN = dict(tau=0.02, eta=0.025, N0=32, beta=4, adaptive_r=1.5, tol=1e-3, M0=1024)


def ref_main_max_loss(norm_cdf_inv) -> float:
    """max_loss of the model main in real_t = float (model_sampler.cpp:144)."""
    import numpy as np
    x = np.float32(norm_cdf_inv(REF_MAIN["eta"] / 2))
    return float(np.float32(REF_MAIN["tau"]) * (x * x - np.float32(1)))


def ref_main_cpu(threads: int | None = None, tol: float | None = None) -> dict:
    """The reference's CPU level sampler (oracle/_ref, OpenMP on `threads`) of the model main under
    the host driver (whose decisions equal the reference's mlmc_t::run): wall seconds and result."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, PKG)
    import oracle as O
    import nmlmc as nm
    threads = threads or os.cpu_count() or 1
    variant = "f32_lzcnt" if O.ref_available("f32_lzcnt") else None
    if variant is None:
        return {"unavailable": "oracle/_ref not built"}
    ml = ref_main_max_loss(O.Reference("f32").L.ref_norm_cdf_inv)
    ref = O.Reference(variant)
    ref.init(threads, REF_MAIN["N0"], REF_MAIN["beta"], REF_MAIN["adaptive_r"], True)
    ref.model_init(0, REF_MAIN["tau"], ml, 0, traced=False)

    def level(ell, M):
        r = ref.sample(ell, M)
        return dict(fsums=r["fsums"], diffsums=r["diffsums"], work=r["work"])

    t = time.perf_counter()
    out = nm.mlmc_run_cb(level, targetTOL=tol or REF_MAIN["tol"], M0=REF_MAIN["M0"], verbose=False)
    return dict(seconds=time.perf_counter() - t, threads=threads, Eg=float(out["Eg"]),
                levels=int(out["nlevels"]), total_work=float(out["total_work"]),
                kind="reference", sample="the whole run (every level call of the reference's sampler)")


def ref_main_case(args):
    """The model main of the reference on the GPU (batched FP32 and the FP64 / REF32 drop-ins on
    the reference's streams, 2048 virtual cores) beside the reference's CPU sampler, all under
    the same host driver; each estimate against the exact eta."""
    sys.path.insert(0, PKG)
    import nmlmc as nm
    ml = ref_main_max_loss(nm.norm_cdf_inv)
    runs = {}
    for name, prec, streams, batched in (("fp32_batched", nm.PREC_FP32, nm.STREAMS_OUTER, True),
                                         ("fp64_dropin", nm.PREC_FP64, nm.STREAMS_CORE, False),
                                         ("ref32_dropin", nm.PREC_REF32, nm.STREAMS_CORE, False)):
        s = nm.Sampler(0, cores=2048, N0=REF_MAIN["N0"], beta=REF_MAIN["beta"],
                       adaptive_r=REF_MAIN["adaptive_r"], precision=prec, streams=streams, seed=1)
        s.set_model(nm.MODEL_REFERENCE, REF_MAIN["tau"], ml)
        if prec == nm.PREC_FP32:
            s.set_autotune(2)
        s.mlmc_run(targetTOL=REF_MAIN["tol"], M0=REF_MAIN["M0"], batched=batched)     # warm-up
        if prec == nm.PREC_FP32:
            s.set_autotune(0)                  # the timed run keeps the warm-up's choices
        s.configure(seed=0)
        t = time.perf_counter()
        out = s.mlmc_run(targetTOL=REF_MAIN["tol"], M0=REF_MAIN["M0"], batched=batched)
        runs[name] = dict(value=float(out["level_time"].sum()), e2e=time.perf_counter() - t,
                          Eg=float(out["Eg"]), abs_err_vs_eta=abs(float(out["Eg"]) - REF_MAIN["eta"]),
                          levels=int(out["nlevels"]), total_work=float(out["total_work"]))
    cpu = ref_main_cpu() if not args.no_cpu else {"skipped": True}
    a = runs["fp32_batched"]
    line = {"metric": "time-to-TOL (s), the reference's model main (TOL = 1e-3)", "value": a["value"],
            "unit": "s", "n_gpus": 1, "higher_is_better": False, "dtype": "f32", "data": "synthetic",
            "config": dict(workload="reference model main: tau 0.02, eta 0.025, N0 32, beta 4, r 1.5",
                           **{k: v for k, v in REF_MAIN.items()}),
            "e2e": {"value": a["e2e"], "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": None},
            "runs": runs, "cpu_baseline": cpu, "vs_baseline": None}
    if "seconds" in cpu:
        line["speedup_vs_cpu_reference"] = {"e2e": cpu["seconds"] / a["e2e"]}
    print(json.dumps(line))


# Lane operations per inner time step of an antithetic Milstein pair on the FP32 path (one normal):
#   Threefry2x64-20 block / 4 = 35, SFU Box-Muller pair / 2 = 11, the Milstein update of both
#   paths (dW, dW^2 - h, correction, two growth factors, two products) = 9, loop and select = 3;
#   the adjoint pass adds the sigma-tangent of both paths (8).
C4_OPS_LOSS = 35 + 11 + 9 + 3
C4_OPS_GRAD = C4_OPS_LOSS + 8


def c4_batch(nm, sizes, d, seed):
    """Portfolios of the path-simulated workload: d GBM stocks (S0 = 100, mu = r = 0.05,
    sigma ~ U[0.1, 0.4]); options on uniformly chosen stocks, 50/50 call/put, strike ~
    U[0.8, 1.2] S0, maturity ~ U[0.25, 2], position ~ N(0, 1); numpy PCG64 seeded per portfolio."""
    import numpy as np
    pfs = []
    for k, P in enumerate(sizes):
        g = np.random.default_rng(seed + k)
        si = g.integers(0, d, P).astype(np.uint32)
        pfs.append(dict(S0=np.full(d, 100.0), mu=np.full(d, 0.05), sigma=0.1 + 0.3 * g.random(d),
                        stock_ind=si, type=np.where(g.random(P) < 0.5, 1, -1).astype(np.int32),
                        strike=100.0 * (0.8 + 0.4 * g.random(P)), maturity=0.25 + 1.75 * g.random(P),
                        w=g.standard_normal(P)))
    return nm.make_batch(pfs, [0.0] * len(sizes), r=0.05, rho=0.2, tau=1 / 52)


def c4_case(args, small=False):
    """Path-simulated loss with adjoint gradients (FP32 paths, FP64 sums): one portfolio of
    P = 1e5 options on d = 50 stocks, and 64 portfolios with sizes log-uniform in [1e3, 1e5]
    in one launch; Milstein on 2^ell steps from tau to maturity.  Thresholds K: the median loss
    of a first loss-only pass; sigmoid width delta = 0.01 |K|."""
    import numpy as np
    sys.path.insert(0, PKG)
    import nmlmc as nm
    s = nm.Sampler(precision=nm.PREC_FP32)
    g = np.random.default_rng(2026)
    runs = [("single", [20_000 if small else 100_000], 64 if small else 256)]
    if not small:
        runs.append(("batch64", [int(x) for x in np.exp(g.uniform(np.log(1e3), np.log(1e5), 64))], 64))
    ell, pairs = 4, 4
    for name, sizes, M in runs:
        b = c4_batch(nm, sizes, 50, 7)
        kw = dict(ell=ell, pairs=pairs, M=M, seed=1, delta_rel=0.01)
        b["K"] = np.median(s.path_adjoint(b, grads=False, loss=True, **kw)["loss"], axis=1)
        for _ in range(max(args.warmup, 1)):
            s.path_adjoint(b, **kw)
        t_loss, t_all = [], []
        cs = ClockSampler(0)
        cs.start()
        for _ in range(args.steps):
            t_loss.append(s.path_adjoint(b, grads=False, **kw)["seconds"])
            t_all.append(s.path_adjoint(b, **kw)["seconds"])
        clk = cs.stop()
        sm_mhz = clk.get("sm_mhz") or 1965.0
        peak = 148 * 128 * sm_mhz * 1e6 / 1e12
        P_tot = int(b["option_off"][-1])
        normals = P_tot * M * pairs * (1 << ell)          # antithetic pair steps per pass
        tl, ta = statistics.median(t_loss), statistics.median(t_all)
        tg = ta - tl
        ops = normals * C4_OPS_LOSS / tl
        line = {"metric": f"path-simulated loss + adjoint, {name}", "value": 2 * normals * 2 / ta,
                "unit": "path-steps/s (loss + adjoint passes)", "n_gpus": 1, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ta * 1e3, "higher_is_better": True,
                "dtype": "f32 paths, f64 sums", "data": "synthetic",
                "config": {"workload": name, "portfolios": len(sizes), "options": P_tot, "stocks_per_portfolio": 50,
                           "ell": ell, "steps_per_path": 1 << ell, "inner_pairs": pairs, "M": M,
                           "method": "Milstein", "delta_rel": 0.01},
                "loss_pass_s": tl, "adjoint_pass_s": tg,
                "roofline": {"bound": "alu", "achieved": ops / 1e12, "peak": peak, "unit": "Tops/s",
                             "frac": ops / 1e12 / peak, "traffic": None,
                             "ops_per_pair_step": C4_OPS_LOSS, "kernel": "k_adj_paths (loss pass)",
                             "peak_source": "issue-slot peak 148 SM x 128 lanes x sampled SM clock"},
                "clocks": clk, "vs_baseline": None}
        print(json.dumps(line))


def c3_portfolio(nm):
    """The large-portfolio configuration: generator seed 1, options sorted by |w| (prob ~ |w|)."""
    import numpy as np
    pf = nm.generate_portfolio(nm.PORTFOLIO_C3, 1)
    order = np.argsort(-np.abs(pf["w"]), kind="stable")
    for k in ("strike", "maturity", "w", "stock_ind", "type"):
        pf[k] = pf[k][order]
    return dict(pf, prob=np.abs(pf["w"]))


def c3_level_case():
    """Profiling case of the large-portfolio phase kernel: two level-10 calls of 8192 outer
    samples (9 adaptive pilot phases and the final phase each), then two level-11 calls of 2^18
    outer samples (the level that carries most of the eps = 1e-4 run), with K = 4726.3 (the 99 %
    loss quantile of the large-portfolio configuration)."""
    sys.path.insert(0, PKG)
    import nmlmc as nm
    s = nm.Sampler(0, N0=64, beta=2, adaptive_r=1.5, precision=nm.PREC_FP32, streams=nm.STREAMS_OUTER, seed=5)
    s.set_portfolio(c3_portfolio(nm), r=0.05, rho=0.0, max_loss=4726.308348894119, tau=nm.TAU_WEEK,
                    subsample=nm.SUB_RANDOM, use_delta_cv=True, discount=False)
    for ell, M in ((10, 8192), (10, 8192), (11, 1 << 18), (11, 1 << 18)):
        r = s.sample(ell, M)
        print(f"level {ell} M {M}: {r['seconds'] * 1e3:.3f} ms, {r['stats'][0] / r['seconds']:.3e} inner/s")


def dropin_extrapolated(s, level_M, budget_s=60.0):
    """Device time the plain FP64 drop-in would take for the level counts `level_M`: each level
    timed on a bounded sample (whole calls of at least one outer sample per virtual core, grown
    until a call takes about budget / levels / 4), its cost per outer sample times M."""
    total, detail = 0.0, []
    per_level = budget_s / max(1, len(level_M))
    for ell, M in enumerate(level_M):
        if M == 0:
            continue
        m = 2048
        while True:
            dt = s.sample(ell, m)["seconds"]
            if dt >= per_level / 4 or m >= M or m >= (1 << 24):
                break
            m = min(M, m * max(2, int(per_level / 4 / max(dt, 1e-4))))
        total += dt / m * M
        detail.append(f"l{ell}:{m}")
    return dict(value=total, e2e=None, extrapolated=True,
                sample="per-level device time on bounded samples [" + ", ".join(detail) +
                       " outer samples] x the level counts of the FP32 run")


def c3_sweep_case():
    """Profiling case of the full-portfolio loss sweep (the K-quantile precompute): the large
    portfolio (d = 200, P = 1e6 packed FP32 records), L(Y) for 8192 outer samples, twice."""
    sys.path.insert(0, PKG)
    import nmlmc as nm
    s = nm.Sampler(0, N0=64, beta=2, precision=nm.PREC_FP32, streams=nm.STREAMS_OUTER, seed=1)
    s.set_portfolio(c3_portfolio(nm), r=0.05, rho=0.0, max_loss=0.0, tau=nm.TAU_WEEK,
                    subsample=nm.SUB_RANDOM, use_delta_cv=True, discount=False)
    for _ in range(2):
        t = time.perf_counter()
        L = s.full_loss(62, 0, 8192)
        dt = time.perf_counter() - t
        print(f"sweep 8192 x 1e6 options: {dt * 1e3:.3f} ms (wall), {8192 * 1e6 / dt:.3e} evaluations/s, "
              f"mean loss {L.mean():.3f}")


def c3_table_case():
    """Profiling case: the large-portfolio phase kernel with option tables of 1e6, 1e4, 1e3 and
    100 options (generator seed 1, d = 200, prob ~ |w|), importance and uniform sub-sampling,
    non-adaptive level 6 (4096 inner samples per outer sample) on 2^14 outer samples: how much of
    the time the table's memory latency takes."""
    import numpy as np
    sys.path.insert(0, PKG)
    import nmlmc as nm
    for P in (1_000_000, 10_000, 1_000, 100):
        pf = nm.generate_portfolio(dict(nm.PORTFOLIO_C3, P=P), 1)
        order = np.argsort(-np.abs(pf["w"]), kind="stable")
        for k in ("strike", "maturity", "w", "stock_ind", "type"):
            pf[k] = pf[k][order]
        pf = dict(pf, prob=np.abs(pf["w"]))
        for sub, name in ((nm.SUB_RANDOM, "importance"), (nm.SUB_UNIFORM, "uniform")):
            s = nm.Sampler(0, N0=64, beta=2, adaptive_r=0.0, precision=nm.PREC_FP32,
                           streams=nm.STREAMS_OUTER, seed=5)
            s.set_portfolio(pf, r=0.05, rho=0.0, max_loss=4726.3, tau=nm.TAU_WEEK, subsample=sub,
                            use_delta_cv=True, discount=False)
            s.set_autotune(0)
            for _ in range(3):
                r = s.sample(6, 1 << 14)
            print(f"P {P} {name}: {r['seconds'] * 1e3:.3f} ms, {r['stats'][0] / r['seconds']:.3e} inner/s")


# Path-simulated large portfolio: d = 50 stocks, P = 1e5 options (the large portfolio's generator,
# seed 1), every option valued by coupled fine / coarse Milstein paths from tau to maturity with
# the reference's Unbiased method (sample_inner_unbiased / sample_inner_approx,
# portfolio_sampler.cpp:521-604): h0 = 1, time steps doubling per path level (dt_beta = 2), level
# L drawn with P(L) ~ 2^(-1.5 L), so 2^L Milstein steps (L = 0..8 covers 99.9999 % of the draws).
C4_MLMC = dict(workload="path-simulated portfolio: d=50 GBM stocks, P=1e5 options, Milstein paths (Unbiased "
                        "method, 2^L steps), P(L>K) with K the 99% Black-Scholes loss quantile",
               stocks=50, options=100_000, generator_seed=1, sub_sampling="importance, prob ~ |w_i|",
               delta_cv=True, N0=64, beta=2, adaptive_r=ADAPTIVE_R, dt_h0inv=1, dt_beta=2, dt_prob_expo=-1.5,
               milstein=True, antithetic_risk=True, eps=1e-3)


def c4_mlmc_portfolio(nm):
    """The path-simulated portfolio of the MLMC line: the large portfolio's generator with d = 50,
    P = 1e5 (seed 1), options sorted by |w|, every option on the Unbiased method."""
    import numpy as np
    pf = nm.generate_portfolio(dict(nm.PORTFOLIO_C3, Q=C4_MLMC["stocks"], P=C4_MLMC["options"]), 1)
    order = np.argsort(-np.abs(pf["w"]), kind="stable")
    for k in ("strike", "maturity", "w", "stock_ind", "type"):
        pf[k] = pf[k][order]
    pf = dict(pf, prob=np.abs(pf["w"]))
    methods = dict(method=np.full(len(pf["w"]), nm.METHOD_UNBIASED, np.int32), dt_h0inv=1, dt_beta=2,
                   dt_prob_expo=-1.5, use_milstein=True, use_antithetic_risk=True)
    return pf, methods


def c4_level_case():
    """Profiling case of the path-simulated phase kernel (FP32): two level-8 calls of 4000 outer
    samples and two level-12 calls of 1000, K = 1676.5 (the 99 % Black-Scholes loss quantile)."""
    sys.path.insert(0, PKG)
    import nmlmc as nm
    pf, methods = c4_mlmc_portfolio(nm)
    s = nm.Sampler(0, N0=64, beta=2, adaptive_r=ADAPTIVE_R, precision=nm.PREC_FP32, streams=nm.STREAMS_OUTER, seed=3)
    s.set_portfolio(pf, r=0.05, rho=0.0, max_loss=1676.5013260915875, tau=nm.TAU_WEEK, subsample=nm.SUB_RANDOM,
                    use_delta_cv=True, discount=True, methods=methods)
    for ell, M in ((8, 4000), (8, 4000), (12, 1000), (12, 1000)):
        r = s.sample(ell, M)
        print(f"level {ell} M {M}: {r['seconds'] * 1e3:.3f} ms, {r['stats'][0] / r['seconds']:.3e} inner/s")


def c4_mlmc_case(args):
    """Time-to-eps of the path-simulated portfolio: the batched FP32 sampler (OUTER streams, each
    path-simulated inner sample on its own counter namespaces) against the FP64 drop-in on the
    reference's stream layout (2048 virtual cores), both measured to the same eps."""
    sys.path.insert(0, PKG)
    import nmlmc as nm
    eps = args.eps if args.eps else C4_MLMC["eps"]
    pf, methods = c4_mlmc_portfolio(nm)

    def mk(prec, streams, K, seed, methods_on=True):
        s = nm.Sampler(0, cores=2048, N0=64, beta=2, adaptive_r=ADAPTIVE_R, precision=prec, streams=streams,
                       seed=seed)
        s.set_portfolio(pf, r=0.05, rho=0.0, max_loss=K, tau=nm.TAU_WEEK, subsample=nm.SUB_RANDOM,
                        use_delta_cv=True, discount=True, methods=methods if methods_on else None)
        return s

    q = mk(nm.PREC_FP32, nm.STREAMS_OUTER, 0.0, 1, methods_on=False)
    K = nm.loss_quantile(q, 0.99, 100_000)
    q.close()
    runs = {}
    clk = None
    for name, prec, streams, batched in (("fp32_batched", nm.PREC_FP32, nm.STREAMS_OUTER, True),
                                         ("fp64_dropin", nm.PREC_FP64, nm.STREAMS_CORE, False)):
        s = mk(prec, streams, K, 3)
        s.mlmc_run(targetTOL=3 * eps, M0=1024, batched=batched)      # warm-up at a looser eps
        s.configure(seed=5)
        cs = ClockSampler(0)
        cs.start()
        t = time.perf_counter()
        out = s.mlmc_run(targetTOL=eps, M0=1024, batched=batched)
        wall = time.perf_counter() - t
        c = cs.stop()
        clk = clk or c
        runs[name] = dict(value=float(out["level_time"].sum()), e2e=wall, Eg=float(out["Eg"]),
                          levels=int(out["nlevels"]), starting_level=int(out["starting_level"]),
                          level_M=[int(x) for x in out["level_M"]], work=float(out["total_work"]))
        s.close()
    a, b = runs["fp32_batched"], runs["fp64_dropin"]
    line = {"metric": f"time-to-eps (s) for MLMC P(L>K), path-simulated portfolio, eps={eps:g} absolute",
            "value": a["value"], "unit": "s", "n_gpus": 1, "higher_is_better": False, "dtype": "f32 paths, f64 states",
            "data": "synthetic (seeded generator)", "config": dict(C4_MLMC, eps=eps, K=K),
            "e2e": {"value": a["e2e"], "unit": "s"}, "runs": runs,
            "speedup_vs_fp64_dropin": {"value": b["value"] / a["value"], "e2e": b["e2e"] / a["e2e"]},
            "clocks": clk, "vs_baseline": None}
    print(json.dumps(line))


C2_CONFIG = dict(workload="portfolio: d=20 GBM stocks, P=1e4 European options, uniform sub-sampling, "
                          "64 * 2^ell inner samples, P(L>K) with K the 99% loss quantile of 1e5 full "
                          "evaluations", stocks=20, options=10_000, generator_seed=1, tau="1/52", r=0.05,
                 rho=0.0, sub_sampling="uniform", delta_cv=False, N0=64, beta=2, adaptive_r=0.0,
                 antithetic=True, eps=1e-4, eps_note="the configuration's relative 1e-2 on P(L>K) ~ 0.01")


def c2_case(args):
    """The C2 portfolio to its eps: K from 1e5 full evaluations (seed 1), a direct estimate of
    P(L > K) from 2e6 more, then the batched FP32 sampler to 1e-3 (a warm-up that also tunes the
    levels, then a timed run) and to eps, and the FP64 drop-in on the reference's streams at 1e-3
    beside the FP32 run at 1e-3."""
    import numpy as np
    sys.path.insert(0, PKG)
    import nmlmc as nm
    eps = args.eps if args.eps else C2_CONFIG["eps"]
    pf = nm.generate_portfolio(nm.PORTFOLIO_C2, 1)

    def mk(prec, streams, K, seed):
        s = nm.Sampler(0, cores=2048, N0=64, beta=2, adaptive_r=0.0, precision=prec, streams=streams, seed=seed)
        s.set_portfolio(pf, r=0.05, rho=0.0, max_loss=K, tau=nm.TAU_WEEK, subsample=nm.SUB_UNIFORM,
                        use_delta_cv=False, discount=False)
        return s

    q = mk(nm.PREC_FP32, nm.STREAMS_OUTER, 0.0, 1)
    K = nm.loss_quantile(q, 0.99, 100_000)
    Ld = np.concatenate([q.full_loss(62, k * 500_000, 500_000) for k in range(4)])
    q.close()
    p_direct = float(np.mean(Ld > K))
    sd = float(np.sqrt(p_direct * (1 - p_direct) / len(Ld)))
    runs = {}
    clk = None

    def timed(name, s, e, batched):
        nonlocal clk
        cs = ClockSampler(0)
        cs.start()
        t = time.perf_counter()
        out = s.mlmc_run(targetTOL=e, M0=1024, batched=batched)
        wall = time.perf_counter() - t
        c = cs.stop()
        clk = clk or c
        runs[name] = dict(eps=e, value=float(out["level_time"].sum()), e2e=wall, Eg=float(out["Eg"]),
                          levels=int(out["nlevels"]), starting_level=int(out["starting_level"]),
                          level_M=[int(x) for x in out["level_M"]], work=float(out["total_work"]))

    s = mk(nm.PREC_FP32, nm.STREAMS_OUTER, K, 3)
    s.mlmc_run(targetTOL=1e-3, M0=1024, batched=True)          # warm-up: tunes the levels
    s.configure(seed=5)
    timed("fp32_batched_1e-3", s, 1e-3, True)
    s.configure(seed=7)
    timed("fp32_batched", s, eps, True)
    s.close()
    d = mk(nm.PREC_FP64, nm.STREAMS_CORE, K, 5)
    timed("fp64_dropin_1e-3", d, 1e-3, False)
    d.close()
    a = runs["fp32_batched"]
    line = {"metric": f"time-to-eps (s) for MLMC P(L>K), d=20 portfolio with uniform sub-sampling, eps={eps:g} absolute",
            "value": a["value"], "unit": "s", "n_gpus": 1, "higher_is_better": False, "dtype": "f32",
            "data": "synthetic (seeded generator)", "config": dict(C2_CONFIG, eps=eps, K=K),
            "e2e": {"value": a["e2e"], "unit": "s"}, "runs": runs,
            "direct_estimate": {"p": p_direct, "sd": sd, "outer_samples": len(Ld)},
            "speedup_vs_fp64_dropin_at_1e-3": {
                "value": runs["fp64_dropin_1e-3"]["value"] / runs["fp32_batched_1e-3"]["value"],
                "e2e": runs["fp64_dropin_1e-3"]["e2e"] / runs["fp32_batched_1e-3"]["e2e"]},
            "clocks": clk, "vs_baseline": None}
    print(json.dumps(line))


def c3_sampler(nm, device, pfw, K, prec, streams, seed, cores=2048):
    s = nm.Sampler(device, cores=cores, N0=64, beta=2, adaptive_r=ADAPTIVE_R, precision=prec,
                   streams=streams, seed=seed)
    s.set_portfolio(pfw, r=0.05, rho=0.0, max_loss=K, tau=nm.TAU_WEEK, subsample=nm.SUB_RANDOM,
                    use_delta_cv=True, discount=False)
    return s


def c3_upload_bytes(P: int, Q: int) -> int:
    """Host->device bytes of set_portfolio on the FP32 path: per option seven float arrays of the
    reference-arithmetic table (strike, maturity, V0, w, prob, W_est, CDF), the stock index (4 B),
    the type (1 B), the alias entry (8 B), its sampling probability (4 B) and two packed 32-byte
    records (full-loss and sampler); per stock S0, mu, sigma and the delta coefficient (4 x 4 B)."""
    return P * (7 * 4 + 4 + 1 + 8 + 4 + 2 * 32) + Q * 16


def c3_fp32_vs_fp64(nm, device, pfw, K, level_M, starting_level, m_max=4096):
    """Each active level's FP32 estimate against the all-FP64 batched sampler on the same OUTER
    streams (at most m_max outer samples per level): level means, phi flips, count mismatches."""
    out = []
    for ell, M in enumerate(level_M):
        if ell < starting_level or M == 0:
            continue
        m = min(int(M), m_max)
        x = c3_sampler(nm, device, pfw, K, nm.PREC_FP32, nm.STREAMS_OUTER, seed=17)
        y = c3_sampler(nm, device, pfw, K, nm.PREC_FP64, nm.STREAMS_OUTER, seed=17)
        x.set_autotune(0)
        rx, ry = x.sample(ell, m, trace=True), y.sample(ell, m, trace=True)
        tx, ty = rx["trace"], ry["trace"]
        flip = (tx["phi_f"] != ty["phi_f"]) | (tx["phi_c"] != ty["phi_c"])
        out.append({"level": ell, "M": m,
                    "fEl_fp32_minus_fp64": (rx["fsums"][0] - ry["fsums"][0]) / m,
                    "dEl_fp32_minus_fp64": (rx["diffsums"][0] - ry["diffsums"][0]) / m,
                    "phi_flips": int(flip.sum()),
                    "count_mismatches": int(((tx["count_f"] != ty["count_f"]) | (tx["count_c"] != ty["count_c"])).sum())})
        x.close()
        y.close()
    return out


def c3_main(args):
    """The large-portfolio line (the default): W warm-up runs and K timed runs of the batched FP32
    sampler to eps, each step uploading the portfolio tables from host buffers (set_portfolio)
    and running the host driver; then the comparators (FP64 drop-in on the same GPU, all-FP64 on
    the same streams per level, the reference CPU sampler), the phase kernel's roofline and the
    K-quantile sweep."""
    import numpy as np
    sys.path.insert(0, PKG)
    import nmlmc as nm
    eps = args.eps if args.eps else EPS
    world, rank, local = ddp_env()
    dist = None
    if world > 1:
        import torch
        import torch.distributed as td
        from datetime import timedelta
        torch.cuda.set_device(local)
        td.init_process_group("nccl", timeout=timedelta(seconds=300))
        dist = (td, torch.device("cuda", local))

    def barrier():
        if dist:
            dist[0].barrier()

    pfw = c3_portfolio(nm)
    P, Q = len(pfw["w"]), len(pfw["S0"])
    # K: the 99 % quantile of the full loss over 1e5 outer samples (FP32 sweep of the packed table)
    q = c3_sampler(nm, local, pfw, 0.0, nm.PREC_FP32, nm.STREAMS_OUTER, seed=1)
    K = nm.loss_quantile(q, 0.99, 100_000)
    t = time.perf_counter()
    Ld = q.full_loss(62, 0, 200_000)
    t_sweep = time.perf_counter() - t
    q.close()
    p_direct = float(np.mean(Ld > K))
    sd = float(np.sqrt(p_direct * (1 - p_direct) / len(Ld)))
    sweep = {"outer_samples": len(Ld), "options": P, "seconds": t_sweep,
             "option_evaluations_per_s": len(Ld) * P / t_sweep,
             "note": "wall time of nmlmc_portfolio_full_loss (outer draws, sweep of the packed records "
                     "32 outer samples per pass, 1.6 MB copy back); the 32 MB table is L2-resident"}

    s = c3_sampler(nm, local, pfw, K, nm.PREC_FP32, nm.STREAMS_OUTER, seed=1000)
    s.set_autotune(2)           # the warm-up runs tune every level: variant and chunk length
    for w in range(args.warmup):
        s.configure(seed=1000 + w)
        run_once(nm, s, batched=True, dist=dist, eps=eps)
    # keep the tuned choices fixed for the timed runs (set_portfolio would otherwise drop them)
    nlev_seen = 0
    for ell in range(64):
        pc = s.phase_config(ell)
        if pc["state"] == 1:
            s.set_phase_config(ell, pc["variant"], pc["chunk"])
            nlev_seen = ell + 1
    s.set_autotune(0)

    clocks = ClockSampler(local)
    clocks.start()
    launches0 = nm.kernel_launches()
    barrier()
    dev_times, walls, outs = [], [], []
    t_region = time.perf_counter()
    for k in range(args.steps):
        s.configure(seed=k)
        t0 = time.perf_counter()
        s.set_portfolio(pfw, r=0.05, rho=0.0, max_loss=K, tau=nm.TAU_WEEK, subsample=nm.SUB_RANDOM,
                        use_delta_cv=True, discount=False)
        out, _ = run_once(nm, s, batched=True, dist=dist, eps=eps)
        walls.append(time.perf_counter() - t0)
        outs.append(out)
        dev_times.append(float(out["level_time"].sum()))
    barrier()
    region = time.perf_counter() - t_region
    launches = nm.kernel_launches() - launches0
    clk = clocks.stop()

    dev_t = sum(dev_times) / len(dev_times)
    wall_t = sum(walls) / len(walls)
    if dist:
        import torch
        tt = torch.tensor([dev_t, wall_t], dtype=torch.float64, device=dist[1])
        dist[0].all_reduce(tt, op=dist[0].ReduceOp.MAX)
        dev_t, wall_t = float(tt[0]), float(tt[1])
    a = outs[0]
    level_M = [int(x) for x in a["level_M"]]
    sl = int(a["starting_level"])
    calls = sum(int(o["calls"]) for o in outs) / len(outs)
    inner = sum(float(o["total_work"]) for o in outs)
    if rank != 0:
        if dist:
            dist[0].destroy_process_group()
        return

    schedule = dict(eps=eps, K=K, levels=list(range(len(level_M))), M=level_M, starting_level=sl,
                    note="outer samples per level of the eps run (seed 0) of the batched sampler")
    if args.schedule_out:
        os.makedirs(os.path.dirname(os.path.abspath(args.schedule_out)), exist_ok=True)
        with open(args.schedule_out, "w") as f:
            json.dump({"c3": schedule}, f)

    # phase-kernel roofline: CUDA events around every phase-kernel launch while the sampler repeats
    # one call per active level of the run (at most 2^18 outer samples each; profiling submits the
    # levels one call at a time, outside the timed region)
    s.set_profiling(True)
    prof_inner = 0.0
    for ell, M in enumerate(level_M):
        if ell >= sl and M > 0:
            prof_inner += float(s.sample(ell, min(M, 1 << 18))["stats"][0])
    n_phase, t_phase = s.phase_kernel_time()
    s.set_profiling(False)
    sm_mhz = clk.get("sm_mhz") or 1965.0
    peak = 148 * 128 * sm_mhz * 1e6 / 1e12
    ach = prof_inner * C3_OPS_PER_INNER / t_phase / 1e12
    roof = {"bound": "alu", "achieved": ach, "peak": peak, "unit": "Tops/s", "frac": ach / peak,
            "traffic": None, "kernel": "k_phase (FP32, portfolio)", "launches": n_phase,
            "kernel_seconds": t_phase, "inner_samples": prof_inner, "ops_per_inner_sample": C3_OPS_PER_INNER,
            "peak_source": "issue-slot peak 148 SM x 4 SMSP x 32 lanes x sampled SM clock (the measured-"
                           "peaks file holds only HBM copy and bf16 GEMM figures)",
            "timing": "CUDA events around each phase-kernel launch of one call per active level "
                      "(<= 2^18 outer samples) after the timed runs",
            "traffic_note": "the 40 MB option and alias tables are L2-resident; DRAM traffic per launch "
                            "is the R_tau rows and per-outer-sample counts (profiles/), so no HBM "
                            "roofline applies"}
    line = {"metric": METRIC, "value": dev_t, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_t * 1e3, "higher_is_better": False,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator)",
            "config": dict(C3_CONFIG, eps=eps),
            "e2e": {"value": wall_t, "unit": "s", "h2d_bytes_per_step": c3_upload_bytes(P, Q),
                    "d2h_bytes_per_step": int(calls * (16 * 8 + 2 * 8)),
                    "h2d_note": "set_portfolio from host buffers every step: the reference-arithmetic "
                                "option arrays, the alias table and the two packed FP32 record tables "
                                "(host-side table construction included); each round's level counts "
                                "travel as kernel arguments",
                    "d2h_note": "per sampled level: 16 FP64 sums and two device clock stamps"},
            "roofline": roof, "clocks": clk, "gpu_launches": int(launches),
            "parallelism": f"outer-sample shards x{world}",
            "phase_config": phase_choices(s, max(nlev_seen, len(level_M))),
            "inner_samples_per_step": inner / len(outs), "inner_samples_per_s": inner / sum(dev_times),
            "Eg": float(a["Eg"]), "p_direct": p_direct, "p_direct_sd": sd, "K": K,
            "levels": len(level_M), "starting_level": sl, "level_M": level_M,
            "timed_region_s": region, "full_loss_sweep": sweep}
    s.close()

    if world == 1 and not args.no_compare:
        # plain FP64 drop-in on the same GPU: per-level cost on bounded samples x the level counts
        # of the FP32 run; calibrated by one complete measured run at eps = 1e-3
        d = c3_sampler(nm, local, pfw, K, nm.PREC_FP64, nm.STREAMS_CORE, seed=5, cores=2048)
        drop = dropin_extrapolated(d, level_M, budget_s=60.0) if eps < 5e-4 else None
        d.close()
        cal_eps = 1e-3
        f = c3_sampler(nm, local, pfw, K, nm.PREC_FP32, nm.STREAMS_OUTER, seed=6)
        f.set_autotune(1)
        of, _ = run_once(nm, f, batched=True, eps=cal_eps)
        f.close()
        d = c3_sampler(nm, local, pfw, K, nm.PREC_FP64, nm.STREAMS_CORE, seed=6, cores=2048)
        od, wd = run_once(nm, d, batched=False, eps=cal_eps)
        d.close()
        d = c3_sampler(nm, local, pfw, K, nm.PREC_FP64, nm.STREAMS_CORE, seed=6, cores=2048)
        ext = dropin_extrapolated(d, [int(x) for x in of["level_M"]], budget_s=20.0)
        d.close()
        cal = {"eps": cal_eps, "measured_s": float(od["level_time"].sum()), "measured_e2e_s": wd,
               "extrapolated_s": ext["value"], "Eg": float(od["Eg"]),
               "extrapolated_over_measured": ext["value"] / float(od["level_time"].sum()),
               "fp32_batched_s": float(of["level_time"].sum()),
               "note": "the drop-in's own complete run at this eps, and the per-level extrapolation "
                       "from the FP32 run's level counts at the same eps"}
        if drop is None:
            drop = {"value": float(od["level_time"].sum()), "e2e": wd, "extrapolated": False}
        drop["calibration"] = cal
        drop["streams"] = "reference (CORE) layout, 2048 virtual cores, one synchronous call per level"
        line["fp64_dropin"] = drop
        line["speedup_vs_fp64_dropin"] = {"value": drop["value"] / dev_t,
                                          "note": "extrapolated drop-in time over the measured FP32 time"
                                                  if drop.get("extrapolated") else "measured"}
        line["fp32_vs_fp64_per_level"] = c3_fp32_vs_fp64(nm, local, pfw, K, level_M, sl)
    if world == 1 and not args.no_cpu:
        line["cpu_baseline"] = c3_cpu_baseline(nm, pfw, K, schedule, budget_s=args.ref_budget,
                                               calibrate_s=args.ref_budget)
    print(json.dumps(line))
    if dist:
        dist[0].destroy_process_group()


# ---------------------------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ref-budget", type=float, default=20.0, help="CPU seconds of reference sampling")
    ap.add_argument("--no-compare", action="store_true", help="skip the FP64 comparison runs")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--eps", type=float, default=None, help="target RMSE of the large-portfolio line (default 1e-4)")
    ap.add_argument("--schedule-out", default=None,
                    help="write the run's outer samples per level (bench_schedule.json format) here")
    ap.add_argument("--case", default=None, choices=["c1", "c2", "small", "c3-level", "c3-table", "c3-sweep", "c4",
                                                      "c4-small", "c4-mlmc", "c4-level", "ref-model"],
                    help="default: the large portfolio to eps; c1: the adaptive model problem to eps; "
                         "c2: the d=20 portfolio with uniform sub-sampling to eps; c4: the "
                         "path-simulated loss with adjoint; c4-mlmc: MLMC of the path-simulated "
                         "portfolio to eps; ref-model: the reference's model main; small, c3-level, "
                         "c3-table, c3-sweep, c4-small, c4-level: profiling cases")
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    if args.case is None:
        return c3_main(args)
    if args.case == "c1":
        return c1_main(args)
    if args.case == "small":
        return small_case()
    if args.case == "c3-level":
        return c3_level_case()
    if args.case == "c3-table":
        return c3_table_case()
    if args.case == "c3-sweep":
        return c3_sweep_case()
    if args.case == "c4-mlmc":
        return c4_mlmc_case(args)
    if args.case == "c2":
        return c2_case(args)
    if args.case == "c4-level":
        return c4_level_case()
    if args.case in ("c4", "c4-small"):
        return c4_case(args, small=args.case == "c4-small")
    if args.case == "ref-model":
        return ref_main_case(args)


def c1_main(args):
    """The adaptive model problem to eps = 1e-4 (X = Y + Z, K = 1): W warm-up and K timed runs of
    the batched FP32 sampler, the all-FP64 run and the FP64 drop-in on the same GPU, the per-level
    FP32 error, the phase kernel's roofline and the reference CPU sampler."""
    sys.path.insert(0, PKG)
    import nmlmc as nm
    world, rank, local = ddp_env()
    dist = None
    if world > 1:
        import torch
        import torch.distributed as td
        from datetime import timedelta
        torch.cuda.set_device(local)
        td.init_process_group("nccl", timeout=timedelta(seconds=120))
        dist = (td, torch.device("cuda", local))

    s = make_sampler(nm, local, nm.PREC_FP32, nm.STREAMS_OUTER, seed=0)
    if world > 1:
        s.set_shard(rank, world)

    def barrier():
        if dist:
            dist[0].barrier()

    for w in range(args.warmup):
        s.configure(seed=1000 + w)
        run_once(nm, s, batched=True, dist=dist)
    s.set_autotune(0)       # the warm-up tuned the levels; the timed runs keep those choices

    clocks = ClockSampler(local)
    clocks.start()
    launches0 = nm.kernel_launches()
    barrier()
    dev_times, walls, outs = [], [], []
    t_region = time.perf_counter()
    for k in range(args.steps):
        s.configure(seed=k)
        out, wall = run_once(nm, s, batched=True, dist=dist)
        outs.append(out)
        walls.append(wall)
        dev_times.append(float(out["level_time"].sum()))
    barrier()
    region = time.perf_counter() - t_region
    launches = nm.kernel_launches() - launches0
    clk = clocks.stop()
    # The phase kernel's own time: a profiled repeat of the timed runs (same seeds) with CUDA
    # events around every phase-kernel launch; profiling submits the levels one call at a time
    # (event pairs have no elapsed time inside a graph), so it stays out of the timed region.
    s.set_profiling(True)
    inner_prof = 0.0
    for k in range(args.steps):
        s.configure(seed=k)
        o, _ = run_once(nm, s, batched=True, dist=dist)
        inner_prof += float(o["total_work"])
    n_phase, t_phase = s.phase_kernel_time()
    s.set_profiling(False)

    dev_t = sum(dev_times) / len(dev_times)
    wall_t = sum(walls) / len(walls)
    if dist:
        import torch
        t = torch.tensor([dev_t, wall_t], dtype=torch.float64, device=dist[1])
        dist[0].all_reduce(t, op=dist[0].ReduceOp.MAX)
        dev_t, wall_t = float(t[0]), float(t[1])

    inner = sum(float(o["total_work"]) for o in outs)  # work = inner samples for this model
    calls = sum(int(o["calls"]) for o in outs)
    if rank != 0:
        if dist:
            dist[0].destroy_process_group()
        return

    ref = outs[0]
    schedule = dict(eps=EPS, levels=list(range(int(ref["nlevels"]))),
                    M=[int(x) for x in ref["level_M"]],
                    note="outer samples per level of the eps run (seed 0) of the batched sampler")
    if args.schedule_out:          # the level counts of this run (the reference arm's schedule)
        os.makedirs(os.path.dirname(os.path.abspath(args.schedule_out)), exist_ok=True)
        with open(args.schedule_out, "w") as f:
            json.dump({"c1": schedule}, f)

    # roofline of the phase kernel (the dominant kernel): lane-ops per inner sample x inner
    # samples / its CUDA-event time; peak = issue slots at the sampled SM clock
    sm_mhz = clk.get("sm_mhz") or 1965.0
    achieved = inner_prof * OPS_PER_INNER / t_phase / 1e9 if t_phase > 0 else None
    peak = 148 * 128 * sm_mhz * 1e6 / 1e9
    roof = {"bound": "alu", "achieved": achieved, "peak": peak, "unit": "Gop/s",
            "frac": (achieved / peak) if achieved else None, "traffic": None,
            "kernel": "k_phase (FP32, X=Y+Z)", "launches": n_phase,
            "kernel_seconds": t_phase, "ops_per_inner_sample": OPS_PER_INNER,
            "timing": "CUDA events around every phase-kernel launch in a profiled repeat of the timed "
                      "runs (same seeds, levels submitted one call at a time)",
            "traffic_note": "DRAM bytes per level-0 launch (ncu): 8 B per outer sample (Y and counts); "
                            "no input data, so no HBM roofline applies",
            "peak_source": "issue-slot peak 148 SM x 4 SMSP x 32 lanes x sampled SM clock "
                           "(not in the measured-peaks file, which holds HBM and bf16 GEMM)"}

    line = {"metric": METRIC, "value": dev_t, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_t * 1e3, "higher_is_better": False,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": C1_WORKLOAD, "parallelism": f"outer-sample shards x{world}",
            "phase_config": phase_choices(s, int(ref["nlevels"])),
            "e2e": {"value": wall_t, "unit": "s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": int(calls / len(outs) * (16 * 8 + 2 * 8)),
                    "h2d_note": "no input arrays: tau, K and each round's level counts travel as kernel "
                                "arguments of the round's graph",
                    "d2h_note": "per sampled level: 16 FP64 sums and two device clock stamps"},
            "roofline": roof, "clocks": clk, "gpu_launches": int(launches),
            "inner_samples_per_step": inner / len(outs),
            "inner_samples_per_s": inner / sum(dev_times),
            "Eg": float(ref["Eg"]), "abs_err_vs_exact": abs(float(ref["Eg"]) - exact_p()),
            "timed_region_s": region}

    if world == 1 and not args.no_compare:
        s64 = make_sampler(nm, local, nm.PREC_FP64, nm.STREAMS_OUTER, seed=0)
        run_once(nm, s64, batched=True)
        s64.configure(seed=0)
        o64, w64 = run_once(nm, s64, batched=True)
        line["fp64_same_streams"] = {
            "value": float(o64["level_time"].sum()), "e2e": w64, "Eg": float(o64["Eg"]),
            "Eg_diff_vs_fp32": float(o64["Eg"]) - float(ref["Eg"]),
            "level_M_equal": bool((o64["level_M"] == ref["level_M"]).all()) if len(o64["level_M"]) == len(ref["level_M"]) else False}
        sdrop = make_sampler(nm, local, nm.PREC_FP64, nm.STREAMS_CORE, seed=0, cores=2048)
        od, wd = run_once(nm, sdrop, batched=False)
        line["fp64_dropin"] = {"value": float(od["level_time"].sum()), "e2e": wd, "Eg": float(od["Eg"]),
                               "streams": "reference (CORE) layout, 2048 virtual cores, per-call launches"}
        line["speedup_vs_fp64_dropin"] = {"value": line["fp64_dropin"]["value"] / dev_t,
                                          "e2e": wd / wall_t}
        line["speedup_vs_fp64_same_streams"] = {"value": line["fp64_same_streams"]["value"] / dev_t,
                                                "e2e": w64 / wall_t}
        line["fp32_vs_fp64_per_level"] = per_level_error(nm, local, int(ref["nlevels"]))
    if world == 1 and not args.no_cpu:
        v, kind, cores, desc = cpu_reference_time(schedule, budget_s=args.ref_budget)
        line["cpu_baseline"] = {"value": v, "unit": "s", "cores": cores, "kind": kind, "sample": desc}
    print(json.dumps(line))
    if dist:
        dist[0].destroy_process_group()


if __name__ == "__main__":
    main()
