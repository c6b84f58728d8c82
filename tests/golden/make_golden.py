"""Generates the golden fixtures of this directory from the UNMODIFIED reference.

Runs oracle/_ref/libref_*.so — the reference sources compiled where they lie by oracle/Makefile
(`make -C oracle ref`) — and records its outputs:

  cases.json   case parameters and scalar results (level sums, work, inner_stats, ABI sizes,
               MLMC driver runs)
  arrays.npz   Threefry blocks, random_state draw scripts, Box-Muller pairs, per-call event logs
               (sample_outer / init_inner_sampler(count) / add_phi(mean, coeff)), BS prices

Usage (in a checkout with the reference available):  python tests/golden/make_golden.py
The tests compare the CPU oracle (oracle/nmlmc_oracle.c) and the GPU library against these.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

ETA = 0.025
TAU = 0.02


def model_max_loss() -> float:
    # model_sampler.cpp:144: max_loss = tau * (norm_cdf_inv(eta / 2)^2 - 1), in real_t = float
    x = np.float32(O.Reference("f32").L.ref_norm_cdf_inv(ETA / 2))
    return float(np.float32(TAU) * (np.float32(x) * np.float32(x) - np.float32(1)))


def engine_cases():
    ml = model_max_loss()
    pf_u = dict(Q=4, P=64, seed=3, prob="uniform")
    pf_w = dict(Q=3, P=50, seed=5, prob="w")
    pf_1 = dict(Q=1, P=20, seed=7, prob="uniform")
    pf_n = dict(Q=5, P=40, seed=9, prob="w")
    pf_m = dict(Q=3, P=24, seed=21, prob="w")
    pf_m2 = dict(Q=2, P=12, seed=22, prob="uniform")
    pf_m3 = dict(Q=2, P=6, seed=23, prob="w")
    g = np.random.default_rng(2024)
    methods_m = [int(x) for x in g.integers(0, 3, 24)]
    methods_m2 = [int(x) for x in g.integers(0, 3, 12)]
    methods_m3 = [0, 1, 2, 1, 2, 0]
    return [
        dict(name="A_refmodel_b4_r15", kind="model", model=0, tau=TAU, max_loss=ml, cores=3, N0=32,
             beta=4, r=1.5, anti=True, seed=0, calls=[(0, 40), (1, 40), (2, 30), (3, 20), (1, 17)]),
        dict(name="B_shift_b2_nonadapt", kind="model", model=1, tau=0.0, max_loss=1.0, cores=4, N0=32,
             beta=2, r=0.0, anti=True, seed=0, calls=[(0, 25), (1, 25), (3, 25), (5, 25)]),
        dict(name="C_shift_b2_r15", kind="model", model=1, tau=0.0, max_loss=1.0, cores=2, N0=32,
             beta=2, r=1.5, anti=True, seed=11, calls=[(0, 25), (2, 25), (4, 25), (6, 25)], lzcnt=True),
        dict(name="D_shift_b2_r2minus", kind="model", model=1, tau=0.0, max_loss=1.0, cores=3, N0=32,
             beta=2, r=float(np.nextafter(np.float32(2), np.float32(0))), anti=True, seed=2,
             calls=[(1, 20), (3, 20), (5, 20)], lzcnt=True),
        dict(name="E_refmodel_nonanti", kind="model", model=0, tau=TAU, max_loss=ml, cores=2, N0=32,
             beta=4, r=1.5, anti=False, seed=4, calls=[(0, 20), (1, 20), (2, 20)]),
        dict(name="F_pf_uniform", kind="portfolio", pf=pf_u, sub=O.SUB_UNIFORM, cv=False, rho=0.0,
             max_loss=0.5, cores=3, N0=64, beta=2, r=0.0, anti=True, seed=5,
             calls=[(0, 20), (1, 20), (2, 20), (3, 20)]),
        dict(name="G_pf_cdf_cv", kind="portfolio", pf=pf_w, sub=O.SUB_RANDOM, cv=True, rho=0.2,
             max_loss=0.3, cores=2, N0=32, beta=4, r=1.5, anti=True, seed=5,
             calls=[(0, 20), (1, 20), (2, 20), (3, 20)]),
        dict(name="H_pf_q1_cv", kind="portfolio", pf=pf_1, sub=O.SUB_UNIFORM, cv=True, rho=0.2,
             max_loss=0.1, cores=3, N0=32, beta=4, r=1.5, anti=True, seed=5,
             calls=[(0, 20), (1, 20), (2, 20), (3, 20)]),
        dict(name="I_pf_none", kind="portfolio", pf=pf_n, sub=O.SUB_NONE, cv=False, rho=0.3,
             max_loss=0.4, cores=3, N0=32, beta=4, r=1.5, anti=True, seed=5,
             calls=[(0, 10), (1, 10), (2, 10)]),
        # mixed compute methods (0 BS, 1 Exact, 2 Unbiased): path-simulated inner samples
        dict(name="J_pf_methods_cdf_cv", kind="portfolio", pf=pf_m, methods=methods_m,
             sub=O.SUB_RANDOM, cv=True, rho=0.2, max_loss=0.3, cores=3, N0=32, beta=4, r=1.5,
             anti=True, seed=6, anti_risk=True, milstein=True, coarse_cv=False,
             calls=[(0, 16), (1, 16), (2, 12)]),
        dict(name="K_pf_methods_euler", kind="portfolio", pf=pf_m2, methods=methods_m2,
             sub=O.SUB_UNIFORM, cv=True, rho=0.0, max_loss=0.2, cores=2, N0=32, beta=2, r=1.5,
             anti=True, seed=8, anti_risk=False, milstein=False, coarse_cv=True, lzcnt=True,
             calls=[(0, 12), (2, 12), (3, 8)]),
        dict(name="L_pf_methods_none", kind="portfolio", pf=pf_m3, methods=methods_m3,
             sub=O.SUB_NONE, cv=True, rho=0.3, max_loss=0.4, cores=3, N0=32, beta=4, r=1.5,
             anti=True, seed=9, anti_risk=True, milstein=True, coarse_cv=True,
             calls=[(0, 6), (1, 6)]),
    ]


def run_engine_case(case: dict, variant: str, arrays: dict) -> dict:
    ref = O.Reference(variant)
    ref.init(case["cores"], case["N0"], case["beta"], case["r"], case["anti"])
    out = dict(variant=variant, calls=[])
    if case["kind"] == "model":
        ref.model_init(case["model"], case["tau"], case["max_loss"], case["seed"], traced=True)
    else:
        pf = O.synthetic_portfolio(**case["pf"])
        if "methods" in case:
            ref.portfolio_init_methods(pf, case["methods"], r=0.05, rho=case["rho"],
                                       max_loss=case["max_loss"], tau=1 / 52,
                                       subsample=case["sub"], use_delta_cv=case["cv"],
                                       use_coarse_delta_cv=case["coarse_cv"],
                                       use_antithetic_risk=case["anti_risk"],
                                       use_milstein=case["milstein"], seed=case["seed"], traced=True)
            return _record_calls(case, variant, ref, arrays, out)
        start, delta = ref.portfolio_init(pf, r=0.05, rho=case["rho"], max_loss=case["max_loss"],
                                          tau=1 / 52, subsample=case["sub"], use_delta_cv=case["cv"],
                                          seed=case["seed"], traced=True)
        key = f"{case['name']}/{variant}"
        arrays[key + "/start"] = start
        arrays[key + "/delta_est"] = delta
    return _record_calls(case, variant, ref, arrays, out)


def _record_calls(case: dict, variant: str, ref, arrays: dict, out: dict) -> dict:
    for i, (ell, M) in enumerate(case["calls"]):
        r = ref.sample(ell, M, events_cap=2_000_000)
        key = f"{case['name']}/{variant}/{i}"
        kinds, vals, aux = r["events"]
        arrays[key + "/kinds"] = np.frombuffer(kinds.encode(), np.uint8)
        arrays[key + "/values"] = vals
        arrays[key + "/aux"] = aux
        out["calls"].append(dict(ell=ell, M=M, fsums=r["fsums"].tolist(), diffsums=r["diffsums"].tolist(),
                                 work=r["work"], stats=[int(x) for x in r["stats"]]))
    return out


def main():
    if not O.ref_available("f32"):
        sys.exit("oracle/_ref is not built: run `make -C oracle ref` where the reference is present")
    arrays: dict = {}
    meta: dict = {}
    rng = np.random.default_rng(20261203)

    # Threefry2x64-20 blocks, edge values included
    ctr = rng.integers(0, 2**64, (64, 2), dtype=np.uint64, endpoint=False)
    key = rng.integers(0, 2**64, (64, 2), dtype=np.uint64, endpoint=False)
    ctr[0] = [0, 0]; key[0] = [0, 0]
    ctr[1] = [2**64 - 1, 2**64 - 1]; key[1] = [2**64 - 1, 2**64 - 1]
    ctr[2] = [2**64 - 1, 0]; key[2] = [0, 7]
    ref = O.Reference("f32")
    arrays["threefry/ctr"] = ctr
    arrays["threefry/key"] = key
    arrays["threefry/out"] = ref.threefry(ctr, key)

    # random_state draw scripts
    ops = "".join(rng.choice(list("runnu"), 3000))
    meta["stream_ops"] = ops
    for variant in ("f32", "f64"):
        R = O.Reference(variant)
        for (s, c) in [(0, 0), (7, 3), (2**63 + 5, 2**32 + 1)]:
            real, u64 = R.stream_draws(s, c, ops)
            arrays[f"stream/{variant}/{s}/{c}/real"] = real
            arrays[f"stream/{variant}/{s}/{c}/u64"] = u64

    # Box-Muller on 64-bit words
    u0 = rng.integers(0, 2**64, 256, dtype=np.uint64, endpoint=False)
    u1 = rng.integers(0, 2**64, 256, dtype=np.uint64, endpoint=False)
    u0[0], u1[0] = 0, 0
    u0[1], u1[1] = 2**64 - 1, 2**64 - 1
    x, y = ref.boxmuller(u0, u1)
    arrays["bm/u0"], arrays["bm/u1"], arrays["bm/x"], arrays["bm/y"] = u0, u1, x, y

    # norm_cdf_inv (common.cpp:53-86), real_t = float
    ps = np.array([1e-6, 0.001, 0.0125, 0.02425, 0.1, 0.5, 0.9, 0.97575, 0.999, 1 - 1e-6])
    arrays["ncdfinv/p"] = ps
    arrays["ncdfinv/f32"] = np.array([O.Reference("f32").L.ref_norm_cdf_inv(p) for p in ps])
    arrays["ncdfinv/f64"] = np.array([O.Reference("f64").L.ref_norm_cdf_inv(p) for p in ps])

    # Black-Scholes price / delta as the reference evaluates them
    n = 200
    S = 80 + 40 * rng.random(n)
    K = 80 + 40 * rng.random(n)
    t = 0.05 + 2 * rng.random(n)
    sg = 0.05 + 0.4 * rng.random(n)
    arrays["bs/S"], arrays["bs/K"], arrays["bs/t"], arrays["bs/sigma"] = S, K, t, sg
    for variant in ("f32", "f64"):
        R = O.Reference(variant)
        for ty in (1, -1):
            pr = np.zeros(n)
            de = np.zeros(n)
            R.L.ref_bs(ty, O._p(S, O._dp), O._p(K, O._dp), 0.05, O._p(t, O._dp), O._p(sg, O._dp),
                       O._p(pr, O._dp), O._p(de, O._dp), n)
            arrays[f"bs/{variant}/{ty}/price"] = pr
            arrays[f"bs/{variant}/{ty}/delta"] = de

    # engine cases
    meta["engine"] = []
    for case in engine_cases():
        c = {k: v for k, v in case.items() if k != "pf"}
        if "pf" in case:
            c["pf"] = case["pf"]
        c["results"] = {}
        for prec in ("f32", "f64"):
            variant = prec + ("_lzcnt" if case.get("lzcnt") else "")
            c["results"][prec] = run_engine_case(case, variant, arrays)
        meta["engine"].append(c)

    # host MLMC driver on a synthetic level sampler
    meta["mlmc"] = []
    for (tol, M0, a, alpha, v, beta, w, gamma, seed) in [
            (1e-2, 100, 0.5, 1.0, 0.2, 1.5, 1.0, 1.0, 1),
            (3e-3, 50, 0.8, 1.0, 0.1, 1.0, 2.0, 1.5, 2),
            (1e-3, 100, 0.3, 2.0, 0.05, 2.0, 1.0, 1.0, 3)]:
        r = ref.mlmc_synthetic(tol, M0, a, alpha, v, beta, w, gamma, seed)
        meta["mlmc"].append(dict(args=[tol, M0, a, alpha, v, beta, w, gamma, seed],
                                 calls_ell=r["calls_ell"].tolist(),
                                 calls_M=[int(x) for x in r["calls_M"]],
                                 levels=r["levels"].tolist(), misc=r["misc"].tolist(),
                                 table=r["table"]))

    meta["abi_sizes"] = [int(x) for x in ref.abi_sizes()]
    meta["model_max_loss_f32"] = model_max_loss()

    with open(os.path.join(HERE, "cases.json"), "w") as f:
        json.dump(meta, f, indent=1)
    np.savez_compressed(os.path.join(HERE, "arrays.npz"), **arrays)
    print("wrote", len(arrays), "arrays;", len(meta["engine"]), "engine cases")


if __name__ == "__main__":
    main()
