"""ctypes front-end to the CPU checkers — TEST INFRASTRUCTURE ONLY.

Loads oracle/_build/liboracle.so (the C restatement, oracle/nmlmc_oracle.c) and, when present,
oracle/_ref/libref_*.so (the unmodified reference sources compiled by oracle/Makefile).  Only
tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs import this module;
the product never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

PREC_REF32, PREC_FP64 = 0, 1
STREAMS_CORE, STREAMS_OUTER = 0, 1
MODEL_REFERENCE, MODEL_SHIFT = 0, 1
SUB_NONE, SUB_RANDOM, SUB_UNIFORM = 0, 1, -1

_u64p = ctypes.POINTER(ctypes.c_uint64)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_i32p = ctypes.POINTER(ctypes.c_int32)
_dp = ctypes.POINTER(ctypes.c_double)


class TraceRec(ctypes.Structure):
    _fields_ = [("count_f", ctypes.c_uint64), ("count_c", ctypes.c_uint64),
                ("phi_f", ctypes.c_double), ("phi_c", ctypes.c_double),
                ("mean_big", ctypes.c_double), ("min_abs_small", ctypes.c_double),
                ("core", ctypes.c_uint32), ("pilots", ctypes.c_uint32)]


TRACE_DTYPE = np.dtype([("count_f", np.uint64), ("count_c", np.uint64), ("phi_f", np.float64),
                        ("phi_c", np.float64), ("mean_big", np.float64),
                        ("min_abs_small", np.float64), ("core", np.uint32), ("pilots", np.uint32)])
assert TRACE_DTYPE.itemsize == ctypes.sizeof(TraceRec)


class Events(ctypes.Structure):
    _fields_ = [("kinds", ctypes.c_char_p), ("values", _dp), ("aux", _dp),
                ("cap", ctypes.c_uint64), ("n", ctypes.c_uint64)]


def _p(a, t):
    return a.ctypes.data_as(t)


def build_oracle(quiet: bool = True) -> str:
    """Builds oracle/_build/liboracle.so with make (gcc only; seconds)."""
    out = subprocess.run(["make", "-C", HERE, "_build/liboracle.so"], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    return ORACLE_SO


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO) or _stale():
            build_oracle()
        _lib = ctypes.CDLL(ORACLE_SO)
        _lib.o_create.restype = ctypes.c_void_p
        _lib.o_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32,
                                  ctypes.c_uint32, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_uint64]
        _lib.o_destroy.argtypes = [ctypes.c_void_p]
        _lib.o_set_model.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        _lib.o_set_portfolio.restype = ctypes.c_int
        _lib.o_set_portfolio.argtypes = [ctypes.c_void_p, ctypes.c_uint32, _dp, _dp, _dp,
                                         ctypes.c_uint32, _dp, _dp, _dp, _u32p, _i32p, _dp,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         _dp, _dp]
        _lib.o_sample.restype = ctypes.c_int
        _lib.o_sample.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, _dp, _dp, _dp,
                                  _u64p, ctypes.c_void_p, ctypes.c_void_p]
        _lib.o_portfolio_full_loss.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64,
                                               ctypes.c_uint64, _dp]
        _lib.o_threefry_batch.argtypes = [_u64p, _u64p, _u64p, ctypes.c_uint64]
        _lib.o_stream_draws.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64,
                                        ctypes.c_char_p, ctypes.c_uint64, _dp, _u64p]
        _lib.o_boxmuller.argtypes = [_u64p, _u64p, _dp, _dp, ctypes.c_uint64]
        _lib.o_norm_cdf_inv.restype = ctypes.c_double
        _lib.o_norm_cdf_inv.argtypes = [ctypes.c_double, ctypes.c_int]
    return _lib


def _stale() -> bool:
    so = os.path.getmtime(ORACLE_SO)
    return any(os.path.getmtime(os.path.join(HERE, f)) > so
               for f in ("nmlmc_oracle.c", "nmlmc_oracle.h", "nmlmc_oracle_body.inc", "adjoint_oracle.c"))


def threefry(ctr: np.ndarray, key: np.ndarray) -> np.ndarray:
    ctr = np.ascontiguousarray(ctr, np.uint64).reshape(-1, 2)
    key = np.ascontiguousarray(key, np.uint64).reshape(-1, 2)
    out = np.zeros_like(ctr)
    lib().o_threefry_batch(_p(ctr, _u64p), _p(key, _u64p), _p(out, _u64p), len(ctr))
    return out


def stream_draws(prec: int, seed: int, core: int, ops: str):
    n = len(ops)
    r = np.zeros(n)
    u = np.zeros(n, np.uint64)
    lib().o_stream_draws(prec, seed, core, ops.encode(), n, _p(r, _dp), _p(u, _u64p))
    return r, u


def boxmuller(u0, u1):
    u0 = np.ascontiguousarray(u0, np.uint64)
    u1 = np.ascontiguousarray(u1, np.uint64)
    x = np.zeros(len(u0))
    y = np.zeros(len(u0))
    lib().o_boxmuller(_p(u0, _u64p), _p(u1, _u64p), _p(x, _dp), _p(y, _dp), len(u0))
    return x, y


def norm_cdf_inv(p: float, prec: int = PREC_REF32) -> float:
    return lib().o_norm_cdf_inv(p, prec)


class Sampler:
    """One oracle context: a nested sampler with its model or portfolio, seed and stream layout."""

    def __init__(self, prec=PREC_REF32, streams=STREAMS_CORE, cores=1, N0=32, beta=2,
                 adaptive_r=0.0, antithetic=True, adaptive_incl_r2=False, seed=0):
        self.L = lib()
        self.h = self.L.o_create(prec, streams, cores, N0, beta, adaptive_r, int(antithetic),
                                 int(adaptive_incl_r2), seed)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.o_destroy(self.h)
            self.h = None

    def set_model(self, kind: int, tau: float = 0.0, max_loss: float = 1.0):
        self.L.o_set_model(self.h, kind, tau, max_loss)

    def set_portfolio(self, pf: dict, r=0.05, rho=0.0, max_loss=0.0, tau=1 / 52,
                      subsample=SUB_UNIFORM, use_delta_cv=False, discount=True):
        Q = len(pf["S0"])
        P = len(pf["strike"])
        d = {k: np.ascontiguousarray(pf[k], np.float64) for k in
             ("S0", "mu", "sigma", "strike", "maturity", "w", "prob")}
        si = np.ascontiguousarray(pf["stock_ind"], np.uint32)
        ty = np.ascontiguousarray(pf["type"], np.int32)
        start = np.zeros(P)
        delta = np.zeros(P)
        rc = self.L.o_set_portfolio(self.h, Q, _p(d["S0"], _dp), _p(d["mu"], _dp),
                                    _p(d["sigma"], _dp), P, _p(d["strike"], _dp),
                                    _p(d["maturity"], _dp), _p(d["w"], _dp), _p(si, _u32p),
                                    _p(ty, _i32p), _p(d["prob"], _dp), r, rho, max_loss, tau,
                                    subsample, int(use_delta_cv), int(discount),
                                    _p(start, _dp), _p(delta, _dp))
        if rc != 0:
            raise ValueError("invalid portfolio (stock index, or prob not positive/non-increasing)")
        return start, delta

    def set_portfolio_methods(self, pf: dict, method, r=0.05, rho=0.0, max_loss=0.0, tau=1 / 52,
                              subsample=SUB_RANDOM, use_delta_cv=False, use_coarse_delta_cv=False,
                              use_antithetic_risk=True, use_milstein=True, dt_h0inv=8, dt_beta=4,
                              dt_prob_expo=-1.5):
        """Mixed compute methods (0 BS, 1 Exact, 2 Unbiased); on the OUTER layout with sub-sampling
        (each path-simulated inner sample draws from its own counter namespaces)."""
        L = _methods_bind()
        Q = len(pf["S0"])
        P = len(pf["strike"])
        d = {k: np.ascontiguousarray(pf[k], np.float64) for k in
             ("S0", "mu", "sigma", "strike", "maturity", "w", "prob")}
        si = np.ascontiguousarray(pf["stock_ind"], np.uint32)
        ty = np.ascontiguousarray(pf["type"], np.int32)
        me = np.ascontiguousarray(method, np.int32)
        rc = L.o_set_portfolio_methods(self.h, Q, _p(d["S0"], _dp), _p(d["mu"], _dp),
                                       _p(d["sigma"], _dp), P, _p(d["strike"], _dp),
                                       _p(d["maturity"], _dp), _p(d["w"], _dp), _p(si, _u32p),
                                       _p(ty, _i32p), _p(d["prob"], _dp), _p(me, _i32p), r, rho,
                                       max_loss, tau, subsample, int(use_delta_cv),
                                       int(use_coarse_delta_cv), int(use_antithetic_risk),
                                       int(use_milstein), dt_h0inv, dt_beta, dt_prob_expo)
        if rc == -2:
            raise ValueError("path-simulated compute methods on the OUTER layout need sub-sampling")
        if rc != 0:
            raise ValueError("invalid portfolio (stock index, or prob not positive/non-increasing)")

    def sample(self, ell: int, M: int, trace: bool = False, events_cap: int = 0, margins: bool = False):
        """One sample(ell, M) call; with `margins`, out["margins"][m] is the smallest
        |ln(new_count / cur)| of outer sample m's adaptive decisions (o_set_margins)."""
        f = np.zeros(4)
        dd = np.zeros(4)
        w = np.zeros(1)
        st = np.zeros(6, np.uint64)
        tr = np.zeros(M, TRACE_DTYPE) if trace else None
        ev = None
        bufs = None
        if events_cap:
            kinds = ctypes.create_string_buffer(events_cap)
            vals = np.zeros(events_cap)
            aux = np.zeros(events_cap)
            bufs = (kinds, vals, aux)
            ev = Events(ctypes.cast(kinds, ctypes.c_char_p), _p(vals, _dp), _p(aux, _dp), events_cap, 0)
        mg = None
        if margins:
            mg = np.full(M, np.inf)
            _margins_bind().o_set_margins(self.h, _p(mg, _dp))
        try:
            rc = self.L.o_sample(self.h, ell, M, _p(f, _dp), _p(dd, _dp), _p(w, _dp), _p(st, _u64p),
                                 tr.ctypes.data if tr is not None else None,
                                 ctypes.addressof(ev) if ev is not None else None)
        finally:
            if margins:
                _margins_bind().o_set_margins(self.h, None)
        if rc != 0:
            raise RuntimeError("event buffer too small")
        out = dict(fsums=f, diffsums=dd, work=float(w[0]), stats=st, trace=tr)
        if margins:
            out["margins"] = mg
        if ev is not None:
            n = ev.n
            out["events"] = (bufs[0].raw[:n].decode(), bufs[1][:n].copy(), bufs[2][:n].copy())
        return out

    def full_loss(self, ell: int, first: int, n: int) -> np.ndarray:
        out = np.zeros(n)
        self.L.o_portfolio_full_loss(self.h, ell, first, n, _p(out, _dp))
        return out


# ------------------------------------------------------------------------------------------
# The reference compiled here (oracle/_ref).  Present only where the reference sources were available
# at build time; callers skip when it is absent.
def ref_available(variant: str = "f32") -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libref_{variant}.so"))


class Reference:
    """ctypes view of oracle/ref_harness.cpp built against the reference sources."""

    def __init__(self, variant: str = "f32"):
        path = os.path.join(REF_DIR, f"libref_{variant}.so")
        self.L = ctypes.CDLL(path)
        L = self.L
        L.ref_threefry.argtypes = [_u64p, _u64p, _u64p, ctypes.c_uint64]
        L.ref_stream_draws.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_char_p,
                                       ctypes.c_uint64, _dp, _u64p]
        L.ref_boxmuller.argtypes = [_u64p, _u64p, _dp, _dp, ctypes.c_uint64]
        L.ref_set_threads.argtypes = [ctypes.c_int]
        L.ref_nested_init.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                      ctypes.c_double, ctypes.c_int]
        L.ref_model_init.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_uint64, ctypes.c_int]
        L.ref_model_sample.restype = ctypes.c_int64
        L.ref_model_sample.argtypes = [ctypes.c_uint32, ctypes.c_uint64, _dp, _dp, _dp, _u64p,
                                       ctypes.c_char_p, _dp, _dp, ctypes.c_uint64]
        L.ref_portfolio_init.argtypes = [ctypes.c_uint32, _dp, _dp, _dp, ctypes.c_uint32, _dp,
                                         _dp, _dp, _u32p, _i32p, _dp, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_int, ctypes.c_int, ctypes.c_uint64,
                                         ctypes.c_int, _dp, _dp]
        L.ref_portfolio_sample.restype = ctypes.c_int64
        L.ref_portfolio_sample.argtypes = L.ref_model_sample.argtypes
        L.ref_norm_cdf_inv.restype = ctypes.c_double
        L.ref_norm_cdf_inv.argtypes = [ctypes.c_double]
        L.ref_bs.argtypes = [ctypes.c_int, _dp, _dp, ctypes.c_double, _dp, _dp, _dp, _dp,
                             ctypes.c_uint64]
        L.ref_mlmc_synthetic.restype = ctypes.c_int64
        L.ref_mlmc_synthetic.argtypes = [ctypes.c_double, ctypes.c_uint64, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_uint64,
                                         _u32p, _u64p, ctypes.c_uint64, _dp, ctypes.c_uint32,
                                         _u32p, _dp, ctypes.c_char_p, ctypes.c_uint64]
        L.ref_abi_sizes.argtypes = [_u64p]
        L.ref_simulate_stock_dt.restype = ctypes.c_double
        L.ref_simulate_stock_dt.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64, _dp,
                                            ctypes.c_uint64, ctypes.c_double, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_uint32, ctypes.c_int,
                                            ctypes.c_uint32]
        self.kind = None

    def threefry(self, ctr, key):
        ctr = np.ascontiguousarray(ctr, np.uint64).reshape(-1, 2)
        key = np.ascontiguousarray(key, np.uint64).reshape(-1, 2)
        out = np.zeros_like(ctr)
        self.L.ref_threefry(_p(ctr, _u64p), _p(key, _u64p), _p(out, _u64p), len(ctr))
        return out

    def stream_draws(self, seed, core, ops):
        n = len(ops)
        r = np.zeros(n)
        u = np.zeros(n, np.uint64)
        self.L.ref_stream_draws(seed, core, ops.encode(), n, _p(r, _dp), _p(u, _u64p))
        return r, u

    def boxmuller(self, u0, u1):
        u0 = np.ascontiguousarray(u0, np.uint64)
        u1 = np.ascontiguousarray(u1, np.uint64)
        x = np.zeros(len(u0))
        y = np.zeros(len(u0))
        self.L.ref_boxmuller(_p(u0, _u64p), _p(u1, _u64p), _p(x, _dp), _p(y, _dp), len(u0))
        return x, y

    def abi_sizes(self):
        out = np.zeros(12, np.uint64)
        self.L.ref_abi_sizes(_p(out, _u64p))
        return out

    def mlmc_synthetic(self, targetTOL, M0, a, alpha, v, beta, w, gamma, seed, cap=100000):
        ells = np.zeros(cap, np.uint32)
        Ms = np.zeros(cap, np.uint64)
        lv = np.zeros((64, 10))
        nl = np.zeros(1, np.uint32)
        misc = np.zeros(4)
        buf = ctypes.create_string_buffer(1 << 16)
        n = self.L.ref_mlmc_synthetic(targetTOL, M0, a, alpha, v, beta, w, gamma, seed,
                                      _p(ells, _u32p), _p(Ms, _u64p), cap, _p(lv, _dp), 64,
                                      _p(nl, _u32p), _p(misc, _dp), buf, len(buf))
        return dict(calls_ell=ells[:n].copy(), calls_M=Ms[:n].copy(), levels=lv[:nl[0]].copy(),
                    misc=misc, table=buf.value.decode())

    def init(self, cores, N0, beta, adaptive_r, antithetic=True):
        self.L.ref_set_threads(cores)
        self.L.ref_nested_init(cores, N0, beta, adaptive_r, int(antithetic))

    def model_init(self, kind, tau, max_loss, seed=0, traced=True):
        self.kind = "model"
        self.L.ref_model_init(kind, tau, max_loss, seed, int(traced))

    def portfolio_init(self, pf, r=0.05, rho=0.0, max_loss=0.0, tau=1 / 52,
                       subsample=SUB_UNIFORM, use_delta_cv=False, seed=0, traced=True):
        self.kind = "portfolio"
        Q = len(pf["S0"])
        P = len(pf["strike"])
        self._pf = {k: np.ascontiguousarray(pf[k], np.float64) for k in
                    ("S0", "mu", "sigma", "strike", "maturity", "w", "prob")}
        d = self._pf
        si = np.ascontiguousarray(pf["stock_ind"], np.uint32)
        ty = np.ascontiguousarray(pf["type"], np.int32)
        self._keep = (si, ty)
        start = np.zeros(P)
        delta = np.zeros(P)
        self.L.ref_portfolio_init(Q, _p(d["S0"], _dp), _p(d["mu"], _dp), _p(d["sigma"], _dp), P,
                                  _p(d["strike"], _dp), _p(d["maturity"], _dp), _p(d["w"], _dp),
                                  _p(si, _u32p), _p(ty, _i32p), _p(d["prob"], _dp), r, rho,
                                  max_loss, tau, subsample, int(use_delta_cv), seed, int(traced),
                                  _p(start, _dp), _p(delta, _dp))
        return start, delta

    def portfolio_init_methods(self, pf, method, r=0.05, rho=0.0, max_loss=0.0, tau=1 / 52,
                               subsample=SUB_RANDOM, use_delta_cv=False, use_coarse_delta_cv=False,
                               use_antithetic_risk=True, use_milstein=True, dt_h0inv=8, dt_beta=4,
                               dt_prob_expo=-1.5, seed=0, traced=True):
        self.kind = "portfolio"
        L = self.L
        L.ref_portfolio_init_methods.argtypes = [
            ctypes.c_uint32, _dp, _dp, _dp, ctypes.c_uint32, _dp, _dp, _dp, _u32p, _i32p, _dp,
            _i32p, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint32,
            ctypes.c_uint32, ctypes.c_double, ctypes.c_uint64, ctypes.c_int]
        Q = len(pf["S0"])
        P = len(pf["strike"])
        self._pf = {k: np.ascontiguousarray(pf[k], np.float64) for k in
                    ("S0", "mu", "sigma", "strike", "maturity", "w", "prob")}
        d = self._pf
        si = np.ascontiguousarray(pf["stock_ind"], np.uint32)
        ty = np.ascontiguousarray(pf["type"], np.int32)
        me = np.ascontiguousarray(method, np.int32)
        self._keep = (si, ty, me)
        L.ref_portfolio_init_methods(Q, _p(d["S0"], _dp), _p(d["mu"], _dp), _p(d["sigma"], _dp), P,
                                     _p(d["strike"], _dp), _p(d["maturity"], _dp), _p(d["w"], _dp),
                                     _p(si, _u32p), _p(ty, _i32p), _p(d["prob"], _dp),
                                     _p(me, _i32p), r, rho, max_loss, tau, subsample,
                                     int(use_delta_cv), int(use_coarse_delta_cv),
                                     int(use_antithetic_risk), int(use_milstein), dt_h0inv,
                                     dt_beta, dt_prob_expo, seed, int(traced))

    def sample(self, ell, M, events_cap=0):
        f = np.zeros(4)
        dd = np.zeros(4)
        w = np.zeros(1)
        st = np.zeros(6, np.uint64)
        cap = max(events_cap, 1)
        kinds = ctypes.create_string_buffer(cap)
        vals = np.zeros(cap)
        aux = np.zeros(cap)
        fn = self.L.ref_model_sample if self.kind == "model" else self.L.ref_portfolio_sample
        n = fn(ell, M, _p(f, _dp), _p(dd, _dp), _p(w, _dp), _p(st, _u64p), kinds, _p(vals, _dp),
               _p(aux, _dp), cap)
        if n < 0:
            raise RuntimeError(f"event buffer too small: need {-n}")
        out = dict(fsums=f, diffsums=dd, work=float(w[0]), stats=st)
        if events_cap:
            out["events"] = (kinds.raw[:n].decode(), vals[:n].copy(), aux[:n].copy())
        return out


def synthetic_portfolio(Q: int, P: int, seed: int, prob: str = "uniform", S0=100.0) -> dict:
    """Small seeded BS portfolio for parity tests (numpy PCG64; not a reference generator)."""
    g = np.random.default_rng(seed)
    pf = dict(S0=np.full(Q, S0) * (1 + 0.1 * (g.random(Q) - 0.5)),
              mu=0.05 + 0.1 * g.random(Q),
              sigma=0.1 + 0.3 * g.random(Q),
              stock_ind=g.integers(0, Q, P).astype(np.uint32),
              type=np.where(g.random(P) < 0.5, 1, -1).astype(np.int32),
              maturity=0.25 + 1.75 * g.random(P))
    pf["strike"] = pf["S0"][pf["stock_ind"]] * (0.8 + 0.4 * g.random(P))
    pf["w"] = g.standard_normal(P)
    if prob == "uniform":
        pf["prob"] = np.ones(P)
    else:  # |w|-proportional, sorted non-increasing as portfolio_update_data requires
        order = np.argsort(-np.abs(pf["w"]), kind="stable")
        for k in ("stock_ind", "type", "maturity", "strike", "w"):
            pf[k] = pf[k][order]
        pf["prob"] = np.abs(pf["w"])
    return pf


def _shard_bind():
    L = lib()
    if not getattr(L, "_shard_bound", False):
        L.o_set_shard.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32]
        L._shard_bound = True
    return L


def _margins_bind():
    L = lib()
    if not getattr(L, "_margins_bound", False):
        L.o_set_margins.argtypes = [ctypes.c_void_p, _dp]
        L._margins_bound = True
    return L


def sampler_set_shard(s: "Sampler", rank: int, world: int):
    _shard_bind().o_set_shard(s.h, rank, world)


Sampler.set_shard = sampler_set_shard


def _methods_bind():
    L = lib()
    if not getattr(L, "_methods_bound", False):
        L.o_set_portfolio_methods.restype = ctypes.c_int
        L.o_set_portfolio_methods.argtypes = [
            ctypes.c_void_p, ctypes.c_uint32, _dp, _dp, _dp, ctypes.c_uint32, _dp, _dp, _dp, _u32p,
            _i32p, _dp, _i32p, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint32,
            ctypes.c_uint32, ctypes.c_double]
        L._methods_bound = True
    return L


def adj_loss(batch: dict, ell: int, pairs: int, M: int, seed: int, milstein: bool = True) -> np.ndarray:
    """Path-simulated loss L[p, m] of a portfolio batch (see adjoint_oracle.c)."""
    L = lib()
    if not getattr(L, "_adj_bound", False):
        L.o_adj_loss.argtypes = [ctypes.c_uint32, _u32p, _u32p, _dp, _dp, _dp, _dp, _dp, _dp, _u32p,
                                 _i32p, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64,
                                 ctypes.c_int, _dp]
        L._adj_bound = True
    so = np.ascontiguousarray(batch["stock_off"], np.uint32)
    oo = np.ascontiguousarray(batch["option_off"], np.uint32)
    d = {k: np.ascontiguousarray(batch[k], np.float64) for k in
         ("S0", "mu", "sigma", "strike", "maturity", "w")}
    si = np.ascontiguousarray(batch["stock_ind"], np.uint32)
    ty = np.ascontiguousarray(batch["type"], np.int32)
    n = len(so) - 1
    out = np.zeros(n * M)
    L.o_adj_loss(n, _p(so, _u32p), _p(oo, _u32p), _p(d["S0"], _dp), _p(d["mu"], _dp),
                 _p(d["sigma"], _dp), _p(d["strike"], _dp), _p(d["maturity"], _dp), _p(d["w"], _dp),
                 _p(si, _u32p), _p(ty, _i32p), batch["r"], batch["rho"], batch["tau"], ell, pairs, M,
                 seed, int(milstein), _p(out, _dp))
    return out.reshape(n, M)


def build_alias(p) -> tuple:
    """Alias table (thr, alias, phat) of the OUTER layout's importance sub-sampling."""
    L = lib()
    if not getattr(L, "_alias_bound", False):
        L.o_build_alias.argtypes = [ctypes.c_uint32, _dp, _u32p, _u32p, _dp]
        L._alias_bound = True
    p = np.ascontiguousarray(p, np.float64)
    P = len(p)
    thr = np.zeros(P, np.uint32)
    al = np.zeros(P, np.uint32)
    ph = np.zeros(P)
    L.o_build_alias(P, _p(p, _dp), _p(thr, _u32p), _p(al, _u32p), _p(ph, _dp))
    return thr, al, ph
