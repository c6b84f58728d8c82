"""nmlmc — Python host bindings of the B200 nested-MLMC level sampler (libnmlmc.so).

Mirrors the reference's extern "C" surface (init_nestedmc_sampler, model_init / model_sample,
portfolio_init / portfolio_sample, ...; haji-ali/nested-risk-mlmc, common.hpp:34-36 "meant to be
used in python") and wraps the native context API (`Sampler`) and the host MLMC driver
(`mlmc_run`).  All computation happens in libnmlmc.so on the GPU: there is no CPU fallback, and
importing this module without the built library raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnmlmc.so")
INCLUDE_H = os.path.join(os.path.dirname(os.path.dirname(HERE)), "include", "nmlmc.h")

OK, ERR_ARG, ERR_CUDA, ERR_STATE, ERR_NOMEM, ERR_TIMEOUT, ERR_LIMIT = range(7)
METHOD_BS, METHOD_EXACT, METHOD_UNBIASED = 0, 1, 2
MAX_PATH_STEPS = 1 << 24
PREC_REF32, PREC_FP64, PREC_FP32 = 0, 1, 2
STREAMS_CORE, STREAMS_OUTER = 0, 1
MODEL_REFERENCE, MODEL_SHIFT = 0, 1
SUB_NONE, SUB_RANDOM, SUB_UNIFORM = 0, 1, -1
MAX_LEVELS = 64

_u64p = ctypes.POINTER(ctypes.c_uint64)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_i32p = ctypes.POINTER(ctypes.c_int32)
_dp = ctypes.POINTER(ctypes.c_double)


class NmlmcError(RuntimeError):
    def __init__(self, status: int, what: str):
        super().__init__(f"{what}: {error_string(status)} (status {status})")
        self.status = status


# ---- C structs (include/nmlmc.h) -----------------------------------------------------------
class NestedSamplerParams(ctypes.Structure):
    _fields_ = [("N0", ctypes.c_uint32), ("beta", ctypes.c_uint32), ("antithetic", ctypes.c_bool),
                ("fine_moments", ctypes.c_uint32), ("diff_moments", ctypes.c_uint32),
                ("adaptive_r", ctypes.c_float)]


class SampleOutput(ctypes.Structure):
    _fields_ = [("M", ctypes.c_uint64), ("fsums", _dp), ("diffsums", _dp),
                ("total_work", ctypes.c_double), ("inner_stats", ctypes.c_uint64 * 6)]


class ModelData(ctypes.Structure):
    _fields_ = [("stau", ctypes.c_float), ("s1tau", ctypes.c_float), ("max_loss", ctypes.c_float),
                ("phi_type", ctypes.c_int32)]


class OptionParams(ctypes.Structure):
    _fields_ = [("strike", ctypes.c_float), ("maturity", ctypes.c_float), ("start", ctypes.c_float),
                ("w", ctypes.c_float), ("delta_est", ctypes.c_float), ("stock_ind", ctypes.c_uint32),
                ("type", ctypes.c_int32), ("prob", ctypes.c_float), ("W_est", ctypes.c_float)]


class StockParams(ctypes.Structure):
    _fields_ = [("S0", ctypes.c_float), ("mu", ctypes.c_float), ("sigma", ctypes.c_float)]


class OptionsSpan(ctypes.Structure):
    _fields_ = [("data", ctypes.POINTER(OptionParams)), ("size", ctypes.c_size_t)]


class StocksSpan(ctypes.Structure):
    _fields_ = [("data", ctypes.POINTER(StockParams)), ("size", ctypes.c_size_t)]


class PortfolioData(ctypes.Structure):
    _fields_ = [("options", OptionsSpan * 3), ("stocks", StocksSpan),
                ("r", ctypes.c_float), ("rho", ctypes.c_float), ("s1_rho2", ctypes.c_float),
                ("max_loss", ctypes.c_float), ("tau", ctypes.c_float),
                ("dt_h0inv", ctypes.c_uint32), ("dt_beta", ctypes.c_uint32),
                ("dt_prob_expo", ctypes.c_float), ("phi_type", ctypes.c_int32),
                ("_phi_size", ctypes.c_uint32), ("subsample", ctypes.c_int32),
                ("use_delta_cv", ctypes.c_bool), ("use_coarse_delta_cv", ctypes.c_bool),
                ("use_antithetic_risk", ctypes.c_bool), ("use_milstein", ctypes.c_bool)]


class Config(ctypes.Structure):
    _fields_ = [("cores", ctypes.c_uint32), ("N0", ctypes.c_uint32), ("beta", ctypes.c_uint32),
                ("adaptive_r", ctypes.c_double), ("antithetic", ctypes.c_int32),
                ("adaptive_incl_r2", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("streams", ctypes.c_int32), ("seed", ctypes.c_uint64), ("batch", ctypes.c_uint64)]


class LevelResult(ctypes.Structure):
    _fields_ = [("fsums", ctypes.c_double * 4), ("diffsums", ctypes.c_double * 4),
                ("total_work", ctypes.c_double), ("M", ctypes.c_uint64),
                ("inner_stats", ctypes.c_uint64 * 6), ("seconds", ctypes.c_double)]

    def as_dict(self) -> dict:
        return dict(fsums=np.array(self.fsums[:]), diffsums=np.array(self.diffsums[:]),
                    work=float(self.total_work), M=int(self.M),
                    stats=np.array(self.inner_stats[:], dtype=np.uint64), seconds=float(self.seconds))


class Portfolio(ctypes.Structure):
    _fields_ = [("Q", ctypes.c_uint32), ("P", ctypes.c_uint32),
                ("S0", _dp), ("mu", _dp), ("sigma", _dp),
                ("strike", _dp), ("maturity", _dp), ("w", _dp), ("prob", _dp),
                ("stock_ind", _u32p), ("type", _i32p),
                ("r", ctypes.c_double), ("rho", ctypes.c_double), ("max_loss", ctypes.c_double),
                ("tau", ctypes.c_double), ("subsample", ctypes.c_int32),
                ("use_delta_cv", ctypes.c_int32), ("discount", ctypes.c_int32)]


class PathMethods(ctypes.Structure):
    _fields_ = [("method", _i32p), ("dt_h0inv", ctypes.c_uint32), ("dt_beta", ctypes.c_uint32),
                ("dt_prob_expo", ctypes.c_double), ("use_coarse_delta_cv", ctypes.c_int32),
                ("use_antithetic_risk", ctypes.c_int32), ("use_milstein", ctypes.c_int32)]


class PortfolioBatch(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint32), ("stock_off", _u32p), ("option_off", _u32p),
                ("S0", _dp), ("mu", _dp), ("sigma", _dp), ("strike", _dp), ("maturity", _dp),
                ("w", _dp), ("stock_ind", _u32p), ("type", _i32p), ("K", _dp),
                ("r", ctypes.c_double), ("rho", ctypes.c_double), ("tau", ctypes.c_double)]


class AdjointConfig(ctypes.Structure):
    _fields_ = [("ell", ctypes.c_uint32), ("inner_pairs", ctypes.c_uint32), ("M", ctypes.c_uint64),
                ("delta_rel", ctypes.c_double), ("precision", ctypes.c_int32),
                ("milstein", ctypes.c_int32), ("seed", ctypes.c_uint64)]


class AdjointResult(ctypes.Structure):
    _fields_ = [("EL", ctypes.c_double), ("P_smooth", ctypes.c_double), ("P_hard", ctypes.c_double)]


class TraceRec(ctypes.Structure):
    _fields_ = [("count_f", ctypes.c_uint64), ("count_c", ctypes.c_uint64),
                ("phi_f", ctypes.c_double), ("phi_c", ctypes.c_double),
                ("mean_big", ctypes.c_double), ("min_abs_small", ctypes.c_double),
                ("core", ctypes.c_uint32), ("pilots", ctypes.c_uint32)]


TRACE_DTYPE = np.dtype([("count_f", np.uint64), ("count_c", np.uint64), ("phi_f", np.float64),
                        ("phi_c", np.float64), ("mean_big", np.float64),
                        ("min_abs_small", np.float64), ("core", np.uint32), ("pilots", np.uint32)])


class MlmcInput(ctypes.Structure):
    _fields_ = [("targetTOL", ctypes.c_double), ("startTOL", ctypes.c_double),
                ("theta", ctypes.c_double), ("starting_level_coeff", ctypes.c_double),
                ("Ca", ctypes.c_double), ("M0", ctypes.c_uint64), ("verbose", ctypes.c_int32),
                ("max_levels", ctypes.c_uint32), ("batched", ctypes.c_int32),
                ("max_iterations", ctypes.c_uint32)]


class MlmcOutput(ctypes.Structure):
    _fields_ = [("nlevels", ctypes.c_uint32), ("starting_level", ctypes.c_uint32),
                ("bias_est", ctypes.c_double), ("stat_error", ctypes.c_double),
                ("TOL", ctypes.c_double), ("Eg", ctypes.c_double),
                ("total_work", ctypes.c_double), ("total_time", ctypes.c_double),
                ("calls", ctypes.c_uint64),
                ("level_M", ctypes.c_uint64 * MAX_LEVELS),
                ("level_fsums", (ctypes.c_double * 4) * MAX_LEVELS),
                ("level_diffsums", (ctypes.c_double * 4) * MAX_LEVELS),
                ("level_work", ctypes.c_double * MAX_LEVELS),
                ("level_time", ctypes.c_double * MAX_LEVELS),
                ("iterations_done", ctypes.c_uint32), ("complete", ctypes.c_uint32)]


class PortfolioSpec(ctypes.Structure):
    _fields_ = [("Q", ctypes.c_uint32), ("P", ctypes.c_uint32), ("S0", ctypes.c_double),
                ("r", ctypes.c_double), ("mu", ctypes.c_double), ("sigma_lo", ctypes.c_double),
                ("sigma_hi", ctypes.c_double), ("strike_lo", ctypes.c_double),
                ("strike_hi", ctypes.c_double), ("maturity_lo", ctypes.c_double),
                ("maturity_hi", ctypes.c_double), ("call_fraction", ctypes.c_double)]


# The benchmark portfolio configurations: d GBM stocks (S0 = 100, r = mu = 0.05,
# sigma ~ U[0.1, 0.4], horizon tau = 1/52), P European options on uniformly chosen stocks,
# 50/50 call/put, strike ~ U[0.8, 1.2] S0, maturity ~ U[0.25, 2], position ~ N(0, 1).
PORTFOLIO_C2 = dict(Q=20, P=10_000, S0=100.0, r=0.05, mu=0.05, sigma_lo=0.1, sigma_hi=0.4,
                    strike_lo=0.8, strike_hi=1.2, maturity_lo=0.25, maturity_hi=2.0, call_fraction=0.5)
PORTFOLIO_C3 = dict(PORTFOLIO_C2, Q=200, P=1_000_000)
TAU_WEEK = 1 / 52

class PhaseConfig(ctypes.Structure):
    """nmlmc_phase_config: phase-kernel variant and chunk length of one level."""
    _fields_ = [("variant", ctypes.c_uint32), ("chunk", ctypes.c_uint32), ("state", ctypes.c_int32),
                ("probe_ms", ctypes.c_double)]


PHASE_DEFAULT, PHASE_TUNED, PHASE_PINNED = 0, 1, 2

SAMPLE_LEVEL_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64,
                                   ctypes.POINTER(LevelResult))
STATE_SAVE_FN = ctypes.CFUNCTYPE(ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t)
STATE_LOAD_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t)


class CheckpointIO(ctypes.Structure):
    """nmlmc_checkpoint_io: checkpoint file of the MLMC driver and the sampler-state hooks."""
    _fields_ = [("path", ctypes.c_char_p), ("resume", ctypes.c_int32), ("save", STATE_SAVE_FN),
                ("load", STATE_LOAD_FN)]
SAMPLE_LEVELS_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_uint32, _u32p, _u64p,
                                    ctypes.POINTER(LevelResult))

# ---- library ---------------------------------------------------------------------------------
_lib = None

# Every symbol include/nmlmc.h declares (checked by the tests against the header and the .so).
EXPORTS = [
    "init_nestedmc_sampler", "cleanup_nestedmc_sampler", "model_update_data", "model_init",
    "model_sample", "portfolio_update_data", "portfolio_init", "portfolio_sample",
    "portfolio_cleanup", "portfolio_comp_params", "portfolio_gen_data", "portfolio_free_data",
    "norm_cdf_inv", "nmlmc_last_error",
    "nmlmc_default_set_precision", "nmlmc_error_string", "nmlmc_version", "nmlmc_create",
    "nmlmc_destroy", "nmlmc_configure", "nmlmc_set_model", "nmlmc_set_portfolio",
    "nmlmc_reset_streams", "nmlmc_sample", "nmlmc_sample_levels", "nmlmc_set_trace",
    "nmlmc_portfolio_full_loss", "nmlmc_mlmc_default_input", "nmlmc_mlmc_run",
    "nmlmc_mlmc_run_cb", "nmlmc_threefry_blocks", "nmlmc_outer_normals", "nmlmc_set_shard",
    "nmlmc_set_profiling", "nmlmc_phase_kernel_time", "nmlmc_kernel_launches",
    "nmlmc_sample_level_noalloc", "nmlmc_portfolio_generate", "nmlmc_set_portfolio_methods",
    "nmlmc_path_adjoint", "nmlmc_graph_stats", "nmlmc_set_autotune", "nmlmc_get_phase_config",
    "nmlmc_set_phase_config", "nmlmc_autotune_level", "nmlmc_mlmc_run_cb_ckpt", "nmlmc_mlmc_run_ckpt",
    "nmlmc_get_sampler_state", "nmlmc_set_sampler_state", "nmlmc_norm_cdf_fast",
    "nmlmc_inject_alloc_failure",
]


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libnmlmc.so is not built ({LIB_PATH}); run "
                          "`make -C nested-risk-mlmc_b200` or __graft_entry__.build()")
    L = ctypes.CDLL(LIB_PATH)
    L.nmlmc_error_string.restype = ctypes.c_char_p
    L.nmlmc_error_string.argtypes = [ctypes.c_int]
    L.nmlmc_create.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int]
    L.nmlmc_destroy.argtypes = [ctypes.c_void_p]
    L.nmlmc_configure.argtypes = [ctypes.c_void_p, ctypes.POINTER(Config)]
    L.nmlmc_set_model.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_double, ctypes.c_double]
    L.nmlmc_set_portfolio.argtypes = [ctypes.c_void_p, ctypes.POINTER(Portfolio), _dp, _dp]
    L.nmlmc_path_adjoint.argtypes = [ctypes.c_void_p, ctypes.POINTER(PortfolioBatch),
                                     ctypes.POINTER(AdjointConfig), ctypes.POINTER(AdjointResult),
                                     _dp, _dp, _dp, _dp, _dp, _dp]
    L.nmlmc_set_portfolio_methods.argtypes = [ctypes.c_void_p, ctypes.POINTER(Portfolio),
                                              ctypes.POINTER(PathMethods), _dp, _dp]
    L.nmlmc_reset_streams.argtypes = [ctypes.c_void_p]
    L.nmlmc_sample.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.POINTER(LevelResult)]
    L.nmlmc_sample_levels.argtypes = [ctypes.c_void_p, ctypes.c_uint32, _u32p, _u64p, ctypes.POINTER(LevelResult)]
    L.nmlmc_set_trace.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64]
    L.nmlmc_portfolio_full_loss.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64,
                                            ctypes.c_uint64, _dp]
    L.nmlmc_mlmc_default_input.restype = MlmcInput
    L.nmlmc_mlmc_run.argtypes = [ctypes.c_void_p, ctypes.POINTER(MlmcInput), ctypes.POINTER(MlmcOutput),
                                 ctypes.c_char_p, ctypes.c_size_t]
    L.nmlmc_mlmc_run_cb.argtypes = [ctypes.POINTER(MlmcInput), SAMPLE_LEVEL_FN, SAMPLE_LEVELS_FN,
                                    ctypes.c_void_p, ctypes.POINTER(MlmcOutput), ctypes.c_char_p,
                                    ctypes.c_size_t]
    L.nmlmc_mlmc_run_cb_ckpt.argtypes = [ctypes.POINTER(MlmcInput), SAMPLE_LEVEL_FN, SAMPLE_LEVELS_FN,
                                         ctypes.c_void_p, ctypes.POINTER(CheckpointIO),
                                         ctypes.POINTER(MlmcOutput), ctypes.c_char_p, ctypes.c_size_t]
    L.nmlmc_mlmc_run_ckpt.argtypes = [ctypes.c_void_p, ctypes.POINTER(MlmcInput), ctypes.c_char_p,
                                      ctypes.c_int32, ctypes.POINTER(MlmcOutput), ctypes.c_char_p,
                                      ctypes.c_size_t]
    L.nmlmc_get_sampler_state.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                          ctypes.POINTER(ctypes.c_size_t)]
    L.nmlmc_set_sampler_state.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]
    L.nmlmc_portfolio_generate.argtypes = [ctypes.POINTER(PortfolioSpec), ctypes.c_uint64, _dp, _dp, _dp,
                                           _dp, _dp, _dp, _u32p, _i32p]
    L.nmlmc_set_shard.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32]
    L.nmlmc_set_profiling.argtypes = [ctypes.c_void_p, ctypes.c_int32]
    L.nmlmc_set_autotune.argtypes = [ctypes.c_void_p, ctypes.c_int32]
    L.nmlmc_inject_alloc_failure.argtypes = [ctypes.c_int32]
    L.nmlmc_get_phase_config.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(PhaseConfig)]
    L.nmlmc_set_phase_config.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(PhaseConfig)]
    L.nmlmc_autotune_level.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64]
    L.nmlmc_phase_kernel_time.argtypes = [ctypes.c_void_p, _u64p, _dp]
    L.nmlmc_kernel_launches.restype = ctypes.c_uint64
    L.nmlmc_sample_level_noalloc.argtypes = [ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                             ctypes.c_uint32, ctypes.c_uint32, ctypes.c_double,
                                             ctypes.c_int32, ctypes.c_int32, ctypes.c_uint64,
                                             ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64,
                                             ctypes.c_void_p, ctypes.c_void_p]
    L.nmlmc_threefry_blocks.argtypes = [_u64p, _u64p, _u64p, ctypes.c_uint64]
    L.nmlmc_norm_cdf_fast.argtypes = [ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
                                      ctypes.c_uint64]
    L.nmlmc_outer_normals.argtypes = [ctypes.c_int32, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32,
                                      ctypes.c_uint64, _dp]
    # reference surface
    L.init_nestedmc_sampler.argtypes = [ctypes.c_uint32, ctypes.POINTER(NestedSamplerParams)]
    L.model_update_data.argtypes = [ctypes.POINTER(ModelData)]
    L.model_init.argtypes = [ctypes.POINTER(ModelData), ctypes.c_uint64]
    L.model_sample.argtypes = [ctypes.c_uint32, ctypes.c_uint64, ctypes.POINTER(SampleOutput)]
    L.portfolio_update_data.argtypes = [ctypes.POINTER(PortfolioData)]
    L.portfolio_init.argtypes = [ctypes.POINTER(PortfolioData), ctypes.c_uint64]
    L.portfolio_sample.argtypes = [ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64, ctypes.POINTER(SampleOutput)]
    L.portfolio_comp_params.argtypes = [ctypes.POINTER(PortfolioData)]
    L.portfolio_gen_data.restype = PortfolioData
    L.portfolio_gen_data.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64,
                                     ctypes.POINTER(ctypes.c_double), ctypes.c_bool, ctypes.c_bool]
    L.portfolio_free_data.restype = None
    L.portfolio_free_data.argtypes = [ctypes.POINTER(PortfolioData)]
    L.norm_cdf_inv.restype = ctypes.c_float
    L.norm_cdf_inv.argtypes = [ctypes.c_float]
    L.nmlmc_default_set_precision.argtypes = [ctypes.c_int32, ctypes.c_int32]
    _lib = L
    return L


def error_string(status: int) -> str:
    try:
        return lib().nmlmc_error_string(status).decode()
    except ImportError:
        return str(status)


def _check(rc: int, what: str):
    if rc != OK:
        raise NmlmcError(rc, what)


def _p(a, t):
    return a.ctypes.data_as(t)


# ---- native context --------------------------------------------------------------------------
class Sampler:
    """One GPU level sampler (nmlmc_ctx): configuration, model or portfolio, streams."""

    def __init__(self, device: int = 0, *, cores=2048, N0=32, beta=2, adaptive_r=0.0,
                 antithetic=True, adaptive_incl_r2=False, precision=PREC_FP32,
                 streams=STREAMS_OUTER, seed=0, batch=0):
        L = lib()
        h = ctypes.c_void_p()
        _check(L.nmlmc_create(ctypes.byref(h), device), "nmlmc_create")
        self.h = h
        self.L = L
        self.cfg = Config(cores, N0, beta, adaptive_r, int(antithetic), int(adaptive_incl_r2),
                          precision, streams, seed, batch)
        _check(L.nmlmc_configure(self.h, ctypes.byref(self.cfg)), "nmlmc_configure")
        self._keep = None

    def close(self):
        if getattr(self, "h", None):
            self.L.nmlmc_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def configure(self, **kw):
        for k, v in kw.items():
            setattr(self.cfg, k, int(v) if isinstance(v, bool) else v)
        _check(self.L.nmlmc_configure(self.h, ctypes.byref(self.cfg)), "nmlmc_configure")

    def set_model(self, kind: int, tau: float = 0.0, max_loss: float = 1.0):
        _check(self.L.nmlmc_set_model(self.h, kind, tau, max_loss), "nmlmc_set_model")

    def set_portfolio(self, pf: dict, r=0.05, rho=0.0, max_loss=0.0, tau=1 / 52,
                      subsample=SUB_UNIFORM, use_delta_cv=False, discount=True, methods=None):
        """Portfolio of European options.  `methods` (optional): dict with `method` ([P] of
        METHOD_BS / METHOD_EXACT / METHOD_UNBIASED) and the path-simulation parameters
        dt_h0inv, dt_beta, dt_prob_expo, use_coarse_delta_cv, use_antithetic_risk,
        use_milstein (defaults 8, 4, -1.5, False, True, True)."""
        d = {k: np.ascontiguousarray(pf[k], np.float64) for k in
             ("S0", "mu", "sigma", "strike", "maturity", "w", "prob")}
        si = np.ascontiguousarray(pf["stock_ind"], np.uint32)
        ty = np.ascontiguousarray(pf["type"], np.int32)
        P, Q = len(d["strike"]), len(d["S0"])
        st = Portfolio(Q, P, _p(d["S0"], _dp), _p(d["mu"], _dp), _p(d["sigma"], _dp),
                       _p(d["strike"], _dp), _p(d["maturity"], _dp), _p(d["w"], _dp),
                       _p(d["prob"], _dp), _p(si, _u32p), _p(ty, _i32p), r, rho, max_loss, tau,
                       subsample, int(use_delta_cv), int(discount))
        start = np.zeros(P)
        delta = np.zeros(P)
        if methods is None:
            _check(self.L.nmlmc_set_portfolio(self.h, ctypes.byref(st), _p(start, _dp), _p(delta, _dp)),
                   "nmlmc_set_portfolio")
            return start, delta
        me = np.ascontiguousarray(methods["method"], np.int32)
        pm = PathMethods(_p(me, _i32p), int(methods.get("dt_h0inv", 8)), int(methods.get("dt_beta", 4)),
                         float(methods.get("dt_prob_expo", -1.5)),
                         int(bool(methods.get("use_coarse_delta_cv", False))),
                         int(bool(methods.get("use_antithetic_risk", True))),
                         int(bool(methods.get("use_milstein", True))))
        _check(self.L.nmlmc_set_portfolio_methods(self.h, ctypes.byref(st), ctypes.byref(pm),
                                                  _p(start, _dp), _p(delta, _dp)),
               "nmlmc_set_portfolio_methods")
        return start, delta

    def path_adjoint(self, batch: dict, ell: int, pairs: int, M: int, delta_rel: float = 0.01,
                     precision: int | None = None, seed: int = 0, milstein: bool = True,
                     grads: bool = True, loss: bool = False) -> dict:
        """Path-simulated loss of a portfolio batch (make_batch) with the adjoint gradients of
        E[L] and of the sigmoid-smoothed P(L > K); see nmlmc_path_adjoint.  precision: the
        sampler's own unless given (PREC_REF32 runs the FP32 paths)."""
        if precision is None:
            precision = PREC_FP64 if self.cfg.precision == PREC_FP64 else PREC_FP32
        so = np.ascontiguousarray(batch["stock_off"], np.uint32)
        oo = np.ascontiguousarray(batch["option_off"], np.uint32)
        d = {k: np.ascontiguousarray(batch[k], np.float64) for k in
             ("S0", "mu", "sigma", "strike", "maturity", "w", "K")}
        si = np.ascontiguousarray(batch["stock_ind"], np.uint32)
        ty = np.ascontiguousarray(batch["type"], np.int32)
        n, NS, NO = len(so) - 1, int(so[-1]), int(oo[-1])
        b = PortfolioBatch(n, _p(so, _u32p), _p(oo, _u32p), _p(d["S0"], _dp), _p(d["mu"], _dp),
                           _p(d["sigma"], _dp), _p(d["strike"], _dp), _p(d["maturity"], _dp),
                           _p(d["w"], _dp), _p(si, _u32p), _p(ty, _i32p), _p(d["K"], _dp),
                           batch["r"], batch["rho"], batch["tau"])
        cfg = AdjointConfig(ell, pairs, M, delta_rel, precision, int(milstein), seed)
        res = (AdjointResult * n)()
        out = {}
        g = [np.zeros(NO), np.zeros(NO), np.zeros(NS), np.zeros(NS)] if grads else [None] * 4
        lo = np.zeros(n * M) if loss else None
        sec = ctypes.c_double(0)
        _check(self.L.nmlmc_path_adjoint(self.h, ctypes.byref(b), ctypes.byref(cfg), res,
                                         *[_p(x, _dp) if x is not None else None for x in g],
                                         _p(lo, _dp) if lo is not None else None, ctypes.byref(sec)),
               "nmlmc_path_adjoint")
        out["EL"] = np.array([r.EL for r in res])
        out["P_smooth"] = np.array([r.P_smooth for r in res])
        out["P_hard"] = np.array([r.P_hard for r in res])
        out["seconds"] = sec.value
        if grads:
            out["grad_w_EL"], out["grad_w_P"], out["grad_sigma_EL"], out["grad_sigma_P"] = g
        if loss:
            out["loss"] = lo.reshape(n, M)
        return out

    def graph_stats(self) -> dict:
        a, b, c = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        _check(self.L.nmlmc_graph_stats(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)),
               "nmlmc_graph_stats")
        return dict(instantiations=a.value, updates=b.value, launches=c.value)

    # ---- phase-kernel autotuner (batched FP32 path) ----
    def set_autotune(self, mode: int):
        """0 off, 1 register/occupancy variant per level (default), 2 variant and chunk length."""
        _check(self.L.nmlmc_set_autotune(self.h, int(mode)), "nmlmc_set_autotune")

    def phase_config(self, ell: int) -> dict:
        """Level ell's phase-kernel configuration: variant, chunk, state (PHASE_*), probe_ms."""
        p = PhaseConfig()
        _check(self.L.nmlmc_get_phase_config(self.h, ell, ctypes.byref(p)), "nmlmc_get_phase_config")
        return dict(variant=p.variant, chunk=p.chunk, state=p.state, probe_ms=p.probe_ms)

    def set_phase_config(self, ell: int, variant=None, chunk=None):
        """Pins level ell's configuration; with no arguments, unpins it."""
        if variant is None and chunk is None:
            _check(self.L.nmlmc_set_phase_config(self.h, ell, None), "nmlmc_set_phase_config")
            return
        cur = self.phase_config(ell)
        p = PhaseConfig(cur["variant"] if variant is None else variant,
                        cur["chunk"] if chunk is None else chunk, 0, 0.0)
        _check(self.L.nmlmc_set_phase_config(self.h, ell, ctypes.byref(p)), "nmlmc_set_phase_config")

    def autotune_level(self, ell: int, M: int) -> dict:
        _check(self.L.nmlmc_autotune_level(self.h, ell, M), "nmlmc_autotune_level")
        return self.phase_config(ell)

    def reset_streams(self):
        _check(self.L.nmlmc_reset_streams(self.h), "nmlmc_reset_streams")

    def sample(self, ell: int, M: int, trace: bool = False) -> dict:
        r = LevelResult()
        tr = None
        if trace:
            tr = np.zeros(M, TRACE_DTYPE)
            _check(self.L.nmlmc_set_trace(self.h, tr.ctypes.data, M), "nmlmc_set_trace")
        _check(self.L.nmlmc_sample(self.h, ell, M, ctypes.byref(r)), "nmlmc_sample")
        out = r.as_dict()
        out["trace"] = tr
        return out

    def sample_levels(self, ells, Ms) -> list:
        ells = np.ascontiguousarray(ells, np.uint32)
        Ms = np.ascontiguousarray(Ms, np.uint64)
        res = (LevelResult * len(ells))()
        _check(self.L.nmlmc_sample_levels(self.h, len(ells), _p(ells, _u32p), _p(Ms, _u64p), res),
               "nmlmc_sample_levels")
        return [r.as_dict() for r in res]

    def set_shard(self, rank: int, world: int):
        _check(self.L.nmlmc_set_shard(self.h, rank, world), "nmlmc_set_shard")

    def set_profiling(self, on: bool):
        _check(self.L.nmlmc_set_profiling(self.h, int(on)), "nmlmc_set_profiling")

    def phase_kernel_time(self):
        n = ctypes.c_uint64(0)
        s = ctypes.c_double(0)
        _check(self.L.nmlmc_phase_kernel_time(self.h, ctypes.byref(n), ctypes.byref(s)), "phase_kernel_time")
        return int(n.value), float(s.value)

    def full_loss(self, ell: int, first: int, n: int) -> np.ndarray:
        out = np.zeros(n)
        _check(self.L.nmlmc_portfolio_full_loss(self.h, ell, first, n, _p(out, _dp)), "full_loss")
        return out

    def mlmc_run(self, targetTOL=1e-3, M0=100, verbose=False, batched=False, max_levels=0,
                 checkpoint=None, resume=False, **kw) -> dict:
        """Continuation MLMC to targetTOL.  With `checkpoint` (a path) the driver writes its state
        after every TOL iteration; `resume` continues from that file (max_iterations=k in kw
        stops after k iterations)."""
        inp = self.L.nmlmc_mlmc_default_input()
        inp.targetTOL, inp.M0, inp.verbose = targetTOL, M0, int(verbose)
        inp.batched, inp.max_levels = int(batched), max_levels
        for k, v in kw.items():
            setattr(inp, k, v)
        out = MlmcOutput()
        buf = ctypes.create_string_buffer(1 << 16)
        if checkpoint is None:
            _check(self.L.nmlmc_mlmc_run(self.h, ctypes.byref(inp), ctypes.byref(out), buf, len(buf)),
                   "nmlmc_mlmc_run")
        else:
            _check(self.L.nmlmc_mlmc_run_ckpt(self.h, ctypes.byref(inp), os.fsencode(checkpoint), int(resume),
                                              ctypes.byref(out), buf, len(buf)), "nmlmc_mlmc_run_ckpt")
        return mlmc_output_dict(out, buf.value.decode())

    def sampler_state(self) -> bytes:
        """The context's stream state (nmlmc_get_sampler_state)."""
        n = ctypes.c_size_t()
        _check(self.L.nmlmc_get_sampler_state(self.h, None, 0, ctypes.byref(n)), "nmlmc_get_sampler_state")
        b = ctypes.create_string_buffer(n.value)
        _check(self.L.nmlmc_get_sampler_state(self.h, b, n.value, ctypes.byref(n)), "nmlmc_get_sampler_state")
        return b.raw[:n.value]

    def set_sampler_state(self, state: bytes):
        _check(self.L.nmlmc_set_sampler_state(self.h, state, len(state)), "nmlmc_set_sampler_state")


def mlmc_output_dict(out: MlmcOutput, table: str) -> dict:
    n = out.nlevels
    return dict(nlevels=n, starting_level=out.starting_level, bias_est=out.bias_est,
                stat_error=out.stat_error, TOL=out.TOL, Eg=out.Eg, total_work=out.total_work,
                total_time=out.total_time, calls=out.calls,
                level_M=np.array(out.level_M[:n], dtype=np.uint64),
                level_fsums=np.array([out.level_fsums[i][:] for i in range(n)]),
                level_diffsums=np.array([out.level_diffsums[i][:] for i in range(n)]),
                level_work=np.array(out.level_work[:n]), level_time=np.array(out.level_time[:n]),
                iterations_done=out.iterations_done, complete=bool(out.complete), table=table)


def mlmc_run_cb(sample_level, sample_levels=None, *, targetTOL=1e-3, M0=100, verbose=False,
                batched=False, checkpoint=None, resume=False, state=None, **kw) -> dict:
    """The host MLMC driver over a Python level sampler: sample_level(ell, M) -> dict with
    fsums, diffsums, work (and optionally seconds); with `batched`, sample_levels(ells, Ms) (if
    given) takes all levels of a round at once.  A sampler that fails leaves the result's M
    at 0 and the driver stops with an error.  With `checkpoint` (a path) the driver writes its
    state after every TOL iteration, `resume` continues from it, and `state` = (save, load)
    stores the sampler's own state in the file: save() -> bytes, load(bytes).  An exception
    raised by a callback stops the run; it is re-raised as NmlmcError (status of the driver) with
    the callback's exception as its cause."""
    L = lib()
    failures = []              # exceptions raised inside the ctypes callbacks, first one first

    def finish(rc, what):
        if failures:
            e = failures[0]
            if rc == OK:
                raise e
            raise NmlmcError(rc, f"{what}: a callback raised {type(e).__name__}: {e}") from e
        _check(rc, what)

    def fill(res, d, M):
        for j in range(4):
            res.fsums[j] = float(d["fsums"][j])
            res.diffsums[j] = float(d["diffsums"][j])
        res.total_work = float(d["work"])
        res.M = M
        res.seconds = float(d.get("seconds", 0.0))

    def _one(user, ell, M, out):
        try:
            fill(out.contents, sample_level(int(ell), int(M)), int(M))
        except Exception as e:     # a failed sampler: M stays 0 and the driver stops
            failures.append(e)
            out.contents.M = 0

    def _many(user, n, ells, Ms, outs):
        try:
            el = [int(ells[i]) for i in range(n)]
            ms = [int(Ms[i]) for i in range(n)]
            rs = sample_levels(el, ms) if sample_levels else [sample_level(e, m) for e, m in zip(el, ms)]
            for i in range(n):
                fill(outs[i], rs[i], ms[i])
        except Exception as e:
            failures.append(e)
            for i in range(n):
                outs[i].M = 0

    f1 = SAMPLE_LEVEL_FN(_one)
    f2 = SAMPLE_LEVELS_FN(_many)
    inp = L.nmlmc_mlmc_default_input()
    inp.targetTOL, inp.M0, inp.verbose, inp.batched = targetTOL, M0, int(verbose), int(batched)
    for k, v in kw.items():
        setattr(inp, k, v)
    out = MlmcOutput()
    buf = ctypes.create_string_buffer(1 << 16)
    if checkpoint is None:
        finish(L.nmlmc_mlmc_run_cb(ctypes.byref(inp), f1, f2, None, ctypes.byref(out), buf, len(buf)),
               "nmlmc_mlmc_run_cb")
        return mlmc_output_dict(out, buf.value.decode())

    def _save(user, p, cap):
        try:
            b = state[0]()
            if p:
                if cap < len(b):
                    return ctypes.c_size_t(-1).value
                ctypes.memmove(p, b, len(b))
            return len(b)
        except Exception as e:     # the run stops with NMLMC_ERR_STATE
            failures.append(e)
            return ctypes.c_size_t(-1).value

    def _load(user, p, n):
        try:
            state[1](ctypes.string_at(p, n))
            return OK
        except Exception as e:
            failures.append(e)
            return ERR_STATE

    fs = STATE_SAVE_FN(_save) if state else STATE_SAVE_FN()
    fl = STATE_LOAD_FN(_load) if state else STATE_LOAD_FN()
    io = CheckpointIO(os.fsencode(checkpoint), int(resume), fs, fl)
    finish(L.nmlmc_mlmc_run_cb_ckpt(ctypes.byref(inp), f1, f2, None, ctypes.byref(io), ctypes.byref(out),
                                    buf, len(buf)), "nmlmc_mlmc_run_cb_ckpt")
    return mlmc_output_dict(out, buf.value.decode())


def norm_cdf_fast(x) -> np.ndarray:
    """Phi(x) as the FP32 Black-Scholes path computes it on the GPU (float32 in and out)."""
    x = np.ascontiguousarray(x, np.float32)
    out = np.empty_like(x)
    fp = ctypes.POINTER(ctypes.c_float)
    _check(lib().nmlmc_norm_cdf_fast(x.ctypes.data_as(fp), out.ctypes.data_as(fp), x.size), "nmlmc_norm_cdf_fast")
    return out


def generate_portfolio(spec: dict, seed: int) -> dict:
    """Seeded synthetic portfolio (nmlmc_portfolio_generate): arrays for Sampler.set_portfolio."""
    sp = PortfolioSpec(**{k: spec[k] for k, _ in PortfolioSpec._fields_})
    Q, P = sp.Q, sp.P
    out = dict(S0=np.zeros(Q), mu=np.zeros(Q), sigma=np.zeros(Q), strike=np.zeros(P),
               maturity=np.zeros(P), w=np.zeros(P), stock_ind=np.zeros(P, np.uint32),
               type=np.zeros(P, np.int32))
    _check(lib().nmlmc_portfolio_generate(ctypes.byref(sp), seed, _p(out["S0"], _dp), _p(out["mu"], _dp),
                                          _p(out["sigma"], _dp), _p(out["strike"], _dp),
                                          _p(out["maturity"], _dp), _p(out["w"], _dp),
                                          _p(out["stock_ind"], _u32p), _p(out["type"], _i32p)),
           "nmlmc_portfolio_generate")
    out["prob"] = np.ones(P)
    return out


def loss_quantile(sampler: "Sampler", q: float, n: int, level: int = 63) -> float:
    """q-quantile of the full portfolio loss L(Y) over n outer samples of the sampler's seed
    (stream level `level`, kept apart from the MLMC levels)."""
    L = sampler.full_loss(level, 0, n)
    return float(np.quantile(L, q, method="inverted_cdf"))


def kernel_launches() -> int:
    """Kernels launched by libnmlmc.so since it was loaded."""
    return int(lib().nmlmc_kernel_launches())


def threefry_blocks(ctr, key) -> np.ndarray:
    """Threefry2x64-20 blocks computed on the GPU."""
    ctr = np.ascontiguousarray(ctr, np.uint64).reshape(-1, 2)
    key = np.ascontiguousarray(key, np.uint64).reshape(-1, 2)
    out = np.zeros_like(ctr)
    _check(lib().nmlmc_threefry_blocks(_p(ctr, _u64p), _p(key, _u64p), _p(out, _u64p), len(ctr)),
           "nmlmc_threefry_blocks")
    return out


def outer_normals(precision: int, seed: int, stream: int, tag: int, n: int) -> np.ndarray:
    out = np.zeros(n)
    _check(lib().nmlmc_outer_normals(precision, seed, stream, tag, n, _p(out, _dp)), "nmlmc_outer_normals")
    return out


# ---- the reference-named surface ---------------------------------------------------------------
def init_nestedmc_sampler(cores: int, params: NestedSamplerParams):
    lib().init_nestedmc_sampler(cores, ctypes.byref(params))
    _check(lib().nmlmc_last_error(), "init_nestedmc_sampler")


def cleanup_nestedmc_sampler():
    lib().cleanup_nestedmc_sampler()


def model_update_data(data: ModelData):
    lib().model_update_data(ctypes.byref(data))
    _check(lib().nmlmc_last_error(), "model_update_data")


def model_init(data: ModelData, seed: int):
    lib().model_init(ctypes.byref(data), seed)
    _check(lib().nmlmc_last_error(), "model_init")


def _sample_output(moments=4):
    f = np.zeros(moments)
    d = np.zeros(moments)
    so = SampleOutput(0, _p(f, _dp), _p(d, _dp), 0.0)
    return so, f, d


def model_sample(ell: int, M: int) -> dict:
    so, f, d = _sample_output()
    lib().model_sample(ell, M, ctypes.byref(so))
    _check(lib().nmlmc_last_error(), "model_sample")
    return dict(M=so.M, fsums=f, diffsums=d, work=so.total_work,
                stats=np.array(so.inner_stats[:], dtype=np.uint64))


def portfolio_update_data(data: PortfolioData):
    lib().portfolio_update_data(ctypes.byref(data))
    _check(lib().nmlmc_last_error(), "portfolio_update_data")


def portfolio_init(data: PortfolioData, seed: int):
    lib().portfolio_init(ctypes.byref(data), seed)
    _check(lib().nmlmc_last_error(), "portfolio_init")


def portfolio_sample(ell: int, override_dyn_inner: int, M: int) -> dict:
    so, f, d = _sample_output()
    lib().portfolio_sample(ell, override_dyn_inner, M, ctypes.byref(so))
    _check(lib().nmlmc_last_error(), "portfolio_sample")
    return dict(M=so.M, fsums=f, diffsums=d, work=so.total_work,
                stats=np.array(so.inner_stats[:], dtype=np.uint64))


def portfolio_cleanup():
    lib().portfolio_cleanup()


def portfolio_comp_params(data: PortfolioData):
    lib().portfolio_comp_params(ctypes.byref(data))


def norm_cdf_inv(p: float) -> float:
    return float(lib().norm_cdf_inv(p))


def make_portfolio_data(pf: dict, r=0.05, rho=0.0, max_loss=0.0, tau=1 / 52,
                        subsample=SUB_UNIFORM, use_delta_cv=False, method=None,
                        use_coarse_delta_cv=False, use_antithetic_risk=True, use_milstein=True,
                        dt_h0inv=8, dt_beta=4, dt_prob_expo=-1.5):
    """Builds a reference-layout portfolio_data from SoA arrays: option j goes to
    options[method[j]] (all BS when `method` is None), in order.  Returns the struct and the
    arrays that back it (keep them alive while the struct is in use)."""
    P, Q = len(pf["strike"]), len(pf["S0"])
    meth = np.zeros(P, np.int32) if method is None else np.asarray(method, np.int32)
    spans = []
    for m in range(3):
        idx = np.flatnonzero(meth == m)
        opts = (OptionParams * max(len(idx), 1))()
        for k, j in enumerate(idx):
            o = opts[k]
            o.strike, o.maturity, o.w = pf["strike"][j], pf["maturity"][j], pf["w"][j]
            o.stock_ind, o.type, o.prob, o.W_est = int(pf["stock_ind"][j]), int(pf["type"][j]), pf["prob"][j], 1.0
        spans.append((opts, len(idx)))
    stocks = (StockParams * Q)()
    for i in range(Q):
        stocks[i].S0, stocks[i].mu, stocks[i].sigma = pf["S0"][i], pf["mu"][i], pf["sigma"][i]
    d = PortfolioData()
    for m in range(3):
        d.options[m] = OptionsSpan(spans[m][0], spans[m][1])
    d.stocks = StocksSpan(stocks, Q)
    d.r, d.rho, d.max_loss, d.tau = r, rho, max_loss, tau
    d.s1_rho2 = float(np.sqrt(np.float32(1) - np.float32(rho) * np.float32(rho)))
    d.dt_h0inv, d.dt_beta, d.dt_prob_expo = dt_h0inv, dt_beta, dt_prob_expo
    d.phi_type, d._phi_size, d.subsample = 0, 1, subsample
    d.use_delta_cv, d.use_coarse_delta_cv = use_delta_cv, use_coarse_delta_cv
    d.use_antithetic_risk, d.use_milstein = use_antithetic_risk, use_milstein
    return d, ([sp[0] for sp in spans], stocks)


def make_batch(portfolios: list, K, r: float = 0.05, rho: float = 0.0, tau: float = TAU_WEEK) -> dict:
    """Concatenates portfolios (dicts of SoA arrays: S0, mu, sigma per stock; strike, maturity, w,
    stock_ind, type per option) into the batch layout of nmlmc_path_adjoint."""
    so, oo = [0], [0]
    cat = {k: [] for k in ("S0", "mu", "sigma", "strike", "maturity", "w", "stock_ind", "type")}
    for pf in portfolios:
        for k in cat:
            cat[k].append(np.asarray(pf[k]))
        so.append(so[-1] + len(pf["S0"]))
        oo.append(oo[-1] + len(pf["strike"]))
    out = {k: np.concatenate(v) for k, v in cat.items()}
    out.update(stock_off=np.array(so, np.uint32), option_off=np.array(oo, np.uint32),
               K=np.asarray(K, np.float64).reshape(-1), r=r, rho=rho, tau=tau)
    return out


from . import checkpoint, tables  # noqa: E402  (file readers: checkpoints, printed reports)
