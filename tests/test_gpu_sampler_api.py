"""The SAMPLER extension interface on the batched path (include/nmlmc_sampler.cuh).

In the reference a new nested problem is a new SAMPLER class (inner_sampler_base, sample_outer,
copy_outer, init_inner_sampler, sample_inner, add_phi; nested_sampler.hpp:36-85, 102-275,
model_sampler.cpp:42-92) run by sample<SAMPLER>(ell, ...) (646-694).  tests/abi/user_sampler.cu
writes the X = Y + Z model of the benchmark as such a class; through the header it runs on the
library's batched kernels, and its level results equal the built-in KIND_SHIFT_MODEL's on the same
streams bit for bit (the same draws, the same FP32 or FP64 arithmetic in the same order), call
after call (each call takes the level's next outer indices).
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG, ROOT

pytestmark = pytest.mark.gpu

SRC = os.path.join(ROOT, "tests", "abi", "user_sampler.cu")
LIB = os.path.join(ROOT, "tests", "abi", "_build", "libuser_sampler.so")


def build_user_sampler():
    """nvcc for sm_100a against the header and libnmlmc.so (what __graft_entry__.build() does)."""
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
           "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(PKG, "csrc"), "-shared", "-o", LIB, SRC,
           "-L", os.path.join(PKG, "nmlmc"), "-lnmlmc", "-Xlinker", "-rpath,$ORIGIN/../../../nested-risk-mlmc_b200/nmlmc"]
    subprocess.run(cmd, check=True, capture_output=True)


def user_lib():
    deps = [SRC, os.path.join(ROOT, "include", "nmlmc_sampler.cuh"), os.path.join(PKG, "nmlmc", "libnmlmc.so")]
    deps += [os.path.join(PKG, "csrc", f) for f in os.listdir(os.path.join(PKG, "csrc")) if f.endswith((".cuh", ".h"))]
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(d) for d in deps):
        build_user_sampler()
    L = ctypes.CDLL(LIB)
    dp = ctypes.POINTER(ctypes.c_double)
    L.user_shift_init.argtypes = [ctypes.c_int32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float,
                                  ctypes.c_uint64, ctypes.c_double]
    L.user_shift_sample.argtypes = [ctypes.c_int32, ctypes.c_uint32, ctypes.c_uint64, dp, dp, dp,
                                    ctypes.POINTER(ctypes.c_uint64)]
    return L


@pytest.mark.parametrize("prec_name", ["fp32", "fp64"])
def test_user_sampler_equals_the_builtin_model(nm, prec_name):
    L = user_lib()
    fp64 = prec_name == "fp64"
    seed, N0, beta, r, K = 31, 32, 2, 1.5, 1.0
    assert L.user_shift_init(int(fp64), N0, beta, r, seed, K) == nm.OK
    s = nm.Sampler(0, N0=N0, beta=beta, adaptive_r=r, precision=nm.PREC_FP64 if fp64 else nm.PREC_FP32,
                   streams=nm.STREAMS_OUTER, seed=seed)
    s.set_model(nm.MODEL_SHIFT, 0.0, K)
    s.set_autotune(0)
    dp = ctypes.POINTER(ctypes.c_double)
    try:
        for ell, M in ((0, 20000), (3, 10000), (7, 3000), (3, 7001), (0, 1)):
            ref = s.sample(ell, M)
            f, d, w = np.zeros(4), np.zeros(4), np.zeros(1)
            st = np.zeros(6, np.uint64)
            rc = L.user_shift_sample(int(fp64), ell, M, f.ctypes.data_as(dp), d.ctypes.data_as(dp),
                                     w.ctypes.data_as(dp), st.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)))
            assert rc == nm.OK, (ell, M, rc)
            np.testing.assert_array_equal(f, ref["fsums"], err_msg=f"ell {ell}")
            np.testing.assert_array_equal(d, ref["diffsums"], err_msg=f"ell {ell}")
            assert w[0] == ref["work"]
            assert st[0] == ref["stats"][0] and st[1] == M
            assert st[2] == ref["stats"][2] and st[3] == ref["stats"][3]
    finally:
        L.user_shift_cleanup()
