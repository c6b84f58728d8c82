"""Shared test set-up: import paths, the `gpu` marker and GPU detection."""
import ctypes
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "nested-risk-mlmc_b200")
for p in (ROOT, PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _gpu_count() -> int:
    try:
        cu = ctypes.CDLL("libcuda.so.1")
    except OSError:
        return 0
    if cu.cuInit(0) != 0:
        return 0
    n = ctypes.c_int(0)
    if cu.cuDeviceGetCount(ctypes.byref(n)) != 0:
        return 0
    return n.value


HAVE_GPU = _gpu_count() > 0


def pytest_collection_modifyitems(config, items):
    if HAVE_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device on this host")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN, "cases.json")) as f:
        meta = json.load(f)
    arrays = dict(np.load(os.path.join(GOLDEN, "arrays.npz")))
    return meta, arrays


@pytest.fixture(scope="session")
def nm():
    """The product's Python host module; builds libnmlmc.so first if it is missing."""
    import subprocess
    lib = os.path.join(PKG, "nmlmc", "libnmlmc.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", PKG, "-j8"], check=True, capture_output=True)
    import nmlmc
    return nmlmc
