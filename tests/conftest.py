"""Shared fixtures.  `-m gpu` tests need a CUDA device (B200); everything else runs on CPU."""
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "oracle"))
GOLDEN = os.path.join(REPO, "tests", "golden", "isvd_golden.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _has_gpu():
    try:
        import ctypes
        rt = ctypes.CDLL("libcuda.so.1")
        n = ctypes.c_int(0)
        if rt.cuInit(0) != 0:
            return False
        return rt.cuDeviceGetCount(ctypes.byref(n)) == 0 and n.value > 0
    except OSError:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(GOLDEN))


@pytest.fixture(scope="session")
def oracle():
    import isvd_oracle
    return isvd_oracle


@pytest.fixture(scope="session")
def reflib():
    """The reference library built from source (oracle/_ref) -- the checker."""
    import build_ref
    from isvd_b200.capi import IsvdLib
    path = build_ref.build()
    return IsvdLib(path)


@pytest.fixture(scope="session")
def lib():
    """The product library (libisvd_gpu_b200.so)."""
    import isvd_b200
    return isvd_b200.load()


@pytest.fixture(scope="session")
def lib64():
    """The ILP64 build of the product library (libisvd_gpu_b200_64.so: isvd_int_t = int64)."""
    import isvd_b200
    if not os.path.exists(isvd_b200.LIB64_PATH):
        raise RuntimeError("libisvd_gpu_b200_64.so is not built; run `python -m isvd_b200.build --ilp64`")
    from isvd_b200.capi import IsvdLib
    return IsvdLib(isvd_b200.LIB64_PATH)
