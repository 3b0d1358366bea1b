"""isvd_b200 -- B200-native integrated randomized SVD behind the iSVD C ABI.

The product is ``isvd_b200/libisvd_gpu_b200.so`` (C ABI declared in ``include/isvd.h``).
This package builds it (``python -m isvd_b200.build``) and binds it for Python callers
(``isvd_b200.load()`` returns an :class:`IsvdLib`).  There is no CPU fallback: loading fails
loudly when the library has not been built.
"""
import os

from .capi import MPI_COMM_WORLD, IsvdLib, Param, ptr  # noqa: F401

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libisvd_gpu_b200.so")
# ILP64 build (isvd_int_t = int64), the reference's "_64" variant: IsvdLib(LIB64_PATH)
LIB64_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libisvd_gpu_b200_64.so")
PRECISION_NATIVE = 0
PRECISION_MIXED = 1

_lib = None


def load():
    """Load libisvd_gpu_b200.so (once)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libisvd_gpu_b200.so is not built; run `python -m isvd_b200.build` "
                               "(needs nvcc for sm_100a)")
        _lib = IsvdLib(LIB_PATH)
    return _lib
