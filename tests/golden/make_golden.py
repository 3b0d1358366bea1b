#!/usr/bin/env python3
"""Convert the reference's Matrix Market goldens into one committed fixture file.

The upstream test suite (``check/check/libisvd/core/stage/*.cxx``) reads
``data/*.mtx`` (dense "array real general", column-major values).  This script
reads those files from a reference checkout and writes
``tests/golden/isvd_golden.npz`` (float64 arrays, same orientation as the
Matrix Market matrices: A is m x n, Qs is m x Nl, ...), plus the iteration counts
the upstream tests pin (KN: 81 at tol 1e-4; WY: 21 at tol 1e-3,
``check/check/libisvd/core/stage/@x@_integrate_kolmogorov_nagumo.cxx:10-16``).

Run once where the reference tree exists:
    python tests/golden/make_golden.py [/path/to/reference]
The fixture is committed so that tests never read the reference tree at run time.
"""
import os
import sys

import numpy as np

NAMES = ["a", "a_sym", "o_gp", "q", "q_hr", "q_kn", "q_wy", "qs", "s", "s_sym", "u", "u_sym", "v", "ys", "ys_gp"]


def read_mtx_array(path):
    """Read a dense Matrix Market 'array real general' file (values column-major)."""
    with open(path) as fh:
        banner = fh.readline()
        if "array" not in banner or "real" not in banner:
            raise ValueError("unsupported Matrix Market banner in %s: %s" % (path, banner))
        line = fh.readline()
        while line.startswith("%"):
            line = fh.readline()
        m, n = (int(t) for t in line.split())
        vals = np.array([float(t) for t in fh.read().split()], dtype=np.float64)
    if vals.size != m * n:
        raise ValueError("%s: expected %d values, got %d" % (path, m * n, vals.size))
    return vals.reshape(n, m).T.copy()


def main(ref):
    data = os.path.join(ref, "data")
    out = {name: read_mtx_array(os.path.join(data, name + ".mtx")) for name in NAMES}
    out["kn_tol"] = np.array(1e-4)
    out["kn_iter"] = np.array(81)
    out["wy_tol"] = np.array(1e-3)
    out["wy_iter"] = np.array(21)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "isvd_golden.npz")
    np.savez_compressed(dst, **out)
    print(dst, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
