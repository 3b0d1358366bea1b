"""The C caller (tests/c/isvd_demo.c) runs on the GPU through the C ABI and reproduces the
singular values of its own test matrix."""
import re
import subprocess

import numpy as np
import pytest

from test_abi import build_c_demo

pytestmark = pytest.mark.gpu


def test_c_demo_runs(tmp_path, lib):
    exe = build_c_demo(tmp_path, lib)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert "Using Real Double Precision GPU Kolmogorov-Nagumo Integration." in out.stdout
    sig = np.array([float(x) for x in re.search(r"sigma:(.*)", out.stdout).group(1).split()])
    m, n = 1200, 800
    i = np.arange(1, m + 1)[:, None]
    j = np.arange(1, n + 1)[None, :]
    a = sum(0.8 ** r * np.cos(0.37 * (r + 1) * i) * np.sin(0.53 * (r + 1) * j) for r in range(12))
    ref = np.linalg.svd(a, compute_uv=False)[:10]
    assert np.abs(sig - ref).max() < 1e-6 * ref[0]
