"""The C callers run on the GPU through the C ABI: tests/c/isvd_demo.c reproduces the singular
values of its own test matrix; tests/c/isvd_mtx_demo.c (the reference demo's flow: Matrix Market
input read by mmio + isvd_dFget, dista 'R', ordera 'C') gives the results of the same solve made
through the Python binding, written back as Matrix Market files."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import REPO
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


def test_mtx_demo_matches_the_binding(tmp_path, lib, golden):
    import scipy.io
    exe = str(tmp_path / "isvd_mtx_demo")
    libdir = os.path.dirname(lib.path)
    subprocess.run(["gcc", "-std=gnu99", "-O1", "-Wall", "-Werror", "-I", os.path.join(REPO, "include"), "-I",
                    os.path.join(REPO, "include", "mpi_shim"), "-I", os.path.join(REPO, "include", "mmio_shim"),
                    os.path.join(REPO, "tests", "c", "isvd_mtx_demo.c"), "-o", exe, "-L" + libdir,
                    "-lisvd_gpu_b200", "-Wl,-rpath," + libdir, "-lm"], check=True, capture_output=True, text=True)
    a = golden["a"]  # the reference's data/a.mtx matrix, 101 x 1001
    m, n = a.shape
    pa, ps, pu, pv = (str(tmp_path / (x + ".mtx")) for x in "asuv")
    scipy.io.mmwrite(pa, a)
    out = subprocess.run([exe, pa, ps, pu, pv], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "readers agree: yes" in out.stdout
    assert "Average sketching time:" in out.stdout
    s_c = np.asarray(scipy.io.mmread(ps)).ravel()
    u_c = np.asarray(scipy.io.mmread(pu))
    v_c = np.asarray(scipy.io.mmread(pv))
    k, p, N = 20, 12, 16
    l = k + p
    prm = lib.create_param(m, n, k, p, N)
    s = np.zeros(l)
    ut = np.zeros((m, l))
    vt = np.zeros((n, l))
    lib.isvd("d", prm, ("GP_gpu", "GR", "KN", "GR_gpu"), np.asfortranarray(a).T.copy(), m, s, ut, l, vt, l,
             seed=0, dista=b"R", ordera=b"C", ut_root=0, vt_root=0)
    assert lib.last_error()[0] == 0
    assert s_c.shape == (l,) and u_c.shape == (m, k) and v_c.shape == (n, k)
    assert np.array_equal(s_c, s)  # the shortest decimal form reads back exactly
    assert np.array_equal(u_c, ut[:, :k]) and np.array_equal(v_c, vt[:, :k])
    assert np.abs(s[:k] - np.linalg.svd(a, compute_uv=False)[:k]).max() < 0.05 * s[0]
