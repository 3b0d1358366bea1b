"""Matrix Market files without a GPU: isvd_?MtxRead against scipy.io.mmread (an independent
reader of the format) on every format / field / symmetry the reference's data files and demo
use or the format allows for real matrices, isvd_?MtxWrite round trips, the reference demo's way
of reading (include/mmio_shim/mmio.h banner + size, one isvd_dFget per value) against
isvd_dMtxRead in a C program, and the errors for malformed files."""
import ctypes
import os
import subprocess

import numpy as np
import pytest
import scipy.io
import scipy.sparse

from conftest import REPO


def mtx_read(lib, path, x="d", ordera=b"C", pad=0):
    return lib.mtx_read(path, x, ordera, pad)


def mtx_write(lib, path, a, x="d"):
    return lib.mtx_write(path, a, x)


def dense(x):
    return x.toarray() if scipy.sparse.issparse(x) else np.asarray(x)


@pytest.mark.parametrize("ordera,pad", [(b"C", 0), (b"R", 0), (b"C", 3), (b"R", 5)])
def test_array_general_matches_scipy(lib, tmp_path, ordera, pad):
    a = np.random.default_rng(0).standard_normal((37, 23)) * 10.0 ** np.random.default_rng(1).integers(-8, 8, (37, 23))
    p = tmp_path / "a.mtx"
    scipy.io.mmwrite(str(p), a, comment="test matrix\nsecond comment line")
    st, b = mtx_read(lib, p, ordera=ordera, pad=pad)
    assert st == 0
    assert np.array_equal(b, dense(scipy.io.mmread(str(p))))


def test_golden_matrix_round_trip(lib, golden, tmp_path):
    """The reference's data/a.mtx matrix (tests/golden), written by scipy and by isvd_dMtxWrite."""
    a = golden["a"]
    p1, p2 = tmp_path / "scipy.mtx", tmp_path / "ours.mtx"
    scipy.io.mmwrite(str(p1), a)
    st, b = mtx_read(lib, p1)
    assert st == 0 and np.array_equal(b, dense(scipy.io.mmread(str(p1))))
    assert mtx_write(lib, p2, a) == 0
    st, c = mtx_read(lib, p2)
    assert st == 0 and np.array_equal(c, a)
    assert np.array_equal(dense(scipy.io.mmread(str(p2))), a)
    head = open(p2).read(80).splitlines()
    assert head[0] == "%%MatrixMarket matrix array real general" and head[1] == "101 1001"


@pytest.mark.parametrize("kind", ["coordinate_general", "coordinate_symmetric", "coordinate_skew", "array_symmetric",
                                  "array_skew", "coordinate_integer", "coordinate_pattern", "array_integer"])
def test_formats_match_scipy(lib, tmp_path, kind):
    rng = np.random.default_rng(2)
    p = tmp_path / (kind + ".mtx")
    if kind == "coordinate_general":
        scipy.io.mmwrite(str(p), scipy.sparse.random(40, 31, density=0.2, random_state=3, format="coo"))
    elif kind == "coordinate_symmetric":
        s = scipy.sparse.random(30, 30, density=0.2, random_state=4)
        scipy.io.mmwrite(str(p), (s + s.T).tocoo(), symmetry="symmetric")
    elif kind == "coordinate_skew":
        s = scipy.sparse.random(30, 30, density=0.2, random_state=5)
        scipy.io.mmwrite(str(p), (s - s.T).tocoo(), symmetry="skew-symmetric")
    elif kind == "array_symmetric":
        s = rng.standard_normal((17, 17))
        scipy.io.mmwrite(str(p), s + s.T, symmetry="symmetric")
    elif kind == "array_skew":
        s = rng.standard_normal((17, 17))
        scipy.io.mmwrite(str(p), s - s.T, symmetry="skew-symmetric")
    elif kind == "coordinate_integer":
        scipy.io.mmwrite(str(p), scipy.sparse.random(20, 25, density=0.3, random_state=6, format="coo",
                                                     data_rvs=lambda k: rng.integers(-50, 50, k)).astype(np.int64))
    elif kind == "coordinate_pattern":
        s = scipy.sparse.random(20, 25, density=0.3, random_state=7, format="coo")
        scipy.io.mmwrite(str(p), s, field="pattern")
    else:
        scipy.io.mmwrite(str(p), rng.integers(-9, 9, (12, 8)), field="integer")
    st, b = mtx_read(lib, p)
    assert st == 0, lib.last_error()
    assert np.array_equal(b, dense(scipy.io.mmread(str(p))).astype(np.float64))
    st, c = mtx_read(lib, p, ordera=b"R", pad=2)
    assert st == 0 and np.array_equal(c, b)


def test_single_precision_reads_each_value_once(lib, tmp_path):
    """isvd_sMtxRead rounds each decimal once to FP32 (as fscanf("%f") does)."""
    a = np.random.default_rng(8).standard_normal((50, 40)).astype(np.float32)
    p = tmp_path / "s.mtx"
    with open(p, "w") as f:
        f.write("%%MatrixMarket matrix array real general\n50 40\n")
        f.write("\n".join(repr(float(v)) for v in a.T.ravel()) + "\n")  # decimal of the double value
    st, b = mtx_read(lib, p, x="s")
    assert st == 0 and b.dtype == np.float32 and np.array_equal(b, a)
    assert mtx_write(lib, tmp_path / "w.mtx", a, x="s") == 0
    st, c = mtx_read(lib, tmp_path / "w.mtx", x="s")
    assert st == 0 and np.array_equal(c, a)


def test_large_file_parsed_in_parallel(lib, tmp_path):
    a = np.random.default_rng(9).standard_normal((1500, 1200))
    p = tmp_path / "big.mtx"
    assert mtx_write(lib, p, a) == 0
    assert os.path.getsize(p) > 16 << 20  # several 4 MB chunks
    st, b = mtx_read(lib, p, ordera=b"R")
    assert st == 0 and np.array_equal(b, a)


@pytest.mark.parametrize("text,needle", [
    ("%%MatrixMarket matrix array real general\n2 2\n1 2 3\n", "3 values for a 2 x 2 array"),
    ("%%MatrixMarket matrix array real general\n2 2\n1 2 x 4\n", "value 3 ('x') is not a number"),
    ("%%MatrixMarket matrix array complex general\n1 1\n1 0\n", "unsupported field 'complex'"),
    ("%MatrixMarket matrix array real general\n1 1\n1\n", "no %%MatrixMarket banner"),
    ("%%MatrixMarket matrix coordinate real general\n3 3 2\n1 1 1.0\n4 1 2.0\n", "outside 3 x 3"),
    ("%%MatrixMarket matrix array real symmetric\n2 3\n1 2 3\n", "non-square"),
    ("%%MatrixMarket matrix array real general\n% only a comment\n", "no size line")])
def test_malformed_files_are_refused(lib, tmp_path, text, needle):
    p = tmp_path / "bad.mtx"
    p.write_text(text)
    lib.clear_error()
    st, b = mtx_read(lib, p)
    assert st == 1 and b is None
    assert needle in lib.last_error()[1], lib.last_error()
    lib.clear_error()
    st, _ = mtx_read(lib, tmp_path / "missing.mtx")
    assert st == 1 and "cannot open" in lib.last_error()[1]


def test_c_reader_like_the_reference_demo(lib, golden, tmp_path):
    """mmio banner / size + isvd_dFget per value (the reference demo's reading) == isvd_dMtxRead."""
    exe = str(tmp_path / "mtx_read_check")
    libdir = os.path.dirname(lib.path)
    subprocess.run(["gcc", "-std=gnu99", "-O1", "-Wall", "-Werror", "-I", os.path.join(REPO, "include"), "-I",
                    os.path.join(REPO, "include", "mpi_shim"), "-I", os.path.join(REPO, "include", "mmio_shim"),
                    os.path.join(REPO, "tests", "c", "mtx_read_check.c"), "-o", exe, "-L" + libdir,
                    "-lisvd_gpu_b200", "-Wl,-rpath," + libdir], check=True, capture_output=True, text=True)
    p = tmp_path / "a.mtx"
    scipy.io.mmwrite(str(p), golden["a"])
    out = subprocess.run([exe, str(p)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "banner 0 [matrix array real general] valid 1" in out.stdout
    assert "size 101 1001 read 101 1001 status 0 fget 0 differ 0" in out.stdout
    sum_c = float(out.stdout.split("sum ")[1])
    assert abs(sum_c - golden["a"].sum(axis=0).sum()) < 1e-9 * np.abs(golden["a"]).sum()


def test_omp_queries(lib):
    """No OpenMP team: the reference's values without OpenMP (la/util/omp.c:20-63)."""
    L = lib.lib
    for name, want in (("isvd_getOmpMaxSize", 1), ("isvd_getOmpSize", 1), ("isvd_getOmpRank", 0)):
        getattr(L, name).restype = ctypes.c_int
        assert getattr(L, name)() == want


@pytest.mark.parametrize("ilp64", [False, True])
def test_headers_compile_as_cpp_and_mmio_writers_round_trip(tmp_path, lib, lib64, ilp64):
    """include/ compiles as C++17 (both index widths) and links with the matching library; the
    mmio writers' banner and size read back through the mmio readers and isvd_dFget."""
    L = lib64 if ilp64 else lib
    exe = str(tmp_path / "header_check")
    libdir = os.path.dirname(L.path)
    name = "isvd_gpu_b200_64" if ilp64 else "isvd_gpu_b200"
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(REPO, "include"), "-I",
           os.path.join(REPO, "include", "mpi_shim"), "-I", os.path.join(REPO, "include", "mmio_shim"),
           os.path.join(REPO, "tests", "c", "header_check.cpp"), "-o", exe, "-L" + libdir, "-l" + name,
           "-Wl,-rpath," + libdir]
    if ilp64:
        cmd.insert(1, "-DISVD_USE_ILP64")
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    out = subprocess.run([exe, str(tmp_path / "w.mtx")], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, (out.returncode, out.stdout, out.stderr)
    assert out.stdout.strip() == "sum 18.0 dim_sketch 6 omp 1 error 0"
