"""C ABI checks that need no GPU: every function and variable declared under include/ is
exported by libisvd_gpu_b200.so; host-only entry points (parameters, memory helpers,
argument errors) behave like the reference's."""
import ctypes
import glob
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import REPO


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(REPO, "include", "isvd", "**", "*.h"), recursive=True):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        text = re.sub(r"static\s+inline[^{;]*\{[^}]*\}", "", text, flags=re.S)
        text = re.sub(r"#[^\n]*", "", text)
        names |= set(re.findall(r"\b(isvd_\w+)\s*\(", text))
        names |= set(re.findall(r"extern\s+[\w\s\*]+?\b(isvd_\w+)\s*;", text))
    return names


def exported_symbols(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if ln.strip()}


def test_library_exports_every_declared_symbol(lib):
    decl = declared_symbols()
    assert len(decl) >= 55
    missing = decl - exported_symbols(lib.path)
    assert not missing, sorted(missing)


def test_only_c_abi_exported(lib):
    extra = {s for s in exported_symbols(lib.path) if not s.startswith("isvd_")}
    assert not extra, sorted(extra)


def test_reference_driver_and_stage_symbols_present(lib, reflib):
    """Every isvd_ entry point the reference's core/gpu/util layers export at the stage/driver level
    is exported by the B200 library too (drop-in link)."""
    wanted = {s for s in exported_symbols(reflib.path)
              if re.match(r"isvd_[sd](Isvd|Sketch|Orthogonalize|Integrate|Postprocess)", s)
              or s in ("isvd_createParam", "isvd_getMpiSize", "isvd_getMpiRank", "isvd_Init_cpu",
                       "isvd_Finalize_cpu", "isvd_PrintEnvironment_cpu")}
    wanted |= {"isvd_%s%s_gpu" % (x, n) for x in "sd" for n in
               ("SketchGaussianProjection", "PostprocessGramian", "PostprocessTallSkinnyQr", "PostprocessSymmetric")}
    wanted |= {"isvd_Init_gpu", "isvd_Finalize_gpu", "isvd_PrintEnvironment_gpu", "isvd_gpu_memory_limit"}
    missing = wanted - exported_symbols(lib.path)
    assert not missing, sorted(missing)


@pytest.mark.parametrize("m,n,k,p,N", [(101, 1001, 11, 0, 12), (2000, 1000, 20, 12, 16), (7, 5, 2, 1, 3)])
def test_create_param_matches_reference(lib, reflib, m, n, k, p, N):
    a = lib.create_param(m, n, k, p, N)
    b = reflib.create_param(m, n, k, p, N)
    for f, _ in a._fields_:
        assert getattr(a, f) == getattr(b, f), f
    assert a.dim_sketch == k + p and a.dim_sketch_total == (k + p) * N


def test_memory_helpers(lib):
    L = lib.lib
    L.isvd_dMalloc.restype = ctypes.c_void_p
    L.isvd_dMalloc.argtypes = [ctypes.c_size_t]
    L.isvd_Free.argtypes = [ctypes.c_void_p]
    L.isvd_dMemset0.argtypes = [ctypes.c_void_p, ctypes.c_size_t]
    p = L.isvd_dMalloc(1000)
    assert p and p % 64 == 0
    L.isvd_dMemset0(p, 1000)
    arr = np.ctypeslib.as_array((ctypes.c_double * 1000).from_address(p))
    assert not arr.any()
    L.isvd_Free(p)


def test_bad_selector_prints_and_returns(lib, capfd):
    """Reference core/driver/@x@_isvd.c:140-144 + util/arg.h:70-78: print and return."""
    lib.clear_error()
    prm = lib.create_param(20, 10, 2, 1, 2)
    _, _, _ = lib.isvd("d", prm, ("GP", "XX", "KN", "GR"), None, 10, None, None, 3, None, 3)
    err = capfd.readouterr().err
    assert "ALG_O ('XX') must be one of the following strings" in err
    assert lib.last_error()[0] == 1


def test_bad_layout_char(lib, capfd):
    lib.clear_error()
    prm = lib.create_param(20, 10, 2, 1, 2)
    lib.sketch("d", prm, np.zeros((20, 10)), 10, np.zeros((20, 6)), 6, 0, dista=b"X")
    assert "DISTA ('X') must be one of the following characters: 'C', 'R'" in capfd.readouterr().err
    assert lib.last_error()[0] == 1


def test_query_defaults_without_gpu(lib, reflib):
    for alg, n in (("KN", 2), ("WY", 9)):
        assert list(lib.query("d", alg, n)) == list(reflib.query("d", alg, n))
        assert np.allclose(lib.query("s", alg, n), reflib.query("s", alg, n))


def test_ilp64_library_exports_the_same_abi(lib, lib64):
    """The ILP64 build (reference cmake/options.cmake:50-61: isvd_int_t = int64, suffix _64) exports
    exactly the LP64 build's entry points."""
    assert exported_symbols(lib64.path) == exported_symbols(lib.path)


@pytest.mark.parametrize("m,n,k,p,N", [(2000, 1000, 20, 12, 16), (5_000_000_000, 3, 2, 1, 3)])
def test_ilp64_param_fields_are_64_bit(lib, lib64, m, n, k, p, N):
    """isvd_Param's index fields are int64 in the ILP64 build: a row count beyond int32 survives."""
    import ctypes as ct
    assert lib64.Param.nrow.size == 8 and lib.Param.nrow.size == 4
    a = lib64.create_param(m, n, k, p, N)
    assert a.nrow == m and a.dim_sketch == k + p and a.dim_sketch_total == (k + p) * N
    if m < 2 ** 31:
        b = lib.create_param(m, n, k, p, N)
        for f, _ in b._fields_:
            assert getattr(a, f) == getattr(b, f), f
    assert ct.sizeof(lib64.Param) > ct.sizeof(lib.Param)


def build_c_demo(tmp_path, lib):
    """Compile tests/c/isvd_demo.c against include/ and link it with the library (plain gcc)."""
    exe = str(tmp_path / "isvd_demo")
    libdir = os.path.dirname(lib.path)
    cmd = ["gcc", "-std=gnu99", "-O1", "-Wall", "-Werror", "-I", os.path.join(REPO, "include"), "-I",
           os.path.join(REPO, "include", "mpi_shim"), os.path.join(REPO, "tests", "c", "isvd_demo.c"), "-o", exe,
           "-L" + libdir, "-lisvd_gpu_b200", "-Wl,-rpath," + libdir, "-lm"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_c_caller_compiles_and_links(tmp_path, lib):
    """A C program written against include/isvd.h builds and links against the library alone."""
    exe = build_c_demo(tmp_path, lib)
    assert os.path.exists(exe)


def test_c_caller_links_ilp64(tmp_path, lib64):
    """The same C program compiled with -DISVD_USE_ILP64 links against the _64 library."""
    exe = str(tmp_path / "isvd_demo64")
    libdir = os.path.dirname(lib64.path)
    cmd = ["gcc", "-std=gnu99", "-O1", "-Wall", "-Werror", "-DISVD_USE_ILP64", "-I", os.path.join(REPO, "include"),
           "-I", os.path.join(REPO, "include", "mpi_shim"), os.path.join(REPO, "tests", "c", "isvd_demo.c"), "-o",
           exe, "-L" + libdir, "-lisvd_gpu_b200_64", "-Wl,-rpath," + libdir, "-lm"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    assert os.path.exists(exe)
