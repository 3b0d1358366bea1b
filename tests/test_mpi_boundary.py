"""The boundary for programs built against a real MPI (no GPU needed).

isvd_Param embeds the caller's MPI_Comm (reference src/include/c/isvd/def.h, core/param.h), whose
type differs between MPI implementations, so the library must be built against the program's
mpi.h (isvd_b200/build.py --mpi-include).  tests/c/mpi_ptr/mpi.h stands in for an MPI whose
communicator is a pointer (as Open MPI's is):

* the layout of isvd_Param (size, alignment, every field's offset and size) under that header and
  under the single-rank stand-in equals the reference's own core/param.h under the same header, for
  both index widths;
* a library built against it reads and writes isvd_Param with the pointer-sized communicator: the
  communicator's size and rank come from its MPI_Comm_size / MPI_Comm_rank, isvd_createParam splits
  the rows as the reference does, the struct passed by value is read at the right offsets, the
  ranks of a communicator with several processes join as row blocks, and only isvd_* symbols are
  exported.
"""
import ctypes
import os
import subprocess
import tempfile

import pytest

from conftest import REPO

MPI_PTR = os.path.join(REPO, "tests", "c", "mpi_ptr")
MPI_SHIM = os.path.join(REPO, "include", "mpi_shim")


def _reference_include():
    import build_ref
    if not os.path.isdir(os.path.join(build_ref.REF, "src", "include", "c")):
        pytest.skip("reference source tree not present")
    d = tempfile.mkdtemp(prefix="isvd_refinc_")
    build_ref.configure(os.path.join(build_ref.REF, "src", "include", "c"), os.path.join(d, "include"))
    return os.path.join(d, "include")


def _layout(include, mpi, ilp64, tmp):
    exe = os.path.join(tmp, "layout_%d_%d" % (hash(include) & 0xffff, ilp64))
    cmd = ["gcc", "-std=gnu99", "-I" + mpi, "-I" + include] + (["-DISVD_USE_ILP64"] if ilp64 else [])
    subprocess.run(cmd + [os.path.join(REPO, "tests", "c", "param_layout.c"), "-o", exe], check=True)
    return subprocess.run([exe], capture_output=True, text=True, check=True).stdout


@pytest.mark.parametrize("ilp64", [False, True])
@pytest.mark.parametrize("mpi", [MPI_PTR, MPI_SHIM], ids=["pointer-comm", "int-comm"])
def test_param_layout_matches_reference(tmp_path, mpi, ilp64):
    ref_inc = _reference_include()
    ours = _layout(os.path.join(REPO, "include"), mpi, ilp64, str(tmp_path))
    theirs = _layout(ref_inc, mpi, ilp64, str(tmp_path))
    assert ours == theirs
    assert len(ours.splitlines()) == 22
    if mpi == MPI_PTR:
        assert ours.splitlines()[1] == "mpi_comm 0 %d" % ctypes.sizeof(ctypes.c_void_p)


class Comm(ctypes.Structure):
    _fields_ = [("size", ctypes.c_int), ("rank", ctypes.c_int),
                ("allreduce", ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p)),
                ("user", ctypes.c_void_p)]


class PtrParam(ctypes.Structure):
    _fields_ = [("mpi_comm", ctypes.c_void_p), ("mpi_size", ctypes.c_int), ("mpi_root", ctypes.c_int),
                ("mpi_rank", ctypes.c_int)] + [(f, ctypes.c_int32) for f in (
                    "nrow", "ncol", "nrow_proc", "ncol_proc", "nrow_each", "ncol_each", "nrow_total", "ncol_total",
                    "rowidxbegin", "rowidxend", "colidxbegin", "colidxend", "rank", "over_rank", "dim_sketch",
                    "dim_sketch_total", "num_sketch")]


@pytest.fixture(scope="module")
def ptrlib(tmp_path_factory):
    from isvd_b200 import build
    out = str(tmp_path_factory.mktemp("mpiptr") / "libisvd_gpu_b200_mpiptr.so")
    path = build.build_mpi(MPI_PTR, out, mpi_libs=())
    lib = ctypes.CDLL(path)
    lib.isvd_createParam.argtypes = [ctypes.c_int32] * 5 + [ctypes.c_int, ctypes.c_void_p]
    lib.isvd_createParam.restype = PtrParam
    lib.isvd_getMpiSize.argtypes = [ctypes.c_void_p]
    lib.isvd_getMpiRank.argtypes = [ctypes.c_void_p]
    lib.isvd_gpu_get_last_error.restype = ctypes.c_int
    lib.isvd_gpu_get_error_string.restype = ctypes.c_char_p
    return path, lib


def _last_error(lib):
    return lib.isvd_gpu_get_last_error(), (lib.isvd_gpu_get_error_string() or b"").decode()


def test_pointer_comm_library(ptrlib, oracle):
    path, lib = ptrlib
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    assert all(ln.split()[-1].startswith("isvd_") for ln in out.splitlines() if ln.strip())
    comm = Comm(3, 1)
    assert lib.isvd_getMpiSize(ctypes.addressof(comm)) == 3
    assert lib.isvd_getMpiRank(ctypes.addressof(comm)) == 1
    assert lib.isvd_getMpiSize(None) == 1
    m, n = 1001, 3000
    prm = lib.isvd_createParam(m, n, 3, 2, 4, 0, ctypes.addressof(comm))
    assert prm.mpi_comm == ctypes.addressof(comm)
    assert (prm.mpi_size, prm.mpi_rank, prm.mpi_root) == (3, 1, 0)
    rb, re = oracle.row_block(m, 3, 1)
    cb, ce = oracle.row_block(n, 3, 1)
    assert (prm.rowidxbegin, prm.rowidxend, prm.nrow_proc) == (rb, re, re - rb)
    assert (prm.colidxbegin, prm.colidxend, prm.ncol_proc) == (cb, ce, ce - cb)
    assert (prm.dim_sketch, prm.dim_sketch_total, prm.num_sketch) == (5, 20, 4)

    # the struct passed by value is read at the right offsets: the one-rank-only entry point names
    # the communicator's size
    fn = lib.isvd_dIntegrateKolmogorovNagumo_noalloc
    fn.argtypes = [PtrParam, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
                   ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    assert fn(prm, None, 0, None, 0, None, 20, None, 5, None) == 6
    code, msg = _last_error(lib)
    assert code == 6 and "MPI size 3" in msg

    # a stage called with the 3-rank parameters joins the communicator's ranks (its argument check
    # then fails before any device work); one-rank parameters leave them again
    orth = lib.isvd_dOrthogonalizeGramian
    orth.argtypes = [PtrParam, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
                     ctypes.c_int32]
    # (observed through the one-rank-only entry point, which reports the joined ranks)
    orth(prm, None, 0, None, 0, None, 0)
    assert _last_error(lib)[0] == 1
    one = lib.isvd_createParam(m, n, 3, 2, 4, 0, None)
    assert one.mpi_size == 1
    assert fn(one, None, 0, None, 0, None, 20, None, 5, None) == 6
    assert "MPI size 1, 3 joined ranks" in _last_error(lib)[1]
    orth(one, None, 0, None, 0, None, 0)
    assert fn(prm, None, 0, None, 0, None, 20, None, 5, None) == 6
    assert "MPI size 3, 1 joined ranks" in _last_error(lib)[1]
