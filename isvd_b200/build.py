"""Build libisvd_gpu_b200.so in-tree with nvcc for sm_100a.

    python -m isvd_b200.build [--force] [--verbose] [--ilp64]
                              [--mpi-include DIR [--mpi-lib DIR] [--mpi-libs "-lmpi ..."] [--out PATH]]

Each CUDA source under isvd_b200/csrc is compiled with
``-gencode arch=compute_100a,code=sm_100a -O3 -lineinfo`` and the objects are linked
into ``isvd_b200/libisvd_gpu_b200.so`` (static CUDA runtime, C ABI of include/isvd.h).
``--ilp64`` builds the 64-bit-index variant (``isvd_int_t`` = int64, ``-DISVD_USE_ILP64``)
as ``isvd_b200/libisvd_gpu_b200_64.so``, the reference's ``_64`` suffix for that build
(reference cmake/options.cmake:50-61).  Sources are rebuilt only when they (or a header) are
newer than their object.

``isvd_Param`` embeds the caller's ``MPI_Comm`` (reference src/include/c/isvd/def.h and
core/param.h), so the library and the program must be compiled against the same ``mpi.h``: its
type and size differ between MPI implementations (an ``int`` handle in MPICH, a pointer in Open
MPI).  By default the library is compiled against the single-rank stand-in
``include/mpi_shim/mpi.h``.  ``--mpi-include DIR`` compiles it against the ``mpi.h`` in DIR instead
and links the MPI library (``--mpi-lib DIR``, ``--mpi-libs``, default ``-lmpi``): then
``isvd_Init_cpu``, ``isvd_Finalize_cpu``, ``isvd_getMpiSize`` and ``isvd_getMpiRank`` call that
MPI, and the ranks of a communicator with more than one process join as row blocks with their
exchanges run as ``MPI_Allreduce`` on the communicator in ``isvd_Param`` (unless the program has
installed its own reduction with ``isvd_gpu_set_allreduce``).  Such a build goes to ``--out``
(default: the in-tree library name) and its objects to a folder of its own.
"""
import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libisvd_gpu_b200.so")
OBJ64 = os.path.join(HERE, "_build64")
LIB64 = os.path.join(HERE, "libisvd_gpu_b200_64.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
MPI_SHIM = os.path.join(REPO, "include", "mpi_shim")
FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "-Xcompiler", "-fvisibility=hidden,-fvisibility-inlines-hidden",
                "--expt-relaxed-constexpr", "-I" + os.path.join(REPO, "include"), "-I" + CSRC]


def _newest_header():
    hs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
    hs += glob.glob(os.path.join(REPO, "include", "**", "*.h"), recursive=True)
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def build(force=False, verbose=False, extra=(), ilp64=False):
    if ilp64:
        return _build(OBJ64, LIB64, force, verbose, tuple(extra) + ("-DISVD_USE_ILP64",))
    return _build(OBJ, LIB, force, verbose, extra)


def build_mpi(mpi_include, out, objdir=None, mpi_lib=None, mpi_libs=("-lmpi",), ilp64=False, force=False,
              verbose=False):
    """The library compiled against the caller's mpi.h (in mpi_include) and linked with its MPI
    library; written to `out`, objects to `objdir` (default: next to `out`)."""
    out = os.path.abspath(out)
    objdir = objdir or out + ".obj"
    extra = ["-DISVD_USE_ILP64"] if ilp64 else []
    link = (["-L" + mpi_lib, "-Xlinker", "-rpath," + mpi_lib] if mpi_lib else []) + list(mpi_libs)
    return _build(objdir, out, force, verbose, tuple(extra), mpi_include=os.path.abspath(mpi_include), link=link)


def build_all(force=False, verbose=False):
    """Both index variants: the LP64 library and the ILP64 (_64) one."""
    lib = build(force, verbose)
    build(force, verbose, ilp64=True)
    return lib


def _build(OBJ, LIB, force, verbose, extra, mpi_include=MPI_SHIM, link=()):
    os.makedirs(OBJ, exist_ok=True)
    extra = tuple(extra) + ("-I" + mpi_include,)
    # a change of compiler flags rebuilds everything
    stamp = os.path.join(OBJ, "flags.txt")
    flags = " ".join([NVCC] + FLAGS + list(extra) + list(link))
    if not os.path.exists(stamp) or open(stamp).read() != flags:
        force = True
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdr = max(_newest_header(), max((os.path.getmtime(h) for h in glob.glob(os.path.join(mpi_include, "*.h"))),
                                    default=0.0))

    def compile_one(src):
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr):
            return obj, False
        cmd = [NVCC] + FLAGS + list(extra) + ["-c", src, "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s%s" % (src, r.stdout, r.stderr))
        if verbose and r.stderr:
            sys.stderr.write(r.stderr)
        return obj, True

    with ThreadPoolExecutor(max_workers=max(2, os.cpu_count() or 2)) as ex:
        results = list(ex.map(compile_one, srcs))
    objs = [o for o, _ in results]
    if force or any(c for _, c in results) or not os.path.exists(LIB):
        # export the C ABI only (isvd_*); template code instantiated from the C++ standard library
        # would otherwise be exported with default visibility
        vmap = os.path.join(OBJ, "exports.map")
        with open(vmap, "w") as fh:
            fh.write("{ global: isvd_*; local: *; };\n")
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcuda", "-Xlinker", "--version-script=" + vmap] + \
            list(link)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s%s" % (r.stdout, r.stderr))
    with open(stamp, "w") as fh:
        fh.write(flags)
    return LIB


def _arg(name, default=None):
    return sys.argv[sys.argv.index(name) + 1] if name in sys.argv else default


if __name__ == "__main__":
    force, verbose, ilp64 = "--force" in sys.argv, "--verbose" in sys.argv, "--ilp64" in sys.argv
    if "--mpi-include" in sys.argv:
        default_out = LIB64 if ilp64 else LIB
        print(build_mpi(_arg("--mpi-include"), _arg("--out", default_out), mpi_lib=_arg("--mpi-lib"),
                        mpi_libs=tuple(_arg("--mpi-libs", "-lmpi").split()), ilp64=ilp64, force=force,
                        verbose=verbose))
    else:
        print(build(force=force, verbose=verbose, ilp64=ilp64))
