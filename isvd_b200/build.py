"""Build libisvd_gpu_b200.so in-tree with nvcc for sm_100a.

    python -m isvd_b200.build [--force] [--verbose] [--ilp64]

Each CUDA source under isvd_b200/csrc is compiled with
``-gencode arch=compute_100a,code=sm_100a -O3 -lineinfo`` and the objects are linked
into ``isvd_b200/libisvd_gpu_b200.so`` (static CUDA runtime, C ABI of include/isvd.h).
``--ilp64`` builds the 64-bit-index variant (``isvd_int_t`` = int64, ``-DISVD_USE_ILP64``)
as ``isvd_b200/libisvd_gpu_b200_64.so``, the reference's ``_64`` suffix for that build
(reference cmake/options.cmake:50-61).  Sources are rebuilt only when they (or a header) are
newer than their object.
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
FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "-Xcompiler", "-fvisibility=hidden,-fvisibility-inlines-hidden",
                "--expt-relaxed-constexpr", "-I" + os.path.join(REPO, "include"),
                "-I" + os.path.join(REPO, "include", "mpi_shim"), "-I" + CSRC]


def _newest_header():
    hs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
    hs += glob.glob(os.path.join(REPO, "include", "**", "*.h"), recursive=True)
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def build(force=False, verbose=False, extra=(), ilp64=False):
    if ilp64:
        return _build(OBJ64, LIB64, force, verbose, tuple(extra) + ("-DISVD_USE_ILP64",))
    return _build(OBJ, LIB, force, verbose, extra)


def build_all(force=False, verbose=False):
    """Both index variants: the LP64 library and the ILP64 (_64) one."""
    lib = build(force, verbose)
    build(force, verbose, ilp64=True)
    return lib


def _build(OBJ, LIB, force, verbose, extra):
    os.makedirs(OBJ, exist_ok=True)
    # a change of compiler flags rebuilds everything
    stamp = os.path.join(OBJ, "flags.txt")
    flags = " ".join([NVCC] + FLAGS + list(extra))
    if not os.path.exists(stamp) or open(stamp).read() != flags:
        force = True
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdr = _newest_header()

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
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcuda", "-Xlinker", "--version-script=" + vmap]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s%s" % (r.stdout, r.stderr))
    with open(stamp, "w") as fh:
        fh.write(flags)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv, ilp64="--ilp64" in sys.argv))
