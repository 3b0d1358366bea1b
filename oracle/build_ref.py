#!/usr/bin/env python3
"""Build the upstream iSVD C library (emfomy/isvd v1.3.2) as a CPU checker.

TEST INFRASTRUCTURE ONLY.  The shared library this script produces,
``oracle/_ref/liboracle_isvd.so``, is the reference's own CPU code path
(BLAS/LAPACK through OpenBLAS, one MPI rank through ``include/mpi_shim``).
Tests and ``bench.py --impl reference`` load it to check and to time against;
the product library never links it.

Recipe (nothing is copied into the repository):
  1. Instantiate the ``@x@`` templates of ``src/include/c`` and ``src/lib`` for
     ``s`` and ``d`` into a temporary directory, the way
     ``cmake/configure.cmake:20-35`` + ``cmake/vars.cmake:2-23`` do
     (``@x@ @X@ @xtype_____@ @XTYPE@ @XName@ @xname@ @XStr@``), and fill
     ``@ISVD_*_VERSION@`` from ``CMakeLists.txt:9-11``.
  2. Compile ``lib/libisvd/{core,la,util,nogpu}`` with
     ``gcc -std=gnu99 -O2 -fopenmp`` against the single-rank ``mpi.h`` shim.
     ``core/param.c`` alone is built with ``-DNDEBUG`` so that tall matrices
     (m > n, rejected by the assert at ``core/param.c:43``) are accepted.  The
     rest keeps its asserts: under NDEBUG ``isvd_assert_pass(MPI_...)`` drops the
     MPI calls themselves (``util/mpi.c:22,34``).
  3. Link against the LP64 OpenBLAS 0.3.15 shipped in the image's
     ``opencv_python_headless.libs`` (exports ``dgemm_``, ``dgesvd_``, ``dsyev_``,
     ``dgelqf_``, ``dorglq_``, ``dgetri_``, ``dlarnv_``, ``lsame_`` ...).

When the reference tree is absent (the GPU box) the prebuilt library travels
with the repository snapshot and this script does nothing.
"""
import os
import shutil
import subprocess
import sys
import sysconfig
import tempfile
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
OUT_DIR = os.path.join(HERE, "_ref")
OUT_LIB = os.path.join(OUT_DIR, "liboracle_isvd.so")
REF = os.environ.get("ISVD_REFERENCE", "/root/reference")

VERSION = {"ISVD_MAJOR_VERSION": "1", "ISVD_MINOR_VERSION": "3", "ISVD_PATCH_VERSION": "2"}
TYPES = {
    "s": dict(x="s", X="S", xtype_____="isvd_s_val_t", XTYPE="ISVD_S_VAL_T", XName="Real Single",
              xname="real single", XStr="RealSingle"),
    "d": dict(x="d", X="D", xtype_____="isvd_d_val_t", XTYPE="ISVD_D_VAL_T", XName="Real Double",
              xname="real double", XStr="RealDouble"),
}


def openblas_dir():
    site = sysconfig.get_paths()["purelib"]
    d = os.path.join(site, "opencv_python_headless.libs")
    libs = [f for f in os.listdir(d) if f.startswith("libopenblas")] if os.path.isdir(d) else []
    if not libs:
        raise RuntimeError("OpenBLAS from opencv_python_headless.libs not found")
    return d, libs[0]


def _subst(text, table):
    for k, v in table.items():
        text = text.replace("@%s@" % k, v)
    return text


def configure(src_root, dst_root):
    for dirpath, _, files in os.walk(src_root):
        rel = os.path.relpath(dirpath, src_root)
        for f in files:
            if f == "CMakeLists.txt":
                continue
            with open(os.path.join(dirpath, f), encoding="utf-8") as fh:
                text = fh.read()
            if "@x@" in f:
                for x, table in TYPES.items():
                    t = dict(VERSION)
                    t.update(table)
                    out = os.path.join(dst_root, rel, f.replace("@x@", x))
                    os.makedirs(os.path.dirname(out), exist_ok=True)
                    with open(out, "w", encoding="utf-8") as fh:
                        fh.write(_subst(text, t))
            else:
                out = os.path.join(dst_root, rel, f)
                os.makedirs(os.path.dirname(out), exist_ok=True)
                with open(out, "w", encoding="utf-8") as fh:
                    fh.write(_subst(text, VERSION))


def build(force=False):
    if os.path.exists(OUT_LIB) and not force:
        return OUT_LIB
    if not os.path.isdir(os.path.join(REF, "src", "lib", "libisvd")):
        if os.path.exists(OUT_LIB):
            return OUT_LIB
        raise RuntimeError("reference tree not found at %s and no prebuilt %s" % (REF, OUT_LIB))
    bdir, blib = openblas_dir()
    tmp = tempfile.mkdtemp(prefix="isvd_ref_")
    try:
        configure(os.path.join(REF, "src", "include", "c"), os.path.join(tmp, "include"))
        configure(os.path.join(REF, "src", "lib"), os.path.join(tmp, "lib"))
        srcs = []
        for sub in ("core", "la", "util", "nogpu"):
            for dirpath, _, files in os.walk(os.path.join(tmp, "lib", "libisvd", sub)):
                srcs += [os.path.join(dirpath, f) for f in files if f.endswith(".c")]
        flags = ["gcc", "-std=gnu99", "-O2", "-fopenmp", "-fPIC", "-w",
                 "-I" + os.path.join(tmp, "include"), "-I" + os.path.join(tmp, "lib"),
                 "-I" + os.path.join(REPO, "include", "mpi_shim")]

        def cc(src):
            obj = src[:-2] + ".o"
            extra = ["-DNDEBUG"] if src.endswith(os.path.join("core", "param.c")) else []
            subprocess.check_call(flags + extra + ["-c", src, "-o", obj])
            return obj

        with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
            objs = list(ex.map(cc, sorted(srcs)))
        os.makedirs(OUT_DIR, exist_ok=True)
        subprocess.check_call(
            ["gcc", "-shared", "-o", OUT_LIB] + objs +
            ["-L" + bdir, "-l:" + blib, "-Wl,--disable-new-dtags", "-Wl,-rpath," + bdir, "-lgomp", "-lm"])
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return OUT_LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
