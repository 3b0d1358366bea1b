"""ctypes binding of the iSVD C ABI (``include/isvd.h``).

The same binding loads any library that exports the iSVD C ABI: the B200 library
(``isvd_b200/libisvd_gpu_b200.so``) or another build of the same interface.  It
is the Python mirror of the reference's C entry points
(``src/include/c/isvd/core/@x@_driver.h:21``, ``core/@x@_stage.h:21-77``,
``gpu/@x@_stage.h:28-90``, ``core/param.h:100``): same names, same argument
meaning, same layouts (``yst``/``qt``/``ut``/``vt`` row-major, ``a`` per
``dista``/``ordera``).  Arrays are passed as raw pointers: NumPy arrays give host
pointers, and anything with ``data_ptr()`` (a CUDA tensor) gives a device pointer.
"""
import ctypes
import os

import numpy as np

c_int_t = ctypes.c_int32          # isvd_int_t (LP64 build, include/isvd/def.h)
c_mpi_int = ctypes.c_int          # mpi_int_t
MPI_COMM_WORLD = 0x44000000       # include/mpi_shim/mpi.h

_PARAM_INT_FIELDS = ["nrow", "ncol", "nrow_proc", "ncol_proc", "nrow_each", "ncol_each", "nrow_total",
                     "ncol_total", "rowidxbegin", "rowidxend", "colidxbegin", "colidxend", "rank", "over_rank",
                     "dim_sketch", "dim_sketch_total", "num_sketch"]


_PARAM_CLASSES = {}


def param_class(cint):
    """isvd_Param (include/isvd/core/param.h; reference core/param.h:27-92) for the index type
    `cint` (ctypes.c_int32: the LP64 build; ctypes.c_int64: the ILP64 build)."""
    if cint not in _PARAM_CLASSES:
        _PARAM_CLASSES[cint] = type("Param" if cint is ctypes.c_int32 else "Param64", (ctypes.Structure,), {
            "_fields_": [("mpi_comm", ctypes.c_int), ("mpi_size", c_mpi_int), ("mpi_root", c_mpi_int),
                         ("mpi_rank", c_mpi_int)] + [(f, cint) for f in _PARAM_INT_FIELDS]})
    return _PARAM_CLASSES[cint]


Param = param_class(c_int_t)


_VP = ctypes.c_void_p
_CH = ctypes.c_char


def ptr(x):
    """Raw address of a NumPy array / CUDA tensor / int / None.  A CUDA tensor's producing work on
    torch's current stream is completed first: the library reads device operands in the order of
    its own stream, which need not be torch's (isvd_gpu_set_stream)."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        if getattr(x, "is_cuda", False):
            import torch
            torch.cuda.current_stream(x.device).synchronize()
        return x.data_ptr()
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    raise TypeError("cannot take the address of %r" % type(x))


def _dt(x):
    return np.float32 if x == "s" else np.float64


# isvd_gpu_allreduce_fn (include/isvd/b200.h): (buf, count, dtype, stream, user)
ALLREDUCE_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_void_p,
                                ctypes.c_void_p)


def host_array(buf, count, dtype):
    """NumPy view of the `count` values at host address `buf` (dtype 0: FP32, 1: FP64)."""
    ct = ctypes.c_float if dtype == 0 else ctypes.c_double
    return np.ctypeslib.as_array((ct * count).from_address(buf))


def torch_host_allreduce(group=None):
    """A host-memory sum-AllReduce over torch.distributed (e.g. the gloo backend) for
    IsvdLib.set_allreduce(..., on_device=False)."""
    import torch
    import torch.distributed as dist

    def fn(buf, count, dtype, stream, user):
        dist.all_reduce(torch.from_numpy(host_array(buf, count, dtype)), group=group)
    return fn


class _DeviceBuffer:
    """`count` values at a device address, exposed through __cuda_array_interface__."""

    def __init__(self, buf, count, dtype):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<f4" if dtype == 0 else "<f8",
                                         "data": (buf, False), "version": 2, "strides": None}


def torch_device_allreduce(group=None):
    """A device-memory sum-AllReduce over torch.distributed (NCCL, or gloo with CUDA tensors) for
    IsvdLib.set_allreduce(..., on_device=True): the reduction is ordered on the library's stream."""
    import torch
    import torch.distributed as dist

    def fn(buf, count, dtype, stream, user):
        with torch.cuda.stream(torch.cuda.ExternalStream(stream or 0)):
            t = torch.as_tensor(_DeviceBuffer(buf, count, dtype), device="cuda")
            dist.all_reduce(t, group=group)
    return fn


class IsvdLib:
    """Thin wrapper over one shared library exporting the iSVD C ABI."""

    def __init__(self, path, mode=ctypes.RTLD_LOCAL, ilp64=None):
        """ilp64: the library's isvd_int_t is int64 (default: a file name ending in _64.so, the
        reference's suffix for that build)."""
        self.path = os.path.abspath(path)
        if ilp64 is None:
            ilp64 = self.path.endswith("_64.so")
        self.ilp64 = bool(ilp64)
        self.c_int_t = ctypes.c_int64 if self.ilp64 else ctypes.c_int32
        self.Param = param_class(self.c_int_t)
        self.STAGE_HEAD = [self.Param, _VP, self.c_int_t, _VP, self.c_int_t]  # param, argv, argc, retv, retc
        self.lib = ctypes.CDLL(self.path, mode=mode)
        L = self.lib
        L.isvd_createParam.restype = self.Param
        L.isvd_createParam.argtypes = [self.c_int_t] * 5 + [c_mpi_int, ctypes.c_int]
        H = self.STAGE_HEAD
        for x in "sd":
            self._decl("isvd_%sSketchGaussianProjection" % x,
                       H + [_CH, _CH, _VP, self.c_int_t, _VP, self.c_int_t, self.c_int_t, c_mpi_int])
            self._decl("isvd_%sSketchGaussianProjection_gpu" % x,
                       H + [_CH, _CH, _VP, self.c_int_t, _VP, self.c_int_t, self.c_int_t, c_mpi_int])
            for name in ("OrthogonalizeTallSkinnyQr", "OrthogonalizeGramian"):
                self._decl("isvd_%s%s" % (x, name), H + [_VP, self.c_int_t])
            for name in ("IntegrateKolmogorovNagumo", "IntegrateWenYin", "IntegrateHierarchicalReduction"):
                self._decl("isvd_%s%s" % (x, name), H + [_VP, self.c_int_t, _VP, self.c_int_t])
            post = H + [_CH, _CH, _VP, self.c_int_t, _VP, self.c_int_t, _VP, _VP, self.c_int_t, _VP, self.c_int_t, c_mpi_int, c_mpi_int]
            for name in ("PostprocessTallSkinnyQr", "PostprocessGramian", "PostprocessSymmetric"):
                self._decl("isvd_%s%s" % (x, name), post)
                self._decl("isvd_%s%s_gpu" % (x, name), post)
            self._decl("isvd_%sIsvd" % x,
                       [self.Param, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                        _VP, _VP, _VP, _VP, _VP, _VP, _CH, _CH, _VP, self.c_int_t, _VP, _VP, self.c_int_t, _VP, self.c_int_t,
                        self.c_int_t, c_mpi_int, c_mpi_int])

        # B200 extensions (include/isvd/b200.h)
        self._decl("isvd_gpu_get_last_error", [], ctypes.c_int)
        self._decl("isvd_gpu_get_error_string", [], ctypes.c_char_p)
        self._decl("isvd_gpu_clear_error", [])
        self._decl("isvd_gpu_set_precision", [ctypes.c_int])
        self._decl("isvd_gpu_get_precision", [], ctypes.c_int)
        self._decl("isvd_gpu_kernel_launch_count", [], ctypes.c_ulonglong)
        self._decl("isvd_gpu_profile_enable", [ctypes.c_int])
        self._decl("isvd_gpu_set_stream", [_VP])
        self._decl("isvd_gpu_get_stream", [], _VP)
        self._decl("isvd_gpu_profile_reset", [])
        self._decl("isvd_gpu_set_allreduce", [ALLREDUCE_FN, _VP, ctypes.c_int, ctypes.c_int, ctypes.c_int])
        self._allreduce_cb = None
        self._decl("isvd_gpu_profile_get", [ctypes.c_char_p, ctypes.POINTER(ctypes.c_double),
                                            ctypes.POINTER(ctypes.c_ulonglong), ctypes.POINTER(ctypes.c_double)],
                   ctypes.c_int)
        for x in "sd":
            self._decl("isvd_%sSketchGaussianProjectionOmega" % x,
                       H + [_CH, _CH, _VP, self.c_int_t, _VP, self.c_int_t, _VP, self.c_int_t])
            self._decl("isvd_%sIsvd_ex" % x,
                       [self.Param, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                        _VP, _VP, _VP, _VP, _VP, _VP, _CH, _CH, _VP, self.c_int_t, _VP, _VP, self.c_int_t, _VP, self.c_int_t,
                        self.c_int_t, c_mpi_int, c_mpi_int, _VP, self.c_int_t, ctypes.c_int], ctypes.c_int)
            it = self.c_int_t
            self._decl("isvd_%sMtxRead" % x, [ctypes.c_char_p, ctypes.POINTER(it), ctypes.POINTER(it), _VP, it, _CH],
                       ctypes.c_int)
            self._decl("isvd_%sMtxWrite" % x, [ctypes.c_char_p, it, it, _VP, it, _CH], ctypes.c_int)

    def _decl(self, name, argtypes, restype=None):
        fn = getattr(self.lib, name, None)
        if fn is None:
            return
        fn.argtypes = argtypes
        fn.restype = restype

    def has(self, name):
        return hasattr(self.lib, name)

    def set_allreduce(self, fn, nranks, rank, on_device=False):
        """Join `nranks` processes as row blocks (isvd_gpu_set_allreduce): fn(buf, count, dtype,
        stream, user) sums in place over the ranks.  fn = None returns to one process."""
        self._allreduce_cb = ALLREDUCE_FN(fn) if fn is not None else ALLREDUCE_FN()
        self.lib.isvd_gpu_set_allreduce(self._allreduce_cb, None, nranks if fn is not None else 1, rank if fn else 0,
                                        1 if on_device else 0)

    # ------------------------------------------------------------------ parameters
    def create_param(self, m, n, k, p, N, root=0, comm=MPI_COMM_WORLD):
        return self.lib.isvd_createParam(m, n, k, p, N, root, comm)

    @staticmethod
    def _args(x, argv, retc):
        av = None if argv is None else np.ascontiguousarray(argv, dtype=_dt(x))
        rv = np.zeros(max(retc, 1), dtype=_dt(x))
        return av, (0 if av is None else len(av)), rv

    # ------------------------------------------------------------------ stages
    def sketch(self, x, param, a, lda, yst, ldyst, seed, dista=b"R", ordera=b"R", gpu=False, root=0):
        fn = getattr(self.lib, "isvd_%sSketchGaussianProjection%s" % (x, "_gpu" if gpu else ""))
        fn(param, None, 0, None, 0, dista, ordera, ptr(a), lda, ptr(yst), ldyst, seed, root)

    def orthogonalize(self, x, alg, param, yst, ldyst):
        name = {"GR": "OrthogonalizeGramian", "TS": "OrthogonalizeTallSkinnyQr"}[alg]
        getattr(self.lib, "isvd_%s%s" % (x, name))(param, None, 0, None, 0, ptr(yst), ldyst)

    def integrate(self, x, alg, param, yst, ldyst, qt, ldqt, argv=None, retc=2):
        name = {"KN": "IntegrateKolmogorovNagumo", "WY": "IntegrateWenYin",
                "HR": "IntegrateHierarchicalReduction"}[alg]
        av, ac, rv = self._args(x, argv, retc)
        getattr(self.lib, "isvd_%s%s" % (x, name))(param, ptr(av), ac, ptr(rv), retc, ptr(yst), ldyst, ptr(qt), ldqt)
        return rv[:retc]

    def query(self, x, alg, retc):
        """Default-argument query protocol (argc < 0)."""
        name = {"KN": "IntegrateKolmogorovNagumo", "WY": "IntegrateWenYin",
                "HR": "IntegrateHierarchicalReduction"}[alg]
        rv = np.zeros(max(retc, 1), dtype=_dt(x))
        p = self.create_param(4, 4, 1, 0, 1)
        getattr(self.lib, "isvd_%s%s" % (x, name))(p, None, -1, ptr(rv), retc, None, 1, None, 1)
        return rv[:retc]

    def postprocess(self, x, alg, param, a, lda, qt, ldqt, s, ut, ldut, vt, ldvt, dista=b"R", ordera=b"R",
                    ut_root=-1, vt_root=-1, gpu=False):
        name = {"GR": "PostprocessGramian", "TS": "PostprocessTallSkinnyQr", "SY": "PostprocessSymmetric"}[alg]
        fn = getattr(self.lib, "isvd_%s%s%s" % (x, name, "_gpu" if gpu else ""))
        fn(param, None, 0, None, 0, dista, ordera, ptr(a), lda, ptr(qt), ldqt, ptr(s), ptr(ut), ldut, ptr(vt),
           ldvt, ut_root, vt_root)

    # ------------------------------------------------------------------ Matrix Market files
    def mtx_read(self, path, x="d", ordera=b"C", pad=0):
        """isvd_?MtxRead: (status, m x n array or None).  ordera / pad choose the layout and the
        leading dimension the library writes (m + pad for 'C', n + pad for 'R')."""
        f = getattr(self.lib, "isvd_%sMtxRead" % x)
        m, n = self.c_int_t(0), self.c_int_t(0)
        p = os.fsencode(str(path))
        st = f(p, ctypes.byref(m), ctypes.byref(n), None, 1, ordera)
        if st:
            return st, None
        dt = _dt(x)
        if ordera == b"C":
            buf = np.zeros((n.value, m.value + pad), dt)  # column j at buf[j, :m]
            st = f(p, ctypes.byref(m), ctypes.byref(n), buf.ctypes.data, m.value + pad, ordera)
            return st, None if st else buf[:, :m.value].T.copy()
        buf = np.zeros((m.value, n.value + pad), dt)
        st = f(p, ctypes.byref(m), ctypes.byref(n), buf.ctypes.data, n.value + pad, ordera)
        return st, None if st else buf[:, :n.value].copy()

    def mtx_write(self, path, a, x="d"):
        """isvd_?MtxWrite of a 2-D array ("matrix array real general"); returns the status."""
        a = np.ascontiguousarray(a, _dt(x))
        return getattr(self.lib, "isvd_%sMtxWrite" % x)(os.fsencode(str(path)), a.shape[0], a.shape[1],
                                                        a.ctypes.data, a.shape[1], b"R")

    # ------------------------------------------------------------------ extensions
    def last_error(self):
        return self.lib.isvd_gpu_get_last_error(), (self.lib.isvd_gpu_get_error_string() or b"").decode()

    def clear_error(self):
        self.lib.isvd_gpu_clear_error()

    def profile(self, tag):
        """(total ms, launches, executed flops) recorded under `tag`, or None."""
        ms, n, fl = ctypes.c_double(), ctypes.c_ulonglong(), ctypes.c_double()
        if self.lib.isvd_gpu_profile_get(tag.encode(), ctypes.byref(ms), ctypes.byref(n), ctypes.byref(fl)) != 0:
            return None
        return ms.value, n.value, fl.value

    def sketch_omega(self, x, param, a, lda, omega, ldomega, yst, ldyst, dista=b"R", ordera=b"R"):
        fn = getattr(self.lib, "isvd_%sSketchGaussianProjectionOmega" % x)
        fn(param, None, 0, None, 0, dista, ordera, ptr(a), lda, ptr(omega), ldomega, ptr(yst), ldyst)

    def isvd(self, x, param, algs, a, lda, s, ut, ldut, vt, ldvt, seed=0, dista=b"R", ordera=b"R",
             argv=None, retc=(0, 0, 2, 0), ut_root=-1, vt_root=-1, omega=None, ldomega=0, precision=None):
        """isvd_?Isvd driver (isvd_?Isvd_ex when omega / precision is given).

        Returns (retv list, time[4], status)."""
        dt = _dt(x)
        keep = []
        argv_arr = (ctypes.c_void_p * 4)()
        argc_arr = (self.c_int_t * 4)()
        for i in range(4):
            av = None if argv is None or argv[i] is None else np.ascontiguousarray(argv[i], dtype=dt)
            keep.append(av)
            argv_arr[i] = ptr(av)
            argc_arr[i] = 0 if av is None else len(av)
        retv_arr = (ctypes.c_void_p * 4)()
        retc_arr = (self.c_int_t * 4)()
        rvs = []
        for i in range(4):
            rv = np.zeros(max(retc[i], 1), dtype=dt)
            rvs.append(rv)
            retv_arr[i] = ptr(rv)
            retc_arr[i] = retc[i]
        times = (ctypes.c_double * 4)()
        common = (param, algs[0].encode(), algs[1].encode(), algs[2].encode(), algs[3].encode(),
                  ctypes.cast(argv_arr, _VP) if argv is not None else None, ctypes.cast(argc_arr, _VP),
                  ctypes.cast(retv_arr, _VP), ctypes.cast(retc_arr, _VP), ctypes.cast(times, _VP), None,
                  dista, ordera, ptr(a), lda, ptr(s), ptr(ut), ldut, ptr(vt), ldvt, seed, ut_root, vt_root)
        status = 0
        if omega is None and precision is None:
            getattr(self.lib, "isvd_%sIsvd" % x)(*common)
        else:
            prec = -1 if precision is None else int(precision)
            status = getattr(self.lib, "isvd_%sIsvd_ex" % x)(*common, ptr(omega), ldomega, prec)
        return [rv[:retc[i]] for i, rv in enumerate(rvs)], list(times), status
