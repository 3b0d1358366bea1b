"""Row blocks over several ranks, host side (no GPU): isvd_createParam splits rows and columns
like the reference's core/param.c:47-55 once isvd_gpu_set_allreduce joins P ranks, and the
reference's row-block exchange algebra -- the oracle's row-block driver with each of the
reference's MPI_Allreduce calls run through the library's capi.torch_host_allreduce callback over
gloo with world_size 2 -- reproduces the one-rank solve, for KN and WY integration."""
import ctypes
import datetime
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from conftest import REPO


@pytest.mark.parametrize("P", [2, 3, 4])
@pytest.mark.parametrize("m,n", [(1001, 3000), (8, 8), (7, 40)])
def test_create_param_blocks(lib, oracle, P, m, n):
    noop = lambda buf, count, dtype, stream, user: None  # noqa: E731
    try:
        for r in range(P):
            lib.set_allreduce(noop, P, r)
            prm = lib.create_param(m, n, 3, 2, 4)
            assert (prm.mpi_size, prm.mpi_rank) == (P, r)
            rb, re = oracle.row_block(m, P, r)
            cb, ce = oracle.row_block(n, P, r)
            assert (prm.rowidxbegin, prm.rowidxend, prm.nrow_proc) == (rb, re, re - rb)
            assert (prm.colidxbegin, prm.colidxend, prm.ncol_proc) == (cb, ce, ce - cb)
            assert prm.nrow_each == (m - 1) // P + 1 and prm.nrow_total == prm.nrow_each * P
            assert prm.ncol_each == (n - 1) // P + 1 and prm.ncol_total == prm.ncol_each * P
    finally:
        lib.set_allreduce(None, 1, 0)
    prm = lib.create_param(m, n, 3, 2, 4)
    assert (prm.mpi_size, prm.mpi_rank, prm.nrow_proc) == (1, 0, m)


def test_set_allreduce_rejects_bad_ranks(lib):
    noop = lambda buf, count, dtype, stream, user: None  # noqa: E731
    lib.clear_error()
    lib.set_allreduce(noop, 2, 2)
    assert lib.last_error()[0] == 1
    lib.clear_error()
    lib.set_allreduce(None, 1, 0)
    assert lib.create_param(10, 10, 2, 1, 2).mpi_size == 1


def _rank(rank, port, a, om, k, p, N, alg, alg_p, dista, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import sys
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import torch.distributed as dist
    import isvd_oracle as orc
    from isvd_b200.capi import torch_host_allreduce
    try:
        dist.init_process_group("gloo", rank=rank, world_size=2, timeout=datetime.timedelta(seconds=60))
        fn = torch_host_allreduce()
        count = [0]

        def allreduce(x):  # the library's callback, on a float64 host buffer
            x = np.ascontiguousarray(x, np.float64)
            fn(x.ctypes.data, x.size, 1, None, None)
            count[0] += 1
            return x

        f32 = np.arange(5, dtype=np.float32) * (rank + 1)
        fn(f32.ctypes.data, 5, 0, None, None)
        rb, re = orc.row_block(a.shape[0], 2, rank)
        if dista == "R":
            s, u, v, it, err = orc.isvd_row_block(a[rb:re], om, k, p, N, allreduce, alg_i=alg, alg_p=alg_p,
                                                  row_begin=rb)
        else:
            cb, ce = orc.row_block(a.shape[1], 2, rank)
            s, u, v, it, err = orc.isvd_col_block(a[:, cb:ce], om, k, p, N, allreduce, slice(rb, re), slice(cb, ce),
                                                  alg_i=alg, alg_p=alg_p)
        q.put((rank, (rb, re), s, u, v, it, count[0], f32))
        dist.destroy_process_group()
    except BaseException as e:
        q.put((rank, "error", repr(e), None, None, None, None, None))


@pytest.mark.parametrize("alg,alg_p,dista", [("KN", "GR", "R"), ("WY", "GR", "R"), ("HR", "GR", "R"),
                                             ("KN", "TS", "R"), ("KN", "SY", "R"), ("KN", "GR", "C"),
                                             ("HR", "TS", "C"), ("WY", "SY", "C")])
def test_exchange_algebra_over_gloo(oracle, alg, alg_p, dista):
    m, n, k, p, N = 301, 120, 6, 4, 5
    rng = np.random.default_rng(3)
    a = (np.linalg.qr(rng.standard_normal((m, 40)))[0] * 0.9 ** np.arange(40)) @ rng.standard_normal((40, n))
    if alg_p == "SY":  # a symmetric A
        a = a[:n] + a[:n].T
        m = n
    om = rng.standard_normal((n, (k + p) * N))
    whole = oracle.isvd(a, om, k, p, N, alg_i=alg, alg_p=alg_p)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    procs = [ctx.Process(target=_rank, args=(r, port, a, om, k, p, N, alg, alg_p, dista, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    res = {}
    for _ in range(2):
        r = q.get(timeout=240)
        assert r[1] != "error", r[2]
        res[r[0]] = r
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    u = np.vstack([res[0][3], res[1][3]])
    for r in (0, 1):
        _, (rb, re), sr, ur, vr, it, calls, f32 = res[r]
        assert np.array_equal(f32, np.arange(5, dtype=np.float32) * 3)
        # column blocks: Y; the block Grams; KN: Bc, one Bgc per iteration; WY: also the first
        # Bgc and the two step-size sums of every iteration but the last; HR: one sum per level;
        # then Z (column blocks: Qbar and Z) and for SY the l x l W
        levels, h2 = 0, N
        while h2 > 1:
            levels, h2 = levels + 1, (h2 + 1) // 2
        integ = {"KN": 1 + it, "WY": 2 + it + (it - 1), "HR": levels}[alg]
        col = dista == "C"
        expected = col + N + integ + (2 if col else 1) + (alg_p == "SY")
        assert it == whole["iters"] and calls == expected
        # column blocks add Y's partial products in another order (last-bit differences); WY stops
        # at tol 1e-3, short of convergence, where such differences grow to about 1e-8
        ts, ta = (1e-7, 1e-6) if (col and alg == "WY") else (1e-12, 1e-10)
        assert np.abs(sr - whole["s"]).max() <= ts * np.abs(whole["s"]).max()
        if alg_p != "SY":
            assert oracle.column_angles(vr, whole["v"]).max() < ta
    assert oracle.column_angles(u, whole["u"]).max() < ta


def test_noalloc_kn_refuses_joined_ranks(lib):
    """The static-scratch Kolmogorov-Nagumo entry point runs on one rank only: it never sums the
    Gram over ranks, so with ranks joined through isvd_gpu_set_allreduce (or an isvd_Param whose MPI
    size is not 1) it returns ISVD_GPU_ERROR_UNSUPPORTED before touching any operand or device."""
    from isvd_b200.capi import Param, c_int_t
    fn = lib.lib.isvd_dIntegrateKolmogorovNagumo_noalloc
    fn.argtypes = [Param, ctypes.c_void_p, c_int_t, ctypes.c_void_p, c_int_t, ctypes.c_void_p, c_int_t,
                   ctypes.c_void_p, c_int_t, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    unsupported = 6  # ISVD_GPU_ERROR_UNSUPPORTED
    noop = lambda buf, count, dtype, stream, user: None  # noqa: E731
    try:
        lib.set_allreduce(noop, 2, 1)
        prm = lib.create_param(1000, 1000, 8, 4, 4)
        assert prm.mpi_size == 2
        lib.clear_error()
        assert fn(prm, None, 0, None, 0, None, 48, None, 12, None) == unsupported
        code, msg = lib.last_error()
        assert code == unsupported and "one rank only" in msg
    finally:
        lib.set_allreduce(None, 1, 0)
    prm = lib.create_param(1000, 1000, 8, 4, 4)
    prm.mpi_size = 2
    lib.clear_error()
    assert fn(prm, None, 0, None, 0, None, 48, None, 12, None) == unsupported
    assert lib.last_error()[0] == unsupported
