"""Row blocks over two processes on one GPU, joined by a caller-supplied AllReduce
(isvd_gpu_set_allreduce with a gloo host reduction): each process holds the rows
[rowidxbegin, rowidxend) that isvd_createParam gives it, and the solve -- every orthogonalization,
integration and postprocessing selector -- matches the one-process
solve of the whole matrix with the same Omega -- singular values within 1e-10 (FP64) / 1e-5
(MIXED), the same iteration counts, U and V column angles within 1e-8 (FP64) / 1e-4 (MIXED), for
the gathered outputs (ut_root = vt_root = 0) and for each rank's own blocks (roots -1).  The
AllReduce runs on host buffers, or on device buffers ordered on the library's stream (gloo with
CUDA tensors, the same interface an NCCL group uses).  The ranks' kernels never wait on each
other: gloo moves the data through the host between launches."""
import datetime
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def lowrank(m, n, rank, decay, noise, seed):
    rng = np.random.default_rng(seed)
    u = np.linalg.qr(rng.standard_normal((m, rank)))[0]
    v = np.linalg.qr(rng.standard_normal((n, rank)))[0]
    return (u * decay ** np.arange(rank)) @ v.T + noise * rng.standard_normal((m, n))


def solve(L, x, prm, a, om, k, p, N, algs, precision, ut_root, vt_root, dista="R"):
    """The driver on this process's rows (dista 'R') or columns ('C'); returns s, ut, vt, retv."""
    l = k + p
    dt = np.float32 if x == "s" else np.float64
    mloc = prm.nrow_proc if ut_root < 0 or ut_root != prm.mpi_rank else prm.nrow
    nloc = prm.ncol_proc if vt_root < 0 else (prm.ncol if vt_root == prm.mpi_rank else prm.ncol_proc)
    s = np.zeros(l, dt)
    ut = np.zeros((max(mloc, 1), l), dt)
    vt = np.zeros((max(nloc, 1), l), dt)
    n = a.shape[1]
    argv = [None, None, [256, 1e-4] if algs[2] == "KN" else None, None]
    retv, _, st = L.isvd(x, prm, algs, np.ascontiguousarray(a.astype(dt)), n, s, ut, l, vt, l, argv=argv,
                         retc=(0, 0, 2, 0), ut_root=ut_root, vt_root=vt_root, dista=dista.encode(),
                         omega=np.ascontiguousarray(om.astype(dt)), ldomega=l * N, precision=precision)
    assert st == 0, L.last_error()
    return s, ut, vt, [list(v) for v in retv]


def _worker(rank, port, args, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist
    from isvd_b200 import LIB_PATH
    from isvd_b200.capi import IsvdLib, torch_device_allreduce, torch_host_allreduce
    try:
        dist.init_process_group("gloo", rank=rank, world_size=2, timeout=datetime.timedelta(seconds=120))
        x, precision, algs, a, om, k, p, N, on_device, dista = args
        L = IsvdLib(LIB_PATH)
        fn = torch_device_allreduce() if on_device else torch_host_allreduce()
        L.set_allreduce(fn, 2, rank, on_device=on_device)
        prm = L.create_param(a.shape[0], a.shape[1], k, p, N)
        held = a[prm.rowidxbegin:prm.rowidxend] if dista == "R" else a[:, prm.colidxbegin:prm.colidxend]
        own = solve(L, x, prm, held, om, k, p, N, algs, precision, -1, -1, dista)
        gathered = solve(L, x, prm, held, om, k, p, N, algs, precision, 0, 0, dista)
        q.put((rank, (prm.rowidxbegin, prm.rowidxend, prm.colidxbegin, prm.colidxend), own, gathered))
        dist.destroy_process_group()
    except BaseException as e:  # report instead of hanging the parent
        q.put((rank, "error", repr(e), None))


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


@pytest.mark.parametrize("x,precision,algs,on_device,dista", [
    ("d", 0, ("GP", "GR", "KN", "GR"), False, "R"), ("s", 1, ("GP", "GR", "KN", "GR"), False, "R"),
    ("d", 0, ("GP", "TS", "WY", "GR"), False, "R"), ("s", 1, ("GP", "TS", "WY", "GR"), False, "R"),
    ("d", 0, ("GP", "GR", "KN", "GR"), True, "R"), ("s", 1, ("GP", "TS", "KN", "GR"), True, "R"),
    ("d", 0, ("GP", "GR", "HR", "GR"), False, "R"), ("s", 1, ("GP", "GR", "HR", "GR"), True, "R"),
    ("d", 0, ("GP", "GR", "KN", "TS"), False, "R"), ("s", 1, ("GP", "TS", "KN", "TS"), True, "R"),
    ("d", 0, ("GP", "GR", "KN", "SY"), False, "R"), ("s", 1, ("GP", "GR", "WY", "SY"), True, "R"),
    ("d", 0, ("GP", "GR", "KN", "GR"), False, "C"), ("s", 1, ("GP", "GR", "KN", "GR"), True, "C"),
    ("d", 0, ("GP", "TS", "HR", "TS"), False, "C"), ("d", 0, ("GP", "GR", "KN", "SY"), True, "C")])
def test_two_row_blocks_match_one_process(lib, oracle, x, precision, algs, on_device, dista):
    """Every selector the driver takes with row blocks: GR or TS orthogonalization, KN, WY or HR
    integration, GR, TS or SY postprocessing (SY: a symmetric A); and column blocks (dista 'C':
    each process holds all rows of its columns, Y summed over the processes)."""
    if algs[3] == "SY":
        m = n = 700
        a = lowrank(m, n, 300, 0.97, 1e-6, 11)
        a = 0.5 * (a + a.T)
    else:
        m, n = 1201, 700
        a = lowrank(m, n, 300, 0.97, 1e-6, 11)
    k, p, N = 16, 8, 8
    om = np.random.default_rng(12).standard_normal((n, (k + p) * N))
    prm1 = lib.create_param(m, n, k, p, N)
    s1, u1, v1, r1 = solve(lib, x, prm1, a, om, k, p, N, algs, precision, -1, -1)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    args = (x, precision, algs, a, om, k, p, N, on_device, dista)
    procs = [ctx.Process(target=_worker, args=(r, port, args, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    out = {}
    for _ in range(2):
        rank, blk, own, gathered = q.get(timeout=300)
        assert blk != "error", own
        out[rank] = (blk, own, gathered)
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    ts, ta = (1e-10, 1e-8) if x == "d" else (1e-5, 1e-4)
    it_tol = 0 if x == "d" else 1
    for rank in (0, 1):
        (rb, re, cb, ce), own, gathered = out[rank]
        for res in (own, gathered):
            assert np.abs(res[0].astype(np.float64) - s1).max() <= ts * np.abs(s1).max()
            assert abs(res[3][2][0] - r1[2][0]) <= it_tol
        uo = own[1][:, :k].astype(np.float64)
        vo = own[2][:, :k].astype(np.float64)
        assert oracle.column_angles(uo, u1[rb:re, :k].astype(np.float64)).max() < ta
        assert oracle.column_angles(vo, v1[cb:ce, :k].astype(np.float64)).max() < ta
    g = out[0][2]
    assert oracle.column_angles(g[1][:, :k].astype(np.float64), u1[:, :k].astype(np.float64)).max() < ta
    assert oracle.column_angles(g[2][:, :k].astype(np.float64), v1[:, :k].astype(np.float64)).max() < ta
