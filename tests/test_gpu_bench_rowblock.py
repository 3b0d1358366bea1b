"""bench.py's multi-GPU mode on one GPU: two ranks (torch.distributed.run) share cuda:0 with the
gloo backend and run the 20000 x 4000 workload split by rows through the library's AllReduce hook
(device buffers staged through the host by gloo, so neither rank's kernels wait on the other's).
A functional check of the row-block bench path that NCCL runs on several GPUs: one JSON line from
rank 0 with the contract's keys, two GPUs' worth of ranks, the row-block parallelism and a
converged Kolmogorov-Nagumo iteration."""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import REPO

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_bench_rowblock_two_ranks_one_gpu():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), os.path.join(REPO, "bench.py"),
           "--gpus", "2", "--size", "small", "--dist-backend", "gloo", "--steps", "2", "--warmup", "3",
           "--skip-fp64", "--skip-cpu", "--skip-extra"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=900, cwd=REPO)
    assert r.returncode == 0, r.stderr[-4000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "scaling", "config", "e2e",
                "roofline", "clocks", "gpu_launches"):
        assert key in d, key
    assert d["n_gpus"] == 2 and d["scaling"] == "strong" and d["value"] > 0
    assert d["config"]["parallelism"].startswith("row blocks over 2 GPUs")
    assert 1 < d["kn_iterations"] <= 256
    assert d["e2e"]["h2d_bytes_per_step"] == 20000 * 4000 * 4
