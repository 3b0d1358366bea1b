"""bench.py's reference arm without a GPU: the reference's own CPU pipeline (built from source as
the checker) on a small row sample prints one JSON line with the contract's keys; a rank other than
0 prints nothing and exits 0."""
import json
import os
import subprocess
import sys

from conftest import REPO


def run_bench(extra_env):
    env = dict(os.environ, ISVD_BENCH_REF_ROWS="512", **extra_env)
    return subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--steps", "1",
                           "--warmup", "0", "--size", "small"], capture_output=True, text=True, timeout=600,
                          env=env, cwd=REPO)


def test_reference_arm_json_line():
    out = run_bench({})
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["steps"] == 1 and d["warmup"] == 0 and d["n_gpus"] == 1
    assert "workload" in d["config"]
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    # ms_per_step is the timed sample step: the steps fit in the run's own wall clock
    assert d["ms_per_step"] * d["steps"] <= 1e3 * d["wall_s"]
    assert abs(d["ms_per_solve_extrapolated"] * d["value"] - 1e3) < 1e-9


def test_reference_arm_other_ranks_exit_quietly():
    out = run_bench({"RANK": "1", "WORLD_SIZE": "2"})
    assert out.returncode == 0, out.stderr[-2000:]
    assert not [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
