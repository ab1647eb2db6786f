"""bench.py --gpus N starts N ranks itself when no torchrun environment is
present (it re-runs under torch.distributed.run).  The --dry-run mode brings
the ranks up over gloo on the CPU and has rank 0 report which ranks ran."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(*extra):
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR",
                                                             "MASTER_PORT")}
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *extra], capture_output=True, text=True,
                       timeout=240, env=env, cwd=ROOT)
    return p


def test_two_ranks_start_and_report():
    p = _run("--gpus", "2", "--dry-run")
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, p.stdout                  # rank 0 alone prints
    line = json.loads(lines[0])
    assert line["n_gpus"] == 2 and sorted(line["ranks"]) == [0, 1] and line["requested"] == 2


def test_one_rank_runs_in_process():
    p = _run("--gpus", "1", "--dry-run")
    assert p.returncode == 0, p.stderr[-2000:]
    line = json.loads([l for l in p.stdout.splitlines() if l.startswith("{")][0])
    assert line["n_gpus"] == 1 and line["ranks"] == [0]


def test_rank_count_mismatch_fails_loudly():
    env = dict(os.environ, WORLD_SIZE="3", RANK="0", LOCAL_RANK="0")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--dry-run"],
                       capture_output=True, text=True, timeout=120, env=env, cwd=ROOT)
    assert p.returncode != 0 and "3 ranks were started" in p.stderr
