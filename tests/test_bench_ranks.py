"""bench.py's rank handling on the host (no GPU): under torchrun only rank 0
runs the reference arm and prints its line; the other ranks exit 0 at once
without work, and the other workloads refuse N > 1 with one `unavailable`
line from rank 0."""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def run_bench(args, rank, world):
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], env=env, capture_output=True, text=True,
                          timeout=120)


def test_reference_arm_other_ranks_exit_without_work():
    r = run_bench(["--impl", "reference", "--gpus", "2", "--steps", "3", "--warmup", "3"], rank=1, world=2)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_other_workloads_refuse_several_ranks():
    for rank in (0, 1):
        r = run_bench(["--workload", "serve", "--gpus", "2"], rank=rank, world=2)
        assert r.returncode == 0, r.stderr
        lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
        if rank == 0:
            assert len(lines) == 1 and "unavailable" in json.loads(lines[0])
        else:
            assert lines == []
