"""bench.py's reference arm (the CPU restatement of the reference's scalar
path, timed on the host cores) keeps the one-JSON-line contract, alone and
under torchrun, where rank 0 alone runs and prints and the other ranks exit 0
without work.  Small batches keep this a few seconds of CPU."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _json_lines(out: str) -> list[dict]:
    return [json.loads(line) for line in out.splitlines() if line.startswith("{")]


def _check_line(line: dict, n_gpus: int, rods: int) -> None:
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference"
    assert line["n_gpus"] == n_gpus
    assert line["warmup"] >= 3
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"]
    assert line["config"]["workload"] == "uneven_batch"
    assert line["config"]["rods"] == rods


def test_reference_arm_one_process():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--rods", "128", "--steps", "2",
                        "--warmup", "3"], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _json_lines(r.stdout)
    assert len(lines) == 1
    _check_line(lines[0], 1, 128)
    assert lines[0]["config"]["parallelism"] == "single GPU"


def test_reference_arm_two_ranks_rank0_shard():
    """Under torchrun the reference arm steps rank 0's shard of the global
    batch: the same rods the GPU arm's rank 0 steps (2 x 128 rods, split by
    the element-balanced partition)."""
    env = dict(os.environ, MASTER_ADDR="127.0.0.1")
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
                        "--master-addr", "127.0.0.1", "--master-port", "29541", "bench.py", "--impl", "reference",
                        "--gpus", "2", "--rods", "128", "--steps", "1", "--warmup", "3"],
                       cwd=ROOT, capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _json_lines(r.stdout)
    assert len(lines) == 1
    line = lines[0]
    # the shard holds about half of 256 rods, balanced by elements
    _check_line(line, 2, line["config"]["rods"])
    assert 64 <= line["config"]["rods"] <= 192
    assert line["cpu_baseline"]["sample"].startswith("rank 0 shard")
