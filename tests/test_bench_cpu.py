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


def test_gpus_flag_without_launcher_runs_that_many_ranks():
    """--gpus N without torchrun relaunches itself as N ranks on this node
    (the line reports n_gpus == N)."""
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--gpus", "2", "--rods", "128",
                        "--steps", "1", "--warmup", "3"], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _json_lines(r.stdout)
    assert len(lines) == 1
    _check_line(lines[0], 2, lines[0]["config"]["rods"])


def test_gpus_flag_disagreeing_with_launcher_is_refused():
    env = dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--gpus", "2", "--rods", "16",
                        "--steps", "1", "--warmup", "3"], cwd=ROOT, capture_output=True, text=True, timeout=300,
                       env=env)
    assert r.returncode != 0
    assert "WORLD_SIZE" in r.stderr


def test_censored_percentiles_are_lower_bounds():
    sys.path.insert(0, ROOT)
    import bench

    done = [1.0, 2.0, 3.0]
    # no censoring: ordinary percentiles
    assert bench.censored_percentiles(done, [])["p50"] == 2.0
    # two requests still running at ages 10 and 20: they enter with their ages
    p = bench.censored_percentiles(done, [10.0, 20.0])
    assert p["p50"] == 3.0 and p["p99"] > 10.0
    assert bench.censored_percentiles([], [])["p99"] is None


def test_compact_line_fits_the_tail():
    """The printed line with every side section in short form stays short."""
    sys.path.insert(0, ROOT)
    import bench

    serving = {k: {"rate_req_s": 200.0, "arrival_window_s": 60.0, "submitted": 12000, "completed": 700,
                   "censored": 11300, "p50_latency_s": 31.123456789, "p99_latency_s": 59.123456789,
                   "latency_percentiles": "censored_lower_bound", "p99_queueing_s": 58.1234567, "value": 1.7e10,
                   "gpu_busy_frac": 0.91234567, "fallbacks": 1, "ticks": 5}
               for k in ("stated_load", "sustained_load")}
    mixed = {"rods": 65536, "elements": 10473311, "steps": 10000, "dt": 4.6e-7, "value": 2.7e10,
             "fp64_default_value": 1.3e10, "fp64_streaming_value": 9.6e9, "fp64_default_plan": "resident",
             "speedup_vs_fp64_default": 2.0123456, "speedup_vs_fp64_streaming": 2.88123456,
             "tip_error_max": 1.1e-7, "tip_error_p99": 4.7e-8, "energy_rel_diff": 2.3e-8, "finite": True,
             "energy_fp64": [1.0, 2.0]}
    batched = {"value": 1.5e10, "plan": {"mode": "resident", "probe_ms": [0.0] * 20}, "ms_per_step": 0.29,
               "pefrl": {"default_plan": {"value": 4e9}, "streaming": {"value": 2.4e9}}}
    contact = {"value": 6.3e8, "ms_per_step": 0.83, "candidate_pairs": 1211410, "launches_per_step": 13,
               "cpu_baseline": {"value": 1.1e6}}
    cant = {"value": 3.6e7, "tip_trajectory": {"max_rel_error": 3e-14}, "cpu_baseline": {"value": 5.6e6}}
    sec = bench.compact_sections(batched, contact, {"stated_load": serving["stated_load"],
                                                    "sustained_load": serving["sustained_load"]}, cant, mixed)
    assert list(sec)[-1] == "mixed"
    assert len(json.dumps(sec, separators=(",", ":"))) < 1500


def test_profile_traffic_only_for_the_profiled_launch():
    """The committed ncu traffic figure of the step kernel is reported for a
    launch over the element count its summary covers, with the sources it
    was captured from, and for nothing else."""
    sys.path.insert(0, ROOT)
    import bench

    srcs = ("rod_step_fp64.cu", "rod_math.cuh", "bulk_copy.cuh")
    path = os.path.join(ROOT, "profiles", "rod_step_fp64_uneven_batch.txt")
    covered = None
    with open(path, encoding="utf-8") as f:
        for line in f:
            if line.startswith("elements_per_launch:"):
                covered = int(line.split(":", 1)[1])
    assert covered is not None
    traffic, note = bench.profile_traffic("rod_step_fp64", "uneven_batch", srcs, covered)
    assert traffic is not None and traffic > 0, note
    traffic, note = bench.profile_traffic("rod_step_fp64", "uneven_batch", srcs, covered // 8)
    assert traffic is None and "covers" in note
    traffic, note = bench.profile_traffic("rod_step_fp64", "no_such_workload", srcs, covered)
    assert traffic is None and note == "no ncu summary"
