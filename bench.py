"""Rod-step throughput (element-steps/s) of the B200 FP64 drop-in.

Default workload: the uneven FP64 batch — 16,384 clamped rods, n ~ U{32..512}
elements (~4.44 M elements), gravity, analytical damper 0.1, one PositionVerlet
step per bench step (one fused kernel launch).  Seeded synthetic inputs.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank runs its own independent batch (seed + rank) on its
own GPU with no data-path collective (weak scaling); the timed region is
bracketed by a barrier and a device synchronize and the max over ranks is
reported.  Rank 0 prints one JSON line.

``--impl reference`` times the CPU restatement of the reference's scalar path
(the oracle, OpenMP over rods on every host core) on the same workload; only
rank 0 runs it.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "element-steps/s"
UNIT = "element-steps/s"
PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
E2E_STEPS_PER_CYCLE = 100  # run_for interval between host syncs (examples/dynamic_cantilever/helpers/data.py:60 uses 100-500)


def algorithmic_bytes(n_elems: np.ndarray, damped: bool) -> float:
    """Bytes one step must move at minimum: the state x, v (nodes) and Q, w
    (elements) read and written once, plus each parameter read once
    (m per node; l0, sigma0, S, J per element; D0, kappa0, B per Voronoi
    point; nu_f / nu_t for explicitly damped rods).  Derived quantities
    (lengths, strains, curvature, loads, 1/m, 1/J) are recomputed, not counted.
    Per element this is 432 B (448 B with explicit damping), the per-unit
    figure times the elements of one launch."""
    per_elem = 432.0 + (16.0 if damped else 0.0)
    return per_elem * float(np.sum(n_elems))


def hbm_peak():
    try:
        with open(PEAKS_PATH, encoding="utf-8") as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def source_digest(*names: str) -> str:
    """First 16 hex digits of the SHA-256 of the named kernel sources."""
    import hashlib

    h = hashlib.sha256()
    for n in names:
        with open(os.path.join(ROOT, "elasticapp_b200", "csrc", n), "rb") as f:
            h.update(f.read())
    return h.hexdigest()[:16]


def profile_traffic(kernel: str, workload: str, sources: tuple, elements: int):
    """DRAM bytes per launch from the committed ncu summary of this kernel
    and workload, if its recorded source digest matches the kernel sources
    as they are now (a summary of an older kernel is not reported) and it
    covers a launch over the same number of elements.
    Returns (bytes or None, note)."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.txt")
    traffic, digest, covered = None, None, None
    try:
        with open(path, encoding="utf-8") as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    traffic = float(line.split(":", 1)[1].strip())
                elif line.startswith("source_digest:"):
                    digest = line.split(":", 1)[1].strip()
                elif line.startswith("elements_per_launch:"):
                    covered = int(line.split(":", 1)[1].strip())
    except OSError:
        return None, "no ncu summary"
    now = source_digest(*sources)
    if digest != now:
        return None, f"stale ncu summary ({digest} != {now})"
    if covered != elements:
        return None, f"ncu summary covers {covered} elements, this launch {elements}"
    return traffic, f"ncu, sources {now}"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = os.path.join("/tmp", f"eb_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path, encoding="utf-8") as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx = float(parts[2])
                except ValueError:
                    continue
                for name, val in zip(names, parts[5:9]):
                    if val.lower().startswith("active"):
                        reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_reference_rate(wl, n_steps: int, budget_s: float = None, max_rods: int | None = None):
    """Oracle (CPU restatement of the reference's scalar path) throughput on
    this host, OpenMP over rods on every core.  Returns (rate, cores, sample)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle  # noqa: F401  (checker / CPU baseline only)
    import oracle_bridge

    sub = wl
    if max_rods is not None and max_rods < len(wl.rods):
        import copy

        sub = copy.copy(wl)
        sub.rods = wl.rods[:max_rods]
        sub.velocities = None if wl.velocities is None else wl.velocities[:max_rods]
        sub.rest_curvature = None if wl.rest_curvature is None else wl.rest_curvature[:max_rods]
        sub.end_torque = None if wl.end_torque is None else wl.end_torque[:max_rods]
    orc = oracle_bridge.oracle_from_workload(sub)
    cores = os.cpu_count() or 1
    orc.step(wl.dt, 1, n_threads=cores)  # warm-up
    done, t0 = 0, time.perf_counter()
    while True:
        orc.step(wl.dt, 1, n_threads=cores)
        done += 1
        el = time.perf_counter() - t0
        if (budget_s is None and done >= n_steps) or (budget_s is not None and el >= budget_s):
            break
    rate = sub.total_elements * done / el
    sample = f"{len(sub.rods)} rods / {sub.total_elements} elements x {done} steps"
    return rate, cores, sample


def bench_workload(args, W, rank, world):
    """The rods this rank steps.  One process: the named workload.  Several
    (weak scaling): one global batch of world x the per-GPU rods, sharded by
    the Karmarkar-Karp partition of its rods (element-balanced); the
    cantilever runs as one replica per rank."""
    if args.workload == "cantilever":
        return W.cantilever()
    if world > 1:
        from elasticapp_b200 import dist as ebdist
        per = args.rods if args.rods is not None else 16384
        return ebdist.shard(W.WORKLOADS[args.workload](n_rods=per * world, seed=1002), rank, world)
    kw = {"seed": 1002 + rank}
    if args.rods is not None:
        kw["n_rods"] = args.rods
    return W.WORKLOADS[args.workload](**kw)


def run_reference(args, W):
    """The reference arm: the CPU restatement of the reference's scalar path
    on all host cores, on the rods rank 0 of the GPU arm steps (the whole
    workload on one process; rank 0's shard under torchrun, where only rank 0
    runs and the others exit at once).  Element-steps/s of this CPU path does
    not depend on how many rods it holds beyond a few thousand, so the shard
    stands for the whole job."""
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    wl = bench_workload(args, W, 0, world)
    cores = os.cpu_count() or 1
    # warm-up steps, then K timed steps over the whole workload
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_bridge as ob  # CPU restatement of the reference path (the checker)

    orc = ob.oracle_from_workload(wl)
    for _ in range(args.warmup):
        orc.step(wl.dt, 1, n_threads=cores)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        orc.step(wl.dt, 1, n_threads=cores)
    el = time.perf_counter() - t0
    value = wl.total_elements * args.steps / el
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": workload_config(wl, world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{'rank 0 shard' if world > 1 else 'whole workload'} "
                                   f"({len(wl.rods)} rods, {wl.total_elements} elements) "
                                   f"x {args.steps} steps; CPU restatement of the reference's scalar "
                                   "path (reference not buildable here: Blaze/TBB absent)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def workload_config(wl, world):
    return {"workload": wl.name, "rods": len(wl.rods), "elements": wl.total_elements,
            "n_elements": [int(wl.n_elements.min()), int(wl.n_elements.max())], "dt": wl.dt,
            "seed": wl.seed, "stepper": "PositionVerlet",
            "constraints": "clamp(node 0) + analytical damper 0.1", "gravity": list(wl.gravity or []),
            "parallelism": f"{world} element-balanced shards of one batch of {world} x the per-GPU rods "
                           "(Karmarkar-Karp partition, weak)" if world > 1 else "single GPU",
            "l2": "no flush: inputs >> 126 MB L2"}


def mixed_comparison(W, eb, torch, args, rank, local, barrier, pg):
    """The mixed batch (65,536 rods, n ~ U{64..256}, helical rest curvature,
    end torque) advanced args.mixed_steps steps three ways from the same
    initial state: the FP64 streaming drop-in (one launch a step), the FP64
    default plan (the planner's choice, resident on this batch) and the
    mixed-precision resident kernel.  Tip positions and total energies after
    the run are compared with the FP64 default plan's."""
    wl = W.mixed_batch(n_rods=args.mixed_rods, seed=1003 + rank)
    out = {"workload": "mixed_batch", "rods": len(wl.rods), "elements": wl.total_elements, "dt": wl.dt,
           "steps": args.mixed_steps, "untimed_steps_before": 128,
           "dt_rule": "0.5 min(l^2/(r c)); 1e-5 s is unstable for these rods in the FP64 reference path"}
    res = {}
    for label, kw in (("fp64_streaming", {"step_mode": "streaming"}), ("fp64_default", {}),
                      ("mixed", {"precision": "mixed"})):
        sim = wl.build(device=local, **kw)
        # one untimed call of 128 steps (one resident launch): the step
        # planner times its candidates here, at the launch length of the
        # timed call, so no probe runs inside the timed region
        t0 = sim.step(eb.PositionVerlet(), 0.0, wl.dt, 128)
        e0 = sim.energy().sum()
        stream = torch.cuda.ExternalStream(sim.stream_handle(), device=torch.device("cuda", local))
        barrier()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sim.step(eb.PositionVerlet(), t0, wl.dt, args.mixed_steps)
        b.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms = torch.tensor([a.elapsed_time(b)], device="cuda")
        if pg is not None:
            pg.all_reduce(ms, op=pg.ReduceOp.MAX)
        tips = np.stack([r.get("Position")[:, -1] for r in sim.rods])
        e1 = sim.energy().sum()
        res[label] = {"ms": float(ms.item()), "tips": tips, "e0": e0, "e1": e1, "plan": sim.step_plan()}
        sim.close()
    lengths = np.array([r.length for r in wl.rods])
    ref = res["fp64_default"]
    err = np.linalg.norm(res["mixed"]["tips"] - ref["tips"], axis=1) / lengths
    err64 = np.linalg.norm(res["fp64_streaming"]["tips"] - ref["tips"], axis=1) / lengths
    n_el = float(wl.total_elements)
    rate = {k: n_el * args.mixed_steps / (v["ms"] / 1e3) for k, v in res.items()}
    out.update({
        "value": rate["mixed"], "unit": UNIT,
        "fp64_streaming_value": rate["fp64_streaming"],
        "fp64_default_value": rate["fp64_default"],
        "fp64_default_plan": ref["plan"]["mode"],
        "mixed_plan": res["mixed"]["plan"]["mode"],
        "tip_error_max": float(np.max(err)), "tip_error_p99": float(np.percentile(err, 99)),
        "tip_error_definition": "|tip_mixed - tip_fp64_default| / rod length after all steps",
        "fp64_plans_tip_diff_max": float(np.max(err64)),
        "energy_fp64": [ref["e0"], ref["e1"]], "energy_mixed": [res["mixed"]["e0"], res["mixed"]["e1"]],
        "energy_rel_diff": abs(res["mixed"]["e1"] - ref["e1"]) / abs(ref["e1"]),
        "finite": bool(np.all(np.isfinite(err))),
    })
    out["speedup_vs_fp64_streaming"] = rate["mixed"] / rate["fp64_streaming"]
    out["speedup_vs_fp64_default"] = rate["mixed"] / rate["fp64_default"]
    return out


def contact_comparison(W, eb, torch, args, rank, local, world, barrier, pg):
    """The contact batch (8,192 free rods of 64 elements, six walls) on the
    FP64 streaming step with the collision system.  Its dynamics diverges
    within tens of microseconds in the reference's model (thin capsules,
    contact torques on a 4e-11 kg m^2 element inertia), so every timed step
    starts from the batch's initial state: the state is restored between
    steps outside the timed region and each step is timed alone."""
    wl = W.contact_batch(n_rods=args.contact_rods, seed=1004 + rank)
    sim = wl.build(device=local)
    names = ("Position", "Velocity", "Director", "AngularVelocity")
    init = {n: sim.get_slots(n).copy() for n in names}
    stream = torch.cuda.ExternalStream(sim.stream_handle(), device=torch.device("cuda", local))
    times = []
    l0 = sim.launch_count()
    for i in range(args.warmup + args.contact_steps):
        for n in names:
            sim.set_slots(n, init[n])
        torch.cuda.synchronize()
        barrier()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sim.step(eb.PositionVerlet(), 0.0, wl.dt, 1)
        b.record(stream)
        torch.cuda.synchronize()
        if i >= args.warmup:
            times.append(a.elapsed_time(b))
    launches = (sim.launch_count() - l0) // (args.warmup + args.contact_steps)
    ms = torch.tensor([sum(times) / len(times)], device="cuda")
    if pg is not None:
        pg.all_reduce(ms, op=pg.ReduceOp.MAX)
    pairs = sim.contact_pairs()
    n_slots = sim.n_slots()
    force = sim.get_slots("ContactForce")
    out = {"workload": "contact_batch", "rods": len(wl.rods), "capsules": wl.total_elements, "dt": wl.dt,
           "planes": len(wl.planes), "seed": wl.seed,
           "value": world * wl.total_elements / (float(ms.item()) / 1e3), "unit": UNIT,
           "ms_per_step": float(ms.item()), "steps_timed": args.contact_steps,
           "launches_per_step": int(launches),
           "candidate_pairs": int(pairs.shape[0]),
           "capsule_plane_pairs": int((pairs[:, 1] >= n_slots).sum()),
           "capsules_with_contact_force": int(np.count_nonzero(np.abs(force).sum(axis=0))),
           "timing": "each step from the initial state (state restored between steps, outside the timing)",
           "parity": "candidate pair set bit-exact and capsule loads equal to the oracle (tests/test_gpu_contact.py)"}
    sim.close()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle  # noqa: F401  (checker / CPU baseline only)
        import oracle_bridge as ob

        orc = ob.oracle_from_workload(wl)
        spec = ob.contact_spec(wl)
        cores = os.cpu_count() or 1
        t0 = time.perf_counter()
        oracle.contact_step(orc, spec, wl.dt, 1, n_threads=cores)
        el = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": wl.total_elements / el, "unit": UNIT, "cores": cores, "kind": "port",
                               "sample": "one contact step of the whole batch (CPU restatement: uniform-grid "
                                         "broad phase, narrow phase, spring-dashpot, rod step)"}
    return out


def cantilever_section(eb, W, torch, args, local):
    """The single-rod cantilever (1 rod, 100 elements, clamp, gravity,
    analytical damper 0.1, dt 1e-5, 1e5 steps): timed run on the planner's
    kernel, then the tip trajectory every 1000 steps against the oracle."""
    wl = W.cantilever()
    n_steps, every = args.cantilever_steps, 1000
    out = {"workload": "cantilever", "rods": 1, "elements": wl.total_elements, "dt": wl.dt, "steps": n_steps}
    for label, kw in (("auto", {}), ("streaming_graph", {"step_mode": "streaming", "cuda_graph": True})):
        sim = wl.build(device=local, **kw)
        t = sim.step(eb.PositionVerlet(), 0.0, wl.dt, 128)  # plan + warm-up
        sim.synchronize()
        stream = torch.cuda.ExternalStream(sim.stream_handle(), device=torch.device("cuda", local))
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sim.step(eb.PositionVerlet(), t, wl.dt, n_steps)
        b.record(stream)
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        out[label] = {"value": wl.total_elements * n_steps / (ms / 1e3), "unit": UNIT, "ms_total": ms,
                      "us_per_step": 1e3 * ms / n_steps, "plan": sim.step_plan()["mode"]}
        sim.close()
    out["value"] = max(out["auto"]["value"], out["streaming_graph"]["value"])
    # tip trajectory against the oracle (fresh runs from the initial state)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_bridge as ob

    sim = wl.build(device=local)
    orc = ob.oracle_from_workload(wl)
    t, errs = 0.0, []
    t0 = time.perf_counter()
    cpu_s = 0.0
    for _ in range(n_steps // every):
        t = sim.step(eb.PositionVerlet(), t, wl.dt, every)
        c0 = time.perf_counter()
        orc.step(wl.dt, every, n_threads=1)
        cpu_s += time.perf_counter() - c0
        tip_g = sim.rods[0].get("Position")[:, -1]
        tip_o = orc.get_rod("x", 0, wl.n_elements[0] + 1)[:, -1]
        errs.append(float(np.linalg.norm(tip_g - tip_o)) / wl.rods[0].length)
    sim.close()
    out["tip_trajectory"] = {"samples": len(errs), "every_steps": every, "max_rel_error": max(errs),
                             "final_rel_error": errs[-1], "final_tip": [float(v) for v in tip_g],
                             "definition": "|tip_gpu - tip_oracle| / rod length, sampled every 1000 steps"}
    out["cpu_baseline"] = {"value": wl.total_elements * n_steps / cpu_s, "unit": UNIT, "cores": 1, "kind": "port",
                           "sample": "the whole 1e5-step run (one rod: one core)"}
    return out


def _serve_request(eb, W, rng):
    """One request of the serving stream: 1-256 rods (log-uniform), n ~
    U{32..1024}, horizon ~ U{1e3..1e5} steps, per-rod parameters as in the
    uneven batch (clamp, damper 0.1, gravity, node velocities N(0, 1e-3^2))."""
    k = int(min(256, max(1, round(float(np.exp(rng.uniform(0.0, np.log(256.0))))))))
    rods, n, L, E, d = W._random_rods(rng, k, 32, 1024)
    vel = [rng.normal(0.0, 1e-3, size=(3, int(m) + 1)) for m in n]
    dt = 0.1 * float(np.min((L / n) / np.sqrt(E / 1000.0)))
    steps = int(rng.integers(1000, 100001))
    return rods, vel, dt, steps, int(n.sum())


def censored_percentiles(done: np.ndarray, censored: np.ndarray, qs=(50, 99)) -> dict:
    """Percentiles of a latency sample in which some requests had not
    finished when the run ended.  An unfinished request contributes its age
    at the end, a lower bound on its latency, so each percentile taken over
    every submitted request is a lower bound of the true one whenever any
    request is censored (and exact when none is)."""
    allv = np.concatenate([np.asarray(done, float), np.asarray(censored, float)])
    if allv.size == 0:
        return {f"p{q}": None for q in qs}
    return {f"p{q}": float(np.percentile(allv, q)) for q in qs}


def serve_stream(eb, W, rate, seconds, drain_s, seed, budget):
    """Poisson arrivals at `rate` requests/s for `seconds`, then up to
    `drain_s` more seconds.  Latency = completion seen - scheduled arrival;
    requests still unfinished at the end count with their age then (censored,
    so the percentiles over all submitted requests are lower bounds).
    Queueing delay = submission to first admission (server clock; still
    queued: age at the end).  Each request is generated at its arrival time
    (the client's work; the server's ticks run for hundreds of milliseconds
    each at this load, so it does not delay them)."""
    from elasticapp_b200.server import Server

    srv = Server(precision="mixed", hbm_budget_bytes=budget)
    arr_rng = np.random.Generator(np.random.PCG64(seed))
    arrivals, t = [], 0.0
    while True:
        t += float(arr_rng.exponential(1.0 / rate))
        if t >= seconds:
            break
        arrivals.append(t)
    arrival_of, lat, qdelay, work = {}, [], [], 0.0
    nxt = 0
    t0 = time.perf_counter()
    while True:
        now = time.perf_counter() - t0
        while nxt < len(arrivals) and arrivals[nxt] <= now:
            rods, vel, dt, steps, elems = _serve_request(
                eb, W, np.random.Generator(np.random.PCG64(seed * 1000003 + nxt)))
            rid = srv.submit(rods, dt, steps, gravity=(0.0, 0.0, -9.81), clamp=True, damper=(0.1, 0.1),
                             velocities=vel)
            arrival_of[rid] = arrivals[nxt]
            work += float(elems) * steps
            nxt += 1
        left = srv.tick()
        done = srv.poll()
        if done:
            seen = time.perf_counter() - t0
            for c in done:
                lat.append(seen - arrival_of.pop(c["request_id"]))
                qdelay.append(c["queued_s"])
                srv.release(c["request_id"])
        if (nxt == len(arrivals) and left == 0) or now > seconds + drain_s:
            break
    end = time.perf_counter() - t0
    # requests still in flight: latency and queueing delay censored at the end
    cens_lat, cens_q, never_admitted = [], [], 0
    for rid, arr in arrival_of.items():
        info = srv.request_status(rid)
        cens_lat.append(end - arr)
        cens_q.append(info["queued_s"])
        never_admitted += info["state"] == "queued"
    st = srv.stats()
    srv.close()
    lp = censored_percentiles(lat, cens_lat)
    qp = censored_percentiles(qdelay, cens_q)
    label = "censored_lower_bound" if cens_lat else "exact"
    return {"rate_req_s": rate, "arrival_window_s": seconds, "drain_s": drain_s, "submitted": len(arrivals),
            "completed": len(lat), "censored": len(cens_lat), "never_admitted": int(never_admitted),
            "fallbacks": int(st["fallbacks"]),
            "p50_latency_s": lp["p50"], "p99_latency_s": lp["p99"], "latency_percentiles": label,
            "p50_latency_completed_s": float(np.percentile(lat, 50)) if lat else None,
            "p99_latency_completed_s": float(np.percentile(lat, 99)) if lat else None,
            "p99_queueing_s": qp["p99"], "p50_queueing_s": qp["p50"],
            "elapsed_s": end, "value": st["element_steps"] / end, "unit": UNIT,
            "offered_element_steps_per_s": work / max(seconds, 1e-9), "ticks": int(st["ticks"]),
            "bins_total": int(st["bins_total"]), "kernel_seconds": st["kernel_seconds"],
            "gpu_busy_frac": st["kernel_seconds"] / end,
            "kernel_element_steps_per_s": st["element_steps"] / max(st["kernel_seconds"], 1e-9)}


def serving_section(eb, W, args, capacity_hint):
    """The serving stream at the stated load (200 requests/s) for a bounded
    arrival window, and at a sustainable load (half the measured capacity)."""
    out = {"workload": "serve_stream", "hbm_budget_bytes": args.serve_budget, "precision": "mixed (FP64 fallback)",
           "steps_per_launch": 128,
           "request": "1-256 rods log-uniform, n ~ U{32..1024} (520-slot bins, one CTA each; rods of 520 or more "
                      "elements on a bin pair run by a 2-CTA cluster), horizon U{1e3..1e5}, "
                      "clamp + damper 0.1 + gravity, velocities N(0, 1e-3^2); dt = 0.1 min(l/c) per request"}
    mean_work = 46.0 * 528.0 * 50500.0  # mean rods x mean n x mean horizon
    out["stated_load"] = serve_stream(eb, W, 200.0, args.serve_seconds, args.serve_drain, 1005, args.serve_budget)
    rate = args.serve_rate if args.serve_rate > 0 else max(1.0, 0.5 * capacity_hint / mean_work)
    out["sustained_load"] = serve_stream(eb, W, rate, args.serve_sustained_seconds, args.serve_drain, 1006,
                                         args.serve_budget)
    return out


def _pick(d, keys):
    return None if d is None else {k: d[k] for k in keys if k in d}


def compact_sections(batched, contact, serving, cantilever, mixed):
    """The side measurements reduced to their figures, so that the whole
    bench line stays short (the full sections go to --detail-out)."""
    out = {}
    if batched is not None:
        out["batched"] = {"value": batched["value"], "plan": batched["plan"]["mode"],
                          "ms_per_step": batched["ms_per_step"],
                          "pefrl_default": batched["pefrl"]["default_plan"]["value"],
                          "pefrl_streaming": batched["pefrl"]["streaming"]["value"]}
    if contact is not None:
        out["contact"] = _pick(contact, ("value", "ms_per_step", "candidate_pairs"))
        if contact.get("cpu_baseline"):
            out["contact"]["cpu_value"] = contact["cpu_baseline"]["value"]
    if cantilever is not None:
        out["cantilever"] = {"value": cantilever["value"],
                             "tip_err_max": cantilever["tip_trajectory"]["max_rel_error"],
                             "cpu_value": cantilever["cpu_baseline"]["value"]}
    if serving is not None:
        keys = ("rate_req_s", "arrival_window_s", "submitted", "completed", "censored", "p50_latency_s",
                "p99_latency_s", "latency_percentiles", "p99_queueing_s", "value", "gpu_busy_frac")
        out["serving"] = {"stated": _pick(serving["stated_load"], keys),
                          "sustained": _pick(serving["sustained_load"], keys)}
    if mixed is not None:
        out["mixed"] = _pick(mixed, ("rods", "elements", "steps", "dt", "value", "fp64_default_value",
                                     "fp64_streaming_value", "fp64_default_plan", "speedup_vs_fp64_default",
                                     "speedup_vs_fp64_streaming", "tip_error_max", "tip_error_p99",
                                     "energy_rel_diff", "finite"))
    return out


def relaunch_under_torchrun(n: int, argv) -> int:
    """bench.py --gpus N started without a launcher: run N ranks on this node
    with torch.distributed.run (rendezvous on 127.0.0.1) and return its exit
    status.  Rank 0 prints the line."""
    import socket

    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + list(argv)
    return subprocess.run(cmd, check=False).returncode


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="uneven_batch")
    ap.add_argument("--rods", type=int, default=None, help="smaller batch (profiling captures only)")
    ap.add_argument("--e2e-cycles", type=int, default=3)
    ap.add_argument("--batched-steps", type=int, default=256,
                    help="steps timed on the resident (batched) kernel; 0 skips it")
    ap.add_argument("--resident-config", type=int, default=0,
                    help="resident configuration (1-based; 0 = chosen by timing)")
    ap.add_argument("--mixed-rods", type=int, default=65536, help="rods of the mixed-precision batch")
    ap.add_argument("--mixed-steps", type=int, default=10000,
                    help="steps of the FP64-vs-mixed comparison on the mixed batch; 0 skips it")
    ap.add_argument("--contact-rods", type=int, default=8192, help="rods of the contact batch")
    ap.add_argument("--contact-steps", type=int, default=10,
                    help="timed steps of the contact batch (each from its initial state); 0 skips it")
    ap.add_argument("--cantilever-steps", type=int, default=100000,
                    help="steps of the single-rod cantilever; 0 skips it")
    ap.add_argument("--serve-seconds", type=float, default=60.0,
                    help="arrival window of the stated-load serving stream; 0 skips serving")
    ap.add_argument("--serve-sustained-seconds", type=float, default=30.0,
                    help="arrival window of the sustained-load serving stream")
    ap.add_argument("--serve-drain", type=float, default=30.0, help="extra seconds to finish in-flight requests")
    ap.add_argument("--serve-rate", type=float, default=0.0,
                    help="sustained-load arrival rate (0: half the measured mixed capacity)")
    ap.add_argument("--serve-budget", type=float, default=40e9, help="HBM budget of the serving pool (bytes)")
    ap.add_argument("--cpu-budget-s", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--reference-rounding", action="store_true",
                    help="FP64 build that rounds every operation as the reference's scalar code")
    ap.add_argument("--window", type=int, default=0, help="slots per CTA of the step kernel (128/256)")
    ap.add_argument("--detail-out", default=None, help="also write every section in full to this JSON file")
    args = ap.parse_args(argv)
    args.warmup = max(args.warmup, 3)

    # --gpus N is the number of ranks: started without a launcher, relaunch
    # under torch.distributed.run; under a launcher, the world size must agree
    launched = "WORLD_SIZE" in os.environ
    if not launched and args.gpus > 1:
        return relaunch_under_torchrun(args.gpus, sys.argv[1:] if argv is None else argv)
    if launched and int(os.environ["WORLD_SIZE"]) != args.gpus:
        print(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={os.environ['WORLD_SIZE']}", file=sys.stderr)
        return 2

    from elasticapp_b200 import workloads as W

    if args.impl == "reference":
        return run_reference(args, W)

    import torch

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        pg = dist

    import elasticapp_b200 as eb

    wl = bench_workload(args, W, rank, world)
    sim = wl.build(device=local, reference_rounding=args.reference_rounding, window=args.window,
                   step_mode="streaming")
    stream = torch.cuda.ExternalStream(sim.stream_handle(), device=torch.device("cuda", local))
    t = 0.0
    t = sim.step(eb.PositionVerlet(), t, wl.dt, args.warmup)
    sim.synchronize()

    def barrier():
        if pg is not None:
            pg.barrier()

    # ---- device-timed region: exactly K steps, one launch each
    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.3)
    launches0 = sim.launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        t = sim.step(eb.PositionVerlet(), t, wl.dt, 1)
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clock_info = clocks.stop()
    launches = sim.launch_count() - launches0
    ms = ev0.elapsed_time(ev1)
    ms_t = torch.tensor([ms], device="cuda")
    elems_t = torch.tensor([float(wl.total_elements)], device="cuda", dtype=torch.float64)
    if pg is not None:
        pg.all_reduce(ms_t, op=pg.ReduceOp.MAX)
        pg.all_reduce(elems_t)
    ms_max = float(ms_t.item())
    total_elems = float(elems_t.item())
    value = total_elems * args.steps / (ms_max / 1e3)

    # ---- roofline of the step kernel (this rank)
    peak, peak_kind = hbm_peak()
    alg = algorithmic_bytes(wl.n_elements, damped=False)
    per_launch_s = (ms / 1e3) / args.steps
    achieved = alg / per_launch_s / 1e9
    traffic, traffic_note = profile_traffic("rod_step_fp64", wl.name, ("rod_step_fp64.cu", "rod_math.cuh", "bulk_copy.cuh"),
                                            int(sum(wl.n_elements)))

    # ---- end to end through the public API with host buffers: each cycle
    # uploads the dynamic state from pinned memory, runs E2E_STEPS_PER_CYCLE
    # steps and reads the state back (the reference's run_for + communicate)
    # in one eb_step_host_state call, which overlaps the copies of each slot
    # group with the steps of the others under a resident plan; a simulator
    # with the default plan (chosen by timing at its first step) and one
    # exchange (building the slot groups) run untimed before the cycles
    names = ("Position", "Velocity", "Director", "AngularVelocity")
    ncomp = {"Position": 3, "Velocity": 3, "Director": 9, "AngularVelocity": 3}
    e2e_plan = None
    if args.e2e_cycles > 0:
        esim = wl.build(device=local)
        estream = torch.cuda.ExternalStream(esim.stream_handle(), device=torch.device("cuda", local))
        S = esim.n_slots()
        host = {n: torch.empty((ncomp[n], S), dtype=torch.float64, pin_memory=True).numpy() for n in names}
        for n in names:
            esim.get_slots(n, out=host[n])
        te = esim.step(eb.PositionVerlet(), 0.0, wl.dt, E2E_STEPS_PER_CYCLE)
        e2e_plan = esim.step_plan()["mode"]
        te = esim.step_host_state(eb.PositionVerlet(), te, wl.dt, E2E_STEPS_PER_CYCLE, inputs=host, outputs=host)
    else:
        esim, estream, S = sim, stream, sim.n_slots()
        host = {n: np.zeros((ncomp[n], S)) for n in names}
    bytes_cycle = sum(8 * ncomp[n] * S for n in names)
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(estream)
    for _ in range(max(args.e2e_cycles, 0)):
        te = esim.step_host_state(eb.PositionVerlet(), te, wl.dt, E2E_STEPS_PER_CYCLE, inputs=host, outputs=host)
    e1.record(estream)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = torch.tensor([e0.elapsed_time(e1)], device="cuda")
    if pg is not None:
        pg.all_reduce(e2e_ms, op=pg.ReduceOp.MAX)
    e2e_value = (total_elems * E2E_STEPS_PER_CYCLE * args.e2e_cycles / (float(e2e_ms.item()) / 1e3)
                 if args.e2e_cycles > 0 else None)
    finite = all(np.isfinite(host[n]).all() for n in names)
    if esim is not sim:
        esim.close()

    # ---- the resident (batched) form of the same step on the same workload
    batched = None
    if args.batched_steps > 0:
        sim.close()
        bsim = wl.build(device=local, step_mode="resident", resident_config=args.resident_config)
        tb = bsim.step(eb.PositionVerlet(), 0.0, wl.dt, 128)  # plan + warm-up
        bsim.synchronize()
        bstream = torch.cuda.ExternalStream(bsim.stream_handle(), device=torch.device("cuda", local))
        barrier()
        torch.cuda.synchronize()
        l0 = bsim.launch_count()
        b0 = torch.cuda.Event(enable_timing=True)
        b1 = torch.cuda.Event(enable_timing=True)
        b0.record(bstream)
        tb = bsim.step(eb.PositionVerlet(), tb, wl.dt, args.batched_steps)
        b1.record(bstream)
        torch.cuda.synchronize()
        barrier()
        bms = torch.tensor([b0.elapsed_time(b1)], device="cuda")
        if pg is not None:
            pg.all_reduce(bms, op=pg.ReduceOp.MAX)
        plan = bsim.step_plan()
        batched = {"value": total_elems * args.batched_steps / (float(bms.item()) / 1e3), "unit": UNIT,
                   "steps": args.batched_steps, "ms_per_step": float(bms.item()) / args.batched_steps,
                   "launches": bsim.launch_count() - l0, "plan": plan,
                   "kernel": "rod_block_fp64 (whole rods resident in shared memory, up to 128 steps per launch)"}
        bsim.close()
        sim = None
        # the same batch with PEFRL (four force evaluations a step): the
        # default plan against the streaming kernel (four launches a step)
        pefrl = {}
        for mode in ("auto", "streaming"):
            psim = wl.build(device=local, stepper=eb.PEFRL(), step_mode=mode)
            tp = psim.step(eb.PEFRL(), 0.0, wl.dt, 128)  # plan + warm-up
            pstream = torch.cuda.ExternalStream(psim.stream_handle(), device=torch.device("cuda", local))
            n_p = 128 if mode == "auto" else 32
            barrier()
            torch.cuda.synchronize()
            p0 = torch.cuda.Event(enable_timing=True)
            p1 = torch.cuda.Event(enable_timing=True)
            p0.record(pstream)
            tp = psim.step(eb.PEFRL(), tp, wl.dt, n_p)
            p1.record(pstream)
            torch.cuda.synchronize()
            barrier()
            pms = torch.tensor([p0.elapsed_time(p1)], device="cuda")
            if pg is not None:
                pg.all_reduce(pms, op=pg.ReduceOp.MAX)
            pefrl[mode] = {"value": total_elems * n_p / (float(pms.item()) / 1e3), "steps": n_p,
                           "ms_per_step": float(pms.item()) / n_p, "plan": psim.step_plan()["mode"]}
            psim.close()
        batched["pefrl"] = {"unit": UNIT, "force_evaluations_per_step": 4, "default_plan": pefrl["auto"],
                            "streaming": pefrl["streaming"]}

    # ---- mixed precision: the mixed batch on the FP64 streaming drop-in and
    # on the mixed-precision resident kernel, tip positions compared
    mixed = None
    if args.mixed_steps > 0:
        mixed = mixed_comparison(W, eb, torch, args, rank, local, barrier, pg)

    cantilever = None
    if args.cantilever_steps > 0 and rank == 0 and world == 1:
        cantilever = cantilever_section(eb, W, torch, args, local)

    serving = None
    if args.serve_seconds > 0 and rank == 0 and world == 1:
        cap = mixed["value"] if mixed else 2.0e10
        serving = serving_section(eb, W, args, cap)

    contact = None
    if args.contact_steps > 0:
        contact = contact_comparison(W, eb, torch, args, rank, local, world, barrier, pg)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, cores, sample = cpu_reference_rate(wl, 0, budget_s=args.cpu_budget_s, max_rods=2048)
        cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": sample + " (CPU restatement of the reference's scalar path, OpenMP over rods)"}

    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": workload_config(wl, world),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_source": f"{peak_kind} hbm_gbs" if peak_kind == "measured" else "fallback 6.65 TB/s",
                         "traffic_source": traffic_note,
                         "kernel": "rod_step_fp64" + ("_reference" if args.reference_rounding else ""),
                         "algorithmic_bytes_per_launch": alg},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": bytes_cycle,
                    "d2h_bytes_per_step": bytes_cycle, "steps_per_e2e_step": E2E_STEPS_PER_CYCLE,
                    "cycles": args.e2e_cycles, "plan": e2e_plan, "call": "eb_step_host_state"},
            "gpu_launches": launches,
            "clocks": clock_info,
            "state_finite": bool(finite),
        }
        if args.detail_out:
            full = dict(line, batched=batched, contact=contact, serving=serving, cantilever=cantilever,
                        mixed=mixed)
            with open(args.detail_out, "w", encoding="utf-8") as f:
                json.dump(full, f, indent=1)
        # the side measurements in short form, the mixed-precision target last
        line.update(compact_sections(batched, contact, serving, cantilever, mixed))
        print(json.dumps(line, separators=(",", ":")), flush=True)
    if sim is not None:
        sim.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
