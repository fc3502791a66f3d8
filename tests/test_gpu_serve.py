"""Serving (continuous batching) on the GPU.

* A served request gives the same state as the plain simulator run of the
  same rods in the same precision, and its mixed-precision tip stays within
  the mixed path's 1e-5 tolerance of the FP64 oracle.
* A request's result is the same served alone and served in a mix of other
  requests (different sizes, time steps, horizons, admitted while it runs):
  bit for bit, since each request's steps are chunked from its own admission.
* The FP64 fallback reruns a request in FP64 and delivers the FP64 result.
* Under a small HBM budget requests queue and are admitted as bins free up.
"""
import numpy as np
import pytest

from oracle_bridge import oracle_from_workload

pytestmark = pytest.mark.gpu

TIP_TOL = 1e-5


@pytest.fixture(scope="module")
def eb():
    import elasticapp_b200
    return elasticapp_b200


def _request(seed, n_rods, n_range=(32, 128)):
    from elasticapp_b200 import workloads as W
    rng = np.random.Generator(np.random.PCG64(seed))
    rods, n, L, E, d = W._random_rods(rng, n_rods, *n_range)
    vel = [rng.normal(0.0, 1e-3, size=(3, int(k) + 1)) for k in n]
    dt = 0.1 * float(np.min((L / n) / np.sqrt(E / 1000.0)))
    return rods, vel, dt


def _serve(eb, requests, budget=2e9, **kw):
    """Serve requests [(rods, vel, dt, steps, submit_at_tick)]; returns
    {index: (completion, [positions per rod], [directors per rod])}."""
    from elasticapp_b200.server import Server
    srv = Server(hbm_budget_bytes=budget, **kw)
    ids, out, tick = {}, {}, 0
    pending = sorted(range(len(requests)), key=lambda i: requests[i][4])
    while True:
        while pending and requests[pending[0]][4] <= tick:
            i = pending.pop(0)
            rods, vel, dt, steps, _ = requests[i]
            ids[srv.submit(rods, dt, steps, gravity=(0.0, 0.0, -9.81), clamp=True, damper=(0.1, 0.1),
                           velocities=vel)] = i
        left = srv.tick()
        tick += 1
        for c in srv.poll():
            i = ids[c["request_id"]]
            n_rods = len(requests[i][0])
            out[i] = (c, [srv.result(c["request_id"], k, "Position") for k in range(n_rods)],
                      [srv.result(c["request_id"], k, "Director") for k in range(n_rods)])
        if left == 0 and not pending:
            break
        assert tick < 200000
    stats = srv.stats()
    srv.close()
    return out, stats


def test_served_request_matches_simulator_and_oracle(eb):
    from elasticapp_b200.workloads import Workload
    rods, vel, dt = _request(11, 8)
    steps = 300  # two full launches of 128 and a partial one
    out, _ = _serve(eb, [(rods, vel, dt, steps, 0)])
    comp, pos, _ = out[0]
    assert comp["precision"] == "mixed" and not comp["fell_back"]
    wl = Workload("served", 11, rods, velocities=vel, dt=dt, n_steps=steps)
    sim = wl.build(precision="mixed")
    sim.step(eb.PositionVerlet(), 0.0, dt, steps)
    for k, ref in enumerate(sim.rods):
        want = ref.get("Position")
        assert np.max(np.abs(pos[k] - want)) <= 1e-12 * np.max(np.abs(want))
    sim.close()
    orc = oracle_from_workload(wl)
    orc.step(dt, steps)
    for k in range(len(rods)):
        tip = orc.get_rod("x", k, rods[k].n_elements + 1)[:, -1]
        assert np.linalg.norm(pos[k][:, -1] - tip) / rods[k].length <= TIP_TOL


def test_result_same_alone_and_in_mix(eb):
    target = _request(21, 6)
    alone, _ = _serve(eb, [(*target, 700, 0)])
    mix = []
    for j in range(12):
        rods, vel, dt = _request(100 + j, 1 + (j * 7) % 20, (16, 500 if j % 3 == 0 else 200))
        mix.append((rods, vel, dt, 200 + 97 * j, j % 4))
    mix.append((*target, 700, 3))  # admitted while others run
    mixed, stats = _serve(eb, mix)
    assert stats["completed"] == len(mix)
    a_pos, a_q = alone[0][1], alone[0][2]
    m_pos, m_q = mixed[len(mix) - 1][1], mixed[len(mix) - 1][2]
    for k in range(len(a_pos)):
        np.testing.assert_array_equal(a_pos[k], m_pos[k])
        np.testing.assert_array_equal(a_q[k], m_q[k])


def test_fp64_fallback_delivers_fp64_result(eb):
    rods, vel, dt = _request(31, 4)
    fb, stats = _serve(eb, [(rods, vel, dt, 260, 0)], force_fallback=True)
    c = fb[0][0]
    assert c["fell_back"] and c["precision"] == "fp64"
    assert stats["fallbacks"] == 1
    ref, _ = _serve(eb, [(rods, vel, dt, 260, 0)], precision="fp64")
    for k in range(len(rods)):
        np.testing.assert_array_equal(fb[0][1][k], ref[0][1][k])


def test_small_budget_queues_and_admits(eb):
    from elasticapp_b200.server import Server
    # a budget of a few bins: requests wait for bins to free up
    reqs = [(*_request(200 + j, 3, (100, 300)), 150 + 10 * j, 0) for j in range(10)]
    out, stats = _serve(eb, reqs, budget=2.0e6)
    assert stats["bins_total"] <= 8
    assert stats["completed"] == 10
    assert all(np.isfinite(p).all() for c, ps, _ in out.values() for p in ps)
    srv = Server(hbm_budget_bytes=2.0e6)
    from elasticapp_b200._lib import EbError
    with pytest.raises(EbError):  # larger than the whole pool
        rods, vel, dt = _request(300, 40, (400, 500))
        srv.submit(rods, dt, 10)
    srv.close()


def test_serve_error_paths(eb):
    from elasticapp_b200._lib import EbError
    from elasticapp_b200.server import Server
    srv = Server(hbm_budget_bytes=1e8)
    rods, vel, dt = _request(41, 2)
    with pytest.raises(EbError):
        srv.submit(rods, -1.0, 10)
    with pytest.raises(EbError):
        srv.submit(rods, dt, 0)
    long_rod = eb.StraightRod(n_elements=1040, material=eb.Material(1000.0, 1e6, 1e6 / 3), radius=0.01, length=1.0)
    with pytest.raises(EbError):
        srv.submit([long_rod], dt, 10)
    srv.close()


def test_request_status_and_queueing_delay(eb):
    """A request waiting for bins reports 'queued' with its age as a lower
    bound on its queueing delay; once done its completion carries the
    delay from submission to admission, no longer than its latency."""
    from elasticapp_b200.server import Server
    srv = Server(hbm_budget_bytes=2.0e6)  # a few bins: the second request waits
    n_bins = srv.stats()["bins_total"]
    # one rod of 300-500 elements a bin (two do not fit in 512 slots): the
    # first request takes every bin
    r1 = _request(500, n_bins, (300, 500))
    r2 = _request(501, 1, (100, 300))
    a = srv.submit(r1[0], r1[2], 300, velocities=r1[1])
    b = srv.submit(r2[0], r2[2], 300, velocities=r2[1])
    srv.tick()
    sa, sb = srv.request_status(a), srv.request_status(b)
    assert sa["state"] in ("active", "finishing", "done")
    assert sb["state"] == "queued" and sb["queued_s"] >= 0.0
    done = {}
    for _ in range(10000):
        left = srv.tick()
        for c in srv.poll():
            done[c["request_id"]] = c
        if left == 0:
            break
    done.update({c["request_id"]: c for c in srv.poll()})
    assert set(done) == {a, b}
    for rid in (a, b):
        c = done[rid]
        assert 0.0 <= c["queued_s"] <= c["latency_s"]
        assert srv.request_status(rid)["state"] == "done"
    assert done[b]["queued_s"] >= sb["queued_s"]
    with pytest.raises(Exception):
        srv.request_status(123456)
    srv.close()
