"""Rods of 520 to 1039 elements on CTA pairs (GPU).

A rod longer than one CTA's 520 slots runs on a cluster of two CTAs, each
holding half of its slots; neighbour reads across the split come from the
partner's shared memory.  Checked here: FP64 parity with the oracle (edge
lengths included: 520 elements, the shortest pair rod, and 1039, two full
halves), chunking invariance, the mixed-precision tip tolerance, and serving
of requests with long rods (same result alone and in a mix; same state as the
simulator)."""
import numpy as np
import pytest

import elasticapp_b200 as eb
from elasticapp_b200 import workloads as W

import oracle_bridge as B

pytestmark = pytest.mark.gpu

TIP_TOL = 1e-5
STATE = (("Position", 0), ("Velocity", 0), ("Director", 1), ("AngularVelocity", 1))


def straight_rods(lengths, seed):
    rng = np.random.default_rng(seed)
    rods = []
    for n in lengths:
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        c = rng.standard_normal(3)
        c -= c.dot(d) * d
        c /= np.linalg.norm(c)
        rods.append(eb.StraightRod(n_elements=n, material=eb.Material(1000.0, 1e6, 1e6 / 3), radius=0.01,
                                   length=float(0.002 * n), origin=tuple(rng.uniform(-1, 1, 3)),
                                   direction=tuple(d), normal=tuple(c)))
    vel = [rng.normal(0, 1e-2, (3, n + 1)) for n in lengths]
    return rods, vel


def check_parity(sim, wl, n_steps):
    orc, spread = B.oracle_spread(wl, n_steps)
    want = B.state_slots(orc)
    bounds = B.parity_bounds(spread)
    for name, place in STATE:
        err = B.max_rel_error_per_rod(sim.get_slots(name), want[name], wl.n_elements, place)
        assert err <= bounds[name], (name, err, bounds[name])


@pytest.mark.parametrize("lengths", [[520], [1039], [520, 1039, 519, 2, 263, 264, 777]])
def test_pair_rods_edge_lengths_vs_oracle(lengths):
    rods, vel = straight_rods(lengths, seed=sum(lengths))
    wl = W.Workload("pairs", 0, rods, velocities=vel, dt=2e-6, n_steps=200)
    sim = wl.build(step_mode="bucketed")
    sim.step(eb.PositionVerlet(), 0.0, wl.dt, 200)
    plan = sim.step_plan()
    assert plan["mode"] == "bucketed"
    assert (plan["config"] // 16) % 4 in (0, 1)  # the pair bucket's configuration
    assert max(plan["probe_ms"][13], plan["probe_ms"][14]) > 0.0  # the pair bucket was timed
    check_parity(sim, wl, 200)


def test_pair_rods_uneven_batch_vs_oracle_and_streaming():
    """Clamped, damped rods under gravity (the uneven batch's setup) with
    lengths across all three buckets, 300 steps: the oracle's parity bounds,
    and the FP64 streaming kernel's state to within the same bounds."""
    wl = W.uneven_batch(n_rods=10, seed=44, n_range=(100, 1039), n_steps=300)
    n = np.array(wl.n_elements)
    assert (n + 1 > 520).sum() >= 3
    sim = wl.build(step_mode="bucketed")
    sim.step(eb.PositionVerlet(), 0.0, wl.dt, 300)
    plan = sim.step_plan()
    assert plan["mode"] == "bucketed"
    assert max(plan["probe_ms"][16:20]) > 0.0  # short and medium rods also timed packed together
    check_parity(sim, wl, 300)
    ref = wl.build(step_mode="streaming")
    ref.step(eb.PositionVerlet(), 0.0, wl.dt, 300)
    for name in ("Position", "Director"):
        a, b = sim.get_slots(name), ref.get_slots(name)
        assert np.max(np.abs(a - b)) <= 1e-10 * max(1.0, np.max(np.abs(b))), name


def test_pair_rods_chunking_invariance():
    wl = W.uneven_batch(n_rods=4, seed=8, n_range=(600, 1000), n_steps=300)
    a = wl.build(step_mode="bucketed")
    b = wl.build(step_mode="bucketed")
    a.step(eb.PositionVerlet(), 0.0, wl.dt, 300)
    for k in (100, 7, 193):
        b.step(eb.PositionVerlet(), 0.0, wl.dt, k)
    for name, _ in STATE:
        assert np.array_equal(a.get_slots(name), b.get_slots(name)), name


def test_mixed_pair_rods_tip_error():
    wl = W.mixed_batch(n_rods=8, seed=91, n_range=(520, 1000))
    ref = wl.build(step_mode="streaming")
    ref.step(eb.PositionVerlet(), 0.0, wl.dt, 2000)
    mix = wl.build(precision="mixed")
    mix.step(eb.PositionVerlet(), 0.0, wl.dt, 2000)
    assert mix.step_plan()["mode"] == "bucketed"
    lengths = np.array([r.length for r in wl.rods])
    tip = lambda s: np.stack([r.get("Position")[:, -1] for r in s.rods])
    err = np.linalg.norm(tip(mix) - tip(ref), axis=1) / lengths
    assert np.all(np.isfinite(err)) and err.max() <= TIP_TOL, err.max()


def _request(seed, n_rods, n_range):
    rng = np.random.Generator(np.random.PCG64(seed))
    rods, n, L, E, d = W._random_rods(rng, n_rods, *n_range)
    vel = [rng.normal(0.0, 1e-3, size=(3, int(k) + 1)) for k in n]
    dt = 0.1 * float(np.min((L / n) / np.sqrt(E / 1000.0)))
    return rods, vel, dt


def _serve(requests, budget=2e9, **kw):
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
            out[i] = (c, [srv.result(c["request_id"], k, "Position") for k in range(len(requests[i][0]))],
                      [srv.result(c["request_id"], k, "Director") for k in range(len(requests[i][0]))])
        if left == 0 and not pending:
            break
        assert tick < 200000
    stats = srv.stats()
    srv.close()
    return out, stats


def test_served_long_rods_same_alone_and_in_mix():
    target = _request(61, 5, (300, 1039))
    assert max(r.n_elements for r in target[0]) > 519
    alone, _ = _serve([(*target, 400, 0)])
    mix = []
    for j in range(8):
        rods, vel, dt = _request(500 + j, 1 + (j * 5) % 9, (32, 1039 if j % 2 else 400))
        mix.append((rods, vel, dt, 150 + 61 * j, j % 3))
    mix.append((*target, 400, 2))
    mixed, stats = _serve(mix)
    assert stats["completed"] == len(mix)
    for k in range(len(target[0])):
        np.testing.assert_array_equal(alone[0][1][k], mixed[len(mix) - 1][1][k])
        np.testing.assert_array_equal(alone[0][2][k], mixed[len(mix) - 1][2][k])


def test_served_long_rods_match_simulator():
    rods, vel, dt = _request(71, 4, (520, 1039))
    steps = 300
    out, _ = _serve([(rods, vel, dt, steps, 0)], precision="fp64")
    comp, pos, _ = out[0]
    assert comp["precision"] == "fp64"
    wl = W.Workload("served_long", 71, rods, velocities=vel, dt=dt, n_steps=steps)
    sim = wl.build(step_mode="bucketed")
    sim.step(eb.PositionVerlet(), 0.0, dt, steps)
    for k, ref in enumerate(sim.rods):
        want = ref.get("Position")
        assert np.max(np.abs(pos[k] - want)) <= 1e-12 * np.max(np.abs(want))
    check_parity(sim, wl, steps)
