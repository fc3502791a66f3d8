"""Clamps at any index and the torque at any element on the GPU, against
the oracle (the FP64 parity rule) on every plan, and the mixed path within
its tip tolerance: rods held at both ends (nodes 0 and n), a rod held at an
inner node, and a torque on an inner element."""
import numpy as np
import pytest

from oracle_bridge import max_rel_error_per_rod, oracle_from_workload, oracle_spread, parity_bounds, state_slots

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eb():
    import elasticapp_b200
    return elasticapp_b200


def _workload(n_rods=10, seed=31, n_range=(20, 300)):
    from elasticapp_b200 import workloads as W
    wl = W.uneven_batch(n_rods=n_rods, seed=seed, n_range=n_range)
    n = wl.n_elements
    wl.clamp_at = [[0, int(m)] for m in n]   # beams held at both ends
    wl.clamp_at[1] = [int(n[1]) // 2]        # held at an inner node only
    wl.clamp_at[3] = [int(n[3])]             # held at the tip only
    wl.end_torque = np.tile([2e-5, -1e-5, 3e-5], (len(n), 1))
    wl.torque_element = [int(m) // 3 for m in n]
    return wl


@pytest.mark.parametrize("kw", [{"step_mode": "streaming"}, {"step_mode": "streaming", "reference_rounding": True},
                                {"step_mode": "streaming", "window": 128}, {"step_mode": "resident"},
                                {"step_mode": "bucketed"}],
                         ids=["streaming", "reference-rounding", "windowed", "resident", "bucketed"])
def test_clamps_and_inner_torque_vs_oracle(eb, kw):
    wl = _workload()
    steps = 600
    base, spread = oracle_spread(wl, steps)
    bounds = parity_bounds(spread)
    sim = wl.build(**kw)
    sim.step(eb.PositionVerlet(), 0.0, wl.dt, steps)
    want = state_slots(base)
    for name, place in (("Position", 0), ("Velocity", 0), ("Director", 1), ("AngularVelocity", 1)):
        err = max_rel_error_per_rod(sim.get_slots(name), want[name], wl.n_elements, place)
        assert err <= bounds[name], (name, err, bounds[name], kw)
    # the held nodes sit exactly at their targets
    for r, at in enumerate(wl.clamp_at):
        x = sim.rods[r].get("Position")
        xo = base.get_rod("x", r, int(wl.n_elements[r]) + 1)
        for k in at:
            np.testing.assert_array_equal(x[:, k], xo[:, k])
    sim.close()


def test_clamps_and_inner_torque_mixed_precision(eb):
    wl = _workload(seed=32)
    steps = 1000
    orc = oracle_from_workload(wl)
    orc.step(wl.dt, steps)
    sim = wl.build(precision="mixed")
    sim.step(eb.PositionVerlet(), 0.0, wl.dt, steps)
    for r, rod in enumerate(wl.rods):
        n = int(wl.n_elements[r])
        x, xo = sim.rods[r].get("Position"), orc.get_rod("x", r, n + 1)
        assert np.max(np.linalg.norm(x - xo, axis=0)) / rod.length <= 1e-5
        for k in wl.clamp_at[r]:
            np.testing.assert_array_equal(x[:, k], xo[:, k])
    sim.close()


def test_constraint_argument_errors(eb):
    from elasticapp_b200._lib import EbError
    rod = eb.StraightRod(n_elements=20, material=eb.Material(1000.0, 1e6, 1e6 / 3), radius=0.01, length=1.0)
    sim = eb.Simulator()
    ref = sim.emplace_back(eb.CosseratRodWithoutDamping, rod)
    with pytest.raises(EbError):
        sim.constrain(ref).at(21).using(eb.Clamp())   # past the last node
    sim.constrain(ref).at(0).using(eb.Clamp())
    with pytest.raises(EbError):
        sim.constrain(ref).at(0).using(eb.Clamp())    # the same index twice
    sim.constrain(ref).at(20).using(eb.Clamp())
    with pytest.raises(EbError):
        sim.constrain(ref).at(10).using(eb.Clamp())   # a third clamp
    sim.force(ref).at(5).using(eb.EndTorque((0.0, 0.0, 1e-3)))
    sim.force(ref).at(5).using(eb.EndTorque((0.0, 1e-3, 0.0)))  # sums on the same element
    with pytest.raises(EbError):
        sim.force(ref).at(6).using(eb.EndTorque((0.0, 0.0, 1e-3)))
    with pytest.raises(EbError):
        sim.force(ref).at(20).using(eb.EndTorque((0.0, 0.0, 1e-3)))  # no element 20
    sim.close()
