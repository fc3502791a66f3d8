"""Connections (joints) between rods on the GPU against the CPU restatement:
the hinge chain of the reference's hinge-joint example (clamped, damped
links under gravity), free joints with dashpots and several connections on
one node, connections beside the collision system, and the argument checks
of eb_connect."""
import numpy as np
import pytest

import elasticapp_b200 as eb
from elasticapp_b200 import _lib as L
from elasticapp_b200 import workloads as W

import oracle_bridge as B

pytestmark = pytest.mark.gpu

STATE = (("Position", 0), ("Velocity", 0), ("Director", 1), ("AngularVelocity", 1))


def check(sim, wl, steps):
    base, spread = B.oracle_spread_loads(wl, steps)
    bounds = B.parity_bounds(spread)
    want = B.state_slots(base)
    for name, place in STATE:
        err = B.max_rel_error_per_rod(sim.get_slots(name), want[name], wl.n_elements, place)
        assert err <= bounds[name], (name, float(err), bounds[name])
    return base


@pytest.mark.parametrize("reference_rounding", [False, True])
def test_hinge_chain_vs_oracle(reference_rounding):
    wl = W.hinge_chain(n_links=3, n_elements=10)
    sim = wl.build(reference_rounding=reference_rounding)
    sim.step(eb.PositionVerlet(), 0.0, wl.dt, 2000)
    assert sim.step_plan()["mode"] == "streaming"
    base = check(sim, wl, 2000)
    # the chain moved and stayed joined: the joint gap is small against the link
    x = sim.get_slots("Position")
    gap = np.linalg.norm(x[:, 11] - x[:, 10])
    assert 0.0 < gap < 1e-3 * 0.2
    assert np.all(np.isfinite(x))


def test_free_joints_several_on_one_node():
    rng = np.random.default_rng(5)
    n = 12
    rods = [eb.StraightRod(n_elements=n, material=eb.Material(1000.0, 1e6, 1e6 / 3), radius=0.01, length=0.15,
                           origin=tuple(rng.uniform(-0.02, 0.02, 3)), direction=tuple(d), normal=tuple(m))
            for d, m in [((1, 0, 0), (0, 1, 0)), ((0, 1, 0), (0, 0, 1)), ((0, 0, 1), (1, 0, 0)), ((-1, 0, 0), (0, 1, 0))]]
    vel = [rng.normal(0, 1e-2, (3, n + 1)) for _ in rods]
    joints = [(0, n - 1, 1, 0, eb.FreeJoint(2e3, -0.5)), (0, n - 1, 2, 0, eb.FreeJoint(1e3, 0.0)),
              (3, 3, 1, 5, eb.FreeJoint(5e2, -0.1)), (2, 0, 1, 0, eb.HingeJoint(1e3, 0.0, 20.0, (0.0, 1.0, 0.0)))]
    wl = W.Workload("joints", 0, rods, clamp=[True, False, False, False], damper=None,
                    gravity=(0.0, 0.0, -9.81), velocities=vel, dt=1e-5, connections=joints)
    sim = wl.build()
    sim.step(eb.PositionVerlet(), 0.0, wl.dt, 1500)
    check(sim, wl, 1500)


def test_connections_beside_contact():
    wl = W.contact_batch(n_rods=32, seed=21, box=0.25, dt=1e-7)
    n = wl.rods[0].n_elements
    wl.connections = [(0, n - 1, 1, 0, eb.FreeJoint(1e2, 0.0)), (2, 10, 3, 20, eb.HingeJoint(1e2, 0.0, 1.0,
                                                                                             (0.0, 0.0, 1.0)))]
    sim = wl.build()
    sim.step(eb.PositionVerlet(), 0.0, wl.dt, 10)
    check(sim, wl, 10)


def test_connect_argument_checks():
    rods = [eb.StraightRod(n_elements=5, material=eb.Material(1000.0, 1e6, 1e6 / 3), radius=0.01, length=0.1)
            for _ in range(2)]
    sim = eb.Simulator()
    a, b = sim.emplace_back_many(eb.CosseratRodWithoutDamping, rods)
    for ia, ib, joint, status in [(5, 0, eb.FreeJoint(1.0), 1), (-1, 0, eb.FreeJoint(1.0), 1),
                                  (4, 6, eb.FreeJoint(1.0), 1), (4, 5, eb.HingeJoint(1.0, 0.0, 1.0, (1, 0, 0)), 1),
                                  (4, 0, eb.FreeJoint(float("nan")), 1)]:
        with pytest.raises(L.EbError) as e:
            sim.connect(a, ia).to(b, ib).using(joint)
        assert e.value.status == status
    sim.connect(a, 4).to(b, 5).using(eb.FreeJoint(1.0))  # node 5 of rod b exists
    bad = eb.RodRef(sim, 7, 5)
    with pytest.raises(L.EbError) as e:
        sim.connect(a, 0).to(bad, 0).using(eb.FreeJoint(1.0))
    assert e.value.status == 6  # unknown rod
    sim.finalize()
    with pytest.raises(L.EbError) as e:
        sim.connect(a, 0).to(b, 0).using(eb.FreeJoint(1.0))
    assert e.value.status == 2  # after finalize
    sim.close()


@pytest.mark.parametrize("joint", ["free", "hinge"])
def test_joint_keeps_total_momentum_on_gpu(joint):
    """A pin of the joint rules that needs no reference value: the joint
    force acts equal and opposite on its two nodes (and the hinge torques
    are internal too), so two free, unloaded rods joined by a stretched
    joint keep their total linear momentum to rounding, while the joint
    moves them (the gap changes)."""
    import elasticapp_b200 as eb
    from test_oracle_connections import two_free_rods
    from elasticapp_b200.simulator import FreeJoint, HingeJoint

    rng = np.random.default_rng(7)
    v = [rng.normal(0, 1e-2, (3, 9)), rng.normal(0, 1e-2, (3, 9))]
    j = FreeJoint(1e3, 0.0) if joint == "free" else HingeJoint(1e3, 0.0, 1e-3, (0.0, 0.0, 1.0))
    wl = two_free_rods((0.01, 0.005, -0.002), j, v=v)
    sim = wl.build()
    m = np.concatenate([r.get("Mass") for r in sim.rods])

    def momentum():
        vel = np.concatenate([r.get("Velocity") for r in sim.rods], axis=1)
        return (vel * m[None, :]).sum(axis=1)

    p0 = momentum()
    x0 = sim.rods[1].get("Position")[:, 0] - sim.rods[0].get("Position")[:, -1]
    sim.step(eb.PositionVerlet(), 0.0, wl.dt, 2000)
    p1 = momentum()
    x1 = sim.rods[1].get("Position")[:, 0] - sim.rods[0].get("Position")[:, -1]
    scale = np.abs(v[0]).max() * m.sum()
    assert np.max(np.abs(p1 - p0)) <= 1e-12 * scale
    assert np.linalg.norm(x1 - x0) > 1e-6  # the joint acted
    sim.close()
