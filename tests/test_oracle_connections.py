"""The CPU restatement of the connections (joints) between rods.

No test of the reference exercises a connection (its joints are written per
case study; examples/hinge_joint/HingeJointCaseStudy.cpp:96-150 is the one
the built-in joints restate), so this is checked by the physics: equal and
opposite joint forces keep the total linear momentum of free rods, a free
joint without damping keeps the mechanical energy of the spring plus the
rods (to the integrator's error), the dashpot term changes it with the sign
the example's rule gives it (-nu ((v_b - v_a) . u) u added to rod a: a
negative nu dissipates, a positive one feeds a separating pair), coincident nodes
(d = 0) give no force, the hinge spring straightens a bent joint, the order
of connections acting on one node does not change the sum beyond rounding,
and out-of-range indices are rejected."""
import numpy as np
import pytest

import oracle
import oracle_bridge as B
from elasticapp_b200 import workloads as W
from elasticapp_b200.simulator import FreeJoint, HingeJoint, Material, StraightRod


def two_free_rods(gap, joint, v=None, n=8):
    rods = [StraightRod(n_elements=n, material=Material(1000.0, 1e6, 1e6 / 3), radius=0.01, length=0.2,
                        origin=(0.0, 0.0, 0.0), direction=(1.0, 0.0, 0.0), normal=(0.0, 1.0, 0.0)),
            StraightRod(n_elements=n, material=Material(1000.0, 1e6, 1e6 / 3), radius=0.01, length=0.2,
                        origin=(0.2 + gap[0], gap[1], gap[2]), direction=(1.0, 0.0, 0.0), normal=(0.0, 1.0, 0.0))]
    return W.Workload("joint", 0, rods, clamp=False, damper=None, gravity=None, velocities=v, dt=1e-5,
                      connections=[(0, n - 1, 1, 0, joint)])


def run(wl, n_steps):
    r = B.oracle_from_workload(wl)
    B.loads_step(r, wl, n_steps)
    return r


def momentum(r, wl):
    m = r.arrays["mass"][: r.n_slots]
    v = r.comp("v")
    return (v * m[None, :]).sum(axis=1)


def energy(r, wl):
    e = r.energy().sum()
    j = wl.connections[0][4]
    n = wl.rods[0].n_elements
    x = r.comp("x")
    d = x[:, n + 1] - x[:, n]  # rod b's node 0 minus rod a's node n
    return e + 0.5 * j.stiffness * float(d @ d)


def test_coincident_nodes_give_no_force():
    wl = two_free_rods((0.0, 0.0, 0.0), FreeJoint(1e4, 5.0))
    r = run(wl, 50)
    # no initial velocity, no loads: nothing moves
    assert np.all(r.comp("v") == 0.0)


def test_momentum_kept_and_spring_energy_exchanged():
    rng = np.random.default_rng(1)
    v = [rng.normal(0, 1e-2, (3, 9)), rng.normal(0, 1e-2, (3, 9))]
    wl = two_free_rods((0.01, 0.005, -0.002), FreeJoint(1e3, 0.0), v=v)
    r0 = B.oracle_from_workload(wl)
    p0, e0 = momentum(r0, wl), energy(r0, wl)
    r = run(wl, 2000)
    p1, e1 = momentum(r, wl), energy(r, wl)
    scale = np.abs(v[0]).max() * r0.arrays["mass"][: r0.n_slots].sum()
    assert np.max(np.abs(p1 - p0)) <= 1e-12 * scale
    # the gap closes (the spring pulls the nodes together) and energy is held
    x = r.comp("x")
    assert np.linalg.norm(x[:, 9] - x[:, 8]) != pytest.approx(np.linalg.norm([0.01, 0.005, -0.002]))
    assert abs(e1 - e0) <= 2e-3 * e0


def test_dashpot_sign_of_the_reference_rule():
    rng = np.random.default_rng(2)
    v = [np.zeros((3, 9)), rng.normal(0, 1e-1, (3, 9))]
    e = {}
    for nu in (-0.05, 0.0, 0.05):
        wl = two_free_rods((0.005, 0.0, 0.0), FreeJoint(1e3, nu), v=v)
        e[nu] = energy(run(wl, 1000), wl)
    assert e[-0.05] < e[0.0] < e[0.05]


def test_hinge_spring_straightens_the_joint():
    # rod b starts tilted about the hinge normal's perpendicular: its first
    # element has a component along the normal, which the spring removes
    n = 8
    rods = [StraightRod(n_elements=n, material=Material(1000.0, 1e6, 1e6 / 3), radius=0.01, length=0.2,
                        origin=(0.0, 0.0, 0.0), direction=(0.0, 0.0, 1.0), normal=(0.0, 1.0, 0.0)),
            StraightRod(n_elements=n, material=Material(1000.0, 1e6, 1e6 / 3), radius=0.01, length=0.2,
                        origin=(0.0, 0.0, 0.2), direction=(np.sin(0.2), 0.0, np.cos(0.2)), normal=(0.0, 1.0, 0.0))]
    def tilt(joint):
        wl = W.Workload("hinge", 0, rods, clamp=[True, False], damper=(2.0, 2.0), gravity=None, dt=1e-5,
                        connections=[(0, n - 1, 1, 0, joint)])
        r = run(wl, 4000)
        x = r.comp("x")
        l = x[:, n + 2] - x[:, n + 1]
        return abs(l[0]) / np.linalg.norm(l)
    assert tilt(HingeJoint(1e4, 0.0, 5e3, (1.0, 0.0, 0.0))) < 0.5 * tilt(FreeJoint(1e4, 0.0))


def test_connection_order_changes_only_rounding():
    rng = np.random.default_rng(3)
    n = 6
    rods = [StraightRod(n_elements=n, material=Material(1000.0, 1e6, 1e6 / 3), radius=0.01, length=0.1,
                        origin=tuple(rng.uniform(-0.05, 0.05, 3)), direction=(1.0, 0.0, 0.0), normal=(0.0, 1.0, 0.0))
            for _ in range(3)]
    c = [(0, n - 1, 1, 0, FreeJoint(1e3, 0.5)), (0, n - 1, 2, 0, FreeJoint(2e3, 0.1))]
    a = run(W.Workload("o", 0, rods, clamp=False, damper=None, gravity=None, dt=1e-5, connections=c), 200)
    b = run(W.Workload("o", 0, rods, clamp=False, damper=None, gravity=None, dt=1e-5, connections=c[::-1]), 200)
    xa, xb = a.comp("x"), b.comp("x")
    assert np.max(np.abs(xa - xb)) <= 1e-13 * np.max(np.abs(xa))


def test_invalid_connections_rejected():
    wl = two_free_rods((0.0, 0.0, 0.0), FreeJoint(1.0))
    r = B.oracle_from_workload(wl)
    for bad in [(0, 8, 1, 0, 0), (0, 7, 1, 9, 0), (0, 7, 1, 8, 1), (2, 0, 1, 0, 0)]:
        spec = oracle.ConnectionSpec([bad + (1.0, 0.0, 0.0, (1.0, 0.0, 0.0))])
        with pytest.raises(RuntimeError):
            oracle.loads_step(r, None, spec, 1e-5, 1)
