"""VelocityVerlet on the GPU (the reference's second symplectic stepper,
elastica/Time/SymplecticSteppers/Algorithms/VelocityVerlet.hpp:49-87): two
launches of the streaming kernel a step (kick dt/2 then drift dt; kick dt/2),
or two force evaluations a step on chip in the resident kernels.

* Parity with the oracle's VelocityVerlet after 300 steps with clamp,
  analytical damper and gravity, in both FP64 builds (the FP64 parity rule).
* Second-order convergence on free rods.
* The damper acts after both kicks with its full-dt factors: the closed
  form of a translating, spinning free rod (tests/analytic_cases.py).
* Graph replay is bit-identical to single launches.
"""
import numpy as np
import pytest

import analytic_cases as A
from oracle_bridge import max_rel_error_per_rod, oracle_spread, parity_bounds, state_slots

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eb():
    import elasticapp_b200
    return elasticapp_b200


@pytest.fixture(scope="module")
def W():
    from elasticapp_b200 import workloads
    return workloads


@pytest.mark.parametrize("kw", [{"step_mode": "streaming"}, {"step_mode": "streaming", "reference_rounding": True},
                                {"step_mode": "resident"}, {"step_mode": "bucketed"}],
                         ids=["streaming", "reference-rounding", "resident", "bucketed"])
def test_velocity_verlet_parity_with_oracle(eb, W, kw):
    wl = W.uneven_batch(n_rods=12, seed=17, n_range=(20, 700))
    steps = 300
    base, spread = oracle_spread(wl, steps, stepper="velocity_verlet")
    bounds = parity_bounds(spread)
    sim = wl.build(stepper=eb.VelocityVerlet(), **kw)
    t = sim.step(eb.VelocityVerlet(), 0.0, wl.dt, steps)
    assert t == pytest.approx(steps * wl.dt, rel=1e-12)
    # rods of more than 519 elements fit no whole-batch resident
    # configuration: a resident request then runs the per-size-bucket plan
    want_mode = {"resident": ("resident", "bucketed")}.get(kw["step_mode"], (kw["step_mode"],))
    assert sim.step_plan()["mode"] in want_mode
    want = state_slots(base)
    for name, place in (("Position", 0), ("Velocity", 0), ("Director", 1), ("AngularVelocity", 1)):
        err = max_rel_error_per_rod(sim.get_slots(name), want[name], wl.n_elements, place)
        assert err <= bounds[name], (name, err, bounds[name], kw)
    if kw["step_mode"] == "streaming":
        assert sim.launch_count() == 2 * steps
    sim.close()


def test_velocity_verlet_second_order_on_gpu(eb, W):
    wl = W.uneven_batch(n_rods=4, seed=3, n_range=(20, 40))
    wl.damper = None
    wl.clamp = False
    horizon = 800 * wl.dt

    def run(f):
        sim = wl.build(stepper=eb.VelocityVerlet())
        dt = wl.dt * f
        sim.step(eb.VelocityVerlet(), 0.0, dt, int(round(horizon / dt)))
        x = sim.get_slots("Position").copy()
        sim.close()
        return x

    ref = run(0.125)
    err = [np.abs(run(f) - ref).max() for f in (2.0, 1.0, 0.5)]
    ratios = [err[0] / err[1], err[1] / err[2]]
    assert all(2.4 < r < 6.4 for r in ratios), (err, ratios)


@pytest.mark.parametrize("step_mode", ["streaming", "resident"])
def test_velocity_verlet_damper_after_both_kicks(eb, step_mode):
    from elasticapp_b200.workloads import Workload
    wl = Workload("analytic", 0, [A.straight_rod(eb)], clamp=False, damper=(A.NU_T, A.NU_R), gravity=None,
                  dt=A.DT)
    sim = wl.build(stepper=eb.VelocityVerlet(), step_mode=step_mode)
    rod = sim.rods[0]
    rod.set("Velocity", A.translating_velocity())
    rod.set("AngularVelocity", A.spinning_omega())
    k = 50
    sim.step(eb.VelocityVerlet(), 0.0, A.DT, k)
    eps = np.finfo(float).eps
    tol = 16.0 * k * eps
    # rounding-level end loads of the fast build (see test_gpu_analytic_pins)
    tol_v = 4.0 * (tol + 2 * k * 2.0 * A.YOUNGS * eps * A.DT / (A.DENSITY * A.L0 * np.linalg.norm(A.V0)))
    v, w = rod.get("Velocity"), rod.get("AngularVelocity")
    assert A.rel(v, np.repeat(A.damped_velocity(2 * k)[:, None], A.N + 1, axis=1)) <= tol_v
    assert A.rel(w[2], np.full(A.N, A.damped_spin(2 * k))) <= tol
    sim.close()


def test_velocity_verlet_graph_replay_bit_identical(eb, W):
    wl = W.uneven_batch(n_rods=16, seed=9, n_range=(20, 200))
    st = eb.VelocityVerlet()
    out = []
    for graph in (False, True):
        sim = wl.build(step_mode="streaming", stepper=st, cuda_graph=graph)
        t = sim.step(st, 0.0, wl.dt, 70)
        t = sim.step(st, t, 0.5 * wl.dt, 33)
        out.append({n: sim.get_slots(n).copy() for n in ("Position", "Velocity", "Director", "AngularVelocity")})
        sim.close()
    for n in out[0]:
        np.testing.assert_array_equal(out[0][n], out[1][n])


def test_velocity_verlet_rejects_mixed_precision(eb, W):
    from elasticapp_b200._lib import EbError
    wl = W.uneven_batch(n_rods=2, seed=1, n_range=(20, 30))
    with pytest.raises(EbError):
        wl.build(precision="mixed", stepper=eb.VelocityVerlet())
