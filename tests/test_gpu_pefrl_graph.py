"""PEFRL and CUDA-graph replay on the GPU.

* PEFRL on the streaming kernel (four launches a step) and on the resident
  kernel (four force evaluations a step on chip) against the oracle's PEFRL
  (the reference declares the stepper without implementing it): the FP64
  parity rule after 200 steps with clamp, damper and gravity, and
  fourth-order convergence on free rods.
* Steps replayed from a captured CUDA graph give bit-identical states to
  the same steps launched one by one, for PositionVerlet and PEFRL, with a
  recorded last step, and after a change of dt (a new capture).
"""
import numpy as np
import pytest

from oracle_bridge import max_rel_error_per_rod, oracle_from_workload, oracle_spread, parity_bounds, state_slots

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eb():
    import elasticapp_b200
    return elasticapp_b200


@pytest.fixture(scope="module")
def W():
    from elasticapp_b200 import workloads
    return workloads


@pytest.mark.parametrize("step_mode", ["streaming", "resident"])
def test_pefrl_parity_with_oracle(eb, W, step_mode):
    wl = W.uneven_batch(n_rods=12, seed=7, n_range=(20, 90))
    steps = 200
    base, spread = oracle_spread(wl, steps, stepper="pefrl")
    bounds = parity_bounds(spread)
    sim = wl.build(stepper=eb.PEFRL(), step_mode=step_mode)
    sim.step(eb.PEFRL(), 0.0, wl.dt, steps)
    want = state_slots(base)
    for name, place in (("Position", 0), ("Velocity", 0), ("Director", 1), ("AngularVelocity", 1)):
        err = max_rel_error_per_rod(sim.get_slots(name), want[name], wl.n_elements, place)
        assert err <= bounds[name], (name, err, bounds[name])
    assert sim.step_plan()["mode"] == step_mode
    sim.close()


def test_pefrl_resident_long_rods_and_chunks(eb, W):
    """PEFRL on the bucketed resident plan (rods on CTA pairs included), in
    chunks that split launches differently, against the streaming kernel."""
    wl = W.uneven_batch(n_rods=6, seed=12, n_range=(100, 900))
    a = wl.build(stepper=eb.PEFRL(), step_mode="bucketed")
    b = wl.build(stepper=eb.PEFRL(), step_mode="bucketed")
    ref = wl.build(stepper=eb.PEFRL(), step_mode="streaming")
    a.step(eb.PEFRL(), 0.0, wl.dt, 300)
    for k in (130, 170):
        b.step(eb.PEFRL(), 0.0, wl.dt, k)
    ref.step(eb.PEFRL(), 0.0, wl.dt, 300)
    assert a.step_plan()["mode"] == "bucketed"
    for name in ("Position", "Director", "Velocity", "AngularVelocity"):
        assert np.array_equal(a.get_slots(name), b.get_slots(name)), name
    for name in ("Position", "Director"):
        x, y = a.get_slots(name), ref.get_slots(name)
        assert np.max(np.abs(x - y)) <= 1e-10 * max(1.0, np.max(np.abs(y))), name
    for s in (a, b, ref):
        s.close()


@pytest.mark.parametrize("step_mode", ["streaming", "resident"])
def test_pefrl_fourth_order_on_gpu(eb, W, step_mode):
    wl = W.uneven_batch(n_rods=4, seed=3, n_range=(20, 40))
    wl.damper = None
    wl.clamp = False
    horizon = 800 * wl.dt

    def run(f):
        sim = wl.build(stepper=eb.PEFRL(), step_mode=step_mode)
        dt = wl.dt * f
        sim.step(eb.PEFRL(), 0.0, dt, int(round(horizon / dt)))
        x = sim.get_slots("Position").copy()
        sim.close()
        return x

    ref = run(0.25)
    err = [np.abs(run(f) - ref).max() for f in (4.0, 2.0, 1.0)]
    ratios = [err[0] / err[1], err[1] / err[2]]
    assert all(9.6 < r < 25.6 for r in ratios), (err, ratios)


def test_pefrl_rejects_mixed_precision_and_wrong_stepper(eb, W):
    from elasticapp_b200._lib import EbError
    wl = W.uneven_batch(n_rods=2, seed=1, n_range=(20, 30))
    with pytest.raises(EbError):
        wl.build(precision="mixed", stepper=eb.PEFRL())
    sim = wl.build(stepper=eb.PEFRL())
    with pytest.raises(TypeError):
        sim.step(eb.PositionVerlet(), 0.0, wl.dt, 1)
    sim.close()


@pytest.mark.parametrize("stepper", ["verlet", "pefrl"])
def test_cuda_graph_replay_is_bit_identical(eb, W, stepper):
    wl = W.uneven_batch(n_rods=16, seed=9, n_range=(20, 200))
    st = eb.PEFRL() if stepper == "pefrl" else eb.PositionVerlet()
    out = []
    for graph in (False, True):
        sim = wl.build(step_mode="streaming", stepper=st, cuda_graph=graph, record_diagnostics=True)
        t = sim.step(st, 0.0, wl.dt, 70)        # two graphs + 6 single steps (last one recorded)
        t = sim.step(st, t, 0.5 * wl.dt, 33)     # a new dt: a new capture
        t = sim.step(st, t, wl.dt, 64)           # back to the first dt, other buffer parity
        out.append({n: sim.get_slots(n).copy() for n in ("Position", "Velocity", "Director", "AngularVelocity",
                                                         "Curvature")})
        sim.close()
    for n in out[0]:
        np.testing.assert_array_equal(out[0][n], out[1][n])
