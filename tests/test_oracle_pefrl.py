"""PEFRL and VelocityVerlet in the oracle.  The reference declares PEFRL
without an implementation, so there is no golden vector: the checks are its
order of accuracy (error ratio about 16 per halving of dt for a
fourth-order method, 4 for PositionVerlet and VelocityVerlet) on free,
undamped rods, where no first-order constraint splitting masks it."""
import numpy as np
import pytest

from oracle_bridge import oracle_from_workload


def _free_batch():
    from elasticapp_b200 import workloads as W
    wl = W.uneven_batch(n_rods=4, seed=3, n_range=(20, 40))
    wl.damper = None
    wl.clamp = False
    return wl


def _positions(wl, stepper, factor, horizon):
    R = oracle_from_workload(wl)
    dt = wl.dt * factor
    R.step(dt, int(round(horizon / dt)), stepper=stepper)
    return R.comp("x").copy()


@pytest.mark.parametrize("stepper,order,factors", [("position_verlet", 2, (2.0, 1.0, 0.5)),
                                                   ("velocity_verlet", 2, (2.0, 1.0, 0.5)),
                                                   ("pefrl", 4, (4.0, 2.0, 1.0))])
def test_order_of_accuracy(stepper, order, factors):
    wl = _free_batch()
    horizon = 800 * wl.dt
    ref = _positions(wl, stepper, factors[2] / 4, horizon)
    err = [np.abs(_positions(wl, stepper, f, horizon) - ref).max() for f in factors]
    ratios = [err[0] / err[1], err[1] / err[2]]
    expect = 2.0 ** order
    assert all(0.6 * expect < r < 1.6 * expect for r in ratios), (err, ratios)


def test_pefrl_more_accurate_than_verlet_at_equal_cost():
    # PEFRL spends four force evaluations a step: compare at 4x the step
    wl = _free_batch()
    horizon = 800 * wl.dt
    ref = _positions(wl, "pefrl", 0.25, horizon)
    e_pv = np.abs(_positions(wl, "position_verlet", 1.0, horizon) - ref).max()
    e_pe = np.abs(_positions(wl, "pefrl", 4.0, horizon) - ref).max()
    assert e_pe < e_pv


def test_velocity_and_position_verlet_agree_to_second_order():
    """Both second-order schemes approach the same trajectory: their
    difference shrinks about 4x per halving of dt."""
    wl = _free_batch()
    horizon = 800 * wl.dt
    d = [np.abs(_positions(wl, "velocity_verlet", f, horizon) - _positions(wl, "position_verlet", f, horizon)).max()
         for f in (1.0, 0.5)]
    assert 2.4 < d[0] / d[1] < 6.4, d
