"""The oracle's analytical damper and energies against closed forms
(tests/analytic_cases.py), which pin them without the reference: the
reference holds no damper or energy values to compare against."""
import numpy as np
import pytest

import analytic_cases as A
from oracle_bridge import oracle_from_workload


@pytest.fixture(scope="module")
def eb():
    import elasticapp_b200
    return elasticapp_b200


def _workload(eb, damper=None):
    from elasticapp_b200.workloads import Workload
    return Workload("analytic", 0, [A.straight_rod(eb)], clamp=False, damper=damper, gravity=None, dt=A.DT)


def test_oracle_damper_decays_as_closed_form(eb, oracle_mod):
    orc = oracle_from_workload(_workload(eb, damper=(A.NU_T, A.NU_R)))
    orc.set_rod("v", 0, A.translating_velocity())
    orc.set_rod("w", 0, A.spinning_omega())
    for k in (1, 10, A.STEPS):
        orc.step(A.DT, k if k == 1 else k - done)
        done = k
        v = orc.get_rod("v", 0, A.N + 1)
        w = orc.get_rod("w", 0, A.N)
        # rounding of k multiplications and of the factors: a few ulp a step
        tol = 8.0 * k * np.finfo(float).eps
        assert A.rel(v, np.repeat(A.damped_velocity(k)[:, None], A.N + 1, axis=1)) <= tol
        assert A.rel(w[2], np.full(A.N, A.damped_spin(k))) <= tol
        # the loads are exactly zero: nothing else moves
        assert np.max(np.abs(w[:2])) == 0.0 and np.max(np.abs(v[0])) == 0.0


def test_oracle_energies_after_damped_steps(eb, oracle_mod):
    """Energies follow the damper: translational by exp(-nu_t dt)^(2k),
    rotational by exp(-nu_r (2 / r^2) dt)^(2k); the elastic ones stay 0."""
    orc = oracle_from_workload(_workload(eb, damper=(A.NU_T, A.NU_R)))
    orc.set_rod("v", 0, A.translating_velocity())
    orc.set_rod("w", 0, A.spinning_omega())
    orc.step(A.DT, A.STEPS)
    et, er, es, eb_ = orc.energy()[0]
    k = A.STEPS
    assert abs(et - A.translational_energy() * np.exp(-A.NU_T * A.DT) ** (2 * k)) <= 1e-13 * et
    assert abs(er - A.rotational_energy() * (A.damped_spin(k) / A.W0) ** 2) <= 1e-13 * er
    assert es == 0.0 and eb_ == 0.0


def test_oracle_energies_equal_closed_forms(eb, oracle_mod):
    wl = _workload(eb)
    orc = oracle_from_workload(wl)
    orc.set_rod("v", 0, A.translating_velocity())
    orc.set_rod("w", 0, A.spinning_omega())
    et, er, es, eb_ = orc.energy()[0]
    assert abs(et - A.translational_energy()) <= 1e-14 * A.translational_energy()
    assert abs(er - A.rotational_energy()) <= 1e-14 * A.rotational_energy()
    assert es == 0.0 and eb_ == 0.0  # unstrained, unbent
    st = oracle_from_workload(wl)
    st.set_rod("x", 0, A.stretched_positions())
    assert abs(st.energy()[0][2] - A.shear_energy()) <= 1e-10 * A.shear_energy()
    bt = oracle_from_workload(wl)
    bt.set_rod("Q", 0, A.bent_directors().reshape(9, A.N))
    assert abs(bt.energy()[0][3] - A.bend_energy()) <= 1e-9 * A.bend_energy()


def test_oracle_velocity_verlet_damps_after_both_kicks(eb, oracle_mod):
    """VelocityVerlet applies the rate constraints after each of its two
    dynamic substeps, and the damper's constants hold the full dt
    (AnalyticalLinearDamper.hpp:15-79): exp(-nu dt) twice a step."""
    orc = oracle_from_workload(_workload(eb, damper=(A.NU_T, A.NU_R)))
    orc.set_rod("v", 0, A.translating_velocity())
    orc.set_rod("w", 0, A.spinning_omega())
    k = 50
    orc.step(A.DT, k, stepper="velocity_verlet")
    tol = 16.0 * k * np.finfo(float).eps
    v, w = orc.get_rod("v", 0, A.N + 1), orc.get_rod("w", 0, A.N)
    assert A.rel(v, np.repeat(A.damped_velocity(2 * k)[:, None], A.N + 1, axis=1)) <= tol
    assert A.rel(w[2], np.full(A.N, A.damped_spin(2 * k))) <= tol
    assert np.max(np.abs(w[:2])) == 0.0 and np.max(np.abs(v[0])) == 0.0
