"""The GPU's analytical damper and energies against closed forms
(tests/analytic_cases.py), through the C-ABI, on every FP64 plan and both
FP64 builds: the damper and the energies are pinned without the oracle."""
import numpy as np
import pytest

import analytic_cases as A

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eb():
    import elasticapp_b200
    return elasticapp_b200


def _sim(eb, damper=None, **kw):
    from elasticapp_b200.workloads import Workload
    wl = Workload("analytic", 0, [A.straight_rod(eb)], clamp=False, damper=damper, gravity=None, dt=A.DT)
    return wl.build(**kw)


@pytest.mark.parametrize("kw", [{"step_mode": "streaming"}, {"step_mode": "streaming", "reference_rounding": True},
                                {"step_mode": "resident"}, {"step_mode": "streaming", "cuda_graph": True}],
                         ids=["streaming", "streaming-reference-rounding", "resident", "graph"])
def test_damper_decays_as_closed_form(eb, kw):
    sim = _sim(eb, damper=(A.NU_T, A.NU_R), **kw)
    rod = sim.rods[0]
    rod.set("Velocity", A.translating_velocity())
    rod.set("AngularVelocity", A.spinning_omega())
    t, done = 0.0, 0
    eps = np.finfo(float).eps
    for k in (1, 10, A.STEPS):
        t = sim.step(eb.PositionVerlet(), t, A.DT, k - done)
        done = k
        v, w = rod.get("Velocity"), rod.get("AngularVelocity")
        tol = 8.0 * k * eps
        # the fast build forms the tangent as dx * (1 / l), which can be one
        # ulp off unit length: the end elements then carry a strain of eps,
        # whose unbalanced load E A eps on the end nodes (mass rho A l0 / 2)
        # moves v by 2 E eps dt / (rho l0 |v0|) relative a step
        tol_v = tol if kw.get("reference_rounding") else \
            4.0 * (tol + k * 2.0 * A.YOUNGS * eps * A.DT / (A.DENSITY * A.L0 * np.linalg.norm(A.V0)))
        assert A.rel(v, np.repeat(A.damped_velocity(k)[:, None], A.N + 1, axis=1)) <= tol_v, (k, kw)
        assert A.rel(w[2], np.full(A.N, A.damped_spin(k))) <= tol, (k, kw)
        # the loads are zero up to the rounding of contracted multiply-adds
        assert np.max(np.abs(w[:2])) <= 1e-12 * A.W0 and np.max(np.abs(v[0])) <= 1e-12
    et, er, es, eb_ = sim.energy()[0]
    assert abs(et - A.translational_energy() * np.exp(-A.NU_T * A.DT) ** (2 * A.STEPS)) <= 1e-13 * et
    assert abs(er - A.rotational_energy() * (A.damped_spin(A.STEPS) / A.W0) ** 2) <= 1e-13 * er
    sim.close()


def test_mixed_precision_damper_within_its_tolerance(eb):
    sim = _sim(eb, damper=(A.NU_T, A.NU_R), precision="mixed")
    rod = sim.rods[0]
    rod.set("Velocity", A.translating_velocity())
    rod.set("AngularVelocity", A.spinning_omega())
    sim.step(eb.PositionVerlet(), 0.0, A.DT, A.STEPS)
    v, w = rod.get("Velocity"), rod.get("AngularVelocity")
    # the damping factors are rounded to FP32 (the same rounding every
    # step): at most one FP32 ulp (2^-23 relative) a step, k steps
    tol = A.STEPS * 2.0 ** -23
    assert A.rel(v, np.repeat(A.damped_velocity(A.STEPS)[:, None], A.N + 1, axis=1)) <= tol
    assert A.rel(w[2], np.full(A.N, A.damped_spin(A.STEPS))) <= tol
    sim.close()


def test_energies_equal_closed_forms(eb):
    sim = _sim(eb)
    rod = sim.rods[0]
    rod.set("Velocity", A.translating_velocity())
    rod.set("AngularVelocity", A.spinning_omega())
    et, er, es, eb_ = sim.energy()[0]
    assert abs(et - A.translational_energy()) <= 1e-13 * A.translational_energy()
    assert abs(er - A.rotational_energy()) <= 1e-13 * A.rotational_energy()
    assert abs(es) <= 1e-25 and abs(eb_) <= 1e-25
    sim.close()
    st = _sim(eb)
    st.rods[0].set("Position", A.stretched_positions())
    assert abs(st.energy()[0][2] - A.shear_energy()) <= 1e-10 * A.shear_energy()
    st.close()
    bt = _sim(eb)
    bt.rods[0].set("Director", A.bent_directors())
    assert abs(bt.energy()[0][3] - A.bend_energy()) <= 1e-9 * A.bend_energy()
    bt.close()
