"""The dynamic cantilever case study on the GPU: the caller sets a modal
initial velocity through communicate(), runs in time spans, and the tip
follows the oracle run from the same initial state (FP64 parity); fused and
chunked runs agree bit for bit; reset restores the initial state."""
import numpy as np
import pytest

import elasticapp_b200 as eb
from elasticapp_b200 import case_study as C
from elasticapp_b200 import workloads as W

from oracle_bridge import oracle_from_workload

pytestmark = pytest.mark.gpu


def first_mode_profile(x, length, amplitude=1e-3):
    # shape of the first clamped-free bending mode (Euler-Bernoulli)
    b = 1.875104068711961 / length
    s = (np.cosh(b * length) + np.cos(b * length)) / (np.sinh(b * length) + np.sin(b * length))
    return amplitude * (np.cosh(b * x) - np.cos(b * x) - s * (np.sinh(b * x) - np.sin(b * x)))


def test_cantilever_case_study_against_oracle():
    cs = C.DynamicCantileverCaseStudy(n_elements=50)
    rod = cs.communicate()
    x0 = np.copy(rod.position_collection)[0, :]
    v = np.asarray(rod.loc[rod.Velocity])
    v[2, :] = first_mode_profile(x0, cs.params.length)
    assert cs.current_dt() == pytest.approx(0.05 * 1.0 / 50)
    tips, times = [], []
    for _ in range(5):
        cs.run_for(additional_time=50 * cs.current_dt())
        tips.append(np.asarray(rod.get_position())[:, -1].copy())
        times.append(cs.current_time())
    assert cs.current_iteration() == 250
    assert times[-1] == pytest.approx(250 * cs.current_dt(), rel=1e-12)
    p = cs.params
    wl = W.Workload("cantilever_case", 0, [eb.StraightRod(
        n_elements=p.n_elements, material=eb.Material(p.density, p.youngs_modulus, p.shear_modulus),
        radius=p.radius, length=p.length, origin=(0.0, 0.0, 0.0), direction=(1.0, 0.0, 0.0),
        normal=(0.0, 1.0, 0.0))], clamp=True, damper=None, gravity=None,
        velocities=[np.vstack([np.zeros_like(x0), np.zeros_like(x0), first_mode_profile(x0, p.length)])],
        dt=cs.current_dt())
    orc = oracle_from_workload(wl)
    for k in range(5):
        orc.step(cs.current_dt(), 50)
        tip = orc.get_rod("x", 0, p.n_elements + 1)[:, -1]
        assert np.linalg.norm(tips[k] - tip) / p.length <= 1e-10, k
    # the tip moved (the mode is excited) and energy is held
    assert abs(tips[-1][2]) > 0.0
    e = [rod.compute_translational_energy(), rod.compute_rotational_energy(), rod.compute_shearing_energy(),
         rod.compute_bending_energy()]
    assert all(np.isfinite(e)) and e[0] + e[3] > 0.0
    cs.close()


def test_fused_and_chunked_runs_agree_and_reset():
    a = C.DynamicCantileverCaseStudy(n_elements=40)
    b = C.DynamicCantileverCaseStudy(n_elements=40)
    for cs in (a, b):
        rod = cs.communicate()
        x0 = np.copy(rod.position_collection)[0, :]
        rod.loc[rod.Velocity][2, :] = first_mode_profile(x0, 1.0)
    p0 = a.communicate().get_position().copy()
    a.run_for(n_iterations=300)
    for _ in range(3):
        b.run_for_n_iterations(100)
    assert np.array_equal(a.communicate().get_position(), b.communicate().get_position())
    assert np.array_equal(a.communicate().get_director(), b.communicate().get_director())
    a.reset()
    assert a.current_iteration() == 0 and a.current_time() == 0.0
    np.testing.assert_array_equal(a.communicate().get_position()[0], p0[0])
    assert np.all(a.communicate().get_velocity() == 0.0)
    a.close()
    b.close()
