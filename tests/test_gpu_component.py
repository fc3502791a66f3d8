"""Internal loads and torques of uniformly strained rods on the GPU.

The pattern of the reference's elasticity component test
(``tests/Unit/Systems/CosseratRods/Components/Elasticity/Test_WithDiagonalLinearHyperElasticModel.cpp:183-249``):
a rod whose elements all carry the same strain has internal loads on its two
end nodes only, equal and opposite, and the same torque on every interior
element.  The rod is set through the C-ABI and stepped once from rest with
diagnostics recorded: the step's force evaluation follows a kinematic half
step that leaves positions and directors bit-identical when v and w are zero,
so its loads and torques are compared with the oracle's force evaluation of
the state that was set.
"""
import math

import numpy as np
import pytest

import elasticapp_b200 as eb

pytestmark = pytest.mark.gpu

N = 8


def _strained_state(oracle_mod, stretch, tilt):
    init = oracle_mod.straight_rod(N, (0.0, 0.0, 0.0), (0.0, 0.0, 1.0), (1.0, 0.0, 0.0), 1.0, 0.05, 1000.0,
                                   1e6, 1e6 / 3)
    x = init["x"] * stretch
    c, s = math.cos(tilt), math.sin(tilt)
    turn = np.array([[1.0, 0.0, 0.0], [0.0, c, s], [0.0, -s, c]])
    q = np.einsum("ab,bje->aje", turn, init["Q"])  # (director, component, element)
    return init, x, q


def _oracle_loads(oracle_mod, init, x, q):
    rods = oracle_mod.RodArrays([N])
    for key, src in (("mass", "mass"), ("rest_length", "l0"), ("rest_voronoi", "D0"), ("volume", "V"),
                     ("shear_diag", "S"), ("bend_diag", "B"), ("inertia_diag", "J"), ("inv_inertia", "Jinv")):
        rods.set_rod(key, 0, init[src])
    rods.set_rod("x", 0, x)
    rods.set_rod("Q", 0, q.reshape(9, N))
    rods.enable_diagnostics()
    rods.force_eval()
    return rods.get_diag("d_loads", 0, N + 1), rods.get_diag("d_torques", 0, N)


@pytest.mark.parametrize("reference_rounding", [False, True])
@pytest.mark.parametrize("stretch,tilt", [(1.125, 0.0), (1.0, 0.01), (1.125, 0.01)])
def test_strained_rod_loads_match_oracle(oracle_mod, stretch, tilt, reference_rounding):
    init, x, q = _strained_state(oracle_mod, stretch, tilt)
    want_f, want_t = _oracle_loads(oracle_mod, init, x, q)

    sim = eb.Simulator(record_diagnostics=True, reference_rounding=reference_rounding, step_mode="streaming")
    rod = sim.emplace_back(eb.CosseratRodWithoutDamping,
                           eb.StraightRod(n_elements=N, material=eb.Material(1000.0, 1e6, 1e6 / 3), radius=0.05,
                                          length=1.0, origin=(0.0, 0.0, 0.0), direction=(0.0, 0.0, 1.0),
                                          normal=(1.0, 0.0, 0.0)))
    sim.finalize()
    rod.set("Position", x.reshape(rod.shape("Position")))
    rod.set("Director", q.reshape(rod.shape("Director")))
    assert np.array_equal(rod.get("Position").reshape(3, N + 1), x)
    assert np.array_equal(rod.get("Director").reshape(3, 3, N), q)
    # the force evaluation of this step sees x and q unchanged (v = w = 0 in
    # the first kinematic half step); the diagnostics are recorded there
    sim.step(eb.PositionVerlet(), 0.0, 1e-6, 1)
    got_f = rod.get("InternalLoads").reshape(3, N + 1)
    got_t = rod.get("InternalTorques").reshape(3, N)

    scale_f = np.abs(want_f).max()
    scale_t = max(np.abs(want_t).max(), 1e-300)
    assert scale_f > 0.0
    assert np.abs(got_f - want_f).max() <= 1e-12 * scale_f
    assert np.abs(got_t - want_t).max() <= 1e-12 * scale_t + 1e-300
    # the component test's structure, on the GPU's own numbers
    assert np.abs(got_f[:, 1:N]).max() <= 1e-12 * scale_f
    assert np.abs(got_f[:, N] + got_f[:, 0]).max() <= 1e-12 * scale_f
    mid = got_t[:, 1]
    assert np.abs(got_t[:, 1:N - 1] - mid[:, None]).max() <= 1e-12 * scale_t + 1e-300
    sim.close()
