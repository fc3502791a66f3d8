"""Case-study layer on the CPU: parameters, iteration counting of run_for,
fused versus per-step runs, and the write-back of rod views (with a stub
simulator; the GPU tests run the real one)."""
import numpy as np
import pytest

from elasticapp_b200 import case_study as C


class StubSim:
    def __init__(self):
        self.calls = []
        self.state = {"Position": np.zeros((3, 5)), "Velocity": np.zeros((3, 5))}
        self.sets = []

    def step(self, stepper, t, dt, n):
        self.calls.append(n)
        return t + n * dt

    def energy(self):
        return np.array([[1.0, 2.0, 3.0, 4.0]])

    def close(self):
        pass


class StubRef:
    def __init__(self, sim):
        self.sim, self.id, self.n_elements = sim, 0, 4

    def get(self, name):
        return self.sim.state[name].copy()

    def set(self, name, values):
        self.sim.sets.append(name)
        self.sim.state[name] = np.array(values)


class Toy(C.CaseStudy):
    parameters = (C.Parameter("n", int, 4, "elements"),
                  C.Parameter("dt", float, lambda p: 0.5 / p.n, "time step"))

    def setup(self, params):
        self.simulator = StubSim()
        self.set_dt(params.dt)
        self.rod = self.view(StubRef(self.simulator))

    def communicate(self):
        return self.rod


class ToyPerStep(Toy):
    def step(self):
        self._advance(1)


def test_parameters_defaults_and_errors():
    p = Toy.make_params()
    assert p.n == 4 and p.dt == 0.125
    p = Toy.make_params(n=10)
    assert p.dt == 0.05  # dependent default
    with pytest.raises(TypeError):
        Toy.make_params(m=3)
    d = C.DynamicCantileverCaseStudy.make_params()
    assert (d.n_elements, d.youngs_modulus, d.density, d.radius, d.length) == (100, 1e5, 2000.0, 0.02, 1.0)
    assert d.shear_modulus == pytest.approx(1e5 / 3) and d.dt == pytest.approx(5e-4)
    assert "Youngs modulus" in C.DynamicCantileverCaseStudy.parameter_help()


def test_multiple_just_greater_than():
    assert C.multiple_just_greater_than(1.0, 0.1) == 10
    assert C.multiple_just_greater_than(0.25, 0.1) == 3
    assert C.multiple_just_greater_than(0.3, 0.1) == 3  # 0.3 / 0.1 rounds above 3
    assert C.multiple_just_greater_than(1e-15, 0.1) == 0


def test_run_for_counts_and_fuses():
    cs = Toy()
    cs.run_for(additional_time=1.0)  # 8 iterations of 0.125
    assert cs.simulator.calls == [8] and cs.current_iteration() == 8
    assert cs.current_time() == pytest.approx(1.0)
    cs.run_for(n_iterations=3)
    cs.run_for_n_iterations(0)
    assert cs.simulator.calls == [8, 3] and cs.current_iteration() == 11
    cs.step_with(0.25)
    assert cs.current_dt() == 0.25 and cs.simulator.calls[-1] == 1
    with pytest.raises(TypeError):
        cs.run_for(additional_time=1.0, n_iterations=2)
    with pytest.raises(TypeError):
        cs.run_for()
    cs.set_current_time(3.0)
    assert cs.current_time() == 3.0
    cs.reset()
    assert cs.current_time() == 0.0 and cs.current_iteration() == 0 and cs.simulator.calls == []
    # an overridden step runs once per iteration
    ps = ToyPerStep()
    ps.run_for(n_iterations=4)
    assert ps.simulator.calls == [1, 1, 1, 1]


def test_view_writes_back_changed_arrays_only():
    cs = Toy()
    rod = cs.communicate()
    v = np.asarray(rod.loc[rod.Velocity])
    assert rod.Velocity == "Velocity" and v.shape == (3, 5)
    _ = rod.position_collection  # read, unchanged
    v[2, :] = 7.0
    cs.step()
    assert cs.simulator.sets == ["Velocity"]
    assert np.all(cs.simulator.state["Velocity"][2] == 7.0)
    # after a step the view reads the device again
    assert np.all(rod.get_velocity()[2] == 7.0)
    assert rod.compute_bending_energy() == 4.0 and rod.compute_translational_energy() == 1.0
    assert rod.n_elems == 4 and len(rod) == 4
    with pytest.raises(AttributeError):
        rod.no_such_thing
