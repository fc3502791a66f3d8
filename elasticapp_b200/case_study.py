"""Case studies: the application layer above the simulator.

Mirrors the reference's case-study interface and its Python binding:

* ``CaseStudy`` — time, time step and iteration bookkeeping with ``step``,
  ``run_for(additional_time=...)`` / ``run_for(n_iterations=...)``,
  ``run_for_n_iterations``, ``step_with``, ``current_time``, ``current_dt``,
  ``current_iteration``, ``set_current_time``, ``reset`` and ``communicate``
  (elastica/Utilities/AppSupport/CaseStudyInterface.hpp and
  Utilities/AppSupport/Python/CaseStudyPybind.hpp:40-110).  The iteration
  count for a time span is the reference's ``multiple_just_greater_than``,
  ceil((seconds - 1e-14) / dt) (Utilities/AppSupport/Helpers/
  MultipleJustGreaterThan.hpp).  A run of n iterations is one ``eb_step``
  call of n steps (a few resident launches), not n calls, unless a subclass
  overrides ``step``.
* Parameters — declared per case study with a type, a default (a value or a
  function of the parameters declared before it) and a help string, as the
  reference's tagged parameter structs (examples/dynamic_cantilever/
  DynamicCantileverCaseStudy.hpp).
* ``RodView`` — what ``communicate`` returns: the rod under the PyElastica
  names (``position_collection``, ``velocity_collection``,
  ``director_collection``, ``omega_collection``, ...;
  Systems/CosseratRods/Python/Generators/BindPyElasticaInterface.hpp:36-66),
  ``get_<variable>()`` accessors, the variable locator ``rod.loc[rod.Velocity]``
  and the energy methods (Python/Generators/BindEnergyMethods.hpp).  The
  reference hands out views into the rod's memory; here the state lives on
  the GPU, so a view holds host copies: read from the device at first use
  after a step, and written back before the next step if the caller changed
  them.
* ``DynamicCantileverCaseStudy`` — the reference's dynamic cantilever example
  (examples/dynamic_cantilever/DynamicCantileverCaseStudy.cpp:25-93).
"""
from __future__ import annotations

import math
import re
from dataclasses import dataclass
from typing import Any, Callable

import numpy as np

from . import _lib as L
from .simulator import (Clamp, CosseratRodWithoutDamping, Material, PositionVerlet, RodRef, Simulator,
                        StraightRod)


def multiple_just_greater_than(value: float, factor: float) -> int:
    """ceil((value - 1e-14) / factor), as the reference counts the steps of a
    time span."""
    return int(math.ceil((value - 1e-14) / factor))


@dataclass(frozen=True)
class Parameter:
    name: str
    type: type
    default: Any  # a value, or a function of the parameters declared before
    help: str = ""


class Params:
    """Parameter values of a case study (attribute access, in declaration
    order)."""

    def __init__(self, declared: tuple, values: dict):
        self._declared = declared
        unknown = set(values) - {p.name for p in declared}
        if unknown:
            raise TypeError(f"unknown parameters: {sorted(unknown)}")
        for p in declared:
            if p.name in values:
                v = values[p.name]
            else:
                v = p.default(self) if callable(p.default) else p.default
            setattr(self, p.name, p.type(v))

    def data(self) -> dict:
        return {p.name: getattr(self, p.name) for p in self._declared}

    def __repr__(self) -> str:
        return "Params(" + ", ".join(f"{k}={v!r}" for k, v in self.data().items()) + ")"


def _snake(name: str) -> str:
    return re.sub(r"(?<!^)(?=[A-Z])", "_", name).lower()


# PyElastica names of the rod variables
_PYELASTICA = {
    "position_collection": "Position", "velocity_collection": "Velocity",
    "director_collection": "Director", "omega_collection": "AngularVelocity",
    "acceleration_collection": "Acceleration", "alpha_collection": "AngularAcceleration",
    "rest_lengths": "ReferenceElementLength", "rest_voronoi_lengths": "ReferenceVoronoiLength",
    "volume": "ElementVolume", "mass": "Mass",
    "mass_second_moment_of_inertia": "MassSecondMomentOfInertia",
    "inv_mass_second_moment_of_inertia": "InvMassSecondMomentOfInertia",
    "dissipation_constant_for_forces": "ForceDampingRate",
    "dissipation_constant_for_torques": "TorqueDampingRate",
    "internal_forces": "InternalLoads", "internal_torques": "InternalTorques",
    "lengths": "ElementLength", "tangents": "Tangent", "dilatation": "ElementDilatation",
    "voronoi_dilatation": "VoronoiDilatation",
}


class _Locator:
    def __init__(self, view: "RodView"):
        self._view = view

    def __getitem__(self, tag: str) -> np.ndarray:
        return self._view._array(tag)

    def __repr__(self) -> str:
        return "Variable indexer"


class RodView:
    """Host view of one rod of a case study (see the module docstring)."""

    def __init__(self, case: "CaseStudy", ref: RodRef):
        self._case = case
        self._ref = ref
        self._cache: dict[str, tuple[np.ndarray, np.ndarray]] = {}

    # variable tags as attributes, for rod.loc[rod.Velocity]
    def __getattr__(self, name: str):
        if name in L.FIELD_ID:
            return name
        if name in _PYELASTICA:
            return self._array(_PYELASTICA[name])
        if name.startswith("get_"):
            snake = name[4:]
            for tag in L.FIELDS:
                if _snake(tag) == snake:
                    return lambda tag=tag: self._array(tag)
        raise AttributeError(name)

    @property
    def loc(self) -> _Locator:
        return _Locator(self)

    @property
    def n_elems(self) -> int:
        return self._ref.n_elements

    def __len__(self) -> int:
        return self._ref.n_elements

    def _array(self, tag: str) -> np.ndarray:
        if tag not in self._cache:
            a = self._ref.get(tag)
            self._cache[tag] = (a, a.copy())
        return self._cache[tag][0]

    def _flush(self) -> None:
        for tag, (a, seen) in self._cache.items():
            if not np.array_equal(a, seen, equal_nan=True):
                self._ref.set(tag, a)
        self._cache.clear()

    # energies (Systems/CosseratRods/Utility/Energy.hpp:46-141)
    def _energy(self, k: int) -> float:
        self._case._flush()
        return float(self._case.simulator.energy()[self._ref.id, k])

    def compute_translational_energy(self) -> float:
        return self._energy(0)

    def compute_rotational_energy(self) -> float:
        return self._energy(1)

    def compute_shearing_energy(self) -> float:
        return self._energy(2)

    def compute_bending_energy(self) -> float:
        return self._energy(3)

    def __str__(self) -> str:
        return "CosseratRodWithoutDamping"


class CaseStudy:
    """Base of a case study.  Subclasses declare ``parameters`` and ``help``,
    implement ``setup(params)`` (create ``self.simulator``, add and finalize
    the rods, call ``self.set_dt``) and ``communicate()``; they may override
    ``step`` (then a run of n iterations calls it n times)."""

    help: str = ""
    parameters: tuple = ()
    stepper = PositionVerlet

    def __init__(self, params: Params | None = None, **values):
        if params is not None and values:
            raise TypeError("pass a Params object or keyword values, not both")
        self.params = params if params is not None else Params(self.parameters, values)
        self.simulator: Simulator | None = None
        self._views: list[RodView] = []
        self._time = 0.0
        self._dt = 0.0
        self._iteration = 0
        self.setup(self.params)

    @classmethod
    def make_params(cls, **values) -> Params:
        return Params(cls.parameters, values)

    @classmethod
    def parameter_help(cls) -> str:
        return "\n".join(f"{p.name} ({p.type.__name__}): {p.help}" for p in cls.parameters)

    # -- to implement ----------------------------------------------------------
    def setup(self, params: Params) -> None:
        raise NotImplementedError

    def communicate(self):
        raise NotImplementedError

    def run(self) -> None:
        raise RuntimeError("run() not implemented : launch the case from python!")

    # -- stepping --------------------------------------------------------------
    def step(self) -> None:
        """One iteration of the time stepper."""
        self._advance(1)

    def _advance(self, n: int) -> None:
        if self.simulator is None:
            raise RuntimeError("the case study has no simulator (setup did not create one)")
        if self._dt <= 0.0:
            raise RuntimeError("the time step is not set (setup must call set_dt)")
        self._flush()
        if n > 0:
            self._time = self.simulator.step(self.stepper(), self._time, self._dt, n)
            self._iteration += n

    def run_for_n_iterations(self, n_iterations: int) -> None:
        n = int(n_iterations)
        if n < 0:
            raise ValueError("n_iterations must be non-negative")
        if type(self).step is CaseStudy.step:
            self._advance(n)  # one fused call
        else:
            for _ in range(n):
                self.step()

    def run_for(self, *, additional_time: float | None = None, n_iterations: int | None = None) -> None:
        if (additional_time is None) == (n_iterations is None):
            raise TypeError("give exactly one of additional_time and n_iterations")
        if n_iterations is not None:
            self.run_for_n_iterations(n_iterations)
        else:
            self.run_for_n_iterations(max(0, multiple_just_greater_than(float(additional_time), self._dt)))

    def step_with(self, dt: float) -> None:
        self.set_dt(dt)
        self.step()

    # -- queries and setters ---------------------------------------------------
    def current_time(self) -> float:
        return self._time

    def current_dt(self) -> float:
        return self._dt

    def current_iteration(self) -> int:
        return self._iteration

    def set_dt(self, value: float) -> None:
        if not value > 0.0:
            raise ValueError("the time step must be positive")
        self._dt = float(value)

    def set_current_time(self, value: float) -> None:
        self._time = float(value)

    def set_current_iteration(self, value: int) -> None:
        self._iteration = int(value)

    def reset(self) -> None:
        """Time and iteration back to zero and the simulator rebuilt from the
        parameters (the reference's reset_case_study with EnableReset)."""
        self._time = 0.0
        self._iteration = 0
        self.close()
        self.setup(self.params)

    # -- checkpoints -----------------------------------------------------------
    def save(self, path) -> None:
        """The simulator's snapshot plus the time, time step and iteration."""
        self._flush()
        snap = self.simulator.snapshot()
        np.savez(path, snapshot=np.frombuffer(snap, dtype=np.uint8),
                 clock=np.array([self._time, self._dt], dtype=np.float64),
                 iteration=np.array([self._iteration], dtype=np.int64))

    def load(self, path) -> None:
        """Restore a checkpoint of this case study (same parameters)."""
        with np.load(path) as z:
            self._views_refresh()
            self.simulator.restore(z["snapshot"].tobytes())
            self._time, self._dt = (float(v) for v in z["clock"])
            self._iteration = int(z["iteration"][0])

    def _views_refresh(self) -> None:
        for v in self._views:
            v._cache.clear()

    # -- views -----------------------------------------------------------------
    def view(self, ref: RodRef) -> RodView:
        v = RodView(self, ref)
        self._views.append(v)
        return v

    def _flush(self) -> None:
        for v in self._views:
            v._flush()

    def close(self) -> None:
        self._views = []
        if self.simulator is not None:
            self.simulator.close()
            self.simulator = None

    def __str__(self) -> str:
        return type(self).__name__


class DynamicCantileverCaseStudy(CaseStudy):
    """A rod clamped at one end (position and directors held at node 0,
    velocity and angular velocity zeroed there), without damping or gravity,
    set oscillating by the caller through ``communicate()``
    (examples/dynamic_cantilever/DynamicCantileverCaseStudy.cpp:25-93 and
    helpers/driver.py)."""

    help = ("DynamicCantilever test-case: response of a clamped CosseratRod, initialised by modal "
            "oscillations at natural frequencies, compared with Euler-Bernoulli beam theory.")
    parameters = (
        Parameter("n_elements", int, 100, "Number of elements in the rod"),
        Parameter("youngs_modulus", float, 1e5, "Youngs modulus of the rod"),
        Parameter("shear_modulus", float, lambda p: p.youngs_modulus / 3.0, "Shear modulus of the rod"),
        Parameter("density", float, 2000.0, "Density of the rod"),
        Parameter("radius", float, 0.02, "Radius of the rod"),
        Parameter("length", float, 1.0, "Length of the rod"),
        Parameter("dt", float, lambda p: 0.05 * p.length / p.n_elements, "Time step of simulation"),
    )

    def setup(self, params: Params) -> None:
        self.simulator = Simulator()
        rod = StraightRod(n_elements=params.n_elements,
                          material=Material(params.density, params.youngs_modulus, params.shear_modulus),
                          radius=params.radius, length=params.length, origin=(0.0, 0.0, 0.0),
                          direction=(1.0, 0.0, 0.0), normal=(0.0, 1.0, 0.0))
        self.rod_ref = self.simulator.emplace_back(CosseratRodWithoutDamping, rod)
        self.simulator.constrain(self.rod_ref).at(0).using(Clamp())
        self.simulator.finalize()
        self.set_dt(params.dt)
        self._rod_view = self.view(self.rod_ref)

    def communicate(self) -> RodView:
        return self._rod_view
