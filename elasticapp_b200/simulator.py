"""Python mirror of the reference's Simulator plugin surface for the rod step.

The reference drives rods as (elastica/Simulator/Interface/...):

    simulator = elastica::make_simulator<...>(config);
    rod = simulator->emplace_back<CosseratRod>(StraightInit{...}.initialize<CosseratRod>());
    simulator->constrain(rod).at(0UL).with(clamp_generator());
    simulator->finalize();
    simulator->step(time_stepper, time, dt);

Here the same calls exist with the same meaning, backed by the C-ABI of
libelastica_b200.so (include/elastica_b200.h):

    sim = Simulator()
    rod = sim.emplace_back(CosseratRod, StraightRod(...))
    sim.constrain(rod).at(0).using(Clamp())
    sim.finalize()
    t = sim.step(PositionVerlet(), t, dt)

Variables are read and written with ``rod.get("Position")`` /
``rod.set("Position", array)`` in the reference's shapes (3 x N, 3 x 3 x N,
N), mirroring ``blocks::get<elastica::tags::Position>(rod)``.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Iterable, Sequence

import numpy as np

from . import _lib as L


# -- rod models (elastica/Systems/CosseratRods/Aliases) ---------------------
class CosseratRod:
    """Circular rod with diagonal linear elasticity and explicit damping
    (Aliases/CosseratRod.hpp:33-40)."""

    model = L.EB_ROD_DAMPED


class CosseratRodWithoutDamping:
    """Same rod without the explicit damping adapter
    (Aliases/CosseratRodWithoutDamping.hpp)."""

    model = L.EB_ROD_UNDAMPED


@dataclass
class Material:
    """The material entries a rod reads (Simulator/Materials/Materials.hpp:436-449)."""

    density: float
    youngs_modulus: float
    shear_modulus: float


@dataclass
class StraightRod:
    """StraightCosseratRodInitializer (Initializers/StraightCosseratRod.hpp)."""

    n_elements: int
    material: Material
    radius: float
    length: float
    origin: Sequence[float] = (0.0, 0.0, 0.0)
    direction: Sequence[float] = (1.0, 0.0, 0.0)
    normal: Sequence[float] = (0.0, 1.0, 0.0)
    force_damping_rate: float = 0.0
    torque_damping_rate: float = 0.0

    def to_c(self, model: int) -> L.EbStraightRod:
        r = L.EbStraightRod()
        r.n_elements = int(self.n_elements)
        r.model = int(model)
        r.density = float(self.material.density)
        r.youngs_modulus = float(self.material.youngs_modulus)
        r.shear_modulus = float(self.material.shear_modulus)
        r.radius = float(self.radius)
        r.length = float(self.length)
        for i in range(3):
            r.origin[i] = float(self.origin[i])
            r.direction[i] = float(self.direction[i])
            r.normal[i] = float(self.normal[i])
        r.force_damping_rate = float(self.force_damping_rate)
        r.torque_damping_rate = float(self.torque_damping_rate)
        return r


# -- constraints, forcing, environments, stepper -----------------------------
@dataclass
class Clamp:
    """Value constraint x_k = x_k(now), Q_k = Q_k(now) plus rate constraint
    v_k = w_k = 0 at the node / element index given with .at(k) (0 if none;
    pattern of examples/dynamic_cantilever/DynamicCantileverCaseStudy.cpp:
    73-89).  At most two clamps per rod, e.g. .at(0) and .at(n)."""


@dataclass
class AnalyticalLinearDamper:
    """Rate constraint of examples/fish_swimming/FishModel/Dissipations/
    AnalyticalLinearDamper.hpp:15-76 (physical version)."""

    translational_rate: float
    rotational_rate: float


@dataclass
class EndTorque:
    """Constant lab-frame torque on one element, the last one unless placed
    with .at(element) (Forcing/MakeForcing.hpp)."""

    torque: Sequence[float]


@dataclass
class GravityField:
    """Environments/GravityField/GravityField.hpp:239-246."""

    gravity: Sequence[float] = (0.0, 0.0, -9.81)


@dataclass
class ContactMaterial:
    """Contact parameters of elastica::create_material (Simulator/Materials/
    Materials.cpp:237-372); a material pair uses 1/(1/a + 1/b) for stiffness
    and dampings and a + b for the friction coefficients."""

    stiffness: float
    normal_damping: float
    tangential_damping: float
    static_friction: float
    dynamic_friction: float


@dataclass
class CollisionSystem:
    """The collision-system environment (Environments/CollisionSystem/
    DEMSolver.hpp:701-727).  Rods take part through Simulator.add_contact;
    planes through Simulator.emplace_plane."""


@dataclass
class FreeJoint:
    """Translational spring (stiffness) and dashpot along the separation
    (damping) between node index_a + 1 of rod a and node index_b of rod b
    (the force rule of examples/hinge_joint/HingeJointCaseStudy.cpp:116-136)."""

    def __init__(self, stiffness: float, damping: float = 0.0):
        self.stiffness, self.damping = float(stiffness), float(damping)

    def to_c(self) -> L.EbJoint:
        j = L.EbJoint()
        j.kind, j.stiffness, j.damping = L.EB_JOINT_FREE, self.stiffness, self.damping
        return j


class HingeJoint(FreeJoint):
    """FreeJoint plus the rotational spring that resists the component of rod
    b's element index_b along `normal` (HingeJointCaseStudy.cpp:137-150)."""

    def __init__(self, stiffness: float, damping: float, rotational_stiffness: float, normal):
        super().__init__(stiffness, damping)
        self.rotational_stiffness = float(rotational_stiffness)
        self.normal = tuple(float(v) for v in normal)

    def to_c(self) -> L.EbJoint:
        j = super().to_c()
        j.kind = L.EB_JOINT_HINGE
        j.rotational_stiffness = self.rotational_stiffness
        for k in range(3):
            j.normal[k] = self.normal[k]
        return j


class _Connect:
    """simulator.connect(rod_a, index_a).to(rod_b, index_b).using(joint), the
    reference's connect(rod_a, at(i)).to(rod_b, at(j)).with(generator)."""

    def __init__(self, sim, rod_a, index_a):
        self.sim, self.rod_a, self.index_a = sim, rod_a, int(index_a)
        self.rod_b = self.index_b = None

    def to(self, rod_b, index_b: int) -> "_Connect":
        self.rod_b, self.index_b = rod_b, int(index_b)
        return self

    def using(self, joint: FreeJoint) -> None:
        if self.rod_b is None:
            raise TypeError("connect(...).to(rod, index) first")
        j = joint.to_c()
        L.call("eb_connect", self.sim._h, self.rod_a.id, self.index_a, self.rod_b.id, self.index_b,
               ctypes.byref(j))

    with_ = using


class PositionVerlet:
    """Time/SymplecticSteppers/Algorithms/PositionVerlet.hpp:49-88."""


@dataclass
class PEFRL:
    """Position-extended Forest-Ruth-like stepper (Omelyan, Mryglod, Folk
    2002), declared in Time/SymplecticSteppers/Algorithms/Types.hpp:31.  A
    simulator steps with the stepper it was created with."""


@dataclass
class VelocityVerlet:
    """Time/SymplecticSteppers/Algorithms/VelocityVerlet.hpp:49-87: kick
    dt/2, drift dt, kick dt/2 (two force evaluations a step)."""


_STEPPERS = {PositionVerlet: L.EB_STEPPER_POSITION_VERLET, PEFRL: L.EB_STEPPER_PEFRL,
             VelocityVerlet: L.EB_STEPPER_VELOCITY_VERLET}


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class RodRef:
    """Stable handle of one emplaced rod (the reference's BlockSlice ref)."""

    def __init__(self, sim: "Simulator", rod_id: int, n_elements: int):
        self.sim = sim
        self.id = int(rod_id)
        self.n_elements = int(n_elements)

    def shape(self, name: str) -> tuple:
        place, nc = L.FIELD_SHAPE[name]
        n = self.n_elements
        count = n + 1 if place == 0 else (n if place == 1 else n - 1)
        if name == "Director":
            return (3, 3, count)
        return (nc, count) if nc > 1 else (count,)

    def get(self, name: str) -> np.ndarray:
        out = np.empty(self.shape(name), dtype=np.float64)
        L.call("eb_get_field", self.sim._h, self.id, L.FIELD_ID[name], _dptr(out), out.size)
        return out

    def set(self, name: str, values) -> None:
        a = np.ascontiguousarray(values, dtype=np.float64)
        if a.size != int(np.prod(self.shape(name))):
            raise ValueError(f"{name} expects shape {self.shape(name)}, got {a.shape}")
        L.call("eb_set_field", self.sim._h, self.id, L.FIELD_ID[name], _dptr(a), a.size)

    # common accessors, as in the reference's rod member API
    # (tests/Unit/Systems/CosseratRods/FullRodTest/Test_RodAPI.cpp:13-40)
    def get_position(self):
        return self.get("Position")

    def get_velocity(self):
        return self.get("Velocity")

    def get_director(self):
        return self.get("Director")

    def get_angular_velocity(self):
        return self.get("AngularVelocity")


class _At:
    def __init__(self, owner, rod: RodRef, kind: str):
        self.owner, self.rod, self.kind, self.index = owner, rod, kind, None

    def at(self, index: int) -> "_At":
        self.index = int(index)
        return self

    def using(self, item) -> None:
        self.owner._attach(self.kind, self.rod, self.index, item)

    with_ = using


class Simulator:
    """Owns one eb_sim (device memory and a CUDA stream)."""

    def __init__(self, device: int = 0, precision: str = "fp64", record_diagnostics: bool = False,
                 reference_rounding: bool = False, window: int = 0, step_mode: str = "auto",
                 resident_config: int = 0, stepper=None, cuda_graph: bool = False):
        cfg = L.EbConfig()
        cfg.device = int(device)
        cfg.precision = {"fp64": L.EB_PRECISION_FP64, "mixed": L.EB_PRECISION_MIXED}[precision]
        cfg.flags = (L.EB_FLAG_RECORD_DIAGNOSTICS if record_diagnostics else 0) | (
            L.EB_FLAG_REFERENCE_ROUNDING if reference_rounding else 0) | {
            "auto": 0, "streaming": L.EB_FLAG_STEP_STREAMING, "resident": L.EB_FLAG_STEP_RESIDENT,
            "bucketed": L.EB_FLAG_STEP_BUCKETED}[step_mode]
        cfg.step_window = int(window)
        cfg.resident_config = int(resident_config)
        if cuda_graph:
            cfg.flags |= L.EB_FLAG_CUDA_GRAPH
        kind = stepper if isinstance(stepper, type) else type(stepper)
        self.stepper = kind if stepper is not None and kind in _STEPPERS else PositionVerlet
        cfg.stepper = _STEPPERS[self.stepper]
        h = ctypes.c_void_p()
        L.call("eb_sim_create", ctypes.byref(cfg), ctypes.byref(h))
        self._h = h
        self.rods: list[RodRef] = []
        self.finalized = False

    def close(self) -> None:
        if getattr(self, "_h", None):
            L.load().eb_sim_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- systems -----------------------------------------------------------
    def emplace_back(self, model, initializer: StraightRod) -> RodRef:
        return self.emplace_back_many(model, [initializer])[0]

    def emplace_back_many(self, model, initializers: Iterable[StraightRod]) -> list[RodRef]:
        inits = list(initializers)
        arr = (L.EbStraightRod * len(inits))(*[i.to_c(model.model) for i in inits])
        ids = (ctypes.c_int64 * len(inits))()
        L.call("eb_emplace_straight_rods", self._h, arr, len(inits), ids)
        refs = [RodRef(self, ids[k], inits[k].n_elements) for k in range(len(inits))]
        self.rods.extend(refs)
        return refs

    # -- modules ---------------------------------------------------------------
    def constrain(self, rod: RodRef) -> _At:
        return _At(self, rod, "constrain")

    def connect(self, rod_a: RodRef, index_a: int) -> _Connect:
        return _Connect(self, rod_a, index_a)

    def force(self, rod: RodRef) -> _At:
        return _At(self, rod, "force")

    def add_environment(self, env) -> None:
        if isinstance(env, GravityField):
            g = np.asarray(env.gravity, dtype=np.float64)
            L.call("eb_add_gravity", self._h, _dptr(g))
        elif isinstance(env, CollisionSystem):
            pass  # active once a rod takes part (add_contact)
        else:
            raise TypeError(f"unsupported environment {env!r}")

    # -- collision system ---------------------------------------------------------
    def create_material(self, material: ContactMaterial) -> int:
        m = L.EbContactMaterial(float(material.stiffness), float(material.normal_damping),
                                float(material.tangential_damping), float(material.static_friction),
                                float(material.dynamic_friction))
        mid = ctypes.c_int32()
        L.call("eb_add_contact_material", self._h, ctypes.byref(m), ctypes.byref(mid))
        return mid.value

    def add_contact(self, rod: RodRef, material: int) -> None:
        """The rod's elements become capsules of the collision system."""
        L.call("eb_add_rod_contact", self._h, rod.id, int(material))

    def emplace_plane(self, point, normal, material: int) -> None:
        """Infinite fixed plane (PlanePrimitive.cpp:60-130)."""
        p = np.ascontiguousarray(point, dtype=np.float64)
        n = np.ascontiguousarray(normal, dtype=np.float64)
        L.call("eb_add_contact_plane", self._h, _dptr(p), _dptr(n), int(material))

    def contact_pairs(self) -> np.ndarray:
        """Sorted candidate pairs (k, 2) of the last step: capsule id = element
        slot, plane p = n_slots + p."""
        count = ctypes.c_int64()
        L.call("eb_contact_pairs", self._h, None, 0, ctypes.byref(count))
        out = np.zeros(2 * max(count.value, 1), dtype=np.int64)
        n2 = ctypes.c_int64()
        L.call("eb_contact_pairs", self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), count.value,
               ctypes.byref(n2))
        return out[:2 * n2.value].reshape(n2.value, 2)

    def _attach(self, kind, rod, index, item):
        if kind == "constrain" and isinstance(item, Clamp):
            L.call("eb_constrain_clamp", self._h, rod.id, 0 if index is None else index)
        elif kind == "constrain" and isinstance(item, AnalyticalLinearDamper):
            L.call("eb_add_analytical_damper", self._h, rod.id, float(item.translational_rate),
                   float(item.rotational_rate))
        elif kind == "force" and isinstance(item, EndTorque):
            t = np.asarray(item.torque, dtype=np.float64)
            element = rod.n_elements - 1 if index is None else index
            L.call("eb_add_element_torque", self._h, rod.id, int(element), _dptr(t))
        else:
            raise TypeError(f"unsupported {kind} item {item!r}")

    def finalize(self) -> None:
        L.call("eb_finalize", self._h)
        self.finalized = True

    # -- time stepping -------------------------------------------------------
    def step(self, stepper, time: float, dt: float, n_steps: int = 1) -> float:
        if not isinstance(stepper, self.stepper):
            raise TypeError(f"this simulator was created for {self.stepper.__name__}")
        t = ctypes.c_double(time)
        L.call("eb_step", self._h, ctypes.byref(t), float(dt), int(n_steps))
        return t.value

    _EXCHANGE = ("Position", "Velocity", "Director", "AngularVelocity")

    def step_host_state(self, stepper, time: float, dt: float, n_steps: int, inputs: dict | None = None,
                        outputs: dict | None = None) -> float:
        """Set the state from host arrays, step, read it back (eb_step_host_state).

        inputs/outputs map "Position", "Velocity", "Director" and
        "AngularVelocity" to float64 C-contiguous arrays in the slot layout,
        shape (ncomp, n_slots); an output may be its input.  The same as
        set_slots, step and get_slots in sequence; under a resident plan the
        copies of one slot group overlap the steps of the others (pinned
        arrays needed for the overlap).
        """
        if not isinstance(stepper, self.stepper):
            raise TypeError(f"this simulator was created for {self.stepper.__name__}")
        hs = L.EbHostState()
        S = self.n_slots()
        for d, arrays in (("in", inputs or {}), ("out", outputs or {})):
            for name, arr in arrays.items():
                if name not in self._EXCHANGE:
                    raise KeyError(f"{name} is not a state field")
                shape = (L.FIELD_SHAPE[name][1], S)
                if (not isinstance(arr, np.ndarray) or arr.dtype != np.float64 or arr.shape != shape
                        or not arr.flags.c_contiguous or (d == "out" and not arr.flags.writeable)):
                    raise ValueError(f"{name} must be a C-contiguous float64 array of shape {shape}")
                setattr(hs, f"{L.FIELD_NAME_SNAKE[name]}_{d}", arr.ctypes.data)
        t = ctypes.c_double(time)
        L.call("eb_step_host_state", self._h, ctypes.byref(t), float(dt), int(n_steps), ctypes.byref(hs))
        return t.value

    def synchronize(self) -> None:
        L.call("eb_synchronize", self._h)

    def energy(self) -> np.ndarray:
        out = np.empty((len(self.rods), 4), dtype=np.float64)
        L.call("eb_energy", self._h, _dptr(out), out.size)
        return out

    def stream_handle(self) -> int:
        """The simulator's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        h = ctypes.c_void_p()
        L.call("eb_get_stream", self._h, ctypes.byref(h))
        return int(h.value or 0)

    def step_plan(self) -> dict:
        """The kernel plan chosen by the first step (see eb_step_plan)."""
        mode, cfg = ctypes.c_int32(), ctypes.c_int32()
        ms = (ctypes.c_float * 20)()
        L.call("eb_step_plan", self._h, ctypes.byref(mode), ctypes.byref(cfg), ms, 20)
        return {"mode": {0: "undecided", 1: "streaming", 2: "resident", 3: "bucketed"}[mode.value], "config": cfg.value,
                "probe_ms": list(ms)}

    def launch_count(self) -> int:
        c = ctypes.c_int64()
        L.call("eb_launch_count", self._h, ctypes.byref(c))
        return c.value

    # -- batch access ----------------------------------------------------------
    def slot_offsets(self) -> np.ndarray:
        out = np.empty(len(self.rods) + 1, dtype=np.int64)
        L.call("eb_slot_offsets", self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), out.size)
        return out

    def n_slots(self) -> int:
        c = ctypes.c_int64()
        L.call("eb_slot_count", self._h, ctypes.byref(c))
        return c.value

    def get_slots(self, name: str, out: np.ndarray | None = None) -> np.ndarray:
        """Field in the device slot layout, shape (ncomp, n_slots)."""
        nc = L.FIELD_SHAPE[name][1]
        if out is None:
            out = np.empty((nc, self.n_slots()), dtype=np.float64)
        L.call("eb_get_field_batch", self._h, L.FIELD_ID[name], L.EB_LAYOUT_SLOTS, _dptr(out), out.size)
        return out

    def set_slots(self, name: str, values: np.ndarray) -> None:
        a = np.ascontiguousarray(values, dtype=np.float64)
        L.call("eb_set_field_batch", self._h, L.FIELD_ID[name], L.EB_LAYOUT_SLOTS, _dptr(a), a.size)

    def get_batch(self, name: str) -> np.ndarray:
        """Field of all rods concatenated in the per-rod layout (flat)."""
        total = sum(int(np.prod(r.shape(name))) for r in self.rods)
        out = np.empty(total, dtype=np.float64)
        L.call("eb_get_field_batch", self._h, L.FIELD_ID[name], L.EB_LAYOUT_PER_ROD, _dptr(out), out.size)
        return out

    def set_batch(self, name: str, values: np.ndarray) -> None:
        a = np.ascontiguousarray(values, dtype=np.float64).ravel()
        L.call("eb_set_field_batch", self._h, L.FIELD_ID[name], L.EB_LAYOUT_PER_ROD, _dptr(a), a.size)

    # -- snapshots and dumps ---------------------------------------------------
    def snapshot(self) -> bytes:
        """Device state, parameters and per-rod settings as one buffer (see
        eb_snapshot_save); restore() loads it into this or an identically
        configured simulator."""
        n = ctypes.c_uint64()
        L.call("eb_snapshot_size", self._h, ctypes.byref(n))
        buf = ctypes.create_string_buffer(n.value)
        L.call("eb_snapshot_save", self._h, buf, n.value)
        return buf.raw

    def restore(self, snapshot: bytes) -> None:
        data = bytes(snapshot)
        L.call("eb_snapshot_load", self._h, data, len(data))

    def save(self, path) -> None:
        with open(path, "wb") as f:
            f.write(self.snapshot())

    def load(self, path) -> None:
        with open(path, "rb") as f:
            self.restore(f.read())

    def dump_rods(self, path, fields=("Position", "Velocity", "Director", "AngularVelocity")) -> None:
        """Per-rod arrays of the given variables in one numpy archive, keys
        ``rod<k>/<Variable>`` (the per-rod datasets the reference writes to
        HDF5 in Simulator/IO/H5/Systems/CosseratRods/CosseratRod.hpp; HDF5
        itself is not available here)."""
        arrays = {f"rod{k}/{name}": ref.get(name) for k, ref in enumerate(self.rods) for name in fields}
        np.savez(path, **arrays)
