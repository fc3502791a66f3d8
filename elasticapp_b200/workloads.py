"""Seeded synthetic rod workloads with the shapes of the reference's target
configurations.  No dataset is involved; every draw is from numpy's PCG64
with the seed recorded in the workload.

* ``cantilever``   — 1 rod, 100 elements, L 1 m, r 0.025 m, rho 1000, E 1e6,
  G = E/3, along +x with normal +y, clamped at node 0, gravity -9.81 z,
  analytical damper 0.1, dt 1e-5 (the template is
  examples/dynamic_cantilever/DynamicCantileverCaseStudy.cpp).
* ``uneven_batch`` — 16,384 clamped rods, n ~ U{32..512}, L ~ U[0.5, 2],
  r ~ U[0.005, 0.05], log10 E ~ U[5, 7], Poisson 0.5 (G = E/3), rho 1000,
  analytical damper 0.1, random direction, node velocities N(0, 1e-3^2),
  gravity -9.81 z, dt = 0.1 min(l / sqrt(E / rho)).
* ``mixed_batch``  — 65,536 rods, n ~ U{64..256}, parameters as above, rest
  curvature k u (k ~ U[0, 10] 1/m, u a random body-frame unit vector) and an
  end torque of 1e-3 N m about the initial tangent.  The step is
  dt = 0.5 min(l^2 / (r c)), c = sqrt(E / rho), the PositionVerlet bound of
  the stiffest bending mode (about 2 r c / l^2) of the batch: 4.6e-7 s for
  the default seed.  A step of 1e-5 s is unstable for these rods in the
  reference algorithm itself (the FP64 oracle's angular velocities grow and
  turn non-finite within 8,000 steps), because the fattest elements have a
  radius up to 25 times their length.
* ``contact_batch`` — 8,192 free rods, n = 64, L 0.2 m, r 0.002 m, E 1e6,
  G = E/3, rho 1000, centres uniform in the unit cube, random directions,
  node velocities N(0, 0.05^2), gravity -9.81 z, six wall planes of the cube
  with inward normals, contact stiffness 1e4 N/m, dashpot 10 N s/m and
  friction 0.3 for every pair (per material 2e4, 20 and 0.15 under the pair
  rules), no damping, dt 1e-5.  With 4 r > l every capsule also overlaps the
  capsules two elements along its own rod; the reference's collision system
  applies contact there too.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .simulator import (AnalyticalLinearDamper, Clamp, CollisionSystem, ContactMaterial,
                        CosseratRodWithoutDamping, EndTorque, GravityField, Material, Simulator, StraightRod)


@dataclass
class Workload:
    name: str
    seed: int
    rods: list  # StraightRod
    model: type = CosseratRodWithoutDamping
    clamp: bool | list = True                 # every rod, or per rod
    damper: tuple | None = (0.1, 0.1)
    gravity: tuple | None = (0.0, 0.0, -9.81)
    end_torque: np.ndarray | None = None      # (n_rods, 3) lab frame
    velocities: list | None = None            # per rod (3, n + 1)
    rest_curvature: list | None = None        # per rod (3, n - 1)
    dt: float = 1e-5
    n_steps: int = 1000
    contact_materials: list | None = None     # ContactMaterial per material id
    contact_rod_material: list | None = None  # per rod material id (-1: none)
    planes: list | None = None                # (point, normal, material id)
    connections: list | None = None           # (rod_a, index_a, rod_b, index_b, FreeJoint or HingeJoint)
    clamp_at: list | None = None              # per rod, the clamped node indices (in place of node 0)
    torque_element: list | None = None        # per rod, the element the end torque acts on

    @property
    def n_elements(self) -> np.ndarray:
        return np.array([r.n_elements for r in self.rods], dtype=np.int64)

    @property
    def total_elements(self) -> int:
        return int(self.n_elements.sum())

    def build(self, device: int = 0, record_diagnostics: bool = False, precision: str = "fp64",
              reference_rounding: bool = False, window: int = 0, step_mode: str = "auto",
              resident_config: int = 0, stepper=None, cuda_graph: bool = False) -> Simulator:
        """Create the simulator through the reference-style plugin surface."""
        sim = Simulator(device=device, precision=precision, record_diagnostics=record_diagnostics,
                        reference_rounding=reference_rounding, window=window, step_mode=step_mode,
                        resident_config=resident_config, stepper=stepper, cuda_graph=cuda_graph)
        refs = sim.emplace_back_many(self.model, self.rods)
        if self.gravity is not None:
            sim.add_environment(GravityField(self.gravity))
        for k, ref in enumerate(refs):
            if self.velocities is not None:
                ref.set("Velocity", self.velocities[k])
            if self.rest_curvature is not None:
                ref.set("ReferenceCurvature", self.rest_curvature[k])
            if self.clamp if isinstance(self.clamp, bool) else self.clamp[k]:
                for idx in (self.clamp_at[k] if self.clamp_at is not None else (0,)):
                    sim.constrain(ref).at(int(idx)).using(Clamp())
            if self.damper is not None:
                sim.constrain(ref).using(AnalyticalLinearDamper(*self.damper))
            if self.end_torque is not None:
                el = ref.n_elements - 1 if self.torque_element is None else int(self.torque_element[k])
                sim.force(ref).at(el).using(EndTorque(self.end_torque[k]))
        if self.contact_materials:
            sim.add_environment(CollisionSystem())
            ids = [sim.create_material(m) for m in self.contact_materials]
            for k, ref in enumerate(refs):
                mat = self.contact_rod_material[k] if self.contact_rod_material is not None else 0
                if mat >= 0:
                    sim.add_contact(ref, ids[mat])
            for point, normal, mat in (self.planes or []):
                sim.emplace_plane(point, normal, ids[mat])
        for ra, ia, rb, ib, joint in (self.connections or []):
            sim.connect(refs[ra], ia).to(refs[rb], ib).using(joint)
        sim.finalize()
        return sim


def _unit_vectors(rng, n):
    v = rng.standard_normal((n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def _normals(rng, directions):
    """Random unit normals exactly orthogonalised against the directions."""
    out = np.empty_like(directions)
    for i, d in enumerate(directions):
        while True:
            c = rng.standard_normal(3)
            c = c - np.dot(c, d) * d
            nrm = np.linalg.norm(c)
            if nrm > 1e-3:
                c = c / nrm
                c = c - np.dot(c, d) * d
                out[i] = c / np.linalg.norm(c)
                break
    return out


def hinge_chain(n_links: int = 2, n_elements: int = 10, seed: int = 1006, n_steps: int = 20_000) -> Workload:
    """Links end to end along +z with the hinge-joint example's parameters
    (examples/hinge_joint/HingeJointCaseStudy.cpp: rho 1750, E 3e7, G 2e7,
    r 0.007, L 0.2, damping rate 0.015, hinge k 1e5, nu 0, k_rot 5e3 about
    normal x direction); the first link clamped at its base.  In place of the
    example's time-dependent tip force (a user-written rule) the chain sags
    under gravity along -y from seeded node velocities N(0, 1e-3^2)."""
    from .simulator import CosseratRod, HingeJoint
    rng = np.random.Generator(np.random.PCG64(seed))
    L, n = 0.2, n_elements
    rods = [StraightRod(n_elements=n, material=Material(1750.0, 3e7, 2e7), radius=0.007, length=L,
                        origin=(0.0, 0.0, k * L), direction=(0.0, 0.0, 1.0), normal=(0.0, 1.0, 0.0),
                        force_damping_rate=0.015, torque_damping_rate=0.015) for k in range(n_links)]
    roll = (1.0, 0.0, 0.0)  # normal x direction
    joints = [(k, n - 1, k + 1, 0, HingeJoint(1e5, 0.0, 5e3, roll)) for k in range(n_links - 1)]
    vel = [rng.normal(0.0, 1e-3, size=(3, n + 1)) for _ in range(n_links)]
    return Workload("hinge_chain", seed, rods, model=CosseratRod, clamp=[k == 0 for k in range(n_links)],
                    damper=None, gravity=(0.0, -9.81, 0.0), velocities=vel, dt=1e-5, n_steps=n_steps,
                    connections=joints)


def cantilever(n_elements: int = 100, seed: int = 1001) -> Workload:
    E = 1e6
    rod = StraightRod(n_elements=n_elements, material=Material(1000.0, E, E / 3.0), radius=0.025,
                      length=1.0, origin=(0.0, 0.0, 0.0), direction=(1.0, 0.0, 0.0),
                      normal=(0.0, 1.0, 0.0))
    return Workload("cantilever", seed, [rod], dt=1e-5, n_steps=100_000)


def _random_rods(rng, n_rods, n_lo, n_hi):
    n = rng.integers(n_lo, n_hi + 1, size=n_rods)
    L = rng.uniform(0.5, 2.0, size=n_rods)
    r = rng.uniform(0.005, 0.05, size=n_rods)
    E = 10.0 ** rng.uniform(5.0, 7.0, size=n_rods)
    d = _unit_vectors(rng, n_rods)
    nv = _normals(rng, d)
    origins = rng.uniform(-1.0, 1.0, size=(n_rods, 3))
    rods = [StraightRod(n_elements=int(n[k]), material=Material(1000.0, float(E[k]), float(E[k]) / 3.0),
                        radius=float(r[k]), length=float(L[k]), origin=tuple(origins[k]),
                        direction=tuple(d[k]), normal=tuple(nv[k])) for k in range(n_rods)]
    return rods, n, L, E, d


def uneven_batch(n_rods: int = 16384, seed: int = 1002, n_range=(32, 512), n_steps: int = 1000) -> Workload:
    rng = np.random.Generator(np.random.PCG64(seed))
    rods, n, L, E, d = _random_rods(rng, n_rods, *n_range)
    vel = [rng.normal(0.0, 1e-3, size=(3, int(n[k]) + 1)) for k in range(n_rods)]
    dt = 0.1 * float(np.min((L / n) / np.sqrt(E / 1000.0)))
    return Workload("uneven_batch", seed, rods, velocities=vel, dt=dt, n_steps=n_steps)


def mixed_batch(n_rods: int = 65536, seed: int = 1003, n_range=(64, 256), n_steps: int = 10_000,
                dt: float | None = None) -> Workload:
    rng = np.random.Generator(np.random.PCG64(seed))
    rods, n, L, E, d = _random_rods(rng, n_rods, *n_range)
    if dt is None:
        radius = np.array([r.radius for r in rods])
        ell = L / n
        dt = 0.5 * float(np.min(ell * ell / (radius * np.sqrt(E / 1000.0))))
    vel = [rng.normal(0.0, 1e-3, size=(3, int(n[k]) + 1)) for k in range(n_rods)]
    k_mag = rng.uniform(0.0, 10.0, size=n_rods)
    axes = _unit_vectors(rng, n_rods)
    kappa = [np.repeat((k_mag[k] * axes[k])[:, None], int(n[k]) - 1, axis=1) for k in range(n_rods)]
    torque = 1e-3 * d
    return Workload("mixed_batch", seed, rods, velocities=vel, rest_curvature=kappa,
                    end_torque=torque, dt=dt, n_steps=n_steps)


def unit_cube_walls(size: float = 1.0, material: int = 0) -> list:
    """The six walls of [0, size]^3 with inward normals."""
    h = 0.5 * size
    return [((0.0, h, h), (1.0, 0.0, 0.0), material), ((size, h, h), (-1.0, 0.0, 0.0), material),
            ((h, 0.0, h), (0.0, 1.0, 0.0), material), ((h, size, h), (0.0, -1.0, 0.0), material),
            ((h, h, 0.0), (0.0, 0.0, 1.0), material), ((h, h, size), (0.0, 0.0, -1.0), material)]


def contact_batch(n_rods: int = 8192, seed: int = 1004, n_elements: int = 64, box: float = 1.0,
                  dt: float = 1e-5, n_steps: int = 10_000, length: float = 0.2) -> Workload:
    rng = np.random.Generator(np.random.PCG64(seed))
    radius, E = 0.002, 1e6
    d = _unit_vectors(rng, n_rods)
    nv = _normals(rng, d)
    centres = rng.uniform(0.0, box, size=(n_rods, 3))
    rods = [StraightRod(n_elements=n_elements, material=Material(1000.0, E, E / 3.0), radius=radius,
                        length=length, origin=tuple(centres[k] - 0.5 * length * d[k]), direction=tuple(d[k]),
                        normal=tuple(nv[k])) for k in range(n_rods)]
    vel = [rng.normal(0.0, 0.05, size=(3, n_elements + 1)) for _ in range(n_rods)]
    mat = ContactMaterial(stiffness=2e4, normal_damping=20.0, tangential_damping=20.0, static_friction=0.15,
                          dynamic_friction=0.15)
    return Workload("contact_batch", seed, rods, clamp=False, damper=None, velocities=vel, dt=dt,
                    n_steps=n_steps, contact_materials=[mat], contact_rod_material=[0] * n_rods,
                    planes=unit_cube_walls(box))


WORKLOADS = {"cantilever": cantilever, "uneven_batch": uneven_batch, "mixed_batch": mixed_batch,
           "contact_batch": contact_batch}
