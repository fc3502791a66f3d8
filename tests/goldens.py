"""Helpers shared by the golden-vector tests.

The fixtures under tests/golden/ were extracted by tests/golden/make_golden.py
from the reference's FullRodTest Catch2 files.  The rod set-up those tests use
(identical in every case) is restated here with citations:

* material ``create_material(7.874, 0.24, 200, 200/(2(1+0.5)), 200, 1e-10,
  1e-10, 0.1, 0.1)`` -> density 7.874, E 200, G 200/3
  (Test_PerturbedRodStep.cpp:39-41; argument order from
  elastica/Simulator/Materials/Materials.hpp:447-449),
* ``StraightCosseratRodInitializer`` with 5 elements, radius 0.007522,
  length 0.18, origin 0, direction +y, normal +z, force and torque damping
  rate 0.2 (Test_PerturbedRodStep.cpp:43-57),
* PositionVerlet with dt = 2e-5 (Test_PerturbedRodStep.cpp:76-82).
"""
from __future__ import annotations

import json
import os

import numpy as np

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

ROD_SETUP = dict(n=5, density=7.874, youngs=200.0, shear=200.0 / (2.0 * (1.0 + 0.50)),
                 radius=0.007522, length=0.18, origin=(0.0, 0.0, 0.0),
                 direction=(0.0, 1.0, 0.0), normal=(0.0, 0.0, 1.0), damping=0.2, dt=2e-5)

# golden field name -> (oracle array name, kind) where kind is
#   "vec"    : 3 x N matrix        "scalar": N vector
#   "tensor" : 3 x 3 x N director  "diag"  : 3 x 3 x N tensor stored as its diagonal
STATE_FIELDS = {
    "Position": ("x", "vec"), "Velocity": ("v", "vec"), "Director": ("Q", "tensor"),
    "AngularVelocity": ("w", "vec"),
}
PARAM_FIELDS = {
    "Mass": ("mass", "scalar"), "ReferenceElementLength": ("rest_length", "scalar"),
    "ReferenceVoronoiLength": ("rest_voronoi", "scalar"), "ElementVolume": ("volume", "scalar"),
    "ReferenceShearStretchStrain": ("rest_sigma", "vec"), "ReferenceCurvature": ("rest_kappa", "vec"),
    "ShearStretchRigidityMatrix": ("shear_diag", "diag"),
    "BendingTwistRigidityMatrix": ("bend_diag", "diag"),
    "MassSecondMomentOfInertia": ("inertia_diag", "diag"),
    "InvMassSecondMomentOfInertia": ("inv_inertia", "diag"),
}
DIAG_FIELDS = {
    "ElementLength": ("d_length", "scalar"), "ElementDilatation": ("d_dilatation", "scalar"),
    "Tangent": ("d_tangent", "vec"), "VoronoiDilatation": ("d_vdilatation", "scalar"),
    "ShearStretchStrain": ("d_sigma", "vec"), "Curvature": ("d_kappa", "vec"),
    "InternalStress": ("d_stress", "vec"), "InternalCouple": ("d_couple", "vec"),
    "InternalLoads": ("d_loads", "vec"), "InternalTorques": ("d_torques", "vec"),
    "Acceleration": ("d_accel", "vec"), "AngularAcceleration": ("d_alpha", "vec"),
    "ElementDimension": ("d_dimension", "scalar"),
}


def load(name: str) -> dict:
    with open(os.path.join(GOLDEN_DIR, f"{name}.json"), "r", encoding="utf-8") as f:
        return json.load(f)


def values(entry: dict) -> np.ndarray:
    """Golden entry -> ndarray in the reference's shape."""
    a = np.array([float.fromhex(h) for h in entry["hex"]], dtype=np.float64)
    return a.reshape(entry["dims"])


def as_component_major(entry: dict, kind: str) -> np.ndarray:
    """Golden entry -> (ncomp, N) array matching the slot layout."""
    a = values(entry)
    if kind == "scalar":
        return a.reshape(1, -1)
    if kind == "vec":
        return a
    if kind == "tensor":
        return a.reshape(9, -1)
    if kind == "diag":
        off = a.copy()
        for k in range(3):
            off[k, k, :] = 0.0
        if np.any(off != 0.0):
            raise ValueError("non-diagonal tensor")
        return np.stack([a[k, k, :] for k in range(3)])
    raise KeyError(kind)


def catch_violation(computed: np.ndarray, expected: np.ndarray, eps: float) -> float:
    """Largest |a - b| / (eps |b|) over the entries, i.e. the reference's
    ``CHECK(a == approx(b))`` with ``Approx::custom().epsilon(eps)`` (scale 0,
    margin 0, TestingFramework.hpp:135-140) passes iff this is <= 1.
    Entries that are exactly equal count as 0."""
    a = np.asarray(computed, dtype=np.float64).ravel()
    b = np.asarray(expected, dtype=np.float64).ravel()
    diff = np.abs(a - b)
    tol = eps * np.abs(b)
    out = np.zeros_like(diff)
    nz = diff > 0
    with np.errstate(divide="ignore"):
        out[nz] = np.where(tol[nz] > 0, diff[nz] / np.where(tol[nz] > 0, tol[nz], 1.0), np.inf)
    return float(out.max()) if out.size else 0.0


def step_cases():
    """Yield (file, case, section, damped) for every stepping golden."""
    for name, damped in (("perturbed_rod_step", True), ("perturbed_rod_step_without_damping", False)):
        doc = load(name)
        for case in doc["cases"]:
            for sec in case["sections"]:
                yield name, case, sec, damped
