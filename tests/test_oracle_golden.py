"""Pin the CPU oracle against the reference's own golden vectors.

Each stepping case restates the reference's Catch2 test: build the straight
rod(s), inject the perturbed state (the ``*_REPLACED`` literals), take N
PositionVerlet steps and compare every checked field with the section's
``approx.epsilon`` under Catch's semantics (|a - b| <= eps |b|).
"""
import numpy as np
import pytest

import goldens as G

pytestmark = []


def build_case(oracle, case, damped):
    n = G.ROD_SETUP["n"]
    rods = oracle.RodArrays([n] * case["n_rods"], damped=damped)
    for r in range(case["n_rods"]):
        init = oracle.straight_rod(n, G.ROD_SETUP["origin"], G.ROD_SETUP["direction"],
                                   G.ROD_SETUP["normal"], G.ROD_SETUP["length"],
                                   G.ROD_SETUP["radius"], G.ROD_SETUP["density"],
                                   G.ROD_SETUP["youngs"], G.ROD_SETUP["shear"])
        rods.set_rod("x", r, init["x"])
        rods.set_rod("Q", r, init["Q"].reshape(9, n))
        rods.set_rod("mass", r, init["mass"])
        rods.set_rod("rest_length", r, init["l0"])
        rods.set_rod("rest_voronoi", r, init["D0"])
        rods.set_rod("volume", r, init["V"])
        rods.set_rod("shear_diag", r, init["S"])
        rods.set_rod("bend_diag", r, init["B"])
        rods.set_rod("inertia_diag", r, init["J"])
        rods.set_rod("inv_inertia", r, init["Jinv"])
        if damped:
            rods.set_rod("nu_force", r, np.full(n + 1, G.ROD_SETUP["damping"]))
            rods.set_rod("nu_torque", r, np.full(n, G.ROD_SETUP["damping"]))
        for field, entry in case["inject"][str(r)].items():
            if field in G.STATE_FIELDS:
                key, kind = G.STATE_FIELDS[field]
            elif field in G.PARAM_FIELDS:
                key, kind = G.PARAM_FIELDS[field]
            else:
                continue  # diagnostics are overwritten by every step
            rods.set_rod(key, r, G.as_component_major(entry, kind))
    rods.enable_diagnostics()
    return rods


def test_fixture_inventory():
    cases = list(G.step_cases())
    assert len(cases) == 10  # 5 + 1 damped sections, 4 undamped sections
    for _, case, sec, _ in cases:
        for r in range(case["n_rods"]):
            assert len(sec["expected"][str(r)]) == 27
        assert sec["epsilon"] is not None


def test_inverse_inertia_is_reciprocal_bitwise():
    """J^-1 in every golden equals 1/J exactly, so the library may derive it."""
    for name in ("perturbed_rod_step", "perturbed_rod_step_without_damping", "perturbed_rod"):
        for case in G.load(name)["cases"]:
            for r, fields in case["inject"].items():
                if "MassSecondMomentOfInertia" not in fields:
                    continue
                J = G.as_component_major(fields["MassSecondMomentOfInertia"], "diag")
                Ji = G.as_component_major(fields["InvMassSecondMomentOfInertia"], "diag")
                assert np.array_equal(1.0 / J, Ji), (name, case["name"], r)


def test_straight_rod_initializer(oracle_mod):
    """Initializer parameters vs the InitializeStraightRod PyElastica values
    (Test_PerturbedRod.cpp:66-143, epsilon 1e-12) and vs the init-time values
    injected by the stepping tests."""
    s = G.ROD_SETUP
    init = oracle_mod.straight_rod(s["n"], s["origin"], s["direction"], s["normal"], s["length"],
                                   s["radius"], s["density"], s["youngs"], s["shear"])
    case = [c for c in G.load("perturbed_rod")["cases"] if c["name"].endswith("InitializeStraightRod")][0]
    exp = case["expected"]["0"]
    checks = {"Mass": init["mass"], "ElementVolume": init["V"],
              "ReferenceElementLength": init["l0"], "ReferenceVoronoiLength": init["D0"],
              "ShearStretchRigidityMatrix": init["S"], "BendingTwistRigidityMatrix": init["B"],
              "MassSecondMomentOfInertia": init["J"], "InvMassSecondMomentOfInertia": init["Jinv"],
              "Position": init["x"], "Director": init["Q"].reshape(9, -1)}
    kinds = {**G.STATE_FIELDS, **G.PARAM_FIELDS}
    for field, got in checks.items():
        want = G.as_component_major(exp[field], kinds[field][1])
        assert G.catch_violation(got, want, 1e-12) <= 1.0, field
    # the stepping goldens inject the same init-time mass, volume and inertia
    step_inject = G.load("perturbed_rod_step")["cases"][0]["inject"]["0"]
    for field, key in (("Mass", "mass"), ("ElementVolume", "V")):
        want = G.as_component_major(step_inject[field], "scalar")
        assert G.catch_violation(init[key], want, 1e-13) <= 1.0, field
    want = G.as_component_major(step_inject["MassSecondMomentOfInertia"], "diag")
    assert G.catch_violation(init["J"], want, 1e-13) <= 1.0


@pytest.mark.parametrize("name,case,sec,damped", list(G.step_cases()),
                         ids=lambda v: v if isinstance(v, str) else (
                             v.get("name", "").split(".")[-1] if isinstance(v, dict) else str(v)))
def test_oracle_step_golden(oracle_mod, name, case, sec, damped):
    rods = build_case(oracle_mod, case, damped)
    n = G.ROD_SETUP["n"]
    if sec["steps"] > 0:
        rods.step(G.ROD_SETUP["dt"], sec["steps"], n_threads=1)
    eps = sec["epsilon"]
    worst = {}
    for r in range(case["n_rods"]):
        for field, entry in sec["expected"][str(r)].items():
            if field in G.STATE_FIELDS:
                key, kind = G.STATE_FIELDS[field]
                count = entry["dims"][-1]
                got = rods.get_rod(key, r, count)
            elif field in G.PARAM_FIELDS:
                key, kind = G.PARAM_FIELDS[field]
                count = entry["dims"][-1]
                got = rods.get_rod(key, r, count)
            else:
                key, kind = G.DIAG_FIELDS[field]
                if sec["steps"] == 0:
                    continue  # NoStep: diagnostics only echo the injection
                count = entry["dims"][-1]
                got = rods.get_diag(key, r, count)
            want = G.as_component_major(entry, kind)
            worst[(r, field)] = G.catch_violation(got, want, eps)
    bad = {k: v for k, v in worst.items() if v > 1.0}
    assert not bad, f"{case['name']}/{sec['name']}: {bad}"
    assert n == 5
