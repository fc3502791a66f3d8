"""Pins the oracle's collision-system restatement against the scenarios of
the reference's own tests (CPU only):

* Detection/Fine/Test_CapsuleCapsule.cpp: contact distance, point and
  normal for capsules touching at their spherical caps, at the cylindrical
  region, with parallel centre lines (two contacts), adjacent rod capsules
  (no contact), separated capsules (no contact), penetration depths 0.25 r,
  0 and -0.9 * contact threshold.
* Detection/Fine/Test_CapsulePlane.cpp: no contact when far or 1.1 *
  threshold away; one contact per penetrating cap.
* Response/DEMForces/Test_LinearSpringDashpot.cpp: a penetrating contact
  gives equal and opposite forces and non-zero torques.
* Detection/Coarse/Test_HashGrids.cpp: the grid search returns exactly the
  exhaustive search's pair set.

The scenarios are restated from the tests' descriptions (positions, radii,
angles); the expected values are the analytic ones those tests assert, at
the reference's Approx tolerance.
"""
import math

import numpy as np
import pytest

THR = 1e-8  # contact threshold for double (Utilities/Thresholds.hpp:138)

P0 = np.array([5.0, 3.0, 6.0])
R1, L1 = 4.0, 8.0
AX = np.array([0.0, 0.0, 1.0])
R2, L2 = 2.0, 8.0
VEL = (1.0, 0.0, 0.0)


def first():
    return {"centre": P0, "axis": AX, "radius": R1, "length": L1, "velocity": VEL}


def close(a, b, tol=1e-9):
    return np.allclose(np.asarray(a), np.asarray(b), rtol=tol, atol=tol)


def unit_from_angles(polar_deg, azim_deg):
    a, b = math.radians(polar_deg), math.radians(azim_deg)
    return np.array([math.sin(a) * math.cos(b), math.sin(a) * math.sin(b), math.cos(a)])


@pytest.mark.parametrize("pen", [0.25 * R1, 0.0, -0.9 * THR])
def test_capsules_atop_each_other(oracle_mod, pen):
    pos2 = P0 + AX * (0.5 * L1 + R1 + 0.5 * L2 + R2 - pen)
    c = oracle_mod.fine_capsule_capsule(first(), {"centre": pos2, "axis": AX, "radius": R2, "length": L2,
                                                  "velocity": VEL})
    assert len(c) >= 1
    pos, n, dist = c[0]
    assert dist == pytest.approx(-pen, rel=1e-9, abs=1e-12)
    assert close(pos, P0 + AX * (0.5 * L1 + R1 - 0.5 * pen))
    assert close(n, -AX)


@pytest.mark.parametrize("pen", [0.25 * R1, 0.0])
def test_capsules_at_an_angle_spherical_regions(oracle_mod, pen):
    ax2 = unit_from_angles(30.0, 80.0)
    anchor = P0 + AX * (0.5 * L1) + (R2 + R1 - pen) * ax2
    pos2 = anchor + (0.5 * L2) * ax2
    c = oracle_mod.fine_capsule_capsule(first(), {"centre": pos2, "axis": ax2, "radius": R2, "length": L2})
    assert len(c) >= 1
    _, n, dist = c[0]
    assert dist == pytest.approx(-pen, rel=1e-9, abs=1e-12)
    assert close(n, -ax2)


@pytest.mark.parametrize("azim", [15.0, 30.0, 45.0, 60.0, 75.0, 90.0, -15.0, -45.0, -90.0])
def test_adjacent_rod_capsules_share_a_vertex_no_contact(oracle_mod, azim):
    ax2 = unit_from_angles(30.0, azim)
    anchor = P0 + 0.5 * L1 * AX
    pos2 = anchor + 0.5 * L2 * ax2
    assert oracle_mod.fine_capsule_capsule(first(), {"centre": pos2, "axis": ax2, "radius": R2,
                                                     "length": L2}) == []


@pytest.mark.parametrize("pen", [0.25 * R1, 0.0])
def test_perpendicular_symmetric_cylindrical_region(oracle_mod, pen):
    # second capsule lies across the top cap, its axis perpendicular to the first
    pos2 = P0 + AX * (0.5 * L1 + R1 + R2 - pen)
    c = oracle_mod.fine_capsule_capsule(first(), {"centre": pos2, "axis": (0.6, 0.8, 0.0), "radius": R2,
                                                  "length": L2})
    assert len(c) == 1
    pos, n, dist = c[0]
    assert dist == pytest.approx(-pen, rel=1e-9, abs=1e-12)
    assert close(pos, P0 + AX * (0.5 * L1 + R1 - 0.5 * pen))
    assert close(n, -AX)


def _radial():
    perp = unit_from_angles(15.0, 30.0)
    r = np.cross(AX, perp)
    return r / np.linalg.norm(r)


@pytest.mark.parametrize("pen", [0.25 * R1, 0.0])
def test_perpendicular_centre_lines_one_contact(oracle_mod, pen):
    rad = _radial()
    pos2 = P0 + (R1 + R2 - pen) * rad
    ax2 = np.cross(AX, rad)
    c = oracle_mod.fine_capsule_capsule(first(), {"centre": pos2, "axis": ax2, "radius": R2, "length": L2})
    assert len(c) == 1
    pos, n, dist = c[0]
    assert dist == pytest.approx(-pen, rel=1e-9, abs=1e-12)
    assert close(pos, P0 + (R1 - 0.5 * pen) * rad)
    assert close(n, -rad)


@pytest.mark.parametrize("pen", [0.25 * R1, 0.0])
def test_parallel_centre_lines_two_contacts(oracle_mod, pen):
    rad = _radial()
    pos2 = P0 + (R1 + R2 - pen) * rad
    c = oracle_mod.fine_capsule_capsule(first(), {"centre": pos2, "axis": AX, "radius": R2, "length": L2})
    assert len(c) == 2
    anchor = P0 + (R1 - 0.5 * pen) * rad
    expected = [anchor - 0.5 * min(L1, L2) * AX, anchor + 0.5 * min(L1, L2) * AX]
    got = sorted((p for p, _, _ in c), key=lambda p: np.linalg.norm(p))
    expected = sorted(expected, key=lambda p: np.linalg.norm(p))
    for g, e in zip(got, expected):
        assert close(g, e)
    for _, n, dist in c:
        assert dist == pytest.approx(-pen, rel=1e-9, abs=1e-12)
        assert close(n, -rad)


def test_separated_capsules_no_contact(oracle_mod):
    rad = unit_from_angles(45.0, 10.0)
    far = P0 + (R1 + 10 * (R2 + L2)) * rad
    for ax2 in (rad, AX, np.cross(rad, AX) / np.linalg.norm(np.cross(rad, AX))):
        assert oracle_mod.fine_capsule_capsule(first(), {"centre": far, "axis": ax2, "radius": R2,
                                                         "length": L2}) == []
    rc = _radial()
    near_radial = P0 + (1.1 * THR + R1 + (R2 + 0.5 * L2)) * rc
    assert oracle_mod.fine_capsule_capsule(first(), {"centre": near_radial, "axis": rc, "radius": R2,
                                                     "length": L2}) == []
    near_parallel = P0 + (R1 + 1.1 * THR + R2) * rc
    assert oracle_mod.fine_capsule_capsule(first(), {"centre": near_parallel, "axis": AX, "radius": R2,
                                                     "length": L2}) == []


def test_capsule_plane_no_contact(oracle_mod):
    cap = {"centre": P0, "axis": AX, "radius": R1, "length": L1, "velocity": VEL}
    assert oracle_mod.fine_capsule_plane(cap, (-10.0, 10.0, 10.0), (0.0, 1.0, 0.0)) == []
    rad = unit_from_angles(45.0, 10.0)
    assert oracle_mod.fine_capsule_plane(cap, P0 + rad * R1 * 2, -rad) == []
    below = P0 - AX * (0.5 * L1 + R1 + 1.1 * THR)
    assert oracle_mod.fine_capsule_plane(cap, below, AX) == []
    rc = _radial()
    assert oracle_mod.fine_capsule_plane(cap, P0 + rc * (R1 + 1.1 * THR), -rc) == []


@pytest.mark.parametrize("tilt", [0.0, 15.0, 30.0, 45.0, 60.0, 75.0])
@pytest.mark.parametrize("side", [-1, 1])
def test_capsule_plane_penetration_at_cap(oracle_mod, tilt, side):
    pen = 0.25 * R1
    cap = {"centre": P0, "axis": AX, "radius": R1, "length": L1}
    n = unit_from_angles(tilt, 0.0)
    point = P0 + side * (0.5 * L1) * AX + side * (R1 - pen) * n
    c = oracle_mod.fine_capsule_plane(cap, point, -side * n)
    assert len(c) >= 1
    # the cap on that side penetrates by pen; its contact sits on the plane
    cap_centre = P0 + side * 0.5 * L1 * AX
    hit = [x for x in c if np.linalg.norm(x[0] - (cap_centre + side * (R1 - pen) * n)) < 1e-9]
    assert len(hit) == 1
    _, normal, dist = hit[0]
    assert dist == pytest.approx(-pen, rel=1e-9)
    assert close(normal, -side * n)


def test_spring_dashpot_equal_and_opposite(oracle_mod):
    pen = 0.25 * R1
    pos2 = P0 + AX * (0.5 * L1 + R1 + 0.5 * L2 + R2 - pen) + np.array([0.3, 0.0, 0.0])
    a = dict(first(), velocity=(1.0, 0.0, 0.0), omega=(0.0, 0.2, 0.0))
    b = {"centre": pos2, "axis": AX, "radius": R2, "length": L2, "velocity": (0.0, 0.5, -1.0)}
    F1, T1, F2, T2 = oracle_mod.fine_pair_loads(a, b, (1e4, 10.0, 10.0, 0.3, 0.3))
    assert np.linalg.norm(F1) > 0 and np.linalg.norm(F2) > 0
    assert np.allclose(F1 + F2, 0.0, atol=1e-9 * np.linalg.norm(F1))
    assert np.linalg.norm(T1) > 0 and np.linalg.norm(T2) > 0
    # normal part: k * delta + c_n * (closing speed) along the contact normal
    n = -AX
    assert F1 @ n > 0.0


def test_spring_dashpot_separated_contact_gives_no_force(oracle_mod):
    # a contact within the threshold but not penetrating: no force
    pos2 = P0 + AX * (0.5 * L1 + R1 + 0.5 * L2 + R2 + 0.5 * THR)
    F1, T1, F2, T2 = oracle_mod.fine_pair_loads(first(), {"centre": pos2, "axis": AX, "radius": R2,
                                                          "length": L2}, (1e4, 10.0, 10.0, 0.3, 0.3))
    assert not F1.any() and not F2.any() and not T1.any() and not T2.any()


def _random_rods(oracle_mod, n_rods, n_el, seed, box=0.3, length=0.2, radius=0.004):
    rng = np.random.default_rng(seed)
    R = oracle_mod.RodArrays([n_el] * n_rods)
    for r in range(n_rods):
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        nrm = np.cross(d, rng.normal(size=3))
        nrm /= np.linalg.norm(nrm)
        centre = rng.uniform(0.0, box, size=3)
        rod = oracle_mod.straight_rod(n_el, centre - 0.5 * length * d, d, nrm, length, radius, 1000.0, 1e6, 1e6 / 3)
        R.set_rod("x", r, rod["x"])
        R.set_rod("Q", r, rod["Q"].reshape(9, -1))
        for key, src in (("mass", "mass"), ("rest_length", "l0"), ("rest_voronoi", "D0"), ("volume", "V"),
                         ("shear_diag", "S"), ("bend_diag", "B"), ("inertia_diag", "J"), ("inv_inertia", "Jinv")):
            R.set_rod(key, r, rod[src])
        R.set_rod("v", r, rng.normal(scale=0.05, size=(3, n_el + 1)))
    return R


WALLS = [((0.0, 0.15, 0.15), (1.0, 0.0, 0.0), 0), ((0.3, 0.15, 0.15), (-1.0, 0.0, 0.0), 0),
         ((0.15, 0.0, 0.15), (0.0, 1.0, 0.0), 0), ((0.15, 0.3, 0.15), (0.0, -1.0, 0.0), 0),
         ((0.15, 0.15, 0.0), (0.0, 0.0, 1.0), 0), ((0.15, 0.15, 0.3), (0.0, 0.0, -1.0), 0)]


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_grid_search_equals_exhaustive(oracle_mod, seed):
    R = _random_rods(oracle_mod, 48, 16, seed)
    spec = oracle_mod.ContactSpec([[2e4, 20.0, 20.0, 0.15, 0.15]], [0] * 48, WALLS)
    for half_dt in (0.0, 5e-6):
        ex = oracle_mod.contact_pairs(R, spec, half_dt, exhaustive=True)
        gr = oracle_mod.contact_pairs(R, spec, half_dt, exhaustive=False)
        assert ex.shape[0] > 48 * 15  # adjacent capsules at least
        assert np.array_equal(ex, gr)
        # sorted, unique, a < b, planes after capsules
        assert (ex[:, 0] < ex[:, 1]).all()
        keys = ex[:, 0] * (R.n_slots + 16) + ex[:, 1]
        assert (np.diff(keys) > 0).all()


def test_rods_without_material_take_no_part(oracle_mod):
    R = _random_rods(oracle_mod, 12, 8, 7, box=0.05)
    mats = [0] * 12
    mats[3] = -1
    spec = oracle_mod.ContactSpec([[2e4, 20.0, 20.0, 0.15, 0.15]], mats, [])
    pairs = oracle_mod.contact_pairs(R, spec, 0.0)
    o3, o4 = R.offset[3], R.offset[4]
    assert not ((pairs >= o3) & (pairs < o4)).any()


def test_contact_step_momentum_balance(oracle_mod):
    """Rod-rod contact forces are internal to the system: with no gravity
    and no planes the total capsule force vanishes."""
    R = _random_rods(oracle_mod, 24, 16, 11, box=0.08)
    spec = oracle_mod.ContactSpec([[2e4, 20.0, 20.0, 0.15, 0.15]], [0] * 24, [])
    oracle_mod.contact_step(R, spec, 1e-5, 3)
    F = spec.capsule_force.reshape(3, -1)
    assert np.abs(F).max() > 0
    assert np.allclose(F.sum(axis=1), 0.0, atol=1e-9 * np.abs(F).sum())
