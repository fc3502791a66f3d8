"""The oracle's element kernels against the reference's own kernel tests.

Test infrastructure: the SO(3) director update and the curvature kernel that
the oracle's step uses, checked one element at a time against

* ``tests/Unit/Systems/States/Expressions/SO3/Test_SO3PrimitiveAddAssign.cpp:36-132``:
  the identity director rotated by u = dt * 76 deg * (1, 3.2, 7) / |(1, 3.2, 7)|
  once and twice, compared with the expected directors it lists (extracted as
  text into ``tests/golden/so3_add_assign.json`` by ``make_golden.py``) under
  the reference's default ``approx`` (epsilon 100 DBL_EPSILON, scale 1,
  ``tests/Unit/Framework/TestingFramework.hpp:76-79``);
* ``tests/Unit/Systems/CosseratRods/Traits/Operations/BlazeBackend/Test_InvRotateDivide_Scalar.cpp``:
  ``correctness`` (lines 26-61: two directors a 120 deg rotation about
  (1, 1, 1) apart, divided by 0.25, epsilon 1.3e-10) and
  ``circle_in_two_dimensions`` (lines 62-135: 512 directors around a planar
  circle in both senses, margin 1e-16 on top of Catch's default epsilon);

and, through the oracle's force evaluation, the pattern of
``tests/Unit/Systems/CosseratRods/Components/Elasticity/Test_WithDiagonalLinearHyperElasticModel.cpp:183-249``
(uniformly strained rods: loads at the end nodes only, equal interior torques).
"""
import ctypes
import math

import numpy as np
import pytest

import goldens

DBL_EPS = np.finfo(np.float64).eps
FLT_EPS = float(np.finfo(np.float32).eps)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _so3(lib, q: np.ndarray, u: np.ndarray) -> None:
    assert lib.orc_so3_add_assign(_ptr(q), _ptr(u)) == 0


def _curvature(lib, qc: np.ndarray, qn: np.ndarray, span: float) -> np.ndarray:
    out = np.zeros(3)
    qc = np.ascontiguousarray(qc, dtype=np.float64)
    qn = np.ascontiguousarray(qn, dtype=np.float64)
    assert lib.orc_inv_rotate_divide(_ptr(qc), _ptr(qn), span, _ptr(out)) == 0
    return out


def _catch(a, b, *, eps, scale=0.0, margin=0.0) -> bool:
    """Catch2's ``a == Approx(b)``: |a - b| <= margin, or
    |a - b| <= eps * (scale + |b|), for every entry."""
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    d = np.abs(a - b)
    return bool(np.all((d <= margin) | (d <= eps * (scale + np.abs(b)))))


def test_so3_fixture_inputs():
    doc = goldens.load("so3_add_assign")
    assert [float.fromhex(h) for h in doc["direction"]] == [1.0, 3.2, 7.0]
    assert float.fromhex(doc["angle_deg"]) == 76.0
    assert float.fromhex(doc["time_delta"]) == 1.0
    assert [e["applications"] for e in doc["expected"]] == [1, 2, 3]


def test_so3_add_assign_expected_rotations(oracle_mod):
    """One and two applications (the two the reference checks) within its
    default approx; the third listed director, which the reference declares
    but never checks, within the same bound."""
    lib = oracle_mod.lib()
    doc = goldens.load("so3_add_assign")
    direction = np.array([float.fromhex(h) for h in doc["direction"]])
    # Test_SO3PrimitiveAddAssign.cpp:75-77, 95: unit direction times the angle, times dt
    u = direction / np.linalg.norm(direction)
    u = u * (float.fromhex(doc["angle_deg"]) * math.pi / 180.0)
    u = float.fromhex(doc["time_delta"]) * u
    q = np.eye(3).ravel().copy()
    for entry in doc["expected"]:
        _so3(lib, q, u)
        want = np.array([float.fromhex(h) for h in entry["hex"]])
        assert _catch(q, want, eps=100 * DBL_EPS, scale=1.0), (entry["name"], q - want)


def test_so3_zero_rotation_is_identity_map(oracle_mod):
    # the 1e-14 guard of SO3PrimitiveAddAssign/Scalar.hpp keeps u = 0 finite
    lib = oracle_mod.lib()
    rng = np.random.default_rng(3)
    q0, _ = np.linalg.qr(rng.standard_normal((3, 3)))
    q = q0.ravel().copy()
    _so3(lib, q, np.zeros(3))
    assert np.array_equal(q, q0.ravel())


def test_so3_keeps_directors_orthonormal(oracle_mod):
    """Orthogonality is kept to rounding.  The row norms move only by the
    1e-14 guard: the axis u / (theta + 1e-14) is short of unit length by
    1e-14 / theta, which changes a row's squared norm by at most about
    theta * 1e-14 per application (Rodrigues' formula with a scaled axis)."""
    lib = oracle_mod.lib()
    rng = np.random.default_rng(11)
    q = np.eye(3).ravel().copy()
    guard_budget = 0.0
    for _ in range(1000):
        u = rng.normal(scale=0.3, size=3)
        guard_budget += np.linalg.norm(u) * 1e-14
        _so3(lib, q, u)
    m = q.reshape(3, 3)
    gram = m @ m.T
    assert np.abs(gram - np.diag(np.diag(gram))).max() < 1e-13
    assert np.abs(np.diag(gram) - 1.0).max() < 2.0 * guard_budget + 1e-13


def test_inv_rotate_divide_correctness(oracle_mod):
    """Directors I and the cyclic permutation (d1, d2, d3) = (y, z, x): a
    120 degree rotation about (1, 1, 1) / sqrt(3); divided by 0.25."""
    lib = oracle_mod.lib()
    qc = np.eye(3).ravel()
    qn = np.array([[0.0, 1.0, 0.0], [0.0, 0.0, 1.0], [1.0, 0.0, 0.0]]).ravel()
    ratio = 0.25
    k = _curvature(lib, qc, qn, ratio)
    angle = np.linalg.norm(k)
    assert _catch(angle, 120.0 * math.pi / 180.0 / ratio, eps=1.3e-10)
    assert _catch(k / angle, np.full(3, 1.0 / math.sqrt(3.0)), eps=1.3e-10)


@pytest.mark.parametrize("sense", ["anticlockwise", "clockwise"])
def test_inv_rotate_divide_circle_in_two_dimensions(oracle_mod, sense):
    lib = oracle_mod.lib()
    n = 512
    if sense == "anticlockwise":
        theta = np.linspace(0.0, 2.0 * math.pi, n)
        axis = np.array([0.0, 0.0, -1.0])
    else:
        theta = np.linspace(2.0 * math.pi, 0.0, n)
        axis = np.array([0.0, 0.0, 1.0])
    dtheta = abs(theta[1] - theta[0])
    # d1 normal, d2 tangent, d3 = -z (Test_InvRotateDivide_Scalar.cpp:99-115)
    q = np.zeros((n, 3, 3))
    q[:, 0, 0], q[:, 0, 1] = -np.cos(theta), -np.sin(theta)
    q[:, 1, 0], q[:, 1, 1] = -np.sin(theta), np.cos(theta)
    q[:, 2, 2] = -1.0
    for i in range(n - 1):
        k = _curvature(lib, q[i].ravel(), q[i + 1].ravel(), 1.0)
        scale = np.linalg.norm(k)
        assert _catch(k / scale, axis, eps=100 * FLT_EPS, margin=1e-16), (i, k)
        assert _catch(scale, dtheta, eps=100 * FLT_EPS, margin=1e-16), (i, scale, dtheta)


def _stretched_rod(oracle_mod, stretch: float, tilt: float = 0.0):
    """One rod of 8 elements along +z, rest length 0.125 per element, every
    node moved to ``stretch`` times its rest position (exactly representable
    for the stretches used), every director turned by ``tilt`` about d1, at
    rest (v = w = 0).  Returns the oracle's rod arrays with diagnostics on."""
    n = 8
    init = oracle_mod.straight_rod(n, (0.0, 0.0, 0.0), (0.0, 0.0, 1.0), (1.0, 0.0, 0.0), 1.0, 0.05, 1000.0,
                                   1e6, 1e6 / 3)
    assert np.array_equal(init["x"][2], 0.125 * np.arange(n + 1))
    rods = oracle_mod.RodArrays([n])
    for key, src in (("mass", "mass"), ("rest_length", "l0"), ("rest_voronoi", "D0"), ("volume", "V"),
                     ("shear_diag", "S"), ("bend_diag", "B"), ("inertia_diag", "J"), ("inv_inertia", "Jinv")):
        rods.set_rod(key, 0, init[src])
    rods.set_rod("x", 0, init["x"] * stretch)
    c, s = math.cos(tilt), math.sin(tilt)
    turn = np.array([[1.0, 0.0, 0.0], [0.0, c, s], [0.0, -s, c]])
    q = init["Q"].transpose(2, 0, 1)  # (element, director, component)
    q = np.einsum("ab,ebj->eaj", turn, q) if tilt else q
    rods.set_rod("Q", 0, q.transpose(1, 2, 0).reshape(9, n))
    rods.enable_diagnostics()
    rods.force_eval()
    return rods, init, n


def test_uniform_stretch_loads_at_the_ends_only(oracle_mod):
    """The pattern of the reference's elasticity component test
    (Components/Elasticity/Test_WithDiagonalLinearHyperElasticModel.cpp:183-209):
    a uniformly strained rod has internal loads +Q^T n_L / e on the first node,
    the opposite on the last and exactly zero in between.  Pure stretch along
    d3 gives n_L = (0, 0, S3 (e - 1)), no couple and no torque."""
    rods, init, n = _stretched_rod(oracle_mod, 1.125)
    loads = rods.get_diag("d_loads", 0, n + 1)
    torques = rods.get_diag("d_torques", 0, n)
    e = 1.125
    s3 = init["S"][2, 0]
    edge = np.array([0.0, 0.0, s3 * (e - 1.0) / e])
    assert np.all(loads[:, 1:n] == 0.0)
    assert _catch(loads[:, 0], edge, eps=1e-15, margin=1e-300)
    assert np.array_equal(loads[:, n], -loads[:, 0])
    assert np.all(torques == 0.0)


def test_uniform_shear_interior_terms_cancel(oracle_mod):
    """Directors turned uniformly against the tangent: every element carries
    the same shear strain, so interior node loads cancel exactly and every
    interior element sees the same torque (shear couple, no curvature
    gradient), while the end elements differ by the boundary terms."""
    rods, _, n = _stretched_rod(oracle_mod, 1.0, tilt=0.01)
    loads = rods.get_diag("d_loads", 0, n + 1)
    torques = rods.get_diag("d_torques", 0, n)
    assert np.all(loads[:, 1:n] == 0.0)
    assert np.array_equal(loads[:, n], -loads[:, 0])
    assert np.abs(loads[1, 0]) > 0.0  # the shear component of n_L
    mid = torques[:, 1]
    for i in range(2, n - 1):
        assert np.array_equal(torques[:, i], mid), i
    assert np.abs(mid[0]) > 0.0  # (Q t) x n_L about d1
