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
  circle in both senses, margin 1e-16 on top of Catch's default epsilon).
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
