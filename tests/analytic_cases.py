"""Closed-form cases that pin the analytical damper and the rod energies
independently of the oracle and of the reference's (absent) numbers.

Rod: one straight rod along +x (normal +y, so d1 = +y, d2 = +z, d3 = +x),
n elements of length l0 = L / n, radius r, density rho, E, G = E / 3, free
(no clamp, no gravity).  With A = pi r^2, I1 = A^2 / (4 pi), M = rho A L:

* Analytical damper (examples/fish_swimming/FishModel/Dissipations/
  AnalyticalLinearDamper.hpp:15-79, physical version), rod translating with
  velocity v0 at every node and spinning about its axis at w0 (material
  frame (0, 0, w0)) on every element.  The velocity is normal to the rod,
  so every node's y and z stay equal and its x does not move: element
  lengths, tangents and directors' tangent rows stay exact, every element
  keeps the same directors, and the internal loads are exactly zero (no
  strain, no curvature, no transport or dilatation term).  Each step then
  only multiplies:
      v_k = v0 exp(-nu_t dt)^k,
      w3_k = w0 (exp(-nu_r m_e J^-1_3 dt) ^ e)^k,   e = 1,
  where the element mass m_e = rho A l0 (interior nodes carry rho A l0, end
  nodes half of it, and the end elements add the other half) and
  J^-1_3 = 1 / (2 I1 rho l0), so m_e J^-1_3 = 2 / r^2 for every element:
      w3_k = w0 exp(-nu_r (2 / r^2) dt k).
* Energies (elastica/Systems/CosseratRods/Utility/Energy.hpp:46-141):
  translating rod: translational 1/2 M |v0|^2; spinning rod: rotational
  1/2 sum J3 w0^2 / e = 1/4 M r^2 w0^2 (the solid cylinder's axial moment);
  uniformly stretched rod (every element length (1 + eps) l0, directors
  unchanged): shear 1/2 sum S3 eps^2 l0 = 1/2 E A eps^2 L; uniformly bent
  rod (element i's directors turned about d1 by kappa (i + 1/2) l0): bend
  1/2 sum B1 kappa^2 D0 = 1/2 E I1 kappa^2 (L - l0), from the n - 1 interior
  Voronoi points of length l0.  The reference's curvature takes
  theta = acos(cos(phi) - 1e-10) for the relative angle phi = kappa l0, but
  the curvature is theta sin(phi) / (sin(theta + 1e-14) l0), so the shift
  moves it by about 1e-10 / 3 relative at phi = 0.05 (theta / sin(theta) is
  flat near 0): the bend energy is pinned to 1e-9.
"""
from __future__ import annotations

import numpy as np

N = 50
LENGTH = 1.0
RADIUS = 0.02
DENSITY = 1000.0
YOUNGS = 1e6
SHEAR = YOUNGS / 3.0
AREA = np.pi * RADIUS ** 2
I1 = AREA ** 2 / (4.0 * np.pi)
MASS = DENSITY * AREA * LENGTH
L0 = LENGTH / N

V0 = np.array([0.0, -0.2, 0.1])  # normal to the rod (along +x)
W0 = 2.0
NU_T, NU_R = 5.0, 0.01
DT = 1e-4
STEPS = 200
EPS = 1e-3
KAPPA = 2.5  # 1/m: relative angle kappa l0 = 0.05 rad per Voronoi point


def straight_rod(eb):
    return eb.StraightRod(n_elements=N, material=eb.Material(DENSITY, YOUNGS, SHEAR), radius=RADIUS,
                          length=LENGTH, origin=(0.0, 0.0, 0.0), direction=(1.0, 0.0, 0.0),
                          normal=(0.0, 1.0, 0.0))


def translating_velocity() -> np.ndarray:
    return np.repeat(V0[:, None], N + 1, axis=1)


def spinning_omega() -> np.ndarray:
    w = np.zeros((3, N))
    w[2] = W0
    return w


def stretched_positions() -> np.ndarray:
    x = np.zeros((3, N + 1))
    x[0] = np.arange(N + 1) * ((1.0 + EPS) * L0)
    return x


def bent_directors() -> np.ndarray:
    """Q(k, j, i): component j of director k of element i; element i turned
    about d1 = +y by kappa (i + 1/2) l0 (d1 stays +y)."""
    q = np.zeros((3, 3, N))
    a = KAPPA * (np.arange(N) + 0.5) * L0
    c, s = np.cos(a), np.sin(a)
    # d1 = +y; d3 = tangent turned from +x towards -z; d2 = d3 x d1
    q[0, 1] = 1.0
    q[2, 0], q[2, 2] = c, -s
    q[1, 0], q[1, 2] = s, c
    return q


def damped_velocity(k: int) -> np.ndarray:
    return V0 * np.exp(-NU_T * DT) ** k


def damped_spin(k: int) -> float:
    return W0 * np.exp(-NU_R * (2.0 / RADIUS ** 2) * DT * k)


def translational_energy() -> float:
    return 0.5 * MASS * float(V0 @ V0)


def rotational_energy() -> float:
    return 0.25 * MASS * RADIUS ** 2 * W0 ** 2


def shear_energy() -> float:
    return 0.5 * YOUNGS * AREA * EPS ** 2 * LENGTH


def bend_energy() -> float:
    return 0.5 * YOUNGS * I1 * KAPPA ** 2 * (LENGTH - L0)


def rel(a, b) -> float:
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / np.max(np.abs(b)))
