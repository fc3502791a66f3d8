"""ctypes front end of the CPU FP64 oracle (rod_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by bench.py's CPU-baseline leg, always as the checker or the timed CPU
baseline, never by the product package.

``RodArrays`` holds one ragged batch of rods in the slot layout described in
``rod_oracle.h`` (rod r owns slots ``offset[r] .. offset[r] + n_r``;
component-major fields).  It is deliberately independent of the product's
host code so that a layout bug on the product side cannot cancel out.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librod_oracle.so")

_P = ctypes.POINTER(ctypes.c_double)


class _OrcRods(ctypes.Structure):
    _fields_ = [
        ("n_rods", ctypes.c_int64),
        ("n_slots", ctypes.c_int64),
        ("offset", ctypes.POINTER(ctypes.c_int64)),
        ("x", _P), ("v", _P), ("Q", _P), ("w", _P),
        ("mass", _P), ("rest_length", _P), ("rest_voronoi", _P), ("volume", _P),
        ("rest_sigma", _P), ("rest_kappa", _P), ("shear_diag", _P), ("bend_diag", _P),
        ("inertia_diag", _P), ("inv_inertia", _P), ("nu_force", _P), ("nu_torque", _P),
        ("clamp", ctypes.POINTER(ctypes.c_uint8)), ("clamp_x", _P), ("clamp_Q", _P),
        ("end_torque", _P), ("damper_nu", _P),
        ("gravity", ctypes.c_double * 3),
        ("d_length", _P), ("d_dilatation", _P), ("d_tangent", _P), ("d_vdilatation", _P),
        ("d_sigma", _P), ("d_kappa", _P), ("d_stress", _P), ("d_couple", _P),
        ("d_loads", _P), ("d_torques", _P), ("d_accel", _P), ("d_alpha", _P),
        ("d_dimension", _P),
        ("clamp_index", ctypes.POINTER(ctypes.c_int64)), ("clamp2_x", _P), ("clamp2_Q", _P),
        ("torque_index", ctypes.POINTER(ctypes.c_int64)),
    ]


class _OrcContactMaterial(ctypes.Structure):
    _fields_ = [("stiffness", ctypes.c_double), ("normal_damping", ctypes.c_double),
                ("tangential_damping", ctypes.c_double), ("static_friction", ctypes.c_double),
                ("dynamic_friction", ctypes.c_double)]


class _OrcContact(ctypes.Structure):
    _fields_ = [
        ("n_materials", ctypes.c_int32),
        ("materials", ctypes.POINTER(_OrcContactMaterial)),
        ("rod_material", ctypes.POINTER(ctypes.c_int32)),
        ("n_planes", ctypes.c_int32),
        ("plane_point", _P), ("plane_normal", _P),
        ("plane_material", ctypes.POINTER(ctypes.c_int32)),
        ("capsule_force", _P), ("capsule_torque", _P),
    ]


_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (in-tree .so)."""
    if force or not os.path.exists(LIB_PATH) or (
        os.path.getmtime(LIB_PATH) < max(os.path.getmtime(os.path.join(HERE, f))
                                         for f in ("rod_oracle.cpp", "rod_oracle.h"))):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.orc_step.argtypes = [ctypes.POINTER(_OrcRods), ctypes.c_double, ctypes.c_int64, ctypes.c_int]
        _lib.orc_force_eval.argtypes = [ctypes.POINTER(_OrcRods), ctypes.c_int]
        _lib.orc_step_pefrl.argtypes = [ctypes.POINTER(_OrcRods), ctypes.c_double, ctypes.c_int64, ctypes.c_int]
        _lib.orc_step_velocity_verlet.argtypes = [ctypes.POINTER(_OrcRods), ctypes.c_double, ctypes.c_int64,
                                                  ctypes.c_int]
        _lib.orc_energy.argtypes = [ctypes.POINTER(_OrcRods), _P, ctypes.c_int]
        _lib.orc_straight_rod.argtypes = [ctypes.c_int64, _P, _P, _P, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_double, ctypes.c_double] + [_P] * 11
        _lib.orc_step_contact.argtypes = [ctypes.POINTER(_OrcRods), ctypes.POINTER(_OrcContact), ctypes.c_double,
                                          ctypes.c_int64, ctypes.c_int]
        _lib.orc_contact_capsules.argtypes = [ctypes.POINTER(_OrcRods), ctypes.POINTER(_OrcContact),
                                              ctypes.c_double, _P]
        _lib.orc_contact_pairs.argtypes = [ctypes.POINTER(_OrcRods), ctypes.POINTER(_OrcContact), ctypes.c_double,
                                           ctypes.c_int, ctypes.POINTER(ctypes.c_int64), ctypes.c_int64]
        _lib.orc_contact_pairs.restype = ctypes.c_int64
        for name in ("orc_fine_capsule_capsule", "orc_fine_capsule_plane"):
            getattr(_lib, name).argtypes = [_P, _P, _P]
        _lib.orc_fine_pair_loads.argtypes = [_P, _P, _P, _P]
        _lib.orc_so3_add_assign.argtypes = [_P, _P]
        _lib.orc_inv_rotate_divide.argtypes = [_P, _P, ctypes.c_double, _P]
        _lib.orc_step_loads.argtypes = [ctypes.POINTER(_OrcRods), ctypes.POINTER(_OrcContact),
                                        ctypes.POINTER(_OrcConnections), ctypes.c_double, ctypes.c_int64,
                                        ctypes.c_int]
    return _lib


STATE = ("x", "v", "Q", "w")
PARAMS = ("mass", "rest_length", "rest_voronoi", "volume", "rest_sigma", "rest_kappa",
          "shear_diag", "bend_diag", "inertia_diag", "inv_inertia")
DIAG = ("d_length", "d_dilatation", "d_tangent", "d_vdilatation", "d_sigma", "d_kappa",
        "d_stress", "d_couple", "d_loads", "d_torques", "d_accel", "d_alpha", "d_dimension")
NCOMP = {"x": 3, "v": 3, "Q": 9, "w": 3, "rest_sigma": 3, "rest_kappa": 3, "shear_diag": 3,
         "bend_diag": 3, "inertia_diag": 3, "inv_inertia": 3, "d_tangent": 3, "d_sigma": 3,
         "d_kappa": 3, "d_stress": 3, "d_couple": 3, "d_loads": 3, "d_torques": 3,
         "d_accel": 3, "d_alpha": 3}


def straight_rod(n, origin, direction, normal, length, radius, density, youngs, shear):
    """Reference straight-rod initializer for one rod; returns a dict of
    per-rod arrays in the reference's shapes (3 x N, 3 x 3 x N, N)."""
    L = lib()
    n = int(n)
    out = {
        "x": np.zeros(3 * (n + 1)), "Q": np.zeros(9 * n), "l0": np.zeros(n), "D0": np.zeros(n - 1),
        "V": np.zeros(n), "radius": np.zeros(n), "mass": np.zeros(n + 1), "J": np.zeros(3 * n),
        "Jinv": np.zeros(3 * n), "S": np.zeros(3 * n), "B": np.zeros(3 * (n - 1)),
    }
    f = lambda a: np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(_P)
    o, d, nm = (np.asarray(a, dtype=np.float64) for a in (origin, direction, normal))
    rc = L.orc_straight_rod(n, f(o), f(d), f(nm), float(length), float(radius), float(density),
                            float(youngs), float(shear), *(out[k].ctypes.data_as(_P) for k in
                                                           ("x", "Q", "l0", "D0", "V", "radius", "mass", "J", "Jinv", "S", "B")))
    if rc != 0:
        raise ValueError("invalid straight rod parameters")
    out["x"] = out["x"].reshape(3, n + 1)
    out["Q"] = out["Q"].reshape(3, 3, n)
    for k in ("J", "Jinv", "S"):
        out[k] = out[k].reshape(3, n)
    out["B"] = out["B"].reshape(3, n - 1)
    return out


class RodArrays:
    """Slot-layout batch of rods for the oracle."""

    def __init__(self, n_elems, damped: bool = False):
        self.n_elems = np.asarray(n_elems, dtype=np.int64)
        self.n_rods = len(self.n_elems)
        self.offset = np.zeros(self.n_rods + 1, dtype=np.int64)
        np.cumsum(self.n_elems + 1, out=self.offset[1:])
        S = self.n_slots = int(self.offset[-1])
        self.arrays = {}
        for k in STATE + PARAMS:
            self.arrays[k] = np.zeros(NCOMP.get(k, 1) * S)
        self.damped = damped
        if damped:
            self.arrays["nu_force"] = np.zeros(S)
            self.arrays["nu_torque"] = np.zeros(S)
        self.clamp = np.zeros(self.n_rods, dtype=np.uint8)
        self.clamp_x = np.zeros(3 * self.n_rods)
        self.clamp_Q = np.zeros(9 * self.n_rods)
        # clamp c of rod r at index clamp_index[2r + c] (-1: none; clamp 0 at
        # index 0 by default), targets clamp_x / clamp_Q (c = 0) or
        # clamp2_x / clamp2_Q (c = 1); end_torque at element torque_index[r]
        # (-1: the last element)
        self.clamp_index = np.tile(np.array([0, -1], dtype=np.int64), self.n_rods)
        self.clamp2_x = np.zeros(3 * self.n_rods)
        self.clamp2_Q = np.zeros(9 * self.n_rods)
        self.torque_index = np.full(self.n_rods, -1, dtype=np.int64)
        self.end_torque = np.zeros(3 * self.n_rods)
        self.damper_nu = np.zeros(2 * self.n_rods)
        self.gravity = np.zeros(3)
        self.diag = None

    # -- per-rod views in the reference's shapes --------------------------
    def comp(self, key):
        a = self.arrays[key]
        return a.reshape(NCOMP.get(key, 1), self.n_slots)

    def rod_view(self, key, r, count):
        """(ncomp, count) view of rod r's first `count` slots."""
        o = int(self.offset[r])
        return self.comp(key)[:, o:o + count]

    def set_rod(self, key, r, values):
        values = np.asarray(values, dtype=np.float64)
        nc = NCOMP.get(key, 1)
        values = values.reshape(nc, -1)
        self.rod_view(key, r, values.shape[1])[...] = values

    def get_rod(self, key, r, count):
        return self.rod_view(key, r, count).copy()

    def enable_diagnostics(self):
        self.diag = {k: np.zeros(NCOMP.get(k, 1) * self.n_slots) for k in DIAG}

    def get_diag(self, key, r, count):
        o = int(self.offset[r])
        return self.diag[key].reshape(NCOMP.get(key, 1), self.n_slots)[:, o:o + count].copy()

    # -- ctypes struct -----------------------------------------------------
    def _struct(self):
        s = _OrcRods()
        s.n_rods = self.n_rods
        s.n_slots = self.n_slots
        s.offset = self.offset.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
        for k, a in self.arrays.items():
            setattr(s, k, a.ctypes.data_as(_P))
        s.clamp = self.clamp.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
        s.clamp_x = self.clamp_x.ctypes.data_as(_P)
        s.clamp_Q = self.clamp_Q.ctypes.data_as(_P)
        s.end_torque = self.end_torque.ctypes.data_as(_P)
        s.damper_nu = self.damper_nu.ctypes.data_as(_P)
        s.clamp_index = self.clamp_index.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
        s.clamp2_x = self.clamp2_x.ctypes.data_as(_P)
        s.clamp2_Q = self.clamp2_Q.ctypes.data_as(_P)
        s.torque_index = self.torque_index.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
        for i in range(3):
            s.gravity[i] = float(self.gravity[i])
        if self.diag is not None:
            for k, a in self.diag.items():
                setattr(s, k, a.ctypes.data_as(_P))
        return s

    def step(self, dt, n_steps=1, n_threads=0, stepper="position_verlet"):
        s = self._struct()
        fn = {"pefrl": lib().orc_step_pefrl, "velocity_verlet": lib().orc_step_velocity_verlet,
              "position_verlet": lib().orc_step}[stepper]
        rc = fn(ctypes.byref(s), float(dt), int(n_steps), int(n_threads))
        if rc != 0:
            raise RuntimeError("orc_step failed")

    def force_eval(self):
        s = self._struct()
        if lib().orc_force_eval(ctypes.byref(s), 0) != 0:
            raise RuntimeError("orc_force_eval failed")

    def energy(self):
        out = np.zeros(4 * self.n_rods)
        s = self._struct()
        if lib().orc_energy(ctypes.byref(s), out.ctypes.data_as(_P), 0) != 0:
            raise RuntimeError("orc_energy failed")
        return out.reshape(self.n_rods, 4)

    def copy(self):
        c = RodArrays.__new__(RodArrays)
        c.__dict__.update(self.__dict__)
        c.arrays = {k: a.copy() for k, a in self.arrays.items()}
        for k in ("clamp", "clamp_x", "clamp_Q", "end_torque", "damper_nu", "gravity", "clamp_index", "clamp2_x",
                  "clamp2_Q", "torque_index"):
            setattr(c, k, getattr(self, k).copy())
        c.diag = None if self.diag is None else {k: a.copy() for k, a in self.diag.items()}
        return c


class ContactSpec:
    """Collision-system description for the oracle: per-material contact
    parameters (stiffness, normal damping, tangential damping, static and
    dynamic friction), the material of each rod (-1: no contact) and planes
    (point, normal, material)."""

    def __init__(self, materials, rod_material, planes=()):
        self.materials = np.asarray(materials, dtype=np.float64).reshape(-1, 5)
        self.rod_material = np.ascontiguousarray(rod_material, dtype=np.int32)
        self.planes = list(planes)
        self.plane_point = np.array([p[0] for p in self.planes], dtype=np.float64).reshape(-1)
        self.plane_normal = np.array([p[1] for p in self.planes], dtype=np.float64).reshape(-1)
        self.plane_material = np.array([p[2] for p in self.planes], dtype=np.int32)
        if self.plane_point.size == 0:
            self.plane_point = np.zeros(3)
            self.plane_normal = np.zeros(3)
            self.plane_material = np.zeros(1, dtype=np.int32)
        self._mats = (_OrcContactMaterial * max(1, len(self.materials)))()
        for i, m in enumerate(self.materials):
            self._mats[i] = _OrcContactMaterial(*[float(v) for v in m])
        self.capsule_force = None
        self.capsule_torque = None

    def _struct(self, n_slots):
        c = _OrcContact()
        c.n_materials = len(self.materials)
        c.materials = ctypes.cast(self._mats, ctypes.POINTER(_OrcContactMaterial))
        c.rod_material = self.rod_material.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        c.n_planes = len(self.planes)
        c.plane_point = self.plane_point.ctypes.data_as(_P)
        c.plane_normal = self.plane_normal.ctypes.data_as(_P)
        c.plane_material = self.plane_material.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        if self.capsule_force is None or self.capsule_force.size != 3 * n_slots:
            self.capsule_force = np.zeros(3 * n_slots)
            self.capsule_torque = np.zeros(3 * n_slots)
        c.capsule_force = self.capsule_force.ctypes.data_as(_P)
        c.capsule_torque = self.capsule_torque.ctypes.data_as(_P)
        return c


_I64 = ctypes.POINTER(ctypes.c_int64)


class _OrcConnections(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("rod_a", _I64), ("index_a", _I64), ("rod_b", _I64), ("index_b", _I64),
                ("kind", ctypes.POINTER(ctypes.c_int32)), ("k", _P), ("nu", _P), ("k_rot", _P), ("normal", _P)]


class ConnectionSpec:
    """Connections for the oracle, in order: (rod_a, index_a, rod_b, index_b,
    kind (0 free, 1 hinge), k, nu, k_rot, normal(3))."""

    def __init__(self, connections):
        c = list(connections)
        self.n = len(c)
        col = lambda i, dt: np.ascontiguousarray([x[i] for x in c] or [0], dtype=dt)
        self.rod_a, self.index_a = col(0, np.int64), col(1, np.int64)
        self.rod_b, self.index_b = col(2, np.int64), col(3, np.int64)
        self.kind = col(4, np.int32)
        self.k, self.nu, self.k_rot = col(5, np.float64), col(6, np.float64), col(7, np.float64)
        self.normal = np.ascontiguousarray(np.array([x[8] for x in c] or [[0.0, 0.0, 0.0]],
                                                    dtype=np.float64).reshape(-1))

    def _struct(self):
        s = _OrcConnections()
        s.n = self.n
        s.rod_a, s.index_a = self.rod_a.ctypes.data_as(_I64), self.index_a.ctypes.data_as(_I64)
        s.rod_b, s.index_b = self.rod_b.ctypes.data_as(_I64), self.index_b.ctypes.data_as(_I64)
        s.kind = self.kind.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        s.k, s.nu, s.k_rot = self.k.ctypes.data_as(_P), self.nu.ctypes.data_as(_P), self.k_rot.ctypes.data_as(_P)
        s.normal = self.normal.ctypes.data_as(_P)
        return s


def loads_step(rods: RodArrays, contact: "ContactSpec | None", connections: ConnectionSpec | None, dt,
               n_steps=1, n_threads=0):
    """PositionVerlet steps with the collision system and/or connections
    (orc_step_loads)."""
    s = rods._struct()
    c = contact._struct(rods.n_slots) if contact is not None else None
    j = connections._struct() if connections is not None else None
    rc = lib().orc_step_loads(ctypes.byref(s), ctypes.byref(c) if c is not None else None,
                              ctypes.byref(j) if j is not None else None, float(dt), int(n_steps), int(n_threads))
    if rc != 0:
        raise RuntimeError("orc_step_loads failed")


def contact_step(rods: RodArrays, spec: ContactSpec, dt, n_steps=1, n_threads=0):
    """PositionVerlet steps with the collision system (orc_step_contact)."""
    s = rods._struct()
    c = spec._struct(rods.n_slots)
    if lib().orc_step_contact(ctypes.byref(s), ctypes.byref(c), float(dt), int(n_steps), int(n_threads)) != 0:
        raise RuntimeError("orc_step_contact failed")


def contact_capsules(rods: RodArrays, spec: ContactSpec, half_dt=0.0):
    """(14, n_slots) capsule table after a drift of half_dt: centre(3),
    length, radius, axis(3), AABB min(3), AABB max(3); NaN where no capsule."""
    out = np.full(14 * rods.n_slots, np.nan)
    s = rods._struct()
    c = spec._struct(rods.n_slots)
    if lib().orc_contact_capsules(ctypes.byref(s), ctypes.byref(c), float(half_dt), out.ctypes.data_as(_P)) != 0:
        raise RuntimeError("orc_contact_capsules failed")
    return out.reshape(14, rods.n_slots)


def contact_pairs(rods: RodArrays, spec: ContactSpec, half_dt=0.0, exhaustive=True):
    """Sorted candidate pairs (k, 2) int64 of the capsules after a drift of
    half_dt; plane p appears as n_slots + p."""
    s = rods._struct()
    c = spec._struct(rods.n_slots)
    n = lib().orc_contact_pairs(ctypes.byref(s), ctypes.byref(c), float(half_dt), int(bool(exhaustive)), None, 0)
    if n < 0:
        raise RuntimeError("orc_contact_pairs failed")
    out = np.zeros(2 * max(n, 1), dtype=np.int64)
    n2 = lib().orc_contact_pairs(ctypes.byref(s), ctypes.byref(c), float(half_dt), int(bool(exhaustive)),
                                 out.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), int(n))
    assert n2 == n
    return out[:2 * n].reshape(n, 2)


def _capsule_desc(c):
    d = np.zeros(14)
    d[0:3] = c["centre"]
    d[3:6] = c["axis"]
    d[6] = c["radius"]
    d[7] = c["length"]
    d[8:11] = c.get("velocity", (0.0, 0.0, 0.0))
    d[11:14] = c.get("omega", (0.0, 0.0, 0.0))
    return d


def fine_capsule_capsule(a, b):
    """Contacts [(position, normal, distance)] of two rod capsules (dicts with
    centre, axis, radius, length[, velocity, omega]), a being the first body."""
    out = np.zeros(14)
    da, db = _capsule_desc(a), _capsule_desc(b)
    n = lib().orc_fine_capsule_capsule(da.ctypes.data_as(_P), db.ctypes.data_as(_P), out.ctypes.data_as(_P))
    return [(out[7 * i:7 * i + 3].copy(), out[7 * i + 3:7 * i + 6].copy(), float(out[7 * i + 6])) for i in range(n)]


def fine_capsule_plane(c, point, normal):
    out = np.zeros(14)
    dc = _capsule_desc(c)
    pl = np.concatenate([np.asarray(point, float), np.asarray(normal, float)])
    n = lib().orc_fine_capsule_plane(dc.ctypes.data_as(_P), pl.ctypes.data_as(_P), out.ctypes.data_as(_P))
    return [(out[7 * i:7 * i + 3].copy(), out[7 * i + 3:7 * i + 6].copy(), float(out[7 * i + 6])) for i in range(n)]


def fine_pair_loads(a, b, pair_material):
    """(force1, torque1, force2, torque2) of the spring-dashpot over all
    contacts of the capsule pair; pair_material = (k, c_n, c_t, mu_s, mu_d)."""
    out = np.zeros(12)
    da, db = _capsule_desc(a), _capsule_desc(b)
    pm = np.asarray(pair_material, dtype=np.float64)
    lib().orc_fine_pair_loads(da.ctypes.data_as(_P), db.ctypes.data_as(_P), pm.ctypes.data_as(_P),
                              out.ctypes.data_as(_P))
    return out.reshape(4, 3)
