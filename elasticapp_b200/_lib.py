"""ctypes binding of libelastica_b200.so (declared in include/elastica_b200.h).

This is the binding a maintainer of the reference's Python layer would add:
plain pointers and sizes, no torch types.  The library must exist: there is
no CPU fallback, and a missing or unbuildable library raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libelastica_b200.so")

EB_OK = 0
STATUS_NAMES = {0: "EB_OK", 1: "EB_ERR_INVALID_ARGUMENT", 2: "EB_ERR_INVALID_STATE",
                3: "EB_ERR_UNSUPPORTED", 4: "EB_ERR_OUT_OF_MEMORY", 5: "EB_ERR_CUDA",
                6: "EB_ERR_NOT_FOUND", 7: "EB_ERR_NUMERICAL"}
EB_ERR_INVALID_ARGUMENT = 1
EB_ERR_CUDA = 5

EB_PRECISION_FP64 = 0
EB_PRECISION_MIXED = 1
EB_FLAG_RECORD_DIAGNOSTICS = 0x1
EB_FLAG_REFERENCE_ROUNDING = 0x2
EB_FLAG_STEP_STREAMING = 0x4
EB_FLAG_STEP_RESIDENT = 0x8
EB_FLAG_CUDA_GRAPH = 0x10
EB_FLAG_STEP_BUCKETED = 0x20
EB_STEPPER_POSITION_VERLET = 0
EB_STEPPER_PEFRL = 1
EB_STEPPER_VELOCITY_VERLET = 2
EB_ROD_DAMPED = 0
EB_ROD_UNDAMPED = 1
EB_LAYOUT_PER_ROD = 0
EB_LAYOUT_SLOTS = 1

# eb_field, in the order of include/elastica_b200.h
FIELDS = [
    "Position", "Velocity", "Director", "AngularVelocity", "Mass", "ReferenceElementLength",
    "ReferenceVoronoiLength", "ElementVolume", "ReferenceShearStretchStrain", "ReferenceCurvature",
    "ShearStretchRigidityMatrix", "BendingTwistRigidityMatrix", "MassSecondMomentOfInertia",
    "InvMassSecondMomentOfInertia", "ForceDampingRate", "TorqueDampingRate", "ElementLength",
    "ElementDilatation", "Tangent", "VoronoiDilatation", "ShearStretchStrain", "Curvature",
    "InternalStress", "InternalCouple", "InternalLoads", "InternalTorques", "Acceleration",
    "AngularAcceleration", "ElementDimension", "ContactForce", "ContactTorque",
]
FIELD_ID = {name: i for i, name in enumerate(FIELDS)}
# (place, ncomp): place 0 = nodes (n+1), 1 = elements (n), 2 = Voronoi (n-1)
FIELD_SHAPE = {
    "Position": (0, 3), "Velocity": (0, 3), "Director": (1, 9), "AngularVelocity": (1, 3),
    "Mass": (0, 1), "ReferenceElementLength": (1, 1), "ReferenceVoronoiLength": (2, 1),
    "ElementVolume": (1, 1), "ReferenceShearStretchStrain": (1, 3), "ReferenceCurvature": (2, 3),
    "ShearStretchRigidityMatrix": (1, 3), "BendingTwistRigidityMatrix": (2, 3),
    "MassSecondMomentOfInertia": (1, 3), "InvMassSecondMomentOfInertia": (1, 3),
    "ForceDampingRate": (0, 1), "TorqueDampingRate": (1, 1), "ElementLength": (1, 1),
    "ElementDilatation": (1, 1), "Tangent": (1, 3), "VoronoiDilatation": (2, 1),
    "ShearStretchStrain": (1, 3), "Curvature": (2, 3), "InternalStress": (1, 3),
    "InternalCouple": (2, 3), "InternalLoads": (0, 3), "InternalTorques": (1, 3),
    "Acceleration": (0, 3), "AngularAcceleration": (1, 3), "ElementDimension": (1, 1),
    "ContactForce": (1, 3), "ContactTorque": (1, 3),
}
DERIVED_FIELDS = set(FIELDS[16:29])
CONTACT_FIELDS = {"ContactForce", "ContactTorque"}


class EbConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("flags", ctypes.c_uint32), ("step_window", ctypes.c_int32),
                ("resident_config", ctypes.c_int32), ("stepper", ctypes.c_int32)]


class EbStraightRod(ctypes.Structure):
    _fields_ = [("n_elements", ctypes.c_int64), ("model", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("density", ctypes.c_double), ("youngs_modulus", ctypes.c_double),
                ("shear_modulus", ctypes.c_double), ("radius", ctypes.c_double),
                ("length", ctypes.c_double), ("origin", ctypes.c_double * 3),
                ("direction", ctypes.c_double * 3), ("normal", ctypes.c_double * 3),
                ("force_damping_rate", ctypes.c_double), ("torque_damping_rate", ctypes.c_double)]


class EbContactMaterial(ctypes.Structure):
    _fields_ = [("stiffness", ctypes.c_double), ("normal_damping", ctypes.c_double),
                ("tangential_damping", ctypes.c_double), ("static_friction", ctypes.c_double),
                ("dynamic_friction", ctypes.c_double)]


class EbServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("precision", ctypes.c_int32), ("steps_per_launch", ctypes.c_int32),
                ("flags", ctypes.c_uint32), ("hbm_budget_bytes", ctypes.c_double),
                ("energy_tolerance", ctypes.c_double)]


class EbRequest(ctypes.Structure):
    _fields_ = [("rods", ctypes.POINTER(EbStraightRod)), ("n_rods", ctypes.c_int64),
                ("velocities", ctypes.POINTER(ctypes.c_double)), ("dt", ctypes.c_double),
                ("n_steps", ctypes.c_int64), ("gravity", ctypes.c_double * 3), ("options", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32), ("damper_translational", ctypes.c_double),
                ("damper_rotational", ctypes.c_double)]


class EbCompletion(ctypes.Structure):
    _fields_ = [("request_id", ctypes.c_int64), ("precision", ctypes.c_int32), ("fell_back", ctypes.c_int32),
                ("latency_s", ctypes.c_double), ("energy_initial", ctypes.c_double),
                ("energy_final", ctypes.c_double), ("elements", ctypes.c_int64), ("steps", ctypes.c_int64),
                ("queued_s", ctypes.c_double)]


class EbServerStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int64) for k in ("queued", "active", "finishing", "completed", "fallbacks",
                                               "bins_total", "bins_used", "ticks")] + \
               [("element_steps", ctypes.c_double), ("kernel_seconds", ctypes.c_double)]


FIELD_NAME_SNAKE = {"Position": "position", "Velocity": "velocity", "Director": "director",
                    "AngularVelocity": "angular_velocity"}


class EbHostState(ctypes.Structure):
    _fields_ = [(f"{n}_{d}", ctypes.c_void_p) for d in ("in", "out")
                for n in ("position", "velocity", "director", "angular_velocity")]


class EbJoint(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("reserved", ctypes.c_int32), ("stiffness", ctypes.c_double),
                ("damping", ctypes.c_double), ("rotational_stiffness", ctypes.c_double),
                ("normal", ctypes.c_double * 3)]


EB_JOINT_FREE = 0
EB_JOINT_HINGE = 1
EB_SERVER_FORCE_FALLBACK = 0x1
EB_REQUEST_CLAMP = 0x1
EB_REQUEST_DAMPER = 0x2
EB_REQUEST_GRAVITY = 0x4


# every entry point of include/elastica_b200.h with its ctypes signature
_P = ctypes.POINTER
_sim = ctypes.c_void_p
SIGNATURES = {
    "eb_sim_create": ([_P(EbConfig), _P(ctypes.c_void_p)], ctypes.c_int),
    "eb_sim_destroy": ([_sim], ctypes.c_int),
    "eb_last_error": ([], ctypes.c_char_p),
    "eb_version": ([], ctypes.c_char_p),
    "eb_emplace_straight_rods": ([_sim, _P(EbStraightRod), ctypes.c_int64, _P(ctypes.c_int64)], ctypes.c_int),
    "eb_rod_count": ([_sim, _P(ctypes.c_int64)], ctypes.c_int),
    "eb_rod_elements": ([_sim, ctypes.c_int64, _P(ctypes.c_int64)], ctypes.c_int),
    "eb_slot_count": ([_sim, _P(ctypes.c_int64)], ctypes.c_int),
    "eb_slot_offsets": ([_sim, _P(ctypes.c_int64), ctypes.c_int64], ctypes.c_int),
    "eb_field_size": ([_sim, ctypes.c_int64, ctypes.c_int32, _P(ctypes.c_int64)], ctypes.c_int),
    "eb_set_field": ([_sim, ctypes.c_int64, ctypes.c_int32, _P(ctypes.c_double), ctypes.c_int64], ctypes.c_int),
    "eb_get_field": ([_sim, ctypes.c_int64, ctypes.c_int32, _P(ctypes.c_double), ctypes.c_int64], ctypes.c_int),
    "eb_set_field_batch": ([_sim, ctypes.c_int32, ctypes.c_int32, _P(ctypes.c_double), ctypes.c_int64], ctypes.c_int),
    "eb_get_field_batch": ([_sim, ctypes.c_int32, ctypes.c_int32, _P(ctypes.c_double), ctypes.c_int64], ctypes.c_int),
    "eb_constrain_clamp": ([_sim, ctypes.c_int64, ctypes.c_int64], ctypes.c_int),
    "eb_add_gravity": ([_sim, _P(ctypes.c_double)], ctypes.c_int),
    "eb_add_end_torque": ([_sim, ctypes.c_int64, _P(ctypes.c_double)], ctypes.c_int),
    "eb_add_element_torque": ([_sim, ctypes.c_int64, ctypes.c_int64, _P(ctypes.c_double)], ctypes.c_int),
    "eb_add_analytical_damper": ([_sim, ctypes.c_int64, ctypes.c_double, ctypes.c_double], ctypes.c_int),
    "eb_add_contact_material": ([_sim, _P(EbContactMaterial), _P(ctypes.c_int32)], ctypes.c_int),
    "eb_add_rod_contact": ([_sim, ctypes.c_int64, ctypes.c_int32], ctypes.c_int),
    "eb_add_contact_plane": ([_sim, _P(ctypes.c_double), _P(ctypes.c_double), ctypes.c_int32], ctypes.c_int),
    "eb_contact_pairs": ([_sim, _P(ctypes.c_int64), ctypes.c_int64, _P(ctypes.c_int64)], ctypes.c_int),
    "eb_connect": ([_sim, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, _P(EbJoint)],
                   ctypes.c_int),
    "eb_finalize": ([_sim], ctypes.c_int),
    "eb_step": ([_sim, _P(ctypes.c_double), ctypes.c_double, ctypes.c_int64], ctypes.c_int),
    "eb_synchronize": ([_sim], ctypes.c_int),
    "eb_step_host_state": ([_sim, _P(ctypes.c_double), ctypes.c_double, ctypes.c_int64, _P(EbHostState)],
                           ctypes.c_int),
    "eb_energy": ([_sim, _P(ctypes.c_double), ctypes.c_int64], ctypes.c_int),
    "eb_get_stream": ([_sim, _P(ctypes.c_void_p)], ctypes.c_int),
    "eb_step_plan": ([_sim, _P(ctypes.c_int32), _P(ctypes.c_int32), _P(ctypes.c_float), ctypes.c_int32], ctypes.c_int),
    "eb_launch_count": ([_sim, _P(ctypes.c_int64)], ctypes.c_int),
    "eb_debug_set_wait_bound": ([_sim, ctypes.c_uint32], ctypes.c_int),
    "eb_server_create": ([_P(EbServerConfig), _P(ctypes.c_void_p)], ctypes.c_int),
    "eb_server_destroy": ([ctypes.c_void_p], ctypes.c_int),
    "eb_server_submit": ([ctypes.c_void_p, _P(EbRequest), _P(ctypes.c_int64)], ctypes.c_int),
    "eb_server_tick": ([ctypes.c_void_p, _P(ctypes.c_int64)], ctypes.c_int),
    "eb_server_poll": ([ctypes.c_void_p, _P(EbCompletion), ctypes.c_int32, _P(ctypes.c_int32)], ctypes.c_int),
    "eb_server_result": ([ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int32, _P(ctypes.c_double),
                          ctypes.c_int64], ctypes.c_int),
    "eb_server_release": ([ctypes.c_void_p, ctypes.c_int64], ctypes.c_int),
    "eb_server_get_stats": ([ctypes.c_void_p, _P(EbServerStats)], ctypes.c_int),
    "eb_server_request_status": ([ctypes.c_void_p, ctypes.c_int64, _P(ctypes.c_int32), _P(ctypes.c_double),
                                  _P(ctypes.c_double)], ctypes.c_int),
    "eb_snapshot_size": ([_sim, _P(ctypes.c_uint64)], ctypes.c_int),
    "eb_snapshot_save": ([_sim, ctypes.c_void_p, ctypes.c_uint64], ctypes.c_int),
    "eb_snapshot_load": ([_sim, ctypes.c_void_p, ctypes.c_uint64], ctypes.c_int),
    "eb_partition_rods": ([_P(ctypes.c_int64), ctypes.c_int64, ctypes.c_int32, _P(ctypes.c_int32)], ctypes.c_int),
    "eb_box_pairs_noalloc": ([ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                              _P(ctypes.c_int64), ctypes.c_void_p], ctypes.c_int),
}


class EbError(RuntimeError):
    def __init__(self, fn: str, status: int, msg: str):
        super().__init__(f"{fn} -> {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_lib = None


def load(build_if_missing: bool = True):
    """Load the library (building it in-tree first if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        if not build_if_missing:
            raise FileNotFoundError(f"{LIB_PATH} is missing; run python -m elasticapp_b200.build")
        from . import build as _build

        _build.build()
    lib = ctypes.CDLL(LIB_PATH)
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def call(fn: str, *args) -> None:
    lib = load()
    rc = getattr(lib, fn)(*args)
    if rc != EB_OK:
        raise EbError(fn, rc, lib.eb_last_error().decode(errors="replace"))
