"""elasticapp_b200: B200-native Cosserat-rod step behind the reference's
Simulator plugin surface (see include/elastica_b200.h for the C-ABI).

The compute path is libelastica_b200.so (hand-written sm_100a kernels); it is
built in-tree by ``python -m elasticapp_b200.build`` and there is no CPU
fallback.
"""
from .simulator import (AnalyticalLinearDamper, Clamp, CollisionSystem, ContactMaterial, CosseratRod,
                        CosseratRodWithoutDamping, EndTorque, FreeJoint, GravityField, HingeJoint, Material, PEFRL,
                        VelocityVerlet,
                        PositionVerlet, RodRef, Simulator, StraightRod)
from . import _lib

__all__ = ["AnalyticalLinearDamper", "Clamp", "CollisionSystem", "ContactMaterial", "CosseratRod", "CosseratRodWithoutDamping", "EndTorque",
           "FreeJoint", "GravityField", "HingeJoint", "Material", "PEFRL", "PositionVerlet", "RodRef", "VelocityVerlet", "Simulator", "StraightRod", "_lib"]
