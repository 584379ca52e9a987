"""flatworld_b200: B200-native explicit 2D FEM step with FlatWorld's API.

Drop-in for the FEM path of FlatWorld (``from flatworld import ...``):
FemDomain / SolidProp(Elastic | HyperElastic | MisesPlastic) /
GroundDomain | HeightFieldDomain | VoxelGridDomain / ExplicitLoop, plus
FEM-FEM contact, SpringMassDomain, and rigid primitives (RigidBodyDomain with
BallRigid | BoxRigid | CapsuleRigid) in contact with FEM bodies.
The step runs as hand-written CUDA kernels for sm_100a (libfwb200.so) behind a
C ABI (include/fwb200.h); there is no CPU fallback.
"""

from .bcs import (EnforceAcc, EnforceRotAcc, EnforceRotVel, EnforceVel, Fixed, FixedAll, Force, Gravity,
                  InitialAngVel, InitialVel, Torque)
from .definitions import *  # noqa: F401,F403
from .domains import FemDomain, GroundDomain, HeightFieldDomain, SpringMassDomain, VoxelGridDomain
from .explicitloop import ExplicitLoop, FemSpringManager
from .femesher import FEMesher
from .materials import J2, Elastic, HyperElastic, MisesPlastic, NeoHookean, SolidProp
from .mesh import Mesh, structured_rectangle
from .rigid import BallRigid, BoxRigid, CapsuleRigid, MeshRigid, RigidBodyDomain, RigidType, Transform


def _out_of_scope(name, why):
    def _raise(*args, **kwargs):
        raise NotImplementedError(f"{name}: {why} -- outside flatworld_b200 (the explicit FEM path)")

    return type(name, (), {"__init__": _raise})


_JOINTS = "joints are solved by the reference's rigid-body constraint solver"
PrismaticJoint = _out_of_scope("PrismaticJoint", _JOINTS)
RevoluteJoint = _out_of_scope("RevoluteJoint", _JOINTS)
SphericalJoint = _out_of_scope("SphericalJoint", _JOINTS)
WeldJoint = _out_of_scope("WeldJoint", _JOINTS)

__version__ = "0.1.0"
