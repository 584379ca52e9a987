"""flatworld_b200: B200-native explicit 2D FEM step with FlatWorld's API.

Drop-in for the FEM path of FlatWorld (``from flatworld import ...``):
FemDomain / SolidProp(Elastic | HyperElastic | MisesPlastic) /
GroundDomain | HeightFieldDomain | VoxelGridDomain / ExplicitLoop.
The step runs as hand-written CUDA kernels for sm_100a (libfwb200.so) behind a
C ABI (include/fwb200.h); there is no CPU fallback.
"""

from .bcs import (EnforceAcc, EnforceRotAcc, EnforceRotVel, EnforceVel, Fixed, FixedAll, Force, Gravity,
                  InitialVel, Torque)
from .definitions import *  # noqa: F401,F403
from .domains import FemDomain, GroundDomain, HeightFieldDomain, SpringMassDomain, VoxelGridDomain
from .explicitloop import ExplicitLoop, FemSpringManager
from .femesher import FEMesher
from .materials import J2, Elastic, HyperElastic, MisesPlastic, NeoHookean, SolidProp
from .mesh import Mesh, structured_rectangle


def _out_of_scope(name, why):
    def _raise(*args, **kwargs):
        raise NotImplementedError(f"{name}: {why} -- outside flatworld_b200 (the explicit FEM path)")

    return type(name, (), {"__init__": _raise})


_RIGID = "rigid bodies, joints and springs are solved by the reference's rigid/spring managers"
RigidBodyDomain = _out_of_scope("RigidBodyDomain", _RIGID)
BallRigid = _out_of_scope("BallRigid", _RIGID)
BoxRigid = _out_of_scope("BoxRigid", _RIGID)
CapsuleRigid = _out_of_scope("CapsuleRigid", _RIGID)
MeshRigid = _out_of_scope("MeshRigid", _RIGID)
Transform = _out_of_scope("Transform", _RIGID)
PrismaticJoint = _out_of_scope("PrismaticJoint", _RIGID)
RevoluteJoint = _out_of_scope("RevoluteJoint", _RIGID)
SphericalJoint = _out_of_scope("SphericalJoint", _RIGID)
WeldJoint = _out_of_scope("WeldJoint", _RIGID)
InitialAngVel = _out_of_scope("InitialAngVel", _RIGID)

__version__ = "0.1.0"
