"""Boundary and initial conditions (reference: flatworld/bcs.py:14-103,
flatworld/initialconditions.py:31-73).  ``processData`` returns
(bit, node ids or None for all nodes, value or None) like the reference."""

import numpy as np

from .definitions import (
    ATYPE,
    FORCETYPE,
    GRAVITY,
    ROTATYPE,
    ROTVTYPE,
    RTYPE,
    TORQUETYPE,
    UTYPE,
    VTYPE,
    BoundaryConditionType,
)


class BcBase:
    pass


class Gravity(BcBase):
    def __init__(self, g):
        self.g = g
        self.type = BoundaryConditionType.GRAVITY

    def processData(self):
        return GRAVITY, None, self.g


class Force(BcBase):
    def __init__(self, nds, force):
        self.nds = nds
        self.force = force
        self.type = BoundaryConditionType.FORCE

    def processData(self):
        return FORCETYPE, self.nds, self.force


class EnforceAcc(BcBase):
    def __init__(self, nds, acc):
        self.nds = nds
        self.acc = acc
        self.type = BoundaryConditionType.ENFORCE_ACCELERATION

    def processData(self):
        return ATYPE, self.nds, self.acc


class EnforceVel(BcBase):
    def __init__(self, nds, vel):
        self.nds = nds
        self.vel = vel
        self.type = BoundaryConditionType.ENFORCE_VELOCITY

    def processData(self):
        return VTYPE, self.nds, self.vel


class Fixed(BcBase):
    def __init__(self, nds):
        self.nds = nds
        self.type = BoundaryConditionType.FIXED

    def processData(self):
        return UTYPE, self.nds, None


class FixedAll(BcBase):
    """Fixes translation and rotation; on FEM nodes only the value slot is
    overwritten (the FEM integrator ignores the rotation bit)."""

    def __init__(self, nds):
        self.nds = nds
        self.type = BoundaryConditionType.FIXED_ALL

    def processData(self):
        return RTYPE, self.nds, None


class EnforceRotVel(BcBase):
    def __init__(self, nds, rotVelocity, origin=(0.0, 0.0, 0.0)):
        self.nds = nds
        self.rotVel = rotVelocity
        self.origin = origin
        self.type = BoundaryConditionType.ENFORCE_ROTATION_VELOCITY

    def processData(self):
        return ROTVTYPE, self.nds, self.rotVel


class EnforceRotAcc(BcBase):
    def __init__(self, nds, rotAcc, origin=(0.0, 0.0, 0.0)):
        self.nds = nds
        self.origin = origin
        self.rotAcc = rotAcc
        self.type = BoundaryConditionType.ENFORCE_ROTATION_ACCELERATION

    def processData(self):
        return ROTATYPE, self.nds, self.rotAcc


class Torque(BcBase):
    def __init__(self, nds, torque):
        self.nds = nds
        self.torque = torque
        self.type = BoundaryConditionType.TORQUE

    def processData(self):
        return TORQUETYPE, self.nds, self.torque


class InitialVel:
    """Initial nodal velocity; ``nds == "ALL"`` applies it to every node."""

    def __init__(self, nds, vel):
        if isinstance(nds, str) and nds == "ALL":
            self.is_all_nodes = True
            self.nds = None
        else:
            self.is_all_nodes = False
            self.nds = np.asarray(nds, dtype=np.int32)
        self.vel = np.asarray(vel, dtype=np.float32)
        self.type = VTYPE


class InitialAngVel:
    """Initial angular velocity of a rigid body (reference:
    initialconditions.py:53-73); ``nds == "ALL"`` applies it to every index."""

    def __init__(self, nds, ang_vel, ref_point=None):
        if isinstance(nds, str) and nds == "ALL":
            self.is_all_nodes = True
            self.nds = None
        else:
            self.is_all_nodes = False
            self.nds = np.asarray(nds, dtype=np.int32)
        self.ang_vel = np.asarray(ang_vel, dtype=np.float32)
        self.ref_point = np.asarray(ref_point, dtype=np.float32) if ref_point is not None else None
        self.type = ROTVTYPE
