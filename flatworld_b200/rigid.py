"""Rigid primitives in contact with FEM bodies (reference: flatworld/rigid.py:20-170,
flatworld/rigiddomain.py:27-160).

``BallRigid``, ``BoxRigid`` and ``CapsuleRigid`` hold the same fields the
reference's classes hold (origin, radius / extents / segment, angle, mass,
body-frame inertia, minSize); ``RigidBodyDomain`` wraps one of them with its
BCs, initial conditions, friction and collision flags.  The loop packs them
into the device world (``PackedWorld.rigid_records``), where the FEM-rigid
penalty contact and the rigid velocity / position update run on the GPU.

Supported: the primitives touching FEM bodies only.  Mesh rigids, joints, and
rigid-rigid or rigid-ground contact (the reference's PGS constraint solve) are
outside flatworld_b200; a world whose rigid meets a ground or another contact
rigid raises at the next step.
"""

from __future__ import annotations

import numpy as np

from .definitions import COLLISION_CATEGORY_ORDINARY_RIGID, COLLISION_MASK_ALL, DomainType


class RigidType:
    """flatworld/definitions.py:50-54"""

    BALL = 0b00001
    BOX = 0b00010
    CAPSULE = 0b01000
    MESH = 0b10000


class RigidBase:
    def __init__(self, d):
        self.d = d
        self.numNodes = 1
        self.mesh = None
        self.initial_quat = None
        self.inertia_body = None
        self.transform = None

    def getRefPoint(self):
        return None

    def getRadius(self):
        return 0.0

    def getPrimary(self):
        return np.zeros((self.d,), dtype=np.float32)


class BallRigid(RigidBase):
    """rigid.py:52-75: inertia 0.5 m r^2 unless given."""

    def __init__(self, d, origin, radius, mass, angle=None, inertia=None):
        super().__init__(d)
        self.origin = np.asarray(origin, dtype=np.float32)
        self.radius = radius
        self.mass = mass
        self.rtype = RigidType.BALL
        self.minSize = radius * 2.0
        self.angle = np.asarray(angle, dtype=np.float32) if angle is not None else np.zeros((d,), dtype=np.float32)
        self.inertia_body = inertia if inertia is not None else 0.5 * self.mass * (self.radius ** 2)

    def getRefPoint(self):
        return self.origin

    def getRadius(self):
        return self.radius


class BoxRigid(RigidBase):
    """rigid.py:86-105: full extents ``ext``; inertia m (w^2 + h^2) / 12 unless given."""

    def __init__(self, d, origin, ext, angle, mass, inertia=None):
        super().__init__(d)
        self.numShapeNodes = 4
        self.ext = np.asarray(ext, dtype=np.float32)
        self.angle = np.asarray(angle, dtype=np.float32)
        self.origin = np.asarray(origin, dtype=np.float32)
        self.mass = mass
        self.rtype = RigidType.BOX
        if inertia is not None:
            self.inertia_body = inertia
        else:
            w = float(self.ext[0])
            h = float(self.ext[1])
            self.inertia_body = (1.0 / 12.0) * self.mass * (w * w + h * h)
        self.minSize = min(float(self.ext[0]), float(self.ext[1]))

    def getRefPoint(self):
        return self.origin

    def getPrimary(self):
        return self.ext


class CapsuleRigid(RigidBase):
    """rigid.py:136-165: segment lc-uc of radius ``radius``, reference point its
    midpoint; inertia m L^2 / 12 + m r^2 / 2 unless given."""

    def __init__(self, d, lc, uc, angle, radius, mass, inertia=None):
        super().__init__(d)
        self.lc = np.asarray(lc, dtype=np.float32)
        self.uc = np.asarray(uc, dtype=np.float32)
        self.radius = radius
        self.mass = mass
        self.rtype = RigidType.CAPSULE
        self.origin = 0.5 * (self.lc + self.uc)
        self.angle = np.asarray(angle, dtype=np.float32)
        axis = self.uc - self.lc
        axis_len = float(np.linalg.norm(axis))
        if inertia is not None:
            self.inertia_body = inertia
        else:
            self.inertia_body = (1.0 / 12.0) * self.mass * (axis_len ** 2) + 0.5 * self.mass * (self.radius ** 2)
        self.minSize = min(self.radius * 2.0, axis_len)

    def getPrimary(self):
        return self.lc

    def getRadius(self):
        return self.radius

    def getRefPoint(self):
        return self.origin


class MeshRigid(RigidBase):
    def __init__(self, *args, **kwargs):
        raise NotImplementedError("MeshRigid: rigid meshes (the reference's spatial-hash FEM-rigid-mesh path) "
                                  "are outside flatworld_b200; use BallRigid, BoxRigid or CapsuleRigid")


class Transform:
    def __init__(self, *args, **kwargs):
        raise NotImplementedError("Transform belongs to MeshRigid, which flatworld_b200 does not implement")


class RigidBodyDomain:
    """rigiddomain.py:27-160.  State reads (ref point, angle, velocities, box)
    come from the device world of the loop the domain was attached to."""

    def __init__(self, rigid, bcs=[], considerContact=True, considerGroundContact=True, initials=[],
                 friction: float = 0.0, restitution=0.9, name="", visual_mesh=None, collision_shapes=None,
                 category_bits=COLLISION_CATEGORY_ORDINARY_RIGID, collide_bits=COLLISION_MASK_ALL):
        if getattr(rigid, "rtype", None) not in (RigidType.BALL, RigidType.BOX, RigidType.CAPSULE):
            raise NotImplementedError("RigidBodyDomain: only BallRigid, BoxRigid and CapsuleRigid are supported")
        if collision_shapes:
            raise NotImplementedError("RigidBodyDomain: compound collision shapes are not supported")
        self.rigid = rigid
        self.d = rigid.d
        self.bcs = bcs
        self.considerContact = considerContact
        self.considerGroundContact = considerGroundContact
        self.type = DomainType.RIGID
        self.ref = rigid.getRefPoint()
        self.nnodes = rigid.numNodes
        self.nelements = 0
        self.initials = initials
        self.friction = float(friction)
        self.restitution = float(restitution)
        self.name = name
        self.visual_mesh = visual_mesh
        self.collision_shapes = []
        self.category_bits = category_bits
        self.collide_bits = collide_bits
        self._loop = None
        self.ndOffset = None

    def attach(self, loop, offset: int):
        self._loop = loop
        self.ndOffset = int(offset)

    def _state(self):
        if self._loop is None:
            raise RuntimeError("RigidBodyDomain: not part of an ExplicitLoop yet")
        return self._loop._rigid_state()[self.ndOffset]

    def getBBox(self):
        s = self._state()
        return s[8:10].astype(np.float32), s[10:12].astype(np.float32)

    def getCurrentRefPoint(self):
        return self._state()[0:2].astype(np.float32)

    def getCurrentRefAngles(self):
        return np.array([self._state()[2]], dtype=np.float32)

    def getCurrentVelocity(self):
        return self._state()[3:5].astype(np.float32)

    def getCurrentAngularVelocity(self):
        return np.array([self._state()[5]], dtype=np.float32)

    def getCurrentDisplacement(self):
        return self._state()[6:8].astype(np.float32)
