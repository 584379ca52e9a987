"""Domain objects of the FEM path (reference: flatworld/femdomain.py,
grounddomain.py, heightfielddomain.py, voxeldomain.py).

Construction arguments, attributes and host-side helpers follow the reference.
The device-side contact arithmetic lives in csrc/fw_device.cuh.
"""

from __future__ import annotations

import numpy as np

from .definitions import COLLISION_CATEGORY_FEM, COLLISION_CATEGORY_GROUND, COLLISION_MASK_ALL, DomainType


class DomainBase:
    pass


class FemDomain(DomainBase):
    """One FEM body (reference: flatworld/femdomain.py:6-60)."""

    def __init__(self, mesh, prop, bcs=[], considerContact=True, considerGroundContact=True,
                 initials=[], friction=0.0):
        self.mesh = mesh
        self.d = mesh.d
        self.prop = prop
        self.bcs = bcs
        self.friction = friction
        self.initials = initials
        self.nnodes = self.mesh.numNodes
        self.nelements = self.mesh.numElements
        self.considerContact = considerContact
        self.considerGroundContact = considerGroundContact
        self.type = DomainType.FEM
        self.category_bits = COLLISION_CATEGORY_FEM
        self.collide_bits = COLLISION_MASK_ALL
        mat = self.prop.mat
        # femdomain.py:24: CFL bound from the shortest element edge
        self.stableTime = 0.4 * self.mesh.charLength / (mat.E / mat.rho) ** 0.5
        self.femManager = None
        self.domainIdx = None

    def attach(self, femManager, domainIdx):
        self.femManager = femManager
        self.domainIdx = domainIdx

    def getBBox(self):
        lb, ub = self.femManager.body_aabb(self.domainIdx)
        return lb, ub

    def getNumDofs(self):
        return self.d * self.mesh.numNodes

    def getNumNodes(self):
        return self.mesh.numNodes

    def getNumElements(self):
        return self.mesh.numElements

    def getCurrentCoords(self):
        return self.femManager.body_coords(self.domainIdx)

    def getCurrentVelocities(self):
        return self.femManager.body_velocities(self.domainIdx)


class GroundDomain(DomainBase):
    """Ground plane through ``point`` with unit ``normal`` (reference:
    flatworld/grounddomain.py:18-77).  With BCs (e.g. ``Fixed([0])``,
    ``EnforceVel``) the rigid manager moves it; as in the reference, FEM bodies
    keep contacting the plane of construction time, while the broad-phase
    boxes of the loop's grounds follow the moving entry."""

    def __init__(self, d, point, normal, bcs=[], considerContact=True, considerGroundContact=True,
                 initials=[]):
        self.d = d
        self.point = np.asarray(point, dtype=np.float32)
        n = np.asarray(normal, dtype=np.float32)
        nlen = float(np.linalg.norm(n))
        self.normal = n / max(nlen, 1e-12)
        self.nnodes = 1
        self.nelements = 0
        self.type = DomainType.ANALYTICAL
        self.considerContact = considerContact
        self.considerGroundContact = considerGroundContact
        self.initials = initials
        self.bcs = bcs
        self.category_bits = COLLISION_CATEGORY_GROUND
        self.collide_bits = COLLISION_MASK_ALL

    def attach(self, loop, entry):
        """A loop with a moving plane holds this ground as rigid-manager entry ``entry``."""
        self._loop = loop
        self._entry = int(entry)

    def getCurrentRefPoint(self):
        if getattr(self, "_loop", None) is not None:
            return self._loop._entry_state()[self._entry, 0:2].astype(np.float32)
        return self.point.copy()

    def getCurrentNormal(self):
        """The normal rotated by the entry's angle (grounddomain.py:47-51)."""
        if getattr(self, "_loop", None) is not None:
            a = float(self._loop._entry_state()[self._entry, 2])
            c, s = np.float32(np.cos(a)), np.float32(np.sin(a))
            n = self.normal.astype(np.float32)
            return np.array([c * n[0] - s * n[1], s * n[0] + c * n[1]], dtype=np.float32)
        return self.normal.astype(np.float32)

    def getBBox(self):
        # grounddomain.py:54-70: +-0.1 along the normal, +-1e4 along the tangent
        buffer = 0.1
        large_span = 10000.0
        p = self.point
        tangent = np.array([-self.normal[1], self.normal[0]], dtype=np.float32)
        lo_raw = p - tangent * large_span - self.normal * buffer
        hi_raw = p + tangent * large_span + self.normal * buffer
        return np.minimum(lo_raw, hi_raw).astype(np.float32), np.maximum(lo_raw, hi_raw).astype(np.float32)


class HeightFieldDomain(DomainBase):
    """Static 1D height field z = h(x) over [lb.x, ub.x]
    (reference: flatworld/heightfielddomain.py:6-222; 2D form)."""

    def __init__(self, d, height_np, lb, ub, considerContact=True, reverse=False):
        if d != 2:
            raise NotImplementedError("flatworld_b200 implements the 2D height field only")
        self.d = d
        self.type = DomainType.HEIGHTFIELD
        self.considerContact = considerContact
        self.initials = []
        self.bcs = []
        self.reverse = reverse
        height_np = np.asarray(height_np, dtype=np.float32)
        assert height_np.ndim == 1, "2D height field expects 1D numpy array of shape (nx,)"
        self.maxHeight = float(np.max(height_np)) + 0.1
        self.minHeight = float(np.min(height_np)) - 0.1
        self.nx = int(height_np.shape[0])
        self.ny = 1
        self.height = height_np.copy()
        self.point = np.array([0.0, -1e6], dtype=np.float32)
        self.normal = np.array([0.0, 1.0], dtype=np.float32)
        self.nnodes = 1
        self.nelements = 0
        self.lb = np.asarray(lb, dtype=np.float32)
        self.ub = np.asarray(ub, dtype=np.float32)
        self.category_bits = COLLISION_CATEGORY_GROUND
        self.collide_bits = COLLISION_MASK_ALL

    @staticmethod
    def _lerp(a, b, t):
        return a + (b - a) * t

    def sample_height_2d(self, x):
        u = (x - self.lb[0]) / (self.ub[0] - self.lb[0])
        u = float(np.clip(u, 0.0, 1.0))
        s = u * (self.nx - 1)
        i0 = int(np.floor(s))
        i1 = min(i0 + 1, self.nx - 1)
        t = s - float(i0)
        return float(self._lerp(self.height[i0], self.height[i1], t))

    def sample_dhdx_2d(self, x):
        u = (x - self.lb[0]) / (self.ub[0] - self.lb[0])
        u = float(np.clip(u, 0.0, 1.0))
        s = u * (self.nx - 1)
        i = int(np.round(s))
        i0 = max(0, i - 1)
        i1 = min(self.nx - 1, i + 1)
        dx_world = (self.ub[0] - self.lb[0]) / (self.nx - 1)
        return (float(self.height[i1]) - float(self.height[i0])) / max(dx_world * (i1 - i0), 1e-6)

    def sample_normal_2d(self, x):
        n = np.array([-self.sample_dhdx_2d(x), 1.0], dtype=np.float32)
        if self.reverse:
            n = -n
        return n / max(float(np.linalg.norm(n)), 1e-12)

    def nearest_on_curve_2d(self, x, z):
        h = self.sample_height_2d(x)
        foot = np.array([x, h], dtype=np.float32)
        n = self.sample_normal_2d(x)
        p = np.array([x, z], dtype=np.float32)
        return foot, n, float(np.dot(p - foot, n))

    def get_maxmin_height_in_range_2d(self, x_min, x_max):
        x0 = float(np.clip(x_min, self.lb[0], self.ub[0]))
        x1 = float(np.clip(x_max, self.lb[0], self.ub[0]))
        span = self.ub[0] - self.lb[0]
        i0 = max(0, min(int(np.floor((x0 - self.lb[0]) / span * (self.nx - 1))), self.nx - 1))
        i1 = max(0, min(int(np.ceil((x1 - self.lb[0]) / span * (self.nx - 1))), self.nx - 1))
        seg = self.height[i0:i1 + 1]
        return float(seg.max()), float(seg.min())

    def getBBox(self):
        return (np.array([self.lb[0], self.minHeight], dtype=np.float32),
                np.array([self.ub[0], self.maxHeight], dtype=np.float32))

    def getBoundaryMesh(self):
        xs = np.linspace(float(self.lb[0]), float(self.ub[0]), self.nx, dtype=np.float32)
        vertices = np.stack([xs, np.zeros_like(xs), self.height], axis=1).astype(np.float32)
        faces = np.stack([np.arange(self.nx - 1), np.arange(1, self.nx)], axis=1).astype(np.int32)
        return vertices, faces


class VoxelGridDomain(DomainBase):
    """Static 2D occupancy grid obstacle (reference: flatworld/voxeldomain.py:6-217).

    ``occ[i, j] == 1`` marks an occupied cell, ``0`` a free one; contact acts on
    nodes inside occupied cells and pushes them out through the nearest free
    face (mixedcontact.py:220-302).
    """

    def __init__(self, d, nx, ny, lb, ub, nz=None, considerContact=True, occupancy_np=None):
        if d != 2:
            raise NotImplementedError("flatworld_b200 implements the 2D voxel grid only")
        self.d = d
        self.type = DomainType.VOXELMAP
        self.considerContact = considerContact
        self.initials = []
        self.bcs = []
        self.nx = int(nx)
        self.ny = int(ny)
        self.lb = np.asarray(lb, dtype=np.float32)
        self.ub = np.asarray(ub, dtype=np.float32)
        self.dx = (self.ub[0] - self.lb[0]) / max(self.nx, 1)
        self.dz = (self.ub[1] - self.lb[1]) / max(self.ny, 1)
        self.occ = np.zeros((self.nx, self.ny), dtype=np.int32)
        if occupancy_np is not None:
            assert occupancy_np.shape == (self.nx, self.ny)
            self.occ[:] = occupancy_np.astype(np.int32)
        self.nnodes = 1
        self.nelements = 0
        self.category_bits = COLLISION_CATEGORY_GROUND
        self.collide_bits = COLLISION_MASK_ALL
        self._edges = None

    def _build_edges(self):
        """Exposed faces of occupied cells (voxeldomain.py:95-129), built lazily:
        only the host-side helpers below use them."""
        occ = self.occ
        p0, p1, nn = [], [], []
        for i in range(self.nx):
            for j in range(self.ny):
                if occ[i, j] != 1:
                    continue
                x0 = self.lb[0] + i * self.dx
                x1 = x0 + self.dx
                z0 = self.lb[1] + j * self.dz
                z1 = z0 + self.dz
                if i - 1 < 0 or occ[i - 1, j] == 0:
                    p0.append([x0, z0]); p1.append([x0, z1]); nn.append([-1.0, 0.0])
                if i + 1 >= self.nx or occ[i + 1, j] == 0:
                    p0.append([x1, z0]); p1.append([x1, z1]); nn.append([1.0, 0.0])
                if j - 1 < 0 or occ[i, j - 1] == 0:
                    p0.append([x0, z0]); p1.append([x1, z0]); nn.append([0.0, -1.0])
                if j + 1 >= self.ny or occ[i, j + 1] == 0:
                    p0.append([x0, z1]); p1.append([x1, z1]); nn.append([0.0, 1.0])
        f = lambda a: np.asarray(a, dtype=np.float32).reshape(-1, 2)  # noqa: E731
        self._edges = (f(p0), f(p1), f(nn))

    @property
    def edge_count(self):
        if self._edges is None:
            self._build_edges()
        return len(self._edges[0])

    def getBBox(self):
        return self.lb, self.ub

    def getBoundaryMesh(self):
        if self._edges is None:
            self._build_edges()
        p0, p1, _ = self._edges
        if len(p0) == 0:
            return np.zeros((0, 2), dtype=np.float32), np.zeros((0, 2), dtype=np.int32)
        verts = np.stack([p0, p1], axis=1).reshape(-1, 2)
        edges = np.arange(2 * len(p0), dtype=np.int32).reshape(-1, 2)
        return verts, edges


class SpringMassDomain(DomainBase):
    """A spring-mass network (reference: flatworld/springmass.py:6-73): nodes
    of equal mass joined by 2-node springs.  prop = [stiffness, damping, node
    mass]; rest lengths are the float32 norms of the initial edge vectors."""

    def __init__(self, d, coords, conns, prop=[100.0, 1.0, 1.0], bcs=[], considerContact=True,
                 considerGroundContact=True, initials=[], friction=0.0):
        if d != 2:
            raise NotImplementedError("flatworld_b200 implements 2D spring-mass domains only")
        self.d = d
        self.prop = prop
        self.bcs = bcs
        self.initials = initials
        self.friction = friction
        self.considerContact = considerContact
        self.considerGroundContact = considerGroundContact
        self.type = DomainType.SPRINGMASS
        self.spring, self.damping, self.mass = prop
        self.massInv = 1.0 / self.mass
        self.coords = np.array(coords, dtype=np.float32)
        self.connectivity = np.array(conns, dtype=np.int32)
        self.nnodes = coords.shape[0]
        self.nelements = conns.shape[0]
        ab = self.coords[self.connectivity[:, 0]] - self.coords[self.connectivity[:, 1]]
        self.restLength = np.array([np.linalg.norm(v) for v in ab], dtype=np.float32)  # springmass.py:43-49
        self.stableTime = 0.5 * np.sqrt(self.mass / self.spring)  # springmass.py:38
        self.category_bits = COLLISION_CATEGORY_FEM
        self.collide_bits = COLLISION_MASK_ALL
        self.femManager = None
        self.domainIdx = None

    def attach(self, femManager, domainIdx):
        self.femManager = femManager
        self.domainIdx = domainIdx

    def getBBox(self):
        if self.femManager is not None:
            return self.femManager.body_aabb(self.domainIdx)
        return np.min(self.coords, axis=0), np.max(self.coords, axis=0)

    def getCurrentCoords(self):
        return self.femManager.body_coords(self.domainIdx)
