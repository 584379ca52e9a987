"""ExplicitLoop and FemSpringManager: the reference's driver API on top of the
B200 world (reference: flatworld/explicitloop.py:71-679,
flatworld/femspringmanager.py:495-1100).

The reference launches 7-9 Warp kernels and performs several blocking
device-to-host reads per substep.  Here one substep is two kernels queued on a
CUDA stream (captured in CUDA graphs for runs of equal substeps); state stays
on the GPU until a ``.numpy()`` read.
"""

from __future__ import annotations

import numpy as np

from . import _native
from .definitions import DomainType
from .world import PackedWorld, SceneLayout, build_native, substep_schedule


class _HostArray:
    """Host-side constant exposed like a Warp array (``.numpy()``)."""

    def __init__(self, arr):
        self._arr = np.asarray(arr)

    def numpy(self):
        return self._arr.copy()

    @property
    def shape(self):
        return self._arr.shape


class _DeviceNodeArray:
    """A node field read from the GPU on ``.numpy()``, padded to MAX_NODES rows
    like the reference's preallocated arrays (femspringmanager.py:546-571)."""

    def __init__(self, mgr, field, width=2, transform=None):
        self._mgr = mgr
        self._field = field
        self._width = width
        self._transform = transform

    def numpy(self):
        m = self._mgr
        shape = (m.MAX_NODES, self._width) if self._width > 1 else (m.MAX_NODES,)
        out = np.zeros(shape, np.float32)
        vals = m._native.read_nodes(self._field, m._n0, m._nn)
        if self._transform is not None:
            vals = self._transform(vals)
        out[: m._nn] = vals
        return out

    @property
    def shape(self):
        return (self._mgr.MAX_NODES, self._width) if self._width > 1 else (self._mgr.MAX_NODES,)


class FemSpringManager:
    """Read-mostly view of the FEM data of one scene (reference names)."""

    def __init__(self, loop, packed: PackedWorld, native: _native.NativeWorld, scene: int = 0):
        self._loop = loop
        self._packed = packed
        self._native = native
        self._scene = scene
        bodies = packed.scene_bodies[scene]
        self._bodies = bodies
        self._n0 = int(packed.noff[bodies[0]])
        self._nn = int(sum(int(packed.ncnt[b]) for b in bodies))
        self._e0 = int(packed.eoff[bodies[0]])
        self._ne = int(sum(int(packed.ecnt[b]) for b in bodies))
        sc = packed.scenes[scene]
        self.domains = sc.fem
        self.domainMeshes = [getattr(d, "mesh", None) for d in sc.fem]
        self.d = 2
        nbound = [d.mesh.numBoundNodes if d.type == DomainType.FEM else d.nnodes for d in sc.fem]
        nb = sum(nbound)
        self.MAX_NODES = max(self._nn + 1024, 2048)
        self.MAX_ELEMENTS = max(self._ne + 2048, 4096)
        self.MAX_BOUNDARY_NODES = max(nb + 1024, self.MAX_NODES)
        self.stableTime = 1.0
        for d in sc.fem:
            self.stableTime = min(d.stableTime, self.stableTime)
        i32 = np.int32
        self.totalNodes = _HostArray(np.array([self._nn], i32))
        self.totalElements = _HostArray(np.array([self._ne], i32))
        n_fem = sum(1 for d in sc.fem if d.type == DomainType.FEM)
        self.totalFEMElements = _HostArray(np.array([sum(d.nelements for d in sc.fem if d.type == DomainType.FEM)], i32))
        self.totalFEMNodes = _HostArray(np.array([sum(d.nnodes for d in sc.fem if d.type == DomainType.FEM)], i32))
        self.numFemDomains = _HostArray(np.array([n_fem], i32))
        self.numSpringDomains = _HostArray(np.array([len(bodies) - n_fem], i32))
        pad = lambda a, n, dt: np.concatenate([a, np.zeros((n - len(a),) + a.shape[1:], dt)])  # noqa: E731
        md = max(len(bodies), 128)
        self.domainNodeOffset = _HostArray(pad(packed.noff[bodies] - self._n0, md, i32))
        self.domainNodeCount = _HostArray(pad(packed.ncnt[bodies], md, i32))
        self.domainElemOffset = _HostArray(pad(packed.eoff[bodies] - self._e0, md, i32))
        self.domainElemCount = _HostArray(pad(packed.ecnt[bodies], md, i32))
        bnoff = np.concatenate([[0], np.cumsum(nbound)[:-1]]).astype(i32)
        self.domainBoundaryNodeOffset = _HostArray(pad(bnoff, md, i32))
        self.domainBoundaryNodeCount = _HostArray(pad(np.array(nbound, i32), md, i32))
        bn = np.concatenate([packed.bnodes[packed.bnoff[b]:packed.bnoff[b] + packed.bncnt[b]] for b in bodies]) - self._n0
        self.boundaryNodes = _HostArray(pad(bn.astype(i32), self.MAX_BOUNDARY_NODES, i32))
        ids = [loop.domains.index(d) for d in sc.fem]
        self.femDomainIds = _HostArray(pad(np.array(ids, i32), md, i32))
        e = slice(self._e0, self._e0 + self._ne)
        nsl = slice(self._n0, self._n0 + self._nn)
        conn4 = np.full((self.MAX_ELEMENTS, 4), -1, i32)
        conn4[: self._ne, :3] = packed.conn[e] - self._n0
        self.connectivity = _HostArray(conn4)
        self.matE = _HostArray(pad(packed.Ev[e], self.MAX_ELEMENTS, np.float32))
        self.matNu = _HostArray(pad(packed.nuv[e], self.MAX_ELEMENTS, np.float32))
        self.matRho = _HostArray(pad(packed.rhov[e], self.MAX_ELEMENTS, np.float32))
        self.matType = _HostArray(pad(packed.mtype[e], self.MAX_ELEMENTS, i32))
        self.matYieldStress = _HostArray(pad(packed.syv[e], self.MAX_ELEMENTS, np.float32))
        self.matH = _HostArray(pad(packed.Hv[e], self.MAX_ELEMENTS, np.float32))
        self.bcNodes = _HostArray(pad(packed.bc_bits[nsl], self.MAX_NODES, i32))
        self.bcValues = _HostArray(pad(packed.bc_vals[nsl], self.MAX_NODES, np.float32))
        self.coords = _DeviceNodeArray(self, _native.FW_FIELD_X)
        self.V = _DeviceNodeArray(self, _native.FW_FIELD_V)
        self.mass = _DeviceNodeArray(self, _native.FW_FIELD_MASS, width=1)
        x0 = packed.coords[nsl]
        # Displacement since construction.  Nothing on the step reads U, so it
        # is formed on demand as x - x0 instead of being streamed every step.
        self.U = _DeviceNodeArray(self, _native.FW_FIELD_X, transform=lambda x: x - x0)
        zeros = np.zeros((self.MAX_NODES, 2), np.float32)
        # A (prescribed acceleration array) is never written and Fext is
        # cleared at the end of every step in the reference (femspringmanager.py:1007-1012).
        self.A = _HostArray(zeros)
        self.Fext = _HostArray(zeros)
        self.aabb = loop.aabb
        for k, dom in enumerate(sc.fem):
            dom.attach(self, k)

    # ---- per-body helpers used by FemDomain
    def body_coords(self, k):
        b = self._bodies[k]
        return self._native.read_nodes(_native.FW_FIELD_X, int(self._packed.noff[b]), int(self._packed.ncnt[b]))

    def body_velocities(self, k):
        b = self._bodies[k]
        return self._native.read_nodes(_native.FW_FIELD_V, int(self._packed.noff[b]), int(self._packed.ncnt[b]))

    def body_aabb(self, k):
        box = self._native.read_aabb(self._packed.B)[self._bodies[k]]
        return box[:2].copy(), box[2:].copy()

    @property
    def elemVolume(self):
        area, _ = self._native.read_reference_shape(self._packed.E)
        return _HostArray(area[self._e0:self._e0 + self._ne])

    @property
    def J_inv(self):
        _, jinv = self._native.read_reference_shape(self._packed.E)
        return _HostArray(jinv[self._e0:self._e0 + self._ne].reshape(-1, 2, 2))

    @property
    def plasticStrain(self):
        ep, _ = self._native.read_plastic(self._packed.E)
        return _HostArray(ep[self._e0:self._e0 + self._ne])

    @property
    def eqPlasticStrain(self):
        _, eq = self._native.read_plastic(self._packed.E)
        return _HostArray(eq[self._e0:self._e0 + self._ne])


class _AABBView:
    """``ExplicitLoop.aabb`` (max_domains x 2 vec2): FEM boxes from the GPU,
    ground boxes from getBBox()."""

    def __init__(self, loop):
        self._loop = loop

    def numpy(self):
        lp = self._loop
        out = np.zeros((lp._max_domains, 2, 2), np.float32)
        boxes = lp._native.read_aabb(lp._packed.B)
        ent = lp._entry_state() if lp._layout.entries else None
        for i, d in enumerate(lp.domains):
            if ent is not None and any(d is e for e in lp._layout.entries):
                k = next(j for j, e in enumerate(lp._layout.entries) if e is d)
                out[i, 0] = ent[k, 8:10]
                out[i, 1] = ent[k, 10:12]
            elif d.type in (DomainType.FEM, DomainType.SPRINGMASS):
                k = lp._packed.scenes[0].fem.index(d)
                b = lp._packed.scene_bodies[0][k]
                out[i, 0] = boxes[b, :2]
                out[i, 1] = boxes[b, 2:]
            elif d.considerContact:
                lo, hi = d.getBBox()
                out[i, 0] = lo
                out[i, 1] = hi
        return out


class RigidManager:
    """Read-only view of the rigid bodies of a loop with the reference's names
    (rigidmanager.py:1410-1790): stableTime (1e-3), numRigids, and the state
    arrays rigidParams (center, primary), quat, V, RotV, U read from the GPU."""

    stableTime = 1.0 / 1000.0

    def __init__(self, loop):
        self._loop = loop
        self.numRigids = len(loop._layout.rigids)
        self.numAnalytical = len(loop._layout.grounds)
        self.movingAnalytical = loop._layout.moving
        self.needUpdate = len(loop._layout.entries) > 0
        self._prim = [np.asarray(loop._packed.rigid_records()[0][k, 2:4]) for k in range(self.numRigids)]

    def _col(self, sl):
        return _HostArray(self._loop._rigid_state()[:, sl].copy())

    @property
    def rigidParams(self):
        st = self._loop._rigid_state()
        out = np.zeros((self.numRigids, 2, 2), np.float32)
        out[:, 0] = st[:, 0:2]
        for k, p in enumerate(self._prim):
            out[k, 1] = p
        return _HostArray(out)

    @property
    def quat(self):
        return self._col(2)

    @property
    def V(self):
        return self._col(slice(3, 5))

    @property
    def RotV(self):
        return self._col(5)

    @property
    def U(self):
        return self._col(slice(6, 8))


class ExplicitLoop:
    """Explicit dynamics driver with the reference's constructor and stepping
    API (explicitloop.py:72-85, 473-589)."""

    def __init__(self, dt, domains, joints=[], ties=None, damping=0.0, useAdapativeDT=True,
                 skip_spatial_hash=False, considerRigidRigidContact=True, use_pd=0,
                 mass_scaling_dt=0.0, max_contact_velocity=50.0, device=0, path="auto", patches=0,
                 front_warps=0, res_sync=0, res_threads=0):
        if joints:
            raise NotImplementedError("joints belong to the rigid-body constraint solver, outside flatworld_b200")
        if not considerRigidRigidContact and any(d.type == DomainType.RIGID for d in domains):
            raise NotImplementedError("considerRigidRigidContact=False with rigid bodies: flatworld_b200 runs "
                                      "FEM-rigid contact with the reference's default broad phase only")
        self.domains = domains
        self.d = domains[0].d
        self.joints = joints
        self.ties = list(ties) if ties is not None else []
        self._max_domains = len(domains) + 10
        self.rigidManager = None
        layout = SceneLayout(domains, dt=dt, damping=damping, useAdapativeDT=useAdapativeDT,
                             mass_scaling_dt=mass_scaling_dt, ties=self.ties)
        self._layout = layout
        self.stableTime = layout.stableTime
        self.useAdapative = layout.useAdapative
        self.damping = layout.damping
        self.dt = layout.dt
        self.default_dt = dt
        self.contacts = layout.contacts
        self.numContacts = len(layout.contacts)
        self._unbatched_contacts = layout.unbatched
        self._counter_py = 0
        self._packed = PackedWorld([layout])
        self._native = build_native(self._packed, device=device, path=path, patches=patches,
                                    front_warps=front_warps, res_sync=res_sync, res_threads=res_threads)
        if layout.mass_scaling_dt > 0.0:  # applyMassScaling after setGlobalAABB (explicitloop.py:168-169)
            self._native.mass_scaling(float(np.float32(layout.mass_scaling_dt)))
        self.path, self.patches = self._native.get_path()
        self.aabb = _AABBView(self)
        self.femSpringManager = FemSpringManager(self, self._packed, self._native, 0)
        self._flex_clock = None
        self._rigid_clock = None
        if layout.entries:  # rigid bodies, or the analytical entries of a loop with a moving plane
            self.rigidManager = RigidManager(self)
            self.rigid_update_times = 0
            for k, d in enumerate(layout.entries):
                if d.type in (DomainType.RIGID, DomainType.ANALYTICAL):  # height fields / voxel grids keep no state
                    d.attach(self, k)

    @property
    def damping(self) -> float:
        return self._damping

    @damping.setter
    def damping(self, value):
        """The reference reads ``self.damping`` at every substep
        (explicitloop.py:528, 537): a new value applies from the next substep,
        to the FEM update and to the rigid update."""
        self._damping = float(value)
        if getattr(self, "_native", None) is not None:
            self._native.set_damping(0, float(np.float32(self._damping)))
            self._rigid_clock = None  # the rigid schedule carries damping: re-sent at the next substep

    def _clock(self, dt: float):
        """Hand the substep's float64 dt to the FEM-FEM hash-refresh clock
        (femspringmanager.py:1035-1039 accumulates ``self.dt`` in float64) and
        to the rigid schedule: the rigids move every N = max(1, 1e-3 // dt)
        substeps by N * dt (explicitloop.py:533-538)."""
        if self._layout.flex and dt != self._flex_clock:
            self._native.set_flex_clock(dt)
            self._flex_clock = dt
        if self._layout.entries and dt != self._rigid_clock:
            every = max(1, RigidManager.stableTime // dt)
            self._native.set_rigid_clock(int(every), float(np.float32(every * dt)),
                                         float(np.float32(self.damping)))
            self._rigid_clock = dt

    def _rigid_state(self):
        """float32[numRigids, 12]: center, angle, V, angular velocity, U, box."""
        return self._entry_state()[:len(self._layout.rigids)]

    def _entry_state(self):
        """float32[entries, 12]: the rigids, then the analytical entries of a
        loop with a moving plane."""
        st, flags = self._native.read_rigids(len(self._layout.entries))
        if flags & 1:
            raise RuntimeError("a rigid body came within 0.01 of a ground or another contact rigid (rigid-rigid "
                               "and rigid-ground contact, the reference's constraint solve, are outside "
                               "flatworld_b200), or its state is no longer finite")
        return st

    # ---- stepping
    def advance(self):
        """One substep of ``self.dt`` (explicitloop.py:473-555)."""
        self._clock(self.dt)
        self._native.step(1, float(np.float32(self.dt)))
        self._counter_py += 1
        if self._layout.entries:
            self.rigid_update_times += 1

    def advance_n(self, n: int, dt: float | None = None):
        """``n`` substeps of ``dt`` (default ``self.dt``) queued in one call."""
        if dt is not None:
            self.dt = dt
        self._clock(self.dt)
        self._native.step(int(n), float(np.float32(self.dt)))
        self._counter_py += int(n)
        if self._layout.entries:
            self.rigid_update_times += int(n)

    def advanceWithTime(self, frame_dt: float = 1.0 / 60.0, verbose: bool = False):
        """Advance by exactly ``frame_dt`` of simulated time in substeps of at
        most stableTime (explicitloop.py:558-589)."""
        runs = substep_schedule(frame_dt, self.stableTime, self.default_dt, self.useAdapative)
        total = 0
        for n, sub in runs:
            self.dt = sub
            self._clock(sub)
            self._native.step(n, float(np.float32(sub)))
            self._counter_py += n
            total += n
        if self._layout.entries:
            self.rigid_update_times += total
        if verbose:
            print(f"Completed {total} substeps for {frame_dt} seconds of simulation time.")

    def synchronize(self):
        self._native.synchronize()

    def reset(self):
        raise NotImplementedError(
            "ExplicitLoop.reset() does not reset FEM state in the reference either "
            "(explicitloop.py:654-656); build a new loop to restart")

    def energy(self) -> dict:
        """Total energy of the scene, reduced in FP64 on the GPU: kinetic,
        strain, external (gravity / constant nodal force potential), contact
        (penalty) and their sum.  No reference counterpart."""
        k, s, e, c = (float(v) for v in self._native.energy(1)[0])
        return {"kinetic": k, "strain": s, "external": e, "contact": c, "total": k + s + e + c}

    def launch_count(self) -> int:
        return self._native.launch_count()

    def enable_cfl_monitor(self, on: bool = True):
        """Report the stable time of the current (deformed) mesh: the step
        also evaluates the reference's 0.4 * L_min / sqrt(E / rho)
        (femdomain.py:24) on every triangle's current shortest edge, reduced
        per scene on the GPU (every step implementation).  dt is not changed
        (the reference fixes it from the rest shape)."""
        self._native.set_cfl_monitor(self._packed.cfl_coefficients() if on else None)

    def currentStableTime(self, reset: bool = True) -> float:
        """Smallest current-shape stable time of the loop's triangles over the
        substeps since the last reset (+inf before any substep)."""
        return float(self._native.read_cfl(1, reset)[0])
