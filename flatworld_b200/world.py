"""Host-side packing of one or many scenes into one device world.

A *scene* is what one reference ``ExplicitLoop`` holds: FEM domains plus static
grounds, one time step, one step counter.  ``SceneLayout`` restates the
construction logic of the reference's ExplicitLoop / FemSpringManager /
MixedContact for one scene (explicitloop.py:72-398, femspringmanager.py:509-813,
femcontact.py:84-303, mixedcontact.py:1756-2270); ``World`` concatenates any
number of scenes into flat node / element / body / pair arrays and hands them
to the native library.  Scenes never interact, so a world of S scenes gives
the same per-scene results as S separate loops.
"""

from __future__ import annotations

import functools
import warnings
from dataclasses import dataclass

import numpy as np

from . import _native
from .definitions import (ATYPE, FORCETYPE, GRAVITY, ROTATYPE, ROTVTYPE, RTYPE, TORQUETYPE, UTYPE, VTYPE,
                          ContactType, DomainType)
from .rigid import RigidType

_SUPPORTED = (DomainType.FEM, DomainType.SPRINGMASS, DomainType.ANALYTICAL, DomainType.HEIGHTFIELD,
              DomainType.VOXELMAP, DomainType.RIGID)
_GROUND_TYPES = (DomainType.ANALYTICAL, DomainType.HEIGHTFIELD, DomainType.VOXELMAP)
_BODY_TYPES = (DomainType.FEM, DomainType.SPRINGMASS)
_SPRING_PENALTY_SCALE = 100.0  # femcontact.py:209, 246, 259, 272


def bulk_modulus(mat) -> float:
    """femcontact.py:94-98"""
    nu = min(mat.nu, 0.4999)
    return mat.E / (3.0 * (1.0 - 2.0 * nu))


def segment_penalty(dom) -> float:
    """femcontact.py:100-119, 2D branch: k = 2 K."""
    return 2.0 * 1.0 * bulk_modulus(dom.prop.mat)


def contact_stable_time(penalty: float, dom) -> float:
    """femcontact.py:121-141: 0.9 sqrt(m_node / k), m_node = rho L^2/2 / 3."""
    mat = dom.prop.mat
    L = dom.mesh.charLength
    m_node = mat.rho * (L * L * 0.5) / 3.0
    return 0.9 * (m_node / penalty) ** 0.5


@dataclass
class ContactSpec:
    kind: str  # "plane" | "heightfield" | "voxel" | "flex" | "rigid" | "spring-fem"
    fem: object     # the FEM domain (for "flex": domain1, the later domain)
    ground: object  # the ground (for "flex": domain2, the earlier FEM domain)
    pair_ids: tuple  # (later domain index, earlier domain index), explicitloop.py:275-276
    penalty: float
    stableTime: float
    friction: float = 0.0
    tied: bool = False  # named in ExplicitLoop(ties=...) (explicitloop.py:265-270)


def _contact_helper(di, dj, ctype, i, j):
    """contactHelper (femcontact.py:283-303) restricted to the FEM-ground,
    FEM-FEM, FEM-rigid and spring-mass pairs."""
    if ctype == ContactType.RIGIDSPRING:
        # ContactSpringRigid (femcontact.py:243-253): penalty 100 k, stable time
        # 0.5 sqrt(m / penalty); every spring node is a work item of the rigid
        # kernel (mixedcontact.py:2006-2018), friction the rigid's
        spring, rig = (di, dj) if di.type == DomainType.SPRINGMASS else (dj, di)
        pen = spring.spring * _SPRING_PENALTY_SCALE
        return ContactSpec("rigid", spring, rig, (i, j), pen, 0.5 * (spring.mass / pen) ** 0.5, float(rig.friction))
    if ctype == ContactType.FLEXRIGID:
        # ContactFlexRigid (femcontact.py:173-179): the FEM side's penalty and
        # stable time; friction = the rigid's (mixedcontact.py:1992)
        fem, rig = (di, dj) if di.type == DomainType.FEM else (dj, di)
        pen = segment_penalty(fem)
        return ContactSpec("rigid", fem, rig, (i, j), pen, contact_stable_time(pen, fem), float(rig.friction))
    if ctype in (ContactType.ANALYTICALSPRING, ContactType.SPRINGHEIGHTFIELD):
        # ContactSpringAnalytical / ContactSpringHeightField (femcontact.py:251-280):
        # penalty 100 k, stable time 0.5 sqrt(m / penalty)
        spring, ground = (di, dj) if di.type == DomainType.SPRINGMASS else (dj, di)
        pen = spring.spring * _SPRING_PENALTY_SCALE
        kind = "plane" if ctype == ContactType.ANALYTICALSPRING else "heightfield"
        return ContactSpec(kind, spring, ground, (i, j), pen, 0.5 * (spring.mass / pen) ** 0.5)
    if ctype == ContactType.FLEXSPRING:
        # ContactSpringFlex (femcontact.py:207-220): a reference contact the loop
        # never executes (it lands in the unbatched list); it bounds the stable
        # time and keeps the broad phase on
        spring, femd = (di, dj) if di.type == DomainType.SPRINGMASS else (dj, di)
        pen = min(spring.spring, segment_penalty(femd)) * _SPRING_PENALTY_SCALE
        return ContactSpec("spring-fem", spring, femd, (i, j), pen, contact_stable_time(pen, femd))
    kinds = {
        ContactType.FLEXANLAYTICAL: "plane",
        ContactType.FEXHEIGHTFIELD: "heightfield",
        ContactType.FLEXVOXELMAP: "voxel",
    }
    if ctype == ContactType.FLEXFLEX:
        # ContactFlexFlex (femcontact.py:199-206): the smaller side penalty, the
        # smaller side stable time; friction = max of the two (mixedcontact.py:1889)
        pen = min(segment_penalty(di), segment_penalty(dj)) * 1.0
        st = min(contact_stable_time(pen, di), contact_stable_time(pen, dj))
        return ContactSpec("flex", di, dj, (i, j), pen, st, max(di.friction, dj.friction))
    if ctype not in kinds:
        return None
    fem, ground = (di, dj) if di.type == DomainType.FEM else (dj, di)
    pen = segment_penalty(fem)
    return ContactSpec(kinds[ctype], fem, ground, (i, j), pen, contact_stable_time(pen, fem))


class SceneLayout:
    """Construction-time state of one scene (one reference ExplicitLoop)."""

    def __init__(self, domains, dt=0.0, damping=0.0, useAdapativeDT=True, mass_scaling_dt=0.0, ties=None):
        for d in domains:
            if d.type not in _SUPPORTED:
                raise NotImplementedError(f"domain type {d.type} is outside flatworld_b200's scope")
        self.domains = list(domains)
        # the bodies: FEM and spring-mass domains in loop order (FemSpringManager.domains)
        self.fem = [d for d in domains if d.type in _BODY_TYPES]
        if not self.fem:
            raise ValueError("a scene needs at least one FemDomain or SpringMassDomain")
        kinds = [d.type for d in self.fem]
        if DomainType.SPRINGMASS in kinds and DomainType.FEM in kinds[kinds.index(DomainType.SPRINGMASS):]:
            raise NotImplementedError(
                "a SpringMassDomain before a FemDomain: the reference's kernels take the first "
                "totalFEMElements elements as triangles (femspringmanager.py:231, 297), so list FEM domains first")
        self.damping = float(damping)
        self.useAdapative = bool(useAdapativeDT)
        # explicitloop.py:145-170: 1.0, capped by the rigid manager's 1e-3 when an
        # analytical plane exists, then by every FEM domain's CFL bound
        stable = 1.0
        if any(d.type in (DomainType.RIGID, DomainType.ANALYTICAL) for d in domains):
            stable = min(1.0 / 1000.0, stable)
        fsm_stable = 1.0
        for d in self.fem:
            fsm_stable = min(d.stableTime, fsm_stable)
        stable = min(fsm_stable, stable)
        # explicitloop.py:168-170: mass scaling lifts the bound to its target
        # (contacts may lower it again below)
        self.mass_scaling_dt = float(mass_scaling_dt)
        if self.mass_scaling_dt > 0.0:
            stable = max(stable, self.mass_scaling_dt)
        # explicitloop.py:237-277: O(D^2) pair loop over contact domains
        contacts = []
        contact_domains = [(i, d) for i, d in enumerate(domains) if d.considerContact]
        if any(d.type in _BODY_TYPES for d in domains if d.considerContact):
            for a, (i, di) in enumerate(contact_domains):
                for b in range(a):
                    j, dj = contact_domains[b]
                    ctype = di.type | dj.type
                    if di.category_bits & dj.collide_bits == 0:
                        continue
                    if di.collide_bits & dj.category_bits == 0:
                        continue
                    if ctype in (ContactType.RIGIDRIGID, ContactType.RIGIDANLAYTICAL,
                                 ContactType.ANALYTICALANALYTICAL):
                        continue
                    if hasattr(di, "env_id") and hasattr(dj, "env_id") and di.env_id != dj.env_id:
                        continue
                    spec = _contact_helper(di, dj, ctype, i, j)
                    if spec is not None:
                        contacts.append(spec)
        # ties (explicitloop.py:400-439): (domain, domain) index pairs, negative
        # indices counted from the end; unresolvable entries are ignored
        tie_pairs = set()
        for t in (ties or []):
            if not isinstance(t, (tuple, list)) or len(t) != 2:
                continue
            a, b = t
            if not isinstance(a, (int, np.integer)) or not isinstance(b, (int, np.integer)):
                continue
            ia, ib = int(a) + (len(domains) if a < 0 else 0), int(b) + (len(domains) if b < 0 else 0)
            if 0 <= ia < len(domains) and 0 <= ib < len(domains) and ia != ib:
                tie_pairs.add((min(ia, ib), max(ia, ib)))
        for c in contacts:
            c.tied = (min(c.pair_ids), max(c.pair_ids)) in tie_pairs
        self.contacts = contacts
        for c in contacts:  # explicitloop.py:313-315
            stable = min(stable, c.stableTime)
        self.stableTime = stable
        self.default_dt = dt
        self.dt = stable if useAdapativeDT else dt  # explicitloop.py:329-334
        # mixedcontact.py:1794-2261: planes, then the single height field, then
        # the single voxel grid; a second distinct height field (or voxel grid)
        # sends all of that kind to the never-executed "unbatched" list
        anal = [c for c in contacts if c.kind == "plane"]
        hf = [c for c in contacts if c.kind == "heightfield"]
        vox = [c for c in contacts if c.kind == "voxel"]
        self.unbatched = [c for c in contacts if c.kind == "spring-fem"]
        if len({id(c.ground) for c in hf}) > 1:
            warnings.warn("more than one HeightFieldDomain in a loop: like the reference, height-field "
                          "contact is not executed for any of them", RuntimeWarning)
            self.unbatched += hf
            hf = []
        if len({id(c.ground) for c in vox}) > 1:
            warnings.warn("more than one VoxelGridDomain in a loop: like the reference, voxel contact "
                          "is not executed for any of them", RuntimeWarning)
            self.unbatched += vox
            vox = []
        # FEM-rigid pairs run after FEM-FEM contact, before the height field
        # (mixedcontact.py:1697-1715), in contact order
        rig = [c for c in contacts if c.kind == "rigid"]
        self.pairs = anal + rig + hf + vox
        # RigidManager: rigid bodies in domain order (rigidmanager.py:2448-2480)
        self.rigids = [d for d in domains if d.type == DomainType.RIGID]
        self.grounds = [d for d in domains if d.type in _GROUND_TYPES]
        # a ground plane with BCs makes the rigid manager move its analytical
        # entries (planes, height fields, voxel grids, in domain order) and
        # recompute their broad-phase boxes (rigidmanager.py:2510-2517, 2580-2586)
        self.moving = any(d.type == DomainType.ANALYTICAL and len(d.bcs) > 0 for d in domains)
        if self.moving and self.rigids:
            raise NotImplementedError("a ground plane with BCs together with rigid bodies: the clearance check "
                                      "of the rigids against a moving plane is not part of flatworld_b200")
        self.entries = self.rigids + (self.grounds if self.moving else [])
        # FEM-FEM pairs in contact-creation order (mixedcontact.py:1869-1935); the
        # loop skips the BVH (all pairs stay active / plain box tests) when it has
        # no ground contact and at most one contact rigid (explicitloop.py:362-373)
        self.flex = [c for c in contacts if c.kind == "flex"]
        rigid_needs_bvh = sum(1 for d in self.rigids if d.considerContact) > 1
        no_bvh = len(contact_domains) <= 1  # explicitloop.py:222-228: no broad phase object
        self.skip_bvh = no_bvh or not (anal or hf or vox or self.unbatched or rigid_needs_bvh)
        self.n_nodes = sum(d.nnodes for d in self.fem)
        self.n_elems = sum(d.nelements for d in self.fem)


class PackedWorld:
    """Flat arrays of a list of scenes (scene-major, FEM domains in order)."""

    def __init__(self, scenes: list[SceneLayout]):
        self.scenes = scenes
        N = sum(s.n_nodes for s in scenes)
        E = sum(s.n_elems for s in scenes)
        self.N, self.E = N, E
        coords = np.zeros((N, 2), np.float32)
        vel = np.zeros((N, 2), np.float32)
        bc_bits = np.zeros(N, np.int32)
        bc_vals = np.zeros((N, 2), np.float32)
        conn = np.zeros((E, 3), np.int32)
        mtype = np.zeros(E, np.int32)
        Ev = np.zeros(E, np.float32)
        nuv = np.zeros(E, np.float32)
        rhov = np.zeros(E, np.float32)
        syv = np.zeros(E, np.float32)
        Hv = np.zeros(E, np.float32)
        noff, ncnt, eoff, ecnt, bscene, bnoff, bncnt, bnodes = [], [], [], [], [], [], [], []
        beoff, becnt, bedges = [], [], []
        spring_bodies = []
        self.body_of = {}  # (scene idx, fem idx) -> global body id
        self.scene_bodies = []
        n0 = e0 = b0 = 0
        for si, sc in enumerate(scenes):
            bodies = []
            for fi, dom in enumerate(sc.fem):
                spring = dom.type == DomainType.SPRINGMASS
                if spring:
                    # addSpringDomain (femspringmanager.py:815-870): 2-node springs,
                    # type 0; stiffness, damping and rest length ride in E, nu, rho
                    nn, ne = dom.nnodes, dom.nelements
                    coords[n0:n0 + nn] = np.asarray(dom.coords, dtype=np.float32)[:, :2]
                    conn[e0:e0 + ne, :2] = np.asarray(dom.connectivity, dtype=np.int64)[:, :2] + n0
                    conn[e0:e0 + ne, 2] = -1
                    mtype[e0:e0 + ne] = 0
                    Ev[e0:e0 + ne] = float(dom.spring)
                    nuv[e0:e0 + ne] = float(dom.damping)
                    rhov[e0:e0 + ne] = dom.restLength
                    spring_bodies.append((b0 + fi, float(np.float32(dom.mass))))
                else:
                    mesh = dom.mesh
                    nn, ne = mesh.numNodes, mesh.numElements
                    coords[n0:n0 + nn] = np.asarray(mesh.coords, dtype=np.float32)[:, :2]
                    conn[e0:e0 + ne] = np.asarray(mesh.connectivity, dtype=np.int64)[:, :3] + n0
                    mat = dom.prop.getMaterial()
                    mtype[e0:e0 + ne] = int(mat.type)
                    ey = getattr(dom, "elementYoung", None)  # optional per-element E (else the material's)
                    Ev[e0:e0 + ne] = float(mat.E) if ey is None else np.asarray(ey, np.float32).reshape(ne)
                    nuv[e0:e0 + ne] = float(mat.nu)
                    rhov[e0:e0 + ne] = float(mat.rho)
                    syv[e0:e0 + ne] = float(getattr(mat, "sigma_y", 0.0))
                    Hv[e0:e0 + ne] = float(getattr(mat, "H", 0.0))
                # processConditions (femspringmanager.py:660-705)
                for bc in dom.bcs:
                    t, nodes, values = bc.processData()
                    if values is None:
                        values = [0.0] * dom.d
                    idx = np.arange(nn) if nodes is None else np.asarray(nodes, dtype=np.int64).reshape(-1)
                    bc_bits[n0 + idx] |= int(t)
                    bc_vals[n0 + idx, 0] = float(values[0])
                    bc_vals[n0 + idx, 1] = float(values[1])
                for ic in dom.initials:
                    if not hasattr(ic, "vel"):
                        raise NotImplementedError(f"initial condition {type(ic).__name__} is not an FEM initial condition")
                    vx, vy = float(ic.vel[0]), float(ic.vel[1])
                    if getattr(ic, "is_all_nodes", False):
                        vel[n0:n0 + nn] = (vx, vy)
                    else:
                        ids = n0 + np.asarray(ic.nds, dtype=np.int64).reshape(-1)
                        vel[ids] = (vx, vy)
                b = b0 + fi
                self.body_of[(si, fi)] = b
                bodies.append(b)
                noff.append(n0)
                ncnt.append(nn)
                eoff.append(e0)
                ecnt.append(ne)
                bscene.append(si)
                bnoff.append(sum(len(x) for x in bnodes))
                # a spring domain's contact work items and box cover all its nodes
                bn = n0 + (np.arange(nn, dtype=np.int64) if spring else np.asarray(mesh.boundaryNodes, dtype=np.int64))
                bncnt.append(len(bn))
                bnodes.append(bn)
                beoff.append(sum(len(x) for x in bedges))
                be = (np.zeros((0, 2), np.int64) if spring
                      else n0 + np.asarray(mesh.boundaryElements, dtype=np.int64).reshape(-1, 2))
                becnt.append(len(be))
                bedges.append(be)
                n0 += nn
                e0 += ne
            b0 += len(sc.fem)
            self.scene_bodies.append(bodies)
        self.coords, self.vel, self.bc_bits, self.bc_vals = coords, vel, bc_bits, bc_vals
        self.conn, self.mtype, self.Ev, self.nuv, self.rhov, self.syv, self.Hv = conn, mtype, Ev, nuv, rhov, syv, Hv
        self.noff = np.asarray(noff, np.int32)
        self.ncnt = np.asarray(ncnt, np.int32)
        self.eoff = np.asarray(eoff, np.int32)
        self.ecnt = np.asarray(ecnt, np.int32)
        self.bscene = np.asarray(bscene, np.int32)
        self.bnoff = np.asarray(bnoff, np.int32)
        self.bncnt = np.asarray(bncnt, np.int32)
        self.bnodes = np.concatenate(bnodes).astype(np.int32) if bnodes else np.zeros(0, np.int32)
        self.spring_bodies = spring_bodies  # (body id, node mass f32)
        self.beoff = np.asarray(beoff, np.int32)
        self.becnt = np.asarray(becnt, np.int32)
        self.bedges = np.concatenate(bedges).astype(np.int32) if bedges else np.zeros((0, 2), np.int32)
        self.B = len(noff)
        self.S = len(scenes)

    def cfl_coefficients(self):
        """Per body, 0.4 / sqrt(E / rho) of its material (the factor of the
        reference's FemDomain.stableTime = 0.4 * L_min / sqrt(E / rho),
        femdomain.py:24), float32; 0 for spring-mass domains."""
        out = np.zeros(self.B, np.float32)
        for si, sc in enumerate(self.scenes):
            for fi, dom in enumerate(sc.fem):
                if dom.type == DomainType.FEM:
                    mat = dom.prop.getMaterial()
                    out[self.body_of[(si, fi)]] = 0.4 / (float(mat.E) / float(mat.rho)) ** 0.5
        return out

    def rigid_records(self):
        """Per rigid, scene-major: float32[16] and int32[4] (type, BC bits,
        considerContact, scene) for fw_set_rigids; per ground of a scene with
        rigids: float32[6] (kind, point + normal or box, scene)."""
        params, ints, boxes = [], [], []
        for si, sc in enumerate(self.scenes):
            if not sc.entries:
                continue
            for dom in sc.rigids:
                p, i = rigid_record(dom)
                params.append(p)
                ints.append([*i, si])
            for g in (sc.grounds if sc.moving else []):
                p, i = analytical_record(g)
                params.append(p)
                ints.append([*i, si])
            if not sc.rigids:
                continue
            for g in sc.grounds:  # plane: kind 0, point, normal; height field / voxel grid: kind 1, box
                if g.type == DomainType.ANALYTICAL:
                    boxes.append([0.0, *np.asarray(g.point, np.float32)[:2], *np.asarray(g.normal, np.float32)[:2],
                                  si])
                else:
                    lo, hi = g.getBBox()
                    boxes.append([1.0, *np.asarray(lo, np.float32).reshape(2), *np.asarray(hi, np.float32).reshape(2),
                                  si])
        as2 = lambda a, w, dt: np.asarray(a, dt).reshape(-1, w)  # noqa: E731
        return as2(params, 20, np.float32), as2(ints, 4, np.int32), as2(boxes, 6, np.float32)

    def rigid_offsets(self):
        """Index of each scene's first entry (rigids, then the analytical
        entries of a loop with a moving plane) in the world's entry list."""
        off, n = [], 0
        for sc in self.scenes:
            off.append(n)
            n += len(sc.entries)
        return off

    def ground_gate_entries(self):
        """Per pair of pair_records(): the entry whose current box gates it
        (a ground pair of a loop with a moving plane), else -1."""
        out = []
        r_off = self.rigid_offsets()
        for si, sc in enumerate(self.scenes):
            for c in sc.pairs:
                moving_ground = sc.moving and c.kind != "rigid"
                out.append(r_off[si] + sc.entries.index(c.ground) if moving_ground else -1)
        return out

    def flex_records(self):
        """Per scene with FEM-FEM pairs: (scene, skip_bvh, dom_obj, dom_body,
        dom_box, [(body1, body2, penalty f32, friction f32, tied)])."""
        out = []
        for si, sc in enumerate(self.scenes):
            if not sc.flex:
                continue
            fem_index = {id(d): k for k, d in enumerate(sc.fem)}
            dom_obj = np.asarray([1 if d.considerContact else 0 for d in sc.domains], np.int32)
            rig_index = {id(d): self.rigid_offsets()[si] + k for k, d in enumerate(sc.entries)}
            dom_body = np.asarray([self.body_of[(si, fem_index[id(d)])] if id(d) in fem_index
                                   else (-2 - rig_index[id(d)] if id(d) in rig_index else -1)
                                   for d in sc.domains], np.int32)
            dom_box = np.zeros((len(sc.domains), 4), np.float32)
            for g, d in enumerate(sc.domains):  # grounds: static boxes; bodies, rigids: boxes on the device
                if id(d) not in fem_index and id(d) not in rig_index and d.considerContact:
                    lo, hi = d.getBBox()
                    dom_box[g, :2] = np.asarray(lo, np.float32).reshape(2)
                    dom_box[g, 2:] = np.asarray(hi, np.float32).reshape(2)
            pairs = [(self.body_of[(si, fem_index[id(c.fem)])], self.body_of[(si, fem_index[id(c.ground)])],
                      np.float32(c.penalty), np.float32(c.friction), bool(c.tied)) for c in sc.flex]
            out.append((si, sc.skip_bvh, dom_obj, dom_body, dom_box, pairs))
        return out

    def pair_records(self):
        """(kind, body, penalty f32, gate lo, gate hi, ground) in launch order."""
        out = []
        r_off = self.rigid_offsets()
        for si, sc in enumerate(self.scenes):
            fem_index = {id(d): k for k, d in enumerate(sc.fem)}
            for c in sc.pairs:
                body = self.body_of[(si, fem_index[id(c.fem)])]
                if c.kind == "rigid":  # the gate box is the rigid's current one, on the device
                    rid = r_off[si] + next(k for k, d in enumerate(sc.rigids) if d is c.ground)
                    out.append((c.kind, body, np.float32(c.penalty), rid, np.float32(c.friction),
                                (sc.skip_bvh, c.tied)))
                    continue
                lo, hi = c.ground.getBBox()
                out.append((c.kind, body, np.float32(c.penalty), np.asarray(lo, np.float32),
                            np.asarray(hi, np.float32), c.ground))
        return out


def build_native(packed: PackedWorld, device: int = 0, path: str = "auto", patches: int = 0,
                 front_warps: int = 0, res_sync: int = 0, stream_patch: int = 0,
                 res_threads: int = 0) -> _native.NativeWorld:
    """Create the device world.  ``path``: "auto" (shared-memory-resident step
    when the world fits on chip, else the gather step), "gather" or "resident";
    ``patches`` / ``front_warps``: resident-step tuning (0 = default);
    ``res_sync``: 0 = flag-in-data hand-off between resident CTAs, 1 = arrival
    counter (FW_OPT_RES_SYNC); ``stream_patch``: owned nodes per patch of the
    stream step (64 or 128; 0 = default); ``res_threads``: threads of a
    resident CTA (512 or 1024; 0 = default)."""
    nw = _native.NativeWorld(device)
    nw.set_path(_native.PATHS[path], patches)
    if res_threads:
        nw.set_option(_native.FW_OPT_RES_THREADS, res_threads)
    if front_warps:
        nw.set_option(_native.FW_OPT_FRONT_WARPS, front_warps)
    if res_sync:
        nw.set_option(_native.FW_OPT_RES_SYNC, res_sync)
    if stream_patch:
        nw.set_option(_native.FW_OPT_STREAM_PATCH, stream_patch)
    stage(nw, packed)
    nw.finalize()
    return nw


def stage(nw: _native.NativeWorld, packed: PackedWorld):
    """Hand a packed world's arrays to the native context (fw_set_* and
    fw_add_*_pair); an arena then commits them as one scene."""
    nw.set_nodes(packed.coords, packed.vel, packed.bc_bits, packed.bc_vals)
    nw.set_elements(packed.conn, packed.mtype, packed.Ev, packed.nuv, packed.rhov, packed.syv, packed.Hv)
    nw.set_bodies(packed.noff, packed.ncnt, packed.eoff, packed.ecnt, packed.bscene, packed.bnoff,
                  packed.bncnt, packed.bnodes)
    if packed.spring_bodies:
        nw.set_spring_bodies(np.asarray([b for b, _ in packed.spring_bodies], np.int32),
                             np.asarray([m for _, m in packed.spring_bodies], np.float32))
    nw.set_scenes(np.asarray([s.damping for s in packed.scenes], np.float32))
    if any(sc.entries for sc in packed.scenes):
        nw.set_rigids(*packed.rigid_records())
    for (kind, body, pen, lo, hi, g), gate in zip(packed.pair_records(), packed.ground_gate_entries()):
        if kind == "rigid":  # (rigid index, friction, (skip_bvh, tied)) in the box and ground slots
            nw.add_rigid_pair(body, lo, pen, hi, 1 if g[0] else 0, 1 if g[1] else 0)
            continue
        if kind == "plane":  # the plane of construction time, also when it moves (mixedcontact.py:1815-1818)
            nw.add_plane(body, pen, lo, hi, g.point, g.normal)
        elif kind == "heightfield":
            nw.add_heightfield(body, pen, lo, hi, g.height, g.lb[0], g.ub[0], 1 if g.reverse else 0)
        else:
            nw.add_voxel(body, pen, lo, hi, np.asarray(g.occ, np.int32), g.lb[0], g.lb[1], g.dx, g.dz)
        if gate >= 0:
            nw.gate_by_rigid(gate)
    flex = packed.flex_records()
    if flex:
        nw.set_boundary_edges(packed.bedges, packed.beoff, packed.becnt)
        n_flex = 0
        for si, skip, obj, body, box, pairs in flex:
            nw.set_flex_scene(si, skip, obj, body, box)
            for b1, b2, pen, fric, tied in pairs:
                nw.add_flex_pair(b1, b2, pen, fric)
                if tied:
                    nw.tie_flex_pair(n_flex)
                n_flex += 1


def _as_float(v) -> float:
    """rigidmanager.py:77-81: the first element of a sequence, else float(v)."""
    if hasattr(v, "__len__") and not isinstance(v, (str, bytes)):
        return float(np.asarray(v, dtype=np.float32).reshape(-1)[0])
    return float(v)


def _as_vec2(v):
    a = np.asarray(v, dtype=np.float32).reshape(-1)
    return float(a[0]), (float(a[1]) if a.size > 1 else 0.0)


def rigid_record(dom):
    """One rigid as RigidManager stores it: RigidBodyDomain.attach (initial
    conditions, rigiddomain.py:118-124), packRigidParams (rigidmanager.py:
    2250-2400) and processConditions / _addBcValue (2527-2567), in that order.
    Returns float32[20] (center, primary, radius, angle, mass, inertia, V,
    angular velocity, BC translation value, gravity, BC rotation value, 4
    unused) and int32[3] (type, BC bits, considerContact)."""
    r = dom.rigid
    f = np.zeros(20, np.float32)
    for ic in dom.initials:
        ids = [0] if getattr(ic, "is_all_nodes", False) else [int(n) for n in np.asarray(ic.nds).reshape(-1)]
        if ids != [0]:
            raise NotImplementedError("a rigid body's initial condition must name index 0 (or 'ALL')")
        if ic.type in (VTYPE, ATYPE):
            f[8], f[9] = _as_vec2(ic.vel)
        else:
            f[10] = _as_float(ic.ang_vel)
    ref = np.asarray(r.getRefPoint(), np.float32).reshape(-1)
    f[0], f[1] = _as_vec2(ref)
    f[6] = _as_float(r.mass)
    if r.rtype == RigidType.BALL:
        f[4] = _as_float(r.getRadius())
    elif r.rtype == RigidType.BOX:
        f[2], f[3] = _as_vec2(r.getPrimary())
    elif r.rtype == RigidType.CAPSULE:
        f[2], f[3] = _as_vec2(r.getPrimary() - r.getRefPoint())
        f[4] = _as_float(r.getRadius())
    f[5] = _as_float(r.angle)
    f[7] = float(r.inertia_body)
    bits = _rigid_bcs(dom.bcs, f)
    return f, np.array([int(r.rtype), bits, 1 if dom.considerContact else 0], np.int32)


def analytical_record(g):
    """The rigid manager's entry for a ground of a loop with a moving plane
    (processDomains_, rigidmanager.py:2486-2517; GroundDomain.attach's initial
    conditions; processConditions): a plane's point and normal as its center
    and primary vector (zero for a height field or voxel grid, whose entries
    the reference never fills), mass 1e10, its BCs, and its getBBox() as the
    first broad-phase box."""
    f = np.zeros(20, np.float32)
    if g.type == DomainType.ANALYTICAL:
        f[0], f[1] = _as_vec2(g.point)
        f[2], f[3] = _as_vec2(g.normal)
    f[6] = 1e10
    for ic in getattr(g, "initials", []):
        if ic.type in (VTYPE, ATYPE):
            f[8], f[9] = _as_vec2(ic.vel)
        else:
            f[10] = _as_float(ic.ang_vel)
    bits = _rigid_bcs(getattr(g, "bcs", []), f)
    lo, hi = g.getBBox()
    f[16], f[17] = _as_vec2(lo)
    f[18], f[19] = _as_vec2(hi)
    return f, np.array([64, bits, 1 if g.considerContact else 0], np.int32)


def _rigid_bcs(bcs, f):
    """processConditions -> _addBcValue (rigidmanager.py:2527-2553) on one
    entry's record; returns its BC bits."""
    bits = 0
    for bc in bcs:
        t, _, value = bc.processData()
        t = int(t)
        bits |= t
        if t == UTYPE:
            f[11:13] = 0.0
            f[6] = 1e10
        elif t == RTYPE:
            f[11:13] = 0.0
            f[6] = 1e10
            f[7] = 1e10
            f[15] = 0.0
        elif t == VTYPE:
            f[11], f[12] = _as_vec2(value)
            f[6] = 1e10
        elif t == ROTVTYPE:
            f[15] = _as_float(value)
            f[7] = 1e10
        elif t in (ROTATYPE, TORQUETYPE):
            f[15] = _as_float(value)
        elif t == GRAVITY:
            f[13], f[14] = _as_vec2(value)
        else:  # ATYPE, FORCETYPE
            f[11], f[12] = _as_vec2(value)
    return bits


def substep_schedule(frame_dt: float, stable: float, default_dt: float, adaptive: bool):
    """advanceWithTime's float64 substep loop (explicitloop.py:573-586) as a list
    of (count, dt) runs.  Memoised: a request loop asks for the same few
    (frame, dt) pairs over and over, and the loop walks every substep."""
    return list(_substep_schedule(float(frame_dt), float(stable), float(default_dt), bool(adaptive)))


@functools.lru_cache(maxsize=4096)
def _substep_schedule(frame_dt: float, stable: float, default_dt: float, adaptive: bool):
    remaining = float(frame_dt)
    runs = []
    while remaining > 1e-12:
        cur = stable if adaptive else default_dt
        sub = max(min(cur, remaining), 1e-8)
        if runs and runs[-1][1] == sub:
            runs[-1][0] += 1
        else:
            runs.append([1, sub])
        remaining -= sub
    return tuple((n, d) for n, d in runs)
