"""Oracle driver: literal restatement of the reference's host-side construction
and stepping logic, running the C oracle (fw_oracle.c) for the device work.

TEST INFRASTRUCTURE ONLY -- imported by tests/, __graft_entry__.smoke() and
bench.py's CPU legs as the checker; never by the product package.

It deliberately shares no code with flatworld_b200: boundary edges, edge
lengths, stable time, contact pairs, penalties, work lists and BC packing are
recomputed here with the reference's own loops:
  flatworld/mesh.py:40-112                 boundary edges, char lengths
  flatworld/femdomain.py:24                FemDomain.stableTime
  flatworld/femcontact.py:94-141, 155-197  penalty 2K, contact stable time
  flatworld/explicitloop.py:145-334        stable dt, O(D^2) contact pairs
  flatworld/femspringmanager.py:660-813    packing, processConditions
  flatworld/mixedcontact.py:1794-2261      work lists (one HF / voxel domain)
  flatworld/grounddomain.py:54-70, heightfielddomain.py:26-27,190-194,
  voxeldomain.py:194-195                   broad-phase boxes
  flatworld/explicitloop.py:558-589        advanceWithTime substep loop
  flatworld/femcontact.py:199-206          ContactFlexFlex penalty, stable time
  flatworld/mixedcontact.py:1869-1935      FEM-FEM work items
  flatworld/explicitloop.py:203-227, 362-373, 383-385  BVH objects, skip_bvh,
                                           initial FEM spatial hash
  flatworld/femspringmanager.py:523-524, 1035-1039  hash refresh every 1/500 s
  flatworld/femcontact.py:173-179          ContactFlexRigid penalty, stable time
  flatworld/mixedcontact.py:1963-2054      FEM-rigid work items (friction of the rigid)
  flatworld/rigiddomain.py:118-124, rigidmanager.py:2250-2400, 2448-2567
                                           rigid packing, BCs, initial conditions
  flatworld/explicitloop.py:533-538        rigid update every max(1, 1e-3 // dt) substeps
Domain objects are read through the reference's attribute names only
(mesh.coords, mesh.connectivity, prop.mat, bcs, initials, point, normal,
height, lb, ub, reverse, occ, nx, ny, dx, dz, considerContact, type, ...).
"""

from __future__ import annotations

import ctypes as C
import os
from collections import defaultdict

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# flatworld/definitions.py
FEM, ANALYTICAL, RIGID, SPRINGMASS, HEIGHTFIELD, VOXELMAP = 0b10, 0b1, 0b100, 0b1000, 0b100000, 0b1000000
FLEXANLAYTICAL, FLEXFLEX, FEXHEIGHTFIELD, FLEXVOXELMAP = 0b11, 0b10, 0b100010, 0b1000010
FLEXSPRING, ANALYTICALSPRING, SPRINGHEIGHTFIELD = 0b1010, 0b1001, 0b101000
FLEXRIGID = 0b110
RIGIDRIGID, RIGIDANLAYTICAL, ANALYTICALANALYTICAL = 0b100, 0b101, 0b1

_LIBS = {}
_f32p = C.POINTER(C.c_float)
_i32p = C.POINTER(C.c_int32)
_f64p = C.POINTER(C.c_double)


def _lib(precision: str):
    name = {"f32": "liboracle_f32.so", "f32fma": "liboracle_f32fma.so", "f32libm": "liboracle_f32libm.so",
            "f64": "liboracle_f64.so"}[precision]
    if name not in _LIBS:
        path = os.path.join(HERE, name)
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: run `make -C oracle`")
        L = C.CDLL(path)
        L.or_create.restype = C.c_void_p
        L.or_create.argtypes = [C.c_int, _f32p, _f32p, _i32p, _f32p, C.c_int, _i32p, _i32p, _f32p, _f32p, _f32p,
                                _f32p, _f32p, C.c_int, _i32p, _i32p, C.c_int, _i32p]
        L.or_add_plane.argtypes = [C.c_void_p, C.c_int, C.c_float, _f32p, _f32p, C.c_float, C.c_float, C.c_float,
                                   C.c_float]
        L.or_add_heightfield.argtypes = [C.c_void_p, C.c_int, C.c_float, _f32p, _f32p, C.c_int, _f32p, C.c_float,
                                         C.c_float, C.c_int]
        L.or_add_voxel.argtypes = [C.c_void_p, C.c_int, C.c_float, _f32p, _f32p, C.c_int, C.c_int, _i32p,
                                   C.c_float, C.c_float, C.c_float, C.c_float]
        L.or_set_threads.argtypes = [C.c_void_p, C.c_int]
        L.or_step.argtypes = [C.c_void_p, C.c_float, C.c_float, C.c_long, C.c_int]
        L.or_get_state.argtypes = [C.c_void_p, _f64p, _f64p, _f64p]
        L.or_get_prepared.argtypes = [C.c_void_p, _f64p, _f64p, _f64p]
        L.or_get_plastic.argtypes = [C.c_void_p, _f64p, _f64p]
        L.or_get_aabb.argtypes = [C.c_void_p, _f64p]
        L.or_set_state.argtypes = [C.c_void_p, _f32p, _f32p]
        L.or_point_stress.argtypes = [C.c_int, C.c_float, C.c_float, C.c_float, C.c_float, _f32p, _f32p, C.c_float,
                                      _f64p, _f64p, _f64p]
        L.or_set_flex.argtypes = [C.c_void_p, C.c_int, _i32p, _i32p, _i32p, C.c_int, _i32p, _i32p, _f32p, C.c_int]
        L.or_add_flex_pair.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_float]
        L.or_set_flex_pair_tied.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.or_flex_counts.argtypes = [C.c_void_p, _i32p]
        L.or_flex_rebuild.argtypes = [C.c_void_p]
        L.or_get_flex_cache.argtypes = [C.c_void_p, _i32p]
        L.or_get_flex_grid.argtypes = [C.c_void_p, _f64p]
        L.or_mass_scaling.argtypes = [C.c_void_p, C.c_float]
        L.or_set_spring_mass.argtypes = [C.c_void_p, C.c_int, C.c_float]
        L.or_destroy.argtypes = [C.c_void_p]
        L.or_log32.argtypes = [C.c_float]
        L.or_log32.restype = C.c_float
        L.or_set_rigids.argtypes = [C.c_void_p, C.c_int, _f32p, _i32p, C.c_int, _f32p]
        L.or_add_rigid_pair.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, C.c_int]
        L.or_rigid_update.argtypes = [C.c_void_p, C.c_float, C.c_float]
        L.or_get_rigids.argtypes = [C.c_void_p, _f64p]
        L.or_get_rigids.restype = C.c_int
        L.or_sincos32.argtypes = [C.c_float, _f32p, _f32p]
        L.or_gate_by_rigid.argtypes = [C.c_void_p, C.c_int]
        L.or_adjoint.argtypes = [C.c_void_p, C.c_int, C.c_float, C.c_float, C.c_long, _f64p, _f64p, _f64p, _f64p,
                                 _f64p]
        L.or_adjoint.restype = C.c_int
        L.or_set_young64.argtypes = [C.c_void_p, _f64p]
        L.or_set_state64.argtypes = [C.c_void_p, _f64p, _f64p]
        _LIBS[name] = L
    return _LIBS[name]


def _fp(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(_f32p)


def _ip(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(_i32p)


# ---------------------------------------------------------------- host restatement

def boundary_edges_literal(conns):
    """mesh.py:53-71, loop for loop: edges seen once, in first-seen order and
    orientation."""
    edge_count = defaultdict(int)
    for cell in np.asarray(conns).tolist():
        for i in range(3):
            v1, v2 = cell[i], cell[(i + 1) % 3]
            if (v2, v1) in edge_count:
                edge_count[(v2, v1)] += 1
            else:
                edge_count[(v1, v2)] += 1
    return np.array([e for e, c in edge_count.items() if c == 1], dtype=np.int64).reshape(-1, 2)


def boundary_nodes_literal(conns):
    """mesh.py:53-71 and 40-47, loop for loop."""
    edge_count = defaultdict(int)
    for cell in np.asarray(conns).tolist():
        for i in range(3):
            v1, v2 = cell[i], cell[(i + 1) % 3]
            if (v2, v1) in edge_count:
                edge_count[(v2, v1)] += 1
            else:
                edge_count[(v1, v2)] += 1
    nodes = set()
    for e, c in edge_count.items():
        if c == 1:
            nodes.update(e)
    return np.array(sorted(nodes), dtype=np.int64)


def char_length_literal(conns, coords):
    """mesh.py:73-78, 90-112: min over float32 norm(a - b) of element edges."""
    coords = np.asarray(coords)
    lengths = []
    for conn in np.asarray(conns):
        for ia, ib in ((0, 1), (1, 2), (2, 0)):
            lengths.append(np.linalg.norm(coords[conn[ia]] - coords[conn[ib]]))
    return float(np.min(np.asarray(lengths, dtype=np.float32)))


def point_stress(mtype, E, nu, F, sigma_y=0.0, H=0.0, eps_p=None, eqps=0.0, precision="f32"):
    """One material-point evaluation of getStress2D / misesReturnMap2D."""
    L = _lib(precision)
    Fa = _fp(np.asarray(F, np.float32).reshape(4))
    ep = _fp(np.zeros(3, np.float32) if eps_p is None else eps_p)
    s = np.zeros(3)
    epo = np.zeros(3)
    eqo = np.zeros(1)
    L.or_point_stress(int(mtype), float(E), float(nu), float(sigma_y), float(H), Fa[1], ep[1], float(eqps),
                      s.ctypes.data_as(_f64p), epo.ctypes.data_as(_f64p), eqo.ctypes.data_as(_f64p))
    return s, epo, float(eqo[0])


def log32(x, precision="f32"):
    """The FP32 log the oracle uses (for its accuracy test)."""
    return float(_lib(precision).or_log32(float(x)))


def sincos32(x):
    """The FP32 (sin, cos) the oracle and the CUDA rigid update use."""
    sv, cv = C.c_float(), C.c_float()
    _lib("f32").or_sincos32(float(x), C.byref(sv), C.byref(cv))
    return sv.value, cv.value


class OracleLoop:
    """CPU restatement of one reference ExplicitLoop over FEM + ground domains."""

    def __init__(self, domains, dt=0.0, damping=0.0, useAdapativeDT=True, precision="f32", threads=1,
                 mass_scaling_dt=0.0, ties=None):
        self.precision = precision
        L = self._L = _lib(precision)
        self.domains = list(domains)
        # bodies: FEM and spring-mass domains in loop order (FemSpringManager.domains)
        fem = [d for d in domains if d.type in (FEM, SPRINGMASS)]
        self.fem = fem
        # --- stable time (explicitloop.py:145-170, femdomain.py:24)
        stable = 1.0
        if any(d.type in (RIGID, ANALYTICAL) for d in domains):
            stable = min(1.0 / 1000.0, stable)
        self.char_len = [char_length_literal(d.mesh.connectivity, d.mesh.coords) if d.type == FEM else 0.0
                         for d in fem]
        fsm = 1.0
        for d, Lc in zip(fem, self.char_len):
            if d.type == FEM:
                fsm = min(0.4 * Lc / (d.prop.mat.E / d.prop.mat.rho) ** 0.5, fsm)
            else:  # springmass.py:38
                fsm = min(0.5 * np.sqrt(d.mass / d.spring), fsm)
        stable = min(fsm, stable)
        if mass_scaling_dt > 0.0:  # explicitloop.py:168-170
            stable = max(stable, mass_scaling_dt)
        # --- contacts (explicitloop.py:237-277; femcontact.py:155-197)
        contacts = []
        cds = [(i, d) for i, d in enumerate(domains) if d.considerContact]
        if any(d.type in (FEM, SPRINGMASS) for d in domains if d.considerContact):
            for a, (i, di) in enumerate(cds):
                for b in range(a):
                    j, dj = cds[b]
                    ct = di.type | dj.type
                    if di.category_bits & dj.collide_bits == 0 or di.collide_bits & dj.category_bits == 0:
                        continue
                    if ct in (RIGIDRIGID, RIGIDANLAYTICAL, ANALYTICALANALYTICAL):
                        continue
                    if ct in (ANALYTICALSPRING, SPRINGHEIGHTFIELD):  # femcontact.py:251-280
                        spr, gnd = (di, dj) if di.type == SPRINGMASS else (dj, di)
                        pen = spr.spring * 100.0
                        contacts.append((FLEXANLAYTICAL if ct == ANALYTICALSPRING else FEXHEIGHTFIELD, spr, gnd, pen,
                                         0.5 * (spr.mass / pen) ** 0.5))
                        continue
                    if ct == FLEXSPRING:  # femcontact.py:207-220: never executed (unbatched), bounds dt
                        spr, fd = (di, dj) if di.type == SPRINGMASS else (dj, di)
                        pen = min(spr.spring, self._seg_penalty(fd)) * 100.0
                        contacts.append((FLEXSPRING, spr, fd, pen, self._contact_stable(pen, fd, fem)))
                        continue
                    if ct == 0b1100:  # ContactSpringRigid (femcontact.py:243-253): every spring node an item
                        spr, rig = (di, dj) if di.type == SPRINGMASS else (dj, di)
                        pen = spr.spring * 100.0
                        contacts.append((FLEXRIGID, spr, rig, pen, 0.5 * (spr.mass / pen) ** 0.5))
                        continue
                    if ct == FLEXRIGID:  # ContactFlexRigid: domain1 = the FEM side
                        femd, rig = (di, dj) if di.type == FEM else (dj, di)
                        pen = self._seg_penalty(femd) * 1.0
                        contacts.append((ct, femd, rig, pen, self._contact_stable(pen, femd, fem)))
                        continue
                    if ct == FLEXFLEX:  # ContactFlexFlex(dom_i, dom_j): domain1 = i, domain2 = j
                        pen = min(self._seg_penalty(di), self._seg_penalty(dj)) * 1.0
                        st = min(self._contact_stable(pen, di, fem), self._contact_stable(pen, dj, fem))
                        contacts.append((ct, di, dj, pen, st))
                        continue
                    if ct not in (FLEXANLAYTICAL, FEXHEIGHTFIELD, FLEXVOXELMAP):
                        continue
                    femd, gnd = (di, dj) if di.type == FEM else (dj, di)
                    pen = self._seg_penalty(femd) * 1.0
                    contacts.append((ct, femd, gnd, pen, self._contact_stable(pen, femd, fem)))
        for c in contacts:
            stable = min(stable, c[4])
        self.stableTime = stable
        self.useAdapative = useAdapativeDT
        self.default_dt = dt
        self.dt = stable if useAdapativeDT else dt
        self.damping = damping
        self.contacts = contacts
        # --- packing (femspringmanager.py:706-813, 660-705)
        xs, vs, bcs, bcv, conns, types, Es, nus, rhos, sys_, Hs = [], [], [], [], [], [], [], [], [], [], []
        bn_off, bn_cnt, bnodes = [], [], []
        off = 0
        self.node_ranges = []
        spring_mass = []
        for d in fem:
            if d.type == SPRINGMASS:  # addSpringDomain (femspringmanager.py:815-870)
                nn = d.nnodes
                xs.append(np.asarray(d.coords, dtype=np.float32)[:, :2])
                v = np.zeros((nn, 2), np.float32)
                bits = np.zeros(nn, np.int64)
                vals = np.zeros((nn, 2), np.float32)
                self._conditions(d, nn, v, bits, vals)
                vs.append(v)
                bcs.append(bits)
                bcv.append(vals)
                cn = np.full((d.nelements, 3), -1, np.int64)
                cn[:, :2] = np.asarray(d.connectivity, np.int64)[:, :2] + off
                conns.append(cn)
                ne = d.nelements
                types.append(np.zeros(ne))
                Es.append(np.full(ne, float(d.spring), np.float32))
                nus.append(np.full(ne, float(d.damping), np.float32))
                ab = np.asarray(d.coords, np.float32)[d.connectivity[:, 0]] - np.asarray(d.coords, np.float32)[d.connectivity[:, 1]]
                rhos.append(np.array([np.linalg.norm(r) for r in ab], dtype=np.float32))  # rest lengths
                sys_.append(np.zeros(ne, np.float32))
                Hs.append(np.zeros(ne, np.float32))
                bn = np.arange(nn, dtype=np.int64) + off
                bn_off.append(sum(len(x) for x in bnodes))
                bn_cnt.append(len(bn))
                bnodes.append(bn)
                spring_mass.append((len(self.node_ranges), float(np.float32(d.mass))))
                self.node_ranges.append((off, nn))
                off += nn
                continue
            m = d.mesh
            nn = m.numNodes
            c = np.asarray(m.coords, dtype=np.float32)[:, :2]
            xs.append(c)
            v = np.zeros((nn, 2), np.float32)
            bits = np.zeros(nn, np.int64)
            vals = np.zeros((nn, 2), np.float32)
            self._conditions(d, nn, v, bits, vals)
            vs.append(v)
            bcs.append(bits)
            bcv.append(vals)
            conns.append(np.asarray(m.connectivity, np.int64)[:, :3] + off)
            ne = m.numElements
            mat = d.prop.getMaterial()
            types.append(np.full(ne, int(mat.type)))
            ey = getattr(d, "elementYoung", None)
            Es.append(np.full(ne, float(mat.E), np.float32) if ey is None else np.asarray(ey, np.float32).reshape(ne))
            nus.append(np.full(ne, float(mat.nu), np.float32))
            rhos.append(np.full(ne, float(mat.rho), np.float32))
            sys_.append(np.full(ne, float(getattr(mat, "sigma_y", 0.0)), np.float32))
            Hs.append(np.full(ne, float(getattr(mat, "H", 0.0)), np.float32))
            bn = boundary_nodes_literal(m.connectivity) + off
            bn_off.append(sum(len(x) for x in bnodes))
            bn_cnt.append(len(bn))
            bnodes.append(bn)
            self.node_ranges.append((off, nn))
            off += nn
        self.N = off
        self.E = sum(len(t) for t in types)
        cat = np.concatenate
        self._keep = [_fp(cat(xs)), _fp(cat(vs)), _ip(cat(bcs)), _fp(cat(bcv)), _ip(cat(conns)), _ip(cat(types)),
                      _fp(cat(Es)), _fp(cat(nus)), _fp(cat(rhos)), _fp(cat(sys_)), _fp(cat(Hs)), _ip(bn_off),
                      _ip(bn_cnt), _ip(cat(bnodes))]
        k = self._keep
        self._w = L.or_create(self.N, k[0][1], k[1][1], k[2][1], k[3][1], self.E, k[4][1], k[5][1], k[6][1],
                              k[7][1], k[8][1], k[9][1], k[10][1], len(fem), k[11][1], k[12][1], len(k[13][0]),
                              k[13][1])
        L.or_set_threads(self._w, int(threads))
        for body, mass in spring_mass:
            L.or_set_spring_mass(self._w, body, mass)
        # --- work lists in launch order (mixedcontact.py:1794-2261)
        anal = [c for c in contacts if c[0] == FLEXANLAYTICAL]
        hf = [c for c in contacts if c[0] == FEXHEIGHTFIELD]
        vox = [c for c in contacts if c[0] == FLEXVOXELMAP]
        flex = [c for c in contacts if c[0] == FLEXFLEX]
        unbatched = sum(1 for c in contacts if c[0] == FLEXSPRING)
        if len({id(c[2]) for c in hf}) > 1:
            unbatched += len(hf)
            hf = []
        if len({id(c[2]) for c in vox}) > 1:
            unbatched += len(vox)
            vox = []
        # a ground plane with BCs: the rigid manager moves its analytical entries
        # (planes, height fields, voxel grids, in domain order), and every
        # ground pair is gated by its entry's current box (rigidmanager.py:
        # 2486-2517, 2580-2586, 950-964); the contact keeps the first plane
        rigid_doms = [d for d in domains if d.type == RIGID]
        grounds = [d for d in domains if d.type in (ANALYTICAL, HEIGHTFIELD, VOXELMAP)]
        self.moving = any(d.type == ANALYTICAL and len(d.bcs) > 0 for d in domains)
        if self.moving and rigid_doms:
            raise NotImplementedError("a moving ground plane together with rigid bodies")
        entries = rigid_doms + (grounds if self.moving else [])
        for ct, femd, g, pen, _ in anal + hf + vox:
            body = fem.index(femd)
            lo, hi = self._ground_box(g)
            pen32 = float(np.float32(pen))
            if ct == FLEXANLAYTICAL:
                pt = np.asarray(g.point, np.float32)
                nm = np.asarray(g.normal, np.float32)
                L.or_add_plane(self._w, body, pen32, lo[1], hi[1], float(pt[0]), float(pt[1]), float(nm[0]),
                               float(nm[1]))
            elif ct == FEXHEIGHTFIELD:
                h = _fp(g.height)
                L.or_add_heightfield(self._w, body, pen32, lo[1], hi[1], len(h[0]), h[1], float(g.lb[0]),
                                     float(g.ub[0]), 1 if g.reverse else 0)
            else:
                occ = _ip(np.asarray(g.occ, np.int32))
                L.or_add_voxel(self._w, body, pen32, lo[1], hi[1], int(g.nx), int(g.ny), occ[1], float(g.lb[0]),
                               float(g.lb[1]), float(np.float32(g.dx)), float(np.float32(g.dz)))
            if self.moving:
                L.or_gate_by_rigid(self._w, entries.index(g))
        self.flex = flex
        # explicitloop.py:222-228, 362-373: no broad phase with <= 1 contact
        # domain; it is skipped without ground contact and with <= 1 contact rigid
        rigid_needs_bvh = sum(1 for d in rigid_doms if d.considerContact) > 1
        no_bvh = len(cds) <= 1
        skip_bvh = 1 if (no_bvh or ((len(anal) + len(hf) + len(vox) + unbatched) == 0 and not rigid_needs_bvh)) else 0
        self.rigids = rigid_doms
        self.entries = entries
        self.rigid_update_times = 0
        if entries:
            prm = np.zeros((len(entries), 20), np.float32)
            ivs = np.zeros((len(entries), 3), np.int32)
            for a, d in enumerate(entries):
                if d.type == RIGID:
                    self._pack_rigid(d, prm[a], ivs[a])
                else:
                    self._pack_analytical(d, prm[a], ivs[a])
            gb = []
            for g in domains:  # plane (kind 0): point, normal; height field / voxel (kind 1): its box
                if g.type == ANALYTICAL:
                    gb.append([0.0, *np.asarray(g.point, np.float32)[:2], *np.asarray(g.normal, np.float32)[:2]])
                elif g.type in (HEIGHTFIELD, VOXELMAP):
                    gb.append([1.0, *self._ground_box(g)[0][0], *self._ground_box(g)[1][0]])
            gbox = _fp(np.asarray(gb, np.float32).reshape(-1, 5))
            rp, ri = _fp(prm), _ip(ivs)
            self._keep += [rp, ri, gbox]
            L.or_set_rigids(self._w, len(entries), rp[1], ri[1], len(gb), gbox[1])
            # _parse_tie_entry / _is_tie_pair (explicitloop.py:400-439)
            tie_set = set()
            for t in (ties or []):
                if isinstance(t, (tuple, list)) and len(t) == 2 and all(isinstance(v, (int, np.integer)) for v in t):
                    a, b = (int(v) + (len(domains) if v < 0 else 0) for v in t)
                    if 0 <= a < len(domains) and 0 <= b < len(domains) and a != b:
                        tie_set.add((min(a, b), max(a, b)))
            dom_index = lambda d: next(k for k, e in enumerate(domains) if e is d)  # noqa: E731
            for ct, femd, rig, pen, _ in contacts:
                if ct == FLEXRIGID:
                    ij = tuple(sorted((dom_index(femd), dom_index(rig))))
                    L.or_add_rigid_pair(self._w, fem.index(femd), rigid_doms.index(rig), float(np.float32(pen)),
                                        float(np.float32(rig.friction)), skip_bvh, 1 if ij in tie_set else 0)
        if flex:
            # boundary edges per fem domain, global node ids, mesh order
            edges, be_off, be_cnt = [], [], []
            for d, (n0, _) in zip(fem, self.node_ranges):
                e = (boundary_edges_literal(d.mesh.connectivity) + n0 if d.type == FEM
                     else np.zeros((0, 2), np.int64))
                be_off.append(sum(len(x) for x in edges))
                be_cnt.append(len(e))
                edges.append(e)
            dom_obj = [1 if d.considerContact else 0 for d in domains]
            # bodies by index, rigids as -2 - rigid index (their boxes move), grounds -1
            in_entries = lambda d: any(d is e for e in entries)  # noqa: E731
            dom_body = [fem.index(d) if d.type in (FEM, SPRINGMASS) else
                        (-2 - next(k for k, e in enumerate(entries) if e is d) if in_entries(d) else -1)
                        for d in domains]
            dom_box = np.zeros((len(domains), 4), np.float32)
            for i, d in enumerate(domains):
                if d.type not in (FEM, SPRINGMASS) and not in_entries(d) and d.considerContact:
                    lo, hi = self._ground_box(d)
                    dom_box[i, :2] = lo[0]
                    dom_box[i, 2:] = hi[0]
            ea, eo, ec = _ip(np.concatenate(edges).reshape(-1)), _ip(be_off), _ip(be_cnt)
            do, db, dbx = _ip(dom_obj), _ip(dom_body), _fp(dom_box)
            self._keep += [ea, eo, ec, do, db, dbx]
            L.or_set_flex(self._w, len(ea[0]) // 2, ea[1], eo[1], ec[1], len(domains), do[1], db[1], dbx[1], skip_bvh)
            # _parse_tie_entry / _is_tie_pair (explicitloop.py:400-439): integer domain pairs
            flex_ties = set()
            for t in (ties or []):
                if isinstance(t, (tuple, list)) and len(t) == 2 and all(isinstance(v, (int, np.integer)) for v in t):
                    a, b = (int(v) + (len(domains) if v < 0 else 0) for v in t)
                    if 0 <= a < len(domains) and 0 <= b < len(domains) and a != b:
                        flex_ties.add((min(a, b), max(a, b)))
            gidx = lambda d: next(k for k, e in enumerate(domains) if e is d)  # noqa: E731
            for _, d1, d2, pen, _ in flex:
                fric = max(d1.friction, d2.friction)
                p = L.or_add_flex_pair(self._w, fem.index(d1), fem.index(d2), float(np.float32(pen)),
                                       float(np.float32(fric)))
                if tuple(sorted((gidx(d1), gidx(d2)))) in flex_ties:
                    L.or_set_flex_pair_tied(self._w, p, 1)
        self.sh_elapsed = 0.0
        self.counter = 0
        # setGlobalAABB -> substep(0.0, 0.0) (femspringmanager.py:872-879)
        L.or_step(self._w, 0.0, 0.0, 0, 1)
        if mass_scaling_dt > 0.0:  # applyMassScaling right after setGlobalAABB
            L.or_mass_scaling(self._w, float(np.float32(mass_scaling_dt)))
        if flex:  # explicitloop.py:383-385: initial FEM spatial hash
            L.or_flex_rebuild(self._w)

    @staticmethod
    def _conditions(d, nn, v, bits, vals):
        """processConditions (femspringmanager.py:660-705) and initial velocities
        (initialconditions.py:31-50) of one body, loop for loop."""
        for bc in d.bcs:
            t, nodes, values = bc.processData()
            if values is None:
                values = [0.0] * d.d
            if nodes is None:
                nodes = range(nn)
            for idx in nodes:
                nd = int(idx)
                bits[nd] |= int(t)
                vals[nd, 0] = float(values[0])
                vals[nd, 1] = float(values[1])
        for ic in d.initials:
            vx, vy = float(ic.vel[0]), float(ic.vel[1])
            if getattr(ic, "is_all_nodes", False):
                v[:, 0] = vx
                v[:, 1] = vy
            else:
                for nid in np.asarray(ic.nds):
                    v[int(nid)] = (vx, vy)

    def _pack_analytical(self, g, f, iv):
        """A ground's rigid-manager entry: processDomains_ (rigidmanager.py:
        2486-2517: mass 1e10, a plane's point and normal in rigidParams),
        GroundDomain.attach's initial velocity, then _addBcValue per BC; its
        first broad-phase box is its getBBox()."""
        if g.type == ANALYTICAL:
            f[0], f[1] = float(np.float32(g.point[0])), float(np.float32(g.point[1]))
            f[2], f[3] = float(np.float32(g.normal[0])), float(np.float32(g.normal[1]))
        f[6] = 1e10
        for ic in g.initials:
            a = np.asarray(ic.vel, np.float32).reshape(-1)
            f[8], f[9] = float(a[0]), float(a[1]) if a.size > 1 else 0.0
        lo, hi = self._ground_box(g)
        f[16], f[17] = lo[0]
        f[18], f[19] = hi[0]
        self._bc_bits(g.bcs, f, iv)
        iv[0], iv[2] = 64, 1 if g.considerContact else 0

    @staticmethod
    def _bc_bits(bcs, f, iv):
        """_addBcValue (rigidmanager.py:2527-2553) for each BC, in order."""
        def first(v):
            if hasattr(v, "__len__") and not isinstance(v, (str, bytes)):
                return float(np.asarray(v, dtype=np.float32).reshape(-1)[0])
            return float(v)

        def vec2(v):
            a = np.asarray(v, dtype=np.float32).reshape(-1)
            return (float(a[0]), float(a[1]) if a.size > 1 else 0.0)

        bits = 0
        for bc in bcs:
            t, _, value = bc.processData()
            bits |= int(t)
            if t == 0b1:  # UTYPE
                f[11], f[12] = 0.0, 0.0
                f[6] = 1e10
            elif t == 0b100000:  # RTYPE
                f[11], f[12] = 0.0, 0.0
                f[6] = 1e10
                f[7] = 1e10
                f[15] = 0.0
            elif t == 0b10:  # VTYPE
                f[11], f[12] = vec2(value)
                f[6] = 1e10
            elif t == 0b1000000:  # ROTVTYPE
                f[15] = first(value)
                f[7] = 1e10
            elif t in (0b10000000, 0b100000000):  # ROTATYPE, TORQUETYPE
                f[15] = first(value)
            elif t == 0b10000:  # GRAVITY
                f[13], f[14] = vec2(value)
            else:
                f[11], f[12] = vec2(value)
        iv[1] = bits

    @staticmethod
    def _pack_rigid(d, f, iv):
        """One rigid, in the reference's order: attach's initial conditions
        (rigiddomain.py:118-124), packRigidParams (rigidmanager.py:2250-2400),
        then each BC through _addBcValue (2527-2553)."""
        def first(v):
            if hasattr(v, "__len__") and not isinstance(v, (str, bytes)):
                return float(np.asarray(v, dtype=np.float32).reshape(-1)[0])
            return float(v)

        def vec2(v):
            a = np.asarray(v, dtype=np.float32).reshape(-1)
            return (float(a[0]), float(a[1]) if a.size > 1 else 0.0)

        r = d.rigid
        for ic in d.initials:
            if ic.type in (0b10, 0b100):  # VTYPE, ATYPE: V[offset]
                f[8], f[9] = vec2(ic.vel)
            else:  # RotV[offset]
                f[10] = first(ic.ang_vel)
        ref = r.getRefPoint()
        f[0], f[1] = vec2(ref)
        f[6] = first(r.mass)
        if r.rtype == 0b1:  # BALL
            f[4] = first(r.getRadius())
        elif r.rtype == 0b10:  # BOX
            f[2], f[3] = vec2(r.getPrimary())
        elif r.rtype == 0b1000:  # CAPSULE
            f[2], f[3] = vec2(r.getPrimary() - ref)
            f[4] = first(r.getRadius())
        f[5] = first(r.angle)
        f[7] = first(r.inertia_body)
        OracleLoop._bc_bits(d.bcs, f, iv)
        iv[0], iv[2] = int(r.rtype), 1 if d.considerContact else 0

    @staticmethod
    def _seg_penalty(dom):
        """femcontact.py:100-119, 2D: 2 K."""
        mat = dom.prop.mat
        nu = min(mat.nu, 0.4999)
        K = mat.E / (3.0 * (1.0 - 2.0 * nu))
        return 2.0 * 1.0 * K

    def _contact_stable(self, pen, dom, fem):
        """femcontact.py:121-141"""
        mat = dom.prop.mat
        Lc = self.char_len[fem.index(dom)]
        m_node = mat.rho * (Lc * Lc * 0.5) / 3.0
        return 0.9 * (m_node / pen) ** 0.5

    @staticmethod
    def _ground_box(g):
        if g.type == ANALYTICAL:
            n = np.asarray(g.normal, np.float32)
            p = np.asarray(g.point, np.float32)
            t = np.array([-n[1], n[0]], dtype=np.float32)
            lo_raw = p - t * 10000.0 - n * 0.1
            hi_raw = p + t * 10000.0 + n * 0.1
            lo, hi = np.minimum(lo_raw, hi_raw), np.maximum(lo_raw, hi_raw)
        elif g.type == HEIGHTFIELD:
            h = np.asarray(g.height, np.float32)
            lo = np.array([g.lb[0], float(np.min(h)) - 0.1], dtype=np.float32)
            hi = np.array([g.ub[0], float(np.max(h)) + 0.1], dtype=np.float32)
        else:
            lo, hi = np.asarray(g.lb, np.float32), np.asarray(g.ub, np.float32)
        return _fp(lo), _fp(hi)

    def close(self):
        if getattr(self, "_w", None):
            self._L.or_destroy(self._w)
            self._w = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def advance(self, n: int = 1, dt: float | None = None):
        d = self.dt if dt is None else dt
        for _ in range(n):
            if self.flex:
                # maybe_rebuild_fem_spatial_hash(self.dt) (femspringmanager.py:1035-1039), called
                # while untied items remain or the ties are not yet initialised (mixedcontact.py:1667-1678)
                cnt = np.zeros(3, np.int32)
                self._L.or_flex_counts(self._w, cnt.ctypes.data_as(_i32p))
                if cnt[1] < cnt[0] or (cnt[1] > 0 and not cnt[2]):
                    self.sh_elapsed += d
                    if self.sh_elapsed >= 1.0 / 500.0:
                        self._L.or_flex_rebuild(self._w)
                        self.sh_elapsed = 0.0
            self._L.or_step(self._w, float(np.float32(d)), float(np.float32(self.damping)), self.counter, 0)
            self.counter += 1
            if self.entries:  # explicitloop.py:533-538
                every = max(1, 1.0e-3 // d)
                self.rigid_update_times += 1
                if self.rigid_update_times % every == 0:
                    self._L.or_rigid_update(self._w, float(np.float32(every * d)), float(np.float32(self.damping)))

    def flex_grid(self):
        """The hash grid: tc, nx, ny, origin x, origin y, cell x, cell y, estimate."""
        out = np.zeros(8)
        self._L.or_get_flex_grid(self._w, out.ctypes.data_as(_f64p))
        return out

    def flex_cache(self):
        """The work items' element caches (edge index, or -1)."""
        n = sum(sum(len(boundary_nodes_literal(d.mesh.connectivity)) for d in (c[1], c[2])) for c in self.flex)
        out = np.zeros(n, np.int32)
        self._L.or_get_flex_cache(self._w, out.ctypes.data_as(_i32p))
        return out

    def advance_with_time(self, frame_dt=1.0 / 60.0):
        remaining = float(frame_dt)
        while remaining > 1e-12:
            cur = self.stableTime if self.useAdapative else self.default_dt
            sub = max(min(cur, remaining), 1e-8)
            self.dt = sub
            self.advance(1)
            remaining -= sub

    def state(self):
        x = np.zeros((self.N, 2))
        v = np.zeros((self.N, 2))
        u = np.zeros((self.N, 2))
        self._L.or_get_state(self._w, x.ctypes.data_as(_f64p), v.ctypes.data_as(_f64p), u.ctypes.data_as(_f64p))
        return x, v, u

    def set_state(self, x, v):
        xa = _fp(x) if x is not None else (None, None)
        va = _fp(v) if v is not None else (None, None)
        self._L.or_set_state(self._w, xa[1], va[1])

    def adjoint(self, n: int, xbar=None, vbar=None, dt: float | None = None):
        """Reverse-mode derivative of the next n substeps (the loop advances
        over them): from the adjoints of the final positions / velocities
        (N x 2, None = 0) to dL/dx0, dL/dv0 (N x 2) and dL/dE (per element).
        The FP64 build gives the exact derivative of the FP64 trajectory."""
        d = self.dt if dt is None else dt
        xt = None if xbar is None else np.ascontiguousarray(xbar, np.float64)
        vt = None if vbar is None else np.ascontiguousarray(vbar, np.float64)
        xb = np.zeros((self.N, 2))
        vb = np.zeros((self.N, 2))
        eb = np.zeros(self.E)
        p = lambda a: None if a is None else a.ctypes.data_as(_f64p)  # noqa: E731
        rc = self._L.or_adjoint(self._w, int(n), float(np.float32(d)), float(np.float32(self.damping)),
                                self.counter, p(xt), p(vt), p(xb), p(vb), p(eb))
        if rc != 0:
            raise NotImplementedError("oracle adjoint: FEM-FEM contact, rigids and springs are not covered")
        self.counter += int(n)
        return xb, vb, eb

    def set_young64(self, young):
        """Per-element Young's modulus in FP64 (no float32 rounding)."""
        y = np.ascontiguousarray(young, np.float64)
        self._L.or_set_young64(self._w, y.ctypes.data_as(_f64p))

    def set_state64(self, x=None, v=None):
        xa = None if x is None else np.ascontiguousarray(x, np.float64)
        va = None if v is None else np.ascontiguousarray(v, np.float64)
        self._L.or_set_state64(self._w, None if xa is None else xa.ctypes.data_as(_f64p),
                               None if va is None else va.ctypes.data_as(_f64p))

    def prepared(self):
        m = np.zeros(self.N)
        a = np.zeros(self.E)
        j = np.zeros((self.E, 4))
        self._L.or_get_prepared(self._w, m.ctypes.data_as(_f64p), a.ctypes.data_as(_f64p), j.ctypes.data_as(_f64p))
        return m, a, j

    def plastic(self):
        ep = np.zeros((self.E, 3))
        eq = np.zeros(self.E)
        self._L.or_get_plastic(self._w, ep.ctypes.data_as(_f64p), eq.ctypes.data_as(_f64p))
        return ep, eq

    def rigid_state(self):
        """(float64[n, 12] per rigid: center, angle, V, angular velocity, U,
        box lb, ub; error flag)."""
        st, err = self.entry_state()
        return st[:len(self.rigids)], err

    def entry_state(self):
        """The same for every rigid-manager entry (rigids, then the analytical
        entries of a loop with a moving plane)."""
        out = np.zeros((max(len(self.entries), 1), 12))
        err = self._L.or_get_rigids(self._w, out.ctypes.data_as(_f64p))
        return out[:len(self.entries)], err

    def aabb(self):
        out = np.zeros((len(self.fem), 4))
        self._L.or_get_aabb(self._w, out.ctypes.data_as(_f64p))
        return out
