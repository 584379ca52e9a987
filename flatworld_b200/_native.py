"""ctypes binding of libfwb200.so (include/fwb200.h).

There is no CPU fallback: if the library is missing or no CUDA device is
visible, constructing a ``NativeWorld`` raises ``RuntimeError``.
"""

from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

from . import build as _build

FW_FIELD_X = 0
FW_FIELD_V = 1
FW_FIELD_MASS = 2
FW_FIELD_X0 = 3

FW_PATH_AUTO = 0
FW_PATH_GATHER = 1
FW_PATH_RESIDENT = 2
FW_PATH_STREAM = 3
PATHS = {"auto": FW_PATH_AUTO, "gather": FW_PATH_GATHER, "resident": FW_PATH_RESIDENT, "stream": FW_PATH_STREAM}
FW_OPT_FRONT_WARPS = 1
FW_OPT_BLOCK_ELEMS = 2
FW_OPT_BLOCK_NODES = 3
FW_OPT_GRID_ELEMS = 4
FW_OPT_RES_SYNC = 5
FW_OPT_WAIT_LIMIT = 6
FW_OPT_TEST_WITHHOLD = 7
FW_OPT_STREAM_PATCH = 8
FW_OPT_STREAM_MINB = 9
FW_OPT_STREAM_BULK = 10
FW_OPT_RES_THREADS = 11
FW_PACK_PINNED = 1

_lock = threading.Lock()
_lib = None

_f32p = C.POINTER(C.c_float)
_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)
_vp = C.c_void_p

_SIGNATURES = {
    "fw_create": (C.c_int, [C.POINTER(_vp), C.c_int]),
    "fw_destroy": (None, [_vp]),
    "fw_last_error": (C.c_char_p, [_vp]),
    "fw_set_stream": (C.c_int, [_vp, _vp]),
    "fw_set_nodes": (C.c_int, [_vp, C.c_int32, _f32p, _f32p, _i32p, _f32p]),
    "fw_set_elements": (C.c_int, [_vp, C.c_int32, _i32p, _i32p, _f32p, _f32p, _f32p, _f32p, _f32p]),
    "fw_set_bodies": (C.c_int, [_vp, C.c_int32, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p, C.c_int32, _i32p]),
    "fw_set_scenes": (C.c_int, [_vp, C.c_int32, _f32p]),
    "fw_add_plane_pair": (C.c_int, [_vp, C.c_int32, C.c_float, _f32p, _f32p, C.c_float, C.c_float, C.c_float, C.c_float]),
    "fw_add_heightfield_pair": (C.c_int, [_vp, C.c_int32, C.c_float, _f32p, _f32p, C.c_int32, _f32p, C.c_float, C.c_float, C.c_int32]),
    "fw_add_voxel_pair": (C.c_int, [_vp, C.c_int32, C.c_float, _f32p, _f32p, C.c_int32, C.c_int32, _i32p, C.c_float, C.c_float, C.c_float, C.c_float]),
    "fw_set_boundary_edges": (C.c_int, [_vp, C.c_int32, _i32p, _i32p, _i32p]),
    "fw_set_flex_scene": (C.c_int, [_vp, C.c_int32, C.c_int32, C.c_int32, _i32p, _i32p, _f32p]),
    "fw_add_flex_pair": (C.c_int, [_vp, C.c_int32, C.c_int32, C.c_float, C.c_float]),
    "fw_tie_flex_pair": (C.c_int, [_vp, C.c_int32]),
    "fw_set_damping": (C.c_int, [_vp, C.c_int32, C.c_float]),
    "fw_set_flex_clock": (C.c_int, [_vp, C.c_double]),
    "fw_set_flex_clocks": (C.c_int, [_vp, C.POINTER(C.c_double)]),
    "fw_mass_scaling": (C.c_int, [_vp, C.c_float]),
    "fw_set_spring_bodies": (C.c_int, [_vp, C.c_int32, _i32p, _f32p]),
    "fw_read_flex_state": (C.c_int, [_vp, _i32p, C.c_int32, _f32p]),
    "fw_set_rigids": (C.c_int, [_vp, C.c_int32, _f32p, _i32p, C.c_int32, _f32p]),
    "fw_add_rigid_pair": (C.c_int, [_vp, C.c_int32, C.c_int32, C.c_float, C.c_float, C.c_int32, C.c_int32]),
    "fw_set_rigid_clock": (C.c_int, [_vp, C.c_int32, C.c_float, C.c_float]),
    "fw_set_rigid_clocks": (C.c_int, [_vp, _i32p, _f32p, _f32p]),
    "fw_gate_by_rigid": (C.c_int, [_vp, C.c_int32]),
    "fw_read_rigids": (C.c_int, [_vp, _f32p, _i32p]),
    "fw_set_path": (C.c_int, [_vp, C.c_int32, C.c_int32]),
    "fw_get_path": (C.c_int, [_vp, _i32p, _i32p]),
    "fw_set_option": (C.c_int, [_vp, C.c_int32, C.c_int32]),
    "fw_get_option": (C.c_int, [_vp, C.c_int32, _i32p]),
    "fw_snapshot": (C.c_int, [_vp, C.c_int32]),
    "fw_set_element_young": (C.c_int, [_vp, C.c_int32, C.c_int32, _vp, C.c_int32]),
    "fw_adj_begin": (C.c_int, [_vp, C.c_int32]),
    "fw_adj_seed": (C.c_int, [_vp, _vp, _vp, C.c_int32]),
    "fw_adj_segment": (C.c_int, [_vp, C.c_int32, C.c_float]),
    "fw_adj_read": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int32]),
    "fw_tan_begin": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int32]),
    "fw_tan_step": (C.c_int, [_vp, C.c_int32, C.c_float]),
    "fw_tan_read": (C.c_int, [_vp, _vp, _vp, C.c_int32]),
    "fw_arena_init": (C.c_int, [_vp, C.c_int64, C.c_int64, C.c_int32, C.c_int32, C.c_int32, C.c_int64, C.c_int64]),
    "fw_arena_commit": (C.c_int, [_vp, _i32p]),
    "fw_arena_remove": (C.c_int, [_vp, C.c_int32]),
    "fw_arena_scene_info": (C.c_int, [_vp, C.c_int32, _i64p]),
    "fw_arena_pack": (C.c_int, [_vp, C.c_int32, C.c_int32, C.POINTER(_vp)]),
    "fw_step_served_budget": (C.c_int, [_vp, _f32p, _i32p, _f32p, _i32p, C.c_int32]),
    "fw_create_stage": (C.c_int, [C.POINTER(_vp)]),
    "fw_arena_commit_pack": (C.c_int, [_vp, _vp, _i32p]),
    "fw_pack_info": (C.c_int, [_vp, _i64p]),
    "fw_pack_destroy": (None, [_vp]),
    "fw_restore": (C.c_int, [_vp, C.c_int32]),
    "fw_finalize": (C.c_int, [_vp]),
    "fw_step": (C.c_int, [_vp, C.c_int32, C.c_float]),
    "fw_step_scenes": (C.c_int, [_vp, C.c_int32, _f32p]),
    "fw_step_served": (C.c_int, [_vp, _f32p]),
    "fw_step_served_n": (C.c_int, [_vp, _f32p, C.c_int32]),
    "fw_set_active": (C.c_int, [_vp, _i32p]),
    "fw_synchronize": (C.c_int, [_vp]),
    "fw_read_nodes": (C.c_int, [_vp, C.c_int32, C.c_int32, C.c_int32, _vp, C.c_int32]),
    "fw_write_nodes": (C.c_int, [_vp, C.c_int32, C.c_int32, C.c_int32, _vp, C.c_int32]),
    "fw_read_aabb": (C.c_int, [_vp, _f32p]),
    "fw_read_plastic": (C.c_int, [_vp, _f32p, _f32p]),
    "fw_read_reference_shape": (C.c_int, [_vp, _f32p, _f32p]),
    "fw_read_counters": (C.c_int, [_vp, _i64p]),
    "fw_energy": (C.c_int, [_vp, C.POINTER(C.c_double)]),
    "fw_scene_status": (C.c_int, [_vp, _vp, C.c_int32]),
    "fw_clear_scene_status": (C.c_int, [_vp, C.c_int32]),
    "fw_set_cfl_monitor": (C.c_int, [_vp, _vp]),
    "fw_read_cfl": (C.c_int, [_vp, _vp, C.c_int32]),
    "fw_launch_count": (C.c_int64, [_vp]),
    "fw_build_info": (C.c_char_p, []),
    "fw_step_noalloc": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_float, C.c_float, _vp, _vp, _vp, _vp, _vp,
                                  _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, C.c_char_p, C.c_int32]),
}


def exported_symbols() -> list[str]:
    return list(_SIGNATURES)


def lib():
    """Load libfwb200.so (built in-tree) and declare every entry point."""
    global _lib
    with _lock:
        if _lib is None:
            path = _build.lib_path()
            if not os.path.exists(path):
                raise RuntimeError(
                    f"{path} is not built; run `python -m flatworld_b200.build` "
                    "(or __graft_entry__.build()) -- there is no CPU fallback")
            handle = C.CDLL(path)
            for name, (res, args) in _SIGNATURES.items():
                fn = getattr(handle, name)
                fn.restype = res
                fn.argtypes = args
            _lib = handle
        return _lib


class ScenePack:
    """A scene prepared for an arena (fw_arena_pack); freed by close() -- no
    commit from it may still be in flight then."""

    def __init__(self, L, handle):
        self._L = L
        self.handle = handle
        info = np.zeros(8, dtype=np.int64)
        L.fw_pack_info(handle, info.ctypes.data_as(_i64p))
        self.device_bytes = int(info[0])
        self.nodes, self.elems, self.bodies = int(info[1]), int(info[2]), int(info[3])
        self.patch_nodes, self.patches, self.patch_elems = int(info[4]), int(info[5]), int(info[6])
        self.pinned = bool(info[7])

    def close(self):
        if self.handle:
            self._L.fw_pack_destroy(self.handle)
            self.handle = None


def _f(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(_f32p)


def _i(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(_i32p)


class NativeError(RuntimeError):
    pass


class NativeWorld:
    """Owner of one fw_ctx (device buffers of a packed world)."""

    def __init__(self, device: int = 0):
        self._L = lib()
        h = _vp()
        rc = self._L.fw_create(C.byref(h), int(device))
        if rc != 0:
            raise NativeError(
                f"fw_create(device={device}) failed with code {rc}: no usable CUDA device "
                "(flatworld_b200 runs on the GPU only)")
        self._h = h
        self.device = device

    @classmethod
    def stage(cls) -> "NativeWorld":
        """A staging context (fw_create_stage): stages one scene at a time
        for arena_pack, touches no device (works without a GPU)."""
        w = cls.__new__(cls)
        w._L = lib()
        h = _vp()
        rc = w._L.fw_create_stage(C.byref(h))
        if rc != 0:
            raise NativeError(f"fw_create_stage failed with code {rc}")
        w._h = h
        w.device = -1
        return w

    def _check(self, rc: int, what: str):
        if rc != 0:
            msg = self._L.fw_last_error(self._h)
            raise NativeError(f"{what}: {msg.decode() if msg else ''} (code {rc})")

    def close(self):
        if getattr(self, "_h", None):
            self._L.fw_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> int:
        return self._h.value

    # ---- construction
    def set_nodes(self, coords, vel, bc_bits, bc_values):
        n = len(coords)
        keep = [_f(coords), _f(vel), _i(bc_bits), _f(bc_values)]
        self._check(self._L.fw_set_nodes(self._h, n, keep[0][1], keep[1][1], keep[2][1], keep[3][1]), "fw_set_nodes")

    def set_elements(self, conn, mtype, E, nu, rho, sy, H):
        k = [_i(conn), _i(mtype), _f(E), _f(nu), _f(rho), _f(sy), _f(H)]
        self._check(self._L.fw_set_elements(self._h, len(mtype), *[x[1] for x in k]), "fw_set_elements")

    def set_bodies(self, noff, ncnt, eoff, ecnt, scene, bnoff, bncnt, bnodes):
        k = [_i(noff), _i(ncnt), _i(eoff), _i(ecnt), _i(scene), _i(bnoff), _i(bncnt)]
        bn = _i(bnodes)
        self._check(self._L.fw_set_bodies(self._h, len(noff), *[x[1] for x in k], len(bn[0]), bn[1]), "fw_set_bodies")

    def set_scenes(self, damping):
        d = _f(damping)
        self._check(self._L.fw_set_scenes(self._h, len(d[0]), d[1]), "fw_set_scenes")

    def add_plane(self, body, penalty, lo, hi, p, n):
        lo, hi = _f(lo), _f(hi)
        self._check(self._L.fw_add_plane_pair(self._h, body, penalty, lo[1], hi[1], float(p[0]), float(p[1]),
                                              float(n[0]), float(n[1])), "fw_add_plane_pair")

    def add_heightfield(self, body, penalty, lo, hi, heights, lbx, ubx, reverse):
        lo, hi, h = _f(lo), _f(hi), _f(heights)
        self._check(self._L.fw_add_heightfield_pair(self._h, body, penalty, lo[1], hi[1], len(h[0]), h[1],
                                                    float(lbx), float(ubx), int(reverse)), "fw_add_heightfield_pair")

    def add_voxel(self, body, penalty, lo, hi, occ, lbx, lby, dx, dz):
        lo, hi = _f(lo), _f(hi)
        o = _i(occ)
        nx, ny = occ.shape
        self._check(self._L.fw_add_voxel_pair(self._h, body, penalty, lo[1], hi[1], nx, ny, o[1], float(lbx),
                                              float(lby), float(dx), float(dz)), "fw_add_voxel_pair")

    def set_boundary_edges(self, edges, body_off, body_cnt):
        e, o, c = _i(np.asarray(edges).reshape(-1)), _i(body_off), _i(body_cnt)
        self._check(self._L.fw_set_boundary_edges(self._h, len(e[0]) // 2, e[1], o[1], c[1]), "fw_set_boundary_edges")

    def set_flex_scene(self, scene, skip_bvh, dom_obj, dom_body, dom_box):
        o, b, x = _i(dom_obj), _i(dom_body), _f(np.asarray(dom_box, np.float32).reshape(-1))
        self._check(self._L.fw_set_flex_scene(self._h, int(scene), int(skip_bvh), len(o[0]), o[1], b[1], x[1]),
                    "fw_set_flex_scene")

    def add_flex_pair(self, body1, body2, penalty, friction):
        self._check(self._L.fw_add_flex_pair(self._h, int(body1), int(body2), float(penalty), float(friction)),
                    "fw_add_flex_pair")

    def set_damping(self, scene, damping):
        self._check(self._L.fw_set_damping(self._h, int(scene), float(damping)), "fw_set_damping")

    def tie_flex_pair(self, pair):
        self._check(self._L.fw_tie_flex_pair(self._h, int(pair)), "fw_tie_flex_pair")

    def read_flex_state(self, n_items: int):
        """(work-item edge caches int32[n_items], hash grid float32[8])."""
        cache = np.zeros(max(n_items, 1), np.int32)
        grid = np.zeros(8, np.float32)
        self._check(self._L.fw_read_flex_state(self._h, cache.ctypes.data_as(_i32p), int(n_items),
                                               grid.ctypes.data_as(_f32p)), "fw_read_flex_state")
        return cache[:n_items], grid

    def set_spring_bodies(self, bodies, node_mass):
        b, m = _i(bodies), _f(node_mass)
        self._check(self._L.fw_set_spring_bodies(self._h, len(b[0]), b[1], m[1]), "fw_set_spring_bodies")

    def set_rigids(self, params, ints, grounds):
        """params float32[n, 20], ints int32[n, 4], grounds float32[g, 6]."""
        p = _f(np.asarray(params, np.float32).reshape(-1))
        i = _i(np.asarray(ints, np.int32).reshape(-1))
        g = _f(np.asarray(grounds, np.float32).reshape(-1))
        self._check(self._L.fw_set_rigids(self._h, len(i[0]) // 4, p[1], i[1], len(g[0]) // 6, g[1]),
                    "fw_set_rigids")

    def add_rigid_pair(self, body, rigid, penalty, friction, skip_bvh, tied=0):
        self._check(self._L.fw_add_rigid_pair(self._h, int(body), int(rigid), float(penalty), float(friction),
                                              int(skip_bvh), int(tied)), "fw_add_rigid_pair")

    def set_rigid_clock(self, every: int, dt: float, damping: float):
        self._check(self._L.fw_set_rigid_clock(self._h, int(every), float(dt), float(damping)), "fw_set_rigid_clock")

    def gate_by_rigid(self, entry: int):
        self._check(self._L.fw_gate_by_rigid(self._h, int(entry)), "fw_gate_by_rigid")

    def set_rigid_clocks(self, every, dt, damping):
        """Per scene: update interval, rigid dt and damping."""
        e, t, m = _i(every), _f(dt), _f(damping)
        self._check(self._L.fw_set_rigid_clocks(self._h, e[1], t[1], m[1]), "fw_set_rigid_clocks")

    def read_rigids(self, n: int):
        """(float32[n, 12] per rigid: center, angle, V, angular velocity, U, box lb, ub; flags)."""
        out = np.zeros((max(n, 1), 12), np.float32)
        flags = np.zeros(1, np.int32)
        self._check(self._L.fw_read_rigids(self._h, out.ctypes.data_as(_f32p), flags.ctypes.data_as(_i32p)),
                    "fw_read_rigids")
        return out[:n], int(flags[0])

    def mass_scaling(self, dt_target: float):
        self._check(self._L.fw_mass_scaling(self._h, float(dt_target)), "fw_mass_scaling")

    def set_flex_clocks(self, dt):
        """Per scene: the substep dt in float64 (FEM-FEM hash clock)."""
        a = np.ascontiguousarray(dt, dtype=np.float64)
        self._check(self._L.fw_set_flex_clocks(self._h, a.ctypes.data_as(C.POINTER(C.c_double))),
                    "fw_set_flex_clocks")

    def set_flex_clock(self, dt: float):
        self._check(self._L.fw_set_flex_clock(self._h, float(dt)), "fw_set_flex_clock")

    def set_path(self, path: int, patches: int = 0):
        self._check(self._L.fw_set_path(self._h, int(path), int(patches)), "fw_set_path")

    def set_option(self, option: int, value: int):
        self._check(self._L.fw_set_option(self._h, int(option), int(value)), "fw_set_option")

    def get_option(self, option: int) -> int:
        v = C.c_int32(0)
        self._check(self._L.fw_get_option(self._h, int(option), C.byref(v)), "fw_get_option")
        return int(v.value)

    def snapshot(self, slot: int = 0):
        self._check(self._L.fw_snapshot(self._h, int(slot)), "fw_snapshot")

    def restore(self, slot: int = 0):
        self._check(self._L.fw_restore(self._h, int(slot)), "fw_restore")

    # ---- differentiable form
    def set_element_young(self, young, first=0):
        y = np.ascontiguousarray(young, dtype=np.float32)
        self._check(self._L.fw_set_element_young(self._h, int(first), len(y), y.ctypes.data, 0),
                    "fw_set_element_young")

    def adj_begin(self, max_segment_steps):
        self._check(self._L.fw_adj_begin(self._h, int(max_segment_steps)), "fw_adj_begin")

    def adj_seed(self, xbar=None, vbar=None):
        xb = None if xbar is None else np.ascontiguousarray(xbar, dtype=np.float32)
        vb = None if vbar is None else np.ascontiguousarray(vbar, dtype=np.float32)
        self._check(self._L.fw_adj_seed(self._h, None if xb is None else xb.ctypes.data,
                                        None if vb is None else vb.ctypes.data, 0), "fw_adj_seed")

    def adj_segment(self, n, dt):
        self._check(self._L.fw_adj_segment(self._h, int(n), float(np.float32(dt))), "fw_adj_segment")

    def adj_read(self, n_nodes, n_elems):
        xb = np.empty((n_nodes, 2), np.float32)
        vb = np.empty((n_nodes, 2), np.float32)
        eb = np.empty((n_elems,), np.float32)
        self._check(self._L.fw_adj_read(self._h, xb.ctypes.data, vb.ctypes.data, eb.ctypes.data, 0), "fw_adj_read")
        return xb, vb, eb

    def tan_begin(self, dx0=None, dv0=None, dE=None):
        arrs = [None if a is None else np.ascontiguousarray(a, np.float32) for a in (dx0, dv0, dE)]
        ptrs = [None if a is None else a.ctypes.data for a in arrs]
        self._check(self._L.fw_tan_begin(self._h, ptrs[0], ptrs[1], ptrs[2], 0), "fw_tan_begin")

    def tan_step(self, n_steps, dt):
        self._check(self._L.fw_tan_step(self._h, int(n_steps), float(dt)), "fw_tan_step")

    def tan_read(self, n_nodes):
        dx = np.empty((n_nodes, 2), np.float32)
        dv = np.empty((n_nodes, 2), np.float32)
        self._check(self._L.fw_tan_read(self._h, dx.ctypes.data, dv.ctypes.data, 0), "fw_tan_read")
        return dx, dv

    # ---- arena (served form)
    def arena_init(self, max_nodes, max_elems, max_bodies, max_scenes, max_pairs, max_heights, max_occ):
        self._check(self._L.fw_arena_init(self._h, int(max_nodes), int(max_elems), int(max_bodies),
                                          int(max_scenes), int(max_pairs), int(max_heights), int(max_occ)),
                    "fw_arena_init")

    def arena_commit(self) -> int:
        s = C.c_int32()
        self._check(self._L.fw_arena_commit(self._h, C.byref(s)), "fw_arena_commit")
        return int(s.value)

    def arena_remove(self, scene: int):
        self._check(self._L.fw_arena_remove(self._h, int(scene)), "fw_arena_remove")

    def arena_pack(self, patch_nodes: int, pinned: bool = False) -> "ScenePack":
        """The scene staged on this (never finalized) context as a pack for
        an arena with ``patch_nodes``-node stream patches (0: gather arena).
        Host work only; the stage is cleared."""
        h = _vp()
        self._check(self._L.fw_arena_pack(self._h, int(patch_nodes), FW_PACK_PINNED if pinned else 0, C.byref(h)),
                    "fw_arena_pack")
        return ScenePack(self._L, h)

    def arena_commit_pack(self, pack: "ScenePack") -> int:
        s = C.c_int32()
        self._check(self._L.fw_arena_commit_pack(self._h, pack.handle, C.byref(s)), "fw_arena_commit_pack")
        return int(s.value)

    def arena_scene_info(self, scene: int):
        out = np.zeros(8, dtype=np.int64)
        self._check(self._L.fw_arena_scene_info(self._h, int(scene), out.ctypes.data_as(_i64p)), "fw_arena_scene_info")
        return out

    def get_path(self):
        p = C.c_int32()
        n = C.c_int32()
        self._check(self._L.fw_get_path(self._h, C.byref(p), C.byref(n)), "fw_get_path")
        return int(p.value), int(n.value)

    def finalize(self):
        self._check(self._L.fw_finalize(self._h), "fw_finalize")

    # ---- stepping
    def step(self, n: int, dt: float):
        self._check(self._L.fw_step(self._h, int(n), float(np.float32(dt))), "fw_step")

    def step_scenes(self, n: int, dt_per_scene):
        d = _f(dt_per_scene)
        self._check(self._L.fw_step_scenes(self._h, int(n), d[1]), "fw_step_scenes")

    def step_served(self, dt_per_scene):
        """One substep; scenes with dt <= 0 stay frozen.  dt must be float32,
        contiguous, one entry per scene (the library copies it before returning)."""
        self._check(self._L.fw_step_served(self._h, dt_per_scene.ctypes.data_as(_f32p)), "fw_step_served")

    def step_served_n(self, dt_per_scene, n_steps: int):
        """n_steps substeps with the same per-scene dt (see step_served)."""
        self._check(self._L.fw_step_served_n(self._h, dt_per_scene.ctypes.data_as(_f32p), int(n_steps)),
                    "fw_step_served_n")

    def step_served_budget(self, dt_per_scene, budget, n_steps: int, dt_next=None, budget_next=None):
        """Stream arenas: n_steps substeps in which scene s runs only its
        first budget[s] substeps, then budget_next[s] at dt_next[s] when
        given (fw_step_served_budget)."""
        b = _i(budget)
        if dt_next is None:
            p_dt2 = p_b2 = None
        else:
            d2, p_dt2 = _f(dt_next)
            b2, p_b2 = _i(budget_next)
        self._check(self._L.fw_step_served_budget(self._h, dt_per_scene.ctypes.data_as(_f32p), b[1], p_dt2, p_b2,
                                                  int(n_steps)), "fw_step_served_budget")

    def set_active(self, active):
        a = _i(active)
        self._check(self._L.fw_set_active(self._h, a[1]), "fw_set_active")

    def synchronize(self):
        self._check(self._L.fw_synchronize(self._h), "fw_synchronize")

    # ---- readback
    def read_nodes(self, field: int, first: int, count: int) -> np.ndarray:
        width = 1 if field == FW_FIELD_MASS else 2
        out = np.empty((count, width), dtype=np.float32)
        self._check(self._L.fw_read_nodes(self._h, field, first, count, out.ctypes.data, 0), "fw_read_nodes")
        return out if width == 2 else out[:, 0]

    def read_nodes_ptr(self, field: int, first: int, count: int, dst_ptr: int, on_device: bool = False):
        """Read into caller memory (host pointer, pinned or not, or a device pointer)."""
        self._check(self._L.fw_read_nodes(self._h, field, first, count, dst_ptr, 1 if on_device else 0),
                    "fw_read_nodes")

    def write_nodes_ptr(self, field: int, first: int, count: int, src_ptr: int, on_device: bool = False):
        self._check(self._L.fw_write_nodes(self._h, field, first, count, src_ptr, 1 if on_device else 0),
                    "fw_write_nodes")

    def set_stream(self, stream_ptr: int | None):
        """Queue this world's work on a caller CUDA stream (None: own stream)."""
        self._check(self._L.fw_set_stream(self._h, stream_ptr or None), "fw_set_stream")

    def write_nodes(self, field: int, first: int, values: np.ndarray):
        v = np.ascontiguousarray(values, dtype=np.float32)
        self._check(self._L.fw_write_nodes(self._h, field, first, len(v), v.ctypes.data, 0), "fw_write_nodes")

    def read_aabb(self, n_bodies: int) -> np.ndarray:
        out = np.empty((n_bodies, 4), dtype=np.float32)
        self._check(self._L.fw_read_aabb(self._h, out.ctypes.data_as(_f32p)), "fw_read_aabb")
        return out

    def read_plastic(self, n_elems: int):
        ep = np.empty((n_elems, 3), dtype=np.float32)
        eq = np.empty((n_elems,), dtype=np.float32)
        self._check(self._L.fw_read_plastic(self._h, ep.ctypes.data_as(_f32p), eq.ctypes.data_as(_f32p)), "fw_read_plastic")
        return ep, eq

    def read_reference_shape(self, n_elems: int):
        area = np.empty((n_elems,), dtype=np.float32)
        jinv = np.empty((n_elems, 4), dtype=np.float32)
        self._check(self._L.fw_read_reference_shape(self._h, area.ctypes.data_as(_f32p), jinv.ctypes.data_as(_f32p)),
                    "fw_read_reference_shape")
        return area, jinv

    def read_counters(self, n_scenes: int) -> np.ndarray:
        out = np.empty((n_scenes,), dtype=np.int64)
        self._check(self._L.fw_read_counters(self._h, out.ctypes.data_as(_i64p)), "fw_read_counters")
        return out

    def energy(self, n_scenes: int) -> np.ndarray:
        """Per-scene energies (FP64, reduced on the device): columns kinetic,
        strain, external potential, contact penalty."""
        out = np.zeros((n_scenes, 4), dtype=np.float64)
        self._check(self._L.fw_energy(self._h, out.ctypes.data_as(C.POINTER(C.c_double))), "fw_energy")
        return out

    def scene_status(self, n_scenes: int, out=None, asynchronous=False):
        """Per-scene non-finite flags (int32).  With asynchronous=True the copy
        is only queued: pass pinned memory (e.g. a pinned torch tensor's numpy
        view) and read it after the stream has passed this point."""
        if out is None:
            out = np.zeros((n_scenes,), dtype=np.int32)
        self._check(self._L.fw_scene_status(self._h, out.ctypes.data, 1 if asynchronous else 0), "fw_scene_status")
        return out

    def set_cfl_monitor(self, coef_per_body):
        """Turn the CFL monitor on with 0.4 / sqrt(E / rho) per body (None: off)."""
        if coef_per_body is None:
            self._check(self._L.fw_set_cfl_monitor(self._h, None), "fw_set_cfl_monitor")
            return
        c = np.ascontiguousarray(coef_per_body, np.float32)
        self._check(self._L.fw_set_cfl_monitor(self._h, c.ctypes.data), "fw_set_cfl_monitor")

    def read_cfl(self, n_scenes: int, reset: bool = True):
        """Smallest current-shape stable time per scene since the last reset."""
        out = np.zeros((n_scenes,), dtype=np.float32)
        self._check(self._L.fw_read_cfl(self._h, out.ctypes.data, 1 if reset else 0), "fw_read_cfl")
        return out

    def clear_scene_status(self, scene: int = -1):
        self._check(self._L.fw_clear_scene_status(self._h, int(scene)), "fw_clear_scene_status")

    def launch_count(self) -> int:
        return int(self._L.fw_launch_count(self._h))
