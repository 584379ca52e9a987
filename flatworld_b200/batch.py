"""Batched form: many independent scenes stepped together in one world.

A *scene* is what one reference ``ExplicitLoop`` holds (FEM domains plus their
grounds).  ``BatchedLoop`` packs S scenes of uneven sizes into one ragged
node / triangle index space and advances all of them with the same two kernels
per substep (captured in CUDA graphs), instead of S separate loops.  Each
scene keeps its own time step, step counter and broad-phase gate, and scenes
never exchange forces, so every scene's result is bit-identical to stepping it
alone in its own ``ExplicitLoop`` (tests/test_batch.py checks this).

The reference cannot batch such scenes in one loop: one ExplicitLoop batches a
single height field and a single voxel grid (flatworld/mixedcontact.py:2140,
2211), so per-body voxel grids need one loop per body.
"""

from __future__ import annotations

import numpy as np

from . import _native
from .world import PackedWorld, SceneLayout, build_native, substep_schedule


class BatchedLoop:
    """Advance S independent scenes together.

    Args:
        scenes: list of domain lists (one per scene, as passed to ExplicitLoop)
        dt, useAdapativeDT, damping: as ExplicitLoop, applied to every scene
            (a sequence gives one value per scene)
        device: CUDA ordinal
        block_elems, block_nodes: launch shape of the step kernels (0: tuned
            default; see flatworld_b200.autotune)
        path: "stream" (one patch-streaming kernel per substep, the faster one
            for many small scenes) or "gather" (two kernels per substep through
            a corner buffer, launch shape tunable); both give the same bits
        stream_patch: owned nodes per patch of the stream step, 64 or 128
            (0: 64); see flatworld_b200.autotune.tune_stream_patch
    """

    def __init__(self, scenes, dt=0.0, useAdapativeDT=True, damping=0.0, device=0,
                 block_elems=0, block_nodes=0, path="stream", stream_patch=0):
        S = len(scenes)
        dts = dt if np.iterable(dt) else [dt] * S
        ada = useAdapativeDT if np.iterable(useAdapativeDT) else [useAdapativeDT] * S
        damp = damping if np.iterable(damping) else [damping] * S
        self.layouts = [SceneLayout(d, dt=a, damping=c, useAdapativeDT=b)
                        for d, a, b, c in zip(scenes, dts, ada, damp)]
        self.packed = PackedWorld(self.layouts)
        self._has_flex = any(lay.flex for lay in self.layouts)
        self._has_rigid = any(lay.entries for lay in self.layouts)
        if path == "stream" and (self.packed.spring_bodies or self._has_flex or self._has_rigid):
            path = "gather"  # the patch-streaming step covers triangles without FEM-FEM / FEM-rigid contact
        self._native = build_native(self.packed, device=device, path=path,
                                    stream_patch=stream_patch if path == "stream" else 0)
        self.path = path
        self.stream_patch = (stream_patch or 64) if path == "stream" else 0
        self.stream_minb = {64: 32, 128: 16}.get(self.stream_patch, 0)  # the built default budgets
        self.stream_bulk = False
        if block_elems or block_nodes:
            self.set_launch(block_elems, block_nodes)
        self.S = S
        self.dt = np.array([lay.dt for lay in self.layouts], dtype=np.float64)
        self.counters = np.zeros(S, dtype=np.int64)
        self._active = np.ones(S, dtype=np.int32)

    # ---- sizes
    @property
    def n_nodes(self):
        return self.packed.N

    @property
    def n_elems(self):
        return self.packed.E

    def scene_elems(self, s):
        return self.layouts[s].n_elems

    def set_launch(self, block_elems=0, block_nodes=0):
        """Change the step kernels' block sizes (cached graphs are rebuilt)."""
        if block_elems:
            self._native.set_option(_native.FW_OPT_BLOCK_ELEMS, block_elems)
        if block_nodes:
            self._native.set_option(_native.FW_OPT_BLOCK_NODES, block_nodes)

    def set_stream_shape(self, minb=0, bulk=None):
        """Stream step launch shape: the CTAs per SM its registers are budgeted
        for (``minb``; 0 keeps it) and whether a patch's triangle records are
        staged by one bulk copy (``bulk``; None keeps it).  Same bits."""
        if minb:
            self._native.set_option(_native.FW_OPT_STREAM_MINB, int(minb))
            self.stream_minb = int(minb)
        if bulk is not None:
            self._native.set_option(_native.FW_OPT_STREAM_BULK, 1 if bulk else 0)
            self.stream_bulk = bool(bulk)

    @property
    def stream_shape(self):
        """The stream step's launch shape as "patch/minb/staged|loads"."""
        return f"{self.stream_patch}/{self.stream_minb}/{'staged' if self.stream_bulk else 'loads'}"

    def set_stream(self, stream_ptr):
        self._native.set_stream(stream_ptr)

    # ---- stepping
    def _set_active(self, active):
        active = np.asarray(active, dtype=np.int32)
        if not np.array_equal(active, self._active):
            self._native.set_active(active)
            self._active = active.copy()

    def _clocks(self, dt):
        """The FEM-FEM hash clocks accumulate each scene's float64 dt
        (femspringmanager.py:1035-1039); each scene's rigids move every
        N = max(1, 1e-3 // dt) substeps by N * dt (explicitloop.py:533-538)."""
        if self._has_flex:
            self._native.set_flex_clocks(np.asarray(dt, np.float64))
        if self._has_rigid:
            every = [int(max(1, 1.0e-3 // float(t))) if t > 0 else 1 for t in dt]
            rdt = [float(np.float32(e * float(t))) for e, t in zip(every, dt)]
            damp = [float(np.float32(lay.damping)) for lay in self.layouts]
            self._native.set_rigid_clocks(np.asarray(every, np.int32), np.asarray(rdt, np.float32),
                                          np.asarray(damp, np.float32))

    def advance(self, n: int = 1):
        """n substeps of every active scene, each with its own dt."""
        self._clocks(self.dt)
        d32 = self.dt.astype(np.float32)
        if np.all(d32 == d32[0]):
            self._native.step(int(n), float(d32[0]))
        else:
            self._native.step_scenes(int(n), d32)
        self.counters += int(n) * self._active

    def advanceWithTime(self, frame_dt=1.0 / 60.0):
        """Every scene advances by frame_dt in its own substeps (the reference's
        advanceWithTime loop per scene, explicitloop.py:558-589).  Scenes with
        fewer substeps are frozen while the others finish."""
        runs = [substep_schedule(frame_dt, lay.stableTime, lay.default_dt, lay.useAdapative)
                for lay in self.layouts]
        pos = [0] * self.S      # index into each scene's run list
        left = [r[0][0] if r else 0 for r in runs]
        base_active = self._active.copy()
        while True:
            live = [s for s in range(self.S) if base_active[s] and pos[s] < len(runs[s])]
            if not live:
                break
            dts = np.zeros(self.S, dtype=np.float32)
            dts64 = np.zeros(self.S, dtype=np.float64)
            act = np.zeros(self.S, dtype=np.int32)
            for s in live:
                dts[s] = np.float32(runs[s][pos[s]][1])
                dts64[s] = runs[s][pos[s]][1]
                act[s] = 1
            n = min(left[s] for s in live)
            self._set_active(act)
            self._clocks(dts64)
            self._native.step_scenes(n, dts)
            for s in live:
                self.counters[s] += n
                left[s] -= n
                self.dt[s] = runs[s][pos[s]][1]
                if left[s] == 0:
                    pos[s] += 1
                    if pos[s] < len(runs[s]):
                        left[s] = runs[s][pos[s]][0]
        self._set_active(base_active)

    def synchronize(self):
        self._native.synchronize()

    # ---- readback
    def _node_range(self, s):
        bodies = self.packed.scene_bodies[s]
        n0 = int(self.packed.noff[bodies[0]])
        nn = int(sum(int(self.packed.ncnt[b]) for b in bodies))
        return n0, nn

    def rigid_state(self, s):
        """float32[rigids of scene s, 12]: center, angle, V, angular velocity,
        U, box (the RigidBodyDomain getters' values)."""
        n = len(self.layouts[s].rigids)
        if n == 0:
            return np.zeros((0, 12), np.float32)
        st, flags = self._native.read_rigids(sum(len(lay.entries) for lay in self.layouts))
        if flags & 1:
            raise RuntimeError("a rigid body came within 0.01 of a ground or another contact rigid, or its state "
                               "is no longer finite")
        r0 = self.packed.rigid_offsets()[s]
        return st[r0:r0 + n]

    def coords(self, s):
        n0, nn = self._node_range(s)
        return self._native.read_nodes(_native.FW_FIELD_X, n0, nn)

    def velocities(self, s):
        n0, nn = self._node_range(s)
        return self._native.read_nodes(_native.FW_FIELD_V, n0, nn)

    def all_coords(self):
        return self._native.read_nodes(_native.FW_FIELD_X, 0, self.packed.N)

    def energies(self):
        """Per-scene energies, FP64 reduced on the GPU: (n_scenes, 4) array of
        kinetic, strain, external potential, contact penalty."""
        return self._native.energy(len(self.packed.scenes))

    def enable_cfl_monitor(self, on: bool = True):
        """Per-scene stable time of the current (deformed) shapes, reduced on
        the GPU in the step (either path; see ExplicitLoop.enable_cfl_monitor).
        dt is not changed."""
        self._native.set_cfl_monitor(self.packed.cfl_coefficients() if on else None)

    def currentStableTimes(self, reset: bool = True):
        """float32[S]: each scene's smallest current-shape stable time since
        the last reset (+inf for scenes that did not step)."""
        return self._native.read_cfl(self.S, reset)

    def launch_count(self):
        return self._native.launch_count()
