"""Served form: a request loop with continuous batching.

A request asks one soft body to advance by ``advanceWithTime(frame_dt)`` in a
given number of substeps.  The ``Server`` keeps every admitted body resident in
a device arena (flatworld_b200 C ABI: fw_arena_*), so a body's state carries
over between its requests, and advances all bodies that have a request in
flight together.  The batch of every substep is exactly the set of requests in
flight: a request leaves at the substep it finishes, and requests that arrive
join at the next native call (a call runs only as many substeps as no
in-flight request finishes within and, with real-time arrivals, as fit before
the next arrival).  A new body is admitted when the arena and the HBM budget
have room for it.
Per-body results do not depend on what else is in the batch -- scenes never
exchange forces -- so every result equals the same requests run alone
(tests/test_serve.py).

``FifoPlainServer`` is the comparison: one request at a time, in arrival
order, each body in its own ExplicitLoop (the plain path).

Reference: each reference ExplicitLoop is built once and stepped by its owner
(flatworld/explicitloop.py:72-589); it has no request loop.
"""

from __future__ import annotations

import collections
import heapq
import time
from dataclasses import dataclass, field

import numpy as np

from . import _native
from .explicitloop import ExplicitLoop
from .world import PackedWorld, SceneLayout, stage, substep_schedule


def scene_device_bytes(layout: SceneLayout) -> int:
    """Device bytes a scene occupies in a gather arena (per-node and
    per-triangle arrays, voxel cells and height samples); a pack reports its
    own exact figure (ScenePack.device_bytes)."""
    nodes = layout.n_nodes
    elems = layout.n_elems
    ground = 0
    for c in layout.pairs:
        if c.kind == "voxel":
            ground += int(c.ground.nx) * int(c.ground.ny)
        elif c.kind == "heightfield":
            ground += 4 * int(c.ground.nx)
    return 48 * nodes + 136 * elems + ground + 64 * len(layout.pairs)


class Arena:
    """Resident scenes in one device arena.

    Args:
        max_*: capacities reserved once
        path: "stream" (the patch-streaming step, one CTA per patch of the
            active scenes; the default) or "gather" (two kernels per
            substep); both give the same bits
        stream_patch: owned nodes per patch of a stream arena (64 or 128)
        stream_minb: CTAs per SM its patch step's registers are budgeted for
            (0: 24 for 64-node patches, 12 for 128-node ones -- the 40-register
            shapes, the fastest at the batch sizes of a request loop)
    """

    def __init__(self, max_nodes, max_elems, max_bodies=4096, max_scenes=4096, max_pairs=4096,
                 max_heights=1 << 20, max_occ=1 << 26, device=0, path="stream", stream_patch=64, stream_minb=0):
        self.native = _native.NativeWorld(device)
        if path == "stream":
            self.native.set_path(_native.FW_PATH_STREAM)
            self.native.set_option(_native.FW_OPT_STREAM_PATCH, int(stream_patch))
        elif path != "gather":
            raise ValueError(f"arena path must be 'stream' or 'gather', not {path!r}")
        self.native.arena_init(max_nodes, max_elems, max_bodies, max_scenes, max_pairs, max_heights, max_occ)
        if path == "stream":
            self.native.set_option(_native.FW_OPT_STREAM_MINB, int(stream_minb or {64: 24, 128: 12}[int(stream_patch)]))
        self.path = path
        self.patch_nodes = int(stream_patch) if path == "stream" else 0
        self.max_scenes = max_scenes
        self.S = max_scenes + 1
        self.layouts = {}
        self._stage = _native.NativeWorld.stage()

    def pack(self, layout: SceneLayout, packed: PackedWorld, pinned: bool = False) -> _native.ScenePack:
        """Host-side preparation of a scene for this arena (validation,
        corner lists, stream patches); touches neither the device nor the
        arena, so another thread may run it while the arena steps (one
        thread at a time per Arena)."""
        if layout.entries:
            raise NotImplementedError("rigid bodies and ground planes with BCs run in an ExplicitLoop or "
                                      "BatchedLoop, not in served worlds")
        stage(self._stage, packed)
        return self._stage.arena_pack(self.patch_nodes, pinned)

    def insert(self, domains, dt=0.0, useAdapativeDT=False, damping=0.0) -> int:
        layout = SceneLayout(domains, dt=dt, damping=damping, useAdapativeDT=useAdapativeDT)
        return self.insert_prepared(layout, PackedWorld([layout]))

    def insert_prepared(self, layout: SceneLayout, packed: PackedWorld) -> int:
        """Upload a scene whose host-side layout and packing are already built."""
        pk = self.pack(layout, packed)
        try:
            return self.insert_pack(layout, pk)
        finally:
            pk.close()  # pageable: its copies were staged when they were queued

    def insert_pack(self, layout: SceneLayout, pk: _native.ScenePack) -> int:
        """Upload a prepared scene (queued on the arena's stream; no wait)."""
        s = self.native.arena_commit_pack(pk)
        self.layouts[s] = layout
        return s

    def remove(self, scene: int):
        self.native.arena_remove(scene)
        self.layouts.pop(scene, None)

    def info(self, scene: int):
        return self.native.arena_scene_info(scene)

    def coords(self, scene: int):
        n0, nn = self.info(scene)[:2]
        return self.native.read_nodes(_native.FW_FIELD_X, int(n0), int(nn))

    def velocities(self, scene: int):
        n0, nn = self.info(scene)[:2]
        return self.native.read_nodes(_native.FW_FIELD_V, int(n0), int(nn))

    def energy(self, scene: int):
        """FP64 energies of one resident scene: kinetic, strain, external, contact."""
        return self.native.energy(self.S)[scene]

    def close(self):
        self._stage.close()
        self.native.close()


@dataclass(order=True)
class Request:
    arrival: float
    rid: int = field(compare=False)
    body: int = field(compare=False)
    substeps: int = field(compare=False)


def poisson_requests(rate, duration, n_bodies, seed=0, substeps=(50, 400)):
    """Poisson arrivals at ``rate`` per second for ``duration`` seconds; each
    request names a body uniformly and a substep count uniform in
    [substeps[0], substeps[1]]."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            break
        out.append(Request(t, len(out), int(rng.integers(n_bodies)),
                           int(rng.integers(substeps[0], substeps[1] + 1))))
    return out


STABLE_MARGIN = 0.5


def request_substeps(req, frame_dt, stable_time):
    """Substeps a request runs: the requested count, raised when the requested
    dt would exceed STABLE_MARGIN x the body's stable time (the reference's
    static CFL / contact bound, explicitloop.py:313-331).  The margin is there
    because the bound itself is not sufficient: soft NeoHookean bodies under
    voxel contact diverge at 0.8 x the bound and stay finite at 0.5 x
    (measured on the CPU oracle)."""
    return max(int(req.substeps), int(np.ceil(frame_dt / (STABLE_MARGIN * stable_time) - 1e-9)))


class _Job:
    __slots__ = ("req", "runs", "pos", "left", "start", "init", "failed")

    def __init__(self, req, frame_dt, stable_time, init=False):
        self.req = req
        self.init = init  # the body was just admitted: its first launch is the zero-dt construction step
        self.failed = False  # its body's state turned non-finite before it was retired
        sub = frame_dt / request_substeps(req, frame_dt, stable_time)
        self.runs = substep_schedule(frame_dt, sub, sub, False)
        self.pos = 0
        self.left = self.runs[0][0]
        self.start = None

    def dt(self):
        return self.runs[self.pos][1]

    def span(self):
        """Substeps this job can run at its current dt (its construction step
        first, if it has not run yet)."""
        return self.left + (1 if self.init else 0)


class Server:
    """Continuous-batching request loop over resident bodies.

    Each iteration runs K substeps in one native call.  On a stream arena
    (fw_step_served_budget) every in-flight request's scene runs only the
    substeps its request has left at its current dt within the call, so a
    request leaves the batch at the very substep it finishes while the call
    goes on for the others; K is capped by max_batch_substeps and, with
    real-time arrivals, by what fits before the next arrival (from the
    measured device time per substep), so new requests join within about one
    arrival gap.  On a gather arena (fw_step_served_n) K also stops at the
    nearest request end.

    Args:
        make_body: body id -> list of domains (the scene of that body)
        budget_bytes: HBM budget for resident bodies (admission control)
        arena_*: arena capacities
        frame_dt: simulated time of one request (advanceWithTime(frame_dt))
        max_inflight: native calls queued ahead of the GPU
        max_batch_substeps: cap on K
    """

    def __init__(self, make_body, budget_bytes=150e9, arena_nodes=8_500_000, arena_elems=17_000_000,
                 arena_bodies=4096, arena_scenes=4096, frame_dt=1.0 / 60.0, max_inflight=4, device=0,
                 max_batch_substeps=64, path="stream", stream_patch=64):
        import torch

        self.make_body = make_body
        self.budget = float(budget_bytes)
        self.frame_dt = frame_dt
        self.arena = Arena(arena_nodes, arena_elems, arena_bodies, arena_scenes, arena_bodies,
                           device=device, path=path, stream_patch=stream_patch)
        self.device = device
        self.stream = torch.cuda.Stream(device=device)
        self.arena.native.set_stream(self.stream.cuda_stream)
        self.max_inflight = max_inflight
        self.max_batch_substeps = int(max_batch_substeps)
        self.us_per_substep = 20.0  # device time per substep, refined from events as calls complete
        self.resident = {}  # body -> scene
        self.used_bytes = 0
        self.body_bytes = {}
        self.deferred_admissions = 0
        self.element_steps = 0
        self.admit_s = 0.0        # host time spent admitting new bodies
        self.last_admit_t = 0.0   # run clock of the last first admission of a body
        self.evicted = 0          # bodies removed because their state turned non-finite
        self.readmitted = 0       # admissions of bodies that were resident before (after an eviction)
        self._prep = {}           # body -> (layout, pack), built ahead by prepare() or at first admission
        self._ever = set()        # bodies admitted at least once
        self.admit_budget_s = 0.002  # host time per loop iteration for admitting new bodies
        self.admit_span = 8          # call length while admissions wait (stream arenas)
        self.host_us = 100.0         # host time of one loop iteration, refined as the loop runs
        self.device_s = 0.0          # device time of the native calls (CUDA events around each call)
        self.trace = None            # a list: one (span, scenes in the call, substeps they ran) per call

    def _build(self, body):
        """Host-side preparation of a body: its domains, scene layout and its
        arena pack in page-locked memory (everything but the upload)."""
        layout = SceneLayout(self.make_body(body))
        return layout, self.arena.pack(layout, PackedWorld([layout]), pinned=True)

    def prepare(self, bodies):
        """Build these bodies' packs ahead of their first request (a catalog
        load); their admission is then an upload queued on the stream.  A
        pack is kept and commits the body afresh if it is evicted."""
        for b in bodies:
            if b not in self._prep:
                self._prep[b] = self._build(b)

    def _queued_work(self, queue, body):
        """Substeps the requests waiting for a body will run (request counts
        raised to the body's stable count, as the jobs will be)."""
        ent = self._prep.get(body)
        if ent is None:
            return sum(r.substeps for r in queue)
        st = ent[0].stableTime
        return sum(request_substeps(r, self.frame_dt, st) for r in queue)

    def close(self):
        """Wait for the arena's stream, then free the packs and the arena."""
        self.arena.native.synchronize()
        for _, pk in self._prep.values():
            pk.close()
        self._prep.clear()
        self.arena.close()

    def _admit(self, body, t0=None):
        """True if resident now; "new" if admitted by this call; False if it
        does not fit (the request waits)."""
        if body in self.resident:
            return True
        ent = self._prep.get(body)
        if ent is None:
            ent = self._prep[body] = self._build(body)
        ta = time.perf_counter()
        layout, pk = ent
        need = pk.device_bytes
        if self.used_bytes + need > self.budget:
            self.deferred_admissions += 1
            return False
        try:
            s = self.arena.insert_pack(layout, pk)
        except _native.NativeError:
            self.deferred_admissions += 1
            return False
        self.resident[body] = s
        self.body_bytes[body] = need
        self.used_bytes += need
        tb = time.perf_counter()
        self.admit_s += tb - ta
        if body in self._ever:
            self.readmitted += 1
        elif t0 is not None:
            self.last_admit_t = tb - t0  # first admissions only: re-admissions follow evictions
        self._ever.add(body)
        return "new"

    def release(self, body):
        s = self.resident.pop(body)
        self.arena.remove(s)
        self.used_bytes -= self.body_bytes.pop(body)

    def run(self, requests, realtime=True):
        """Serve ``requests`` (sorted by arrival).  With realtime, arrivals
        follow the wall clock; otherwise every request is present at t = 0.
        Returns per-request latency (s), wall time and counters.

        Per-scene job state lives in arrays (dt of the current run, substeps
        left in it, busy / construction-step flags), so one iteration costs
        O(scenes) vector work plus Python only for requests whose run ends."""
        arrivals = list(requests)
        heapq.heapify(arrivals)
        return self._run(arrivals, requests, realtime)

    def _run(self, arrivals, requests, realtime):
        import torch

        queues = collections.defaultdict(collections.deque)  # body -> waiting requests
        ready = set()      # idle bodies with a waiting request
        busy = {}          # scene -> job
        busy_bodies = set()
        S = self.arena.S
        cur_dt = np.zeros(S, dtype=np.float32)
        left = np.zeros(S, dtype=np.int64)        # substeps left at the current dt (construction step included)
        busy_m = np.zeros(S, dtype=bool)
        init_m = np.zeros(S, dtype=bool)
        n_el = np.zeros(S, dtype=np.int64)
        adm_set, adm_order = set(), []           # bodies waiting for admission, most queued work first
        ran = np.zeros(S, dtype=np.int32)        # substeps each scene runs in the current call
        bud2 = np.zeros(S, dtype=np.int32)       # ... in its second segment (stream arenas)
        dt2 = np.zeros(S, dtype=np.float32)
        budgets = self.arena.path == "stream"  # per-scene budgets: a call need not stop at each request end
        dts = np.zeros(S, dtype=np.float32)
        inflight = collections.deque()
        done_at = {}
        failed = {}  # rid -> run clock when the request was failed (its body's state turned non-finite)
        pending_done = []  # (event, [jobs finished in that call], start event, substeps, status slot)
        # per-call copies of the non-finite flags, read when the call retires
        ring = 2 * self.max_inflight + 4
        status = torch.zeros((ring, S), dtype=torch.int32, pin_memory=True).numpy()
        slot = 0
        t0 = time.perf_counter()
        n_sub = 0
        n_calls = 0

        def evict(bad_scenes):
            """Fail the requests of bodies whose state turned non-finite and
            remove the bodies (a later request admits them afresh)."""
            scene_body = {sc: b for b, sc in self.resident.items()}
            now_ = time.perf_counter() - t0
            for sc in bad_scenes:
                body = scene_body.get(int(sc))
                if body is None:
                    continue
                job = busy.pop(int(sc), None)
                if job is not None:
                    failed[job.req.rid] = now_
                    busy_m[sc] = False
                    busy_bodies.discard(body)
                for r in queues[body]:
                    failed[r.rid] = now_
                queues[body].clear()
                for entry in pending_done:  # finished in calls not yet retired: ran on the broken state
                    for j in entry[1]:
                        if j.req.body == body:
                            j.failed = True
                ready.discard(body)
                self.release(body)  # waits for the stream, clears the flag
                status[:, sc] = 0   # copies queued before the release must not flag the slot's next body
                self.evicted += 1
        while arrivals or busy or ready or pending_done:
            t_iter = time.perf_counter()
            now = t_iter - t0
            while arrivals and (not realtime or arrivals[0].arrival <= now):
                r = heapq.heappop(arrivals)
                queues[r.body].append(r)
                if r.body not in busy_bodies:
                    ready.add(r.body)
            # start the next request of every idle body that has one; new
            # bodies are uploaded within a host-time budget per iteration, so a
            # burst of first requests cannot stall the requests in flight
            t_adm = time.perf_counter()
            # resident bodies first; then bodies to admit, the most queued work
            # first (the longest queues set the end of a burst)
            new_bodies = {b for b in ready if b not in self.resident}
            if new_bodies != adm_set:  # bodies joined (or left) the wait: order them again
                adm_set = new_bodies
                adm_order = sorted(new_bodies, key=lambda b: (-self._queued_work(queues[b], b), b))
            for body in sorted(b for b in ready if b in self.resident) + adm_order:
                if body not in self.resident and time.perf_counter() - t_adm > self.admit_budget_s:
                    break  # admitted in a later iteration
                adm = self._admit(body, t0)
                if not adm:
                    continue
                s = self.resident[body]
                job = _Job(queues[body].popleft(), self.frame_dt, self.arena.layouts[s].stableTime,
                           init=(adm == "new"))
                job.start = now
                busy[s] = job
                busy_bodies.add(body)
                ready.discard(body)
                cur_dt[s] = job.dt()
                left[s] = job.span()
                busy_m[s] = True
                init_m[s] = job.init
                n_el[s] = self.arena.layouts[s].n_elems
            if adm_set:
                adm_order = [b for b in adm_order if b not in self.resident]
                adm_set = set(adm_order)
            if not busy:
                if not arrivals and not pending_done and ready and not any(b in self.resident for b in ready) \
                        and time.perf_counter() - t_adm <= self.admit_budget_s:
                    raise RuntimeError("requests wait for bodies that cannot be admitted (arena or budget full)")
                # nothing on the GPU: retire finished work, then wait for the next arrival
                evict(self._retire(pending_done, done_at, failed, status, t0, block=True))
                if arrivals and realtime:
                    time.sleep(max(0.0, arrivals[0].arrival - (time.perf_counter() - t0)))
                continue
            waiting = budgets and bool(adm_set)  # bodies wait for admission
            if waiting and len(pending_done) >= 2:
                # bodies wait for admission and the GPU still has two calls to run:
                # spend this iteration admitting rather than queueing a third call
                evict(self._retire(pending_done, done_at, failed, status, t0, block=False))
                continue
            np.copyto(dts, np.where(busy_m, cur_dt, np.float32(0.0)))
            # a call shorter than one host iteration's worth of device time idles the GPU
            floor = max(1, int(self.host_us / self.us_per_substep))
            cap = self.max_batch_substeps
            if realtime and arrivals:  # end the call near the next arrival
                gap_us = (arrivals[0].arrival - (time.perf_counter() - t0)) * 1e6
                cap = min(cap, max(floor, int(gap_us / self.us_per_substep)))
            if waiting:
                cap = min(cap, max(floor, self.admit_span))  # bodies wait for admission: let it catch up
            ev0 = torch.cuda.Event(enable_timing=True)
            ev0.record(self.stream)
            second = []  # (scene, the body's next job or None for the request's own next run)
            if budgets:
                # one call spans request ends: each scene runs its own remaining
                # substeps, then its next run -- the request's remainder at its
                # own dt, or the body's next queued request -- within the call
                span = int(min(cap, left[busy_m].max()))
                np.copyto(ran, np.where(busy_m, np.minimum(left, span), 0))
                bud2.fill(0)
                for s in np.nonzero(busy_m & (left < span))[0].tolist():
                    job = busy[s]
                    if job.pos + 1 < len(job.runs):
                        n2, d2 = job.runs[job.pos + 1]
                        nxt = None
                    elif queues[job.req.body]:
                        nxt = _Job(queues[job.req.body][0], self.frame_dt, self.arena.layouts[s].stableTime)
                        n2, d2 = nxt.runs[0]
                    else:
                        continue
                    bud2[s] = min(n2, span - int(left[s]))
                    dt2[s] = np.float32(d2)
                    second.append((s, nxt))
                if second:
                    self.arena.native.step_served_budget(dts, ran, span, dt2, bud2)
                else:
                    self.arena.native.step_served_budget(dts, ran, span)
            else:
                span = int(min(cap, left[busy_m].min()))
                np.copyto(ran, np.where(busy_m, span, 0))
                self.arena.native.step_served_n(dts, span)
            self.arena.native.scene_status(S, out=status[slot], asynchronous=True)
            if self.trace is not None:
                self.trace.append((span, int(busy_m.sum()), int(ran.sum()) + int(bud2.sum()) if second else int(ran.sum())))
            n_sub += span
            n_calls += 1
            self.element_steps += int((n_el * ran).sum()) - int(n_el[busy_m & init_m].sum())
            init_m[busy_m] = False
            left[busy_m] -= ran[busy_m]
            finished = []
            for s, nxt in second:  # the second segments (their first run has just ended)
                job = busy[s]
                self.element_steps += int(n_el[s]) * int(bud2[s])
                if nxt is None:
                    job.pos += 1
                else:
                    finished.append(job)
                    queues[job.req.body].popleft()
                    nxt.start = now
                    busy[s] = job = nxt
                cur_dt[s] = job.runs[job.pos][1]
                left[s] = job.runs[job.pos][0] - int(bud2[s])
            for s in np.nonzero(busy_m & (left == 0))[0].tolist():
                job = busy[s]
                job.pos += 1
                if job.pos < len(job.runs):  # next run of the same request, at its own dt
                    cur_dt[s] = job.runs[job.pos][1]
                    left[s] = job.runs[job.pos][0]
                    continue
                finished.append(job)
                del busy[s]
                busy_m[s] = False
                body = job.req.body
                busy_bodies.discard(body)
                if queues[body]:
                    ready.add(body)
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(self.stream)
            pending_done.append((ev, finished, ev0, span, slot))
            slot = (slot + 1) % ring
            inflight.append(ev)
            # host time of an iteration that issues a call (before any wait on the GPU)
            self.host_us = 0.9 * self.host_us + 0.1 * (time.perf_counter() - t_iter) * 1e6
            if len(inflight) > self.max_inflight:
                inflight.popleft().synchronize()
            evict(self._retire(pending_done, done_at, failed, status, t0, block=False))
        evict(self._retire(pending_done, done_at, failed, status, t0, block=True))
        wall = time.perf_counter() - t0
        ends = {**done_at, **failed}
        lat = np.array([ends[r.rid] - r.arrival if realtime else ends[r.rid] for r in requests])
        return {"latency_s": lat, "wall_s": wall, "substeps": n_sub, "native_calls": n_calls,
                "failed": sorted(failed), "evicted_bodies": self.evicted, "readmitted_bodies": self.readmitted,
                "element_steps": self.element_steps, "deferred_admissions": self.deferred_admissions,
                "resident_bodies": len(self.resident), "used_bytes": self.used_bytes,
                "admit_s": self.admit_s, "last_admit_t": self.last_admit_t, "device_s": self.device_s}

    def _retire(self, pending_done, done_at, failed, status, t0, block):
        """Retire completed calls in order; returns the scenes whose state
        turned non-finite in them (their finished requests count as failed)."""
        bad = set()
        while pending_done:
            ev, jobs, ev0, span, slot = pending_done[0]
            if block:
                ev.synchronize()
            elif not ev.query():
                break
            t = time.perf_counter() - t0
            flagged = set(np.nonzero(status[slot])[0].tolist())
            bad |= flagged
            for j in jobs:
                if j.failed or self.resident.get(j.req.body) in flagged:
                    failed[j.req.rid] = t
                else:
                    done_at[j.req.rid] = t
            call_ms = ev0.elapsed_time(ev)
            self.device_s += call_ms * 1e-3
            self.us_per_substep = 0.8 * self.us_per_substep + 0.2 * max(1.0, call_ms * 1e3 / span)
            pending_done.pop(0)
        return bad

    def coords(self, body):
        return self.arena.coords(self.resident[body])


class FifoPlainServer:
    """Comparison server: requests one at a time in arrival order, each body
    in its own ExplicitLoop (created at its first request, kept afterwards)."""

    def __init__(self, make_body, frame_dt=1.0 / 60.0, device=0):
        self.make_body = make_body
        self.frame_dt = frame_dt
        self.device = device
        self.loops = {}
        self.element_steps = 0

    def run(self, requests, realtime=True, time_limit=None):
        t0 = time.perf_counter()
        done_at = {}
        for r in sorted(requests):
            now = time.perf_counter() - t0
            if realtime and r.arrival > now:
                time.sleep(r.arrival - now)
            if time_limit is not None and time.perf_counter() - t0 > time_limit:
                break
            lp = self.loops.get(r.body)
            if lp is None:
                lp = ExplicitLoop(0.0, self.make_body(r.body), useAdapativeDT=False, device=self.device)
                self.loops[r.body] = lp
            sub = self.frame_dt / request_substeps(r, self.frame_dt, lp.stableTime)
            lp.default_dt = sub
            lp.advanceWithTime(self.frame_dt)
            lp.synchronize()
            self.element_steps += lp._packed.E * sum(n for n, _ in substep_schedule(self.frame_dt, sub, sub, False))
            done_at[r.rid] = time.perf_counter() - t0
        served = [r for r in requests if r.rid in done_at]
        lat = np.array([done_at[r.rid] - r.arrival if realtime else done_at[r.rid] for r in served])
        return {"latency_s": lat, "wall_s": time.perf_counter() - t0, "served": len(served),
                "element_steps": self.element_steps}
