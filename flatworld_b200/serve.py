"""Served form: a request loop with continuous batching.

A request asks one soft body to advance by ``advanceWithTime(frame_dt)`` in a
given number of substeps.  The ``Server`` keeps every admitted body resident in
a device arena (flatworld_b200 C ABI: fw_arena_*), so a body's state carries
over between its requests, and advances all bodies that have a request in
flight together, one substep at a time: the batch is rebuilt every substep
(requests that arrive join at the next substep; finished ones leave), and a
new body is admitted when the arena and the HBM budget have room for it.
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
    """Device bytes a scene occupies in the arena (per-node and per-triangle
    arrays, voxel cells and height samples)."""
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
    """Resident scenes in one device arena."""

    def __init__(self, max_nodes, max_elems, max_bodies=4096, max_scenes=4096, max_pairs=4096,
                 max_heights=1 << 20, max_occ=1 << 26, device=0):
        self.native = _native.NativeWorld(device)
        self.native.arena_init(max_nodes, max_elems, max_bodies, max_scenes, max_pairs, max_heights, max_occ)
        self.max_scenes = max_scenes
        self.S = max_scenes + 1
        self.layouts = {}

    def insert(self, domains, dt=0.0, useAdapativeDT=False, damping=0.0) -> int:
        layout = SceneLayout(domains, dt=dt, damping=damping, useAdapativeDT=useAdapativeDT)
        stage(self.native, PackedWorld([layout]))
        s = self.native.arena_commit()
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
    __slots__ = ("req", "runs", "pos", "left", "start", "init")

    def __init__(self, req, frame_dt, stable_time, init=False):
        self.req = req
        self.init = init  # the body was just admitted: its first launch is the zero-dt construction step
        sub = frame_dt / request_substeps(req, frame_dt, stable_time)
        self.runs = substep_schedule(frame_dt, sub, sub, False)
        self.pos = 0
        self.left = self.runs[0][0]
        self.start = None

    def dt(self):
        return self.runs[self.pos][1]

    def advance(self):
        if self.init:
            self.init = False
            return False
        self.left -= 1
        if self.left == 0:
            self.pos += 1
            if self.pos < len(self.runs):
                self.left = self.runs[self.pos][0]
        return self.pos >= len(self.runs)


class Server:
    """Continuous-batching request loop over resident bodies.

    Args:
        make_body: body id -> list of domains (the scene of that body)
        budget_bytes: HBM budget for resident bodies (admission control)
        arena_*: arena capacities
        frame_dt: simulated time of one request (advanceWithTime(frame_dt))
        max_inflight: substeps queued ahead of the GPU
    """

    def __init__(self, make_body, budget_bytes=150e9, arena_nodes=8_500_000, arena_elems=17_000_000,
                 arena_bodies=4096, arena_scenes=4096, frame_dt=1.0 / 60.0, max_inflight=4, device=0):
        import torch

        self.make_body = make_body
        self.budget = float(budget_bytes)
        self.frame_dt = frame_dt
        self.arena = Arena(arena_nodes, arena_elems, arena_bodies, arena_scenes, arena_bodies,
                           device=device)
        self.device = device
        self.stream = torch.cuda.Stream(device=device)
        self.arena.native.set_stream(self.stream.cuda_stream)
        self.max_inflight = max_inflight
        self.resident = {}  # body -> scene
        self.used_bytes = 0
        self.body_bytes = {}
        self.deferred_admissions = 0
        self.element_steps = 0

    def _admit(self, body):
        """True if resident now; "new" if admitted by this call; False if it
        does not fit (the request waits)."""
        if body in self.resident:
            return True
        doms = self.make_body(body)
        need = scene_device_bytes(SceneLayout(doms))
        if self.used_bytes + need > self.budget:
            self.deferred_admissions += 1
            return False
        try:
            s = self.arena.insert(doms)
        except _native.NativeError:
            self.deferred_admissions += 1
            return False
        self.resident[body] = s
        self.body_bytes[body] = need
        self.used_bytes += need
        return "new"

    def release(self, body):
        s = self.resident.pop(body)
        self.arena.remove(s)
        self.used_bytes -= self.body_bytes.pop(body)

    def run(self, requests, realtime=True):
        """Serve ``requests`` (sorted by arrival).  With realtime, arrivals
        follow the wall clock; otherwise every request is present at t = 0.
        Returns per-request latency (s), wall time and counters."""
        import torch

        arrivals = list(requests)
        heapq.heapify(arrivals)
        queues = collections.defaultdict(collections.deque)  # body -> waiting requests
        busy = {}  # scene -> job
        dts = np.zeros(self.arena.S, dtype=np.float32)
        inflight = collections.deque()
        done_at = {}
        pending_done = []  # (event, [jobs finished at that substep])
        t0 = time.perf_counter()
        n_sub = 0
        while arrivals or busy or any(queues.values()) or pending_done:
            now = time.perf_counter() - t0
            while arrivals and (not realtime or arrivals[0].arrival <= now):
                r = heapq.heappop(arrivals)
                queues[r.body].append(r)
            # start the next request of every idle body that has one
            busy_bodies = {j.req.body for j in busy.values()}
            for body, q in queues.items():
                if q and body not in busy_bodies:
                    adm = self._admit(body)
                    if not adm:
                        continue
                    s = self.resident[body]
                    job = _Job(q.popleft(), self.frame_dt, self.arena.layouts[s].stableTime, init=(adm == "new"))
                    job.start = now
                    busy[s] = job
            if not busy:
                if not arrivals and not pending_done and any(queues.values()):
                    raise RuntimeError("requests wait for bodies that cannot be admitted (arena or budget full)")
                # nothing on the GPU: retire finished work, then wait for the next arrival
                self._retire(pending_done, done_at, t0, block=True)
                if arrivals and realtime:
                    time.sleep(max(0.0, arrivals[0].arrival - (time.perf_counter() - t0)))
                continue
            dts[:] = 0.0
            for s, job in busy.items():
                dts[s] = job.dt()
            self.arena.native.step_served(dts)
            n_sub += 1
            finished = []
            for s, job in list(busy.items()):
                if not job.init:
                    self.element_steps += self.arena.layouts[s].n_elems
                if job.advance():
                    finished.append(job)
                    del busy[s]
            ev = torch.cuda.Event()
            ev.record(self.stream)
            pending_done.append((ev, finished))
            inflight.append(ev)
            if len(inflight) > self.max_inflight:
                inflight.popleft().synchronize()
            self._retire(pending_done, done_at, t0, block=False)
        self._retire(pending_done, done_at, t0, block=True)
        wall = time.perf_counter() - t0
        lat = np.array([done_at[r.rid] - r.arrival if realtime else done_at[r.rid] for r in requests])
        return {"latency_s": lat, "wall_s": wall, "substeps": n_sub, "element_steps": self.element_steps,
                "deferred_admissions": self.deferred_admissions, "resident_bodies": len(self.resident),
                "used_bytes": self.used_bytes}

    @staticmethod
    def _retire(pending_done, done_at, t0, block):
        while pending_done:
            ev, jobs = pending_done[0]
            if block:
                ev.synchronize()
            elif not ev.query():
                break
            t = time.perf_counter() - t0
            for j in jobs:
                done_at[j.req.rid] = t
            pending_done.pop(0)

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
