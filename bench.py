"""Benchmark: FEM element-steps/s of the explicit 2D FEM step on B200.

Default workload (N=1): the plain large single mesh -- unit square at (0, 0.2),
256 x 256 quads split in two (131072 triangles, 66049 nodes), NeoHookean
E=1e5 nu=0.35 rho=100, v0 = (0, -0.5) + N(0, 0.01^2), height field of 4096
samples (8 sinusoids, amplitude 0.05), adaptive (static CFL) dt.  One bench
"step" is one ``advanceWithTime(1/60)`` frame (548 substeps at dt = 3.04e-5);
L2 is flushed (256 MiB write) between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

For N > 1 (torchrun, one rank per GPU) every rank steps its own replica of the
workload (weak scaling; the bodies of different ranks never interact, so there
is no collective on the data path).  ``--impl reference`` times the CPU
restatement of the reference's scheme (the reference itself, Python + NVIDIA
Warp, is not installable here) on this host's cores.
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from flatworld_b200 import _native, shard  # noqa: E402

FRAME = 1.0 / 60.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--mesh", type=int, default=256, help="quads per side of the large mesh")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--workload", choices=["plain_large", "batched", "served", "adjoint", "flex", "rigid"],
                    default="plain_large")
    ap.add_argument("--rigid-mesh", type=int, default=256,
                    help="rigid: quads along the slab (and a quarter of that across)")
    ap.add_argument("--rigid-scenes", type=int, default=1,
                    help="rigid: > 1 batches that many independent 32 x 8-quad slab scenes (BatchedLoop)")
    ap.add_argument("--flex-side", type=int, default=12, help="flex: disks per row and column of the pile")
    ap.add_argument("--flex-scenes", type=int, default=1,
                    help="flex: > 1 batches that many independent 3 x 3 piles (BatchedLoop) instead of one pile")
    ap.add_argument("--fd-directions", type=int, default=16, help="adjoint: FP64 central-FD directions checked")
    ap.add_argument("--rate", type=float, default=2000.0, help="served: requests per second")
    ap.add_argument("--duration", type=float, default=10.0, help="served: seconds of arrivals")
    ap.add_argument("--fifo-seconds", type=float, default=5.0, help="served: wall-time cap of the FIFO server")
    ap.add_argument("--scenes", type=int, default=2048, help="batched: number of bodies")
    ap.add_argument("--plain-sample", type=int, default=64, help="batched: bodies timed alone")
    ap.add_argument("--stream-patch", choices=["auto", "64", "128"], default="auto",
                    help="batched, stream path: owned nodes per patch (auto: tuned on a sample)")
    ap.add_argument("--stream-minb", type=int, default=0,
                    help="batched, stream path: CTAs per SM of the register budget (0: tuned)")
    ap.add_argument("--stream-bulk", type=int, choices=[-1, 0, 1], default=-1,
                    help="batched, stream path: stage triangle records by bulk copy (-1: tuned)")
    ap.add_argument("--serve-path", choices=["gather", "stream"], default="stream",
                    help="served: arena step implementation (same bits)")
    ap.add_argument("--batch-path", choices=["gather", "stream"], default="stream",
                    help="batched: step implementation (same bits)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def dist_init(world, local):
    """One process per GPU (torchrun): an NCCL group with a short timeout for
    the barriers and the whole-job reductions; None on one GPU."""
    if world <= 1:
        return None
    import datetime

    import torch
    import torch.distributed as dist

    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    return dist


def barrier(dist):
    if dist is not None:
        import torch

        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()


def workload(fw, mesh):
    from tests import scenes

    return scenes.plain_large_scene(fw, n=mesh)


def algorithmic_bytes_per_substep(n_nodes, n_elems, n_j2, n_contact_nodes, ground_bytes):
    """Compulsory traffic of one substep: nodes read+write x, v and read the
    inverse mass (36 B); elements read connectivity (12), Dm^-1 (16), rest area
    (4) and the two Lame constants (8) = 40 B; J2 elements read+write eps_p and
    eqps (32 B); each boundary contact item reads a node id and a penalty (8);
    ground tables once (height field 4 B/sample)."""
    return 36 * n_nodes + 40 * n_elems + 32 * n_j2 + 8 * n_contact_nodes + ground_bytes


class ClockSampler:
    """Samples SM clock and throttle reasons through NVML while running."""

    REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
               0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting"}

    def __init__(self, device_index):
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self._stop = threading.Event()
        self._ok = False
        try:
            import pynvml
            import torch

            pynvml.nvmlInit()
            p = torch.cuda.get_device_properties(device_index)
            bus = f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
            self._h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            self._nv = pynvml
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
            self._ok = True
        except Exception as e:  # pragma: no cover - depends on the box
            self.error = str(e)

    def _run(self):
        nv = self._nv
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                for bit, name in self.REASONS.items():
                    if r & bit and bit != 0x1:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.005)  # 5 ms: several samples even in a timed region of ~40 ms

    def __enter__(self):
        if self._ok:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._ok:
            self._t.join()

    def summary(self):
        if not self._ok or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                    "note": getattr(self, "error", "no samples")}
        return {"sm_mhz": float(np.median(self.samples)), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic():
    """Per-substep DRAM bytes of the step kernels from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "traffic_plain_large.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f).get("dram_bytes_per_substep")
    return None


def ncu_traffic_ratio_batched(step_path="gather", shape=None):
    """(DRAM bytes / algorithmic bytes, where it was measured) of the batched
    step kernels, from ncu captures of a 256-body batch (per-triangle and
    per-node traffic do not depend on the batch size, so the ratio scales to
    the full batch).  On the stream path the ratio of the launch shape in use
    (``BatchedLoop.stream_shape``) where one was captured."""
    path = os.path.join(ROOT, "profiles", "traffic_batched.json")
    if not os.path.exists(path):
        return None, None
    with open(path) as f:
        d = json.load(f)
    if step_path != "stream":
        return d.get("traffic_over_algorithmic"), d.get("source")
    shapes = d.get("stream_shapes", {})
    if shape in shapes:
        return shapes[shape], f"{d.get('stream_shapes_source')}, shape {shape}"
    return d.get("stream_traffic_over_algorithmic"), d.get("stream_source")


def flex_work_items(pk):
    """FEM-FEM contact work items of a packed world: per pair, the boundary
    nodes of both bodies (each node a query against the other body)."""
    return sum(int(pk.bncnt[b1] + pk.bncnt[b2]) for _, _, _, _, _, prs in pk.flex_records() for b1, b2, *_ in prs)


def cpu_oracle_rate(fw, mesh, seconds, threads):
    """Element-steps/s of the CPU restatement on this host (bounded sample)."""
    import oracle

    o = oracle.OracleLoop(workload(fw, mesh), 0.0, useAdapativeDT=True, precision="f32", threads=threads)
    o.advance(3)
    t0 = time.perf_counter()
    n = 0
    while time.perf_counter() - t0 < seconds:
        o.advance(5)
        n += 5
    dt = time.perf_counter() - t0
    return o.E * n / dt, n


def run_reference(args, rank, world):
    if rank != 0:
        return
    import flatworld_b200 as fw

    threads = os.cpu_count() or 1
    import oracle

    o = oracle.OracleLoop(workload(fw, args.mesh), 0.0, useAdapativeDT=True, precision="f32", threads=threads)
    # one bench step = advanceWithTime(1/60), the same frame of substeps the GPU arm times
    for _ in range(args.warmup):
        o.advance_with_time(FRAME)
    c0 = o.counter
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.advance_with_time(FRAME)
    el = time.perf_counter() - t0
    sample = (o.counter - c0) // args.steps
    value = o.E * (o.counter - c0) / el
    line = {
        "impl": "reference", "metric": "FEM element-steps/s", "value": value, "unit": "element-steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": el / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"plain large single mesh {args.mesh}x{args.mesh} quads, NeoHookean, height field",
                   "elements": o.E, "nodes": o.N, "step": "advanceWithTime(1/60)", "substeps_per_step": sample,
                   "dt": o.stableTime},
        "cpu_baseline": {"value": value, "unit": "element-steps/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} steps of advanceWithTime(1/60) ({sample} substeps each) of the "
                                   f"workload, FP32 C restatement of the reference scheme, {threads} threads"},
        "e2e": {"value": value, "unit": "element-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def percentile_ms(samples, q):
    return float(np.percentile(np.asarray(samples), q))


def run_batched(args, rank, world, local):
    """Ragged batch: 2048 independent bodies (node count log-uniform in
    [100, 20000], aspect U[0.25, 4], Elastic / NeoHookean / J2 in thirds, each
    on its own 128 x 128 Bernoulli(0.15) voxel grid), dt = 5e-5, 1000 substeps,
    all bodies in one world (two kernels per substep).  Baseline: the same
    bodies stepped one at a time by the plain path (a random sample of
    --plain-sample bodies, each alone for 1000 substeps)."""
    import torch

    import flatworld_b200 as fw
    from flatworld_b200 import autotune
    from flatworld_b200.batch import BatchedLoop
    from tests import scenes

    torch.cuda.set_device(local)
    dist = dist_init(world, local)
    substeps = 100 * args.steps
    t0 = time.perf_counter()
    batch = scenes.ragged_batch(fw, args.scenes, seed=rank)
    patch_tuning = None
    stream_patch = 0
    if args.batch_path == "stream":
        if args.stream_patch == "auto":
            # the patch size is fixed when a loop is built: pick it on a sample
            # of the batch (every 8th body), each size with its tuned launch shape
            sample = batch[::8]
            stream_patch, patch_tuning = autotune.tune_stream_patch(
                lambda p: BatchedLoop(sample, dt=5e-5, useAdapativeDT=False, device=local, path="stream",
                                      stream_patch=p))
        else:
            stream_patch = int(args.stream_patch)
    b = BatchedLoop(batch, dt=5e-5, useAdapativeDT=False, device=local, path=args.batch_path,
                    stream_patch=stream_patch)
    build_s = time.perf_counter() - t0
    if args.batch_path == "stream" and (args.stream_minb or args.stream_bulk >= 0):
        b.set_stream_shape(args.stream_minb, None if args.stream_bulk < 0 else bool(args.stream_bulk))
        tuned = {"path": "stream", "shape": b.stream_shape, "chosen_by": "command line"}
    else:
        tuned = autotune.tune_batched(b)
    if patch_tuning is not None:
        tuned = dict(tuned, patch_candidates=patch_tuning)
    stream = torch.cuda.Stream()
    b.set_stream(stream.cuda_stream)
    with torch.cuda.stream(stream):
        b.advance(100 * args.warmup)
        barrier(dist)
        l0 = b.launch_count()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(substeps)]
        with ClockSampler(local) as clk:
            for s_, e_ in ev:
                s_.record(stream)
                b.advance(1)
                e_.record(stream)
            torch.cuda.synchronize()
        launches = b.launch_count() - l0
        # ---- end to end: every body's positions and velocities in from pinned
        # host memory, one step of 100 substeps, and back out
        N = b.n_nodes
        xh = torch.empty((N, 2), dtype=torch.float32, pin_memory=True)
        vh = torch.empty((N, 2), dtype=torch.float32, pin_memory=True)
        b._native.read_nodes_ptr(0, 0, N, xh.data_ptr())
        b._native.read_nodes_ptr(1, 0, N, vh.data_ptr())
        ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for s_, e_ in ev2:
            s_.record(stream)
            b._native.write_nodes_ptr(0, 0, N, xh.data_ptr())
            b._native.write_nodes_ptr(1, 0, N, vh.data_ptr())
            b.advance(100)
            b._native.read_nodes_ptr(0, 0, N, xh.data_ptr())
            b._native.read_nodes_ptr(1, 0, N, vh.data_ptr())
            e_.record(stream)
        torch.cuda.synchronize()
    barrier(dist)
    lat = [s_.elapsed_time(e_) for s_, e_ in ev]
    E = b.n_elems
    work, ms = shard.aggregate(E * substeps, float(sum(lat)))
    work_e2e, ms_e2e = shard.aggregate(E * 100 * args.steps, float(sum(s_.elapsed_time(e_) for s_, e_ in ev2)))
    finite = bool(np.isfinite(b.all_coords()).all())
    value = work / (ms / 1e3)
    # plain path: sample of the same bodies, one loop per body
    rng = np.random.default_rng(1234)
    pick = rng.choice(args.scenes, size=min(args.plain_sample, args.scenes), replace=False)
    plain_e, plain_ms, plain_lat = 0, 0.0, []
    for i in pick:
        doms = scenes.ragged_batch_one(fw, int(i), seed=rank)
        lp = fw.ExplicitLoop(5e-5, doms, useAdapativeDT=False, device=local)
        lp._native.set_stream(stream.cuda_stream)
        lp.advance_n(20)
        s_, e_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s_.record(stream)
        lp.advance_n(substeps)
        e_.record(stream)
        e_.synchronize()
        t = s_.elapsed_time(e_)
        plain_ms += t
        plain_e += doms[1].nelements
        plain_lat.append(t / substeps)
        lp._native.close()
    plain_value = plain_e * substeps / (plain_ms / 1e3)
    nb = int(sum(b.packed.bncnt))
    nj2 = int(np.sum(b.packed.mtype == 3))
    ground = sum(c.ground.nx * c.ground.ny // 8 for lay in b.layouts for c in lay.pairs)
    bstep = algorithmic_bytes_per_substep(b.n_nodes, E, nj2, nb, ground)
    achieved = bstep / (ms / 1e3 / substeps) / 1e9
    peak, which = peaks()
    ratio, ratio_src = ncu_traffic_ratio_batched(args.batch_path, b.stream_shape if b.stream_patch else None)
    line = {
        "metric": "FEM element-steps/s (batched ragged bodies)", "value": value, "unit": "element-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded bodies, materials and voxel grids)",
        "config": {"workload": f"ragged batch of {args.scenes} bodies on voxel grids, dt 5e-5",
                   "elements": E, "nodes": b.n_nodes, "bodies": args.scenes, "substeps": substeps,
                   "step": "100 substeps", "l2": "working set larger than L2", "launch": tuned,
                   "host_build_s": build_s, "state_finite": finite, "replicas": world,
                   "step_path": args.batch_path},
        "batched_vs_plain": {"plain_value": plain_value, "ratio": value / plain_value,
                             "plain_sample_bodies": len(pick),
                             "plain_p50_ms_per_substep": percentile_ms(plain_lat, 50)},
        "latency_ms_per_substep": {"p50": percentile_ms(lat, 50), "p99": percentile_ms(lat, 99),
                                   "p99.9": percentile_ms(lat, 99.9)},
        "roofline": {"bound": "hbm",
                     "kernel": ("substep = k_control + k_stream" if args.batch_path == "stream"
                                else "substep = k_elements + k_nodes"), "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": which,
                     "algorithmic_bytes_per_substep": bstep,
                     "traffic": None if ratio is None else round(ratio * bstep),
                     "traffic_from": ("DRAM bytes per substep scaled from an ncu capture of a 256-body batch: "
                                      f"{ratio_src}")},
        "e2e": {"value": work_e2e / (ms_e2e / 1e3), "unit": "element-steps/s",
                "h2d_bytes_per_step": 2 * N * 8, "d2h_bytes_per_step": 2 * N * 8},
        "gpu_launches": launches, "clocks": clk.summary(),
    }
    if rank == 0 and not args.no_cpu_baseline:
        import oracle

        threads = os.cpu_count() or 1
        work, t_cpu, bodies = 0, 0.0, 0
        for i in pick[:8]:  # a bounded sample: 8 of the same bodies, 100 substeps each
            o = oracle.OracleLoop(scenes.ragged_batch_one(fw, int(i), seed=rank), 5e-5, useAdapativeDT=False,
                                  precision="f32", threads=threads)
            t1 = time.perf_counter()
            o.advance(100)
            t_cpu += time.perf_counter() - t1
            work += o.E * 100
            bodies += 1
        line["cpu_baseline"] = {"value": work / t_cpu, "unit": "element-steps/s", "cores": threads, "kind": "port",
                                "sample": f"{bodies} bodies of the batch x 100 substeps, FP32 C restatement of the "
                                          f"reference scheme, {threads} threads"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def run_served(args, rank, world, local):
    """Request stream: Poisson arrivals at --rate per second for --duration s;
    each request advances one body (drawn as in the ragged batch, a population
    of --scenes bodies) by advanceWithTime(1/60) in U{50..400} substeps.  Bodies
    stay resident between their requests; admission by free HBM (150 GB
    budget).  Compared with a FIFO server that runs requests one at a time on
    the plain path (one ExplicitLoop per body) on the same stream."""
    import torch

    import flatworld_b200 as fw
    from flatworld_b200.serve import FifoPlainServer, Server, poisson_requests
    from tests import scenes

    torch.cuda.set_device(local)
    dist = dist_init(world, local)
    t0 = time.perf_counter()
    population = scenes.ragged_batch(fw, args.scenes, seed=rank)  # request payloads, built client-side
    build_s = time.perf_counter() - t0
    reqs = poisson_requests(args.rate, args.duration, args.scenes, seed=17 + rank)
    srv = Server(lambda b: population[b], budget_bytes=150e9, device=local, path=args.serve_path)
    # catalog load: every body's pack (host-side layout, corner lists, stream
    # patches, in page-locked memory) built before the stream starts;
    # admission (an upload queued on the arena's stream) happens at its first request
    t1 = time.perf_counter()
    srv.prepare(range(args.scenes))
    prepare_s = time.perf_counter() - t1
    # warm-up: compile paths and touch the allocator with a few bodies
    warm = poisson_requests(200.0, 0.05, 8, seed=5)
    wsrv = Server(lambda b: scenes.ragged_batch_one(fw, 10_000 + b), arena_nodes=200_000, arena_elems=400_000,
                  arena_bodies=64, arena_scenes=64, device=local, path=args.serve_path)
    wsrv.run(warm, realtime=False)
    wsrv.close()
    barrier(dist)
    l0 = srv.arena.native.launch_count()
    with ClockSampler(local) as clk:
        out = srv.run(reqs, realtime=True)
    launches = srv.arena.native.launch_count() - l0
    srv.close()
    # capacity: the requests of the first 10 s all queued at t = 0 (a fresh server)
    cap_reqs = [r for r in reqs if r.arrival < 10.0]
    cap_srv = Server(lambda b: population[b], budget_bytes=150e9, device=local, path=args.serve_path)
    cap_srv.prepare(range(args.scenes))
    cap = cap_srv.run(cap_reqs, realtime=False)
    cap_srv.close()
    steps_all, wall = shard.aggregate(out["element_steps"], out["wall_s"])
    lat = out["latency_s"] * 1e3
    steady = np.asarray([l for l, r in zip(lat, reqs) if r.arrival > out["last_admit_t"]])
    if dist is not None:  # every rank's requests count in the percentiles
        gathered = [None] * world
        dist.all_gather_object(gathered, lat.tolist())
        lat = np.asarray([v for g in gathered for v in g])
    fifo = FifoPlainServer(lambda b: population[b], device=local)
    fo = fifo.run(reqs, realtime=True, time_limit=args.fifo_seconds)
    flat = fo["latency_s"] * 1e3
    line = {
        "metric": "FEM element-steps/s (served, continuous batching)",
        "value": steps_all / wall, "unit": "element-steps/s", "n_gpus": world,
        "steps": len(lat), "warmup": len(warm), "ms_per_step": float(np.mean(lat)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded bodies, Poisson arrivals)",
        "config": {"workload": f"served: {args.rate:.0f} req/s Poisson for {args.duration:.0f} s, "
                               f"{args.scenes} resident bodies, advanceWithTime(1/60) in U{{50..400}} substeps",
                   "requests": len(reqs), "population_build_s": build_s, "catalog_prepare_s": prepare_s,
                   "step_path": args.serve_path,
                   "budget_bytes": 150e9,
                   "resident_bodies": out["resident_bodies"], "resident_bytes": out["used_bytes"],
                   "deferred_admissions": out["deferred_admissions"], "substeps_run": out["substeps"]},
        "capacity": {"requests": len(cap_reqs), "wall_s": cap["wall_s"],
                     "sims_per_s": len(cap_reqs) / cap["wall_s"],
                     "element_steps_per_s": cap["element_steps"] / cap["wall_s"],
                     "native_calls": cap["native_calls"], "substeps": cap["substeps"],
                     "device_busy_s": cap["device_s"], "admit_s": cap["admit_s"],
                     "note": "same requests all queued at t = 0 (saturated GPU); includes admitting 2048 bodies"},
        "served": {"sims_per_s": len(lat) / wall, "wall_s": wall, "substeps": out["substeps"],
                   "native_calls": out["native_calls"], "admit_s": out["admit_s"], "device_busy_s": out["device_s"],
                   "last_admission_at_s": out["last_admit_t"], "evicted_bodies": out["evicted_bodies"],
                   "readmitted_bodies": out["readmitted_bodies"], "failed_requests": len(out["failed"]),
                   "failed_note": "bodies whose state turned non-finite (flagged on the device) are evicted and "
                                  "their requests failed; a later request re-admits them afresh",
                   "latency_ms_after_last_admission": {
                       "requests": int(len(steady)),
                       "p50": percentile_ms(steady, 50) if len(steady) else None,
                       "p99": percentile_ms(steady, 99) if len(steady) else None,
                       "p99.9": percentile_ms(steady, 99.9) if len(steady) else None},
                   "latency_ms": {"p50": percentile_ms(lat, 50), "p99": percentile_ms(lat, 99),
                                  "p99.9": percentile_ms(lat, 99.9)}},
        "fifo_plain": {"served": fo["served"], "wall_s": fo["wall_s"],
                       "sims_per_s": fo["served"] / fo["wall_s"],
                       "element_steps_per_s": fo["element_steps"] / fo["wall_s"],
                       "latency_ms": {"p50": percentile_ms(flat, 50) if len(flat) else None,
                                      "p99": percentile_ms(flat, 99) if len(flat) else None}},
        "gpu_launches": launches, "clocks": clk.summary(),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def fd_check(fw, build, sim, v0, steps, dt, target, eb32, vb32, eb64, vb64, n_dirs, threads):
    """CPU leg of the adjoint workload: FP64 central finite differences of the
    loss on the oracle along n_dirs random directions (half in the moduli,
    half in the initial velocities).  The oracle takes float32 inputs, so the
    perturbed inputs are rounded to float32 and the adjoint is dotted with the
    direction the rollouts saw.  Returns (seconds per rollout, errors)."""
    import oracle

    def rollout(young, v):
        o = oracle.OracleLoop(build(young), dt, useAdapativeDT=False, precision="f64", threads=threads)
        o.set_state(None, v)
        o.advance(steps)
        return o.state()[0]

    def perturbed(p0, d, eps):
        hi = (p0.astype(np.float64) + eps * d).astype(np.float32)
        lo = (p0.astype(np.float64) - eps * d).astype(np.float32)
        return hi, lo, (hi.astype(np.float64) - lo.astype(np.float64)) / (2.0 * eps)

    loss = lambda x: float(np.sum((x - target) ** 2))  # noqa: E731
    rng = np.random.default_rng(2024)
    eps, out, t_roll, n_roll = 1e-4, {"E": [], "v": []}, 0.0, 0
    for k in range(n_dirs):
        kind = "E" if k % 2 == 0 else "v"
        if kind == "E":
            Ep, Em, dE = perturbed(sim.E0, sim.E0 * rng.standard_normal(sim.E), eps)
            vp = vm = v0
            a32, a64 = float(np.dot(eb32.astype(np.float64), dE)), float(np.dot(eb64.astype(np.float64), dE))
        else:
            vp, vm, dv = perturbed(v0, rng.standard_normal((sim.N, 2)), eps)
            Ep = Em = sim.E0
            a32 = float(np.sum(vb32.astype(np.float64) * dv))
            a64 = float(np.sum(vb64.astype(np.float64) * dv))
        t0 = time.perf_counter()
        fd = (loss(rollout(Ep, vp)) - loss(rollout(Em, vm))) / (2 * eps)
        t_roll += time.perf_counter() - t0
        n_roll += 2
        out[kind].append((abs(a32 - fd) / abs(fd), abs(a64 - fd) / abs(fd)))
    return t_roll / n_roll, out


def run_adjoint(args, rank, world, local):
    """Differentiable form: 64 x 64-quad NeoHookean block (8192 triangles,
    per-element E log-normal, mean 1e5, sigma 0.3), dropped from y = 0.5 with
    v0 = (0, -2) onto the plane y = 0, 2000 substeps at dt = 1e-4, checkpoints
    every 50.  Loss |x_T - x_T(1.1 E)|^2.  One bench step = one gradient
    evaluation: the forward rollout (storing checkpoints) and the adjoint
    (recompute + reverse per segment), dL/dE per triangle and dL/dv0 per node
    returned to the host."""
    import torch

    import flatworld_b200 as fw
    from flatworld_b200.diff import DiffSim
    from tests import scenes

    torch.cuda.set_device(local)
    dist = dist_init(world, local)
    dt, steps, K = 1e-4, 2000, 50
    build = lambda y=None: scenes.gradient_block_scene(fw, n=64, young=y, seed=rank)  # noqa: E731
    sim = DiffSim(build(), dt, steps, checkpoint_every=K, device=local)
    stream = torch.cuda.Stream()
    sim.native.set_stream(stream.cuda_stream)
    v0 = np.tile(np.array([0.0, -2.0], np.float32), (sim.N, 1))
    target = sim.forward(sim.E0 * 1.1, v0).astype(np.float64)
    for _ in range(args.warmup):
        x = sim.forward(sim.E0, v0)
        sim.backward(2.0 * (x - target))
    barrier(dist)
    l0 = sim.native.launch_count()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    walls = []
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB > L2
    with ClockSampler(local) as clk:
        for a, b, c in ev:
            with torch.cuda.stream(stream):
                flush.zero_()  # between timed iterations, on the stream the rollout runs on
            w0 = time.perf_counter()
            a.record(stream)
            x = sim.forward(sim.E0, v0)
            b.record(stream)
            eb, vb, _ = sim.backward(2.0 * (x - target))
            c.record(stream)
            walls.append(time.perf_counter() - w0)
        torch.cuda.synchronize()
    launches = sim.native.launch_count() - l0
    barrier(dist)
    fwd_ms = [a.elapsed_time(b) for a, b, _ in ev]
    bwd_ms = [b.elapsed_time(c) for _, b, c in ev]
    evals, ms = shard.aggregate(args.steps, float(np.sum(fwd_ms) + np.sum(bwd_ms)))
    per_eval_s = ms / 1e3 / evals
    # dot-product test at full size: adjoint of L = <w, x_T> against the tangent
    rng_t = np.random.default_rng(77)
    w = rng_t.standard_normal((sim.N, 2))
    sim.forward(sim.E0, v0)
    eb_w, vb_w, _ = sim.backward(w)
    dot = []
    for _ in range(2):
        dE = (sim.E0 * rng_t.standard_normal(sim.E)).astype(np.float32)
        dv = rng_t.standard_normal((sim.N, 2)).astype(np.float32)
        _, dx = sim.jvp(sim.E0, v0, dE, dv)
        a_e, a_v = float(np.dot(eb_w.astype(np.float64), dE)), float(np.sum(vb_w.astype(np.float64) * dv))
        dot.append(abs(float(np.sum(w * dx.astype(np.float64))) - a_e - a_v) / (abs(a_e) + abs(a_v)))
    # the block must reach the plane: minimum height over the forward rollout
    probe = fw.ExplicitLoop(dt, build(), useAdapativeDT=False, path="gather", device=local)
    low = 1e9
    for _ in range(steps // 100):
        probe.advance_n(100)
        low = min(low, float(probe.femSpringManager.coords.numpy()[: sim.N, 1].min()))
    line = {
        "metric": "gradient evaluations/s (forward + adjoint rollout)", "value": 1.0 / per_eval_s,
        "unit": "gradients/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (adjoint accumulators f64)", "data": "synthetic (seeded moduli)",
        "config": {"workload": "differentiable 64x64-quad NeoHookean block, 2000 substeps dt 1e-4, K=50",
                   "elements": sim.E, "nodes": sim.N, "substeps": steps, "checkpoint_every": K,
                   "min_height_m": low, "contact": bool(low < 0.0),
                   "l2": "flushed between rollouts (256 MiB write)"},
        "adjoint": {"forward_ms": float(np.median(fwd_ms)), "backward_ms": float(np.median(bwd_ms)),
                    "forward_element_steps_per_s": sim.E * steps / (np.median(fwd_ms) / 1e3),
                    "backward_over_forward": float(np.median(bwd_ms) / np.median(fwd_ms)),
                    "dot_product_test_max_rel": max(dot)},
        "e2e": {"value": args.steps / float(np.sum(walls)), "unit": "gradients/s",
                "h2d_bytes_per_step": sim.N * 8 * 2 + sim.E * 4, "d2h_bytes_per_step": sim.N * 8 * 2 + sim.E * 4},
        "gpu_launches": launches, "clocks": clk.summary(),
    }
    if not args.no_cpu_baseline and rank == 0:
        import oracle

        threads = os.cpu_count() or 1
        o = oracle.OracleLoop(build(), dt, useAdapativeDT=False, precision="f64", threads=threads)
        o.set_state(None, v0)
        o.advance(steps)
        x64 = o.state()[0]
        sim.forward(sim.E0, v0)
        eb64, vb64, _ = sim.backward(2.0 * (x64 - target))
        sim.forward(sim.E0, v0)
        eb32, vb32, _ = sim.backward(2.0 * (sim.native.read_nodes(0, 0, sim.N) - target))
        t_roll, errs = fd_check(fw, build, sim, v0, steps, dt, target, eb32, vb32, eb64, vb64,
                                args.fd_directions, threads)
        n_params = sim.E + 2 * sim.N
        line["cpu_baseline"] = {"value": 1.0 / (2 * n_params * t_roll), "unit": "gradients/s", "cores": threads,
                                "kind": "port",
                                "sample": f"{2 * args.fd_directions} FP64 oracle rollouts of the workload "
                                          f"({t_roll:.3f} s each); a full gradient by central differences "
                                          f"takes 2 x {n_params} of them"}
        line["fd_check"] = {
            "directions": args.fd_directions, "eps": 1e-4,
            "max_rel_err_dE": max((e[0] for e in errs["E"]), default=None),
            "max_rel_err_dv0": max((e[0] for e in errs["v"]), default=None),
            "max_rel_err_dE_fp64_seed": max((e[1] for e in errs["E"]), default=None),
            "max_rel_err_dv0_fp64_seed": max((e[1] for e in errs["v"]), default=None),
            "median_rel_err": float(np.median([e[0] for k in errs for e in errs[k]]))}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def run_flex(args, rank, world, local):
    """FEM-FEM contact: a pile of --flex-side^2 touching disks (16 x 16
    mapped-grid cells, alternately Elastic / NeoHookean, E 1e5, rho 1000,
    friction 0.2) settling under gravity on a ground plane; every pair of disks
    is a FEM-FEM contact pair (broad-phase gated), plus each disk's plane
    contact.  dt = 0.5 x the loop's adaptive dt (at the adaptive dt itself the
    disks diverge on landing, in the oracle too).  A step is 100 substeps."""
    import torch

    import flatworld_b200 as fw
    from flatworld_b200.world import SceneLayout
    from tests import scenes

    torch.cuda.set_device(local)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB > L2
    dist = dist_init(world, local)
    side = args.flex_side
    build = lambda: scenes.flex_pile(fw, side, side, gap=0.0)  # noqa: E731  (touching: contact from the start)
    dt = 0.5 * SceneLayout(build(), useAdapativeDT=True).dt
    t0 = time.perf_counter()
    loop = fw.ExplicitLoop(dt, build(), useAdapativeDT=False, device=local)
    build_s = time.perf_counter() - t0
    stream = torch.cuda.Stream()
    loop._native.set_stream(stream.cuda_stream)
    pk = loop._packed
    N, E = pk.N, pk.E
    n_items = flex_work_items(pk)
    per = 100
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            loop.advance_n(per)
        torch.cuda.synchronize()
        barrier(dist)
        l0 = loop.launch_count()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        with ClockSampler(local) as clk:
            for s_, e_ in ev:
                flush.zero_()
                s_.record(stream)
                loop.advance_n(per)
                e_.record(stream)
            torch.cuda.synchronize()
        launches = loop.launch_count() - l0
        cache, _ = loop._native.read_flex_state(n_items)
        in_contact = int((cache >= 0).sum())
        x_mid = loop.femSpringManager.coords.numpy()[:N].copy()
        v_mid = loop.femSpringManager.V.numpy()[:N].copy()
        # ---- end to end: positions and velocities in from pinned host memory, a step, and out
        xh = torch.empty((N, 2), dtype=torch.float32, pin_memory=True)
        vh = torch.empty((N, 2), dtype=torch.float32, pin_memory=True)
        loop._native.read_nodes_ptr(0, 0, N, xh.data_ptr())
        loop._native.read_nodes_ptr(1, 0, N, vh.data_ptr())
        ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for s_, e_ in ev2:
            flush.zero_()
            s_.record(stream)
            loop._native.write_nodes_ptr(0, 0, N, xh.data_ptr())
            loop._native.write_nodes_ptr(1, 0, N, vh.data_ptr())
            loop.advance_n(per)
            loop._native.read_nodes_ptr(0, 0, N, xh.data_ptr())
            loop._native.read_nodes_ptr(1, 0, N, vh.data_ptr())
            e_.record(stream)
        torch.cuda.synchronize()
    barrier(dist)
    lat = [s_.elapsed_time(e_) for s_, e_ in ev]
    work, ms = shard.aggregate(E * per * args.steps, float(sum(lat)))
    work_e2e, ms_e2e = shard.aggregate(E * per * args.steps, float(sum(s_.elapsed_time(e_) for s_, e_ in ev2)))
    finite = bool(np.isfinite(loop.femSpringManager.coords.numpy()[:N]).all())
    value = work / (ms / 1e3)
    nb_plane = int(sum(pk.bncnt))
    bstep = algorithmic_bytes_per_substep(N, E, 0, nb_plane + n_items, 0)
    achieved = bstep / (ms / 1e3 / (per * args.steps)) / 1e9
    peak, which = peaks()
    line = {
        "metric": "FEM element-steps/s (FEM-FEM contact pile)", "value": value, "unit": "element-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded pile of disks)",
        "config": {"workload": f"pile of {side * side} touching disks with FEM-FEM contact on a plane, dt 0.5 x adaptive",
                   "elements": E, "nodes": N, "bodies": side * side, "flex_pairs": side * side * (side * side - 1) // 2,
                   "flex_work_items": n_items, "items_with_contact_at_end": in_contact, "dt": dt,
                   "step": "100 substeps", "l2": "flushed between steps (256 MiB write)",
                   "host_build_s": build_s, "state_finite": finite, "replicas": world, "path": "gather"},
        "latency_ms_per_step": {"p50": percentile_ms(lat, 50), "p99": percentile_ms(lat, 99)},
        "roofline": {"bound": "hbm", "kernel": "substep = k_flex_pre + k_flex_contact + k_elements + k_nodes_flex",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": which,
                     "algorithmic_bytes_per_substep": bstep, "traffic": None,
                     "note": "latency-bound: a substep is 4 dependent launches over a world of ~1 MB of state"},
        "e2e": {"value": work_e2e / (ms_e2e / 1e3), "unit": "element-steps/s",
                "h2d_bytes_per_step": 2 * N * 8, "d2h_bytes_per_step": 2 * N * 8},
        "gpu_launches": launches, "clocks": clk.summary(),
    }
    if rank == 0 and not args.no_cpu_baseline:
        import oracle

        threads = os.cpu_count() or 1
        o = oracle.OracleLoop(build(), dt=dt, useAdapativeDT=False, precision="f32", threads=threads)
        o.set_state(x_mid, v_mid)  # the same landed state the GPU was timed on
        o.advance(1)
        o._L.or_flex_rebuild(o._w)  # its spatial hash from that state, too
        t1 = time.perf_counter()
        o.advance(500)
        t_cpu = time.perf_counter() - t1
        line["cpu_baseline"] = {"value": E * 500 / t_cpu, "unit": "element-steps/s", "cores": threads, "kind": "port",
                                "sample": f"500 substeps of the same pile from the GPU's timed state, FP32 C "
                                          f"restatement ({threads} threads for the element / node work, FEM-FEM "
                                          f"contact serial as in the reference's CPU device)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def run_rigid(args, rank, world, local):
    """FEM-rigid contact: a NeoHookean slab of --rigid-mesh x --rigid-mesh/4
    quads on a ground plane, with 12 BC-driven ball / box / capsule rigids
    pressing into its top (tests/scenes.py rigid_row): per substep the plane
    items, 12 x (slab boundary nodes) FEM-rigid items with their reactions,
    and the rigid update every max(1, 1e-3 // dt) substeps.  Adaptive dt; a
    step is 100 substeps."""
    import torch

    import flatworld_b200 as fw
    from tests import scenes

    torch.cuda.set_device(local)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB > L2
    dist = dist_init(world, local)
    nx = args.rigid_mesh
    build = lambda: scenes.rigid_row(fw, nx, max(4, nx // 4))  # noqa: E731
    t0 = time.perf_counter()
    loop = fw.ExplicitLoop(0.0, build(), useAdapativeDT=True, device=local)
    build_s = time.perf_counter() - t0
    stream = torch.cuda.Stream()
    loop._native.set_stream(stream.cuda_stream)
    pk = loop._packed
    N, E = pk.N, pk.E
    n_rigid = len(loop._layout.rigids)
    n_items = n_rigid * int(pk.bncnt[0])
    dt = loop.dt
    per = 100
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            loop.advance_n(per)
        torch.cuda.synchronize()
        barrier(dist)
        l0 = loop.launch_count()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        with ClockSampler(local) as clk:
            for s_, e_ in ev:
                flush.zero_()
                s_.record(stream)
                loop.advance_n(per)
                e_.record(stream)
            torch.cuda.synchronize()
        launches = loop.launch_count() - l0
        # ---- end to end: positions and velocities in from pinned host memory, a step, and out
        xh = torch.empty((N, 2), dtype=torch.float32, pin_memory=True)
        vh = torch.empty((N, 2), dtype=torch.float32, pin_memory=True)
        loop._native.read_nodes_ptr(0, 0, N, xh.data_ptr())
        loop._native.read_nodes_ptr(1, 0, N, vh.data_ptr())
        ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for s_, e_ in ev2:
            flush.zero_()
            s_.record(stream)
            loop._native.write_nodes_ptr(0, 0, N, xh.data_ptr())
            loop._native.write_nodes_ptr(1, 0, N, vh.data_ptr())
            loop.advance_n(per)
            loop._native.read_nodes_ptr(0, 0, N, xh.data_ptr())
            loop._native.read_nodes_ptr(1, 0, N, vh.data_ptr())
            e_.record(stream)
        torch.cuda.synchronize()
    barrier(dist)
    loop.synchronize()  # raises if a rigid met the ground or another rigid
    rig = loop._rigid_state()
    lat = [s_.elapsed_time(e_) for s_, e_ in ev]
    work, ms = shard.aggregate(E * per * args.steps, float(sum(lat)))
    work_e2e, ms_e2e = shard.aggregate(E * per * args.steps, float(sum(s_.elapsed_time(e_) for s_, e_ in ev2)))
    finite = bool(np.isfinite(loop.femSpringManager.coords.numpy()[:N]).all())
    value = work / (ms / 1e3)
    bstep = algorithmic_bytes_per_substep(N, E, 0, int(pk.bncnt[0]) + n_items, 0)
    achieved = bstep / (ms / 1e3 / (per * args.steps)) / 1e9
    peak, which = peaks()
    line = {
        "metric": "FEM element-steps/s (FEM-rigid contact)", "value": value, "unit": "element-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (slab and a row of rigid primitives)",
        "config": {"workload": f"NeoHookean slab {nx}x{max(4, nx // 4)} quads on a plane, 12 BC-driven "
                               f"ball / box / capsule rigids pressing into it",
                   "elements": E, "nodes": N, "rigids": n_rigid, "rigid_work_items": n_items, "dt": dt,
                   "rigid_update_every": int(max(1, 1e-3 // dt)), "step": "100 substeps",
                   "l2": "flushed between steps (256 MiB write)", "host_build_s": build_s, "state_finite": finite,
                   "rigid_x_range_at_end": [float(rig[:, 0].min()), float(rig[:, 0].max())],
                   "replicas": world, "path": "gather"},
        "latency_ms_per_step": {"p50": percentile_ms(lat, 50), "p99": percentile_ms(lat, 99)},
        "roofline": {"bound": "hbm", "kernel": "substep = k_elements + k_nodes_rigid + k_rigid",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": which,
                     "algorithmic_bytes_per_substep": bstep, "traffic": None,
                     "note": "latency-bound: 3 dependent launches per substep over ~1 MB of state"},
        "e2e": {"value": work_e2e / (ms_e2e / 1e3), "unit": "element-steps/s",
                "h2d_bytes_per_step": 2 * N * 8, "d2h_bytes_per_step": 2 * N * 8},
        "gpu_launches": launches, "clocks": clk.summary(),
    }
    if rank == 0 and not args.no_cpu_baseline:
        import oracle

        threads = os.cpu_count() or 1
        o = oracle.OracleLoop(build(), useAdapativeDT=True, precision="f32", threads=threads)
        o.advance(20)
        t1 = time.perf_counter()
        n_cpu = 3000
        o.advance(n_cpu)
        t_cpu = time.perf_counter() - t1
        line["cpu_baseline"] = {"value": E * n_cpu / t_cpu, "unit": "element-steps/s", "cores": threads,
                                "kind": "port",
                                "sample": f"{n_cpu} substeps of the same scene, FP32 C restatement ({threads} "
                                          f"threads for the element / node work, FEM-rigid contact and the "
                                          f"rigid update serial as in the reference's CPU device)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def run_rigid_batched(args, rank, world, local):
    """FEM-rigid contact, batched: --rigid-scenes independent scenes of the
    rigid workload at 32 x 8 quads (a slab with 12 BC-driven rigids, balls at
    0.01 m/s) in one
    BatchedLoop, each scene with its own rigid clock; a step is 100 substeps
    at the scene's adaptive dt.  Baseline: the same scene stepped alone in an
    ExplicitLoop (the reference runs one loop per scene)."""
    import torch

    import flatworld_b200 as fw
    from flatworld_b200.batch import BatchedLoop
    from flatworld_b200.world import SceneLayout
    from tests import scenes

    torch.cuda.set_device(local)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB > L2
    dist = dist_init(world, local)
    build = lambda: scenes.rigid_row(fw, 32, 8, ball_speed=0.01)  # noqa: E731  (clearances last the whole run)
    dt = SceneLayout(build(), useAdapativeDT=True).dt
    K = args.rigid_scenes
    t0 = time.perf_counter()
    b = BatchedLoop([build() for _ in range(K)], dt=dt, useAdapativeDT=False, device=local)
    build_s = time.perf_counter() - t0
    stream = torch.cuda.Stream()
    b.set_stream(stream.cuda_stream)
    per = 100
    E = b.n_elems
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            b.advance(per)
        torch.cuda.synchronize()
        barrier(dist)
        l0 = b.launch_count()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        with ClockSampler(local) as clk:
            for s_, e_ in ev:
                flush.zero_()
                s_.record(stream)
                b.advance(per)
                e_.record(stream)
            torch.cuda.synchronize()
        launches = b.launch_count() - l0
        lp = fw.ExplicitLoop(dt, build(), useAdapativeDT=False, device=local)
        lp._native.set_stream(stream.cuda_stream)
        for _ in range(args.warmup):
            lp.advance_n(per)
        a_, z_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a_.record(stream)
        for _ in range(args.steps):
            lp.advance_n(per)
        z_.record(stream)
        torch.cuda.synchronize()
    barrier(dist)
    b.synchronize()  # raises if a rigid met a ground or another rigid
    work, ms = shard.aggregate(E * per * args.steps, float(sum(s_.elapsed_time(e_) for s_, e_ in ev)))
    e_one = lp._packed.E
    plain_value = e_one * per * args.steps / (a_.elapsed_time(z_) / 1e3)
    value = work / (ms / 1e3)
    line = {
        "metric": "FEM element-steps/s (batched FEM-rigid contact scenes)", "value": value,
        "unit": "element-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (slabs and rows of rigid primitives)",
        "config": {"workload": f"{K} slabs of 32 x 8 quads with 12 BC-driven rigids each, FEM-rigid contact",
                   "elements": E, "scenes": K, "rigids": 12 * K, "dt": dt, "step": "100 substeps", "l2": "flushed between steps (256 MiB write)",
                   "host_build_s": build_s, "path": "gather",
                   "state_finite": bool(np.isfinite(b.all_coords()).all())},
        "batched_vs_plain": {"plain_value": plain_value, "ratio": value / plain_value,
                             "plain": "the same scene alone in an ExplicitLoop"},
        "gpu_launches": launches, "clocks": clk.summary(),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def run_flex_batched(args, rank, world, local):
    """FEM-FEM contact, batched: --flex-scenes independent piles of 3 x 3
    touching disks (as the flex workload) in one BatchedLoop, each scene with
    its own spatial hash; a step is 100 substeps at 0.5 x the adaptive dt.
    Baseline: the same pile stepped alone in an ExplicitLoop (the reference
    runs one loop per scene)."""
    import torch

    import flatworld_b200 as fw
    from flatworld_b200.batch import BatchedLoop
    from flatworld_b200.world import SceneLayout
    from tests import scenes

    torch.cuda.set_device(local)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB > L2
    dist = dist_init(world, local)
    build = lambda: scenes.flex_pile(fw, 3, 3, gap=0.0)  # noqa: E731
    dt = 0.5 * SceneLayout(build(), useAdapativeDT=True).dt
    K = args.flex_scenes
    t0 = time.perf_counter()
    b = BatchedLoop([build() for _ in range(K)], dt=dt, useAdapativeDT=False, device=local)
    build_s = time.perf_counter() - t0
    stream = torch.cuda.Stream()
    b.set_stream(stream.cuda_stream)
    per = 100
    E = b.n_elems
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            b.advance(per)
        torch.cuda.synchronize()
        barrier(dist)
        l0 = b.launch_count()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        with ClockSampler(local) as clk:
            for s_, e_ in ev:
                flush.zero_()
                s_.record(stream)
                b.advance(per)
                e_.record(stream)
            torch.cuda.synchronize()
        launches = b.launch_count() - l0
        lp = fw.ExplicitLoop(dt, build(), useAdapativeDT=False, device=local)
        lp._native.set_stream(stream.cuda_stream)
        for _ in range(args.warmup):
            lp.advance_n(per)
        a_, z_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a_.record(stream)
        for _ in range(args.steps):
            lp.advance_n(per)
        z_.record(stream)
        torch.cuda.synchronize()
    barrier(dist)
    work, ms = shard.aggregate(E * per * args.steps, float(sum(s_.elapsed_time(e_) for s_, e_ in ev)))
    e_one = lp._packed.E
    plain_value = e_one * per * args.steps / (a_.elapsed_time(z_) / 1e3)
    value = work / (ms / 1e3)
    line = {
        "metric": "FEM element-steps/s (batched FEM-FEM contact scenes)", "value": value, "unit": "element-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded piles of disks)",
        "config": {"workload": f"{K} piles of 3 x 3 touching disks, FEM-FEM contact, dt 0.5 x adaptive",
                   "elements": E, "scenes": K, "step": "100 substeps", "l2": "flushed between steps (256 MiB write)", "host_build_s": build_s, "path": "gather",
                   "state_finite": bool(np.isfinite(b.all_coords()).all())},
        "batched_vs_plain": {"plain_value": plain_value, "ratio": value / plain_value,
                             "plain": "the same pile alone in an ExplicitLoop"},
        "gpu_launches": launches, "clocks": clk.summary(),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload == "batched":
        run_batched(args, rank, world, local)
        return
    if args.workload == "served":
        run_served(args, rank, world, local)
        return
    if args.workload == "adjoint":
        run_adjoint(args, rank, world, local)
        return
    if args.workload == "rigid":
        if args.rigid_scenes > 1:
            run_rigid_batched(args, rank, world, local)
        else:
            run_rigid(args, rank, world, local)
        return
    if args.workload == "flex":
        if args.flex_scenes > 1:
            run_flex_batched(args, rank, world, local)
        else:
            run_flex(args, rank, world, local)
        return
    import torch

    import flatworld_b200 as fw
    from flatworld_b200.world import substep_schedule

    torch.cuda.set_device(local)
    dist = dist_init(world, local)
    domains = workload(fw, args.mesh)
    loop = fw.ExplicitLoop(0.0, domains, useAdapativeDT=True, device=local)
    stream = torch.cuda.Stream()
    loop._native.set_stream(stream.cuda_stream)
    fsm = loop.femSpringManager
    N = int(fsm.totalNodes.numpy()[0])
    E = int(fsm.totalElements.numpy()[0])
    runs = substep_schedule(FRAME, loop.stableTime, loop.default_dt, True)
    substeps = sum(n for n, _ in runs)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            flush.zero_()
            loop.advanceWithTime(FRAME)
        barrier(dist)
        launches0 = loop.launch_count()
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        with ClockSampler(local) as clk:
            for k in range(args.steps):
                flush.zero_()
                starts[k].record(stream)
                loop.advanceWithTime(FRAME)
                ends[k].record(stream)
            torch.cuda.synchronize()
        barrier(dist)
        launches = loop.launch_count() - launches0
        ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
        # ---- end to end: host state in, one frame, host state out (pinned)
        xh = torch.empty((N, 2), dtype=torch.float32, pin_memory=True)
        vh = torch.empty((N, 2), dtype=torch.float32, pin_memory=True)
        loop._native.read_nodes_ptr(0, 0, N, xh.data_ptr())
        loop._native.read_nodes_ptr(1, 0, N, vh.data_ptr())
        e_s = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        e_e = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        for k in range(args.steps):
            flush.zero_()
            e_s[k].record(stream)
            loop._native.write_nodes_ptr(0, 0, N, xh.data_ptr())
            loop._native.write_nodes_ptr(1, 0, N, vh.data_ptr())
            loop.advanceWithTime(FRAME)
            loop._native.read_nodes_ptr(0, 0, N, xh.data_ptr())
            loop._native.read_nodes_ptr(1, 0, N, vh.data_ptr())
            e_e[k].record(stream)
        torch.cuda.synchronize()
        ms_e2e = sum(s.elapsed_time(e) for s, e in zip(e_s, e_e))
    t = torch.tensor([ms, ms_e2e], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms, ms_e2e = float(t[0]), float(t[1])
    if rank == 0:
        work = world * E * substeps * args.steps
        value = work / (ms / 1e3)
        e2e = work / (ms_e2e / 1e3)
        nb = sum(d.mesh.numBoundNodes for d in loop._layout.fem)
        ground = sum(4 * c.ground.nx for c in loop._layout.pairs if c.kind == "heightfield")
        bstep = algorithmic_bytes_per_substep(N, E, 0, nb * len(loop._layout.pairs), ground)
        per_sub_s = (ms / 1e3) / (substeps * args.steps)
        achieved = bstep / per_sub_s / 1e9
        peak, which = peaks()
        traffic = ncu_traffic()
        line = {
            "metric": "FEM element-steps/s", "value": value, "unit": "element-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded mesh, velocities and height field)",
            "config": {"workload": f"plain large single mesh {args.mesh}x{args.mesh} quads, NeoHookean, "
                                   f"height field 4096 samples",
                       "elements": E, "nodes": N, "step": "advanceWithTime(1/60)",
                       "substeps_per_step": substeps, "dt": loop.stableTime,
                       "l2": "flushed between steps (256 MiB write)", "replicas": world,
                       "path": {1: "gather", 2: "resident"}.get(loop.path, loop.path), "patches": loop.patches,
                       "front_warps": loop._native.get_option(_native.FW_OPT_FRONT_WARPS) if loop.path == 2 else None},
            "roofline": {"bound": "hbm",
                         "kernel": "k_resident (all substeps of a step)" if loop.path == 2 else
                                   "substep = k_elements + k_nodes",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": which, "algorithmic_bytes_per_substep": bstep,
                         "us_per_substep": per_sub_s * 1e6,
                         "traffic": traffic,
                         "traffic_from": "profiles/traffic_plain_large.json (ncu capture of this workload, "
                                         "committed; not measured in this run)"},
            "e2e": {"value": e2e, "unit": "element-steps/s", "h2d_bytes_per_step": 2 * N * 8,
                    "d2h_bytes_per_step": 2 * N * 8},
            "gpu_launches": launches,
            "clocks": clk.summary(),
            "energy_fp64": loop.energy(),
        }
        if not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            rate, n = cpu_oracle_rate(fw, args.mesh, args.cpu_seconds, threads)
            rate1, n1 = cpu_oracle_rate(fw, args.mesh, args.cpu_seconds / 2, 1)
            line["cpu_baseline"] = {"value": rate, "unit": "element-steps/s", "cores": threads, "kind": "port",
                                    "sample": f"{n} substeps of the same workload, FP32 C restatement of the "
                                              f"reference scheme, {threads} threads",
                                    "one_thread": {"value": rate1, "sample": f"{n1} substeps, 1 thread"}}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
