"""Served form (GPU): continuous batching over an arena of resident bodies.

Each body's result after its requests must be bit-identical to running the
same requests alone, one ExplicitLoop per body; bodies admitted, removed and
re-admitted reuse arena ranges correctly."""

import numpy as np
import pytest

import flatworld_b200 as fw
from flatworld_b200.serve import Arena, FifoPlainServer, Request, Server, poisson_requests, request_substeps
from flatworld_b200.world import substep_schedule
from tests import scenes

pytestmark = pytest.mark.gpu
FRAME = 1.0 / 60.0


def small_body(i):
    rng = np.random.default_rng([99, i])
    while True:
        sc = scenes.ragged_body_scene(fw, rng, i)
        if sc[1].nnodes <= 2500:
            return sc


def alone(body, reqs):
    lp = fw.ExplicitLoop(0.0, small_body(body), useAdapativeDT=False, path="gather")
    for r in reqs:
        lp.default_dt = FRAME / request_substeps(r, FRAME, lp.stableTime)
        lp.advanceWithTime(FRAME)
    return lp.femSpringManager.coords.numpy()[: lp._packed.N], lp.femSpringManager.V.numpy()[: lp._packed.N]


def test_served_results_equal_alone():
    reqs = poisson_requests(rate=400.0, duration=0.1, n_bodies=6, seed=3, substeps=(20, 60))
    assert len(reqs) >= 20
    srv = Server(small_body, arena_nodes=60_000, arena_elems=120_000, arena_bodies=64, arena_scenes=64)
    out = srv.run(reqs, realtime=False)
    assert len(out["latency_s"]) == len(reqs)
    for body in sorted({r.body for r in reqs}):
        mine = [r for r in reqs if r.body == body]
        x, v = alone(body, mine)
        xs = srv.coords(body)
        assert np.isfinite(xs).all()
        assert np.array_equal(xs, x), body
        assert np.array_equal(srv.arena.velocities(srv.resident[body]), v), body


def exploding_body(i):
    """A soft NeoHookean block thrown apart by random 50 m/s nodal velocities:
    its triangles fold over (J <= 0) within a few substeps and the state turns
    non-finite -- the same on the FP32 oracle."""
    conn, coords = fw.structured_rectangle(12, 12, 0.12, 0.12, origin=(0.0, 0.0))
    v0 = np.random.default_rng(5).normal(0.0, 50.0, size=coords.shape)
    ics = [fw.InitialVel([k], v0[k]) for k in range(coords.shape[0])]
    fem = fw.FemDomain(fw.Mesh(2, conn, coords), fw.SolidProp(fw.HyperElastic(1e4, 0.45, 1000.0)), [],
                       initials=ics)
    return [fem]


def test_nonfinite_body_is_evicted_and_others_are_untouched():
    """A body whose state turns NaN is flagged on the device, its requests fail,
    it is removed from the arena, and the other bodies' results are the same
    bits as alone."""
    body_fn = lambda b: exploding_body(b) if b == 4 else small_body(b)  # noqa: E731
    reqs = [Request(0.0, k, k % 5, 40) for k in range(15)]
    srv = Server(body_fn, arena_nodes=60_000, arena_elems=120_000, arena_bodies=64, arena_scenes=64)
    out = srv.run(reqs, realtime=False)
    bad = {r.rid for r in reqs if r.body == 4}
    assert set(out["failed"]) == bad
    assert out["evicted_bodies"] == 1 and 4 not in srv.resident
    for body in range(4):
        x, v = alone(body, [r for r in reqs if r.body == body])
        assert np.array_equal(srv.coords(body), x), body
    # the flag itself, through the C ABI on a plain loop (both step paths)
    for path in ("gather", "resident"):
        lp = fw.ExplicitLoop(0.0, exploding_body(0), useAdapativeDT=True, path=path)
        assert lp._native.scene_status(1)[0] == 0
        lp.advance_n(200)
        assert lp._native.scene_status(1)[0] == 1, path
        lp._native.clear_scene_status(0)
        assert lp._native.scene_status(1)[0] == 0


def test_arena_reuses_ranges_after_remove():
    ar = Arena(40_000, 80_000, 16, 16, 16, 1 << 16, 1 << 20)
    a = ar.insert(small_body(0), dt=5e-5)
    b = ar.insert(small_body(1), dt=5e-5)
    info_a = ar.info(a)
    ar.remove(a)
    c = ar.insert(small_body(0), dt=5e-5)  # same size: first fit takes the freed range
    assert ar.info(c)[0] == info_a[0] and ar.info(c)[2] == info_a[2]
    dts = np.zeros(ar.S, np.float32)
    dts[b] = dts[c] = np.float32(5e-5)
    for _ in range(101):  # 1 construction step + 100 substeps
        ar.native.step_served(dts)
    lp = fw.ExplicitLoop(5e-5, small_body(0), useAdapativeDT=False, path="gather")
    lp.advance_n(100)
    assert np.array_equal(ar.coords(c), lp.femSpringManager.coords.numpy()[: lp._packed.N])


def test_fifo_plain_server_runs():
    reqs = [Request(0.0, 0, 0, 30), Request(0.0, 1, 1, 40), Request(0.0, 2, 0, 25)]
    f = FifoPlainServer(small_body)
    out = f.run(reqs, realtime=False)
    assert out["served"] == 3
    x, _ = alone(0, [reqs[0], reqs[2]])
    assert np.array_equal(f.loops[0].femSpringManager.coords.numpy()[: len(x)], x)
