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
