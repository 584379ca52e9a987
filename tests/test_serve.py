"""Served form (GPU): continuous batching over an arena of resident bodies.

Each body's result after its requests must be bit-identical to running the
same requests alone, one ExplicitLoop per body, on both arena step paths
(stream: one CTA per patch of the active scenes; gather); bodies admitted,
removed and re-admitted reuse arena ranges correctly; scenes that sit out
some calls (of odd or even substep counts) keep their state."""

import numpy as np
import pytest

import flatworld_b200 as fw
from flatworld_b200 import _native
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


@pytest.mark.parametrize("path", ["stream", "gather"])
def test_served_results_equal_alone(path):
    reqs = poisson_requests(rate=400.0, duration=0.1, n_bodies=6, seed=3, substeps=(20, 60))
    assert len(reqs) >= 20
    srv = Server(small_body, arena_nodes=60_000, arena_elems=120_000, arena_bodies=64, arena_scenes=64, path=path)
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


@pytest.mark.parametrize("path", ["stream", "gather"])
def test_nonfinite_body_is_evicted_and_others_are_untouched(path):
    """A body whose state turns NaN is flagged on the device, its requests fail,
    it is removed from the arena, and the other bodies' results are the same
    bits as alone."""
    body_fn = lambda b: exploding_body(b) if b == 4 else small_body(b)  # noqa: E731
    reqs = [Request(0.0, k, k % 5, 40) for k in range(15)]
    srv = Server(body_fn, arena_nodes=60_000, arena_elems=120_000, arena_bodies=64, arena_scenes=64, path=path)
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


@pytest.mark.parametrize("path", ["stream", "gather"])
def test_arena_reuses_ranges_after_remove(path):
    ar = Arena(40_000, 80_000, 16, 16, 16, 1 << 16, 1 << 20, path=path)
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


@pytest.mark.parametrize("patch", [64, 128])
def test_stream_arena_idle_scenes_keep_their_state(patch):
    """Three scenes on a stream arena step in calls of odd and even substep
    counts while the others sit out (the active scenes' state is carried back
    into the first buffers after an odd count); each ends bit-identical to
    its own run alone.  The pack of scene 0 is committed twice (a second
    resident copy), as a server re-admits an evicted body."""
    ar = Arena(60_000, 120_000, 16, 16, 16, 1 << 16, 1 << 22, path="stream", stream_patch=patch)
    from flatworld_b200.world import PackedWorld, SceneLayout

    lay = SceneLayout(small_body(0))
    pk = ar.pack(lay, PackedWorld([lay]), pinned=True)
    assert pk.patch_nodes == patch and pk.patches >= (pk.nodes + patch - 1) // patch and pk.patch_elems >= pk.elems
    a = ar.insert_pack(lay, pk)
    b = ar.insert(small_body(1))
    a2 = ar.insert_pack(lay, pk)
    dt = np.float32(5e-5)
    plan = [({a, b, a2}, 1), ({a}, 7), ({b, a2}, 12), ({a, b}, 5), ({a2}, 3), ({a, b, a2}, 8)]
    ran = {a: 0, b: 0, a2: 0}
    for active, n in plan:
        dts = np.zeros(ar.S, np.float32)
        for s_ in active:
            dts[s_] = dt
            ran[s_] += n
        ar.native.step_served_n(dts, n)
    ar.native.synchronize()
    pk.close()
    for s_, body in ((a, 0), (b, 1), (a2, 0)):
        lp = fw.ExplicitLoop(5e-5, small_body(body), useAdapativeDT=False, path="gather")
        lp.advance_n(ran[s_] - 1)  # the first substep of a committed scene is its construction step
        n = lp._packed.N
        assert np.array_equal(ar.coords(s_), lp.femSpringManager.coords.numpy()[:n]), (s_, ran[s_])
        assert np.array_equal(ar.velocities(s_), lp.femSpringManager.V.numpy()[:n]), (s_, ran[s_])
    ar.close()


def test_stream_arena_budgets_equal_separate_calls():
    """fw_step_served_budget: in one call of n substeps each scene runs its
    budget at its dt, then (second segment) its next budget at another dt,
    then sits out (its state carried unchanged between the buffers) -- the
    same bits as running each scene's runs alone, in order."""
    ar = Arena(60_000, 120_000, 16, 16, 16, 1 << 16, 1 << 22, path="stream")
    sc = [ar.insert(small_body(i)) for i in range(3)]
    d1, d2 = np.float32(5e-5), np.float32(3e-5)
    runs = {s_: [] for s_ in sc}  # (substeps, dt) in order, per scene
    plan = (  # n, per scene (budget, budget of the second segment at d2)
        (9, ((9, 0), (4, 5), (1, 0))),
        (16, ((3, 13), (16, 0), (11, 2))),
        (7, ((7, 0), (0, 0), (2, 5))),
        (12, ((1, 11), (12, 0), (12, 0))),
    )
    for n, budgets in plan:
        dts = np.zeros(ar.S, np.float32)
        bud = np.zeros(ar.S, np.int32)
        dt_next = np.zeros(ar.S, np.float32)
        bud_next = np.zeros(ar.S, np.int32)
        for s_, (b1, b2) in zip(sc, budgets):
            if b1:
                dts[s_], bud[s_] = d1, b1
                runs[s_].append((b1, d1))
                if b2:
                    dt_next[s_], bud_next[s_] = d2, b2
                    runs[s_].append((b2, d2))
        ar.native.step_served_budget(dts, bud, n, dt_next, bud_next)
    ar.native.synchronize()
    for s_, body in zip(sc, range(3)):
        lp = fw.ExplicitLoop(5e-5, small_body(body), useAdapativeDT=False, path="gather")
        first = True
        for k, d in runs[s_]:
            k -= 1 if first else 0  # the first substep is the construction step
            first = False
            if k:
                lp.advance_n(k, float(d))
        n = lp._packed.N
        assert np.array_equal(ar.coords(s_), lp.femSpringManager.coords.numpy()[:n]), (s_, runs[s_])
        assert np.array_equal(ar.velocities(s_), lp.femSpringManager.V.numpy()[:n]), (s_, runs[s_])
    gather = Arena(10_000, 20_000, 4, 4, 4, 1, 1, path="gather")
    with pytest.raises(_native.NativeError, match="stream arena"):
        gather.native.step_served_budget(np.zeros(gather.S, np.float32), np.zeros(gather.S, np.int32), 1)
    ar.close()
    gather.close()


def test_fifo_plain_server_runs():
    reqs = [Request(0.0, 0, 0, 30), Request(0.0, 1, 1, 40), Request(0.0, 2, 0, 25)]
    f = FifoPlainServer(small_body)
    out = f.run(reqs, realtime=False)
    assert out["served"] == 3
    x, _ = alone(0, [reqs[0], reqs[2]])
    assert np.array_equal(f.loops[0].femSpringManager.coords.numpy()[: len(x)], x)
