"""FEM-FEM penalty contact (the reference's ContactFlexFlex on its spatial-hash
path, flatworld/mixedcontact.py:886-1018).

CPU tests pin the oracle's restatement on the reference's own FEM-FEM scene
(test2D/test_2Dfem_contact.py: two circles pulled together meet and bounce
apart, and pass through each other when contact is off) and check that the
host layout agrees with the oracle's.  GPU tests require the CUDA path to give
the oracle's bits, substep after substep, through spatial-hash rebuilds, the
per-item edge caches, friction, the broad-phase gate and the launch order of
plane / height-field contact around it."""

import numpy as np
import pytest

import flatworld_b200 as fw
import oracle
from flatworld_b200.world import SceneLayout
from tests import scenes

FRAME = 1.0 / 60.0


def _centres(x, n1):
    return x[:n1].mean(axis=0), x[n1:].mean(axis=0)


def test_oracle_circles_meet_and_bounce():
    """test2D/test_2Dfem_contact.py: with contact the circles touch (a work item
    finds an edge) and are pushed apart again; without it they pass through."""
    doms = scenes.flex_circles(fw)
    n1 = doms[0].mesh.numNodes
    o = oracle.OracleLoop(doms, useAdapativeDT=True)
    touched = False
    for f in range(12):
        o.advance_with_time(FRAME)
        touched |= bool((o.flex_cache() >= 0).any())
    x, _, _ = o.state()
    c1, c2 = _centres(x, n1)
    assert touched
    assert c2[1] - c1[1] > 0.2, "the circles must bounce apart"
    free = oracle.OracleLoop(scenes.flex_circles(fw, contact=False), useAdapativeDT=True)
    for f in range(12):
        free.advance_with_time(FRAME)
    x, _, _ = free.state()
    c1, c2 = _centres(x, n1)
    assert c2[1] < c1[1], "without contact the circles pass through each other"


def test_oracle_circles_no_deep_penetration():
    """While they touch, no boundary node of one circle gets deeper than 5% of
    the radius into the other (point-in-polygon depth over the boundary edges)."""
    doms = scenes.flex_circles(fw)
    n1 = doms[0].mesh.numNodes
    o = oracle.OracleLoop(doms, useAdapativeDT=True)
    edges = [oracle.scene.boundary_edges_literal(d.mesh.connectivity) + off
             for d, off in zip(doms, (0, n1))]
    worst = 0.0
    for s in range(int(0.2 / o.dt)):
        o.advance(1)
        x, _, _ = o.state()
        for k, other in ((1, 0), (0, 1)):
            e = edges[other]
            a, b = x[e[:, 0]], x[e[:, 1]]
            d = (b - a) / np.linalg.norm(b - a, axis=1)[:, None]
            nrm = np.stack([d[:, 1], -d[:, 0]], axis=1)
            pts = x[n1:] if k == 1 else x[:n1]
            pen = ((pts[:, None, :] - a[None]) * nrm[None]).sum(-1)  # < 0 inside that edge's half plane
            inside = (pen < 0).all(axis=1)
            if inside.any():
                worst = max(worst, float((-pen.max(axis=1))[inside].max()))
    assert worst < 0.005, worst


def test_oracle_stamp_quirk_one_sided():
    """With the far plane as domain 0, only the items whose target is the second
    circle (FEM-local 1) ever find an edge."""
    doms = scenes.flex_stamp_quirk(fw)
    o = oracle.OracleLoop(doms, useAdapativeDT=True)
    n_b = len(oracle.scene.boundary_nodes_literal(doms[2].mesh.connectivity))
    hit = np.zeros(len(o.flex_cache()), bool)
    for f in range(10):
        o.advance_with_time(FRAME)
        hit |= o.flex_cache() >= 0
    # pair (domain1 = second circle, domain2 = first): items 0..n_b-1 are the first
    # circle's nodes against the second's edges (target FEM-local 1), the rest target FEM-local 0
    n_a = len(hit) - n_b
    assert hit[:n_a].any() and not hit[n_a:].any()


def test_layout_matches_oracle():
    """Stable dt, pair order, penalty and friction of the host layout equal the
    oracle's literal restatement."""
    for build in (scenes.flex_circles, scenes.flex_stack, scenes.flex_blocks):
        lay = SceneLayout(build(fw), useAdapativeDT=True)
        o = oracle.OracleLoop(build(fw), useAdapativeDT=True)
        assert lay.stableTime == o.stableTime
        assert len(lay.flex) == len(o.flex) == 1
        assert np.float32(lay.flex[0].penalty) == np.float32(o.flex[0][3])
        assert lay.skip_bvh == (build is scenes.flex_circles)


@pytest.mark.gpu
@pytest.mark.parametrize("name,frames", [("circles", 24), ("stack", 40), ("stamp-quirk", 16)])
def test_gpu_equals_oracle_frames(name, frames):
    build = {"circles": scenes.flex_circles, "stack": scenes.flex_stack, "stamp-quirk": scenes.flex_stamp_quirk}[name]
    lp = fw.ExplicitLoop(0.0, build(fw), useAdapativeDT=True)
    assert lp.path == 1  # FEM-FEM contact runs on the gather path
    o = oracle.OracleLoop(build(fw), useAdapativeDT=True)
    n = o.N
    touched = False
    for f in range(frames):
        lp.advanceWithTime(FRAME)
        o.advance_with_time(FRAME)
        xo, vo, _ = o.state()
        x = lp.femSpringManager.coords.numpy()[:n].astype(np.float64)
        v = lp.femSpringManager.V.numpy()[:n].astype(np.float64)
        assert np.array_equal(x, xo), (name, f)
        assert np.array_equal(v, vo), (name, f)
        touched |= bool((o.flex_cache() >= 0).any())
    assert touched
    cache, _ = lp._native.read_flex_state(len(o.flex_cache()))
    assert np.array_equal(cache, o.flex_cache())  # every work item's edge cache, too


@pytest.mark.gpu
def test_gpu_equals_oracle_blocks_heightfield():
    """Larger bodies, several hash rebuilds, friction, FEM-FEM contact between a
    height field's and the internal forces; fixed dt 0.3 x the adaptive one."""
    st = oracle.OracleLoop(scenes.flex_blocks(fw), useAdapativeDT=True).dt
    dt = 0.3 * st
    lp = fw.ExplicitLoop(dt, scenes.flex_blocks(fw), useAdapativeDT=False)
    o = oracle.OracleLoop(scenes.flex_blocks(fw), dt=dt, useAdapativeDT=False, threads=4)
    n = o.N
    hits = 0
    for k in range(30):
        lp.advance_n(100)
        o.advance(100)
        xo, vo, _ = o.state()
        assert np.array_equal(lp.femSpringManager.coords.numpy()[:n].astype(np.float64), xo), k
        assert np.array_equal(lp.femSpringManager.V.numpy()[:n].astype(np.float64), vo), k
        hits += int((o.flex_cache() >= 0).sum())
    assert hits > 0


@pytest.mark.gpu
def test_gpu_flex_world_limits():
    """FEM-FEM worlds run on the gather path; the resident path and snapshots
    are refused with a clear error."""
    with pytest.raises(RuntimeError, match="gather path only"):
        fw.ExplicitLoop(0.0, scenes.flex_circles(fw), useAdapativeDT=True, path="resident")
    lp = fw.ExplicitLoop(0.0, scenes.flex_circles(fw), useAdapativeDT=True)
    with pytest.raises(RuntimeError, match="FEM-FEM"):
        lp._native.snapshot(0)


@pytest.mark.gpu
def test_gpu_batched_flex_scenes_equal_alone():
    """FEM-FEM scenes batched with others (each scene its own spatial hash,
    clock and broad phase; per-scene dt schedules): every scene equals the same
    scene in its own loop, frame after frame."""
    from flatworld_b200.batch import BatchedLoop

    builds = [scenes.flex_circles, scenes.flex_stack, scenes.flex_stamp_quirk, scenes.plain_small_scene]
    b = BatchedLoop([f(fw) for f in builds], useAdapativeDT=True)
    assert len(set(np.round(b.dt, 12))) > 1
    alone = [fw.ExplicitLoop(0.0, f(fw), useAdapativeDT=True) for f in builds]
    for frame in range(8):
        b.advanceWithTime(FRAME)
        for s, lp in enumerate(alone):
            lp.advanceWithTime(FRAME)
            n = len(b.coords(s))
            assert np.array_equal(b.coords(s), lp.femSpringManager.coords.numpy()[:n]), (frame, s)


def test_oracle_tied_pair_holds_the_slabs_together():
    """ExplicitLoop(ties=[(0, 1)]): the upper slab slides at 0.2 m/s over the
    cantilever; tied, its bottom face stays on the cantilever's top face
    (within 2 mm); untied, it slides on by more than 5 mm in the same 3000
    substeps."""
    doms = scenes.tied_slabs_scene(fw)
    n_a, n_b = doms[0].mesh.numNodes, doms[1].mesh.numNodes
    out = {}
    for ties in ([(0, 1)], None):
        o = oracle.OracleLoop(scenes.tied_slabs_scene(fw), 1.25e-5, useAdapativeDT=False, ties=ties)
        x0, _, _ = o.state()
        o.advance(3000)
        x, _, _ = o.state()
        out[bool(ties)] = (x0, x)
    x0, x = out[True]
    a_top = np.arange(4, n_a, 5)  # node i * 5 + 4: the cantilever's top row (ny = 4)
    b_bot = n_a + np.arange(0, n_b, 5)  # the upper slab's bottom row
    shift_tied = float(np.abs((x[b_bot, 0] - x0[b_bot, 0]) - (x[a_top[4:13], 0] - x0[a_top[4:13], 0])).max())
    x0u, xu = out[False]
    shift_free = float(((xu[b_bot, 0] - x0u[b_bot, 0]) - (xu[a_top[4:13], 0] - x0u[a_top[4:13], 0])).mean())
    assert shift_tied < 2e-3, shift_tied
    assert shift_free > 5e-3, shift_free


@pytest.mark.gpu
def test_gpu_tied_pairs_equal_oracle():
    """Tied pair plus untied FEM-FEM contact in one loop: the GPU gives the
    oracle's bits every 300 substeps (the ties resolve at the first substep,
    tie forces come before contact forces on every node)."""
    lp = fw.ExplicitLoop(1.25e-5, scenes.tied_slabs_scene(fw), useAdapativeDT=False, ties=[(0, 1)])
    o = oracle.OracleLoop(scenes.tied_slabs_scene(fw), 1.25e-5, useAdapativeDT=False, ties=[(0, 1)])
    n = o.N
    for k in range(10):
        lp.advance_n(300)
        o.advance(300)
        xo, vo, _ = o.state()
        assert np.array_equal(lp.femSpringManager.coords.numpy()[:n].astype(np.float64), xo), k
        assert np.array_equal(lp.femSpringManager.V.numpy()[:n].astype(np.float64), vo), k

