"""Batched form: many independent scenes in one world (GPU).

Each scene's result must be bit-identical to the same scene stepped alone by
the plain path, and to the FP32 oracle; freezing, snapshots and the autotuner
must not change results."""

import numpy as np
import pytest

import flatworld_b200 as fw
import oracle
from flatworld_b200 import autotune
from flatworld_b200.batch import BatchedLoop
from tests import scenes

pytestmark = pytest.mark.gpu
FRAME = 1.0 / 60.0


def small_batch(n=9, seed=7):
    """Ragged scenes capped at ~3000 nodes so the oracle stays quick."""
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < n:
        sc = scenes.ragged_body_scene(fw, rng, len(out))
        if sc[1].nnodes <= 3000:
            out.append(sc)
    return out


@pytest.mark.parametrize("path", ["gather", "stream"])
def test_batched_equals_alone_and_oracle_fixed_dt(path):
    build = lambda: small_batch()  # noqa: E731
    b = BatchedLoop(build(), dt=5e-5, useAdapativeDT=False, path=path)
    b.advance(300)
    alone = build()
    for s, doms in enumerate(alone):
        lp = fw.ExplicitLoop(5e-5, doms, useAdapativeDT=False, path="gather")
        lp.advance_n(300)
        xa = lp.femSpringManager.coords.numpy()[: doms[1].nnodes]
        assert np.array_equal(b.coords(s), xa), s
        assert np.array_equal(b.velocities(s), lp.femSpringManager.V.numpy()[: doms[1].nnodes]), s
    for s in (0, 1, 2):  # one scene per material law
        o = oracle.OracleLoop(build()[s], 5e-5, useAdapativeDT=False, threads=8)
        o.advance(300)
        xo, vo, _ = o.state()
        assert np.array_equal(b.coords(s).astype(np.float64), xo), s
        assert np.array_equal(b.velocities(s).astype(np.float64), vo), s


@pytest.mark.parametrize("path", ["gather", "stream"])
def test_batched_advance_with_time_per_scene_dt(path):
    """Adaptive dt differs per scene: each scene takes its own substeps (the
    reference's own test scenes, each stable at its adaptive dt); finished
    scenes freeze while the others go on."""
    build = lambda: [scenes.hf_disk_scene(fw), scenes.voxel_disk_scene(fw), scenes.plain_small_scene(fw),  # noqa: E731
                     [scenes.two_triangle_square(fw)]]
    b = BatchedLoop(build(), useAdapativeDT=True, path=path)
    assert len(set(np.round(b.dt, 12))) > 1
    for _ in range(2):
        b.advanceWithTime(FRAME)
    for s, doms in enumerate(build()):
        lp = fw.ExplicitLoop(0.0, doms, useAdapativeDT=True, path="gather")
        for _ in range(2):
            lp.advanceWithTime(FRAME)
        n = sum(d.nnodes for d in doms if d.type == fw.DomainType.FEM)
        assert np.isfinite(b.coords(s)).all()
        assert np.array_equal(b.coords(s), lp.femSpringManager.coords.numpy()[:n]), s
        assert b.counters[s] == lp._counter_py


@pytest.mark.parametrize("path", ["gather", "stream"])
def test_snapshot_restore_and_frozen_scenes(path):
    b = BatchedLoop(small_batch(n=4), dt=5e-5, useAdapativeDT=False, path=path)
    b.advance(50)
    b._native.snapshot(3)
    b.advance(60)
    xa = b.all_coords()
    b._native.restore(3)
    b.advance(60)
    assert np.array_equal(xa, b.all_coords())
    frozen = b.coords(1)
    b._set_active([1, 0, 1, 1])
    b.advance(40)
    assert np.array_equal(frozen, b.coords(1))
    assert not np.array_equal(xa[: len(b.coords(0))], b.coords(0))


def test_autotune_keeps_results(tmp_path, monkeypatch):
    monkeypatch.setenv("FLATWORLD_B200_CACHE", str(tmp_path))
    a = BatchedLoop(small_batch(n=5), dt=5e-5, useAdapativeDT=False, path="gather")
    c = BatchedLoop(small_batch(n=5), dt=5e-5, useAdapativeDT=False, path="gather")
    best = autotune.tune_batched(a, blocks=(128, 256), steps=4)
    assert best["block_elems"] in (128, 256) and len(best["candidates"]) == 4
    a.advance(100)
    c.advance(100)
    assert np.array_equal(a.all_coords(), c.all_coords())
    again = autotune.tune_batched(a, blocks=(128, 256), steps=4)
    assert again.get("cached")


def test_stream_young_change_equals_gather():
    """A Young's modulus change mid-run reaches the stream path's patch
    records: both paths give the same bits afterwards."""
    loops = [BatchedLoop(small_batch(n=4), dt=5e-5, useAdapativeDT=False, path=p) for p in ("gather", "stream")]
    rng = np.random.default_rng(3)
    young = None
    for lp in loops:
        lp.advance(50)
        if young is None:
            young = rng.uniform(5e3, 4e4, lp.n_elems).astype(np.float32)
        lp._native.set_element_young(young)
        lp.advance(100)
    assert np.array_equal(loops[0].all_coords(), loops[1].all_coords())
    assert not np.array_equal(loops[0].all_coords(), BatchedLoop(small_batch(n=4), dt=5e-5, useAdapativeDT=False,
                                                                  path="stream").all_coords())
