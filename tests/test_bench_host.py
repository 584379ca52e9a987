"""Host-side helpers of bench.py on the CPU (the GPU parts run on a B200):
what they compute from a packed world must keep up with the packing."""

import flatworld_b200 as fw
from flatworld_b200.world import PackedWorld, SceneLayout

import bench
from tests import scenes


def test_flex_work_items_counts_both_bodies_of_every_pair():
    doms = scenes.flex_circles(fw)
    pk = PackedWorld([SceneLayout(doms)])
    # one FEM-FEM pair; each circle's boundary nodes query the other circle
    assert bench.flex_work_items(pk) == int(pk.bncnt[0] + pk.bncnt[1])
    tied = PackedWorld([SceneLayout(scenes.flex_circles(fw), ties=[(0, 1)])])
    assert bench.flex_work_items(tied) == bench.flex_work_items(pk)


def test_algorithmic_bytes_formula():
    assert bench.algorithmic_bytes_per_substep(66049, 131072, 0, 1024, 16384) == 7645220


def test_stream_traffic_record_of_the_tuned_shape():
    """The bench line reports the DRAM traffic ratio captured for the launch
    shape it ran; the autotuner's pick on the 2048-body batch (128-node
    patches, 12 CTAs per SM, per-thread loads) moves at most 1.25x its
    algorithmic bytes, and every captured ratio is at least 1 (a capture
    below the algorithmic bytes would mean the kernel skipped work)."""
    ratio, source = bench.ncu_traffic_ratio_batched("stream", "128/12/loads")
    assert ratio is not None and 1.0 <= ratio <= 1.25
    assert "128/12/loads" in source
    gather, _ = bench.ncu_traffic_ratio_batched("gather")
    assert gather is not None and gather >= 1.0
    import json
    import os
    with open(os.path.join(bench.ROOT, "profiles", "traffic_batched.json")) as f:
        shapes = json.load(f)["stream_shapes"]
    assert all(v >= 1.0 for v in shapes.values())
