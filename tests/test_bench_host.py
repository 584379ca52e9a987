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
