"""The product's host-side packing (flatworld_b200.world) against the oracle's
literal restatement of the reference's construction loops.  CPU only."""

import numpy as np
import pytest

import flatworld_b200 as fw
import oracle
from flatworld_b200.world import PackedWorld, SceneLayout
from tests import scenes


def _scenes():
    return {
        "plain_small": scenes.plain_small_scene(fw),
        "heightfield": scenes.hf_disk_scene(fw),
        "voxel": scenes.voxel_disk_scene(fw),
        "two_triangles": [scenes.two_triangle_square(fw)],
        "elastic10000": [fw.FemDomain(scenes.elastic10000_mesh(fw, 40), fw.SolidProp(fw.Elastic(2e4, 0.2, 40.0)),
                                      [fw.Gravity([0, -1.0])])],
    }


@pytest.mark.parametrize("name", list(_scenes()))
def test_layout_matches_oracle(name):
    doms = _scenes()[name]
    lay = SceneLayout(doms, dt=0.0, useAdapativeDT=True)
    o = oracle.OracleLoop(doms, 0.0, useAdapativeDT=True)
    assert lay.stableTime == o.stableTime
    assert lay.dt == o.dt
    assert [c.penalty for c in lay.contacts] == [c[3] for c in o.contacts]
    assert [c.stableTime for c in lay.contacts] == [c[4] for c in o.contacts]
    for d, Lc in zip(lay.fem, o.char_len):
        assert d.mesh.charLength == Lc
        assert np.array_equal(np.asarray(d.mesh.boundaryNodes), oracle.boundary_nodes_literal(d.mesh.connectivity))


def test_boundary_edges_first_seen_order():
    conn = np.array([[0, 1, 3], [0, 3, 2], [2, 3, 5], [2, 5, 4]], np.int32)
    coords = np.array([[0, 0], [1, 0], [0, 1], [1, 1], [0, 2], [1, 2]], np.float32)
    m = fw.Mesh(2, conn, coords)
    # dict-order reference result: edges seen once, in insertion order
    from collections import defaultdict
    cnt = defaultdict(int)
    for cell in conn.tolist():
        for i in range(3):
            a, b = cell[i], cell[(i + 1) % 3]
            if (b, a) in cnt:
                cnt[(b, a)] += 1
            else:
                cnt[(a, b)] += 1
    ref = [e for e, c in cnt.items() if c == 1]
    assert [tuple(e) for e in m.boundaryElements.tolist()] == ref


def test_bc_packing_last_value_wins():
    dom = scenes.two_triangle_square(fw, bcs_fn=lambda: [fw.Gravity([0, -1.0]), fw.Force([0, 1], [0, -100.0]),
                                                          fw.Fixed([2, 3]), fw.EnforceVel([1], [0.5, 0.0])])
    pw = PackedWorld([SceneLayout([dom])])
    assert pw.bc_bits.tolist() == [fw.GRAVITY | fw.FORCETYPE, fw.GRAVITY | fw.FORCETYPE | fw.VTYPE,
                                   fw.GRAVITY | fw.UTYPE, fw.GRAVITY | fw.UTYPE]
    assert pw.bc_vals.tolist() == [[0, -100.0], [0.5, 0.0], [0, 0], [0, 0]]


def test_substep_schedule_matches_reference_loop():
    from flatworld_b200.world import substep_schedule
    for stable in (3.0446e-5, 1e-3, 0.0035777, 0.02):
        runs = substep_schedule(1 / 60, stable, 0.0, True)
        remaining, ref = 1 / 60, []
        while remaining > 1e-12:
            sub = max(min(stable, remaining), 1e-8)
            ref.append(sub)
            remaining -= sub
        flat = [d for n, d in runs for _ in range(n)]
        assert flat == ref


def test_unbatched_second_heightfield_drops_hf_contact():
    doms = scenes.hf_disk_scene(fw)
    hf2 = fw.HeightFieldDomain(2, scenes.heightfield_bowl(), lb=[0.0, 0.0], ub=[1.0, 1.0])
    with pytest.warns(RuntimeWarning):
        lay = SceneLayout([doms[0], hf2, doms[1]])
    assert lay.pairs == [] and len(lay.unbatched) == 2


def test_fem_fem_pairs_are_built():
    """Two contact-enabled FEM domains make one ContactFlexFlex pair (domain1 =
    the later one); without ground contact the broad phase is skipped; a pair
    named in ties= is marked tied; considerContact=False makes no pair."""
    a = scenes.two_triangle_square(fw)
    b = scenes.two_triangle_square(fw)
    lay = SceneLayout([a, b])
    assert len(lay.flex) == 1 and lay.flex[0].fem is b and lay.flex[0].ground is a
    assert lay.skip_bvh
    assert not lay.flex[0].tied
    assert SceneLayout([a, b], ties=[(0, 1)]).flex[0].tied
    assert not SceneLayout([a, b], ties=[(0, 2)]).flex[0].tied  # unresolvable entries are ignored
    lay = SceneLayout([fw.FemDomain(a.mesh, a.prop, a.bcs, False), fw.FemDomain(b.mesh, b.prop, b.bcs, False)])
    assert not lay.flex
