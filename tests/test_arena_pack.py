"""Arena packs on the CPU: a scene staged on a staging context (no device)
becomes a pack -- validation, corner lists and, for stream arenas, its
patches -- through the C ABI, with the sizes a stream arena reserves for it,
and staging mistakes are refused with a clear error."""

import numpy as np
import pytest

import flatworld_b200 as fw
from flatworld_b200 import _native
from flatworld_b200.world import PackedWorld, SceneLayout, stage
from tests import scenes


def _layout(i=3):
    return SceneLayout(scenes.ragged_batch_one(fw, i, seed=0))


@pytest.mark.parametrize("patch", [0, 64, 128])
def test_pack_sizes(patch):
    lay = _layout()
    packed = PackedWorld([lay])
    st = _native.NativeWorld.stage()
    stage(st, packed)
    pk = st.arena_pack(patch)
    assert (pk.nodes, pk.elems, pk.bodies) == (packed.N, packed.E, len(packed.noff))
    assert pk.patch_nodes == patch and not pk.pinned
    if patch:
        # each body is cut into ceil(nodes / patch) patches; every triangle
        # touching an owned node is held by that patch (cut triangles twice)
        want = sum((int(n) + patch - 1) // patch for n in packed.ncnt)
        assert pk.patches == want
        assert packed.E <= pk.patch_elems <= 3 * packed.E
    else:
        assert pk.patches == 0 and pk.patch_elems == 0
    assert pk.device_bytes >= 48 * packed.N + 136 * packed.E
    pk.close()
    # the stage was cleared: a second pack without staging is refused
    with pytest.raises(_native.NativeError, match="nothing staged"):
        st.arena_pack(patch)
    st.close()


def test_pack_refuses_bad_input():
    st = _native.NativeWorld.stage()
    lay = _layout()
    stage(st, PackedWorld([lay]))
    with pytest.raises(_native.NativeError, match="patch_nodes must be 0, 64 or 128"):
        st.arena_pack(32)
    st.close()
    st = _native.NativeWorld.stage()
    packed = PackedWorld([lay])
    bad = packed.conn.copy()
    bad[0, 0] = packed.N + 5  # a node id outside the scene
    st.set_nodes(packed.coords, packed.vel, packed.bc_bits, packed.bc_vals)
    st.set_elements(bad, packed.mtype, packed.Ev, packed.nuv, packed.rhov, packed.syv, packed.Hv)
    st.set_bodies(packed.noff, packed.ncnt, packed.eoff, packed.ecnt, packed.bscene, packed.bnoff, packed.bncnt,
                  packed.bnodes)
    st.set_scenes(np.zeros(1, np.float32))
    with pytest.raises(_native.NativeError, match="bad node id"):
        st.arena_pack(64)
    st.close()


def test_stage_context_cannot_be_finalized():
    st = _native.NativeWorld.stage()
    with pytest.raises(_native.NativeError, match="staging context"):
        st.arena_init(100, 100, 1, 1, 1, 1, 1)
    st.close()


def test_options_read_back():
    """fw_get_option reads the launch-shape options back (a staging context
    needs no device), and refuses an option it cannot read."""
    st = _native.NativeWorld.stage()
    assert st.get_option(_native.FW_OPT_FRONT_WARPS) == 6
    assert st.get_option(_native.FW_OPT_RES_THREADS) == 512
    st.set_option(_native.FW_OPT_RES_THREADS, 1024)
    st.set_option(_native.FW_OPT_FRONT_WARPS, 16)
    assert (st.get_option(_native.FW_OPT_RES_THREADS), st.get_option(_native.FW_OPT_FRONT_WARPS)) == (1024, 16)
    st.set_option(_native.FW_OPT_STREAM_PATCH, 128)
    assert (st.get_option(_native.FW_OPT_STREAM_PATCH), st.get_option(_native.FW_OPT_STREAM_MINB)) == (128, 16)
    with pytest.raises(_native.NativeError):
        st.get_option(_native.FW_OPT_WAIT_LIMIT)
    st.close()
