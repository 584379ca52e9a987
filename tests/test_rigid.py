"""Rigid primitives in contact with FEM bodies (RigidBodyDomain with BallRigid /
BoxRigid / CapsuleRigid; the reference's _batched_rigid_prim_kernel,
mixedcontact.py:1026-1115, and RigidManager.substep without a constraint
solve, rigidmanager.py:832-964, 2102-2197).

CPU: the oracle reproduces the reference's FEM-rigid scene
(test2D/test_2Dfemcontact_types.py:26-38: an FEM circle dropped on a fixed
ball stays on it, mean y > 0.2), a free ball is stopped by an FEM block
through the reaction impulses alone, the host's packing of rigids and pairs
equals the oracle's, the FP32 sin/cos is accurate, and scenes outside the
scope are refused.  GPU: the CUDA path gives the oracle's bits for the FEM
nodes and for every rigid's state, frame after frame, and raises when a rigid
meets the ground; batched rigid scenes equal the same scenes alone."""

import numpy as np
import pytest

import flatworld_b200 as fw
import oracle
from flatworld_b200.world import PackedWorld, SceneLayout
from oracle.scene import OracleLoop, sincos32
from tests import scenes

FRAME = 1.0 / 60.0


def test_oracle_sincos_accuracy():
    """The FP32 sin / cos of the rigid rotation (Cody-Waite reduction + Taylor)
    within 2 ulp of 1 on [-8 pi, 8 pi] and exact at 0."""
    xs = np.concatenate([np.linspace(-8 * np.pi, 8 * np.pi, 20001), [0.0, np.pi / 2, -np.pi, 1e-6, -3.0]])
    worst = 0.0
    for x in xs.astype(np.float32):
        s, c = sincos32(float(x))
        worst = max(worst, abs(s - np.sin(np.float64(x))), abs(c - np.cos(np.float64(x))))
    assert worst < 2 * 2.0 ** -23, worst
    assert sincos32(0.0) == (0.0, 1.0)


def test_oracle_fem_rests_on_fixed_ball():
    """test2D/test_2Dfemcontact_types.py:26-38 (60 frames, mean y > 0.2); the
    circle settles on top of the ball (centre about r_ball + r_fem above it)."""
    o = OracleLoop(scenes.rigid_fixed_ball(fw), useAdapativeDT=True)
    for _ in range(60):
        o.advance_with_time(FRAME)
    x, _, _ = o.state()
    st, err = o.rigid_state()
    assert err == 0
    assert np.mean(x[:, 1]) > 0.2
    assert abs(x[:, 1].mean() - (0.3 + 0.15 + 0.05)) < 0.02
    assert np.array_equal(st[0, :2], [np.float32(0.5), np.float32(0.3)])  # FixedAll: the ball never moves


def test_oracle_free_ball_stopped_by_reactions():
    """A free ball (gravity 9.8, spin 3 rad/s) on an FEM block: the FEM-rigid
    reactions stop its fall; it then rattles on the block (undamped penalty
    contact, as in the reference) with its centre about one radius above the
    block's top, and rolls (friction turns its spin into travel)."""
    o = OracleLoop(scenes.rigid_free_ball(fw), useAdapativeDT=True)
    ys = []
    for f in range(60):
        o.advance_with_time(FRAME)
        st, err = o.rigid_state()
        assert err == 0
        if f >= 20:
            ys.append(st[0, 1])
    assert 0.24 < min(ys) and max(ys) < 0.30, (min(ys), max(ys))
    assert abs(st[0, 4]) < 1.0
    assert st[0, 0] < 0.49 and st[0, 2] > 0.5  # rolled to the left, turned


def test_oracle_box_across_two_blocks():
    """One rigid in two pairs: the box rests across both blocks (reactions
    from both), level within a few degrees, clear of the ground."""
    o = OracleLoop(scenes.rigid_shared(fw), useAdapativeDT=True)
    for _ in range(40):
        o.advance_with_time(FRAME)
    st, err = o.rigid_state()
    assert err == 0
    assert abs(st[0, 1] - (0.15 + 0.03)) < 0.01 and abs(st[0, 2]) < 0.1, st[0]


def test_oracle_rigid_bcs():
    """EnforceAcc zeroes the contact impulse (the box moves straight down at
    the enforced acceleration, slowed only by damping); Fixed keeps the capsule
    in place while EnforceRotAcc spins it up (angle near a t^2 / 2)."""
    o = OracleLoop(scenes.rigid_bcs(fw), useAdapativeDT=True, damping=0.5)
    st0, _ = o.rigid_state()
    for _ in range(24):
        o.advance_with_time(FRAME)
    st, err = o.rigid_state()
    assert err == 0
    assert st[1, 0] == st0[1, 0] and st[1, 3] == 0.0 and -0.2 < st[1, 4] < -0.17
    assert np.array_equal(st[2, :2], st0[2, :2])
    assert 0.3 < st[2, 2] < 0.42 and st[2, 5] > 0.0


def test_oracle_flags_unstable_rigid():
    """The same box at 1.5 kg is too light for the rigid update interval (its
    contact frequency times N dt nears 1): it blows up, as the reference's
    scheme would, and the non-finite state is flagged rather than reported."""
    o = OracleLoop(scenes.rigid_shared(fw, mass=1.5), useAdapativeDT=True)
    for _ in range(40):
        o.advance_with_time(FRAME)
    assert o.rigid_state()[1] == 1


def test_oracle_flags_rigid_near_ground():
    """A rigid falling toward the ground plane sets the error flag: rigid-ground
    contact belongs to the constraint solver."""
    doms = scenes.rigid_fixed_ball(fw)
    doms[1] = fw.RigidBodyDomain(fw.BallRigid(2, [0.2, 0.3], 0.05, 1.0), [fw.Gravity([0, -10.0])])
    o = OracleLoop(doms, useAdapativeDT=True)
    for _ in range(30):
        o.advance_with_time(FRAME)
    assert o.rigid_state()[1] == 1


def test_layout_matches_oracle():
    """Stable dt, pair order and penalties, skip_bvh and the rigid records of
    the host equal the oracle's restatement."""
    for build in (scenes.rigid_fixed_ball, scenes.rigid_pusher, scenes.rigid_free_ball):
        lay = SceneLayout(build(fw), useAdapativeDT=True)
        o = OracleLoop(build(fw), useAdapativeDT=True)
        assert lay.stableTime == o.stableTime, build.__name__
        rig = [c for c in lay.pairs if c.kind == "rigid"]
        orc = [c for c in o.contacts if c[0] == 0b110]
        assert len(rig) == len(orc) > 0
        for a, b in zip(rig, orc):
            assert np.float32(a.penalty) == np.float32(b[3])
            assert lay.rigids.index(a.ground) == o.rigids.index(b[2])
        params, ints, grounds = PackedWorld([lay]).rigid_records()
        for k, d in enumerate(lay.rigids):
            f = np.zeros(20, np.float32)
            iv = np.zeros(3, np.int32)
            OracleLoop._pack_rigid(d, f, iv)
            assert np.array_equal(params[k], f) and np.array_equal(ints[k, :3], iv), (build.__name__, k)
        assert grounds.shape == (1, 6) and grounds[0, 0] == 0.0
    # every rigid BC kind, and a moving ground's analytical entries (plane + the
    # entries a height field gets), packed as the oracle packs them
    for doms in (scenes.rigid_bcs(fw), scenes.ground_circle(fw, [fw.EnforceVel([0], [0.1, -0.2])]),
                 scenes.fixed_ground_heightfield(fw, True)):
        lay = SceneLayout(doms, useAdapativeDT=True)
        o = OracleLoop(doms, useAdapativeDT=True)
        params, ints, _ = PackedWorld([lay]).rigid_records()
        assert len(lay.entries) == len(o.entries) == len(params)
        for k, d in enumerate(lay.entries):
            f = np.zeros(20, np.float32)
            iv = np.zeros(3, np.int32)
            (OracleLoop._pack_rigid(d, f, iv) if d.type == fw.DomainType.RIGID else o._pack_analytical(d, f, iv))
            assert np.array_equal(params[k], f) and np.array_equal(ints[k, :3], iv), k
    # FEM + one rigid, no ground: the loop skips the broad phase (plain box test)
    assert SceneLayout([scenes.rigid_fixed_ball(fw)[i] for i in (0, 1)], useAdapativeDT=True).skip_bvh
    assert not SceneLayout(scenes.rigid_fixed_ball(fw), useAdapativeDT=True).skip_bvh


def test_out_of_scope_refused():
    with pytest.raises(NotImplementedError):
        fw.MeshRigid(2, None, 0.0, 1.0)
    with pytest.raises(NotImplementedError):
        fw.RevoluteJoint()
    with pytest.raises(NotImplementedError):
        fw.ExplicitLoop(0.0, scenes.rigid_fixed_ball(fw), considerRigidRigidContact=False)
    from flatworld_b200.diff import DiffSim

    with pytest.raises(NotImplementedError):
        DiffSim(scenes.rigid_fixed_ball(fw), 1e-4, 10)


def _compare(lp, o, n, tag):
    xo, vo, _ = o.state()
    assert np.array_equal(lp.femSpringManager.coords.numpy()[:n].astype(np.float64), xo), tag
    assert np.array_equal(lp.femSpringManager.V.numpy()[:n].astype(np.float64), vo), tag
    st, err = o.rigid_state()
    assert err == 0, tag
    assert np.array_equal(lp._rigid_state().astype(np.float64), st), tag


@pytest.mark.gpu
@pytest.mark.parametrize("name,frames", [("fixed-ball", 40), ("pusher", 14), ("free-ball", 40), ("shared", 30)])
def test_gpu_equals_oracle_frames(name, frames):
    build = {"fixed-ball": scenes.rigid_fixed_ball, "pusher": scenes.rigid_pusher,
             "free-ball": scenes.rigid_free_ball, "shared": scenes.rigid_shared}[name]
    lp = fw.ExplicitLoop(0.0, build(fw), useAdapativeDT=True)
    assert lp.path == 1  # FEM-rigid contact runs on the gather path
    o = oracle.OracleLoop(build(fw), useAdapativeDT=True)
    for f in range(frames):
        lp.advanceWithTime(FRAME)
        o.advance_with_time(FRAME)
        _compare(lp, o, o.N, (name, f))
    lp.synchronize()
    if name == "fixed-ball":
        assert np.mean(lp.femSpringManager.coords.numpy()[:o.N, 1]) > 0.2
    d = lp._layout.rigids[-1]
    assert np.array_equal(d.getCurrentRefPoint(), lp._rigid_state()[-1, :2])


@pytest.mark.gpu
def test_gpu_equals_oracle_bcs_damping():
    """Force, Torque, EnforceAcc, Fixed + EnforceRotAcc and loop damping."""
    lp = fw.ExplicitLoop(0.0, scenes.rigid_bcs(fw), useAdapativeDT=True, damping=0.5)
    o = oracle.OracleLoop(scenes.rigid_bcs(fw), useAdapativeDT=True, damping=0.5)
    for f in range(24):
        lp.advanceWithTime(FRAME)
        o.advance_with_time(FRAME)
        _compare(lp, o, o.N, f)


@pytest.mark.gpu
def test_gpu_batched_rigid_scenes_equal_alone():
    """Scenes with rigids batched with each other and with a plain scene (each
    scene its own rigid clock, counter and clearance check; per-scene dt and
    damping; 42 rigids, more than one block of the rigid kernel holds, so the
    scene updates run from the last warp of each scene): every scene's nodes
    and rigids equal the same scene in its own loop, frame after frame."""
    from flatworld_b200.batch import BatchedLoop

    row = lambda f: scenes.rigid_row(f, 32, 8, ball_speed=0.01)  # noqa: E731  (12 rigids each)
    builds = [scenes.rigid_fixed_ball, scenes.plain_small_scene, scenes.rigid_free_ball, scenes.rigid_bcs,
              scenes.rigid_shared, row, row, row]
    damp = [0.0, 0.0, 0.0, 0.5, 0.0, 0.0, 0.0, 0.0]
    b = BatchedLoop([f(fw) for f in builds], useAdapativeDT=True, damping=damp)
    assert len(set(np.round(b.dt, 12))) > 1
    alone = [fw.ExplicitLoop(0.0, f(fw), useAdapativeDT=True, damping=c) for f, c in zip(builds, damp)]
    for frame in range(10):
        b.advanceWithTime(FRAME)
        for s, lp in enumerate(alone):
            lp.advanceWithTime(FRAME)
            n = len(b.coords(s))
            assert np.array_equal(b.coords(s), lp.femSpringManager.coords.numpy()[:n]), (frame, s)
            if lp._layout.rigids:
                assert np.array_equal(b.rigid_state(s), lp._rigid_state()), (frame, s)


@pytest.mark.gpu
def test_gpu_equals_oracle_fixed_dt_advance():
    """advance() at a fixed dt whose rigid schedule is N = 1e-3 // dt = 6."""
    dt = 1.6e-4
    lp = fw.ExplicitLoop(dt, scenes.rigid_free_ball(fw), useAdapativeDT=False)
    o = oracle.OracleLoop(scenes.rigid_free_ball(fw), dt=dt, useAdapativeDT=False)
    for k in range(8):
        lp.advance_n(97)
        o.advance(97)
        _compare(lp, o, o.N, k)


@pytest.mark.gpu
def test_gpu_rigid_near_ground_raises():
    doms = scenes.rigid_fixed_ball(fw)
    doms[1] = fw.RigidBodyDomain(fw.BallRigid(2, [0.2, 0.3], 0.05, 1.0), [fw.Gravity([0, -10.0])])
    lp = fw.ExplicitLoop(0.0, doms, useAdapativeDT=True)
    for _ in range(30):
        lp.advanceWithTime(FRAME)
    with pytest.raises(RuntimeError, match="rigid"):
        lp.synchronize()
    with pytest.raises(RuntimeError):
        lp._native.snapshot(0)


# ---- ground planes with BCs (the rigid manager's moving analytical entries)

def test_oracle_fixed_ground_equals_static():
    """A ground with Fixed([0]) (common in the reference's example scripts)
    gives the same bits as a static one while the body stays within the
    moving-plane boxes' +-100 span."""
    a = OracleLoop(scenes.ground_circle(fw), useAdapativeDT=True)
    b = OracleLoop(scenes.ground_circle(fw, [fw.Fixed([0])]), useAdapativeDT=True)
    for _ in range(60):
        a.advance_with_time(FRAME)
        b.advance_with_time(FRAME)
    assert np.array_equal(a.state()[0], b.state()[0])
    st, err = b.entry_state()
    assert err == 0 and np.allclose(st[0, 8:12], [-100.0, 0.2, 100.0, 0.4])  # box now +-100 x +-0.1


def test_oracle_moving_plane_moves_gates_not_contact():
    """EnforceVel moves the plane's entry (and its broad-phase box) down at
    0.5 m/s; the contact keeps the plane of construction time, so once the
    box has left the body, the body falls through y = 0.3
    (mixedcontact.py:1815-1818 copy the plane at build time)."""
    m = OracleLoop(scenes.ground_circle(fw, [fw.EnforceVel([0], [0.0, -0.5])]), useAdapativeDT=True)
    for _ in range(30):
        m.advance_with_time(FRAME)
    st, err = m.entry_state()
    assert err == 0 and abs(st[0, 1] - (0.3 - 0.5 * 30 * FRAME)) < 0.02  # whole rigid updates of N dt
    assert m.state()[0][:, 1].min() < 0.25


def test_oracle_fixed_ground_collapses_heightfield_box():
    """With a plane under BCs the height field's entry box becomes the origin
    point after the first update and the circle falls through the bowl onto
    the plane (without the BC it rests in the bowl)."""
    runs = {}
    for fixed in (False, True):
        o = OracleLoop(scenes.fixed_ground_heightfield(fw, fixed), useAdapativeDT=True)
        for _ in range(60):
            o.advance_with_time(FRAME)
        runs[fixed] = o
    assert runs[False].state()[0][:, 1].min() > 0.3
    assert runs[True].state()[0][:, 1].min() < 0.2
    assert np.array_equal(runs[True].entry_state()[0][1, 8:12], [0.0, 0.0, 0.0, 0.0])


@pytest.mark.gpu
@pytest.mark.parametrize("name,frames", [("fixed", 40), ("moving", 30), ("hf", 40)])
def test_gpu_moving_ground_equals_oracle(name, frames):
    build = {"fixed": lambda: scenes.ground_circle(fw, [fw.Fixed([0])]),
             "moving": lambda: scenes.ground_circle(fw, [fw.EnforceVel([0], [0.0, -0.5])]),
             "hf": lambda: scenes.fixed_ground_heightfield(fw, True)}[name]
    lp = fw.ExplicitLoop(0.0, build(), useAdapativeDT=True)
    o = oracle.OracleLoop(build(), useAdapativeDT=True)
    n = o.N
    for f in range(frames):
        lp.advanceWithTime(FRAME)
        o.advance_with_time(FRAME)
        xo, vo, _ = o.state()
        assert np.array_equal(lp.femSpringManager.coords.numpy()[:n].astype(np.float64), xo), (name, f)
        assert np.array_equal(lp.femSpringManager.V.numpy()[:n].astype(np.float64), vo), (name, f)
        assert np.array_equal(lp._entry_state().astype(np.float64), o.entry_state()[0]), (name, f)
    g = lp.domains[0]
    assert np.array_equal(g.getCurrentRefPoint(), lp._entry_state()[0, :2])


# ---- tied FEM-rigid pairs (ExplicitLoop ties=...)

def test_oracle_tied_pair():
    """A tied pair (explicitloop.py:265-270) takes the tied branch of the
    rigid kernel: the node is pulled to its contact point with no 1e-4 offset
    and no friction (mixedcontact.py:1073-1087).  The circle still rests on
    the ball, on a trajectory of its own; negative indices name domains from
    the end, and the host marks the same pair."""
    free = OracleLoop(scenes.rigid_fixed_ball(fw), useAdapativeDT=True)
    tied = OracleLoop(scenes.rigid_fixed_ball(fw), useAdapativeDT=True, ties=[(0, -2)])
    for _ in range(40):
        free.advance_with_time(FRAME)
        tied.advance_with_time(FRAME)
    xf, xt = free.state()[0], tied.state()[0]
    assert not np.array_equal(xf, xt) and xt[:, 1].mean() > 0.45
    lay = SceneLayout(scenes.rigid_fixed_ball(fw), useAdapativeDT=True, ties=[(0, -2)])
    assert [c.tied for c in lay.pairs if c.kind == "rigid"] == [True]
    assert [c.tied for c in SceneLayout(scenes.rigid_fixed_ball(fw), ties=[(0, 2)]).pairs if c.kind == "rigid"] == [False]


@pytest.mark.gpu
@pytest.mark.parametrize("name,ties,frames", [("fixed-ball", [(0, 1)], 30), ("pusher", [(1, 2), (1, 3)], 14)])
def test_gpu_tied_equals_oracle(name, ties, frames):
    build = {"fixed-ball": scenes.rigid_fixed_ball, "pusher": scenes.rigid_pusher}[name]
    lp = fw.ExplicitLoop(0.0, build(fw), useAdapativeDT=True, ties=ties)
    o = oracle.OracleLoop(build(fw), useAdapativeDT=True, ties=ties)
    for f in range(frames):
        lp.advanceWithTime(FRAME)
        o.advance_with_time(FRAME)
        _compare(lp, o, o.N, (name, f))


def test_oracle_spring_net_rests_on_box():
    """Spring-rigid pairs (femcontact.py:243-253): penalty 100 k, stable time
    0.5 sqrt(m / penalty), every spring node a work item; the net lands on the
    fixed box and stays above it, while the ball lands on the FEM block."""
    doms = scenes.rigid_spring_net(fw)
    lay = SceneLayout(doms, useAdapativeDT=True)
    o = OracleLoop(scenes.rigid_spring_net(fw), useAdapativeDT=True)
    assert lay.stableTime == o.stableTime
    assert [c.kind for c in lay.pairs] == ["rigid"] * 4  # block and net, each against box and ball
    for _ in range(30):
        o.advance_with_time(FRAME)
    x, _, _ = o.state()
    n_block = doms[0].nnodes
    assert x[n_block:, 1].min() > 0.41 - 0.01  # the box top is at 0.41
    st, err = o.rigid_state()
    assert err == 0 and abs(st[1, 1] - (0.4 + 0.04)) < 0.01  # the ball on the block top


@pytest.mark.gpu
def test_gpu_spring_rigid_equals_oracle():
    lp = fw.ExplicitLoop(0.0, scenes.rigid_spring_net(fw), useAdapativeDT=True)
    o = oracle.OracleLoop(scenes.rigid_spring_net(fw), useAdapativeDT=True)
    for f in range(24):
        lp.advanceWithTime(FRAME)
        o.advance_with_time(FRAME)
        _compare(lp, o, o.N, f)


