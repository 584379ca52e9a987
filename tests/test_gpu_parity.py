"""GPU parity: flatworld_b200 (CUDA, sm_100a) against the CPU oracle.

Bar (from the project's correctness target): node positions and velocities
within 1e-5 relative, L-infinity over nodes, of the FP32 scheme; the distance
to the FP64 oracle is reported.  Where the step uses only IEEE-rounded
operations (+ - * / sqrt floor round) the GPU path is expected to be
bit-identical to the FP32 oracle, and the tests assert equality.  The
NeoHookean log(J) is evaluated by the same IEEE-only method on both sides
(fw_log / or_logf), so NeoHookean runs are bit-identical too; the distance to
an oracle that uses the C library's logf instead is measured in
tests/test_noise_floor.py.
"""

import numpy as np
import pytest

import flatworld_b200 as fw
from flatworld_b200 import _native
import oracle
from tests import scenes

pytestmark = pytest.mark.gpu
RTOL = 1e-5
FRAME = 1.0 / 60.0


@pytest.fixture(params=["gather", "resident", "resident-counter", "stream"])
def path(request):
    """Every step implementation must meet the same bar: the gather path, the
    resident path with either hand-off between CTAs (flag-in-data words, the
    default for <= 8 bodies, or the arrival counter) and the patch-streaming
    path."""
    return request.param


def loop_kw(path):
    """ExplicitLoop keyword arguments for a ``path`` fixture value."""
    if path == "resident-counter":
        return {"path": "resident", "res_sync": 1}
    return {"path": path}


def rel_linf(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(np.abs(b).max(), 1e-30)
    return float(np.abs(a - b).max() / scale)


def gpu_state(loop):
    m = loop.femSpringManager
    n = int(m.totalNodes.numpy()[0])
    return m.coords.numpy()[:n], m.V.numpy()[:n]


def hf_gap(domains, x):
    """Smallest height of a node above the scene's height field (its first
    domain), linear interpolation between samples: negative = penetrating."""
    hf = domains[0]
    h = np.asarray(hf.height, np.float64)
    xs = np.linspace(float(hf.lb[0]), float(hf.ub[0]), len(h))
    return float((np.asarray(x, np.float64)[:, 1] - np.interp(np.asarray(x, np.float64)[:, 0], xs, h)).min())


def run_pair(domains, steps, every, dt=None, adaptive=True, exact=False, build=None, track=None, path="auto",
             track_fn=None):
    """Step GPU and FP32 oracle side by side; compare every `every` steps.
    ``track`` (a list) receives the lowest node height at every checkpoint,
    or ``track_fn(x)`` of the GPU positions when that is given."""
    doms_gpu = build() if build else domains
    doms_or = build() if build else domains
    loop = fw.ExplicitLoop(dt or 0.0, doms_gpu, useAdapativeDT=adaptive, **loop_kw(path))
    o32 = oracle.OracleLoop(doms_or, dt or 0.0, useAdapativeDT=adaptive, precision="f32", threads=8)
    assert loop.dt == o32.dt
    worst = (0.0, 0.0)
    done = 0
    while done < steps:
        n = min(every, steps - done)
        loop.advance_n(n)
        o32.advance(n)
        done += n
        xg, vg = gpu_state(loop)
        xo, vo, _ = o32.state()
        ex, ev = rel_linf(xg, xo), rel_linf(vg, vo)
        if track is not None:
            track.append(track_fn(xg) if track_fn else float(xg[:, 1].min()))
        worst = (max(worst[0], ex), max(worst[1], ev))
        if exact:
            assert np.array_equal(xg.astype(np.float64), xo), f"x differs at step {done}: {ex:.3e}"
            assert np.array_equal(vg.astype(np.float64), vo), f"v differs at step {done}: {ev:.3e}"
        assert ex <= RTOL and ev <= RTOL, f"step {done}: x {ex:.3e} v {ev:.3e}"
    return loop, o32, worst


def fp64_error(domains, steps, dt, xg, adaptive=False):
    o64 = oracle.OracleLoop(domains, dt, useAdapativeDT=adaptive, precision="f64", threads=8)
    o64.advance(steps)
    return rel_linf(xg, o64.state()[0])


def test_plain_small_2000_steps_bitwise(path):
    doms = scenes.plain_small_scene(fw)
    loop, o32, worst = run_pair(doms, 2000, 100, dt=1e-4, adaptive=False, exact=True, path=path)
    xg, _ = gpu_state(loop)
    e64 = fp64_error(scenes.plain_small_scene(fw), 2000, 1e-4, xg)
    print(f"plain small 2000 steps: vs FP32 oracle {worst}, vs FP64 {e64:.3e}")


def test_plain_small_with_ground_contact_bitwise(path):
    """12000 steps of 1e-4: the body lands on the plane (about 0.77 s of fall)."""
    doms = scenes.plain_small_scene(fw)
    low = []
    run_pair(doms, 12000, 500, dt=1e-4, adaptive=False, exact=True, track=low, path=path)
    assert min(low) < 0.01  # it reached the plane (and bounced: the plane penalty is undamped)
    assert min(low) > -0.05


def test_heightfield_disk_bitwise(path):
    loop = fw.ExplicitLoop(0.0, scenes.hf_disk_scene(fw), useAdapativeDT=True, **loop_kw(path))
    o32 = oracle.OracleLoop(scenes.hf_disk_scene(fw), 0.0, useAdapativeDT=True)
    for f in range(60):
        loop.advanceWithTime(FRAME)
        o32.advance_with_time(FRAME)
        if f % 10 == 9:
            xg, vg = gpu_state(loop)
            xo, vo, _ = o32.state()
            assert np.array_equal(xg.astype(np.float64), xo) and np.array_equal(vg.astype(np.float64), vo), f
    xg, _ = gpu_state(loop)
    assert xg[:, 1].min() > 0.05  # test_2Dfem_heightfield_contact.py:66


def test_voxel_disk_bitwise(path):
    loop = fw.ExplicitLoop(0.0, scenes.voxel_disk_scene(fw), useAdapativeDT=True, **loop_kw(path))
    o32 = oracle.OracleLoop(scenes.voxel_disk_scene(fw), 0.0, useAdapativeDT=True)
    for f in range(60):
        loop.advanceWithTime(FRAME)
        o32.advance_with_time(FRAME)
    xg, vg = gpu_state(loop)
    xo, vo, _ = o32.state()
    assert np.array_equal(xg.astype(np.float64), xo) and np.array_equal(vg.astype(np.float64), vo)
    assert xg[:, 1].min() > 0.02  # test_2Dfem_voxel_contact.py:70


def test_neohookean_heightfield_bitwise(path):
    """Reduced large-mesh workload (64 x 64 quads, NeoHookean, height field)."""
    build = lambda: scenes.plain_large_scene(fw, n=64, hf_offset=0.17)  # noqa: E731
    gaps = []
    loop, o32, worst = run_pair(None, 3000, 250, adaptive=True, build=build, path=path, exact=True, track=gaps,
                                track_fn=lambda x: hf_gap(build(), x))
    assert min(gaps) < 0.0, "the body must press into the height field (contact active)"
    xg, _ = gpu_state(loop)
    e64 = fp64_error(build(), 3000, loop.dt, xg, adaptive=True)
    print(f"NeoHookean 64x64: vs FP32 oracle {worst}, vs FP64 {e64:.3e}")


def test_j2_plastic_block_on_plane_bitwise(path):
    def build():
        conn, coords = fw.structured_rectangle(24, 12, 0.4, 0.2, origin=(0.1, 0.05), jitter=0.1, seed=3)
        mat = fw.MisesPlastic(E=1e5, nu=0.3, rho=100.0, sigma_y=2e3, H=1e3)
        fem = fw.FemDomain(fw.Mesh(2, conn, coords), fw.SolidProp(mat), [fw.Gravity([0.0, -9.8])],
                           initials=[fw.InitialVel("ALL", [0.3, -2.0])])
        return [fw.GroundDomain(2, [0.0, 0.0], [0.0, 1.0]), fem]
    loop, o32, _ = run_pair(None, 4000, 500, dt=5e-5, adaptive=False, exact=True, build=build, path=path)
    ep_g = loop.femSpringManager.eqPlasticStrain.numpy()
    _, eq_o = o32.plastic()
    assert ep_g.max() > 0.0, "the block must yield"
    assert np.array_equal(ep_g.astype(np.float64), eq_o)


def test_bcs_scene_bitwise(path):
    """test_2Dfem_bcs.py: Force+Fixed, EnforceVel+Fixed, EnforceAcc+Fixed bodies."""
    def build():
        conn = np.array([[0, 1, 3], [0, 3, 2]], dtype=np.int32)
        c = np.array([[0.5, 0.5], [0.7, 0.5], [0.5, 0.7], [0.7, 0.7]], dtype=np.float32)
        prop = fw.SolidProp(fw.Elastic(E=2e4, nu=0.2, rho=40.0))
        d0 = fw.FemDomain(fw.Mesh(2, conn, c), prop, [fw.Force([0, 1], [0, -100.0]), fw.Fixed([2, 3])], False)
        d1 = fw.FemDomain(fw.Mesh(2, conn, c + 0.25), prop, [fw.EnforceVel([0, 1], [0, -1.0]), fw.Fixed([2, 3])],
                          False)
        d2 = fw.FemDomain(fw.Mesh(2, conn, c - 0.25), prop, [fw.EnforceAcc([0, 1], [0, -10.0]), fw.Fixed([2, 3])],
                          False)
        d3 = fw.FemDomain(fw.Mesh(2, conn, c + 0.5), prop, [], False, initials=[fw.InitialVel([0, 1], [0, -1.0])])
        return [d0, d1, d2, d3]
    loop = fw.ExplicitLoop(0.0, build(), useAdapativeDT=True, **loop_kw(path))
    o32 = oracle.OracleLoop(build(), 0.0, useAdapativeDT=True)
    for _ in range(60):
        loop.advanceWithTime(FRAME)
        o32.advance_with_time(FRAME)
    xg, vg = gpu_state(loop)
    xo, vo, _ = o32.state()
    assert np.array_equal(xg.astype(np.float64), xo) and np.array_equal(vg.astype(np.float64), vo)


def test_prepared_data_bitwise():
    doms = scenes.plain_small_scene(fw)
    loop = fw.ExplicitLoop(1e-4, doms, useAdapativeDT=False)
    o32 = oracle.OracleLoop(doms, 1e-4, useAdapativeDT=False)
    m, a, j = o32.prepared()
    n = int(loop.femSpringManager.totalNodes.numpy()[0])
    assert np.array_equal(loop.femSpringManager.mass.numpy()[:n].astype(np.float64), m)
    assert np.array_equal(loop.femSpringManager.elemVolume.numpy().astype(np.float64), a)
    assert np.array_equal(loop.femSpringManager.J_inv.numpy().reshape(-1, 4).astype(np.float64), j)


def test_gpu_kats_through_public_api():
    loop = fw.ExplicitLoop(0.0, [scenes.two_triangle_square(fw)], useAdapativeDT=True)
    t = 0.0
    while t < 3.0:
        loop.advanceWithTime(FRAME)
        t += FRAME
        if loop.femSpringManager.coords.numpy()[0, 1] < 0.0:
            break
    assert np.isclose(t, 1.0, atol=FRAME)
    mesh = scenes.elastic10000_mesh(fw)
    loop = fw.ExplicitLoop(0.0, [fw.FemDomain(mesh, fw.SolidProp(fw.Elastic(2e4, 0.2, 40.0)),
                                              [fw.Gravity([0, -1.0])])], useAdapativeDT=True)
    t = 0.0
    while t < 3.0:
        loop.advanceWithTime(FRAME)
        t += FRAME
        if loop.femSpringManager.coords.numpy()[0, 1] < 0.0:
            break
    assert np.isclose(t, np.sqrt(0.6), atol=FRAME)


def test_run_to_run_determinism():
    a = fw.ExplicitLoop(0.0, scenes.hf_disk_scene(fw), useAdapativeDT=True)
    b = fw.ExplicitLoop(0.0, scenes.hf_disk_scene(fw), useAdapativeDT=True)
    for _ in range(30):
        a.advanceWithTime(FRAME)
        b.advanceWithTime(FRAME)
    xa, va = gpu_state(a)
    xb, vb = gpu_state(b)
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)


def test_aabb_and_getbbox(path):
    doms = scenes.plain_small_scene(fw)
    loop = fw.ExplicitLoop(1e-4, doms, useAdapativeDT=False, **loop_kw(path))
    loop.advance_n(50)
    lb, ub = doms[1].getBBox()
    xg, _ = gpu_state(loop)
    bn = doms[1].mesh.boundaryNodes
    assert np.array_equal(lb, xg[bn].min(axis=0)) and np.array_equal(ub, xg[bn].max(axis=0))


def test_resident_is_chosen_for_large_mesh_and_matches_gather():
    """The 256 x 256 workload runs on the resident path by default; it and the
    gather path give identical bits (same sums in the same order)."""
    a = fw.ExplicitLoop(0.0, scenes.plain_large_scene(fw, n=256), useAdapativeDT=True)
    assert a.path == 2 and a.patches >= 64, (a.path, a.patches)
    b = fw.ExplicitLoop(0.0, scenes.plain_large_scene(fw, n=256), useAdapativeDT=True, path="gather")
    assert b.path == 1
    for _ in range(3):
        a.advanceWithTime(FRAME)
        b.advanceWithTime(FRAME)
    xa, va = gpu_state(a)
    xb, vb = gpu_state(b)
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)
    assert np.array_equal(np.asarray(a.femSpringManager.domains[0].getBBox()),
                          np.asarray(b.femSpringManager.domains[0].getBBox()))


@pytest.mark.parametrize("res_sync", [0, 1], ids=["flag-in-data", "counter"])
@pytest.mark.parametrize("patches", [1, 7, 64, 148])
def test_resident_patch_counts_bitwise(patches, res_sync):
    doms = lambda: scenes.plain_large_scene(fw, n=32, hf_offset=0.17)  # noqa: E731
    a = fw.ExplicitLoop(0.0, doms(), useAdapativeDT=True, path="resident", patches=patches, res_sync=res_sync)
    b = fw.ExplicitLoop(0.0, doms(), useAdapativeDT=True, path="gather")
    for _ in range(20):
        a.advanceWithTime(FRAME)
        b.advanceWithTime(FRAME)
    xa, va = gpu_state(a)
    xb, vb = gpu_state(b)
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)


@pytest.mark.parametrize("res_sync", [0, 1], ids=["flag-in-data", "counter"])
@pytest.mark.parametrize("threads,front", [(512, 2), (512, 8), (1024, 8), (1024, 12), (1024, 16)])
def test_resident_launch_shapes_bitwise(threads, front, res_sync):
    """Every resident CTA size and split of front warps gives the gather
    path's bits (the node pass and the warp split change no sum's order)."""
    doms = lambda: scenes.plain_large_scene(fw, n=64, hf_offset=0.17)  # noqa: E731
    a = fw.ExplicitLoop(0.0, doms(), useAdapativeDT=True, path="resident", res_threads=threads, front_warps=front,
                        res_sync=res_sync)
    b = fw.ExplicitLoop(0.0, doms(), useAdapativeDT=True, path="gather")
    assert a.path == 2
    assert a._native.get_option(_native.FW_OPT_FRONT_WARPS) == front
    assert a._native.get_option(_native.FW_OPT_RES_THREADS) == threads
    for _ in range(10):
        a.advanceWithTime(FRAME)
        b.advanceWithTime(FRAME)
    xa, va = gpu_state(a)
    xb, vb = gpu_state(b)
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)


@pytest.mark.parametrize("n_bodies", [3, 10])
def test_resident_multi_body_bitwise(n_bodies):
    """Several bodies in one scene, all three laws, plane contact: the body
    boxes (and so the broad-phase gates) are reduced per body across CTAs.
    3 bodies use the flag-in-data hand-off, 10 bodies (> 8) the counter."""
    build = lambda: scenes.multi_block_scene(fw, n_bodies)  # noqa: E731
    a = fw.ExplicitLoop(0.0, build(), useAdapativeDT=True, path="resident", patches=37)
    b = fw.ExplicitLoop(0.0, build(), useAdapativeDT=True, path="gather")
    assert a.path == 2
    low = 1e9
    for _ in range(6):
        a.advanceWithTime(FRAME)
        b.advanceWithTime(FRAME)
        xa, va = gpu_state(a)
        low = min(low, float(xa[:, 1].min()))
        xb, vb = gpu_state(b)
        assert np.array_equal(xa, xb) and np.array_equal(va, vb)
    assert low < 0.0, "the blocks must reach the plane"
    for d in a.femSpringManager.domains:
        assert np.isfinite(np.asarray(d.getBBox())).all()


def test_plain_large_full_size_5000_steps_bitwise():
    """The large single-mesh workload at full size (256 x 256 quads, 131072
    triangles, NeoHookean, height field), 5000 substeps, bit-identical to the
    FP32 oracle at every checkpoint; the FP64 distance is reported."""
    build = lambda: scenes.plain_large_scene(fw, n=256)  # noqa: E731
    low = []
    loop, o32, worst = run_pair(None, 5000, 1000, adaptive=True, build=build, exact=True, track=low,
                                track_fn=lambda x: hf_gap(build(), x))
    assert loop.path == 2
    assert min(low) < 0.0, "the body must reach the height field within the 5000 substeps (contact active)"
    xg, vg = gpu_state(loop)
    o64 = oracle.OracleLoop(build(), 0.0, useAdapativeDT=True, precision="f64", threads=16)
    o64.advance(5000)
    x64, v64, _ = o64.state()
    print(f"plain large 5000 substeps: bitwise vs FP32 oracle; vs FP64 x {rel_linf(xg, x64):.3e} "
          f"v {rel_linf(vg, v64):.3e}; deepest penetration of the height field {-min(low):.2e}")


@pytest.mark.parametrize("path", ["gather", "resident"])
def test_damping_assigned_mid_run_applies_from_the_next_substep(path):
    """The reference reads ExplicitLoop.damping at every substep
    (explicitloop.py:528, 537): a value assigned between substeps applies from
    the next one, on every step path."""
    loop = fw.ExplicitLoop(1e-4, scenes.plain_small_low_scene(fw), useAdapativeDT=False, path=path)
    o32 = oracle.OracleLoop(scenes.plain_small_low_scene(fw), 1e-4, useAdapativeDT=False)
    loop.advance_n(200)
    o32.advance(200)
    loop.damping = 0.05
    o32.damping = 0.05
    loop.advance_n(300)
    o32.advance(300)
    xg, vg = gpu_state(loop)
    xo, vo, _ = o32.state()
    assert np.array_equal(xg.astype(np.float64), xo) and np.array_equal(vg.astype(np.float64), vo)
