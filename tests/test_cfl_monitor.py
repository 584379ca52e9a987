"""CFL monitor: the stable time of the current (deformed) mesh, reduced on the
GPU inside the step (warp shuffles; gather and stream steps one atomic per
warp and scene, the resident step one per CTA and launch).

The reference's dt is fixed at construction from the rest shape
(explicitloop.py:160-166; FemDomain.stableTime = 0.4 * L_min / sqrt(E / rho),
femdomain.py:24).  The monitor evaluates that same bound on every triangle's
current shortest edge and reports the minimum; it never changes dt, so the
trajectory is the same bits with it on or off."""

import numpy as np
import pytest

import flatworld_b200 as fw
from flatworld_b200.batch import BatchedLoop
from tests import scenes

pytestmark = pytest.mark.gpu


def host_bound(x, conn, coef):
    """The kernel's arithmetic in float32, on host: min over triangles of
    sqrt(min squared edge) * coef."""
    x = x.astype(np.float32)
    a, b, c = x[conn[:, 0]], x[conn[:, 1]], x[conn[:, 2]]

    def sq(p, q):
        d = (p - q).astype(np.float32)
        return d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]

    m = np.minimum(sq(a, b), np.minimum(sq(b, c), sq(c, a)))
    return float((np.sqrt(m) * np.float32(coef)).min())


def test_cfl_monitor_reports_the_current_shape_bound_and_changes_nothing():
    doms = scenes.j2_block_scene(fw)
    loop = fw.ExplicitLoop(5e-5, doms, useAdapativeDT=False, path="gather")
    ref = fw.ExplicitLoop(5e-5, scenes.j2_block_scene(fw), useAdapativeDT=False, path="gather")
    loop.enable_cfl_monitor()
    fem = doms[1]
    mat = fem.prop.getMaterial()
    coef = np.float32(0.4 / (mat.E / mat.rho) ** 0.5)
    conn = np.asarray(fem.mesh.connectivity)[:, :3]
    n = int(loop.femSpringManager.totalNodes.numpy()[0])
    x0 = loop.femSpringManager.coords.numpy()[:n]
    loop.advance()
    ref.advance()
    # one substep: the bound of the shape at its start (the rest shape), which
    # is the reference's stableTime of the domain
    got = loop.currentStableTime()
    assert got == host_bound(x0, conn, coef)
    assert abs(got - fem.stableTime) <= 1e-6 * fem.stableTime
    lowest = got
    for _ in range(40):
        loop.advance_n(100)
        ref.advance_n(100)
        lowest = min(lowest, loop.currentStableTime())
    # the block hits the plane and yields: its shortest edges shrink
    assert lowest < 0.95 * fem.stableTime
    # dt never changed: the same bits as without the monitor
    assert np.array_equal(loop.femSpringManager.coords.numpy()[:n], ref.femSpringManager.coords.numpy()[:n])
    assert np.array_equal(loop.femSpringManager.V.numpy()[:n], ref.femSpringManager.V.numpy()[:n])


def test_cfl_monitor_per_scene_in_a_batch():
    sc = [scenes.j2_block_scene(fw), scenes.plain_small_low_scene(fw)]
    bl = BatchedLoop(sc, dt=[5e-5, 1e-4], useAdapativeDT=False, path="gather")
    bl.enable_cfl_monitor()
    bl.advance(1)
    got = bl.currentStableTimes()
    for s, doms in enumerate(sc):
        assert abs(got[s] - doms[1].stableTime) <= 1e-6 * doms[1].stableTime, (s, got[s], doms[1].stableTime)


@pytest.mark.parametrize("path", ["resident", "stream"])
def test_cfl_monitor_same_on_every_step(path):
    """The resident and stream steps report the gather step's bound bit for
    bit (the same operations on the same positions), window by window, and
    the trajectory is unchanged by the monitor."""
    build = lambda: scenes.plain_large_scene(fw, n=32, hf_offset=0.17)  # noqa: E731
    if path == "resident":
        a = fw.ExplicitLoop(0.0, build(), useAdapativeDT=True, path="resident")
        assert a.path == 2
        a.enable_cfl_monitor()
        read = lambda: a.currentStableTime()  # noqa: E731
        step = lambda n: a.advance_n(n)  # noqa: E731
    else:
        a = BatchedLoop([build(), scenes.j2_block_scene(fw)], dt=3e-5, useAdapativeDT=False, path="stream")
        assert a.path == "stream"
        a.enable_cfl_monitor()
        read = lambda: a.currentStableTimes()  # noqa: E731
        step = lambda n: a.advance(n)  # noqa: E731
    if path == "resident":
        g = fw.ExplicitLoop(0.0, build(), useAdapativeDT=True, path="gather")
        g.enable_cfl_monitor()
        gread, gstep = (lambda: g.currentStableTime()), (lambda n: g.advance_n(n))
    else:
        g = BatchedLoop([build(), scenes.j2_block_scene(fw)], dt=3e-5, useAdapativeDT=False, path="gather")
        g.enable_cfl_monitor()
        gread, gstep = (lambda: g.currentStableTimes()), (lambda n: g.advance(n))
    for n in (1, 37, 300, 1000):
        step(n)
        gstep(n)
        assert np.array_equal(np.asarray(read()), np.asarray(gread())), n
    xa = a.femSpringManager.coords.numpy() if path == "resident" else a.all_coords()
    xg = g.femSpringManager.coords.numpy() if path == "resident" else g.all_coords()
    assert np.array_equal(xa, xg)
