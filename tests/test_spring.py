"""Spring-mass domains (SpringMassDomain, flatworld/springmass.py;
_spring_force_kernel, femspringmanager.py:283-312; packing, 815-870).

CPU: the oracle reproduces the reference's own spring tests
(test2D/test_2Dspring_bcs.py: Force / EnforceVel / EnforceAcc with Fixed
nodes, final minimum (0.0, -0.252) within 1e-3; test2D/test_2Dspring_10000.py:
a 100 x 100 spring grid under gravity 100, final minimum (0.25, -0.5278)
within 1e-2).  GPU: the CUDA path gives the oracle's bits on those scenes, on
FEM and spring bodies together over a ground plane (spring-plane contact at
100 k, the spring-FEM pair bounding dt), and with mass scaling."""

import numpy as np
import pytest

import flatworld_b200 as fw
import oracle
from flatworld_b200.world import SceneLayout

FRAME = 1.0 / 60.0


def bcs_scene():
    """test2D/test_2Dspring_bcs.py:17-27"""
    conn = np.array([[0, 1], [1, 2], [0, 2], [2, 3], [3, 1], [0, 3]], dtype=np.int32)
    coords = np.array([[0.5, 0.5], [0.7, 0.5], [0.5, 0.7], [0.7, 0.7]], dtype=np.float32)
    d0 = fw.SpringMassDomain(2, coords, conn, [100.0, 1.0, 1.0], [fw.Force([0, 1], [0, -1.0]), fw.Fixed([2, 3])],
                             False)
    d1 = fw.SpringMassDomain(2, coords - 0.25, conn, [100.0, 1.0, 1.0],
                             [fw.EnforceVel([0, 1], [0, -1.0]), fw.Fixed([2, 3])], False)
    d2 = fw.SpringMassDomain(2, coords - 0.5, conn, [100.0, 1.0, 1.0],
                             [fw.EnforceAcc([0, 1], [0, -10.0]), fw.Fixed([2, 3])], False)
    return [d0, d1, d2]


def grid_scene(n=100):
    """test2D/test_2Dspring_10000.py:26-48 (n x n cells, four springs each)."""
    dx = 0.6 / n
    ii, jj = np.meshgrid(np.arange(n + 1), np.arange(n + 1), indexing="ij")
    coords = np.stack([dx * ii, dx * jj], axis=-1).reshape(-1, 2).astype(np.float32)
    conn = []
    for i in range(n):
        for j in range(n):
            a, b, c = i * (n + 1) + j, i * (n + 1) + j + 1, (i + 1) * (n + 1) + j
            conn += [[a, b], [b, c], [c, a], [a, b]]
    conn = np.asarray(conn, np.int32)
    return [fw.SpringMassDomain(2, coords + 0.25, conn, [10.0, 1.0, 1.0], [fw.Gravity([0, -100.0])], False)]


def mixed_scene():
    """An Elastic block and a spring net (a 6 x 6 grid of the grid scene's
    pattern) falling on the ground plane y = 0, side by side."""
    conn, coords = fw.structured_rectangle(8, 4, 0.2, 0.1, origin=(0.0, 0.05))
    block = fw.FemDomain(fw.Mesh(2, conn, coords), fw.SolidProp(fw.Elastic(E=2e4, nu=0.3, rho=100.0)),
                         [fw.Gravity([0.0, -9.8])])
    net = grid_scene(6)[0]
    xy = (net.coords - np.float32(0.25)) * np.float32(0.25) + np.float32([0.3, 0.03])  # [0.3, 0.45] x [0.03, 0.18]
    net = fw.SpringMassDomain(2, xy.astype(np.float32), net.connectivity, [200.0, 0.5, 0.01], [fw.Gravity([0.0, -9.8])],
                              friction=0.1)
    return [fw.GroundDomain(2, [0.0, 0.0], [0.0, 1.0]), block, net]


def _run_frames(loop, t_end):
    t = 0.0
    while t < t_end:
        loop(FRAME)
        t += FRAME


def test_oracle_reference_spring_bcs():
    o = oracle.OracleLoop(bcs_scene(), useAdapativeDT=True)
    _run_frames(o.advance_with_time, 0.2)
    x, _, _ = o.state()
    assert np.allclose(x.min(axis=0), [0.0, -0.252], atol=1e-3)


def test_oracle_reference_spring_grid():
    o = oracle.OracleLoop(grid_scene(), useAdapativeDT=True, threads=8)
    _run_frames(o.advance_with_time, 0.1)
    x, _, _ = o.state()
    assert np.allclose(x.min(axis=0), [0.25, -0.5278], atol=1e-2)


def test_layout_matches_oracle():
    for build in (bcs_scene, grid_scene, mixed_scene):
        lay = SceneLayout(build(), useAdapativeDT=True)
        o = oracle.OracleLoop(build(), useAdapativeDT=True)
        assert lay.stableTime == o.stableTime, build.__name__
    lay = SceneLayout(mixed_scene(), useAdapativeDT=True)
    assert [c.kind for c in lay.pairs] == ["plane", "plane"] and len(lay.unbatched) == 1


def test_spring_before_fem_is_refused():
    d = mixed_scene()
    with pytest.raises(NotImplementedError):
        SceneLayout([d[0], d[2], d[1]])


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["bcs", "grid", "mixed"])
def test_gpu_equals_oracle(name):
    build = {"bcs": bcs_scene, "grid": lambda: grid_scene(40), "mixed": mixed_scene}[name]
    lp = fw.ExplicitLoop(0.0, build(), useAdapativeDT=True)
    assert lp.path == 1  # spring-mass worlds run on the gather path
    o = oracle.OracleLoop(build(), useAdapativeDT=True, threads=4)
    n = o.N
    m_orc, _, _ = o.prepared()
    assert np.array_equal(lp.femSpringManager.mass.numpy()[:n].astype(np.float64), m_orc)
    for f in range(12):
        lp.advanceWithTime(FRAME)
        o.advance_with_time(FRAME)
        xo, vo, _ = o.state()
        assert np.array_equal(lp.femSpringManager.coords.numpy()[:n].astype(np.float64), xo), (name, f)
        assert np.array_equal(lp.femSpringManager.V.numpy()[:n].astype(np.float64), vo), (name, f)
    assert np.isfinite(lp.energy()["total"])


@pytest.mark.gpu
def test_gpu_mass_scaling_with_springs():
    """The spring part of the mass-scaling kernel: spring nodes get at least 4 k dt^2."""
    t = 4.0 * SceneLayout(mixed_scene(), useAdapativeDT=True).stableTime
    lp = fw.ExplicitLoop(0.0, mixed_scene(), useAdapativeDT=True, mass_scaling_dt=t)
    o = oracle.OracleLoop(mixed_scene(), useAdapativeDT=True, mass_scaling_dt=t)
    n = o.N
    m_orc, _, _ = o.prepared()
    assert np.array_equal(lp.femSpringManager.mass.numpy()[:n].astype(np.float64), m_orc)
    for f in range(6):
        lp.advanceWithTime(FRAME)
        o.advance_with_time(FRAME)
        xo, _, _ = o.state()
        assert np.array_equal(lp.femSpringManager.coords.numpy()[:n].astype(np.float64), xo), f


@pytest.mark.gpu
def test_gpu_batched_spring_scenes_equal_alone():
    """A BatchedLoop of spring scenes steps on the gather path; each scene
    equals the same scene stepped alone."""
    from flatworld_b200.batch import BatchedLoop

    builds = [bcs_scene, lambda: grid_scene(20), mixed_scene]
    b = BatchedLoop([f() for f in builds], dt=2e-4, useAdapativeDT=False)
    b.advance(150)
    for s, f in enumerate(builds):
        lp = fw.ExplicitLoop(2e-4, f(), useAdapativeDT=False)
        lp.advance_n(150)
        n = len(b.coords(s))
        assert np.array_equal(b.coords(s), lp.femSpringManager.coords.numpy()[:n]), s
