"""Selective mass scaling (ExplicitLoop(mass_scaling_dt=...), the reference's
applyMassScaling, femspringmanager.py:139-196, explicitloop.py:168-170).

CPU: the host's stable-dt rule equals the oracle's, and the oracle's scaled
masses are what the rule says (every triangle under the target gets the
density that brings it to the target).  GPU: scaled masses and the trajectory
at the larger dt equal the oracle's bit for bit, on the resident and the
gather step."""

import numpy as np
import pytest

import flatworld_b200 as fw
import oracle
from flatworld_b200.world import SceneLayout


def jittered_scene():
    """A 32 x 8 rectangle with interior nodes jittered by up to 0.4 cells (so
    some edges are short), Elastic, gravity, over the ground plane."""
    conn, coords = fw.structured_rectangle(32, 8, 0.4, 0.1, origin=(0.0, 0.02), jitter=0.4, seed=5)
    body = fw.FemDomain(fw.Mesh(2, conn, coords), fw.SolidProp(fw.Elastic(E=2e4, nu=0.25, rho=40.0)),
                        [fw.Gravity([0.0, -9.8])])
    return [fw.GroundDomain(2, [0.0, 0.0], [0.0, 1.0]), body]


def _target():
    return 2.0 * SceneLayout(jittered_scene(), useAdapativeDT=True).stableTime


def test_stable_time_rule_matches_oracle():
    t = _target()
    lay = SceneLayout(jittered_scene(), useAdapativeDT=True, mass_scaling_dt=t)
    o = oracle.OracleLoop(jittered_scene(), useAdapativeDT=True, mass_scaling_dt=t)
    assert lay.stableTime == o.stableTime
    # the plane contact still bounds the step (explicitloop.py:313-315 after the scaling)
    assert lay.stableTime <= t


def test_oracle_scaled_masses_follow_the_rule():
    t = _target()
    plain = oracle.OracleLoop(jittered_scene(), useAdapativeDT=True, precision="f64")
    scaled = oracle.OracleLoop(jittered_scene(), useAdapativeDT=True, precision="f64", mass_scaling_dt=t)
    m0, area, _ = plain.prepared()
    m1, _, _ = scaled.prepared()
    assert (m1 >= m0).all() and (m1 > m0).any()
    d = jittered_scene()[1]
    x = np.asarray(d.mesh.coords, np.float64)
    c = np.asarray(d.mesh.connectivity)
    t32 = float(np.float32(t))
    expect = m0.copy()
    for e, (a, b, k) in enumerate(c):
        L = min(np.linalg.norm(x[b] - x[a]), np.linalg.norm(x[k] - x[b]), np.linalg.norm(x[a] - x[k]))
        mat = d.prop.mat
        if 0.4 * L / np.sqrt(mat.E / mat.rho) < t32:
            rho_new = mat.E * (t32 / (0.4 * L)) ** 2
            for n in (a, b, k):
                expect[n] += (rho_new - mat.rho) * area[e] / 3.0
    assert np.allclose(m1, expect, rtol=1e-9)


@pytest.mark.gpu
@pytest.mark.parametrize("path", ["auto", "gather"])
def test_gpu_scaled_masses_and_trajectory_equal_oracle(path):
    t = _target()
    lp = fw.ExplicitLoop(0.0, jittered_scene(), useAdapativeDT=True, mass_scaling_dt=t, path=path)
    o = oracle.OracleLoop(jittered_scene(), useAdapativeDT=True, mass_scaling_dt=t, threads=4)
    n = o.N
    m_gpu = lp.femSpringManager.mass.numpy()[:n].astype(np.float64)
    m_orc, _, _ = o.prepared()
    assert np.array_equal(m_gpu, m_orc)
    assert lp.dt == o.dt
    for k in range(5):
        lp.advance_n(100)
        o.advance(100)
        xo, vo, _ = o.state()
        assert np.array_equal(lp.femSpringManager.coords.numpy()[:n].astype(np.float64), xo), k
        assert np.array_equal(lp.femSpringManager.V.numpy()[:n].astype(np.float64), vo), k
