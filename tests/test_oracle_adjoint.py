"""The oracle's adjoint (FP64 build) against FP64 central differences.

``OracleLoop.adjoint`` restates the reverse-mode derivative of the substep
(elements column by column in dual numbers through the same formulas as the
forward, contact of every kind with its velocity damping, the J2 plastic state
carried backward).  Here it is checked on 12 x 12-quad NeoHookean / J2 blocks
that land on a plane, a height field and a voxel grid: along random
directions in the per-element Young's moduli and in the initial velocities,
the adjoint must equal the FP64 central difference (inputs set in FP64, no
float32 rounding) to 1e-6 relative.  A direction whose central difference is
not converged -- a contact starts inside the interval, where the damping term
switches on with a jump -- is replaced by another one.  This proves the linearisation itself;
the CUDA adjoint's distance to it is then the FP32 trajectory's rounding
(tests/test_adjoint.py)."""

import numpy as np
import pytest

import flatworld_b200 as fw
import oracle
from tests import scenes

STEPS, DT, EPS, RTOL = 400, 5e-5, 1e-5, 1e-6


def block(kind, n=12):
    def build(young=None):
        ground, fem = scenes.gradient_block_scene(fw, n=n, side=0.1, bottom=0.02, young=young, v0=(0.3, -1.0))
        if kind == "heightfield":
            xs = np.linspace(0.0, 1.0, 257)
            ground = fw.HeightFieldDomain(2, (0.005 * np.sin(20 * xs)).astype(np.float32), lb=[0.0, -1.0],
                                          ub=[1.0, 1.0])
        elif kind == "voxel":
            # a flat floor (the nearest free face of a penetrating node is the
            # top one, so the signed distance is smooth there), cell faces
            # offset from the mesh's node columns
            occ = np.zeros((40, 20), np.int32)
            occ[:, :15] = 1
            ground = fw.VoxelGridDomain(2, 40, 20, [0.0123, -0.05], [1.0123, 0.03], occupancy_np=occ)
        elif kind == "j2":
            fem.prop = fw.SolidProp(fw.MisesPlastic(1e5, 0.3, 1000.0, 3e3, 1e3))
        return [ground, fem]
    return build


@pytest.mark.parametrize("kind", ["plane", "heightfield", "voxel", "j2"])
def test_oracle_adjoint_equals_fp64_central_differences(kind):
    build = block(kind)
    doms = build()
    o = oracle.OracleLoop(doms, DT, useAdapativeDT=False, precision="f64")
    E0 = np.asarray(doms[1].elementYoung, np.float64)
    x0, v0, _ = o.state()
    rng = np.random.default_rng(7)
    w = rng.standard_normal((o.N, 2))
    _, vb, eb = o.adjoint(STEPS, xbar=w)  # L = <w, x_T>
    if kind == "j2":
        _, eq = o.plastic()
        assert eq.max() > 0.0  # the block yields, so the return map is differentiated

    def loss(E, v):
        q = oracle.OracleLoop(build(), DT, useAdapativeDT=False, precision="f64")
        q.set_young64(E)
        q.set_state64(x0, v)
        q.advance(STEPS)
        return float(np.sum(w * q.state()[0]))

    def central(f, d):
        """Central difference along d at EPS, or None when the one at EPS / 2
        disagrees (a contact switches on inside the interval: the damping term
        starts with a jump, so the loss is not smooth there)."""
        a = (f(EPS * d) - f(-EPS * d)) / (2 * EPS)
        b = (f(0.5 * EPS * d) - f(-0.5 * EPS * d)) / EPS
        return a if abs(a - b) <= 0.5 * RTOL * abs(a) else None

    checked = {"E": 0, "v": 0}
    for _ in range(8):
        if min(checked.values()) >= 2:
            break
        dE = E0 * rng.standard_normal(o.E)
        fd = central(lambda p: loss(E0 + p, v0), dE)
        if fd is not None and checked["E"] < 2:
            assert abs(float(eb @ dE) - fd) <= RTOL * abs(fd), (kind, float(eb @ dE), fd)
            checked["E"] += 1
        dv = rng.standard_normal((o.N, 2))
        fd = central(lambda p: loss(E0, v0 + p), dv)
        if fd is not None and checked["v"] < 2:
            assert abs(float(np.sum(vb * dv)) - fd) <= RTOL * abs(fd), (kind, float(np.sum(vb * dv)), fd)
            checked["v"] += 1
    assert min(checked.values()) >= 2, checked
