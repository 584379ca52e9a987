"""GPU against the golden fixtures made by the reference's own code.

The fixtures (``tests/golden/*.npz``, written by ``tests/golden/make_golden.py``
from FlatWorld's unmodified source on a serial CPU stand-in for Warp) hold node
positions and velocities at fixed substeps / frames.  Every step
implementation runs the same scene through the public API and is compared
at every snapshot:

* no ``log`` / ``sin`` / ``cos`` of a changing argument on the path
  (Elastic, J2, ground contact, FEM-FEM contact, boundary conditions,
  springs): the GPU must give the fixture's bits;
* NeoHookean (``log J``) and rotating rigids (``sin`` / ``cos`` of the
  angle): the reference evaluates the C library's functions, the GPU
  IEEE-only methods of its own (within 2 ulp), so the bar is the case's own
  rounding noise floor, never tighter than 1e-5 relative in positions
  (``tests/golden/bars.py``); the velocity distance is reported.
"""

import os

import numpy as np
import pytest

import flatworld_b200 as fw
from tests import scenes
from tests.golden.bars import TRANSCENDENTAL_CASES, noise_floor, position_bar, rel_linf
from tests.golden.make_golden import CASES, FRAME, GATHER_ONLY, LOOP_KW

pytestmark = pytest.mark.gpu
HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PATHS = {"gather": {"path": "gather"}, "resident": {"path": "resident"},
         "resident-counter": {"path": "resident", "res_sync": 1}, "stream": {"path": "stream"}}


@pytest.mark.parametrize("path", sorted(PATHS))
@pytest.mark.parametrize("name", sorted(CASES))
def test_gpu_matches_reference_fixture(name, path):
    g = dict(np.load(os.path.join(HERE, f"{name}.npz")))
    builder, kw, dt, adaptive, (mode, total, every) = CASES[name]
    if name in GATHER_ONLY and path != "gather":
        pytest.skip("FEM-FEM contact, rigid bodies and springs step on the gather path only")
    loop = fw.ExplicitLoop(dt, getattr(scenes, builder)(fw, **kw), useAdapativeDT=adaptive, **PATHS[path],
                           **LOOP_KW.get(name, {}))
    assert loop.dt == float(g["dt"])
    m = loop.femSpringManager
    n = int(m.totalNodes.numpy()[0])
    assert np.array_equal(m.mass.numpy()[:n], g["mass"])
    worst_x = worst_v = 0.0
    done = 0
    for i, mark in enumerate(g["marks"]):
        if mode == "steps":
            loop.advance_n(int(mark) - done)
        else:
            for _ in range(int(mark) - done):
                loop.advanceWithTime(FRAME)
        done = int(mark)
        x, v = m.coords.numpy()[:n], m.V.numpy()[:n]
        if name in TRANSCENDENTAL_CASES:
            worst_x = max(worst_x, rel_linf(x, g["x"][i]))
            worst_v = max(worst_v, rel_linf(v, g["v"][i]))
        else:
            assert np.array_equal(x, g["x"][i]), (name, path, int(mark), rel_linf(x, g["x"][i]))
            assert np.array_equal(v, g["v"][i]), (name, path, int(mark), rel_linf(v, g["v"][i]))
        if "eqps" in g:
            assert np.array_equal(m.eqPlasticStrain.numpy()[: g["eqps"].shape[1]], g["eqps"][i]), (name, int(mark))
    if name in TRANSCENDENTAL_CASES:
        print(f"{name} [{path}]: GPU vs reference fixture x {worst_x:.2e}, v {worst_v:.2e} (relative, L-inf); "
              f"noise floor {noise_floor(name):.2e}")
        assert worst_x <= position_bar(name), (worst_x, position_bar(name))
