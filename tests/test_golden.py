"""The oracle against golden fixtures made by the reference's own code.

``tests/golden/*.npz`` were written by ``tests/golden/make_golden.py``, which
runs FlatWorld's unmodified Python source (``ExplicitLoop``, its contact
build, ``FemSpringManager`` and every Warp kernel they launch) on a serial CPU
stand-in for the Warp runtime (``tests/golden/warp_standin.py``: IEEE float32
per operation, kernels run thread by thread, ``wp.log`` = the C library's
``logf``).  These tests pin the oracle to those outputs:

* the oracle build that uses the C library's ``logf`` (``f32libm``) must give
  the fixtures' bits at every snapshot, for every case -- the restatement and
  the reference agree operation for operation;
* the default FP32 oracle (``f32``, the GPU's arithmetic: ``log`` by an
  IEEE-only method) must give the same bits wherever no ``log`` is evaluated
  (every case but the NeoHookean one), and stay within 1e-5 relative in
  positions on the NeoHookean case.
"""

import os

import numpy as np
import pytest

import flatworld_b200 as fw
import oracle
from tests import scenes
from tests.golden.make_golden import CASES, FRAME, LOOP_KW

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RTOL = 1e-5
NEOHOOKEAN_CASES = {"nh_heightfield32", "tied_slabs"}


def load(name):
    path = os.path.join(HERE, f"{name}.npz")
    if not os.path.exists(path):
        pytest.fail(f"missing golden fixture {path}: run tests/golden/make_golden.py")
    return dict(np.load(path))


def rel_linf(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def run_oracle(name, precision):
    """Yield (mark, x, v, oracle) at the fixture's snapshots."""
    builder, kw, dt, adaptive, (mode, total, every) = CASES[name]
    o = oracle.OracleLoop(getattr(scenes, builder)(fw, **kw), dt, useAdapativeDT=adaptive, precision=precision,
                          **LOOP_KW.get(name, {}))
    yield 0, None, None, o
    for k in range(1, total + 1):
        if mode == "steps":
            o.advance(1)
        else:
            o.advance_with_time(FRAME)
        if k % every == 0:
            x, v, _ = o.state()
            yield k, x, v, o


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_libm_equals_reference_fixture(name):
    g = load(name)
    it = run_oracle(name, "f32libm")
    _, _, _, o = next(it)
    assert o.dt == float(g["dt"]), (o.dt, float(g["dt"]))
    m, _, _ = o.prepared()
    assert np.array_equal(m.astype(np.float32), g["mass"])
    i = 0
    for k, x, v, o in it:
        assert k == g["marks"][i]
        assert np.array_equal(x.astype(np.float32), g["x"][i]), (name, k, rel_linf(x, g["x"][i]))
        assert np.array_equal(v.astype(np.float32), g["v"][i]), (name, k, rel_linf(v, g["v"][i]))
        if "eqps" in g:
            _, eq = o.plastic()
            assert np.array_equal(eq.astype(np.float32), g["eqps"][i]), (name, k)
        i += 1
    assert i == len(g["marks"])


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_f32_against_reference_fixture(name):
    g = load(name)
    worst_x = worst_v = 0.0
    i = 0
    for k, x, v, o in run_oracle(name, "f32"):
        if x is None:
            continue
        if name in NEOHOOKEAN_CASES:
            worst_x = max(worst_x, rel_linf(x, g["x"][i]))
            worst_v = max(worst_v, rel_linf(v, g["v"][i]))
        else:
            assert np.array_equal(x.astype(np.float32), g["x"][i]), (name, k, rel_linf(x, g["x"][i]))
            assert np.array_equal(v.astype(np.float32), g["v"][i]), (name, k, rel_linf(v, g["v"][i]))
        i += 1
    if name in NEOHOOKEAN_CASES:
        print(f"{name}: f32 oracle vs reference fixture: x {worst_x:.2e}, v {worst_v:.2e} (relative, L-inf)")
        assert worst_x <= RTOL, worst_x


def test_fixtures_exercise_contact_and_plasticity():
    """The fixtures must cover what they are for: bodies reach their ground,
    the J2 block yields."""
    low = load("plain_small_contact")["x"][:, :, 1].min()
    assert low < 0.0  # nodes pressed below the plane y = 0 (penalty contact active)
    hf = load("nh_heightfield32")
    assert hf["x"][-1][:, 1].min() < 0.2 - 0.5 * 250 * float(hf["dt"]) * 12 + 0.5  # moved
    assert load("j2_block")["eqps"][-1].max() > 0.0
    assert load("hf_disk")["x"][-1][:, 1].min() > 0.05  # test_2Dfem_heightfield_contact.py:66
    assert load("voxel_disk")["x"][-1][:, 1].min() > 0.02  # test_2Dfem_voxel_contact.py:70
