"""The oracle against golden fixtures made by the reference's own code.

``tests/golden/*.npz`` were written by ``tests/golden/make_golden.py``, which
runs FlatWorld's unmodified Python source (``ExplicitLoop``, its contact
build, ``FemSpringManager``, the rigid manager and every Warp kernel they
launch) on a serial CPU stand-in for the Warp runtime
(``tests/golden/warp_standin.py``: IEEE float32 per operation, kernels run
thread by thread, ``wp.log`` / ``wp.sin`` / ``wp.cos`` = the C library's
``logf`` / ``sinf`` / ``cosf``).  These tests pin the oracle to those outputs:

* the oracle build that uses the C library's functions (``f32libm``) must
  give the fixtures' bits at every snapshot, for every case -- the
  restatement and the reference agree operation for operation;
* the default FP32 oracle (``f32``, the GPU's arithmetic: those functions by
  IEEE-only methods) must give the same bits wherever none of them is
  evaluated on a changing argument, and stay within the case's bar
  (``tests/golden/bars.py``) on the NeoHookean and rotating-rigid cases.
"""

import os

import numpy as np
import pytest

from tests.golden.bars import TRANSCENDENTAL_CASES, noise_floor, position_bar, rel_linf, run_oracle
from tests.golden.make_golden import CASES

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    path = os.path.join(HERE, f"{name}.npz")
    if not os.path.exists(path):
        pytest.fail(f"missing golden fixture {path}: run tests/golden/make_golden.py")
    return dict(np.load(path))


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
        if name in TRANSCENDENTAL_CASES:
            worst_x = max(worst_x, rel_linf(x, g["x"][i]))
            worst_v = max(worst_v, rel_linf(v, g["v"][i]))
        else:
            assert np.array_equal(x.astype(np.float32), g["x"][i]), (name, k, rel_linf(x, g["x"][i]))
            assert np.array_equal(v.astype(np.float32), g["v"][i]), (name, k, rel_linf(v, g["v"][i]))
        i += 1
    if name in TRANSCENDENTAL_CASES:
        print(f"{name}: f32 oracle vs reference fixture: x {worst_x:.2e}, v {worst_v:.2e} (relative, L-inf); "
              f"noise floor {noise_floor(name):.2e}")
        assert worst_x <= position_bar(name), (worst_x, position_bar(name))


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
    fc = load("flex_circles")  # two circles pulled together: they meet and bounce apart
    h = fc["x"].shape[1] // 2
    assert fc["v"][0][:h, 1].mean() > 0.0 > fc["v"][1][:h, 1].mean()
    assert abs(float(fc["x"][1][h:, 1].min() - fc["x"][1][:h, 1].max())) < 0.01  # in contact at the bounce
    fb = load("rigid_fixed_ball")  # the circle lands on the fixed ball's top (y = 0.45) and bounces
    assert min(float(x[:, 1].min()) for x in fb["x"]) > 0.44 and fb["x"][1][:, 1].min() > fb["x"][0][:, 1].min()
    assert not np.array_equal(fb["x"], load("rigid_fixed_ball_tied")["x"])  # the tie changes the motion
    assert np.abs(load("rigid_pusher")["x"][-1] - load("rigid_pusher")["x"][0]).max() > 0.03  # the box drags the block
    assert min(float(x[:, 1].min()) for x in load("spring_mixed")["x"]) < 0.0  # spring-plane penalty active
