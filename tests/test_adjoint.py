"""Differentiable form (GPU): adjoint gradients of a rollout w.r.t.
per-element Young's modulus and initial velocities, checked against central
finite differences of the FP64 oracle along random directions.

The oracle takes its inputs in float32, like the reference, so a perturbed
input p0 +- eps*d is rounded to float32 before the FP64 rollout; the adjoint
is dotted with the direction the rollouts actually saw,
(p+ - p-) / (2 eps), which keeps the central difference consistent."""

import numpy as np
import pytest

import flatworld_b200 as fw
import oracle
from flatworld_b200.diff import DiffSim
from tests import scenes

pytestmark = pytest.mark.gpu


def rollout64(domains_fn, young, v0, steps, dt, damping=0.0):
    o = oracle.OracleLoop(domains_fn(young), dt, damping=damping, useAdapativeDT=False, precision="f64", threads=8)
    o.set_state(None, v0)
    o.advance(steps)
    return o.state()[0]


def perturbed(p0, d, eps):
    """(p0 + eps d, p0 - eps d) in float32 and the direction they span."""
    hi = (p0.astype(np.float64) + eps * d).astype(np.float32)
    lo = (p0.astype(np.float64) - eps * d).astype(np.float32)
    return hi, lo, (hi.astype(np.float64) - lo.astype(np.float64)) / (2.0 * eps)


def directional_errors(sim, build, v0, steps, dt, seed_fn, loss_fn, n_dirs, seed, eps=1e-4, damping=0.0):
    """Relative error |adj - fd| / |fd| along random directions: n_dirs in
    the moduli (dE) and n_dirs in the initial velocities (dv), each checked
    on its own (a mixed direction's two parts can cancel, which magnifies
    the relative error of the sum).  seed_fn(x32, x64) gives dL/dx_T from
    the GPU rollout and from the FP64 oracle rollout of the unperturbed
    inputs."""
    x32 = sim.forward(sim.E0, v0)
    x64 = rollout64(build, sim.E0, v0, steps, dt, damping)
    eb, vb, _ = sim.backward(seed_fn(x32, x64))
    rng = np.random.default_rng(seed)
    errs = []
    for kind in ("E", "v") * n_dirs:
        if kind == "E":
            Ep, Em, dE = perturbed(sim.E0, sim.E0 * rng.standard_normal(sim.E), eps)
            vp = vm = v0
            adj = float(np.dot(eb.astype(np.float64), dE))
        else:
            vp, vm, dv = perturbed(v0, rng.standard_normal((sim.N, 2)), eps)
            Ep = Em = sim.E0
            adj = float(np.sum(vb.astype(np.float64) * dv))
        fd = (loss_fn(rollout64(build, Ep, vp, steps, dt, damping))
              - loss_fn(rollout64(build, Em, vm, steps, dt, damping))) / (2 * eps)
        errs.append(abs(adj - fd) / max(abs(fd), 1e-30))
    return errs


@pytest.mark.parametrize("bottom,steps,seed_from", [(0.04, 600, "fp32"), (0.04, 600, "fp64"), (0.5, 300, "fp64")],
                         ids=["contact-fp32seed", "contact", "free"])
def test_adjoint_matches_fp64_central_differences(bottom, steps, seed_from):
    """Quadratic loss |x_T - target|^2 (target: the rollout with 1.1 x the
    moduli).  With seed_from="fp64" the adjoint is seeded with dL/dx_T at the
    FP64 state, so the check measures the adjoint alone; "fp32" seeds it from
    the GPU's FP32 state, as FEMRollout does.  In free flight the
    centre-of-mass part of x_T - target is FP32 rounding (~2e-6 of ~8e-4),
    which the FP64 differences do not see, so that case uses the FP64 seed.

    Tolerance 2.5e-3 relative: the adjoint differentiates the FP32 forward,
    whose element strains differ from the FP64 rollout's by a median 1.4e-3
    relative in the free case and 4.4e-4 in the contact case (strain is
    (F^T F - I) / 2, a difference of nearly equal numbers; measured with the
    FP32 and FP64 oracles), and dL/dE is a sum over those stresses.  The
    measured errors are 1e-4..1.6e-3.  The contact cases must touch the plane."""
    dt = 1e-4
    build = lambda y=None: scenes.gradient_block_scene(fw, n=12, side=0.12, bottom=bottom, young=y, seed=1)  # noqa: E731
    sim = DiffSim(build(), dt, steps, checkpoint_every=50)
    rng = np.random.default_rng(5)
    v0 = (np.tile([0.0, -2.0], (sim.N, 1)) + 0.3 * rng.standard_normal((sim.N, 2))).astype(np.float32)
    target = sim.forward(sim.E0 * 1.1, v0).astype(np.float64)
    if bottom < 0.1:
        probe = fw.ExplicitLoop(dt, build(), useAdapativeDT=False, path="gather")
        probe._native.write_nodes(fw._native.FW_FIELD_V, 0, v0)
        low = []
        for _ in range(steps // 50):
            probe.advance_n(50)
            low.append(float(probe.femSpringManager.coords.numpy()[: sim.N, 1].min()))
        assert min(low) < 0.0, "the block must reach the plane (penalty contact active)"
    pick = 0 if seed_from == "fp32" else 1
    errs = directional_errors(sim, build, v0, steps, dt, lambda *xs: 2.0 * (xs[pick] - target),
                              lambda x: float(np.sum((x - target) ** 2)), 2, seed=0)
    print("relative error of directional derivatives:", errs)
    assert max(errs) < 2.5e-3, errs


def test_adjoint_of_linear_functional():
    """L = w . x_T for a fixed random w: the adjoint is J^T w exactly, with
    no error from the seed."""
    dt, steps = 1e-4, 600
    build = lambda y=None: scenes.gradient_block_scene(fw, n=12, side=0.12, bottom=0.04, young=y, seed=4)  # noqa: E731
    sim = DiffSim(build(), dt, steps, checkpoint_every=50)
    v0 = np.tile(np.array([0.0, -2.0], np.float32), (sim.N, 1))
    w = np.random.default_rng(9).standard_normal((sim.N, 2))
    errs = directional_errors(sim, build, v0, steps, dt, lambda *xs: w, lambda x: float(np.sum(w * x)), 2, seed=1)
    print("relative error of directional derivatives:", errs)
    assert max(errs) < 1e-3, errs


def test_adjoint_with_damping_matches_fp64_central_differences():
    """Velocity damping c enters the update as v' = v (1 - dt c / m) + dt f / m."""
    dt, steps, c = 1e-4, 600, 0.05
    build = lambda y=None: scenes.gradient_block_scene(fw, n=12, side=0.12, bottom=0.04, young=y, seed=4)  # noqa: E731
    sim = DiffSim(build(), dt, steps, checkpoint_every=50, damping=c)
    v0 = np.tile(np.array([0.0, -2.0], np.float32), (sim.N, 1))
    w = np.random.default_rng(11).standard_normal((sim.N, 2))
    errs = directional_errors(sim, build, v0, steps, dt, lambda *xs: w, lambda x: float(np.sum(w * x)), 2, seed=2,
                              damping=c)
    print("relative error of directional derivatives (damping):", errs)
    assert max(errs) < 1e-3, errs


@pytest.mark.parametrize("damping", [0.0, 0.05])
def test_adjoint_is_the_transpose_of_the_tangent(damping):
    """Dot-product test on one FP32 trajectory: for L = <w, x_T>, the adjoint's
    <dL/dE, dE> + <dL/dv0, dv0> equals <w, dx_T> of the forward-mode tangent
    along (dE, dv0) to rounding (1e-5 of the terms' magnitude), for
    directions in E only, v0 only and both; with plane contact."""
    dt, steps = 1e-4, 600
    build = lambda y=None: scenes.gradient_block_scene(fw, n=12, side=0.12, bottom=0.04, young=y, seed=6)  # noqa: E731
    sim = DiffSim(build(), dt, steps, checkpoint_every=50, damping=damping)
    rng = np.random.default_rng(21)
    v0 = (np.tile([0.0, -2.0], (sim.N, 1)) + 0.3 * rng.standard_normal((sim.N, 2))).astype(np.float32)
    w = rng.standard_normal((sim.N, 2))
    sim.forward(sim.E0, v0)
    eb, vb, _ = sim.backward(w)
    for kind in ("E", "v", "both"):
        dE = (sim.E0 * rng.standard_normal(sim.E)).astype(np.float32) if kind != "v" else np.zeros(sim.E, np.float32)
        dv = rng.standard_normal((sim.N, 2)).astype(np.float32) if kind != "E" else np.zeros((sim.N, 2), np.float32)
        _, dx = sim.jvp(sim.E0, v0, dE, dv)
        tangent = float(np.sum(w * dx.astype(np.float64)))
        a_e = float(np.dot(eb.astype(np.float64), dE))
        a_v = float(np.sum(vb.astype(np.float64) * dv))
        err = abs(tangent - (a_e + a_v)) / (abs(a_e) + abs(a_v))
        print(f"dot-product test ({kind}, damping {damping}): tangent {tangent:.9e} adjoint {a_e + a_v:.9e} rel {err:.2e}")
        assert err < 1e-5, (kind, tangent, a_e + a_v)


def test_resident_reverse_pass_equals_gather_reverse_pass():
    """The resident recompute + reverse (one cooperative launch each per
    segment) and the gather ones give the same bits, with contact and damping."""
    dt, steps = 1e-4, 300
    build = lambda: scenes.gradient_block_scene(fw, n=12, side=0.12, bottom=0.02, seed=8)  # noqa: E731
    a = DiffSim(build(), dt, steps, checkpoint_every=50, damping=0.03)
    b = DiffSim(build(), dt, steps, checkpoint_every=50, damping=0.03, path="gather")
    assert a.native.get_path()[0] == 2 and b.native.get_path()[0] == 1
    rng = np.random.default_rng(3)
    v0 = (np.tile([0.0, -2.0], (a.N, 1)) + 0.3 * rng.standard_normal((a.N, 2))).astype(np.float32)
    w = rng.standard_normal((a.N, 2)).astype(np.float32)
    xa = a.forward(a.E0, v0)
    xb_ = b.forward(b.E0, v0)
    assert np.array_equal(xa, xb_)
    for u, v in zip(a.backward(w), b.backward(w)):
        assert np.array_equal(u, v)


def test_checkpoint_interval_does_not_change_gradients():
    build = lambda: scenes.gradient_block_scene(fw, n=10, side=0.1, bottom=0.03, seed=2)  # noqa: E731
    a = DiffSim(build(), 1e-4, 300, checkpoint_every=50)
    b = DiffSim(build(), 1e-4, 300, checkpoint_every=300)
    v0 = np.tile(np.array([0.0, -1.5], np.float32), (a.N, 1))
    xa = a.forward(a.E0, v0)
    xb = b.forward(b.E0, v0)
    assert np.array_equal(xa, xb)
    ga = a.backward(xa)
    gb = b.backward(xb)
    for u, w in zip(ga, gb):
        assert np.array_equal(u, w)


def test_torch_autograd_function():
    import torch

    from flatworld_b200.diff import FEMRollout

    sim = DiffSim(scenes.gradient_block_scene(fw, n=8, side=0.08, bottom=0.02, seed=3), 1e-4, 200, checkpoint_every=50)
    E = torch.tensor(sim.E0, device="cuda", requires_grad=True)
    v0 = torch.tensor(np.tile([0.0, -1.0], (sim.N, 1)).astype(np.float32), device="cuda", requires_grad=True)
    x = FEMRollout.apply(E, v0, sim)
    loss = (x ** 2).sum()
    loss.backward()
    eb, vb, _ = sim.backward(2.0 * x.detach().cpu().numpy())
    assert np.allclose(E.grad.cpu().numpy(), eb) and np.allclose(v0.grad.cpu().numpy(), vb)
    assert torch.isfinite(E.grad).all() and E.grad.abs().sum() > 0


@pytest.mark.parametrize("kind", ["plane", "heightfield", "voxel", "j2"])
def test_gpu_adjoint_against_fp64_oracle_adjoint(kind):
    """The CUDA adjoint (FP32 trajectory) against the oracle's FP64 adjoint
    (FP64 trajectory; itself equal to FP64 central differences to 1e-6,
    tests/test_oracle_adjoint.py) on a 12 x 12 block landing on a plane, a
    height field and a voxel floor (contact with its velocity damping), and a
    J2 block that yields on the plane (plastic state carried backward), for
    L = <w, x_T> over 400 substeps.  What separates them is the FP32
    trajectory's rounding; the tolerance is stated on the L2 norm of dL/dE and
    dL/dv0."""
    from tests.test_oracle_adjoint import DT, STEPS, block

    build = block(kind)
    doms = build()
    sim = DiffSim(doms, DT, STEPS, checkpoint_every=50, path="gather")
    o = oracle.OracleLoop(build(), DT, useAdapativeDT=False, precision="f64")
    _, v0, _ = o.state()
    w = np.random.default_rng(7).standard_normal((sim.N, 2))
    _, vb64, eb64 = o.adjoint(STEPS, xbar=w)
    sim.forward(sim.E0, v0.astype(np.float32))
    eb, vb, _ = sim.backward(w)
    e_err = float(np.linalg.norm(eb - eb64) / np.linalg.norm(eb64))
    v_err = float(np.linalg.norm(vb - vb64) / np.linalg.norm(vb64))
    print(f"{kind}: CUDA adjoint vs FP64 adjoint: dL/dE {e_err:.2e}, dL/dv0 {v_err:.2e} (relative L2)")
    assert e_err < 1e-2 and v_err < 1e-2, (e_err, v_err)


@pytest.mark.parametrize("kind", ["heightfield", "voxel"])
def test_adjoint_is_the_transpose_of_the_tangent_with_ground_contact(kind):
    """Dot-product test with height-field and voxel contact (penetration and
    velocity-damping terms), with loop damping, on one FP32 trajectory."""
    from tests.test_oracle_adjoint import DT, STEPS, block

    sim = DiffSim(block(kind)(), DT, STEPS, checkpoint_every=50, damping=0.02)
    rng = np.random.default_rng(31)
    v0 = np.tile(np.array([0.3, -1.0], np.float32), (sim.N, 1))
    w = rng.standard_normal((sim.N, 2))
    sim.forward(sim.E0, v0)
    eb, vb, _ = sim.backward(w)
    for what in ("E", "v"):
        dE = (sim.E0 * rng.standard_normal(sim.E)).astype(np.float32) if what == "E" else np.zeros(sim.E, np.float32)
        dv = rng.standard_normal((sim.N, 2)).astype(np.float32) if what == "v" else np.zeros((sim.N, 2), np.float32)
        _, dx = sim.jvp(sim.E0, v0, dE, dv)
        tangent = float(np.sum(w * dx.astype(np.float64)))
        a = float(np.dot(eb.astype(np.float64), dE)) + float(np.sum(vb.astype(np.float64) * dv))
        err = abs(tangent - a) / max(abs(a), 1e-30)
        print(f"dot-product test ({kind}, {what}): tangent {tangent:.9e} adjoint {a:.9e} rel {err:.2e}")
        assert err < 1e-5, (kind, what, tangent, a)


@pytest.mark.parametrize("kind", ["heightfield", "voxel"])
def test_resident_reverse_equals_gather_reverse_with_ground_contact(kind):
    from tests.test_oracle_adjoint import DT, STEPS, block

    a = DiffSim(block(kind)(), DT, STEPS, checkpoint_every=50, damping=0.03)
    b = DiffSim(block(kind)(), DT, STEPS, checkpoint_every=50, damping=0.03, path="gather")
    assert a.native.get_path()[0] == 2 and b.native.get_path()[0] == 1
    v0 = np.tile(np.array([0.3, -1.0], np.float32), (a.N, 1))
    w = np.random.default_rng(4).standard_normal((a.N, 2)).astype(np.float32)
    assert np.array_equal(a.forward(a.E0, v0), b.forward(b.E0, v0))
    for u, v in zip(a.backward(w), b.backward(w)):
        assert np.array_equal(u, v)
