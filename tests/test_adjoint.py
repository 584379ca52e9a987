"""Differentiable form (GPU): adjoint gradients of a rollout w.r.t.
per-element Young's modulus and initial velocities, checked against central
finite differences of the FP64 oracle along random directions."""

import numpy as np
import pytest

import flatworld_b200 as fw
import oracle
from flatworld_b200.diff import DiffSim
from tests import scenes

pytestmark = pytest.mark.gpu


def fd_loss64(domains_fn, young, v0, steps, dt, target):
    doms = domains_fn(young)
    o = oracle.OracleLoop(doms, dt, useAdapativeDT=False, precision="f64", threads=8)
    o.set_state(None, v0)
    o.advance(steps)
    x, _, _ = o.state()
    return float(np.sum((x - target) ** 2))


@pytest.mark.parametrize("n,steps", [(12, 600)])
def test_adjoint_matches_fp64_central_differences(n, steps):
    dt = 1e-4
    build = lambda y=None: scenes.gradient_block_scene(fw, n=n, side=0.12, bottom=0.04, young=y, seed=1)  # noqa: E731
    sim = DiffSim(build(), dt, steps, checkpoint_every=50)
    E0 = sim.E0.copy()
    v0 = np.tile(np.array([0.0, -2.0], np.float32), (sim.N, 1))
    target = sim.forward(E0 * 1.1, v0).astype(np.float64)
    xT = sim.forward(E0, v0)
    assert xT[:, 1].min() < 0.005, "the block must touch the plane"
    eb, vb, _ = sim.backward(2.0 * (xT - target))
    rng = np.random.default_rng(0)
    errs = []
    for _ in range(4):
        dE = E0 * rng.standard_normal(sim.E).astype(np.float32)
        dv = rng.standard_normal((sim.N, 2)).astype(np.float32)
        adj = float(np.dot(eb.astype(np.float64), dE) + np.sum(vb.astype(np.float64) * dv))
        eps = 1e-4
        lp = fd_loss64(build, (E0 + eps * dE).astype(np.float64), v0 + eps * dv, steps, dt, target)
        lm = fd_loss64(build, (E0 - eps * dE).astype(np.float64), v0 - eps * dv, steps, dt, target)
        fd = (lp - lm) / (2 * eps)
        errs.append(abs(adj - fd) / max(abs(fd), 1e-30))
    print("relative error of directional derivatives:", errs)
    assert max(errs) < 2e-2, errs


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
