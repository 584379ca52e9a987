"""Differentiable form: gradients of a rollout w.r.t. per-element Young's
modulus and initial velocities, by a hand-written adjoint of the FEM substep
(csrc/fw_adjoint.cuh) with checkpoint-and-recompute.

    sim = DiffSim(domains, dt=1e-4, n_steps=2000, checkpoint_every=50)
    x_T = FEMRollout.apply(E, v0, sim)       # torch tensors, E per triangle, v0 per node
    loss = ((x_T - target) ** 2).sum(); loss.backward()   # E.grad, v0.grad

Forward: the rollout runs on the GPU (the resident step when the mesh fits on
chip, else the gather step) and stores the state at
the start of every segment of ``checkpoint_every`` substeps (fw_snapshot).
Backward: for each segment, last first, the checkpoint is restored, the
segment is recomputed with its positions and broad-phase gates recorded, and
the substeps are reversed (fw_adj_segment).  Memory: one state per segment
plus one segment of positions.

The reference has no differentiation (no Warp tape; its kernels write state
in place, flatworld/femspringmanager.py:355-358).
"""

from __future__ import annotations

import numpy as np

from . import _native
from .world import PackedWorld, SceneLayout, build_native


class DiffSim:
    """A single-scene rollout of ``n_steps`` substeps of ``dt`` with its adjoint."""

    def __init__(self, domains, dt, n_steps, checkpoint_every=50, device=0, damping=0.0, path="auto"):
        self.layout = SceneLayout(domains, dt=dt, damping=damping, useAdapativeDT=False)
        if self.layout.entries:
            raise NotImplementedError("the adjoint covers FEM triangles; rigid bodies and ground planes with BCs "
                                      "are not differentiated")
        self.packed = PackedWorld([self.layout])
        # forward, recompute and reverse on the resident step when the mesh
        # (and the adjoint state) fits on chip; otherwise on the gather step --
        # the same bits either way
        self.native = build_native(self.packed, device=device, path=path)
        self.N, self.E = self.packed.N, self.packed.E
        self.dt = float(np.float32(dt))
        self.n_steps = int(n_steps)
        self.K = int(checkpoint_every)
        self.segments = [(s, min(self.K, self.n_steps - s)) for s in range(0, self.n_steps, self.K)]
        self.native.adj_begin(self.K)
        self.native.snapshot(0)  # state after construction (the zero-dt step)
        self.E0 = self.packed.Ev.copy()

    def forward(self, young, v0):
        """Run the rollout from the construction state with per-triangle moduli
        ``young`` and initial velocities ``v0`` (N x 2); return x_T (N x 2)."""
        self.native.set_element_young(np.asarray(young, np.float32))
        self.native.restore(0)
        self.native.write_nodes(_native.FW_FIELD_V, 0, np.asarray(v0, np.float32).reshape(self.N, 2))
        for i, (_, n) in enumerate(self.segments):
            self.native.snapshot(1 + i)
            self.native.step(n, self.dt)
        return self.native.read_nodes(_native.FW_FIELD_X, 0, self.N)

    def jvp(self, young, v0, dE=None, dv0=None):
        """Forward-mode derivative of the rollout: (x_T, dx_T) along the
        moduli direction dE (per triangle) and velocity direction dv0."""
        self.native.set_element_young(np.asarray(young, np.float32))
        self.native.restore(0)
        self.native.write_nodes(_native.FW_FIELD_V, 0, np.asarray(v0, np.float32).reshape(self.N, 2))
        self.native.tan_begin(None, None if dv0 is None else np.asarray(dv0, np.float32).reshape(self.N, 2),
                              None if dE is None else np.asarray(dE, np.float32))
        self.native.tan_step(self.n_steps, self.dt)
        x = self.native.read_nodes(_native.FW_FIELD_X, 0, self.N)
        dx, _ = self.native.tan_read(self.N)
        return x, dx

    def backward(self, xbar_T, vbar_T=None):
        """Reverse the last forward rollout from dL/dx_T (and dL/dv_T);
        returns (dL/dE per triangle, dL/dv0 per node, dL/dx0 per node)."""
        self.native.adj_seed(np.asarray(xbar_T, np.float32).reshape(self.N, 2),
                             None if vbar_T is None else np.asarray(vbar_T, np.float32).reshape(self.N, 2))
        for i in reversed(range(len(self.segments))):
            self.native.restore(1 + i)
            self.native.adj_segment(self.segments[i][1], self.dt)
        xb, vb, eb = self.native.adj_read(self.N, self.E)
        return eb, vb, xb


try:
    import torch

    class FEMRollout(torch.autograd.Function):
        """x_T = rollout(E, v0) as an autograd op (E per triangle, v0 per node)."""

        @staticmethod
        def forward(ctx, young, v0, sim):
            ctx.young = young.detach().cpu().numpy()
            ctx.v0 = v0.detach().cpu().numpy()
            ctx.device = young.device
            x = sim.forward(ctx.young, ctx.v0)
            ctx.sim = sim
            return torch.from_numpy(x).to(young.device)

        @staticmethod
        def backward(ctx, grad_x):
            eb, vb, _ = ctx.sim.backward(grad_x.detach().cpu().numpy())
            dev = grad_x.device
            return torch.from_numpy(eb).to(dev), torch.from_numpy(vb).to(dev), None

        @staticmethod
        def jvp(ctx, young_t, v0_t, sim_t):
            """Forward-mode AD (torch.func.jvp / forward_ad) through the tangent."""
            sim = ctx.sim
            _, dx = sim.jvp(ctx.young, ctx.v0, None if young_t is None else young_t.detach().cpu().numpy(),
                            None if v0_t is None else v0_t.detach().cpu().numpy())
            return torch.from_numpy(dx).to(ctx.device)

except ImportError:  # pragma: no cover
    FEMRollout = None


def lognormal_young(n, mean=1e5, sigma=0.3, seed=0):
    """Per-element moduli, log-normal with the given mean and log-std."""
    rng = np.random.default_rng(seed)
    mu = np.log(mean) - 0.5 * sigma * sigma
    return np.exp(mu + sigma * rng.standard_normal(n)).astype(np.float32)
