"""fw_step_noalloc: the allocation-free substep for callers that cannot call
cudaMalloc (a real-time loop where an allocation may block and synchronise the
device, or a process whose device memory belongs to its own pool allocator).

The caller owns every buffer (here torch tensors stand in for that caller's
memory); the library only uses its fixed, built-in scratch array.  The test
checks the result against the context entry point fw_step on the same world,
for two calls in a row (the second call finds the scratch array holding the
first call's values), within the suite's 1e-5 relative tolerance, and that a
mesh larger than the scratch limit is refused with a clear error.

This file is collected last so that a run stopping at the first failure has
run every other test already; it builds everything it uses, so it also passes
alone in a fresh process.
"""

import ctypes

import numpy as np
import pytest

import flatworld_b200 as fw
from flatworld_b200 import _native
from flatworld_b200.world import PackedWorld, SceneLayout, build_native

pytestmark = pytest.mark.gpu
RTOL = 1e-5
FW_NOALLOC_MAX_ELEMS = 131072


def _scene():
    conn, coords = fw.structured_rectangle(32, 8, 0.5, 0.125, origin=(0.0, 0.3), jitter=0.1, seed=1)
    a = fw.FemDomain(fw.Mesh(2, conn, coords), fw.SolidProp(fw.Elastic(2e4, 0.2, 40.0)),
                     [fw.Gravity([0, -1.0]), fw.Fixed([0, 1, 2])], considerContact=False)
    conn2, coords2 = fw.structured_rectangle(16, 8, 0.3, 0.15, origin=(0.7, 0.3), jitter=0.1, seed=2)
    b = fw.FemDomain(fw.Mesh(2, conn2, coords2), fw.SolidProp(fw.MisesPlastic(1e5, 0.3, 100.0, 2e3, 1e3)),
                     [fw.EnforceVel([0, 1], [0.0, -3.0]), fw.Gravity([0, -9.8])], considerContact=False,
                     initials=[fw.InitialVel("ALL", [0.5, -1.0])])
    return [a, b]


def _rel(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / max(np.abs(b).max(), 1e-30))


def test_noalloc_step_matches_context_step():
    import torch

    dt = 5e-5
    packed = PackedWorld([SceneLayout(_scene(), dt=dt, useAdapativeDT=False)])
    ref = build_native(packed, path="gather")  # the context entry point, fw_step
    N, E = packed.N, packed.E
    # state after construction (the zero-dt step the context runs in fw_finalize)
    x0 = ref.read_nodes(_native.FW_FIELD_X, 0, N)
    v0 = ref.read_nodes(_native.FW_FIELD_V, 0, N)
    mass = ref.read_nodes(_native.FW_FIELD_MASS, 0, N)
    area, jinv = ref.read_reference_shape(E)
    ep, eq = ref.read_plastic(E)
    one, two = np.float32(1.0), np.float32(2.0)
    Ev, nu = packed.Ev, packed.nuv
    lam = Ev * nu / ((one + nu) * (one - two * nu))
    mu = Ev / (two * (one + nu))
    elem_mat = np.stack([area, lam, mu, packed.mtype.astype(np.float32)], axis=1)
    counts = np.bincount(packed.conn.reshape(-1), minlength=N)
    csr_off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    order = np.argsort(packed.conn.reshape(-1), kind="stable")  # ascending element within a node
    csr_slot = order.astype(np.int32)
    j2p = np.stack([packed.syv, packed.Hv], axis=1).astype(np.float32)
    j2s = np.concatenate([ep, eq[:, None]], axis=1).astype(np.float32)

    dev = torch.device("cuda", 0)
    T = lambda a, dt_: torch.from_numpy(np.ascontiguousarray(a, dtype=dt_)).to(dev)  # noqa: E731
    x, v = T(x0, np.float32), T(v0, np.float32)
    bufs = dict(bc=T(packed.bc_bits, np.int32), bcv=T(packed.bc_vals, np.float32), m=T(mass, np.float32),
                conn=T(packed.conn, np.int32), jinv=T(jinv, np.float32), mat=T(elem_mat, np.float32),
                j2s=T(j2s, np.float32), j2p=T(j2p, np.float32), off=T(csr_off, np.int32),
                slot=T(csr_slot, np.int32))
    L = _native.lib()
    err = ctypes.create_string_buffer(256)
    for call in range(2):
        rc = L.fw_step_noalloc(N, E, 40, float(np.float32(dt)), 0.0, x.data_ptr(), v.data_ptr(),
                               bufs["bc"].data_ptr(), bufs["bcv"].data_ptr(), bufs["m"].data_ptr(),
                               bufs["conn"].data_ptr(), bufs["jinv"].data_ptr(), bufs["mat"].data_ptr(),
                               bufs["j2s"].data_ptr(), bufs["j2p"].data_ptr(), bufs["off"].data_ptr(),
                               bufs["slot"].data_ptr(), None, err, len(err))
        assert rc == 0, err.value.decode()
        torch.cuda.synchronize()
        ref.step(40, dt)
        xr = ref.read_nodes(_native.FW_FIELD_X, 0, N)
        vr = ref.read_nodes(_native.FW_FIELD_V, 0, N)
        xn, vn = x.cpu().numpy(), v.cpu().numpy()
        assert _rel(xn, xr) <= RTOL and _rel(vn, vr) <= RTOL, (call, _rel(xn, xr), _rel(vn, vr))
        _, eq_r = ref.read_plastic(E)
        assert _rel(bufs["j2s"].cpu().numpy()[:, 3], eq_r) <= RTOL
    assert float(eq_r.max()) > 0.0  # the J2 body yielded
    ref.close()


def test_noalloc_rejects_meshes_beyond_the_scratch_limit():
    L = _native.lib()
    err = ctypes.create_string_buffer(256)
    rc = L.fw_step_noalloc(10, FW_NOALLOC_MAX_ELEMS + 1, 1, 1e-4, 0.0, *([None] * 12), None, err, len(err))
    assert rc == -1 and b"scratch limit" in err.value
