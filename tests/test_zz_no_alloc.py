"""fw_step_noalloc: the allocation-free substep for callers that cannot call
cudaMalloc (a real-time loop where an allocation may block and synchronise the
device, or a process whose device memory belongs to its own pool allocator).

The caller owns every buffer (here torch tensors stand in for that caller's
memory); the library only uses its fixed, built-in scratch array.  The main
test checks the result against the context entry point fw_step on the same
world, bit for bit (both run the same arithmetic in the same order), for two
calls in a row (the second call finds the scratch array holding the first
call's values).  The others check the documented edge behaviour: J2 triangles
without state arrays respond elastically, a record that is not a triangle adds
no force, and bad arguments are refused with a clear error.

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
DT = 5e-5


def _scene(j2_material=True):
    conn, coords = fw.structured_rectangle(32, 8, 0.5, 0.125, origin=(0.0, 0.3), jitter=0.1, seed=1)
    a = fw.FemDomain(fw.Mesh(2, conn, coords), fw.SolidProp(fw.Elastic(2e4, 0.2, 40.0)),
                     [fw.Gravity([0, -1.0]), fw.Fixed([0, 1, 2])], considerContact=False)
    conn2, coords2 = fw.structured_rectangle(16, 8, 0.3, 0.15, origin=(0.7, 0.3), jitter=0.1, seed=2)
    mat = fw.MisesPlastic(1e5, 0.3, 100.0, 2e3, 1e3) if j2_material else fw.Elastic(1e5, 0.3, 100.0)
    b = fw.FemDomain(fw.Mesh(2, conn2, coords2), fw.SolidProp(mat),
                     [fw.EnforceVel([0, 1], [0.0, -3.0]), fw.Gravity([0, -9.8])], considerContact=False,
                     initials=[fw.InitialVel("ALL", [0.5, -1.0])])
    return [a, b]


def _rel(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / max(np.abs(b).max(), 1e-30))


class _Caller:
    """What a caller of fw_step_noalloc holds: every input and output as its
    own device memory, filled from a context world after construction."""

    def __init__(self, packed, ref, extra_records=0):
        import torch

        N, E = packed.N, packed.E
        self.N, self.E = N, E + extra_records
        x0 = ref.read_nodes(_native.FW_FIELD_X, 0, N)
        v0 = ref.read_nodes(_native.FW_FIELD_V, 0, N)
        mass = ref.read_nodes(_native.FW_FIELD_MASS, 0, N)
        area, jinv = ref.read_reference_shape(E)
        ep, eq = ref.read_plastic(E)
        # Lame constants with the reference's float32 formula and operation
        # order (materialfunctions.py:12-13), as the context computes them
        one, two = np.float32(1.0), np.float32(2.0)
        Ev, nu = packed.Ev.astype(np.float32), packed.nuv.astype(np.float32)
        lam = Ev * nu / ((one + nu) * (one - two * nu))
        mu = Ev / (two * (one + nu))
        elem_mat = np.stack([area, lam, mu, packed.mtype.astype(np.float32)], axis=1)
        conn = packed.conn.astype(np.int32)
        counts = np.bincount(conn.reshape(-1), minlength=N)
        csr_off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
        csr_slot = np.argsort(conn.reshape(-1), kind="stable").astype(np.int32)  # ascending element per node
        j2p = np.stack([packed.syv, packed.Hv], axis=1).astype(np.float32)
        j2s = np.concatenate([ep, eq[:, None]], axis=1).astype(np.float32)
        if extra_records:
            # spring-like records (type 0, third node -1) after the triangles;
            # no node's CSR list names their corners
            conn = np.concatenate([conn, np.tile(np.array([[0, 1, -1]], np.int32), (extra_records, 1))])
            elem_mat = np.concatenate([elem_mat, np.tile(np.array([[1.0, 1.0, 1.0, 0.0]], np.float32),
                                                         (extra_records, 1))])
            jinv = np.concatenate([jinv, np.zeros((extra_records, 4), np.float32)])
            j2p = np.concatenate([j2p, np.zeros((extra_records, 2), np.float32)])
            j2s = np.concatenate([j2s, np.zeros((extra_records, 4), np.float32)])
        dev = torch.device("cuda", 0)
        T = lambda a, t: torch.from_numpy(np.ascontiguousarray(a, dtype=t)).to(dev)  # noqa: E731
        self.x, self.v = T(x0, np.float32), T(v0, np.float32)
        self.b = dict(bc=T(packed.bc_bits, np.int32), bcv=T(packed.bc_vals, np.float32), m=T(mass, np.float32),
                      conn=T(conn, np.int32), jinv=T(jinv, np.float32), mat=T(elem_mat, np.float32),
                      j2s=T(j2s, np.float32), j2p=T(j2p, np.float32), off=T(csr_off, np.int32),
                      slot=T(csr_slot, np.int32))

    def step(self, n, with_j2=True):
        import torch

        L = _native.lib()
        err = ctypes.create_string_buffer(256)
        b = self.b
        j2s = b["j2s"].data_ptr() if with_j2 else None
        j2p = b["j2p"].data_ptr() if with_j2 else None
        rc = L.fw_step_noalloc(self.N, self.E, n, float(np.float32(DT)), 0.0, self.x.data_ptr(),
                               self.v.data_ptr(), b["bc"].data_ptr(), b["bcv"].data_ptr(), b["m"].data_ptr(),
                               b["conn"].data_ptr(), b["jinv"].data_ptr(), b["mat"].data_ptr(), j2s, j2p,
                               b["off"].data_ptr(), b["slot"].data_ptr(), None, err, len(err))
        assert rc == 0, err.value.decode()
        torch.cuda.synchronize()
        return self.x.cpu().numpy(), self.v.cpu().numpy()


def _context(j2_material=True):
    packed = PackedWorld([SceneLayout(_scene(j2_material), dt=DT, useAdapativeDT=False)])
    return packed, build_native(packed, path="gather")  # the context entry point, fw_step


def test_noalloc_step_matches_context_step():
    packed, ref = _context()
    caller = _Caller(packed, ref)
    for call in range(2):
        xn, vn = caller.step(40)
        ref.step(40, DT)
        xr = ref.read_nodes(_native.FW_FIELD_X, 0, packed.N)
        vr = ref.read_nodes(_native.FW_FIELD_V, 0, packed.N)
        assert np.array_equal(xn, xr) and np.array_equal(vn, vr), (call, _rel(xn, xr), _rel(vn, vr))
        _, eq_r = ref.read_plastic(packed.E)
        assert np.array_equal(caller.b["j2s"].cpu().numpy()[:, 3], eq_r), call
    assert float(eq_r.max()) > 0.0  # the J2 body yielded
    ref.close()


def test_noalloc_j2_without_state_arrays_is_elastic():
    """With j2_state = j2_param = NULL the J2 triangles never yield: the
    result equals the context step on the same world with the J2 material
    replaced by Elastic of the same E, nu, rho (within the suite's tolerance)."""
    packed, ref = _context(j2_material=True)
    caller = _Caller(packed, ref)
    ref.close()
    packed_el, ref_el = _context(j2_material=False)
    xn, vn = caller.step(80, with_j2=False)
    ref_el.step(80, DT)
    xr = ref_el.read_nodes(_native.FW_FIELD_X, 0, packed_el.N)
    vr = ref_el.read_nodes(_native.FW_FIELD_V, 0, packed_el.N)
    assert _rel(xn, xr) <= RTOL and _rel(vn, vr) <= RTOL, (_rel(xn, xr), _rel(vn, vr))
    ref_el.close()


def test_noalloc_non_triangle_records_add_no_force():
    packed, ref = _context()
    plain = _Caller(packed, ref)
    extra = _Caller(packed, ref, extra_records=5)
    xa, va = plain.step(30)
    xb, vb = extra.step(30)
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)
    ref.close()


def test_noalloc_rejects_bad_arguments():
    L = _native.lib()
    err = ctypes.create_string_buffer(256)
    rc = L.fw_step_noalloc(10, FW_NOALLOC_MAX_ELEMS + 1, 1, 1e-4, 0.0, *([None] * 12), None, err, len(err))
    assert rc == -1 and b"scratch limit" in err.value
    fake = ctypes.c_void_p(16)  # never dereferenced: the call is refused before any launch
    args = [fake] * 8 + [fake, None] + [fake] * 2  # j2_state given, j2_param NULL
    rc = L.fw_step_noalloc(10, 4, 1, 1e-4, 0.0, *args, None, err, len(err))
    assert rc == -1 and b"both be given or both be NULL" in err.value
