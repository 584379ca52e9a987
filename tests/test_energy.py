"""Total energy, reduced in FP64 on the GPU (fw_energy), checked against an
independent numpy FP64 restatement evaluated on the GPU's own state, plus
conservation and determinism checks."""

import numpy as np
import pytest

import flatworld_b200 as fw
import oracle
from flatworld_b200.batch import BatchedLoop
from tests import scenes

pytestmark = pytest.mark.gpu
FRAME = 1.0 / 60.0


def numpy_energy(loop, build):
    """Kinetic, strain, external and contact energy of scene 0 in numpy FP64
    from the GPU state (positions, velocities, J2 state) and the prepared
    masses / areas / inverse reference shapes (bit-identical to the GPU's)."""
    pk = loop._packed
    n = pk.N
    x = loop._native.read_nodes(fw._native.FW_FIELD_X, 0, n).astype(np.float64)
    v = loop._native.read_nodes(fw._native.FW_FIELD_V, 0, n).astype(np.float64)
    mass, area, jinv = oracle.OracleLoop(build(), 0.0, useAdapativeDT=True).prepared()
    ke = 0.5 * np.sum(mass * np.sum(v * v, axis=1))
    bc = pk.bc_bits
    grav = ((bc & 0x10) != 0) & ((bc & 0x5) == 0)
    ext = -np.sum(mass[grav] * np.sum(pk.bc_vals[grav].astype(np.float64) * x[grav], axis=1))
    # strain energy per triangle; Lame constants in FP32 as the device prepares them
    E32, nu32 = pk.Ev.astype(np.float32), pk.nuv.astype(np.float32)
    one, two = np.float32(1.0), np.float32(2.0)
    lam = ((E32 * nu32) / ((one + nu32) * (one - two * nu32))).astype(np.float64)
    mu = (E32 / (two * (one + nu32))).astype(np.float64)
    c = pk.conn.reshape(-1, 3)
    a, b, cc = x[c[:, 0]], x[c[:, 1]], x[c[:, 2]]
    ji = jinv.reshape(-1, 4)
    j00, j01 = a[:, 0] - cc[:, 0], b[:, 0] - cc[:, 0]
    j10, j11 = a[:, 1] - cc[:, 1], b[:, 1] - cc[:, 1]
    F00, F01 = j00 * ji[:, 0] + j01 * ji[:, 2], j00 * ji[:, 1] + j01 * ji[:, 3]
    F10, F11 = j10 * ji[:, 0] + j11 * ji[:, 2], j10 * ji[:, 1] + j11 * ji[:, 3]
    C00, C01, C11 = F00 ** 2 + F10 ** 2, F00 * F01 + F10 * F11, F01 ** 2 + F11 ** 2
    e0, e1, e2 = 0.5 * (C00 - 1.0), 0.5 * (C11 - 1.0), 0.5 * C01
    j2 = pk.mtype == 3
    if j2.any():
        ep, _ = loop._native.read_plastic(pk.E)
        e0 = e0 - np.where(j2, ep[:, 0], 0.0)
        e1 = e1 - np.where(j2, ep[:, 1], 0.0)
        e2 = e2 - np.where(j2, ep[:, 2], 0.0)
    W = 0.5 * lam * (e0 + e1) ** 2 + mu * (e0 ** 2 + e1 ** 2 + 2.0 * e2 ** 2)
    nh = pk.mtype == 2
    lj = np.log(np.where(nh, F00 * F11 - F01 * F10, 1.0))
    W = np.where(nh, 0.5 * mu * (C00 + C11 - 2.0) - mu * lj + 0.5 * lam * lj ** 2, W)
    strain = float(np.sum(area * W))
    # plane penalty from the FP32 force, as on the device
    x32 = x.astype(np.float32)
    pen_e = 0.0
    for kind, body, k, _lo, _hi, g in pk.pair_records():
        assert kind == "plane"
        k = np.float32(k)
        nodes = pk.bnodes[pk.bnoff[body]: pk.bnoff[body] + pk.bncnt[body]]
        p0, p1 = np.float32(g.point[0]), np.float32(g.point[1])
        n0, n1 = np.float32(g.normal[0]), np.float32(g.normal[1])
        pen = (x32[nodes, 0] - p0) * n0 + (x32[nodes, 1] - p1) * n1
        pen = pen[pen < 0]
        fx, fy = -(n0 * k * pen), -(n1 * k * pen)
        pen_e += float(np.sum(0.5 * (fx.astype(np.float64) ** 2 + fy.astype(np.float64) ** 2) / np.float64(k)))
    return np.array([ke, strain, ext, pen_e])


def test_energy_matches_numpy_fp64_all_laws_with_contact():
    """Three blocks (Elastic, NeoHookean, J2) falling onto a plane: every term
    of the device reduction equals the numpy FP64 restatement to summation
    order (1e-12 relative), once the blocks penetrate the plane."""
    build = lambda: scenes.multi_block_scene(fw, 3)  # noqa: E731
    for path in ("gather", "resident"):
        loop = fw.ExplicitLoop(0.0, build(), useAdapativeDT=True, path=path)
        for _ in range(6):
            loop.advanceWithTime(FRAME)
        gpu = loop.energy()
        ref = numpy_energy(loop, build)
        got = np.array([gpu["kinetic"], gpu["strain"], gpu["external"], gpu["contact"]])
        assert ref[3] > 0.0, "the blocks must penetrate the plane"
        assert ref[1] > 0.0 and ref[0] > 0.0
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=0.0)
        assert gpu["total"] == pytest.approx(got.sum(), rel=1e-15)


def vibrating_block(n=16):
    """NeoHookean block, no gravity, no ground, smooth initial velocity field
    (a shear wave plus a bending-like mode, peak 0.3 m/s)."""
    conn, coords = fw.structured_rectangle(n, n, 0.2, 0.2, origin=(0.4, 0.4))
    xc = (coords - coords.mean(axis=0)) / 0.1
    v0 = np.stack([0.3 * np.sin(0.5 * np.pi * xc[:, 1]), 0.3 * xc[:, 0] * xc[:, 1]], axis=1)
    ics = [fw.InitialVel([i], v0[i]) for i in range(coords.shape[0])]
    return [fw.FemDomain(fw.Mesh(2, conn, coords), fw.SolidProp(fw.HyperElastic(E=1e5, nu=0.3, rho=1000.0)), [],
                         initials=ics)]


def test_energy_is_conserved_in_free_flight():
    """No gravity, no contact, no damping: over 80 ms (about four vibration
    periods) symplectic Euler at the static CFL step keeps the total energy
    within 5% of its start (measured: 1.9%), while energy moves between its
    kinetic and strain parts."""
    loop = fw.ExplicitLoop(0.0, vibrating_block(), useAdapativeDT=True)
    e0 = loop.energy()
    assert e0["kinetic"] > 0.0 and e0["strain"] < 1e-9 * e0["kinetic"]  # rest shape (F = I up to FP32 rounding)
    totals, strains = [], []
    for _ in range(20):
        loop.advanceWithTime(FRAME / 4)
        e = loop.energy()
        totals.append(e["total"])
        strains.append(e["strain"])
    drift = max(abs(t - e0["total"]) for t in totals) / e0["total"]
    print(f"free-flight energy: start {e0['total']:.6f} J, max relative deviation {drift:.2e}")
    assert max(strains) > 0.1 * e0["total"], "energy must move between kinetic and strain"
    assert drift < 5e-2


def test_energy_deterministic_and_same_in_batch():
    """Two calls give the same bits; a scene's energies in a batch equal the
    same scene's energies stepped alone."""
    build = lambda: [scenes.multi_block_scene(fw, 3), scenes.plain_small_scene(fw)]  # noqa: E731
    b = BatchedLoop(build(), dt=1e-4, useAdapativeDT=False)
    b.advance(400)
    e1, e2 = b.energies(), b.energies()
    assert np.array_equal(e1, e2)
    for s, doms in enumerate(build()):
        lp = fw.ExplicitLoop(1e-4, doms, useAdapativeDT=False, path="gather")
        lp.advance_n(400)
        e = lp.energy()
        assert np.array_equal(e1[s], [e["kinetic"], e["strain"], e["external"], e["contact"]]), s
