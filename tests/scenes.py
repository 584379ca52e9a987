"""Scene builders shared by the tests and the benchmark (seeded, synthetic).

The small scenes restate the reference's own test fixtures
(test2D/test_2Dfem_elastic.py:17-25, test_2Dfem_elastic10000.py:17-32,
test_2Dfem_force.py:17-24, test_2Dfem_heightfield_contact.py:14-46,
test_2Dfem_voxel_contact.py:14-50); the large ones follow the benchmark
workload descriptions (plain small / large mesh, ragged batch, gradient block).
"""

from __future__ import annotations

import numpy as np


def two_triangle_square(fw, bcs_fn=None, mat=None):
    conn = np.array([[0, 1, 3], [0, 3, 2]], dtype=np.int32)
    coords = np.array([[0.5, 0.5], [0.7, 0.5], [0.5, 0.7], [0.7, 0.7]], dtype=np.float32)
    mesh = fw.Mesh(2, conn, coords)
    mat = mat or fw.Elastic(E=2e4, nu=0.2, rho=40.0)
    bcs = bcs_fn() if bcs_fn else [fw.Gravity([0, -1.0])]
    return fw.FemDomain(mesh, fw.SolidProp(mat), bcs)


def elastic10000_mesh(fw, num_el=100):
    """test_2Dfem_elastic10000.py:17-32, loop for loop."""
    dx = 0.6 / num_el
    conn = np.zeros((2 * num_el * num_el, 3), dtype=np.int32)
    coords = np.zeros(((num_el + 1) * (num_el + 1), 2), dtype=np.float32)
    nd = 0
    for i in range(num_el + 1):
        for j in range(num_el + 1):
            coords[nd] = np.array([dx * i, dx * j])
            nd += 1
    el = 0
    for i in range(num_el):
        for j in range(num_el):
            conn[el] = [i * (num_el + 1) + j, i * (num_el + 1) + j + 1, (i + 1) * (num_el + 1) + j]
            conn[el + 1] = [i * (num_el + 1) + j + 1, (i + 1) * (num_el + 1) + j + 1, (i + 1) * (num_el + 1) + j]
            el += 2
    return fw.Mesh(2, conn, coords + 0.3)


def heightfield_bowl(nx=513, cx=0.5, r=0.5, zc=0.7):
    xs = np.linspace(0.0, 1.0, nx, dtype=np.float32)
    h = np.empty(nx, dtype=np.float32)
    for i, x in enumerate(xs):
        dx = x - cx
        inside = r * r - dx * dx
        h[i] = zc - np.sqrt(inside) if inside >= 0.0 else zc
    return h


def voxel_pit(nx=160, ny=100):
    occ = np.zeros((nx, ny), dtype=np.int32)
    cx = nx * 0.5
    r = nx * 0.45
    max_h = int(ny * 0.55)
    for i in range(nx):
        dx = i - cx
        inside = r * r - dx * dx
        if inside > 0:
            depth = inside / (r * r)
            h = int(max_h * (1.3 - depth))
        else:
            h = max_h
        if h > 0:
            occ[i, :h] = 1
    return occ


def hf_disk_scene(fw):
    mesh = fw.FEMesher(2).createCircle([0.5, 0.65], 0.1)
    fem = fw.FemDomain(mesh, fw.SolidProp(fw.Elastic(E=2e4, nu=0.2, rho=40.0)), [fw.Gravity([0.0, -10.0])],
                       considerContact=True, initials=[])
    hf = fw.HeightFieldDomain(2, heightfield_bowl(), lb=[0.0, 0.0], ub=[1.0, 1.0], considerContact=True)
    return [hf, fem]


def voxel_disk_scene(fw):
    mesh = fw.FEMesher(2).createCircle([0.5, 0.75], 0.07)
    fem = fw.FemDomain(mesh, fw.SolidProp(fw.Elastic(E=2e4, nu=0.25, rho=50.0)), [fw.Gravity([0.0, -9.8])],
                       considerContact=True, initials=[])
    vox = fw.VoxelGridDomain(d=2, nx=12, ny=8, lb=[0.0, 0.0], ub=[1.0, 1.0], considerContact=True,
                             occupancy_np=voxel_pit(12, 8))
    return [vox, fem]


def plain_small_scene(fw, seed=0):
    """Plain small workload: 1.0 x 0.25 rectangle at (0, 0.3), 64 x 16 quads
    split in two (2048 triangles, 1105 nodes), interior nodes jittered
    U(+-0.1h); Elastic E=2e4 nu=0.2 rho=40; gravity (0, -1); ground plane y=0."""
    conn, coords = fw.structured_rectangle(64, 16, 1.0, 0.25, origin=(0.0, 0.3), jitter=0.1, seed=seed)
    fem = fw.FemDomain(fw.Mesh(2, conn, coords), fw.SolidProp(fw.Elastic(E=2e4, nu=0.2, rho=40.0)),
                       [fw.Gravity([0.0, -1.0])])
    ground = fw.GroundDomain(2, [0.0, 0.0], [0.0, 1.0])
    return [ground, fem]


def plain_large_scene(fw, seed=0, n=256, hf_offset=0.15):
    """Plain large workload: unit square at (0, 0.2), n x n quads (n=256: 131072
    triangles, 66049 nodes); NeoHookean E=1e5 nu=0.35 rho=100; v0 = (0, -0.5) +
    N(0, 0.01^2) per component; height field of 4096 samples over x in [-1, 2],
    sum of 8 sinusoids of total amplitude 0.05 with random phase, raised by
    ``hf_offset`` so that the body reaches it within the run; no gravity."""
    rng = np.random.default_rng(seed)
    conn, coords = fw.structured_rectangle(n, n, 1.0, 1.0, origin=(0.0, 0.2))
    nn = coords.shape[0]
    v0 = np.array([0.0, -0.5]) + rng.normal(0.0, 0.01, size=(nn, 2))
    ics = [fw.InitialVel([i], v0[i]) for i in range(nn)]
    fem = fw.FemDomain(fw.Mesh(2, conn, coords), fw.SolidProp(fw.HyperElastic(E=1e5, nu=0.35, rho=100.0)), [],
                       initials=ics)
    xs = np.linspace(-1.0, 2.0, 4096)
    amps = rng.uniform(0.5, 1.0, size=8)
    amps = amps / amps.sum() * 0.05
    omegas = 2.0 * np.pi * rng.uniform(0.5, 6.0, size=8)
    phases = rng.uniform(0.0, 2.0 * np.pi, size=8)
    h = hf_offset + sum(a * np.sin(w * xs + p) for a, w, p in zip(amps, omegas, phases))
    hf = fw.HeightFieldDomain(2, h.astype(np.float32), lb=[-1.0, -1.0], ub=[2.0, 1.0])
    return [hf, fem]


def multi_block_scene(fw, n_bodies, n=10, side=0.08):
    """n_bodies blocks of n x n quads side by side over the ground plane y=0,
    bottoms staggered in [0.01, 0.06], falling at (0, -1) under gravity;
    materials cycle Elastic / NeoHookean / J2 so every law meets contact.
    The blocks do not collide with each other (collision masks)."""
    from flatworld_b200.definitions import COLLISION_CATEGORY_FEM, COLLISION_MASK_ALL

    doms = [fw.GroundDomain(2, [0.0, 0.0], [0.0, 1.0])]
    for b in range(n_bodies):
        conn, coords = fw.structured_rectangle(n, n, side, side, origin=(b * 1.25 * side, 0.01 + 0.05 * ((b * 7) % 11) / 10))
        mat = (fw.Elastic(E=5e4, nu=0.3, rho=500.0), fw.HyperElastic(E=5e4, nu=0.3, rho=500.0),
               fw.MisesPlastic(E=5e4, nu=0.3, rho=500.0, sigma_y=400.0, H=1e3))[b % 3]
        fem = fw.FemDomain(fw.Mesh(2, conn, coords), fw.SolidProp(mat), [fw.Gravity([0.0, -9.8])],
                           initials=[fw.InitialVel("ALL", [0.0, -1.0])])
        fem.collide_bits = COLLISION_MASK_ALL & ~COLLISION_CATEGORY_FEM  # blocks touch the ground only
        doms.append(fem)
    return doms


def ragged_body_scene(fw, rng, index, h=0.01, rho=2000.0, voxel_cells=128, voxel_h=0.02, v0=0.0):
    """One scene of the ragged batch: a structured rectangle with node count
    log-uniform in [100, 20000] and aspect ratio U[0.25, 4]; material by
    index % 3 (Elastic, NeoHookean, J2 with yield stress 0.02 E, H = 0),
    E ~ U[1e4, 1e6], nu ~ U[0.2, 0.45]; its own 128 x 128 voxel grid with
    Bernoulli(0.15) occupancy.  Fixed here (unspecified by the workload): 1 cm
    elements, density 2000, 2 cm voxel cells, the body at rest 1 cm above the
    grid under gravity 9.8, so it drops into the voxel field within the first
    ~900 substeps and settles there.  With these, dt = 5e-5 is at most 0.77 of
    every body's CFL and contact bound (the worst is 6.5e-5).  A faster entry
    (1 m/s down) drives some NeoHookean bodies 5 cm into the random field,
    where the nearest-free-face normals fold elements until J <= 0 and the
    state turns non-finite -- the same on the FP32 oracle, i.e. a property of
    the scheme on that input, not of the kernels."""
    n = float(np.exp(rng.uniform(np.log(100.0), np.log(20000.0))))
    asp = float(rng.uniform(0.25, 4.0))
    nx = max(1, int(round(np.sqrt(n * asp) - 1)))
    ny = max(1, int(round(np.sqrt(n / asp) - 1)))
    E = float(rng.uniform(1e4, 1e6))
    nu = float(rng.uniform(0.2, 0.45))
    kind = index % 3
    if kind == 0:
        mat = fw.Elastic(E, nu, rho)
    elif kind == 1:
        mat = fw.HyperElastic(E, nu, rho)
    else:
        mat = fw.MisesPlastic(E, nu, rho, sigma_y=0.02 * E, H=0.0)
    W, Hh = nx * h, ny * h
    extent = voxel_cells * voxel_h
    lb = np.array([-0.5 * extent + 0.5 * W, -extent - 0.01], np.float32)
    occ = (rng.random((voxel_cells, voxel_cells)) < 0.15).astype(np.int32)
    vox = fw.VoxelGridDomain(2, voxel_cells, voxel_cells, lb, lb + extent, occupancy_np=occ)
    conn, coords = fw.structured_rectangle(nx, ny, W, Hh, origin=(0.0, 0.0))
    fem = fw.FemDomain(fw.Mesh(2, conn, coords), fw.SolidProp(mat), [fw.Gravity([0.0, -9.8])],
                       initials=[fw.InitialVel("ALL", [0.0, v0])])
    return [vox, fem]


def ragged_batch(fw, n_scenes=2048, seed=0):
    """Scene i draws from its own generator (seed, i), so any one scene can be
    rebuilt alone (ragged_batch_one) for the one-body-at-a-time baseline."""
    return [ragged_batch_one(fw, i, seed) for i in range(n_scenes)]


def ragged_batch_one(fw, index, seed=0):
    return ragged_body_scene(fw, np.random.default_rng([seed, index]), index)


def gradient_block_scene(fw, n=64, side=0.4, bottom=0.5, young=None, v0=(0.0, -2.0), seed=0):
    """Differentiation workload: n x n quads (2 n^2 NeoHookean triangles) of
    side ``side`` with its bottom at y = ``bottom``, dropped onto the ground
    plane y = 0 with initial velocity v0 under gravity 9.8.  Per-element
    Young's modulus log-normal with mean 1e5 and sigma 0.3 (unless given).
    Fixed here (unspecified by the workload): nu = 0.3, rho = 1000, side 0.4 m,
    v0 = (0, -2) so that the block reaches the plane within 0.2 s."""
    from flatworld_b200.diff import lognormal_young

    conn, coords = fw.structured_rectangle(n, n, side, side, origin=(0.5 - 0.5 * side, bottom))
    fem = fw.FemDomain(fw.Mesh(2, conn, coords), fw.SolidProp(fw.HyperElastic(1e5, 0.3, 1000.0)),
                       [fw.Gravity([0.0, -9.8])], initials=[fw.InitialVel("ALL", list(v0))])
    fem.elementYoung = lognormal_young(2 * n * n, seed=seed) if young is None else np.asarray(young, np.float32)
    return [fw.GroundDomain(2, [0.0, 0.0], [0.0, 1.0]), fem]


# ---- FEM-FEM contact scenes

def flex_circles(fw, contact=True):
    """The reference's FEM-FEM scene (test2D/test_2Dfem_contact.py:14-26): two
    16-segment circles of radius 0.1 at y = 0.5 and 0.8, pulled toward each
    other by gravity +10 and -10, Elastic E = 2e4, nu = 0.2, rho = 40."""
    msh = fw.FEMesher(2)
    prop = fw.SolidProp(fw.Elastic(E=2e4, nu=0.2, rho=40.0))
    a = fw.FemDomain(msh.createCircle([0.5, 0.5], 0.1), prop, [fw.Gravity([0, 10.0])], considerContact=contact)
    b = fw.FemDomain(msh.createCircle([0.5, 0.8], 0.1), prop, [fw.Gravity([0, -10.0])], considerContact=contact)
    return [a, b]


def flex_stack(fw):
    """A circle resting on the ground plane and a NeoHookean circle with
    friction 0.3 dropped onto it, slightly off centre (plane + FEM-FEM
    contact, so the broad phase gates the FEM-FEM pair)."""
    msh = fw.FEMesher(2)
    g = fw.GroundDomain(2, [0.0, 0.0], [0.0, 1.0])
    a = fw.FemDomain(msh.createCircle([0.5, 0.101], 0.1), fw.SolidProp(fw.Elastic(E=2e4, nu=0.2, rho=40.0)),
                     [fw.Gravity([0, -10.0])])
    b = fw.FemDomain(msh.createCircle([0.52, 0.35], 0.1), fw.SolidProp(fw.HyperElastic(E=2e4, nu=0.2, rho=40.0)),
                     [fw.Gravity([0, -10.0])], friction=0.3)
    return [g, a, b]


def ccw_rectangle(fw, nx, ny, lx, ly, origin):
    """structured_rectangle with counter-clockwise triangles, so boundary-edge
    normals point outward as FEM-FEM contact expects."""
    conn, coords = fw.structured_rectangle(nx, ny, lx, ly, origin=origin)
    return fw.Mesh(2, np.ascontiguousarray(conn[:, [0, 2, 1]]), coords)


def flex_blocks(fw):
    """A 16 x 4 Elastic slab falling onto a rippled height field and an 8 x 8
    NeoHookean block (friction 0.3, 0.3 m/s down) falling onto the slab;
    height field + FEM-FEM contact.  Stable at a fixed dt of 0.3 x the loop's
    adaptive dt (at the adaptive dt itself the two soft bodies' two-sided
    penalty contact diverges, in the oracle as on the GPU)."""
    xs = np.linspace(-0.2, 0.5, 64)
    g = fw.HeightFieldDomain(2, (0.004 * np.sin(25 * xs)).astype(np.float32), [-0.2, -1.0], [0.5, 1.0])
    a = fw.FemDomain(ccw_rectangle(fw, 16, 4, 0.2, 0.05, (0.0, 0.01)), fw.SolidProp(fw.Elastic(E=2e4, nu=0.3, rho=100.0)),
                     [fw.Gravity([0.0, -9.8])])
    b = fw.FemDomain(ccw_rectangle(fw, 8, 8, 0.08, 0.08, (0.05, 0.075)),
                     fw.SolidProp(fw.HyperElastic(E=2e4, nu=0.3, rho=100.0)), [fw.Gravity([0.0, -9.8])],
                     initials=[fw.InitialVel("ALL", [0.0, -0.3])], friction=0.3)
    return [g, a, b]


def ccw_disk(fw, cells, radius, centre):
    """A disk meshed by mapping the counter-clockwise cells x cells square grid
    onto the circle (elliptical grid mapping x sqrt(1 - y^2/2), y sqrt(1 - x^2/2)):
    a round boundary of 4 cells edges without corners."""
    conn, coords = fw.structured_rectangle(cells, cells, 2.0, 2.0, origin=(-1.0, -1.0))
    u, v = coords[:, 0].astype(np.float64), coords[:, 1].astype(np.float64)
    x = u * np.sqrt(np.maximum(0.0, 1.0 - 0.5 * v * v))
    y = v * np.sqrt(np.maximum(0.0, 1.0 - 0.5 * u * u))
    pts = np.stack([centre[0] + radius * x, centre[1] + radius * y], axis=1).astype(np.float32)
    return fw.Mesh(2, np.ascontiguousarray(conn[:, [0, 2, 1]]), pts)


def flex_pile(fw, cols=8, rows=8, cells=16, radius=0.025, gap=0.01, E=1e5, rho=1000.0):
    """cols x rows disks (cells x cells mapped grid each) in a grid above the
    ground plane y = 0, alternately Elastic and NeoHookean, friction 0.2,
    every pair in FEM-FEM contact; the columns fall, land and stack."""
    doms = [fw.GroundDomain(2, [0.0, 0.0], [0.0, 1.0])]
    pitch = 2 * radius + gap
    for r in range(rows):
        for c in range(cols):
            k = r * cols + c
            mat = (fw.Elastic if k % 2 == 0 else fw.HyperElastic)(E=E, nu=0.3, rho=rho)
            mesh = ccw_disk(fw, cells, radius, (radius + c * pitch + 0.002 * (r % 2), radius + 0.002 + r * pitch))
            doms.append(fw.FemDomain(mesh, fw.SolidProp(mat), [fw.Gravity([0.0, -9.8])], friction=0.2))
    return doms


def flex_stamp_quirk(fw):
    """A ground plane far below (never in a broad-phase pair) as domain 0, then
    two circles pulled together (tests/scenes.flex_circles).  The reference
    reads the broad-phase stamp of the FEM-FEM item's target at its FEM-local
    index (mixedcontact.py:925) in an array indexed by global domain index
    (explicitloop.py:451-463): items targeting the first circle (FEM-local 0)
    read the far plane's stamp and never run; items targeting the second read
    the first circle's and do."""
    return [fw.GroundDomain(2, [0.0, -5.0], [0.0, 1.0])] + flex_circles(fw)


def rigid_fixed_ball(fw):
    """The reference's FEM-rigid scene (test2D/test_2Dfemcontact_types.py:26-38):
    an Elastic circle of radius 0.05 at (0.5, 0.6) falling under gravity 10
    onto a fixed BallRigid of radius 0.15 at (0.5, 0.3), ground plane y = 0."""
    mesh = fw.FEMesher(2).createCircle([0.5, 0.6], 0.05)
    fem = fw.FemDomain(mesh, fw.SolidProp(fw.Elastic(E=2e4, nu=0.2, rho=40.0)), [fw.Gravity([0, -10.0])])
    rigid = fw.RigidBodyDomain(fw.BallRigid(2, [0.5, 0.3], 0.15, 100.0), [fw.FixedAll([0])], considerContact=True)
    ground = fw.GroundDomain(2, [0, 0.0], [0, 1])
    return [fem, rigid, ground]


def rigid_block(fw, nx=16, ny=4, w=0.4, h=0.1, y0=0.0, mat=None):
    conn, coords = fw.structured_rectangle(nx, ny, w, h, origin=(0.3, y0))
    mat = mat or fw.Elastic(E=5e4, nu=0.3, rho=100.0)
    return fw.FemDomain(fw.Mesh(2, conn, coords), fw.SolidProp(mat), [fw.Gravity([0.0, -9.8])])


def rigid_pusher(fw):
    """A box driven at constant velocity and spin (EnforceVel + EnforceRotVel)
    sweeping across the top of an FEM block (0.4 x 0.2) that rests on the
    ground, with friction 0.3 (the rigid's), plus a free capsule (gravity, no
    BCs) dropped onto the block's far end: FEM-rigid contact with both
    BC-driven and free rigids, friction, and reaction impulses.  The rigids
    stay clear of the ground plane's box (y <= 0.1)."""
    block = rigid_block(fw, nx=16, ny=8, h=0.2)
    box = fw.RigidBodyDomain(fw.BoxRigid(2, [0.25, 0.262], [0.08, 0.1], [0.3], 5.0),
                             [fw.EnforceVel([0], [0.6, -0.05]), fw.EnforceRotVel([0], 2.0)], friction=0.3)
    cap = fw.RigidBodyDomain(fw.CapsuleRigid(2, [0.55, 0.26], [0.65, 0.28], [0.0], 0.02, 2.0),
                             [fw.Gravity([0.0, -9.8])], friction=0.1)
    return [fw.GroundDomain(2, [0.0, 0.0], [0.0, 1.0]), block, box, cap]


def rigid_free_ball(fw):
    """A free ball (gravity, initial spin) dropped onto an FEM block resting on
    the ground: its fall is stopped by the reaction impulses alone."""
    block = rigid_block(fw, nx=20, ny=5, w=0.4, h=0.2, y0=0.0, mat=fw.HyperElastic(E=4e4, nu=0.3, rho=80.0))
    ball = fw.RigidBodyDomain(fw.BallRigid(2, [0.5, 0.32], 0.06, 2.0), [fw.Gravity([0.0, -9.8])],
                              initials=[fw.InitialAngVel([0], 3.0)], friction=0.2)
    return [fw.GroundDomain(2, [0.0, 0.0], [0.0, 1.0]), block, ball]


def rigid_row(fw, nx=128, ny=32, n_rigid=12, ball_speed=0.05):
    """A NeoHookean slab (1.0 x 0.25, nx x ny quads) on the ground plane under
    gravity, with a row of n_rigid BC-driven primitives touching its top
    (0.5 mm deep at the start), 0.08 apart, cycled: balls rolling right at
    ball_speed m/s (EnforceVel, friction 0.2), fixed box indenters (FixedAll)
    and capsules spinning in place at 1 rad/s (Fixed + EnforceRotVel,
    friction 0.1), which press deeper as they turn.  BC-driven rigids keep
    their clearances (a ball reaches the next box after about 0.035 /
    ball_speed s), so the scene runs for as long as a benchmark needs."""
    conn, coords = fw.structured_rectangle(nx, ny, 1.0, 0.25, origin=(0.0, 0.0))
    slab = fw.FemDomain(fw.Mesh(2, conn, coords), fw.SolidProp(fw.HyperElastic(E=1e5, nu=0.3, rho=500.0)),
                        [fw.Gravity([0.0, -9.8])])
    doms = [fw.GroundDomain(2, [0.0, 0.0], [0.0, 1.0]), slab]
    for k in range(n_rigid):
        x = 0.06 + 0.08 * k
        if k % 3 == 0:
            r = fw.RigidBodyDomain(fw.BallRigid(2, [x, 0.2745], 0.025, 0.5), [fw.EnforceVel([0], [ball_speed, 0.0])],
                                   friction=0.2)
        elif k % 3 == 1:
            r = fw.RigidBodyDomain(fw.BoxRigid(2, [x, 0.2745], [0.04, 0.05], [0.0], 1.0), [fw.FixedAll([0])])
        else:
            r = fw.RigidBodyDomain(fw.CapsuleRigid(2, [x - 0.02, 0.2695], [x + 0.02, 0.2695], [0.0], 0.02, 0.5),
                                   [fw.Fixed([0]), fw.EnforceRotVel([0], 1.0)], friction=0.1)
        doms.append(r)
    return doms


def rigid_shared(fw, mass=20.0):
    """A free box (gravity) lying across two FEM blocks that stand on the
    ground 5 cm apart: one rigid in two FEM-rigid pairs (its reactions summed
    over both pairs in pair order), next to the blocks' own FEM-FEM pair."""
    def block(x0, mat):
        conn, coords = fw.structured_rectangle(12, 6, 0.3, 0.15, origin=(x0, 0.0))
        return fw.FemDomain(fw.Mesh(2, conn, coords), fw.SolidProp(mat), [fw.Gravity([0.0, -9.8])])

    a = block(0.1, fw.Elastic(E=6e4, nu=0.3, rho=100.0))
    b = block(0.45, fw.HyperElastic(E=4e4, nu=0.25, rho=120.0))
    box = fw.RigidBodyDomain(fw.BoxRigid(2, [0.425, 0.1795], [0.5, 0.06], [0.02], mass), [fw.Gravity([0.0, -9.8])],
                             friction=0.15)
    return [fw.GroundDomain(2, [0.0, 0.0], [0.0, 1.0]), a, b, box]


def rigid_bcs(fw):
    """The remaining rigid BCs over an FEM slab (0.9 x 0.1) on the ground: a
    ball under gravity pushed sideways by a Force and turned by a Torque, a
    box driven down into the slab by EnforceAcc, and a capsule held by Fixed
    and spun up by EnforceRotAcc, with loop damping 0.5."""
    conn, coords = fw.structured_rectangle(36, 4, 0.9, 0.1, origin=(0.05, 0.0))
    slab = fw.FemDomain(fw.Mesh(2, conn, coords), fw.SolidProp(fw.Elastic(E=8e4, nu=0.3, rho=200.0)),
                        [fw.Gravity([0.0, -9.8])])
    ball = fw.RigidBodyDomain(fw.BallRigid(2, [0.2, 0.14], 0.03, 4.0),
                              [fw.Gravity([0.0, -9.8]), fw.Force([0], [0.5, 0.0]), fw.Torque([0], 0.01)],
                              friction=0.2)
    box = fw.RigidBodyDomain(fw.BoxRigid(2, [0.5, 0.1205], [0.06, 0.04], [0.1], 2.0),
                             [fw.EnforceAcc([0], [0.0, -0.5])], friction=0.1)
    cap = fw.RigidBodyDomain(fw.CapsuleRigid(2, [0.76, 0.1195], [0.84, 0.1195], [0.0], 0.02, 1.0),
                             [fw.Fixed([0]), fw.EnforceRotAcc([0], 5.0)], friction=0.3)
    return [fw.GroundDomain(2, [0.0, 0.0], [0.0, 1.0]), slab, ball, box, cap]


def ground_circle(fw, bcs=None, plane_y=0.3):
    """The reference's FEM-analytical scene (test2D/test_2Dfem_contact.py,
    test_2Dfemanalytic_contact.py): an Elastic circle of radius 0.1 at
    (0.5, 0.5) under gravity 10 over the plane y = plane_y; ``bcs`` on the
    ground (the reference's example scripts often fix it: [Fixed([0])])."""
    mesh = fw.FEMesher(2).createCircle([0.5, 0.5], 0.1)
    fem = fw.FemDomain(mesh, fw.SolidProp(fw.Elastic(E=2e4, nu=0.2, rho=40.0)), [fw.Gravity([0, -10.0])])
    return [fw.GroundDomain(2, [0.0, plane_y], [0.0, 1.0], bcs or []), fem]


def fixed_ground_heightfield(fw, fixed=True):
    """A circle dropped on a height-field bowl, with a ground plane far below;
    the plane fixed by a BC or not.  With the BC the rigid manager recomputes
    every ground's broad-phase box each update, and the height field's entry
    (whose point and normal the reference never fills) collapses to the
    origin, so the circle falls through the bowl onto the plane."""
    x = np.linspace(0.0, 1.0, 64)
    h = (0.3 + 0.4 * (x - 0.5) ** 2).astype(np.float32)
    hf = fw.HeightFieldDomain(2, h, [0.0, 0.0], [1.0, 1.0])
    mesh = fw.FEMesher(2).createCircle([0.5, 0.55], 0.08)
    fem = fw.FemDomain(mesh, fw.SolidProp(fw.Elastic(E=2e4, nu=0.2, rho=40.0)), [fw.Gravity([0, -10.0])])
    ground = fw.GroundDomain(2, [0.0, 0.0], [0.0, 1.0], [fw.Fixed([0])] if fixed else [])
    return [ground, hf, fem]


def rigid_spring_net(fw):
    """A spring net (6 x 6 cells of the reference's spring-grid pattern)
    dropped onto a fixed box, next to an FEM block that a free ball lands on:
    spring-rigid pairs (every spring node an item, penalty 100 k) beside
    FEM-rigid ones.  No ground, so the broad phase is skipped."""
    n, dx = 6, 0.03
    ii, jj = np.meshgrid(np.arange(n + 1), np.arange(n + 1), indexing="ij")
    coords = (np.stack([dx * ii, dx * jj], axis=-1).reshape(-1, 2) + np.float32([0.1, 0.42])).astype(np.float32)
    conn = []
    for i in range(n):
        for j in range(n):
            a, b, c = i * (n + 1) + j, i * (n + 1) + j + 1, (i + 1) * (n + 1) + j
            conn += [[a, b], [b, c], [c, a]]
    net = fw.SpringMassDomain(2, coords, np.asarray(conn, np.int32), [400.0, 0.5, 0.01], [fw.Gravity([0.0, -9.8])])
    conn2, coords2 = fw.structured_rectangle(8, 4, 0.2, 0.1, origin=(0.5, 0.3))
    block = fw.FemDomain(fw.Mesh(2, conn2, coords2), fw.SolidProp(fw.Elastic(E=3e4, nu=0.3, rho=100.0)),
                         [fw.Fixed(list(range(9)))])
    box = fw.RigidBodyDomain(fw.BoxRigid(2, [0.19, 0.36], [0.3, 0.1], [0.0], 5.0), [fw.FixedAll([0])],
                             friction=0.2)
    ball = fw.RigidBodyDomain(fw.BallRigid(2, [0.6, 0.44], 0.04, 1.0), [fw.Gravity([0.0, -9.8])])
    return [block, net, box, ball]



def plain_small_low_scene(fw, seed=0):
    """The plain small body (64 x 16 jittered quads, Elastic, gravity (0, -1))
    placed 5 mm above the ground plane y = 0 and moving down at 0.5 m/s, so
    that plane contact starts within the first 100 substeps of 1e-4."""
    conn, coords = fw.structured_rectangle(64, 16, 1.0, 0.25, origin=(0.0, 0.005), jitter=0.1, seed=seed)
    fem = fw.FemDomain(fw.Mesh(2, conn, coords), fw.SolidProp(fw.Elastic(E=2e4, nu=0.2, rho=40.0)),
                       [fw.Gravity([0.0, -1.0])], initials=[fw.InitialVel("ALL", [0.0, -0.5])])
    ground = fw.GroundDomain(2, [0.0, 0.0], [0.0, 1.0])
    return [ground, fem]


def j2_block_scene(fw):
    """A J2 (MisesPlastic) block, 24 x 12 jittered quads, thrown at the ground
    plane at (0.3, -2) m/s under gravity 9.8; it yields on impact."""
    conn, coords = fw.structured_rectangle(24, 12, 0.4, 0.2, origin=(0.1, 0.05), jitter=0.1, seed=3)
    mat = fw.MisesPlastic(E=1e5, nu=0.3, rho=100.0, sigma_y=2e3, H=1e3)
    fem = fw.FemDomain(fw.Mesh(2, conn, coords), fw.SolidProp(mat), [fw.Gravity([0.0, -9.8])],
                       initials=[fw.InitialVel("ALL", [0.3, -2.0])])
    return [fw.GroundDomain(2, [0.0, 0.0], [0.0, 1.0]), fem]


def bcs_scene(fw):
    """test2D/test_2Dfem_bcs.py: two-triangle squares under Force + Fixed,
    EnforceVel + Fixed, EnforceAcc + Fixed, and an initial velocity."""
    conn = np.array([[0, 1, 3], [0, 3, 2]], dtype=np.int32)
    c = np.array([[0.5, 0.5], [0.7, 0.5], [0.5, 0.7], [0.7, 0.7]], dtype=np.float32)
    prop = fw.SolidProp(fw.Elastic(E=2e4, nu=0.2, rho=40.0))
    d0 = fw.FemDomain(fw.Mesh(2, conn, c), prop, [fw.Force([0, 1], [0, -100.0]), fw.Fixed([2, 3])], False)
    d1 = fw.FemDomain(fw.Mesh(2, conn, c + 0.25), prop, [fw.EnforceVel([0, 1], [0, -1.0]), fw.Fixed([2, 3])],
                      False)
    d2 = fw.FemDomain(fw.Mesh(2, conn, c - 0.25), prop, [fw.EnforceAcc([0, 1], [0, -10.0]), fw.Fixed([2, 3])],
                      False)
    d3 = fw.FemDomain(fw.Mesh(2, conn, c + 0.5), prop, [], False, initials=[fw.InitialVel([0, 1], [0, -1.0])])
    return [d0, d1, d2, d3]


def tied_slabs_scene(fw, disk=True):
    """Two slabs glued by a tie (ExplicitLoop(ties=[(0, 1)])): a 16 x 4 Elastic
    cantilever clamped at its left end, and an 8 x 4 NeoHookean slab resting on
    its top face, sliding sideways at 0.2 m/s, held by the tie; both under
    gravity.  With ``disk``, a free Elastic disk drops onto the upper slab:
    untied FEM-FEM contact in the same loop, so nodes of the upper slab take
    tie and contact forces in one substep.  Stable at a fixed dt of 1.25e-5
    (half the loop's adaptive dt; at the adaptive dt the soft bodies' penalty
    contact diverges, in the oracle as in the reference's scheme)."""
    a = fw.FemDomain(ccw_rectangle(fw, 16, 4, 0.2, 0.05, (0.0, 0.01)), fw.SolidProp(fw.Elastic(E=5e4, nu=0.3, rho=100.0)),
                     [fw.Gravity([0.0, -9.8]), fw.Fixed(list(range(5)))])
    b = fw.FemDomain(ccw_rectangle(fw, 8, 4, 0.1, 0.05, (0.06, 0.06)),
                     fw.SolidProp(fw.HyperElastic(E=5e4, nu=0.3, rho=100.0)), [fw.Gravity([0.0, -9.8])],
                     initials=[fw.InitialVel("ALL", [0.2, 0.0])])
    doms = [a, b]
    if disk:
        c = fw.FemDomain(ccw_disk(fw, 8, 0.02, (0.1, 0.14)), fw.SolidProp(fw.Elastic(E=5e4, nu=0.3, rho=100.0)),
                         [fw.Gravity([0.0, -9.8])], initials=[fw.InitialVel("ALL", [0.0, -0.5])])
        doms.append(c)
    return doms


def ground_circle_fixed(fw):
    """ground_circle with the plane held by Fixed([0]) (the rigid manager moves it: static bits)."""
    return ground_circle(fw, [fw.Fixed([0])])


def ground_circle_moving(fw):
    """ground_circle with the plane driven by EnforceVel: its gate box moves, its contact stays."""
    return ground_circle(fw, [fw.EnforceVel([0], [0.0, -0.5])])


def fixed_heightfield(fw):
    return fixed_ground_heightfield(fw, True)


def spring_bcs_scene(fw):
    """test2D/test_2Dspring_bcs.py:17-27: three spring squares under Force /
    EnforceVel / EnforceAcc with two fixed nodes each."""
    conn = np.array([[0, 1], [1, 2], [0, 2], [2, 3], [3, 1], [0, 3]], dtype=np.int32)
    coords = np.array([[0.5, 0.5], [0.7, 0.5], [0.5, 0.7], [0.7, 0.7]], dtype=np.float32)
    d0 = fw.SpringMassDomain(2, coords, conn, [100.0, 1.0, 1.0], [fw.Force([0, 1], [0, -1.0]), fw.Fixed([2, 3])],
                             False)
    d1 = fw.SpringMassDomain(2, coords - 0.25, conn, [100.0, 1.0, 1.0],
                             [fw.EnforceVel([0, 1], [0, -1.0]), fw.Fixed([2, 3])], False)
    d2 = fw.SpringMassDomain(2, coords - 0.5, conn, [100.0, 1.0, 1.0],
                             [fw.EnforceAcc([0, 1], [0, -10.0]), fw.Fixed([2, 3])], False)
    return [d0, d1, d2]


def spring_mixed_scene(fw):
    """An Elastic block and a 6 x 6 spring net (friction 0.1) falling on the
    ground plane y = 0 side by side (spring-plane contact at 100 k, the
    spring-FEM pair bounding dt)."""
    n = 6
    dx = 0.6 / n
    ii, jj = np.meshgrid(np.arange(n + 1), np.arange(n + 1), indexing="ij")
    grid = np.stack([dx * ii, dx * jj], axis=-1).reshape(-1, 2).astype(np.float32) + np.float32(0.25)
    sconn = []
    for i in range(n):
        for j in range(n):
            a, b, c = i * (n + 1) + j, i * (n + 1) + j + 1, (i + 1) * (n + 1) + j
            sconn += [[a, b], [b, c], [c, a], [a, b]]
    sconn = np.asarray(sconn, np.int32)
    conn, coords = fw.structured_rectangle(8, 4, 0.2, 0.1, origin=(0.0, 0.05))
    block = fw.FemDomain(fw.Mesh(2, conn, coords), fw.SolidProp(fw.Elastic(E=2e4, nu=0.3, rho=100.0)),
                         [fw.Gravity([0.0, -9.8])])
    xy = (grid - np.float32(0.25)) * np.float32(0.25) + np.float32([0.3, 0.03])
    net = fw.SpringMassDomain(2, xy.astype(np.float32), sconn, [200.0, 0.5, 0.01], [fw.Gravity([0.0, -9.8])],
                              friction=0.1)
    return [fw.GroundDomain(2, [0.0, 0.0], [0.0, 1.0]), block, net]
