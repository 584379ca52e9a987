"""Generate the golden fixtures in this folder by running the REFERENCE's own
Python source (FlatWorld: ``ExplicitLoop``, ``FemSpringManager``, the batched
contact code and every ``@wp.kernel`` / ``@wp.func`` they launch, unmodified)
on ``warp_standin`` -- a serial CPU stand-in for the Warp runtime, written from
Warp's public documentation, because ``warp-lang`` is not installable here.

Usage (in a checkout that has the reference at REFERENCE below):

    python tests/golden/make_golden.py            # every case, in parallel
    python tests/golden/make_golden.py plain_small j2_block

Each case builds one scene of ``tests/scenes.py`` through the reference's API
(the same builder the tests use with ``flatworld_b200``), steps it with the
reference's ``advance()`` / ``advanceWithTime()`` and writes ``<case>.npz``:

    marks   int64 [K]     substeps (or frames) completed at each snapshot
    x, v    float32 [K, n, 2]  node positions / velocities at the snapshots
    dt      float64       the loop's dt right after construction
    mass    float32 [n]   lumped masses as prepared by the reference
    eqps    float32 [K, E] (J2 cases) equivalent plastic strain

Test infrastructure only; the product never reads these files' generator.
"""

from __future__ import annotations

import contextlib
import io
import os
import subprocess
import sys
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REFERENCE = "/root/reference"
FRAME = 1.0 / 60.0

# name -> (scene builder in tests/scenes.py, kwargs, ExplicitLoop dt, adaptive, schedule)
# schedule: ("steps", total substeps, snapshot every) with loop.advance(), or
#           ("frames", total frames, snapshot every) with loop.advanceWithTime(1/60)
CASES = {
    "plain_small": ("plain_small_scene", {}, 1e-4, False, ("steps", 2000, 200)),
    "plain_small_contact": ("plain_small_low_scene", {}, 1e-4, False, ("steps", 1500, 150)),
    "hf_disk": ("hf_disk_scene", {}, 0.0, True, ("frames", 60, 10)),
    "voxel_disk": ("voxel_disk_scene", {}, 0.0, True, ("frames", 60, 10)),
    "nh_heightfield32": ("plain_large_scene", {"n": 32, "hf_offset": 0.17}, 0.0, True, ("steps", 3000, 250)),
    "j2_block": ("j2_block_scene", {}, 5e-5, False, ("steps", 4000, 400)),
    "bcs": ("bcs_scene", {}, 0.0, True, ("frames", 60, 10)),
    "tied_slabs": ("tied_slabs_scene", {}, 1.25e-5, False, ("steps", 3000, 300)),
    # row (f): FEM-FEM contact, rigid primitives, grounds with BCs, springs
    "flex_circles": ("flex_circles", {}, 0.0, True, ("frames", 24, 4)),
    "flex_stack": ("flex_stack", {}, 0.0, True, ("frames", 40, 8)),
    "rigid_fixed_ball": ("rigid_fixed_ball", {}, 0.0, True, ("frames", 40, 8)),
    "rigid_fixed_ball_tied": ("rigid_fixed_ball", {}, 0.0, True, ("frames", 40, 8)),
    "rigid_pusher": ("rigid_pusher", {}, 0.0, True, ("frames", 14, 2)),
    "rigid_free_ball": ("rigid_free_ball", {}, 0.0, True, ("frames", 40, 8)),
    "rigid_bcs": ("rigid_bcs", {}, 0.0, True, ("frames", 30, 6)),
    "ground_circle_fixed": ("ground_circle_fixed", {}, 0.0, True, ("frames", 30, 6)),
    "ground_circle_moving": ("ground_circle_moving", {}, 0.0, True, ("frames", 30, 6)),
    "fixed_heightfield": ("fixed_heightfield", {}, 0.0, True, ("frames", 30, 6)),
    "spring_bcs": ("spring_bcs_scene", {}, 0.0, True, ("frames", 60, 10)),
    "spring_mixed": ("spring_mixed_scene", {}, 0.0, True, ("frames", 30, 6)),
}
# ExplicitLoop keyword arguments beyond dt / useAdapativeDT, per case
LOOP_KW = {"tied_slabs": {"ties": [(0, 1)]}, "rigid_fixed_ball_tied": {"ties": [(0, 1)]},
           "rigid_bcs": {"damping": 0.5}}
# cases whose worlds step on the gather path only (FEM-FEM contact, rigids, springs)
GATHER_ONLY = {"tied_slabs", "flex_circles", "flex_stack", "rigid_fixed_ball", "rigid_fixed_ball_tied",
               "rigid_pusher", "rigid_free_ball", "rigid_bcs", "ground_circle_fixed", "ground_circle_moving",
               "fixed_heightfield", "spring_bcs", "spring_mixed"}


def reference_api():
    """Import the reference package on the Warp stand-in and return a
    namespace with its public names (plus the structured-mesh generator the
    scene builders use to make their inputs)."""
    sys.path.insert(0, HERE)
    import warp_standin

    sys.modules["warp"] = warp_standin
    # femesher imports meshio only inside its file readers; the circle
    # generator the scenes use does not need it
    sys.modules.setdefault("meshio", types.ModuleType("meshio"))
    if REFERENCE not in sys.path:
        sys.path.insert(0, REFERENCE)
    with contextlib.redirect_stdout(io.StringIO()):
        import flatworld as rf
    sys.path.insert(0, REPO)
    from flatworld_b200.mesh import structured_rectangle

    ns = types.SimpleNamespace(**{k: getattr(rf, k) for k in dir(rf) if not k.startswith("_")})
    ns.structured_rectangle = structured_rectangle
    return ns, rf


def run_case(name: str) -> str:
    builder, kw, dt, adaptive, (mode, total, every) = CASES[name]
    ns, rf = reference_api()
    from tests import scenes

    quiet = io.StringIO()
    t0 = time.time()
    with contextlib.redirect_stdout(quiet):
        loop = rf.ExplicitLoop(dt, getattr(scenes, builder)(ns, **kw), useAdapativeDT=adaptive,
                               **LOOP_KW.get(name, {}))
    dt0 = float(loop.dt)  # advanceWithTime changes loop.dt (its last substep is the remainder)
    fsm = loop.femSpringManager
    n = int(fsm.totalNodes.numpy()[0])
    ne = int(fsm.totalFEMElements.numpy()[0])
    has_j2 = bool((fsm.matType.numpy()[:ne] == int(rf.MaterialType.MISES)).any())
    marks, xs, vs, eq = [], [], [], []
    with contextlib.redirect_stdout(quiet):
        for k in range(1, total + 1):
            if mode == "steps":
                loop.advance()
            else:
                loop.advanceWithTime(FRAME)
            if k % every == 0:
                marks.append(k)
                xs.append(fsm.coords.numpy()[:n].copy())
                vs.append(fsm.V.numpy()[:n].copy())
                if has_j2:
                    eq.append(fsm.eqPlasticStrain.numpy()[:ne].copy())
    out = {
        "marks": np.asarray(marks, np.int64),
        "x": np.asarray(xs, np.float32),
        "v": np.asarray(vs, np.float32),
        "dt": np.float64(dt0),
        "mass": fsm.mass.numpy()[:n].astype(np.float32),
    }
    if has_j2:
        out["eqps"] = np.asarray(eq, np.float32)
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    return f"{name}: {len(marks)} snapshots, n={n}, dt={dt0:.6e}, {time.time() - t0:.0f} s -> {path}"


def main(argv):
    names = argv or list(CASES)
    if len(names) == 1:
        print(run_case(names[0]), flush=True)
        return 0
    procs = [(nm, subprocess.Popen([sys.executable, __file__, nm], cwd=REPO)) for nm in names]
    rc = 0
    for nm, p in procs:
        rc |= p.wait()
    return rc


if __name__ == "__main__":
    if REPO not in sys.path:
        sys.path.insert(0, REPO)
    sys.exit(main(sys.argv[1:]))
