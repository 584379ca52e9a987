"""Rounding noise floor of the FP32 scheme itself (CPU only).

Three FP32 evaluations of the same reference scheme that differ only in
rounding -- the oracle as written, the oracle with FMA contraction (as the
reference's NVRTC-compiled GPU path does), and the oracle with the C library's
logf (as the reference's CPU device does) -- are compared with each other and
with FP64.  Positions stay within 1e-5 relative of each other; velocities of
the stiff NeoHookean workload drift apart by ~1e-2 relative within a few
hundred substeps, which is the scale any FP32 implementation that is not
bit-identical operation for operation will show.
"""

import numpy as np

import flatworld_b200 as fw
import oracle
from tests import scenes


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def test_noise_floor_neohookean():
    build = lambda: scenes.plain_large_scene(fw, n=32, hf_offset=0.17)  # noqa: E731
    loops = {p: oracle.OracleLoop(build(), 0.0, precision=p, threads=4) for p in ("f32", "f32fma", "f32libm", "f64")}
    for o in loops.values():
        o.advance(1000)
    st = {p: o.state() for p, o in loops.items()}
    x = {p: s[0] for p, s in st.items()}
    v = {p: s[1] for p, s in st.items()}
    report = {p: (rel(x[p], x["f64"]), rel(v[p], v["f64"])) for p in ("f32", "f32fma", "f32libm")}
    print("vs FP64 after 1000 substeps (x, v):", report)
    for p in ("f32fma", "f32libm"):
        assert rel(x[p], x["f32"]) < 1e-5
    # the FP32 variants are all equally far from FP64
    assert max(r[0] for r in report.values()) < 1e-5


def test_log_method_accuracy():
    """or_logf (the log of the FP32 oracle and of the kernels) against FP64
    log: < 2 ulp on a sweep of [0.5, 2) (the range of J in the workloads) and
    across the float range; exact specials."""
    from oracle.scene import log32
    rng = np.random.default_rng(0)
    xs = np.concatenate([np.linspace(0.5, 2.0, 20001), 10.0 ** rng.uniform(-37, 38, 20000)]).astype(np.float32)
    worst = 0.0
    for x in xs:
        ref = np.log(np.float64(x))
        got = log32(x)
        r32 = np.float32(ref)
        ulp = float(np.spacing(np.abs(r32)))
        worst = max(worst, abs(got - ref) / ulp)
    assert worst < 2.0, worst
    assert log32(1.0) == 0.0 and log32(0.0) == -np.inf and np.isnan(log32(-1.0)) and log32(np.inf) == np.inf
