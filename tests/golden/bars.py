"""How close this build must come to the golden fixtures, per case (test
infrastructure: used by tests/test_golden.py and tests/test_gpu_golden.py).

The fixtures were made by the reference's own code on a CPU whose ``log``,
``sin`` and ``cos`` are the C library's.  The GPU and the default FP32 oracle
compute these three by IEEE-only methods of their own (bit-identical to each
other, within 2 ulp of the C library).  So:

* a case that evaluates none of them on a changing argument must match the
  fixture bit for bit;
* a *transcendental* case (a NeoHookean body: ``log J``; a rigid body whose
  angle changes: ``sin`` / ``cos`` of it) starts from the same bits but may
  drift by the last bit of those functions.  In a quiet scene that drift stays
  near 1e-6; in a scene where contact switches on and off (a ball landing on a
  block, a box driven through a stack) it grows like any other rounding
  difference.  The bar is the case's own rounding noise floor: the distance
  between two faithful FP32 builds of the scheme that differ only in rounding
  (the C library's functions without FMA contraction against the IEEE-only
  functions with FMA contraction), times NOISE_FACTOR, and never tighter than
  RTOL (the project's 1e-5 relative correctness target).
"""

from __future__ import annotations

import functools

import numpy as np

import flatworld_b200 as fw
import oracle
from tests import scenes
from tests.golden.make_golden import CASES, FRAME, LOOP_KW

RTOL = 1e-5
NOISE_FACTOR = 2.0
# cases with a rigid body whose angle changes (a free ball rolled by friction,
# a box turned by EnforceRotVel, rigids under boundary conditions)
TRIG_CASES = {"rigid_bcs", "rigid_pusher", "rigid_free_ball"}


def _uses_log(name):
    from flatworld_b200.definitions import MaterialType

    builder, kw = CASES[name][:2]
    return any(hasattr(getattr(d, "prop", None), "getMaterial") and d.prop.getMaterial().type == MaterialType.NEOHOOKEAN
               for d in getattr(scenes, builder)(fw, **kw))


TRANSCENDENTAL_CASES = {name for name in CASES if _uses_log(name)} | TRIG_CASES


def rel_linf(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def run_oracle(name, precision):
    """Yield (mark, x, v, oracle) at the fixture's snapshots, after a first
    (0, None, None, oracle) for the freshly built loop."""
    builder, kw, dt, adaptive, (mode, total, every) = CASES[name]
    o = oracle.OracleLoop(getattr(scenes, builder)(fw, **kw), dt, useAdapativeDT=adaptive, precision=precision,
                          **LOOP_KW.get(name, {}))
    yield 0, None, None, o
    for k in range(1, total + 1):
        if mode == "steps":
            o.advance(1)
        else:
            o.advance_with_time(FRAME)
        if k % every == 0:
            x, v, _ = o.state()
            yield k, x, v, o


@functools.lru_cache(maxsize=None)
def noise_floor(name):
    """Largest relative (L-inf) position distance, over the snapshots, between
    the f32libm and f32fma oracle builds on this case."""
    a = [x for _, x, _, _ in run_oracle(name, "f32libm") if x is not None]
    b = [x for _, x, _, _ in run_oracle(name, "f32fma") if x is not None]
    return max(rel_linf(p, q) for p, q in zip(b, a))


def position_bar(name):
    """Relative (L-inf) position bar for a transcendental case."""
    return max(RTOL, NOISE_FACTOR * noise_floor(name))
