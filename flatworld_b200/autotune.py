"""Project autotuner for the step's launch shapes.

* ``tune_batched(loop)``: times the gather step of a BatchedLoop for each
  (element block, node block) candidate on the loop's own world -- the state
  is saved with fw_snapshot before and restored after, so tuning does not move
  the simulation -- and applies the fastest.  On the stream path it tunes the
  register budget and record staging instead (``tune_stream``);
  ``tune_stream_patch`` picks the patch size from sample batches.
* ``tune_resident(build_domains)``: builds the single-scene resident step with
  each (front warps, patches) candidate and times it; returns the best kwargs
  for ExplicitLoop.

Results are cached per (GPU name, world size) in
``$FLATWORLD_B200_CACHE`` (default ~/.cache/flatworld_b200/autotune.json).
"""

from __future__ import annotations

import json
import os

import numpy as np

_SNAP = 1023  # snapshot slot reserved for tuning


def _cache_path():
    d = os.environ.get("FLATWORLD_B200_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "flatworld_b200"))
    os.makedirs(d, exist_ok=True)
    return os.path.join(d, "autotune.json")


def _load_cache():
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store_cache(key, value):
    c = _load_cache()
    c[key] = value
    tmp = _cache_path() + ".tmp"
    with open(tmp, "w") as f:
        json.dump(c, f, indent=1)
    os.replace(tmp, _cache_path())


def _gpu_name(device):
    import torch

    return torch.cuda.get_device_name(device)


def _time_steps(native, steps, dt, stream):
    import torch

    s = torch.cuda.Event(enable_timing=True)
    e = torch.cuda.Event(enable_timing=True)
    s.record(stream)
    native.step(steps, dt)
    e.record(stream)
    e.synchronize()
    return s.elapsed_time(e) / steps


STREAM_MINB = {64: (32, 24, 20, 16), 128: (16, 12, 10, 8)}  # register budgets built per patch size


def tune_stream(loop, steps=16, use_cache=True):
    """Pick the stream step's register budget (CTAs per SM) and record staging
    (bulk copy or per-thread loads) for ``loop`` (a BatchedLoop on the stream
    path), timed on the loop's own world from a snapshot, as tune_batched."""
    import torch

    key = (f"stream|{_gpu_name(loop._native.device)}|N={loop.n_nodes}|E={loop.n_elems}|S={loop.S}"
           f"|patch={loop.stream_patch}")
    if use_cache:
        hit = _load_cache().get(key)
        if hit:
            loop.set_stream_shape(hit["minb"], hit["bulk"])
            return dict(hit, cached=True)
    stream = torch.cuda.Stream(device=loop._native.device)
    loop.set_stream(stream.cuda_stream)
    dt = float(np.float32(loop.dt.min()))
    nat = loop._native
    nat.snapshot(_SNAP)
    results = []
    for minb in STREAM_MINB[loop.stream_patch]:
        for bulk in (False, True):
            try:
                loop.set_stream_shape(minb, bulk)
            except RuntimeError:  # e.g. the staged records do not fit in shared memory
                continue
            nat.restore(_SNAP)
            nat.step(2, dt)
            nat.restore(_SNAP)
            results.append((_time_steps(nat, steps, dt, stream), minb, bulk))
    nat.restore(_SNAP)
    nat.synchronize()
    ms, minb, bulk = min(results)
    loop.set_stream_shape(minb, bulk)
    loop.set_stream(None)
    out = {"path": "stream", "patch": loop.stream_patch, "minb": minb, "bulk": bool(bulk), "ms_per_step": ms,
           "candidates": [{"minb": m, "bulk": bool(b), "ms": t} for t, m, b in results]}
    _store_cache(key, out)
    return out


def tune_stream_patch(make_loop, patches=(64, 128), steps=16):
    """Pick the stream step's patch size: ``make_loop(patch)`` builds a
    BatchedLoop (a representative sample of the batch) with that patch size;
    each is tuned with tune_stream and timed.  Returns (best patch, results)."""
    results = []
    for p in patches:
        lp = make_loop(p)
        r = tune_stream(lp, steps=steps, use_cache=False)
        results.append((r["ms_per_step"], p, r))
        lp._native.close()
    ms, p, _ = min(results, key=lambda t: t[0])
    return p, [{"patch": q, "ms": m, "minb": r["minb"], "bulk": r["bulk"]} for m, q, r in results]


def tune_batched(loop, blocks=(128, 256, 512), steps=16, use_cache=True):
    """Pick the launch shape for ``loop`` (a BatchedLoop): on the gather path
    the kernels' block sizes; on the stream path its register budget and
    record staging (tune_stream; the patch size is fixed when the loop is
    built, see tune_stream_patch)."""
    import torch

    if getattr(loop, "path", "gather") == "stream":
        return tune_stream(loop, steps=steps, use_cache=use_cache)
    if getattr(loop, "_has_flex", False) or getattr(loop, "_has_rigid", False):
        # candidates are timed from one snapshot, which holds neither the FEM-FEM
        # contact state nor the rigid bodies: keep the default launch shape
        return {"path": loop.path, "block_elems": 0, "block_nodes": 0, "candidates": [],
                "skipped": "snapshots hold no FEM-FEM contact or rigid-body state"}

    key = f"batched|{_gpu_name(loop._native.device)}|N={loop.n_nodes}|E={loop.n_elems}|S={loop.S}"
    if use_cache:
        hit = _load_cache().get(key)
        if hit:
            loop.set_launch(hit["block_elems"], hit["block_nodes"])
            return dict(hit, cached=True)
    stream = torch.cuda.Stream(device=loop._native.device)
    loop.set_stream(stream.cuda_stream)
    dt = float(np.float32(loop.dt.min()))
    nat = loop._native
    nat.snapshot(_SNAP)
    results = []
    for be in blocks:
        for bn in blocks:
            loop.set_launch(be, bn)
            nat.restore(_SNAP)
            nat.step(2, dt)
            nat.restore(_SNAP)
            ms = _time_steps(nat, steps, dt, stream)
            results.append((ms, be, bn))
    nat.restore(_SNAP)
    nat.synchronize()
    ms, be, bn = min(results)
    loop.set_launch(be, bn)
    loop.set_stream(None)
    out = {"block_elems": be, "block_nodes": bn, "ms_per_step": ms,
           "candidates": [{"block_elems": b, "block_nodes": n, "ms": m} for m, b, n in results]}
    _store_cache(key, out)
    return out


def tune_resident(build_domains, fronts=(4, 6, 8), patches=(0, 128, 96), steps=200, device=0, use_cache=True):
    """Pick (front_warps, patches) of the resident step for the single-scene
    world returned by ``build_domains()``; returns ExplicitLoop kwargs."""
    import torch

    from .explicitloop import ExplicitLoop

    probe = ExplicitLoop(0.0, build_domains(), device=device)
    key = f"resident|{_gpu_name(device)}|N={probe._packed.N}|E={probe._packed.E}"
    if use_cache:
        hit = _load_cache().get(key)
        if hit:
            return {"front_warps": hit["front_warps"], "patches": hit["patches"]}
    results = []
    stream = torch.cuda.Stream(device=device)
    for fwp in fronts:
        for p in patches:
            lp = ExplicitLoop(0.0, build_domains(), device=device, path="resident", patches=p, front_warps=fwp)
            lp._native.set_stream(stream.cuda_stream)
            dt = float(np.float32(lp.stableTime))
            lp._native.step(20, dt)
            ms = _time_steps(lp._native, steps, dt, stream)
            results.append((ms, fwp, p))
            lp._native.close()
    ms, fwp, p = min(results)
    _store_cache(key, {"front_warps": fwp, "patches": p, "ms_per_step": ms,
                       "candidates": [{"front_warps": f, "patches": q, "ms": m} for m, f, q in results]})
    return {"front_warps": fwp, "patches": p}
