"""Autotuner for the sweep kernel's temporal-blocking depth T and segment length.

For an image shape it times candidate (T, rows_per_segment) pairs with CUDA events on
the device (a fixed number of sweeps over synthetic coefficient planes of that shape)
and keeps the fastest; for a batch (`best_batch_config`) it times the persistent batched
launch of that exact batch under each candidate (T, rows per tile).  Results are cached
per (device name, shape or batch signature, mode) in memory and, when HS_AUTOTUNE_CACHE
names a file, in that JSON file.  HS_AUTOTUNE_LOG names a file that receives every
candidate's timing as one JSON line per tuning.
"""
from __future__ import annotations

import json
import os
import threading
from typing import Dict, Tuple

_cache: Dict[str, Tuple[int, int]] = {}
_lock = threading.Lock()

T_CANDIDATES = (1, 2, 3, 4, 5, 6, 7, 8)


def _seg_candidates(H: int, W: int, T: int):
    out = {0}
    for L in (12, 16, 20, 24, 32, 48, 64, 128, 256):
        if 2 * T <= L < H:
            out.add(L)
    return sorted(out)


def _key(dev_name, H, W, ld, fast_math):
    return f"{dev_name}|{H}x{W}|ld{ld}|{'fast' if fast_math else 'exact'}"


DEFAULT_TUNING_SWEEPS = 240


def _sweep_key(dev_name, H, W, ld, fast_math, sweeps):
    """Cache key of a sweep tuning; a run over another sweep count is cached apart."""
    key = _key(dev_name, H, W, ld, fast_math) + "|layout"
    return key if sweeps == DEFAULT_TUNING_SWEEPS else key + f"|s{sweeps}"


def _file():
    return os.environ.get("HS_AUTOTUNE_CACHE")


def _load_file():
    path = _file()
    if path and os.path.exists(path):
        try:
            with open(path) as f:
                for k, v in json.load(f).items():
                    _cache.setdefault(k, tuple(v))
        except (OSError, ValueError):
            pass


def _save_file():
    path = _file()
    if path:
        try:
            with open(path, "w") as f:
                json.dump({k: list(v) for k, v in _cache.items()}, f, indent=1)
        except OSError:
            pass


def time_config(Ix, Iy, It, u, v, T, seg, fast_math, sweeps, reps=5, layout=0):
    import torch

    from . import _lib as L
    from . import device as D

    cfg = L.make_config(sweeps_per_pass=T, rows_per_segment=seg, fast_math=fast_math, layout=layout)
    D.hs_sweeps(Ix, Iy, It, 1.0, T, u, v, cfg)  # warm-up, first-launch attributes
    best = float("inf")
    for _ in range(reps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        D.hs_sweeps(Ix, Iy, It, 1.0, sweeps, u, v, cfg)
        b.record()
        b.synchronize()
        best = min(best, a.elapsed_time(b))
    return best


def best_sweep_config(H: int, W: int, ld: int, fast_math: bool = True,
                      candidates=T_CANDIDATES,
                      sweeps: int = DEFAULT_TUNING_SWEEPS) -> Tuple[int, int, int]:
    """(sweeps_per_pass, rows_per_segment, layout) fastest on the current device for HxW;
    both layouts (2 and 4 columns per lane) compete in the fast form.  Every candidate is timed
    over `sweeps` sweeps: pass the workload's own count when it is known (the last, partial
    pass differs by depth)."""
    import torch

    from . import device as D

    dev_name = torch.cuda.get_device_name()
    key = _sweep_key(dev_name, H, W, ld, fast_math, sweeps)
    with _lock:
        if not _cache:
            _load_file()
        if key in _cache:
            return tuple(_cache[key])
    g = torch.Generator(device="cuda")
    g.manual_seed(0)
    planes = D.empty_planes(5, H, W)
    for p in planes:
        p.copy_(torch.rand((H, W), device="cuda", generator=g) - 0.5)
    Ix, Iy, It, u, v = planes
    # the same sweep count for every candidate (by default whole passes at depths 1-6 and 8,
    # one partial at 7; candidates 1-2 % apart, such as T = 6 and 7 at 1080p, need long runs)
    results = []
    for layout in ((1, 2) if fast_math else (1,)):
        for T in candidates:
            for seg in _seg_candidates(H, W, T):
                ms = time_config(Ix, Iy, It, u, v, T, seg, fast_math, sweeps, layout=layout)
                results.append((ms, T, seg, layout))
    results.sort()
    best = tuple(results[0][1:])
    log = os.environ.get("HS_AUTOTUNE_LOG")
    if log:
        try:
            with open(log, "a") as f:
                f.write(json.dumps({"key": key, "sweeps": sweeps,
                                    "ms": [[round(r[0], 5), *r[1:]] for r in results]}) + "\n")
        except OSError:
            pass
    with _lock:
        _cache[key] = best
        _save_file()
    return best


def clear():
    with _lock:
        _cache.clear()


# (T, rows per tile, layout): 1 = 2 columns per lane, 2 = 4 (fast form only)
BATCH_CANDIDATES = ((3, 96, 1), (4, 64, 1), (4, 96, 1), (5, 96, 1), (5, 128, 1), (6, 128, 1),
                    (6, 96, 1), (6, 128, 2), (6, 96, 2), (6, 192, 2), (5, 128, 2), (5, 96, 2),
                    (5, 64, 2), (5, 160, 2), (5, 192, 2), (4, 128, 2), (4, 96, 2), (4, 192, 2))


def _log(entry):
    log = os.environ.get("HS_AUTOTUNE_LOG")
    if log:
        try:
            with open(log, "a") as f:
                f.write(json.dumps(entry) + "\n")
        except OSError:
            pass


def best_batch_config(specs, fast_math: bool = True, candidates=BATCH_CANDIDATES,
                      reps: int = 3) -> Tuple[int, int, int]:
    """(sweeps_per_pass, rows_per_segment, layout) fastest for the persistent batched launch of
    `specs` = [(H, W, alpha, iters)] on the current device (timed as CUDA-graph replays
    of the batch itself over seeded random planes)."""
    import hashlib

    import torch

    from . import _lib as L
    from .batched import BatchPlan

    sig = hashlib.sha1(repr(sorted((int(H), int(W), float(a), int(n)) for H, W, a, n in specs))
                       .encode()).hexdigest()[:16]
    key = f"{torch.cuda.get_device_name()}|batch{len(specs)}:{sig}|{'fast' if fast_math else 'exact'}|layout"
    with _lock:
        if not _cache:
            _load_file()
        if key in _cache:
            return tuple(_cache[key])
    g = torch.Generator(device="cuda")
    g.manual_seed(0)
    results = []
    for T, rows, layout in candidates:
        if layout != 1 and not fast_math:
            if (T, rows, 1) in candidates:
                continue
            layout = 1
        plan = BatchPlan(specs, L.make_config(sweeps_per_pass=T, rows_per_segment=rows,
                                              fast_math=fast_math, layout=layout))
        for a, b in zip(plan.I0, plan.I1):
            a.copy_(torch.rand(a.shape, device="cuda", generator=g))
            b.copy_(torch.rand(b.shape, device="cuda", generator=g))
        plan.capture()
        plan.replay()
        plan.check()
        best = float("inf")
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            plan.replay()
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        plan.check()
        results.append((best, T, rows, layout))
        del plan
    results.sort()
    best = tuple(results[0][1:])
    _log({"key": key, "ms": [[round(r[0], 4), *r[1:]] for r in results]})
    with _lock:
        _cache[key] = best
        _save_file()
    return best
