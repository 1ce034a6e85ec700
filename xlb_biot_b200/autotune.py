"""Autotuner of the fused sweeps' launch shape.

The sweeps take a runtime launch shape (``XlbbSweepConfig``: owned columns per
CTA, prefetch depth in rows, CTAs per SM, minimum strip height).  ``tune``
times every candidate on the caller's own sweep (CUDA events on the current
stream, after a warm-up) and keeps the fastest; results are cached per GPU,
kernel family, dtype and grid size in a JSON file so later runs skip the
search.  The cache path is ``$XLBB_TUNE_CACHE`` or ``~/.cache/xlbb_tune.json``.
"""
import itertools
import json
import os

import torch

from . import _lib

ELASTICITY, DARCY = 0, 1
TX = (128, 256)
# per pipeline: CTA+registers / CTA+bulk ring / warps / collide-and-push (one thread per cell)
DEPTH = {0: (1, 2), 1: (2, 4, 6), 2: (1, 2), 3: (1,), 4: (1,)}
CTAS_PER_SM = (1, 2, 3, 4, 6)
MIN_ROWS = (8, 16, 32)


def get_config(kernel):
    c = _lib.SweepConfig()
    _lib.check(_lib.lib().xlbb_sweep_get_config(kernel, c), "xlbb_sweep_get_config")
    return {"tx": c.tx, "depth": c.depth, "ctas_per_sm": c.ctas_per_sm, "min_rows": c.min_rows,
            "pipeline": c.pipeline}


def set_config(kernel, tx, depth, ctas_per_sm, min_rows, pipeline=0):
    c = _lib.SweepConfig(int(tx), int(depth), int(ctas_per_sm), int(min_rows), int(pipeline))
    _lib.check(_lib.lib().xlbb_sweep_set_config(kernel, c), "xlbb_sweep_set_config")


def candidates(dtype_bytes=4, kernel=ELASTICITY):
    """Every launch shape the library instantiates for the given element size
    and kernel family (pipelines 3 and 4 ignore depth, CTAs per SM and strip
    height; pipeline 4, the four-column form of eligible FP32 sweeps -- the
    periodic elasticity sweep and the D2Q9 Darcy sweep -- is pipeline 3 for
    every other sweep)."""
    out = []
    for pipe, depths in DEPTH.items():
        ctas, rows = (CTAS_PER_SM, MIN_ROWS) if pipe < 3 else ((1,), (8,))   # pipelines 3, 4: only tx matters
        for t, d, c, m in itertools.product(TX if pipe != 2 else (128,), depths, ctas, rows):
            if dtype_bytes == 8 and (t > 128 or d > 4 or pipe == 4):
                continue
            out.append(dict(tx=t, depth=d, ctas_per_sm=c, min_rows=m, pipeline=pipe))
    return out


def device_status(reset=True):
    """Status word of the kernels' bounded waits (0 or XLBB_ETIMEOUT)."""
    import ctypes
    v = ctypes.c_int(0)
    _lib.check(_lib.lib().xlbb_device_status(ctypes.byref(v), 1 if reset else 0), "xlbb_device_status")
    return v.value


def _cache_path():
    return os.environ.get("XLBB_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "xlbb_tune.json"))


def _load():
    try:
        with open(_cache_path()) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _store(cache):
    path = _cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as fh:
            json.dump(cache, fh, indent=1, sort_keys=True)
    except OSError:
        pass


def _time(run, reps):
    run()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        run()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def tune(kernel, run, key, reps=5, cands_override=None, use_cache=True):
    """Pick the fastest launch shape for ``run`` (a callable issuing the sweeps
    to tune, e.g. 20 sweeps of the production grid).  ``key`` identifies the
    problem (dtype, grid).  Returns (config, ms, table)."""
    dev = torch.cuda.get_device_name()
    full_key = f"{dev}|{kernel}|{key}"
    cache = _load() if use_cache else {}
    if full_key in cache:
        cfg = cache[full_key]["config"]
        set_config(kernel, **cfg)
        return cfg, cache[full_key]["ms"], None
    cands = candidates(kernel=kernel) if cands_override is None else cands_override
    table = []
    for cfg in cands:
        set_config(kernel, **cfg)
        table.append((_time(run, reps), cfg))
    table.sort(key=lambda e: e[0])
    ms, best = table[0]
    set_config(kernel, **best)
    if use_cache:
        cache[full_key] = {"config": best, "ms": ms}
        _store(cache)
    return best, ms, table
