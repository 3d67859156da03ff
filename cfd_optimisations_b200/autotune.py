"""Autotuner of the step kernels' launch shape, cached per GPU, precision, limiter and size
class.

Candidates: the tiled kernels with 64, 128 or 256 cells per tile (one compute thread per
cell, or 128 threads over 256 cells — two cells per thread), and the per-cell kernels with
128 or 256 threads per block (no tile staging: the other fusion split).  A size class is
round(log2(real cells)); each class is tuned once on a supersonic wedge of about that many
triangles and the winner is stored in a JSON cache ($HCFD_AUTOTUNE_CACHE, default
~/.cache/hcfd_b200/autotune.json).
"""
from __future__ import annotations

import json
import math
import os
import subprocess

from . import (FP32, FP64, GLOBAL_CFL, KERNEL_CELL, KERNEL_TILED, LIMITER_BJ, NUMBER_RANDOM, Mesh, Solver,
               wedge_case)

CANDIDATES = (
    dict(kernel=KERNEL_TILED, tile=64, block=64),
    dict(kernel=KERNEL_TILED, tile=128, block=128),
    dict(kernel=KERNEL_TILED, tile=256, block=256),
    dict(kernel=KERNEL_TILED, tile=256, block=128),
    dict(kernel=KERNEL_CELL, tile=0, block=128),
    dict(kernel=KERNEL_CELL, tile=0, block=256),
)


def cache_path() -> str:
    return os.environ.get("HCFD_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "hcfd_b200", "autotune.json"))


def gpu_name() -> str:
    try:
        out = subprocess.run(["nvidia-smi", "--query-gpu=name", "--format=csv,noheader", "-i", "0"],
                             capture_output=True, text=True, timeout=20).stdout.strip()
        return out or "unknown"
    except (OSError, subprocess.SubprocessError):
        return "unknown"


def size_class(ncells: int) -> int:
    return max(10, min(24, int(round(math.log2(max(ncells, 2))))))


def _key(cls: int, precision: int, limiter: int, arena_shapes: bool) -> str:
    return f"{gpu_name()}|{'fp32' if precision == FP32 else 'fp64'}|lim{limiter}|c{cls}|{'arena' if arena_shapes else 'all'}"


def _load() -> dict:
    try:
        with open(cache_path()) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _store(d: dict) -> None:
    p = cache_path()
    os.makedirs(os.path.dirname(p), exist_ok=True)
    tmp = p + ".tmp"
    with open(tmp, "w") as fh:
        json.dump(d, fh, indent=1, sort_keys=True)
    os.replace(tmp, p)


def tune_class(cls: int, precision: int = FP64, limiter: int = LIMITER_BJ, steps: int = 40,
               arena_shapes: bool = False) -> dict:
    """Times every candidate on a wedge of about 2**cls triangles; returns the timings.
    With `arena_shapes` only the shapes an arena can run (tiled, one thread per cell)."""
    ny1 = max(2, int(round(math.sqrt(2 ** cls / 4.0))))
    mesh = Mesh.wedge(2 * ny1 + 1, ny1 + 1, seed=4321, numbering=NUMBER_RANDOM)
    bcmap, qbc, q = wedge_case(2.5)
    res = []
    for c in CANDIDATES:
        if arena_shapes and (c["kernel"] != KERNEL_TILED or c["block"] != c["tile"]):
            continue
        s = Solver(mesh, precision=precision, limiter=limiter, **c)
        s.gather_bcs(bcmap, qbc)
        s.initialise(q)
        s.step(5, GLOBAL_CFL, 0.5)
        ms = s.step_timed(steps, GLOBAL_CFL, 0.5) / steps
        res.append(dict(c, ms_per_step=ms))
        del s
    res.sort(key=lambda r: r["ms_per_step"])
    return dict(best=res[0], timings=res, cells=mesh.Nc)


def best(ncells: int, precision: int = FP64, limiter: int = LIMITER_BJ, tune: bool = True,
         arena_shapes: bool = False) -> dict:
    """The cached winner for this size class ({kernel, tile, block}); tunes and caches it
    when missing and `tune` is true, else returns the default shape."""
    cls = size_class(ncells)
    key = _key(cls, precision, limiter, arena_shapes)
    d = _load()
    if key not in d:
        if not tune:
            return dict(kernel=KERNEL_TILED, tile=128, block=128)
        d[key] = tune_class(cls, precision, limiter, arena_shapes=arena_shapes)
        _store(d)
    b = d[key]["best"]
    return dict(kernel=b["kernel"], tile=b["tile"], block=b["block"])
