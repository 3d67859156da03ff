"""Autotuner of the step kernels' launch shape, cached per GPU, precision, limiter and size
class.

Two tunings:
  - a single-mesh solver (Solver): the tiled kernels with 64, 128 or 256 cells per tile for
    both passes (one compute thread per cell, or 128 threads over 256 cells — two cells per
    thread), with separate pass-1 / pass-2 tilings (the library's default, 224 / 192 cells in
    FP64 and 256 / 128 in FP32, and 256 / 128), against the per-cell kernels with 128 or
    256 threads per block (no tile staging: the other fusion split), timed on one wedge of
    the size class;
  - an arena (Arena): its tile size (64, 128 or 256 cells, one thread per cell), timed on
    an arena holding copies of a wedge of the size class, about 2 million cells in all, so
    that the timing is that of a full device and not of one launch-bound instance.
A size class is round(log2(real cells)), clamped to [10, 24].  The winners are stored in a
JSON cache ($HCFD_AUTOTUNE_CACHE, default ~/.cache/hcfd_b200/autotune.json).

    python -m cfd_optimisations_b200.autotune --cells N [--fp32] [--arena]
"""
from __future__ import annotations

import json
import math
import os
import subprocess
import time

from . import (FP64, GLOBAL_CFL, KERNEL_CELL, KERNEL_TILED, LIMITER_BJ, NUMBER_RANDOM, Mesh, Solver, device_sync,
               wedge_case)

SOLVER_SHAPES = (
    dict(kernel=KERNEL_TILED, tile=0, tile2=0, block=0),          # the library's default split
    dict(kernel=KERNEL_TILED, tile=256, tile2=128, block=0),
    dict(kernel=KERNEL_TILED, tile=64, tile2=0, block=64),
    dict(kernel=KERNEL_TILED, tile=128, tile2=0, block=128),
    dict(kernel=KERNEL_TILED, tile=256, tile2=0, block=256),
    dict(kernel=KERNEL_TILED, tile=256, tile2=0, block=128),
    dict(kernel=KERNEL_CELL, tile=0, tile2=0, block=128),
    dict(kernel=KERNEL_CELL, tile=0, tile2=0, block=256),
)
DEFAULT_SHAPE = SOLVER_SHAPES[0]
ARENA_TILES = (64, 128, 256)


def cache_path() -> str:
    return os.environ.get("HCFD_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "hcfd_b200", "autotune.json"))


def gpu_name() -> str:
    try:
        out = subprocess.run(["nvidia-smi", "--query-gpu=name", "--format=csv,noheader", "-i", "0"],
                             capture_output=True, text=True, timeout=20).stdout.strip()
        return out.splitlines()[0] if out else "unknown"
    except (OSError, subprocess.SubprocessError):
        return "unknown"


def size_class(ncells: int) -> int:
    return max(10, min(24, int(round(math.log2(max(ncells, 2))))))


def class_mesh(cls: int) -> Mesh:
    """A wedge on a 2:1 node grid with about 2**cls triangles."""
    ny1 = max(2, int(round(math.sqrt(2 ** cls / 4.0))))
    return Mesh.wedge(2 * ny1 + 1, ny1 + 1, seed=4321, numbering=NUMBER_RANDOM)


def _key(kind: str, cls: int, precision: int, limiter: int) -> str:
    return f"{gpu_name()}|{kind}|{'fp64' if precision == FP64 else 'fp32'}|lim{limiter}|c{cls}"


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


def tune_solver(cls: int, precision: int = FP64, limiter: int = LIMITER_BJ, steps: int = 40) -> dict:
    """Times every solver shape on one wedge of the class; returns the timings, best first."""
    mesh = class_mesh(cls)
    bcmap, qbc, q = wedge_case(2.5)
    res = []
    for c in SOLVER_SHAPES:
        s = Solver(mesh, precision=precision, limiter=limiter, **c)
        s.gather_bcs(bcmap, qbc)
        s.initialise(q)
        s.step(5, GLOBAL_CFL, 0.5)
        res.append(dict(c, ms_per_step=s.step_timed(steps, GLOBAL_CFL, 0.5) / steps))
        del s
    res.sort(key=lambda r: r["ms_per_step"])
    return dict(best=res[0], timings=res, cells=mesh.Nc)


def tune_arena(cls: int, precision: int, limiter: int = LIMITER_BJ, steps: int = 40,
               target_cells: int = 2_000_000) -> dict:
    """Times every arena tile size on an arena of copies of a wedge of the class."""
    from .arena import Arena
    mesh = class_mesh(cls)
    copies = max(1, min(512, target_cells // mesh.Nc))
    bcmap, qbc, q = wedge_case(2.5)
    res = []
    for tile in ARENA_TILES:
        a = Arena(int(max(1e9, 600.0 * copies * mesh.Nc)), precision=precision, limiter=limiter, tile=tile,
                  max_instances=copies)
        for _ in range(copies):
            if a.admit(mesh, bcmap, qbc, q, 0.5) is None:
                raise RuntimeError("autotune: arena full")
        a.step(4)
        a.poll()
        device_sync()
        t0 = time.perf_counter()
        a.step(steps)
        a.poll()
        res.append(dict(tile=tile, ms_per_step=1e3 * (time.perf_counter() - t0) / steps))
        del a
    res.sort(key=lambda r: r["ms_per_step"])
    return dict(best=res[0], timings=res, cells=mesh.Nc, copies=copies)


def best_solver_shape(ncells: int, precision: int = FP64, limiter: int = LIMITER_BJ, tune: bool = True) -> dict:
    """The cached winner for a single mesh of this size ({kernel, tile, tile2, block}, the
    Solver keywords); tuned and cached when missing and `tune` is true, else the library's
    default shape."""
    cls = size_class(ncells)
    key = _key("solver", cls, precision, limiter)
    d = _load()
    if key not in d or "tile2" not in d[key]["best"]:
        if not tune:
            return dict(DEFAULT_SHAPE)
        d[key] = tune_solver(cls, precision, limiter)
        _store(d)
    b = d[key]["best"]
    return dict(kernel=b["kernel"], tile=b["tile"], tile2=b["tile2"], block=b["block"])


def best_arena_tile(ncells: int, precision: int, limiter: int = LIMITER_BJ, tune: bool = True) -> int:
    """The cached arena tile size for instances of about this size."""
    cls = size_class(ncells)
    key = _key("arena", cls, precision, limiter)
    d = _load()
    if key not in d:
        if not tune:
            return 128
        d[key] = tune_arena(cls, precision, limiter)
        _store(d)
    return int(d[key]["best"]["tile"])


def main():
    import argparse
    from . import FP32
    ap = argparse.ArgumentParser(description="tune (or read from the cache) the launch shape for a mesh size")
    ap.add_argument("--cells", type=int, required=True, help="real cells of the mesh (or of a typical instance)")
    ap.add_argument("--fp32", action="store_true")
    ap.add_argument("--arena", action="store_true", help="the arena tile size instead of the single-mesh shape")
    a = ap.parse_args()
    prec = FP32 if a.fp32 else FP64
    out = (dict(tile=best_arena_tile(a.cells, prec)) if a.arena else best_solver_shape(a.cells, prec))
    print(json.dumps(dict(size_class=size_class(a.cells), cache=cache_path(), **out)))


if __name__ == "__main__":
    main()
