"""Batched solves: many wedge instances of uneven size packed into one device arena and
advanced together, against the plain FP64 solver looped over the same instances.

    python -m cfd_optimisations_b200.batched [--instances 512 --steps 2000 --seed 2024]

Instances: triangle counts log-uniform in [2,000, 200,000] on a 2:1 node grid, M ~ U[1.8, 4.0],
ramp angle ~ U[5, 15] degrees, a jitter/permutation seed per instance; freestream initial
state; Barth-Jespersen limiter; global CFL 0.5 per instance; a fixed number of steps each.
The arena runs in FP32 with compensated residual sums, its tile size picked by the
autotuner (autotune.py) for the median instance size; the loop runs each instance alone
through the plain FP64 solver.  Prints one JSON object: device throughput of both, the
speed-up, and per instance the FP32 arena's relative L-inf error against the FP64 loop beside
the spread one rounding of the initial state gives the FP64 solve itself.
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

from . import FP32, FP64, GLOBAL_CFL, LIMITER_BJ, NUMBER_RANDOM, Mesh, Solver, wedge_case
from . import autotune
from .arena import Arena


def instance_specs(n: int = 512, seed: int = 2024, lo: float = 2e3, hi: float = 2e5):
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n):
        ntri = math.exp(rng.uniform(math.log(lo), math.log(hi)))
        ny1 = max(2, int(round(math.sqrt(ntri / 4.0))))
        specs.append(dict(nx=2 * ny1 + 1, ny=ny1 + 1, mach=float(rng.uniform(1.8, 4.0)),
                          theta=float(rng.uniform(5.0, 15.0)), seed=1234 + i))
    return specs


def build(specs, workers: int = 8):
    """The instances' meshes, generated by `workers` threads (the generator releases the GIL)."""
    from concurrent.futures import ThreadPoolExecutor
    gen = lambda s: Mesh.wedge(s["nx"], s["ny"], theta_deg=s["theta"], seed=s["seed"], numbering=NUMBER_RANDOM)
    with ThreadPoolExecutor(max_workers=max(1, workers)) as ex:
        return list(ex.map(gen, specs))


def rel_linf_max(a, b) -> float:
    """max over variables of max|a-b| / max|b| (the tests' relative L-infinity)."""
    return float((np.abs(a - b).max(axis=1) / np.maximum(np.abs(b).max(axis=1), 1e-300)).max())


def accuracy_summary(e32, e64, bound: float = 1e-5) -> dict:
    """FP32-vs-FP64 errors beside the FP64 one-rounding spreads of the same solves."""
    e32, e64 = np.asarray(e32, dtype=float), np.asarray(e64, dtype=float)
    return dict(n=int(e32.size), bound=bound,
                fp32_vs_fp64=dict(median=float(np.median(e32)), max=float(e32.max())),
                fp64_one_rounding_spread=dict(median=float(np.median(e64)), max=float(e64.max())),
                fp32_within_bound=int((e32 <= bound).sum()),
                fp64_spread_above_bound=int((e64 > bound).sum()),
                fp32_within_10x_fp64_spread=int((e32 <= 10.0 * e64).sum()),
                fp32_within_bound_or_10x_spread=int(((e32 <= bound) | (e32 <= 10.0 * e64)).sum()))


def run_arena(meshes, specs, steps, precision=FP32, limiter=LIMITER_BJ, cfl=0.5, tile=0):
    cells = sum(m.Nc for m in meshes)
    a = Arena(int(max(2e9, 400.0 * cells)), precision=precision, limiter=limiter, tile=tile,
              max_instances=len(meshes) + 8)
    slots = []
    t0 = time.perf_counter()
    for m, s in zip(meshes, specs):
        bcmap, qbc, q = wedge_case(s["mach"])
        k = a.admit(m, bcmap, qbc, q, cfl)
        if k is None:
            raise RuntimeError("arena full")
        slots.append(k)
    t_admit = time.perf_counter() - t0
    a.step(2)
    a.poll()
    t0 = time.perf_counter()
    a.step(steps - 2)
    stats = a.poll()
    t_run = time.perf_counter() - t0
    return a, slots, stats, t_admit, t_run


def run_loop(meshes, specs, steps, precision=FP64, limiter=LIMITER_BJ, cfl=0.5, rho_scale=1.0):
    ms, t_create, out = 0.0, 0.0, []
    for m, s in zip(meshes, specs):
        bcmap, qbc, q = wedge_case(s["mach"])
        t0 = time.perf_counter()
        sol = Solver(m, precision=precision, limiter=limiter)
        sol.gather_bcs(bcmap, qbc)
        qi = list(q)
        qi[0] *= rho_scale
        sol.initialise(qi)
        t_create += time.perf_counter() - t0
        sol.step(2, GLOBAL_CFL, cfl)
        ms += sol.step_timed(steps - 2, GLOBAL_CFL, cfl)
        out.append(sol.U())
        del sol
    return ms, t_create, out


def run(instances: int = 512, steps: int = 2000, seed: int = 2024, loop: bool = True, tile: int = 0,
        spread_every: int = 1, per_instance: bool = False) -> dict:
    """Config-4 batched solves: the FP32 arena against the plain FP64 loop on the same instances.

    Both sides are timed on the device over steps 3..`steps` of every instance (the first two
    steps, which build the CUDA graphs, stay out); mesh generation and admission are reported
    apart.  Every `spread_every`-th instance is also solved in FP64 from an initial density one
    rounding step larger (x (1 + 2^-52)): that solve's distance from the unperturbed FP64 solve
    is the spread rounding alone produces, reported beside the FP32 error of the same instance."""
    specs = instance_specs(instances, seed)
    t0 = time.perf_counter()
    meshes = build(specs)
    t_gen = time.perf_counter() - t0
    real = [m.Nc - (2 * (s["nx"] - 1) + 2 * (s["ny"] - 1)) for m, s in zip(meshes, specs)]
    median = int(np.median(real))
    tile = tile or autotune.best_arena_tile(median, FP32, LIMITER_BJ)
    arena, slots, stats, t_admit, t_run = run_arena(meshes, specs, steps, tile=tile)
    upd = sum(real) * (steps - 2)
    out = dict(workload=dict(instances=instances, steps=steps, triangles_total=int(sum(real)),
                             triangles_median=median, seed=seed, limiter="barth-jespersen", cfl=0.5),
               mesh_generation_s=t_gen,
               arena=dict(precision="fp32-compensated", tile=tile, admit_s=t_admit, run_s=t_run,
                          cell_updates_per_s=upd / t_run, solves_per_s=instances / t_run,
                          nonfinite=sum(1 for s in stats.values() if s["nonfinite"])))
    if loop:
        ms, t_create, U64 = run_loop(meshes, specs, steps)
        U32 = [arena.fetch(k) for k in slots]
        del arena
        out["fp64_loop"] = dict(device_s=ms / 1e3, create_s=t_create, cell_updates_per_s=upd / (ms / 1e3),
                                solves_per_s=instances / (ms / 1e3))
        out["speedup_solves_per_s"] = out["arena"]["solves_per_s"] / out["fp64_loop"]["solves_per_s"]
        sub = list(range(0, len(meshes), max(1, spread_every)))
        _, _, U64p = run_loop([meshes[i] for i in sub], [specs[i] for i in sub], steps, rho_scale=1.0 + 2.0 ** -52)
        e32 = [rel_linf_max(U32[i], U64[i]) for i in sub]
        e64 = [rel_linf_max(up, U64[i]) for i, up in zip(sub, U64p)]
        out["fp32_vs_fp64_rel_linf"] = dict(n=instances, median=float(np.median([rel_linf_max(u, v) for u, v in
                                                                             zip(U32, U64)])),
                                            max=max(rel_linf_max(u, v) for u, v in zip(U32, U64)))
        out["accuracy"] = accuracy_summary(e32, e64)
        if per_instance:
            out["per_instance"] = [dict(instance=i, triangles=real[i], fp32_vs_fp64=a, fp64_one_rounding_spread=b)
                                   for i, a, b in zip(sub, e32, e64)]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--instances", type=int, default=512)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--no-loop", action="store_true", help="skip the FP64 loop baseline")
    ap.add_argument("--tile", type=int, default=0, help="arena tile size (0: autotuned for the median instance)")
    ap.add_argument("--spread-every", type=int, default=1,
                    help="FP64 one-rounding spread on every k-th instance (1: all)")
    a = ap.parse_args()
    print(json.dumps(run(a.instances, a.steps, a.seed, not a.no_loop, a.tile, a.spread_every, per_instance=True)))


if __name__ == "__main__":
    main()
