"""Runs every kernel of the library a few times on one mid-sized case, so that a profiler
can report each kernel's device time and DRAM traffic from one run:

    python -m cfd_optimisations_b200.kernel_tour [--mesh 1025x513 --instances 64]

Single mesh (a 1025 x 513-node wedge, 1,048,576 triangles, RCM numbering, Venkatakrishnan
K = 5, M 2.5): the tiled FP64 and FP32 solvers and the per-cell FP64 and FP32 solvers, each
through set-up (geometry, renumbering, face records), initialise and boundary cells, steps in
global and local CFL mode, an asynchronous snapshot, download, upload, the wall pressure
coefficient and a checkpoint / restore.  Arena: `instances` wedges of 10,000 to 60,000
triangles admitted to one FP32 arena (admission kernels), stepped, polled, fetched,
checkpointed, restored and released.  An FP64 step on the single mesh moves 0.45 GB, well
above the 126 MB L2, so its kernels' DRAM figures are those of a full-size run; the FP32 and
arena passes move 0.1-0.2 GB each, about the L2's size, so part of their traffic can hit in L2.
Prints one JSON line with the cells touched and the steps taken.
"""
from __future__ import annotations

import argparse
import json
import os
import tempfile

import numpy as np

from . import (FP32, FP64, GLOBAL_CFL, KERNEL_CELL, KERNEL_TILED, LIMITER_BJ, LIMITER_VENKAT, LOCAL_CFL,
               NUMBER_RANDOM, NUMBER_RCM, Mesh, Solver, device_sync, wedge_case)
from .arena import Arena

LOWER_WALL = 2   # colour of the ramp in the generated wedge


def single(mesh: Mesh, precision: int, kernel: int, steps: int, tmp: str) -> dict:
    bcmap, qbc, q = wedge_case(2.5)
    s = Solver(mesh, limiter=LIMITER_VENKAT, venkat_K=5.0, precision=precision, kernel=kernel)
    s.gather_bcs(bcmap, qbc)
    s.initialise(q)
    s.step(steps, GLOBAL_CFL, 0.5)
    s.step(steps, LOCAL_CFL, 0.5)
    out = np.empty((4, mesh.Nc), dtype=np.float64)
    s.snapshot(out, prims=True).wait()
    U = s.U()
    s.upload(U)
    s.wall_cp(LOWER_WALL, q[0], q[3], float(np.hypot(q[1], q[2])))
    path = os.path.join(tmp, "tour.ckpt")
    s.checkpoint(path)
    s.restore(path)
    s.step(1, GLOBAL_CFL, 0.5)
    device_sync()
    st = s.stats()
    del s
    return dict(cells=mesh.Nc, faces=mesh.Nf, steps=2 * steps + 1, residual_l2=st["res_l2"])


def arena(n: int, steps: int, tmp: str, seed: int = 7) -> dict:
    rng = np.random.default_rng(seed)
    a = Arena(int(2e9), precision=FP32, limiter=LIMITER_BJ, max_instances=n + 8)
    slots, cells = [], 0
    for i in range(n):
        ntri = float(np.exp(rng.uniform(np.log(1e4), np.log(6e4))))
        ny1 = max(2, int(round(np.sqrt(ntri / 4.0))))
        m = Mesh.wedge(2 * ny1 + 1, ny1 + 1, theta_deg=float(rng.uniform(5.0, 15.0)), seed=100 + i,
                       numbering=NUMBER_RANDOM)
        bcmap, qbc, q = wedge_case(float(rng.uniform(1.8, 4.0)))
        k = a.admit(m, bcmap, qbc, q, 0.5)
        if k is None:
            raise RuntimeError("arena full")
        slots.append(k)
        cells += m.Nc
    a.step(steps)
    a.poll()
    a.fetch(slots[0])
    path = os.path.join(tmp, "tour_arena.ckpt")
    a.checkpoint(slots[0], path)
    a.restore(slots[0], path)
    a.step(2)
    a.poll()
    for k in slots:
        a.release(k)
    device_sync()
    del a
    return dict(instances=n, cells=cells, steps=steps + 2)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--mesh", default="1025x513")
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--instances", type=int, default=64)
    a = ap.parse_args()
    nx, ny = (int(x) for x in a.mesh.lower().split("x"))
    mesh = Mesh.wedge(nx, ny, theta_deg=15.0, seed=1234, numbering=NUMBER_RCM)
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, prec, kern in (("tiled_fp64", FP64, KERNEL_TILED), ("tiled_fp32", FP32, KERNEL_TILED),
                                 ("cell_fp64", FP64, KERNEL_CELL), ("cell_fp32", FP32, KERNEL_CELL)):
            out[name] = single(mesh, prec, kern, a.steps, tmp)
        out["arena_fp32"] = arena(a.instances, a.steps, tmp)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
