#!/usr/bin/env python
"""Benchmark of the per-step residual-and-update loop on the large supersonic wedge.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step" = one solver time step over the whole mesh): the triangulated wedge
of 2001 x 1001 nodes (4,000,000 triangles + 6,000 ghost cells, 6,003,000 faces), x in
[0, 3], top wall y = 1.5, ramp of 15 degrees from x = 0.5, interior nodes jittered by
U(+-0.15) of the local spacing, seeded diagonals; freestream rho 1.4, p 1, u 2.5 (M 2.5);
Venkatakrishnan limiter K = 5; global CFL 0.5; FP64; cells RCM-renumbered.  Synthetic,
generated in-process from fixed seeds.

Metric: cell-updates/s = real cells x steps / time.  The per-step working set (~1.7 GB)
is far larger than the 126 MB L2, so no flush is needed between steps.

Under torchrun (N > 1) every rank runs its own replica of the workload on its own GPU
(the path does not shard: replicas only, no collective on the data path); the reported
time is the maximum over ranks and the value is the total over ranks.

`--impl reference` times the reference's own CPU solver (compiled unchanged into
oracle/_ref): its fastest layout that matches its Base layout to 1e-12 after one step
(VEC, AVX2 build), fixed dt, Barth-Jespersen limiter (the reference has no
Venkatakrishnan limiter and no CFL control), one independent instance per host core.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX, NY = 2001, 1001
THETA, MACH, SEED = 15.0, 2.5, 1234
VENKAT_K, CFL = 5.0, 0.5
WORKLOAD = (f"supersonic wedge {NX}x{NY} nodes ({2 * (NX - 1) * (NY - 1):,} triangles), M{MACH} "
            f"{THETA:g}deg, Venkatakrishnan K{VENKAT_K:g}, global CFL {CFL}, FP64")


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.out = None

    def __enter__(self):
        try:
            self.out = tempfile.TemporaryFile(mode="w+")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.out.seek(0)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "samples": len(sm), "reasons": sorted(reasons)}


def dist_setup(nproc: int):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as td
        torch.cuda.set_device(local)
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = td
    return rank, world, local, dist


def allmax(dist, x: float) -> float:
    """Maximum of x over the ranks (the slowest rank's time)."""
    if dist is None:
        return x
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate(units_per_rank: float, world: int, ms_max: float) -> float:
    """Whole-job throughput: every rank processed the same units; the job took the slowest
    rank's time."""
    return units_per_rank * world / (ms_max * 1e-3)


def barrier(dist):
    if dist is not None:
        dist.barrier()


def make_mesh(numbering):
    import cfd_optimisations_b200 as H
    return H.Mesh.wedge(NX, NY, theta_deg=THETA, jitter=0.15, seed=SEED, numbering=numbering)


def traffic_from_profiles(kernel: str, workload_key: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if one matches."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as fh:
        d = json.load(fh)
    e = d.get(workload_key, {}).get(kernel)
    return None if e is None else float(e)


def cpu_reference(mesh, steps: int, dt: float, threads: int | None = None):
    """The reference solver's VEC layout (AVX2 build, compiled unchanged) over `threads`
    independent instances; returns (cell-updates/s, threads, seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import cfd_optimisations_b200 as H
    if not O.RefSolver.available():
        return None
    nthreads = threads or os.cpu_count() or 1
    try:  # about 1.7 GB per instance of this mesh
        with open("/proc/meminfo") as fh:
            avail = next(int(l.split()[1]) for l in fh if l.startswith("MemAvailable")) * 1024
        nthreads = max(1, min(nthreads, int(0.6 * avail / 1.8e9)))
    except (OSError, StopIteration):
        pass
    bcmap, qbc, q = H.wedge_case(MACH)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "wedge.hmsh")
        mesh.write(path)
        secs = O.RefSolver.bench("VEC", path, bcmap, qbc, q, nthreads, 1, steps, dt)
    ntri = 2 * (NX - 1) * (NY - 1)
    return ntri * steps * nthreads / secs, nthreads, secs


def run_reference_arm(args):
    rank, world, local, dist = int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), 0, None
    if rank != 0:
        return 0
    import cfd_optimisations_b200 as H
    try:
        mesh = make_mesh(H.NUMBER_RCM)
    except Exception as e:  # no native library: the mesh generator is part of it
        print(json.dumps({"impl": "reference", "unavailable": f"mesh generator unavailable: {e}"}))
        return 0
    # dt: the global CFL-0.5 dt of the freestream state (constant while the flow is uniform).
    bcmap, qbc, q = H.wedge_case(MACH)
    a = (1.4 * q[3] / q[0]) ** 0.5
    dx = 3.0 / (NX - 1)
    dt = CFL * 0.5 * dx / (q[1] + a)
    steps = max(1, min(args.steps, 2))
    r = cpu_reference(mesh, steps, dt)
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libhcfd_ref.so not built"}))
        return 0
    value, threads, secs = r
    sample = (f"reference VEC layout (AVX2 build, compiled unchanged), {threads} independent instances x "
              f"{steps} steps of the {NX}x{NY} wedge after 1 warm-up step; fixed dt {dt:.3e}; "
              f"Barth-Jespersen (the reference has no Venkatakrishnan limiter or CFL control)")
    line = {"metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": args.gpus,
            "steps": steps, "warmup": 1, "ms_per_step": secs / steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD + ", RCM numbering", "parallelism": f"{threads} CPU replicas"},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": threads, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def e2e_run(H, mesh, steps: int):
    """Through the C ABI with host buffers: pinned initial state uploaded, `steps` steps each
    reading back its statistics (dt and residual), final primitive state downloaded into a
    pinned host buffer.  Host wall clock around the whole sequence."""
    s = H.Solver(mesh, limiter=H.LIMITER_VENKAT, venkat_K=VENKAT_K, precision=H.FP64)
    bcmap, qbc, q = H.wedge_case(MACH)
    s.gather_bcs(bcmap, qbc)
    s.initialise(q)
    U0 = np.ascontiguousarray(s.U())
    Q = np.empty_like(U0)
    H.pin(U0)
    H.pin(Q)
    try:
        s.step(2, H.GLOBAL_CFL, CFL)
        s.upload(U0)
        t0 = time.perf_counter()
        s.upload(U0)
        for _ in range(steps):
            s.step(1, H.GLOBAL_CFL, CFL, wait=True)
        s.download(prims=True, out=Q)
        t = time.perf_counter() - t0
    finally:
        H.unpin(U0)
        H.unpin(Q)
    nbytes = U0.nbytes
    stats_bytes = 40
    return t, nbytes / steps, (nbytes + stats_bytes * steps) / steps


def main():
    global NX, NY, WORKLOAD
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-variants", action="store_true", help="skip the random-numbering and FP32 lines")
    ap.add_argument("--mesh", default=f"{NX}x{NY}", help="node grid NXxNY (profiling of smaller cases)")
    ap.add_argument("--kernel", choices=["tiled", "cell"], default="tiled",
                    help="step kernel family (the per-cell gather kernels are the other fusion split)")
    ap.add_argument("--profile-only", action="store_true",
                    help="warm-up and timed steps only (no end-to-end, variants or CPU legs): for ncu")
    args = ap.parse_args()
    NX, NY = (int(x) for x in args.mesh.lower().split("x"))
    WORKLOAD = (f"supersonic wedge {NX}x{NY} nodes ({2 * (NX - 1) * (NY - 1):,} triangles), M{MACH} "
                f"{THETA:g}deg, Venkatakrishnan K{VENKAT_K:g}, global CFL {CFL}, FP64")
    if args.profile_only:
        args.no_cpu = args.no_variants = True
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference_arm(args)

    import cfd_optimisations_b200 as H
    rank, world, local, dist = dist_setup(args.gpus)
    H.set_device(local)
    mesh = make_mesh(H.NUMBER_RCM)
    bcmap, qbc, q = H.wedge_case(MACH)
    kernel = H.KERNEL_CELL if args.kernel == "cell" else H.KERNEL_TILED
    s = H.Solver(mesh, limiter=H.LIMITER_VENKAT, venkat_K=VENKAT_K, precision=H.FP64, kernel=kernel)
    s.gather_bcs(bcmap, qbc)
    s.initialise(q)
    ntri = s.Nreal
    Nc, Nf = s.Nc, s.Nf
    s.step(args.warmup, H.GLOBAL_CFL, CFL)
    # per-kernel events on every 10th step of the timed region (the events' own gaps stay
    # out of the other nine)
    s.profile(True, every=10)
    barrier(dist)
    H.device_sync()
    with ClockSampler(local) as clk:
        ms = s.step_timed(args.steps, H.GLOBAL_CFL, CFL)
    H.device_sync()
    barrier(dist)
    prof = s.profile_read()
    s.profile(False)
    st = s.stats()
    ms_max = allmax(dist, ms)
    value = aggregate(ntri * args.steps, world, ms_max)

    # Roofline of the dominant kernel.  Algorithmic bytes (two-pass minimum, w = 8):
    #   pass 1: U (4w) + iv (w) + phiG (8w) per cell, (8 + 7w) per face
    #   pass 2: U (4w) + phiG (8w) + iv (w) + U' (4w) per cell, (8 + 7w) per face
    w = 8
    b1 = 13 * w * Nc + (8 + 7 * w) * Nf
    b2 = 17 * w * Nc + (8 + 7 * w) * Nf
    t1 = prof["ms_pass1"] / max(prof["n_pass1"], 1)
    t2 = prof["ms_pass2"] / max(prof["n_pass2"], 1)
    dom, b, t = ("pass2", b2, t2) if t2 >= t1 else ("pass1", b1, t1)
    peak, peak_kind = peaks()
    achieved = b / (t * 1e-3) / 1e9
    step_achieved = (b1 + b2) / (ms_max / args.steps * 1e-3) / 1e9
    traffic = traffic_from_profiles(dom, f"fp64_rcm_{NX}x{NY}" + ("_cell" if args.kernel == "cell" else ""))

    line = {"metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD + ", RCM numbering" + (", per-cell kernels" if args.kernel == "cell" else ""),
                       "cells": Nc, "real_cells": ntri, "faces": Nf,
                       "parallelism": f"{world} replica(s), one per GPU, no collective",
                       "l2": "per-step working set > 1.6 GB, far above the 126 MB L2; no flush"},
            "gpu_launches": s.launches_per_step() * args.steps,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": f"{peak_kind} hbm_gbs",
                         "algorithmic_bytes_per_launch": b,
                         "ms_per_launch": {"pass1": t1, "pass2": t2},
                         "step_achieved": step_achieved, "step_frac": step_achieved / peak},
            "clocks": clk.summary(),
            "residual_l2_last": st["res_l2"]}

    # End to end through the C ABI with host buffers.
    del s
    if not args.profile_only:
        et, h2d, d2h = e2e_run(H, mesh, args.steps)
        et = allmax(dist, et)
        line["e2e"] = {"value": ntri * args.steps * world / et, "unit": "cell-updates/s",
                       "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                       "how": "hcfd_gpu_upload of the pinned state, per step hcfd_gpu_step + stats read, "
                              "hcfd_gpu_download of the primitive state into pinned memory; host wall clock"}

    if not args.no_variants and rank == 0:
        var = {}
        for name, num, prec in (("fp64_random", H.NUMBER_RANDOM, H.FP64), ("fp32_rcm", H.NUMBER_RCM, H.FP32)):
            m2 = mesh if num == H.NUMBER_RCM else make_mesh(num)
            v = H.Solver(m2, limiter=H.LIMITER_VENKAT, venkat_K=VENKAT_K, precision=prec)
            v.gather_bcs(bcmap, qbc)
            v.initialise(q)
            v.step(args.warmup, H.GLOBAL_CFL, CFL)
            k = min(args.steps, 200)
            mv = v.step_timed(k, H.GLOBAL_CFL, CFL)
            ww = 8 if prec == H.FP64 else 4
            balg = 30 * ww * Nc + 2 * (8 + 7 * ww) * Nf
            var[name] = {"cell_updates_per_s": ntri * k / (mv * 1e-3), "ms_per_step": mv / k,
                         "step_achieved_GBs": balg / (mv / k * 1e-3) / 1e9,
                         "step_frac": balg / (mv / k * 1e-3) / 1e9 / peak}
            del v
        line["variants"] = var

    if rank == 0 and world == 1 and not args.no_cpu:
        dt_cpu = st["dt"]
        r = cpu_reference(mesh, 2, dt_cpu)
        if r is not None:
            cv, threads, secs = r
            line["cpu_baseline"] = {"value": cv, "unit": "cell-updates/s", "cores": threads, "kind": "reference",
                                    "sample": f"reference VEC layout (AVX2 build, compiled unchanged), {threads} "
                                              f"independent instances x 2 steps of this mesh (BJ limiter, fixed "
                                              f"dt {dt_cpu:.3e}), {secs:.1f} s"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
