#!/usr/bin/env python
"""Benchmark of the per-step residual-and-update loop on the large supersonic wedge, with the
batched and served legs.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Headline workload (one "step" = one solver time step over the whole mesh): the triangulated
wedge of 2001 x 1001 nodes (4,000,000 triangles + 6,000 ghost cells, 6,003,000 faces), x in
[0, 3], top wall y = 1.5, ramp of 15 degrees from x = 0.5, interior nodes jittered by
U(+-0.15) of the local spacing, seeded diagonals; freestream rho 1.4, p 1, u 2.5 (M 2.5);
Venkatakrishnan limiter K = 5; global CFL 0.5; FP64; cells RCM-renumbered.  Synthetic,
generated in-process from fixed seeds.

Metric: cell-updates/s = real cells x steps / time.  The per-step working set (~1.7 GB)
is far larger than the 126 MB L2, so no flush is needed between steps.

Legs beside the headline (rank 0, one GPU):
* variants: random cell numbering; FP32; and the reference's own arithmetic on the same mesh
  (Barth-Jespersen, fixed dt), the configuration the reference arm can run;
* cpu_baseline: the reference's fastest valid CPU layout on the host cores, same mesh, same
  fixed-dt configuration;
* batched: 512 wedges of 2,000-200,000 triangles in one FP32 arena, 2000 steps each, against
  the plain FP64 solver looped over them (cfd_optimisations_b200/batched.py);
* served: the first requests of the seeded 10,000-request stream (Poisson arrivals at 100/s),
  continuous batching into one FP32 arena, against the plain sequential FP64 loop run on every
  one of the same requests (cfd_optimisations_b200/serve.py).

Under torchrun (N > 1) every rank runs its own replica of the headline workload on its own GPU
(the path does not shard: replicas only, no collective on the data path); the reported time
is the maximum over ranks and the value is the total over ranks.

`--impl reference` times the reference's own CPU solver (compiled unchanged into oracle/_ref):
its fastest layout that matches its Base layout to 1e-12 after one step (VEC, AVX2 build), on
the same mesh written by the oracle's generator (the product library is not loaded), fixed dt
(the reference has no CFL control) and the Barth-Jespersen limiter (it has no Venkatakrishnan
limiter), one independent instance per host core.
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
REF_MAX_STEPS, REF_MAX_WARMUP = 60, 5      # keeps the reference arm within about two minutes


def workload(precision: str = "fp64") -> str:
    return (f"supersonic wedge {NX}x{NY} nodes ({2 * (NX - 1) * (NY - 1):,} triangles), M{MACH} "
            f"{THETA:g}deg, Venkatakrishnan K{VENKAT_K:g}, global CFL {CFL}, {precision.upper()}, RCM numbering")


def freestream_case(mach: float = MACH, rho: float = 1.4, p: float = 1.0, gma: float = 1.4):
    """BC map and states of the wedge case (the same values as the package's wedge_case):
    colour tags 1 upper / 2 lower SYMMETRY, 3 inlet SUPINLET, 4 outlet SUPOUTLET
    (src/Test.cpp:64); uniform freestream (rho, M a, 0, p)."""
    a = (gma * p / rho) ** 0.5
    q = np.array([rho, mach * a, 0.0, p])
    return np.array([0, 0, 0, 2, 4], dtype=np.int32), np.tile(q, (4, 1)), q


def reference_dt() -> float:
    """The fixed dt of the reference's configuration (it has no CFL control, so both arms use
    this one number): 0.009 / (NX - 1), 4.5e-6 on the 2001 x 1001 mesh, where the global CFL-0.5
    dt of the freestream is 1.22e-5 (the jittered cells near the ramp are the smallest): a
    CFL number of about 0.18, stable while the shock forms over the benchmark's steps."""
    return 0.009 / (NX - 1)


def reference_workload() -> str:
    return (f"supersonic wedge {NX}x{NY} nodes ({2 * (NX - 1) * (NY - 1):,} triangles), M{MACH} "
            f"{THETA:g}deg, Barth-Jespersen, fixed dt {reference_dt():.6e}, FP64, RCM numbering")


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


def cpu_reference(steps: int, warmup: int, threads: int | None = None):
    """The reference solver's VEC layout (AVX2 build, compiled unchanged) over `threads`
    independent instances of the wedge (written by the oracle's generator, not the product
    library), Barth-Jespersen, fixed dt reference_dt(); returns (cell-updates/s, threads,
    seconds, sample text) or None when the reference library was not built."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not O.RefSolver.available():
        return None
    nthreads = threads or os.cpu_count() or 1
    try:  # about 1.8 GB per instance of this mesh
        with open("/proc/meminfo") as fh:
            avail = next(int(l.split()[1]) for l in fh if l.startswith("MemAvailable")) * 1024
        nthreads = max(1, min(nthreads, int(0.6 * avail / (1.8e9 * NX * NY / 2.003e6))))
    except (OSError, StopIteration):
        pass
    bcmap, qbc, q = freestream_case()
    dt = reference_dt()
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "wedge.hmsh")
        O.wedge_hmsh(path, NX, NY, theta_deg=THETA, jitter=0.15, seed=SEED, numbering=O.NUMBER_RCM)
        secs = O.RefSolver.bench("VEC", path, bcmap, qbc, q, nthreads, warmup, steps, dt)
    ntri = 2 * (NX - 1) * (NY - 1)
    sample = (f"reference VEC layout (AVX2 build, compiled unchanged), {nthreads} independent instances x {steps} "
              f"steps of the {NX}x{NY} wedge after {warmup} warm-up steps; Barth-Jespersen, fixed dt {dt:.6e} "
              f"(the reference has no Venkatakrishnan limiter or CFL control); mesh from the oracle's generator")
    return ntri * steps * nthreads / secs, nthreads, secs, sample


def run_reference_arm(args):
    """Rank 0 alone times the reference (the other ranks exit without work)."""
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    steps, warm = max(1, min(args.steps, REF_MAX_STEPS)), max(1, min(args.warmup, REF_MAX_WARMUP))
    r = cpu_reference(steps, warm)
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libhcfd_ref.so not built"}))
        return 0
    value, threads, secs, sample = r
    line = {"metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": args.gpus,
            "steps": steps, "warmup": warm, "ms_per_step": secs / steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": reference_workload(), "parallelism": f"{threads} CPU replicas, one per host thread"},
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


def timed_variant(H, mesh, ntri, Nc, Nf, peak, steps, warmup, limiter, prec, mode, value):
    """Device time of `steps` steps of one more configuration on the same kind of mesh."""
    v = H.Solver(mesh, limiter=limiter, venkat_K=VENKAT_K, precision=prec)
    bcmap, qbc, q = H.wedge_case(MACH)
    v.gather_bcs(bcmap, qbc)
    v.initialise(q)
    v.step(warmup, mode, value)
    mv = v.step_timed(steps, mode, value)
    ww = 8 if prec == H.FP64 else 4
    balg = 30 * ww * Nc + 2 * (8 + 7 * ww) * Nf
    return {"cell_updates_per_s": ntri * steps / (mv * 1e-3), "ms_per_step": mv / steps, "steps": steps,
            "step_achieved_GBs": balg / (mv / steps * 1e-3) / 1e9,
            "step_frac": balg / (mv / steps * 1e-3) / 1e9 / peak}


def main():
    global NX, NY
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-variants", action="store_true", help="skip the random-numbering, FP32 and BJ lines")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched leg")
    ap.add_argument("--no-served", action="store_true", help="skip the served leg")
    ap.add_argument("--batched-instances", type=int, default=512)
    ap.add_argument("--batched-steps", type=int, default=2000)
    ap.add_argument("--served-requests", type=int, default=100)
    ap.add_argument("--mesh", default=f"{NX}x{NY}", help="node grid NXxNY (profiling of smaller cases)")
    ap.add_argument("--kernel", choices=["tiled", "cell"], default="tiled",
                    help="step kernel family (the per-cell gather kernels are the other fusion split)")
    ap.add_argument("--precision", choices=["fp64", "fp32"], default="fp64",
                    help="precision of the headline solve (FP64 is the headline; FP32 for profiling its kernels)")
    ap.add_argument("--profile-only", action="store_true",
                    help="warm-up and timed steps only (no end-to-end, variants, CPU, batched or served legs): for ncu")
    ap.add_argument("--tour", action="store_true",
                    help="run every kernel of the library a few times (default mesh 1025x513) for a launch list")
    args = ap.parse_args()
    if args.tour:
        nx, ny = (int(x) for x in (args.mesh if args.mesh != f"{NX}x{NY}" else "1025x513").lower().split("x"))
        print(json.dumps(run_tour(nx, ny)), flush=True)
        return 0
    NX, NY = (int(x) for x in args.mesh.lower().split("x"))
    if args.profile_only:
        args.no_cpu = args.no_variants = args.no_batched = args.no_served = True
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference_arm(args)

    import cfd_optimisations_b200 as H
    rank, world, local, dist = dist_setup(args.gpus)
    H.set_device(local)
    mesh = make_mesh(H.NUMBER_RCM)
    bcmap, qbc, q = H.wedge_case(MACH)
    kernel = H.KERNEL_CELL if args.kernel == "cell" else H.KERNEL_TILED
    f32 = args.precision == "fp32"
    s = H.Solver(mesh, limiter=H.LIMITER_VENKAT, venkat_K=VENKAT_K, precision=H.FP32 if f32 else H.FP64,
                 kernel=kernel)
    s.gather_bcs(bcmap, qbc)
    s.initialise(q)
    ntri = s.Nreal
    Nc, Nf = s.Nc, s.Nf
    s.step(args.warmup, H.GLOBAL_CFL, CFL)
    # per-kernel events on every 4th step of the timed region (the events' own gaps stay out
    # of the other three)
    s.profile(True, every=4)
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

    # Roofline of the dominant kernel.  Algorithmic bytes (two-pass minimum, w = 8 in FP64,
    # 4 in FP32):
    #   pass 1: U (4w) + iv (w) + phiG (8w) per cell, (8 + 7w) per face
    #   pass 2: U (4w) + phiG (8w) + iv (w) + U' (4w) per cell, (8 + 7w) per face
    w = 4 if f32 else 8
    b1 = 13 * w * Nc + (8 + 7 * w) * Nf
    b2 = 17 * w * Nc + (8 + 7 * w) * Nf
    t1 = prof["ms_pass1"] / max(prof["n_pass1"], 1)
    t2 = prof["ms_pass2"] / max(prof["n_pass2"], 1)
    dom, b, t = ("pass2", b2, t2) if t2 >= t1 else ("pass1", b1, t1)
    peak, peak_kind = peaks()
    achieved = b / (t * 1e-3) / 1e9
    step_achieved = (b1 + b2) / (ms_max / args.steps * 1e-3) / 1e9
    traffic = traffic_from_profiles(dom, f"{args.precision}_rcm_{NX}x{NY}" + ("_cell" if args.kernel == "cell" else ""))

    line = {"metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32" if f32 else "f64",
            "data": "synthetic",
            "config": {"workload": workload(args.precision) + (", per-cell kernels" if args.kernel == "cell" else ""),
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

    single = rank == 0 and world == 1
    if not args.no_variants and rank == 0:
        k = min(args.steps, 200)
        var = {"fp64_random": timed_variant(H, make_mesh(H.NUMBER_RANDOM), ntri, Nc, Nf, peak, k, args.warmup,
                                            H.LIMITER_VENKAT, H.FP64, H.GLOBAL_CFL, CFL),
               "fp32_rcm": timed_variant(H, mesh, ntri, Nc, Nf, peak, k, args.warmup, H.LIMITER_VENKAT, H.FP32,
                                         H.GLOBAL_CFL, CFL),
               "fp64_bj_fixed_dt": timed_variant(H, mesh, ntri, Nc, Nf, peak, k, args.warmup,
                                                 H.LIMITER_BJ, H.FP64, H.FIXED_DT, reference_dt())}
        var["fp64_bj_fixed_dt"]["workload"] = reference_workload()
        line["variants"] = var

    if single and not args.no_cpu:
        r = cpu_reference(max(1, min(args.steps, 2)), 1)
        if r is not None:
            cv, threads, secs, sample = r
            line["cpu_baseline"] = {"value": cv, "unit": "cell-updates/s", "cores": threads, "kind": "reference",
                                    "sample": sample}
            if "variants" in line:
                g = line["variants"]["fp64_bj_fixed_dt"]["cell_updates_per_s"]
                line["same_config_as_reference"] = {
                    "workload": reference_workload(), "gpu_cell_updates_per_s": g, "cpu_cell_updates_per_s": cv,
                    "gpu_over_cpu": g / cv,
                    "note": "the reference arm's own configuration (Barth-Jespersen, fixed dt) on the GPU, "
                            "against the reference on the host cores in this run"}

    if single and not args.no_batched:
        from cfd_optimisations_b200 import batched
        t0 = time.perf_counter()
        b = batched.run(args.batched_instances, args.batched_steps, spread_every=4)
        b["wall_s"] = time.perf_counter() - t0
        line["batched"] = b

    if single and not args.no_served:
        from cfd_optimisations_b200 import serve
        t0 = time.perf_counter()
        sv = serve.run_prefix(args.served_requests)
        sv["wall_s"] = time.perf_counter() - t0
        per = sv.pop("per_request")
        sv["per_request"] = {k: [p[k] for p in per] for k in ("triangles", "latency_s", "fp32_vs_fp64",
                                                              "fp64_one_rounding_spread")}
        line["served"] = sv

    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------------------
# --tour: every kernel of the library a few times on one mid-sized case, so that one
# profiler run (a launch list of device times) covers all of them.  Single mesh: a
# 1025 x 513-node wedge (1,048,576 triangles, RCM numbering, Venkatakrishnan K = 5, M 2.5),
# the tiled FP64 and FP32 solvers and the per-cell FP64 and FP32 solvers, each through set-up
# (geometry, renumbering, face records), initialise and boundary cells, steps in global and
# local CFL mode, an asynchronous snapshot, download, upload, the wall pressure coefficient
# and a checkpoint / restore.  Arena: `instances` wedges of 10,000 to 60,000 triangles
# admitted to one FP32 arena (admission kernels), stepped, polled, fetched, checkpointed,
# restored and released.  Prints one JSON line with the cells touched and the steps taken.

def _tour_single(H, mesh, precision: int, kernel: int, steps: int, tmp: str) -> dict:
    bcmap, qbc, q = H.wedge_case(2.5)
    s = H.Solver(mesh, limiter=H.LIMITER_VENKAT, venkat_K=5.0, precision=precision, kernel=kernel)
    s.gather_bcs(bcmap, qbc)
    s.initialise(q)
    s.step(steps, H.GLOBAL_CFL, 0.5)
    s.step(steps, H.LOCAL_CFL, 0.5)
    out = np.empty((4, mesh.Nc), dtype=np.float64)
    s.snapshot(out, prims=True).wait()
    U = s.U()
    s.upload(U)
    s.wall_cp(2, q[0], q[3], float(np.hypot(q[1], q[2])))    # colour 2: the ramp
    path = os.path.join(tmp, "tour.ckpt")
    s.checkpoint(path)
    s.restore(path)
    s.step(1, H.GLOBAL_CFL, 0.5)
    H.device_sync()
    st = s.stats()
    del s
    return dict(cells=mesh.Nc, faces=mesh.Nf, steps=2 * steps + 1, residual_l2=st["res_l2"])


def _tour_arena(H, n: int, steps: int, tmp: str, seed: int = 7) -> dict:
    from cfd_optimisations_b200.arena import Arena
    rng = np.random.default_rng(seed)
    a = Arena(int(2e9), precision=H.FP32, limiter=H.LIMITER_BJ, max_instances=n + 8)
    slots, cells = [], 0
    for i in range(n):
        ntri = float(np.exp(rng.uniform(np.log(1e4), np.log(6e4))))
        ny1 = max(2, int(round(np.sqrt(ntri / 4.0))))
        m = H.Mesh.wedge(2 * ny1 + 1, ny1 + 1, theta_deg=float(rng.uniform(5.0, 15.0)), seed=100 + i,
                         numbering=H.NUMBER_RANDOM)
        bcmap, qbc, q = H.wedge_case(float(rng.uniform(1.8, 4.0)))
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
    H.device_sync()
    del a
    return dict(instances=n, cells=cells, steps=steps + 2)


def run_tour(nx: int = 1025, ny: int = 513, steps: int = 3, instances: int = 64) -> dict:
    import cfd_optimisations_b200 as H
    mesh = H.Mesh.wedge(nx, ny, theta_deg=15.0, seed=1234, numbering=H.NUMBER_RCM)
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, prec, kern in (("tiled_fp64", H.FP64, H.KERNEL_TILED), ("tiled_fp32", H.FP32, H.KERNEL_TILED),
                                 ("cell_fp64", H.FP64, H.KERNEL_CELL), ("cell_fp32", H.FP32, H.KERNEL_CELL)):
            out[name] = _tour_single(H, mesh, prec, kern, steps, tmp)
        out["arena_fp32"] = _tour_arena(H, instances, steps, tmp)
    return out


if __name__ == "__main__":
    sys.exit(main())
