"""Precision study: the FP32 path (float state, gradients, limiter and fluxes, compensated
per-cell residual sums, double geometry and residual norm) against the FP64 path on the
same mesh, both on the GPU, both run to convergence.

    python -m cfd_optimisations_b200.precision [--nx 1025 --ny 513 --mach 3.0 --theta 20
                                                 --cfl 0.8 --orders 8 --max-steps 50000]

Defaults are the 1025 x 513-node wedge (1,048,576 triangles), M 3.0, ramp 20 degrees, local
time stepping at CFL 0.8, Venkatakrishnan limiter K = 5, stop when the L2 density residual
has dropped `orders` orders below its first value or after `max-steps`.  Without limiter
freezing (--freeze N: steps after N reuse step N's limiter values) the residual of either
limiter stalls after one or two orders, the limiter switching back and forth.  Prints one
JSON object: for each precision the steps and device time to convergence, and the FP32 errors
against FP64 (relative L-inf and L2 of each conserved variable, and the L-inf and L2 error of
the wall pressure coefficient on the lower wall, the ramp).  A third run, FP64 from an initial
density one rounding step larger, gives the same errors for a perturbation the size of one
rounding: the floor that no precision can go below while the limiter keeps switching.
With --track N the three solves instead step side by side to --max-steps, their errors
against FP64 recorded every N steps, to show how long each stays within 1e-5.  With
--handoff --freeze N --track K the FP64 solve is handed over to the FP32 path at step N (its
checkpoint converted to FP32, so the FP32 solver freezes the FP64 limiter values) and both
that solve and an FP32 solve freezing its own values are tracked against FP64.
"""
from __future__ import annotations

import argparse
import json
import os
import tempfile
import time

import numpy as np

from . import (FP32, FP64, GLOBAL_CFL, LIMITER_BJ, LIMITER_VENKAT, LOCAL_CFL, NUMBER_RANDOM, Mesh, Solver,
               convert_checkpoint, wedge_case)
from .native import ENONFINITE, HcfdError

LOWER_WALL = 2   # colour of the lower wall (the ramp) in the generated wedge


def converge(mesh: Mesh, precision: int, mach: float, cfl: float, orders: float, max_steps: int,
             mode: int = LOCAL_CFL, limiter: int = LIMITER_VENKAT, K: float = 5.0, chunk: int = 200,
             freeze: int = 0, rho_scale: float = 1.0) -> dict:
    """Runs one solve to convergence; returns its state, wall Cp and timing.  `rho_scale`
    scales the initial density (1 + 2**-52: a perturbation the size of one rounding)."""
    bcmap, qbc, q = wedge_case(mach)
    s = Solver(mesh, limiter=limiter, venkat_K=K, precision=precision, freeze_limiter_after=freeze)
    s.gather_bcs(bcmap, qbc)
    qi = list(q)
    qi[0] *= rho_scale
    s.initialise(qi)
    steps, ms, hist = 0, 0.0, []
    st = s.step(1, mode, cfl)
    steps += 1
    res0 = st["res_first"]
    diverged = False
    while steps < max_steps:
        n = min(chunk, max_steps - steps)
        try:
            ms += s.step_timed(n, mode, cfl)
        except HcfdError as e:
            if e.code != ENONFINITE:
                raise
            diverged = True
        steps += n
        if diverged:
            st = dict(res_l2=None, nonfinite=True)
            break
        st = s.stats()
        hist.append((steps, st["res_l2"]))
        if st["res_l2"] <= res0 * 10.0 ** (-orders):
            break
    rho, p = q[0], q[3]
    speed = float(np.hypot(q[1], q[2]))
    U = cp = None
    if not diverged:
        U, cp = s.U(), s.wall_cp(LOWER_WALL, rho, p, speed)
    return dict(U=U, cp=cp, steps=steps, ms=ms, res0=res0, diverged=diverged,
                res=st["res_l2"], drop=float(np.log10(res0 / st["res_l2"])) if st["res_l2"] else None,
                history=hist)


def errors(a: dict, b: dict) -> dict:
    """Errors of solve `a` against reference solve `b`."""
    Ua, Ub = a["U"], b["U"]
    den = np.abs(Ub).max(axis=1)
    linf = (np.abs(Ua - Ub).max(axis=1) / den).tolist()
    l2 = (np.sqrt(((Ua - Ub) ** 2).mean(axis=1)) / np.sqrt((Ub ** 2).mean(axis=1))).tolist()
    dcp = a["cp"] - b["cp"]
    return dict(rel_linf=linf, rel_l2=l2, cp_linf=float(np.abs(dcp).max()),
                cp_l2=float(np.sqrt((dcp ** 2).mean())), cp_range=float(b["cp"].max() - b["cp"].min()))


def _rel_linf(Ua: np.ndarray, Ub: np.ndarray) -> float:
    return float((np.abs(Ua - Ub).max(axis=1) / np.abs(Ub).max(axis=1)).max())


def _rel_l2(Ua: np.ndarray, Ub: np.ndarray) -> float:
    return float((np.sqrt(((Ua - Ub) ** 2).mean(axis=1)) / np.sqrt((Ub ** 2).mean(axis=1))).max())


def _lockstep(runs: dict, others: tuple, done: int, steps: int, every: int, mode: int, cfl: float,
              bound: float) -> dict:
    """Steps every solve of `runs` side by side from step `done` to `steps`.  At the start and
    every `every` steps it records the relative L-inf and L2 errors (each the max over the
    conserved variables) of the solves named in `others` against runs["fp64"].  For each of
    those, `steps_within_bound` is the last recorded step up to which its L-inf error stayed
    within `bound` (None if it did not start within it).  A solve that produces a NaN or Inf
    ends the stepping; `diverged` names it and the step by which it did (the end of the
    interval it failed in)."""
    hist, within, still = [], {k: None for k in others}, {k: True for k in others}

    def record(step):
        U64 = runs["fp64"].U()
        row = dict(step=step, res_l2=runs["fp64"].stats()["res_l2"] if step else None)
        for k in others:
            Uk = runs[k].U()
            row[k] = _rel_linf(Uk, U64)
            row[k + "_l2"] = _rel_l2(Uk, U64)
            still[k] = still[k] and row[k] <= bound
            if still[k]:
                within[k] = step
        hist.append(row)

    record(done)
    diverged = None
    while done < steps:
        n = min(every, steps - done)
        for name, s in runs.items():
            try:
                s.step(n, mode, cfl)
            except HcfdError as e:
                if e.code != ENONFINITE:
                    raise
                diverged = dict(solve=name, by_step=done + n)
                break
        if diverged is not None:
            break
        done += n
        record(done)
    return dict(bound=bound, steps_within_bound=within, diverged=diverged, history=hist)


def _solver(mesh, precision, limiter, K, freeze, mach, rho_scale=1.0):
    bcmap, qbc, q = wedge_case(mach)
    s = Solver(mesh, limiter=limiter, venkat_K=K, precision=precision, freeze_limiter_after=freeze)
    s.gather_bcs(bcmap, qbc)
    qi = list(q)
    qi[0] *= rho_scale
    s.initialise(qi)
    return s


def track(mesh: Mesh, mach: float, cfl: float, steps: int, every: int, mode: int = LOCAL_CFL,
          limiter: int = LIMITER_VENKAT, K: float = 5.0, freeze: int = 0, bound: float = 1e-5) -> dict:
    """Steps the FP64 solve, the FP32 solve and the FP64 solve from an initial density one
    rounding step larger side by side from the start; the errors of the last two against the
    first are recorded as _lockstep records them."""
    runs = {name: _solver(mesh, prec, limiter, K, freeze, mach, scale)
            for name, prec, scale in (("fp64", FP64, 1.0), ("fp32", FP32, 1.0),
                                      ("fp64_perturbed", FP64, 1.0 + 2.0 ** -52))}
    return _lockstep(runs, ("fp32", "fp64_perturbed"), 0, steps, every, mode, cfl, bound)


def handoff(mesh: Mesh, mach: float, cfl: float, steps: int, every: int, freeze: int, mode: int = GLOBAL_CFL,
            limiter: int = LIMITER_BJ, K: float = 5.0, bound: float = 1e-5) -> dict:
    """An FP64 solve with the limiter frozen after step `freeze` is handed over to the FP32
    path at that step: its checkpoint, converted to FP32 (convert_checkpoint), is restored
    into an FP32 solver freezing after the same step, which therefore continues with the FP64
    solve's limiter values.  Beside it an FP32 solve that ran from the start freezes its own.
    From step `freeze` on, the three step side by side and the two FP32 solves' errors against
    FP64 are recorded as _lockstep records them."""
    fp64 = _solver(mesh, FP64, limiter, K, freeze, mach)
    own = _solver(mesh, FP32, limiter, K, freeze, mach)
    fp64.step(freeze, mode, cfl)
    own.step(freeze, mode, cfl)
    with tempfile.TemporaryDirectory() as tmp:
        p64, p32 = os.path.join(tmp, "fp64.ckpt"), os.path.join(tmp, "fp32.ckpt")
        fp64.checkpoint(p64)
        convert_checkpoint(p64, p32, FP32)
        handed = _solver(mesh, FP32, limiter, K, freeze, mach)
        handed.restore(p32)
    runs = {"fp64": fp64, "fp32_handoff": handed, "fp32_own_limiter": own}
    return _lockstep(runs, ("fp32_handoff", "fp32_own_limiter"), freeze, steps, every, mode, cfl, bound)


def study(nx=1025, ny=513, mach=3.0, theta=20.0, cfl=0.8, orders=8.0, max_steps=50000, seed=1234,
          mode=LOCAL_CFL, limiter=LIMITER_VENKAT, K=5.0, freeze=0) -> dict:
    mesh = Mesh.wedge(nx, ny, theta_deg=theta, seed=seed, numbering=NUMBER_RANDOM)
    out = dict(workload=dict(nx=nx, ny=ny, triangles=2 * (nx - 1) * (ny - 1), mach=mach, theta_deg=theta, cfl=cfl,
                             time_mode="local" if mode == LOCAL_CFL else "global", orders=orders,
                             max_steps=max_steps, limiter="venkatakrishnan" if limiter == LIMITER_VENKAT else "bj",
                             K=K, freeze_limiter_after=freeze))
    runs = {}
    for name, prec, scale in (("fp64", FP64, 1.0), ("fp32", FP32, 1.0), ("fp64_perturbed", FP64, 1.0 + 2.0 ** -52)):
        t0 = time.perf_counter()
        runs[name] = converge(mesh, prec, mach, cfl, orders, max_steps, mode=mode, limiter=limiter, K=K,
                              freeze=freeze, rho_scale=scale)
        r = runs[name]
        out[name] = dict(steps=r["steps"], device_ms=r["ms"], wall_s=time.perf_counter() - t0, diverged=r["diverged"],
                         residual_drop_orders=r["drop"], converged=bool(r["drop"] is not None and r["drop"] >= orders))
    ok = lambda k: runs[k]["U"] is not None
    out["fp32_vs_fp64"] = errors(runs["fp32"], runs["fp64"]) if ok("fp32") and ok("fp64") else None
    # the same FP64 solve from an initial density one rounding step larger: the spread that
    # rounding alone gives in this solve, whatever the precision
    out["fp64_perturbed_vs_fp64"] = (errors(runs["fp64_perturbed"], runs["fp64"])
                                     if ok("fp64_perturbed") and ok("fp64") else None)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=1025)
    ap.add_argument("--ny", type=int, default=513)
    ap.add_argument("--mach", type=float, default=3.0)
    ap.add_argument("--theta", type=float, default=20.0)
    ap.add_argument("--cfl", type=float, default=0.8)
    ap.add_argument("--orders", type=float, default=8.0)
    ap.add_argument("--max-steps", type=int, default=50000)
    ap.add_argument("--global-dt", action="store_true", help="global instead of local time stepping")
    ap.add_argument("--bj", action="store_true", help="Barth-Jespersen instead of Venkatakrishnan")
    ap.add_argument("--K", type=float, default=5.0)
    ap.add_argument("--freeze", type=int, default=0,
                    help="freeze the limiter after this many steps (0: never)")
    ap.add_argument("--track", type=int, default=0,
                    help="instead of the convergence runs: step all three solves to --max-steps and "
                         "record their errors every this many steps")
    ap.add_argument("--handoff", action="store_true",
                    help="with --freeze N and --track K: hand the FP64 solve over to FP32 at step N "
                         "(FP64 limiter values) and track both FP32 solves against FP64")
    a = ap.parse_args()
    mode = GLOBAL_CFL if a.global_dt else LOCAL_CFL
    limiter = LIMITER_BJ if a.bj else LIMITER_VENKAT
    if a.handoff:
        if a.freeze <= 0 or a.track <= 0:
            ap.error("--handoff needs --freeze N and --track K")
        mesh = Mesh.wedge(a.nx, a.ny, theta_deg=a.theta, seed=1234, numbering=NUMBER_RANDOM)
        out = handoff(mesh, a.mach, a.cfl, a.max_steps, a.track, a.freeze, mode=mode, limiter=limiter, K=a.K)
        out["workload"] = dict(nx=a.nx, ny=a.ny, mach=a.mach, theta_deg=a.theta, cfl=a.cfl,
                               time_mode="local" if mode == LOCAL_CFL else "global",
                               limiter="bj" if a.bj else "venkatakrishnan", K=a.K, steps=a.max_steps,
                               handoff_at=a.freeze)
        print(json.dumps(out))
        return
    if a.track:
        mesh = Mesh.wedge(a.nx, a.ny, theta_deg=a.theta, seed=1234, numbering=NUMBER_RANDOM)
        out = track(mesh, a.mach, a.cfl, a.max_steps, a.track, mode=mode, limiter=limiter, K=a.K, freeze=a.freeze)
        out["workload"] = dict(nx=a.nx, ny=a.ny, mach=a.mach, theta_deg=a.theta, cfl=a.cfl,
                               time_mode="local" if mode == LOCAL_CFL else "global",
                               limiter="bj" if a.bj else "venkatakrishnan", K=a.K, steps=a.max_steps,
                               freeze_limiter_after=a.freeze)
        print(json.dumps(out))
        return
    print(json.dumps(study(a.nx, a.ny, a.mach, a.theta, a.cfl, a.orders, a.max_steps,
                           mode=mode, limiter=limiter, K=a.K, freeze=a.freeze)))


if __name__ == "__main__":
    main()
