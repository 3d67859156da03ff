"""Serving loop: wedge-solve requests admitted into one resident arena as they arrive
(continuous batching), against the plain one-mesh-at-a-time FP64 GPU loop on the same stream.

    python -m cfd_optimisations_b200.serve [--requests 10000 --rate 100 --seed 7 --budget-gb 160
                                            --orders 6 --max-steps 20000 --chunk 100
                                            --baseline-sample 24]

Requests arrive as a Poisson process (`rate` per second).  Each carries a wedge: triangle count
lognormal (median 50,000, sigma 1.0) clipped to [5,000, 2,000,000] on a 2:1 node grid, Mach
number ~ U[1.8, 4.0], ramp angle ~ U[5, 15] degrees, its own jitter/permutation seed.  A
request is done when its L2 density residual has dropped `orders` orders below its first value
or after `max-steps` steps (or when a step produced a NaN/Inf, reported as failed).

The server: worker threads build each arrived request's mesh and prepare its admission (tile
plan, BC table: hcfd_arena_prepare) while the server thread steps the arena.  Between chunks of
`chunk` steps the server polls every instance's residual, retires the finished ones (state
copied to the host, ranges freed) and admits prepared requests, oldest first, as long as the
HBM budget has room: the batch is never drained.  Admissions and checks happen only between
chunks, so an instance is checked after the same numbers of its own steps alone and in any
mix, and its arithmetic does not depend on its neighbours: its result is the same alone and in
the mix.  Latency is result time minus arrival time, mesh construction included.

The baseline runs each request alone through the plain FP64 solver (Solver, one mesh at a
time, the same stopping rule checked every `chunk` steps).  Timing it over the whole stream
would take hours; it is run on `baseline-sample` requests (every k-th request in arrival
order) and the stream's sequential service time is estimated from them per cell-step, stated
in the output (the headline ratio).  One rate per cell-step is exact when a step's cost is
proportional to its cells; with a fixed cost per step as well, it is right only when the
sample's cell-step-weighted mean size matches the stream's.  A second estimate therefore fits
a step cost a + b * triangles to the sample and applies it request by request.  A third adds
each request's own overhead (mesh construction, solver set-up, download: wall time less
device time on the sample, fitted as c + d * triangles), so that the sequential loop is
charged what the served latencies include.  The same sample gives the served results' errors
against FP64.  `run_prefix` (the bench's served leg) runs the sequential loop for real on
every request of a stream prefix instead.
"""
from __future__ import annotations

import argparse
import json
import math
import time
from collections import deque
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from . import FP32, FP64, GLOBAL_CFL, LIMITER_BJ, NUMBER_RANDOM, Mesh, Solver, device_mem_info, wedge_case
from .native import ENONFINITE, HcfdError


@dataclass
class Request:
    rid: int
    t_arrive: float
    nx: int
    ny: int
    mach: float
    theta: float
    seed: int

    @property
    def triangles(self) -> int:
        return 2 * (self.nx - 1) * (self.ny - 1)


@dataclass
class Result:
    rid: int
    t_arrive: float
    t_admit: float
    t_done: float
    steps: int
    drop: float
    converged: bool
    failed: bool
    triangles: int
    U: np.ndarray | None = field(default=None, repr=False)

    @property
    def latency(self) -> float:
        return self.t_done - self.t_arrive


def request_stream(n: int = 10000, rate: float = 100.0, seed: int = 7, median: float = 5e4, sigma: float = 1.0,
                   lo: float = 5e3, hi: float = 2e6) -> list[Request]:
    """The seeded request stream (arrival times in seconds from the start)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    ntri = np.clip(np.exp(math.log(median) + sigma * rng.standard_normal(n)), lo, hi)
    mach = rng.uniform(1.8, 4.0, n)
    theta = rng.uniform(5.0, 15.0, n)
    out = []
    for i in range(n):
        ny1 = max(2, int(round(math.sqrt(ntri[i] / 4.0))))
        out.append(Request(i, float(t[i]), 2 * ny1 + 1, ny1 + 1, float(mach[i]), float(theta[i]), 1234 + i))
    return out


def build_mesh(r: Request) -> Mesh:
    return Mesh.wedge(r.nx, r.ny, theta_deg=r.theta, seed=r.seed, numbering=NUMBER_RANDOM)


def done_reason(st: dict, orders: float, max_steps: int) -> str | None:
    """Why an instance with these statistics is finished, or None."""
    if st["nonfinite"]:
        return "failed"
    if st["res_first"] > 0 and st["res_l2"] <= st["res_first"] * 10.0 ** (-orders):
        return "converged"
    if st["steps"] >= max_steps:
        return "cap"
    return None


def drop_of(st: dict) -> float:
    return float(math.log10(st["res_first"] / st["res_l2"])) if st["res_l2"] > 0 and st["res_first"] > 0 else 0.0


class Server:
    """Continuous batching of requests into one arena.

    `arena` is an Arena (or any object with prepare/admit_prepared/step/poll/fetch/release);
    `mesh_for` builds a request's mesh.  Both are parameters so that the scheduling can be
    exercised without a GPU."""

    def __init__(self, arena, cfl: float = 0.5, orders: float = 6.0, max_steps: int = 20000, chunk: int = 100,
                 workers: int = 8, lookahead: int = 64, keep=None, mesh_for=build_mesh, clock=time.perf_counter):
        if max_steps % chunk:
            raise ValueError("max_steps must be a multiple of chunk")
        self.arena = arena
        self.cfl, self.orders, self.max_steps, self.chunk = cfl, orders, max_steps, chunk
        self.workers, self.lookahead = workers, lookahead
        self.keep = keep if keep is not None else (lambda rid: False)
        self.mesh_for = mesh_for
        self.clock = clock
        self.busy_s = 0.0          # wall time with at least one instance on the device
        self.max_active = 0
        self.max_cells = 0

    def _prepare(self, r: Request):
        bcmap, qbc, q = wedge_case(r.mach)
        return self.arena.prepare(self.mesh_for(r), bcmap, qbc, q, self.cfl)

    def run(self, reqs: list[Request]) -> list[Result]:
        reqs = sorted(reqs, key=lambda r: r.t_arrive)
        t0 = self.clock()
        now = lambda: self.clock() - t0
        pool = ThreadPoolExecutor(max_workers=self.workers)
        pending = deque()        # (request, future) in arrival order, not yet admitted
        active = {}              # slot -> (request, t_admit, cells)
        results = []
        nxt = 0
        cells = 0
        try:
            while len(results) < len(reqs):
                t = now()
                # hand arrived requests to the workers, at most `lookahead` waiting
                while nxt < len(reqs) and reqs[nxt].t_arrive <= t and len(pending) < self.lookahead:
                    pending.append((reqs[nxt], pool.submit(self._prepare, reqs[nxt])))
                    nxt += 1
                # admit prepared requests, oldest first, while the budget has room
                blocked = False
                for item in list(pending):
                    r, fut = item
                    if not fut.done():
                        continue
                    adm = fut.result()
                    slot = self.arena.admit_prepared(adm)
                    if slot is None:
                        blocked = True
                        break
                    pending.remove(item)
                    active[slot] = (r, now(), adm.cells)
                    cells += adm.cells
                    del adm
                self.max_active = max(self.max_active, len(active))
                self.max_cells = max(self.max_cells, cells)
                if not active:
                    if blocked:
                        raise RuntimeError("serve: a request does not fit in an empty arena")
                    # idle: wait for the next arrival or preparation
                    waits = [reqs[nxt].t_arrive - now()] if nxt < len(reqs) and len(pending) < self.lookahead else []
                    time.sleep(min([0.002] + [w for w in waits if w > 0]))
                    continue
                tb = now()
                self.arena.step(self.chunk)
                stats = self.arena.poll()
                self.busy_s += now() - tb
                for slot, st in stats.items():
                    why = done_reason(st, self.orders, self.max_steps)
                    if why is None:
                        continue
                    r, t_adm, c = active.pop(slot)
                    U = self.arena.fetch(slot) if self.keep(r.rid) else None
                    self.arena.release(slot)
                    cells -= c
                    results.append(Result(r.rid, r.t_arrive, t_adm, now(), int(st["steps"]), drop_of(st),
                                          why == "converged", why == "failed", r.triangles, U))
        finally:
            pool.shutdown(wait=True, cancel_futures=True)
        return sorted(results, key=lambda x: x.rid)


def partition(reqs: list[Request], ndev: int) -> list[list[Request]]:
    """Replicas over several GPUs: each request, in arrival order, goes to the device with the
    fewest triangles assigned so far (its arena's memory and work grow with them)."""
    loads = [0] * ndev
    parts = [[] for _ in range(ndev)]
    for r in sorted(reqs, key=lambda r: r.t_arrive):
        d = min(range(ndev), key=lambda i: (loads[i], i))
        parts[d].append(r)
        loads[d] += r.triangles
    return parts


def serve_devices(reqs: list[Request], make_server, devices) -> tuple[list[Result], list[list[Request]]]:
    """One Server with its own arena per device, each in its own thread (the thread's current
    device is the one it serves); no data crosses devices.  `make_server(device)` builds the
    server in that thread.  Returns all results by request id and the partition."""
    import threading
    parts = partition(reqs, len(devices))
    out = [None] * len(devices)
    errors = []

    def work(i, dev):
        try:
            out[i] = make_server(dev).run(parts[i]) if parts[i] else []
        except BaseException as e:          # reported after all threads end
            errors.append(e)

    threads = [threading.Thread(target=work, args=(i, d)) for i, d in enumerate(devices)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if errors:
        raise errors[0]
    return sorted((r for part in out for r in part), key=lambda r: r.rid), parts


def solve_alone_fp64(r: Request, cfl: float, orders: float, max_steps: int, chunk: int, rho_scale: float = 1.0,
                     **kw):
    """One request through the plain FP64 solver; returns (device ms, Result-like dict, U).
    `rho_scale` scales the initial density (a rounding-sized perturbation with 1 + 2**-52)."""
    bcmap, qbc, q = wedge_case(r.mach)
    s = Solver(build_mesh(r), precision=FP64, limiter=LIMITER_BJ, **kw)
    s.gather_bcs(bcmap, qbc)
    qi = list(q)
    qi[0] *= rho_scale
    s.initialise(qi)
    ms, steps = 0.0, 0
    while True:
        try:
            ms += s.step_timed(chunk, GLOBAL_CFL, cfl)
            st = s.stats()
        except HcfdError as e:
            if e.code != ENONFINITE:
                raise
            st = dict(res_l2=0.0, res_first=0.0, nonfinite=True)
        steps += chunk
        st["steps"] = steps
        why = done_reason(st, orders, max_steps)
        if why is not None:
            return ms, dict(steps=steps, drop=drop_of(st), why=why), s.U()


def sequential_service(reqs, steps_by_rid: dict, s_per_step, overhead=None) -> tuple[float, list[float]]:
    """Makespan and latencies of serving `reqs` one at a time in arrival order, request r
    taking steps_by_rid[r.rid] steps of s_per_step(r.triangles) seconds each, plus
    overhead(r.triangles) seconds when given."""
    t_free, lat = 0.0, []
    for r in reqs:
        t = steps_by_rid[r.rid] * s_per_step(r.triangles) + (overhead(r.triangles) if overhead else 0.0)
        t_free = max(t_free, r.t_arrive) + t
        lat.append(t_free - r.t_arrive)
    return t_free, lat


def affine_step_model(triangles, s_per_step) -> tuple[float, float]:
    """Least-squares fit s_per_step = a + b * triangles over the sampled requests: a step's
    fixed cost (launches, small meshes) and its cost per cell (large meshes).  a is clamped
    at 0."""
    x = np.asarray(triangles, dtype=float)
    y = np.asarray(s_per_step, dtype=float)
    A = np.column_stack([np.ones_like(x), x])
    (a, b), *_ = np.linalg.lstsq(A, y, rcond=None)
    if a < 0:
        a, b = 0.0, float((x * y).sum() / (x * x).sum())
    return float(a), float(b)


def percentiles(x) -> dict:
    x = np.asarray(x, dtype=float)
    return dict(p50=float(np.percentile(x, 50)), p99=float(np.percentile(x, 99)), mean=float(x.mean()))


def arena_budget(budget_gb: float) -> int:
    """The HBM budget: `budget_gb` GB, capped at the device's free memory less 4 GB."""
    free, _ = device_mem_info()
    return int(min(budget_gb * 1e9, free - 4e9))


def run_prefix(n: int = 100, rate: float = 100.0, seed: int = 7, orders: float = 6.0, max_steps: int = 20000,
               chunk: int = 100, cfl: float = 0.5, budget_gb: float = 160.0, spread_every: int = 4,
               workers: int = 8) -> dict:
    """The first `n` requests of the seeded stream, served, against the plain sequential FP64
    GPU loop run on every one of the same requests (nothing extrapolated).

    Served: continuous batching into one FP32 arena (Server); host clock from the first
    arrival, mesh construction, admission and result download included.  Sequential: each
    request alone through the plain FP64 solver in arrival order, started once it has arrived
    and the previous one is done, measured the same way (mesh, set-up, steps, download); the
    same loop charged only the device time of its steps is reported beside it
    (`device_only`).  Every request's FP32 result is compared with its FP64 result; every
    `spread_every`-th request is also solved in FP64 from an initial density one rounding step
    larger, the spread rounding alone produces in that solve."""
    from . import autotune
    from .arena import Arena
    from .batched import accuracy_summary, rel_linf_max
    reqs = request_stream(10000, rate, seed)[:n]
    budget = arena_budget(budget_gb)
    med = int(np.median([r.triangles for r in reqs]))
    tile = autotune.best_arena_tile(med, FP32, LIMITER_BJ)
    arena = Arena(budget, precision=FP32, limiter=LIMITER_BJ, time_mode=GLOBAL_CFL, tile=tile,
                  max_instances=max(64, 2 * n))
    srv = Server(arena, cfl, orders, max_steps, chunk, workers=workers, keep=lambda rid: True)
    res = srv.run(reqs)
    span = max(r.t_done for r in res)
    del srv.arena, arena
    # the sequential loop, run for real on the same arrivals: each request, once it has arrived
    # and the previous one is done, builds its mesh, creates its solver, steps and downloads its
    # result; host clock, as the served latencies are
    dev_s, U64, info64, t_end = {}, {}, {}, {}
    t0 = time.perf_counter()
    for r in reqs:
        wait = r.t_arrive - (time.perf_counter() - t0)
        if wait > 0:
            time.sleep(wait)
        ms, info, U = solve_alone_fp64(r, cfl, orders, max_steps, chunk)
        t_end[r.rid] = time.perf_counter() - t0
        dev_s[r.rid], U64[r.rid], info64[r.rid] = ms / 1e3, U, info
    wall = max(t_end.values())
    lat_wall = [t_end[r.rid] - r.t_arrive for r in reqs]
    # the same loop charged only the device time of its steps (no mesh construction, set-up or
    # download): the ratio against it is the conservative one
    t_free, lat_seq = 0.0, []
    for r in reqs:
        t_free = max(t_free, r.t_arrive) + dev_s[r.rid]
        lat_seq.append(t_free - r.t_arrive)
    by = {x.rid: x for x in res}
    e32 = {r.rid: rel_linf_max(by[r.rid].U, U64[r.rid]) for r in reqs}
    sub = [r for i, r in enumerate(reqs) if i % max(1, spread_every) == 0]
    e64 = {}
    for r in sub:
        _, _, Up = solve_alone_fp64(r, cfl, orders, max_steps, chunk, rho_scale=1.0 + 2.0 ** -52)
        e64[r.rid] = rel_linf_max(Up, U64[r.rid])
    served = dict(precision="fp32-compensated", tile=tile, budget_bytes=budget, makespan_s=span,
                  solves_per_s=n / span, latency_s=percentiles([x.latency for x in res]),
                  queue_s=percentiles([x.t_admit - x.t_arrive for x in res]),
                  converged=sum(x.converged for x in res), failed=sum(x.failed for x in res),
                  steps=percentiles([x.steps for x in res]), device_busy_fraction=srv.busy_s / span,
                  max_active=srv.max_active)
    seq = dict(precision="fp64", makespan_s=wall, solves_per_s=n / wall, latency_s=percentiles(lat_wall),
               converged=sum(i["why"] == "converged" for i in info64.values()),
               steps=percentiles([i["steps"] for i in info64.values()]),
               how="every request alone through the plain FP64 solver in arrival order, each started once it "
                   "has arrived and the previous one is done: mesh, solver set-up, steps (stopping rule checked "
                   "every chunk), download; host clock, like the served latencies",
               device_only=dict(makespan_s=t_free, solves_per_s=n / t_free, latency_s=percentiles(lat_seq),
                                device_s=sum(dev_s.values()),
                                how="the same requests charged only the device time of their steps"))
    return dict(workload=dict(requests=n, of_stream=10000, rate_per_s=rate, seed=seed,
                              triangles="lognormal median 5e4 sigma 1.0 clipped [5e3, 2e6]",
                              triangles_total=int(sum(r.triangles for r in reqs)), mach="U[1.8,4.0]",
                              theta_deg="U[5,15]", stop=f"{orders} orders or {max_steps} steps", chunk=chunk,
                              limiter="barth-jespersen", cfl=cfl),
                served=served, fp64_sequential=seq, speedup_solves_per_s=served["solves_per_s"] / seq["solves_per_s"],
                speedup_solves_per_s_vs_device_only=served["solves_per_s"] / seq["device_only"]["solves_per_s"],
                accuracy=accuracy_summary([e32[r.rid] for r in sub], [e64[r.rid] for r in sub]),
                fp32_vs_fp64_rel_linf=dict(n=n, median=float(np.median(list(e32.values()))),
                                           max=float(max(e32.values()))),
                per_request=[dict(rid=r.rid, triangles=r.triangles, latency_s=by[r.rid].latency,
                                  steps=by[r.rid].steps, fp32_vs_fp64=e32[r.rid],
                                  fp64_one_rounding_spread=e64.get(r.rid)) for r in reqs])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--requests", type=int, default=10000)
    ap.add_argument("--rate", type=float, default=100.0)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--budget-gb", type=float, default=160.0)
    ap.add_argument("--orders", type=float, default=6.0)
    ap.add_argument("--max-steps", type=int, default=20000)
    ap.add_argument("--chunk", type=int, default=100)
    ap.add_argument("--cfl", type=float, default=0.5)
    ap.add_argument("--tile", type=int, default=0, help="arena tile size (0: autotuned for the median request)")
    ap.add_argument("--workers", type=int, default=8)
    ap.add_argument("--baseline-sample", type=int, default=24)
    ap.add_argument("--devices", type=int, default=1, help="GPUs, one arena each (replicas, no collective)")
    ap.add_argument("--max-instances", type=int, default=65536,
                    help="resident instance slots (admission is by the HBM budget below this cap)")
    a = ap.parse_args()

    from . import autotune
    from .arena import Arena

    reqs = request_stream(a.requests, a.rate, a.seed)
    budget = arena_budget(a.budget_gb)
    med = int(np.median([r.triangles for r in reqs]))
    tile = a.tile or autotune.best_arena_tile(med, FP32, LIMITER_BJ)
    k = max(1, len(reqs) // max(1, a.baseline_sample))
    sample = set(r.rid for r in reqs[::k][:a.baseline_sample])
    servers = []

    def make_server(dev):
        from . import set_device
        set_device(dev)
        arena = Arena(budget, precision=FP32, limiter=LIMITER_BJ, time_mode=GLOBAL_CFL, tile=tile,
                      max_instances=a.max_instances)
        srv = Server(arena, a.cfl, a.orders, a.max_steps, a.chunk, workers=a.workers, keep=lambda rid: rid in sample)
        servers.append(srv)
        return srv

    t0 = time.perf_counter()
    res, _ = serve_devices(reqs, make_server, list(range(a.devices)))
    wall = time.perf_counter() - t0
    busy = sum(srv.busy_s for srv in servers) / len(servers)
    span = max(r.t_done for r in res)
    lat = [r.latency for r in res]
    cell_steps = sum(r.triangles * r.steps for r in res)
    out = dict(
        workload=dict(requests=a.requests, rate_per_s=a.rate, seed=a.seed, triangles="lognormal median 5e4 sigma 1.0 "
                      "clipped [5e3, 2e6]", mach="U[1.8,4.0]", theta_deg="U[5,15]", stop=f"{a.orders} orders or "
                      f"{a.max_steps} steps", chunk=a.chunk, limiter="barth-jespersen", cfl=a.cfl,
                      time_mode="global per instance"),
        served=dict(precision="fp32-compensated", tile=tile, budget_bytes=budget, max_instances=a.max_instances, wall_s=wall, makespan_s=span,
                    solves_per_s=len(res) / span, latency_s=percentiles(lat),
                    queue_s=percentiles([r.t_admit - r.t_arrive for r in res]),
                    converged=sum(r.converged for r in res), failed=sum(r.failed for r in res),
                    steps=percentiles([r.steps for r in res]), cell_updates_per_s=cell_steps / span,
                    devices=a.devices, device_busy_fraction=busy / span,
                    max_active=max(srv.max_active for srv in servers), max_cells=max(srv.max_cells for srv in servers)))
    for srv in servers:
        del srv.arena
    servers.clear()
    # baseline on the sample
    base, errs, errs64 = [], [], []
    for r in reqs:
        if r.rid not in sample:
            continue
        tw = time.perf_counter()
        ms, info, U64 = solve_alone_fp64(r, a.cfl, a.orders, a.max_steps, a.chunk)
        info["wall_s"] = time.perf_counter() - tw      # mesh, set-up, steps and download
        base.append((r, ms / 1e3, info))
        served = next(x for x in res if x.rid == r.rid)
        den = np.abs(U64).max(axis=1)
        errs.append(dict(rid=r.rid, triangles=r.triangles, steps_fp32=served.steps, steps_fp64=info["steps"],
                         rel_linf=float((np.abs(served.U - U64).max(axis=1) / den).max())))
        # the same FP64 solve from an initial density one rounding step larger: the spread
        # that rounding alone produces in this solve, whatever the precision
        _, info2, U64b = solve_alone_fp64(r, a.cfl, a.orders, a.max_steps, a.chunk, rho_scale=1.0 + 2.0 ** -52)
        errs64.append(float((np.abs(U64b - U64).max(axis=1) / den).max()))
    per_cell_step = sum(s for _, s, _ in base) / sum(r.triangles * i["steps"] for r, _, i in base)
    # sequential service of the whole stream, each request's time estimated from its cell-steps
    # (steps per request as served); the headline ratio
    steps_by_rid = {x.rid: x.steps for x in res}
    t_free, lat_b = sequential_service(reqs, steps_by_rid, lambda tri: per_cell_step * tri)
    out["fp64_sequential"] = dict(sample=len(base), sample_device_s=sum(s for _, s, _ in base),
                                  s_per_cell_step=per_cell_step, estimated_makespan_s=t_free,
                                  solves_per_s=len(reqs) / t_free, latency_s=percentiles(lat_b),
                                  note="device time of the sampled requests, extrapolated per cell-step to the "
                                       "stream (steps per request as served)")
    out["speedup_solves_per_s"] = out["served"]["solves_per_s"] / out["fp64_sequential"]["solves_per_s"]
    # the same with a step cost a + b * triangles fitted to the sample: the fixed cost per step
    # charged request by request, whatever the sample's mean size
    a0, b0 = affine_step_model([r.triangles for r, _, _ in base], [s / i["steps"] for r, s, i in base])
    t_aff, lat_aff = sequential_service(reqs, steps_by_rid, lambda tri: a0 + b0 * tri)
    out["fp64_sequential_affine"] = dict(s_per_step_fixed=a0, s_per_cell_step=b0, estimated_makespan_s=t_aff,
                                         solves_per_s=len(reqs) / t_aff, latency_s=percentiles(lat_aff))
    out["speedup_solves_per_s_affine"] = out["served"]["solves_per_s"] / out["fp64_sequential_affine"]["solves_per_s"]
    # end to end, as the served latencies are measured: each sampled request's wall time (mesh,
    # solver set-up, steps, download) as device time plus a per-request overhead, the overhead
    # fitted as c + d * triangles on the sample and charged request by request with the affine
    # step cost above
    oh = [max(0.0, i["wall_s"] - s) for _, s, i in base]
    c0, d0 = affine_step_model([r.triangles for r, _, _ in base], oh)
    t_e2e, lat_e2e = sequential_service(reqs, steps_by_rid, lambda tri: a0 + b0 * tri,
                                        overhead=lambda tri: c0 + d0 * tri)
    out["fp64_sequential_end_to_end"] = dict(overhead_s_fixed=c0, overhead_s_per_triangle=d0,
                                             sample_wall_s=sum(i["wall_s"] for _, _, i in base),
                                             estimated_makespan_s=t_e2e, solves_per_s=len(reqs) / t_e2e,
                                             latency_s=percentiles(lat_e2e))
    out["speedup_solves_per_s_end_to_end"] = out["served"]["solves_per_s"] / out["fp64_sequential_end_to_end"]["solves_per_s"]
    e32 = [e["rel_linf"] for e in errs]
    out["fp32_vs_fp64_rel_linf"] = dict(n=len(e32), max=max(e32), median=float(np.median(e32)), per_request=errs)
    out["fp64_vs_fp64_initial_density_plus_one_ulp_rel_linf"] = dict(n=len(errs64), max=max(errs64),
                                                                    median=float(np.median(errs64)))
    print(json.dumps(out))


if __name__ == "__main__":
    main()
