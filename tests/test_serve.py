"""Serving loop scheduling without a GPU: a fake arena stands in for the device (its
residual falls at a per-request rate), so admission by budget, oldest-first order, backfill
on retirement, the stopping rules and the latency bookkeeping are checked on the CPU."""
import math

import numpy as np
import pytest

from cfd_optimisations_b200 import serve


class FakeAdmission:
    def __init__(self, r):
        self.r = r
        self.cells = 128 * math.ceil(r.triangles / 128)


class FakeArena:
    """prepare/admit_prepared/step/poll/fetch/release with a cell budget; instance k's
    residual after n steps is 10**(-n * rate_k)."""

    def __init__(self, capacity, rates, nonfinite=()):
        self.capacity, self.used = capacity, 0
        self.rates, self.nonfinite = rates, set(nonfinite)
        self.inst = {}
        self.admitted = []
        self.max_used = 0

    def prepare(self, mesh, bcmap, qbc, qic, cfl):
        assert mesh.rid >= 0 and cfl > 0
        return FakeAdmission(mesh)

    def admit_prepared(self, adm):
        if self.used + adm.cells > self.capacity:
            return None
        slot = next(k for k in range(10 ** 6) if k not in self.inst)
        self.inst[slot] = dict(r=adm.r, steps=0, cells=adm.cells)
        self.used += adm.cells
        self.max_used = max(self.max_used, self.used)
        self.admitted.append(adm.r.rid)
        return slot

    def step(self, n):
        for I in self.inst.values():
            I["steps"] += n

    def poll(self):
        out = {}
        for k, I in self.inst.items():
            rid = I["r"].rid
            res = 10.0 ** (-I["steps"] * self.rates[rid])
            out[k] = dict(dt=1e-3, res_l2=res, res_first=1.0, steps=I["steps"],
                          nonfinite=rid in self.nonfinite and I["steps"] >= 200)
        return out

    def fetch(self, slot):
        return np.full((4, 3), float(self.inst[slot]["r"].rid))

    def release(self, slot):
        self.used -= self.inst.pop(slot)["cells"]


def small_stream(n=40, rate=2000.0, seed=3):
    reqs = serve.request_stream(n, rate, seed, median=2e3, sigma=0.8, lo=500, hi=2e4)
    return reqs


def test_request_stream_is_seeded_and_clipped():
    a = serve.request_stream(500, 100.0, 11)
    b = serve.request_stream(500, 100.0, 11)
    assert [(r.t_arrive, r.nx, r.mach) for r in a] == [(r.t_arrive, r.nx, r.mach) for r in b]
    tri = np.array([r.triangles for r in a])
    assert tri.min() >= 0.8 * 5e3 and tri.max() <= 1.2 * 2e6
    assert 3e4 < np.median(tri) < 8e4
    t = np.array([r.t_arrive for r in a])
    assert np.all(np.diff(t) > 0) and 3.5 < t[-1] < 6.5          # 500 arrivals at 100/s
    assert all(1.8 <= r.mach <= 4.0 and 5.0 <= r.theta <= 15.0 for r in a)
    assert all(r.nx == 2 * (r.ny - 1) + 1 for r in a)             # 2:1 node grid


def test_done_reason():
    st = dict(res_l2=1e-7, res_first=1.0, steps=100, nonfinite=False)
    assert serve.done_reason(st, 6.0, 1000) == "converged"
    assert serve.done_reason(dict(st, res_l2=1e-3), 6.0, 1000) is None
    assert serve.done_reason(dict(st, res_l2=1e-3, steps=1000), 6.0, 1000) == "cap"
    assert serve.done_reason(dict(st, nonfinite=True), 6.0, 1000) == "failed"


def run_fake(reqs, capacity, rates, nonfinite=(), chunk=50, max_steps=1000, workers=4):
    arena = FakeArena(capacity, rates, nonfinite)
    srv = serve.Server(arena, orders=6.0, max_steps=max_steps, chunk=chunk, workers=workers, lookahead=16,
                       keep=lambda rid: True, mesh_for=lambda r: r)
    return arena, srv, srv.run(reqs)


def test_server_budget_backfill_and_stopping_rules():
    reqs = small_stream()
    rng = np.random.default_rng(5)
    rates = {r.rid: float(rng.choice([0.0, 0.01, 0.02, 0.05])) for r in reqs}
    rates[reqs[3].rid] = 0.0
    cap = 6 * max(FakeAdmission(r).cells for r in reqs)
    arena, srv, res = run_fake(reqs, cap, rates, nonfinite={reqs[3].rid})
    assert [x.rid for x in res] == sorted(r.rid for r in reqs)
    assert arena.max_used <= cap
    assert srv.max_active >= 2                                      # batched
    assert len(arena.admitted) == len(reqs)
    for x in res:
        rate = rates[x.rid]
        if x.rid == reqs[3].rid:
            assert x.failed and x.steps == 200
            continue
        # first chunk boundary at which 10**(-rate*n) <= 1e-6, else the cap
        want = min((math.ceil(6.0 / rate / 50) * 50) if rate > 0 else 10 ** 9, 1000)
        assert x.steps == want, (x.rid, rate)
        assert x.converged == (rate > 0 and want < 1000 or rate * 1000 >= 6.0)
        assert x.t_arrive <= x.t_admit <= x.t_done
        assert np.all(x.U == x.rid)


def test_server_admits_oldest_first_when_full():
    reqs = small_stream(24)
    rates = {r.rid: 0.0 for r in reqs}
    biggest = max(FakeAdmission(r).cells for r in reqs)
    # one worker prepares in arrival order; the arena holds the largest request alone
    arena, srv, res = run_fake(reqs, biggest, rates, max_steps=100, workers=1)
    assert arena.admitted == [r.rid for r in sorted(reqs, key=lambda r: r.t_arrive)]
    assert arena.max_used <= biggest
    assert all(x.steps == 100 for x in res)


def test_server_rejects_request_larger_than_arena():
    reqs = small_stream(3)
    with pytest.raises(RuntimeError, match="does not fit"):
        run_fake(reqs, 64, {r.rid: 0.0 for r in reqs})


def test_max_steps_multiple_of_chunk():
    with pytest.raises(ValueError):
        serve.Server(FakeArena(1, {}), max_steps=1000, chunk=300)


def test_partition_balances_triangles():
    reqs = serve.request_stream(200, 100.0, 4)
    parts = serve.partition(reqs, 3)
    assert sorted(r.rid for p in parts for r in p) == list(range(200))
    loads = [sum(r.triangles for r in p) for p in parts]
    assert max(loads) - min(loads) <= max(r.triangles for r in reqs)
    assert serve.partition(reqs, 1)[0] == sorted(reqs, key=lambda r: r.t_arrive)


def test_serve_devices_runs_one_server_per_device():
    reqs = small_stream(30)
    rates = {r.rid: 0.02 for r in reqs}
    made = []

    def make_server(dev):
        arena = FakeArena(10 ** 9, rates)
        made.append((dev, arena))
        return serve.Server(arena, orders=6.0, max_steps=1000, chunk=50, workers=2, keep=lambda rid: True,
                            mesh_for=lambda r: r)

    res, parts = serve.serve_devices(reqs, make_server, [0, 1])
    assert sorted(d for d, _ in made) == [0, 1]
    assert [x.rid for x in res] == sorted(r.rid for r in reqs)
    for (dev, arena), part in zip(sorted(made, key=lambda m: m[0]), parts):
        assert sorted(arena.admitted) == sorted(r.rid for r in part)     # each device served its share
    assert all(x.steps == 300 for x in res)                               # 10**(-0.02 n) <= 1e-6 at n = 300


def test_sequential_service_and_step_models():
    """The FP64 sequential baseline's estimators: queueing in arrival order, and the affine
    step-cost fit recovering a known fixed cost and per-cell cost."""
    reqs = [serve.Request(i, t, 0, 0, 2.0, 10.0, i) for i, t in enumerate((0.0, 0.5, 10.0))]
    steps = {0: 10, 1: 10, 2: 20}
    # 0.1 s per step: request 0 runs 0..1, request 1 waits until 1 and runs to 2, request 2 runs 10..12
    span, lat = serve.sequential_service(reqs, steps, lambda t: 0.1)
    assert span == pytest.approx(12.0) and lat == pytest.approx([1.0, 1.5, 2.0])
    x = np.array([5e3, 2e4, 8e4, 3e5, 1e6, 2e6])
    a, b = serve.affine_step_model(x, 2e-5 + 1.1e-10 * x)
    assert a == pytest.approx(2e-5, rel=1e-6) and b == pytest.approx(1.1e-10, rel=1e-6)
    a, b = serve.affine_step_model(x, 1.1e-10 * x - 1e-6)              # a negative fixed cost is clamped
    assert a == 0.0 and b > 0


def test_sequential_service_charges_each_request_its_overhead():
    """The end-to-end sequential estimate: each request takes its steps plus its own overhead
    (mesh, set-up, download), one at a time in arrival order."""
    from cfd_optimisations_b200.serve import Request, sequential_service
    reqs = [Request(0, 0.0, 11, 6, 2.0, 10.0, 1), Request(1, 0.5, 11, 6, 2.0, 10.0, 2), Request(2, 10.0, 11, 6, 2.0, 10.0, 3)]
    steps = {0: 100, 1: 100, 2: 100}
    span, lat = sequential_service(reqs, steps, lambda tri: 0.01, overhead=lambda tri: 0.5)
    # request 0: 0 -> 1.5; request 1 waits: 1.5 -> 3.0; request 2 arrives at 10: 10 -> 11.5
    assert span == pytest.approx(11.5)
    assert lat == pytest.approx([1.5, 2.5, 1.5])
    span0, _ = sequential_service(reqs, steps, lambda tri: 0.01)
    assert span0 == pytest.approx(11.0)
