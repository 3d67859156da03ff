"""The precision study's lockstep tracking (precision.track) on the CPU, with stand-in solvers
whose states drift from the FP64 one at set rates: the bookkeeping of the errors, of the last
step within the bound, and of a solve that produces a NaN or Inf."""
import numpy as np
import pytest

from cfd_optimisations_b200 import precision as P
from cfd_optimisations_b200.native import ENONFINITE, HcfdError


def fake_solver(drift, fail_after=None):
    """A stand-in for Solver: state 1 + drift(step) per precision, NaN/Inf error after
    `fail_after` steps of one precision."""
    class S:
        def __init__(self, mesh, precision, freeze_limiter_after=0, **kw):
            self.prec, self.n, self.scale = precision, 0, 1.0

        def gather_bcs(self, bcmap, qbc):
            pass

        def initialise(self, q):
            self.scale = q[0] / 1.4

        def step(self, n, mode, cfl):
            self.n += n
            if fail_after is not None and self.prec == P.FP32 and self.n > fail_after:
                raise HcfdError(ENONFINITE, "a step produced a NaN or Inf")

        def stats(self):
            return dict(res_l2=1.0 / (1 + self.n))

        def U(self):
            e = drift(self.n) if self.prec == P.FP32 else (self.scale - 1.0) * 1e6 * self.n
            return np.full((4, 8), 1.0 + e)
    return S


def test_track_records_errors_and_the_horizon(monkeypatch):
    monkeypatch.setattr(P, "Solver", fake_solver(lambda n: 1e-7 * 2.0 ** (n / 10)))
    out = P.track(None, 2.5, 0.5, steps=100, every=10)
    steps = [r["step"] for r in out["history"]]
    assert steps == list(range(0, 101, 10)) and out["diverged"] is None
    # FP32 drift 1e-7 * 2**(n/10): within 1e-5 while 2**(n/10) <= 100, i.e. up to step 60
    assert out["steps_within_bound"]["fp32"] == 60
    r = out["history"][1]
    assert r["fp32"] == pytest.approx(2e-7, rel=1e-6) and r["fp32_l2"] == pytest.approx(2e-7, rel=1e-6)
    # the perturbed FP64 solve: (2**-52 * 1e6) * n stays far below the bound
    assert out["steps_within_bound"]["fp64_perturbed"] == 100


def test_track_ends_at_a_nonfinite_step(monkeypatch):
    monkeypatch.setattr(P, "Solver", fake_solver(lambda n: 1e-8, fail_after=35))
    out = P.track(None, 2.5, 0.5, steps=100, every=10)
    assert out["diverged"] == dict(solve="fp32", by_step=40)
    assert [r["step"] for r in out["history"]] == [0, 10, 20, 30]


def test_handoff_restores_the_converted_fp64_checkpoint_into_fp32(monkeypatch):
    """precision.handoff with stand-in solvers that write and read the real checkpoint format
    (and, like the library, refuse a checkpoint of the other precision): the FP32 solver that
    takes over starts from the FP64 state rounded to floats and follows FP64; the FP32 solve
    with its own limiter values (here: a fixed offset) never is within the bound."""
    import struct
    HDR = struct.Struct("<8siiiiqdddii")
    Nc = 8

    class S:
        def __init__(self, mesh, precision, freeze_limiter_after=0, **kw):
            self.prec, self.freeze, self.n = precision, freeze_limiter_after, 0
            base = np.linspace(1.0, 2.0, 4 * Nc).reshape(4, Nc) * (1 + 1e-9 * np.pi)
            self.u = base + (1e-3 if precision == P.FP32 else 0.0)
            if precision == P.FP32:
                self.u = self.u.astype(np.float32).astype(np.float64)

        def gather_bcs(self, bcmap, qbc):
            pass

        def initialise(self, q):
            pass

        def step(self, n, mode, cfl):
            self.n += n
            self.u = self.u + 1e-4 * n
            if self.prec == P.FP32:
                self.u = self.u.astype(np.float32).astype(np.float64)

        def stats(self):
            return dict(res_l2=1.0 / (1 + self.n))

        def U(self):
            return self.u.copy()

        def checkpoint(self, path):
            with open(path, "wb") as fh:
                fh.write(HDR.pack(b"HCFDCKP1", 1, self.prec, Nc, 1, self.n, 1.0, 1.0, 1e-3, 0, 0))
                fh.write(np.concatenate([self.u.ravel(), np.ones(4 * Nc)]).astype("<f8").tobytes())

        def restore(self, path):
            raw = open(path, "rb").read()
            h = HDR.unpack_from(raw, 0)
            if h[2] != self.prec or h[3] != Nc or h[4] != 1:
                raise HcfdError(-1, "restore: mismatch")
            vals = np.frombuffer(raw, dtype="<f8", offset=HDR.size)
            self.u, self.n = vals[:4 * Nc].reshape(4, Nc).copy(), h[5]

    monkeypatch.setattr(P, "Solver", S)
    out = P.handoff(None, 2.5, 0.5, steps=400, every=100, freeze=100)
    assert out["diverged"] is None
    assert [r["step"] for r in out["history"]] == [100, 200, 300, 400]
    first = out["history"][0]
    assert 0 < first["fp32_handoff"] <= 2.0 ** -23            # the FP64 state rounded to floats
    assert out["steps_within_bound"] == dict(fp32_handoff=400, fp32_own_limiter=None)
