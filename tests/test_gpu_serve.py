"""Serving loop on the device: a stream of requests served with continuous batching gives
each request the same state, bit for bit, as serving it alone."""
import numpy as np
import pytest

from cfd_optimisations_b200 import FP32, LIMITER_BJ, serve
from cfd_optimisations_b200.arena import Arena

pytestmark = pytest.mark.gpu


def arena(budget=16 << 20):
    return Arena(budget, precision=FP32, limiter=LIMITER_BJ, tile=128, max_instances=64)


def test_served_results_same_alone_and_in_the_mix():
    reqs = serve.request_stream(12, 400.0, 9, median=2e4, sigma=0.6, lo=4e3, hi=5e4)
    # a 16 MiB arena holds about 100k cells: the stream needs backfill
    srv = serve.Server(arena(), orders=0.2, max_steps=600, chunk=50, workers=4, keep=lambda rid: True)
    mix = {x.rid: x for x in srv.run(reqs)}
    assert len(mix) == len(reqs)
    assert srv.max_active >= 2
    first_done = min(x.t_done for x in mix.values())
    assert any(x.t_admit >= first_done for x in mix.values())   # admitted after a retirement
    assert not any(x.failed for x in mix.values())
    assert len({x.steps for x in mix.values()}) >= 2          # some retire early, others at the cap
    for r in reqs:
        alone = serve.Server(arena(), orders=0.2, max_steps=600, chunk=50, workers=1,
                             keep=lambda rid: True).run([serve.Request(r.rid, 0.0, r.nx, r.ny, r.mach, r.theta, r.seed)])
        assert alone[0].steps == mix[r.rid].steps
        assert np.array_equal(alone[0].U, mix[r.rid].U), r.rid
