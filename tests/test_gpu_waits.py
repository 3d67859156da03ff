"""The bounded waits of the tiled step kernels run out without faulting, hanging or poisoning
the context.

hcfd_gpu_test_waits makes the staging warp arm nothing for one tile, so the compute warps'
wait for that tile has nothing in flight and runs out (after a short poll limit).  The step
must come back with HCFD_ETIMEOUT; the CTA must leave no copy in flight (the staging warp of
that CTA has armed later tiles on the larger mesh, and drains them before it exits); and after
re-initialising, the same handle must step bit-identically to a fresh handle.  No GPU fault is
made: every address stays valid, only a wait is left unsatisfied.
"""
import ctypes as ct

import numpy as np
import pytest

import cfd_optimisations_b200 as H
from cfd_optimisations_b200 import native as N

pytestmark = pytest.mark.gpu


def _solver(m, precision):
    s = H.Solver(m, precision=precision, limiter=H.LIMITER_VENKAT, venkat_K=5.0)
    s.gather_bcs(*H.wedge_case(2.5)[:2])
    s.initialise(H.wedge_case(2.5)[2])
    return s


@pytest.mark.parametrize("precision", [H.FP64, H.FP32])
@pytest.mark.parametrize("nx,ny,skip", [(81, 41, 1), (401, 201, 1), (401, 201, 0)])
def test_a_wait_that_runs_out_reports_etimeout_and_the_handle_recovers(precision, nx, ny, skip):
    m = H.Mesh.wedge(nx, ny, seed=9, numbering=H.NUMBER_RCM)
    s = _solver(m, precision)
    s.step(2, H.GLOBAL_CFL, 0.5)
    L = N.lib()
    N.check(L.hcfd_gpu_test_waits(s._h, 1 << 16, skip))
    with pytest.raises(H.HcfdError) as e:
        s.step(1, H.GLOBAL_CFL, 0.5)
    assert e.value.code == N.ETIMEOUT
    # the error stays until the state is re-initialised
    with pytest.raises(H.HcfdError):
        s.sync()
    N.check(L.hcfd_gpu_test_waits(s._h, 0, -1))
    s.initialise(H.wedge_case(2.5)[2])
    st = s.step(6, H.GLOBAL_CFL, 0.5)
    fresh = _solver(m, precision)
    st_f = fresh.step(6, H.GLOBAL_CFL, 0.5)
    assert np.array_equal(s.U(), fresh.U())
    assert st["dt"] == st_f["dt"] and st["res_l2"] == st_f["res_l2"]


def test_test_hook_rejects_a_poll_limit_above_2_to_30():
    s = _solver(H.Mesh.wedge(41, 21, seed=1), H.FP64)
    assert N.lib().hcfd_gpu_test_waits(s._h, (1 << 30) + 1, -1) == N.EINVAL
