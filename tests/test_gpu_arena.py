"""The device arena (many meshes in one set of device arrays): each instance's state is
bit-identical to the single-mesh solver with the same tile size, alone or in a mix; budget
admission, release and backfill leave the other instances untouched."""
import numpy as np
import pytest

import cfd_optimisations_b200 as H
from cfd_optimisations_b200.arena import Arena
import oracle as O

pytestmark = pytest.mark.gpu


def _single(mesh, mach, precision, limiter, steps, tile=128):
    bcmap, qbc, q = H.wedge_case(mach)
    s = H.Solver(mesh, precision=precision, limiter=limiter, venkat_K=5.0, tile=tile)
    s.gather_bcs(bcmap, qbc)
    s.initialise(q)
    st = s.step(steps, H.GLOBAL_CFL, 0.5)
    return s.U(), st


@pytest.mark.parametrize("precision", [H.FP64, H.FP32])
def test_instances_match_the_single_mesh_solver_alone_and_mixed(precision):
    lim = H.LIMITER_VENKAT
    cases = [(H.Mesh.wedge(41, 21, theta_deg=8.0, seed=1), 2.0), (H.Mesh.wedge(121, 61, theta_deg=12.0, seed=2), 3.1),
             (H.Mesh.wedge(81, 41, theta_deg=5.0, seed=3), 2.4), (H.Mesh.wedge(61, 31, theta_deg=15.0, seed=4), 1.9)]
    steps = 30
    ref = [_single(m, M, precision, lim, steps) for m, M in cases]
    # alone
    for (m, M), (U, st) in zip(cases[:2], ref[:2]):
        a = Arena(1 << 28, precision=precision, limiter=lim)
        bcmap, qbc, q = H.wedge_case(M)
        k = a.admit(m, bcmap, qbc, q, 0.5)
        a.step(steps)
        assert np.array_equal(a.fetch(k), U)
        assert a.poll()[k]["dt"] == st["dt"]
    # mixed
    a = Arena(1 << 28, precision=precision, limiter=lim)
    slots = []
    for m, M in cases:
        bcmap, qbc, q = H.wedge_case(M)
        slots.append(a.admit(m, bcmap, qbc, q, 0.5))
    a.step(steps)
    stats = a.poll()
    for k, (U, st) in zip(slots, ref):
        assert np.array_equal(a.fetch(k), U)
        assert stats[k]["dt"] == st["dt"]
        assert stats[k]["steps"] == steps
        assert stats[k]["res_l2"] == pytest.approx(st["res_l2"], rel=1e-12)


def test_budget_admission_release_and_backfill():
    big = H.Mesh.wedge(201, 101, seed=5)
    small = H.Mesh.wedge(41, 21, seed=6)
    bcmap, qbc, q = H.wedge_case(2.5)
    a = Arena(24 << 20, precision=H.FP32)          # room for about two of the big meshes
    admitted = []
    while True:
        k = a.admit(big, bcmap, qbc, q, 0.5)
        if k is None:
            break
        admitted.append(k)
        assert len(admitted) < 50
    assert len(admitted) >= 1
    keep = admitted[-1]
    a.step(10)
    U_keep = a.fetch(keep)
    # retire one, backfill with small meshes while `keep` continues
    a.release(admitted[0])
    backfill = a.admit(small, bcmap, qbc, q, 0.5)
    assert backfill is not None
    a.step(10)
    # `keep` advanced 20 steps exactly as it would alone
    U_ref, _ = _single(big, 2.5, H.FP32, H.LIMITER_BJ, 20)
    assert np.array_equal(a.fetch(keep), U_ref)
    U_small, _ = _single(small, 2.5, H.FP32, H.LIMITER_BJ, 10)
    assert np.array_equal(a.fetch(backfill), U_small)
    info = a.info()
    assert info["active"] == len(admitted) and info["cells_used"] <= info["cell_capacity"]


def test_arena_fp32_tracks_the_fp64_oracle():
    """FP32 arena instances stay within 1e-5 relative L-inf of the FP64 oracle over 50 steps."""
    m = H.Mesh.wedge(81, 41, seed=8)
    bcmap, qbc, q = H.wedge_case(2.5)
    a = Arena(1 << 27, precision=H.FP32, limiter=H.LIMITER_VENKAT)
    k = a.admit(m, bcmap, qbc, q, 0.5)
    o = O.Oracle(m.arrays())
    o.gather_bcs(bcmap, qbc)
    o.initialise(q)
    o.set_limiter(O.VENKAT, 5.0)
    a.step(50)
    for _ in range(50):
        o.step(O.GLOBAL_CFL, 0.5)
    assert np.all(O.rel_linf(a.fetch(k), o.U()) <= 1e-5)


def test_arena_limiter_freezing_per_instance():
    """Instances admitted at different times freeze their limiter after their own N steps."""
    m1, m2 = H.Mesh.wedge(81, 41, seed=11), H.Mesh.wedge(61, 31, seed=12)
    bcmap, qbc, q = H.wedge_case(2.5)
    a = Arena(1 << 27, precision=H.FP64, freeze_limiter_after=15)
    k1 = a.admit(m1, bcmap, qbc, q, 0.5)
    a.step(10)
    k2 = a.admit(m2, bcmap, qbc, q, 0.5)
    a.step(20)
    for k, m, n in ((k1, m1, 30), (k2, m2, 20)):
        s = H.Solver(m, precision=H.FP64, freeze_limiter_after=15)
        s.gather_bcs(bcmap, qbc)
        s.initialise(q)
        s.step(n, H.GLOBAL_CFL, 0.5)
        assert np.array_equal(a.fetch(k), s.U())
