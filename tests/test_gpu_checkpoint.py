"""Checkpoint and resume on the device: a solve interrupted by checkpoint, discarded and
restored into a new solver (or arena instance) continues bit for bit."""
import numpy as np
import pytest

import cfd_optimisations_b200 as H
from cfd_optimisations_b200.arena import Arena
from cfd_optimisations_b200.native import HcfdError

pytestmark = pytest.mark.gpu


def make(mesh, case, **kw):
    s = H.Solver(mesh, **kw)
    s.gather_bcs(case[0], case[1])
    s.initialise(case[2])
    return s


@pytest.mark.parametrize("precision", [H.FP64, H.FP32])
@pytest.mark.parametrize("freeze", [0, 15])
def test_solver_resume_is_bit_identical(tmp_path, precision, freeze):
    m = H.Mesh.wedge(121, 61, theta_deg=12.0, seed=3, numbering=H.NUMBER_RANDOM)
    case = H.wedge_case(2.7)
    kw = dict(precision=precision, limiter=H.LIMITER_BJ, freeze_limiter_after=freeze)
    a = make(m, case, **kw)
    a.step(20, H.GLOBAL_CFL, 0.5)
    path = str(tmp_path / "s.ckpt")
    a.checkpoint(path)
    info = H.checkpoint_info(path)
    assert info == dict(Nc=m.Nc, precision=precision, steps=20, has_limiter=freeze > 0)
    st_a = a.step(12, H.GLOBAL_CFL, 0.5)
    Ua = a.U()
    del a
    b = make(m, case, **kw)
    b.restore(path)
    st_b = b.step(12, H.GLOBAL_CFL, 0.5)
    assert np.array_equal(b.U(), Ua)
    assert st_b["steps"] == st_a["steps"] == 32
    assert st_b["res_first"] == st_a["res_first"] and st_b["res_l2"] == st_a["res_l2"]


def test_solver_restore_rejects_mismatch(tmp_path):
    m = H.Mesh.wedge(41, 21, seed=3)
    case = H.wedge_case(2.5)
    a = make(m, case)
    a.step(3, H.GLOBAL_CFL, 0.5)
    path = str(tmp_path / "m.ckpt")
    a.checkpoint(path)
    for kw, mesh in ((dict(precision=H.FP32), m), (dict(freeze_limiter_after=5), m), ({}, H.Mesh.wedge(43, 22, seed=3))):
        b = make(mesh, case, **kw)
        with pytest.raises(HcfdError) as e:
            b.restore(path)
        assert e.value.code == H.native.EINVAL


@pytest.mark.parametrize("freeze", [0, 10])
def test_arena_instance_preempt_and_resume(tmp_path, freeze):
    meshes = [H.Mesh.wedge(81, 41, theta_deg=t, seed=s, numbering=H.NUMBER_RANDOM) for t, s in ((8.0, 1), (13.0, 2))]
    cases = [H.wedge_case(2.2), H.wedge_case(3.1)]
    A = Arena(64 << 20, precision=H.FP32, limiter=H.LIMITER_BJ, max_instances=8, freeze_limiter_after=freeze)
    k0 = A.admit(meshes[0], *cases[0], 0.5)
    k1 = A.admit(meshes[1], *cases[1], 0.5)
    A.step(18)
    path = str(tmp_path / "i.ckpt")
    A.checkpoint(k1, path)
    A.step(9)
    ref = A.fetch(k1)
    ref_stats = A.poll()[k1]
    # preempt instance 1, run the other on, then resume it in a fresh arena
    A.release(k1)
    A.step(5)
    B = Arena(64 << 20, precision=H.FP32, limiter=H.LIMITER_BJ, max_instances=8, freeze_limiter_after=freeze)
    j = B.admit(meshes[1], *cases[1], 0.5)
    B.restore(j, path)
    B.step(9)
    assert np.array_equal(B.fetch(j), ref)
    st = B.poll()[j]
    assert st["steps"] == ref_stats["steps"] == 27 and st["res_l2"] == ref_stats["res_l2"]


@pytest.mark.parametrize("precision", [H.FP64, H.FP32])
def test_snapshot_while_stepping_matches_download(precision):
    """A snapshot taken between steps holds that step's state even though the solver steps on
    while it is copied; two snapshots in a row reuse the staging buffer safely."""
    m = H.Mesh.wedge(161, 81, seed=9, numbering=H.NUMBER_RANDOM)
    case = H.wedge_case(2.5)
    a = make(m, case, precision=precision)
    b = make(m, case, precision=precision)
    outs = [np.empty((4, m.Nc)), np.empty((4, m.Nc))]
    for o in outs:
        H.pin(o)
    try:
        a.step(7, H.GLOBAL_CFL, 0.5)
        t1 = a.snapshot(outs[0], prims=True)
        a.step(5, H.GLOBAL_CFL, 0.5)
        t2 = a.snapshot(outs[1], prims=False)
        a.step(3, H.GLOBAL_CFL, 0.5)
        b.step(7, H.GLOBAL_CFL, 0.5)
        assert np.array_equal(t1.wait(), b.Q())
        b.step(5, H.GLOBAL_CFL, 0.5)
        assert np.array_equal(t2.wait(), b.U())
        b.step(3, H.GLOBAL_CFL, 0.5)
        assert np.array_equal(a.U(), b.U())
    finally:
        del t1, t2
        for o in outs:
            H.unpin(o)
