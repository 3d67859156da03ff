"""Parity of the CUDA solver (through the C ABI) with the reference and with the oracle.

Tolerances are the FP64 bar for this path: relative L-infinity (max |a-b| / max |b| per
conserved variable, ghost cells included) <= 1e-12 after one step and <= 1e-9 after 1000
steps.  The GPU forms each per-cell sum in the reference's order but stores the limited
gradient premultiplied (phi * grad U) and fuses multiply-adds where nvcc chooses, so it
agrees with the reference to rounding, not bit for bit.
"""
import os

import numpy as np
import pytest

import cfd_optimisations_b200 as H
import oracle as O

pytestmark = pytest.mark.gpu

ONE_STEP = 1e-12
MANY_STEPS = 1e-9


def wedge_reference_case():
    # src/Test.cpp:51-64: gamma 1.4, M = 2, QIC = QBC = (1, 1, 0, 1/(gamma M^2)), dt 1e-3.
    gma, M = 1.4, 2.0
    p = 1.0 / (gma * M * M)
    q = np.array([1.0, 1.0, 0.0, p])
    return np.array([H.SYMMETRY, H.SYMMETRY, H.SYMMETRY, H.SUPINLET, H.SUPOUTLET]), np.tile(q, (4, 1)), q


def solver_for(mesh, bcmap, qbc, q, **kw):
    s = H.Solver(mesh, **kw)
    s.gather_bcs(bcmap, qbc)
    s.initialise(q)
    return s


def oracle_for(mesh, bcmap, qbc, q, limiter=O.BJ, K=0.0):
    o = O.Oracle(mesh.arrays())
    o.gather_bcs(bcmap, qbc)
    o.initialise(q)
    o.set_limiter(limiter, K)
    return o


def test_initial_state_matches_base0(golden):
    m = H.Mesh(os.path.join(golden, "wedge.hmsh"))
    s = solver_for(m, *wedge_reference_case())
    _, b0 = O.read_hsln(os.path.join(golden, "Base_0.hsln"))
    assert np.all(O.rel_linf(s.Q(), b0) <= 1e-15)


@pytest.mark.parametrize("kernel", [H.KERNEL_TILED, H.KERNEL_CELL])
def test_one_step_matches_oracle_wedge(golden, kernel):
    m = H.Mesh(os.path.join(golden, "wedge.hmsh"))
    case = wedge_reference_case()
    s = solver_for(m, *case, kernel=kernel)
    o = oracle_for(m, *case)
    s.step(1, H.FIXED_DT, 1e-3)
    o.step(O.FIXED_DT, 1e-3)
    assert np.all(O.rel_linf(s.U(), o.U()) <= ONE_STEP)


@pytest.mark.parametrize("kernel", [H.KERNEL_TILED, H.KERNEL_CELL])
def test_1000_steps_match_base1(golden, kernel):
    """The reference's shipped golden: wedge.hmsh, 1000 steps of dt = 1e-3."""
    m = H.Mesh(os.path.join(golden, "wedge.hmsh"))
    s = solver_for(m, *wedge_reference_case(), kernel=kernel)
    s.step(1000, H.FIXED_DT, 1e-3)
    _, b1 = O.read_hsln(os.path.join(golden, "Base_1.hsln"))
    assert np.all(O.rel_linf(s.Q(), b1) <= MANY_STEPS)
    assert np.all(O.rel_linf(s.U(), O.prim_to_cons(b1)) <= MANY_STEPS)


def test_generated_wedge_matches_reference_fixture(golden):
    """The reference (compiled unchanged) on a generated 41 x 21 wedge, random numbering."""
    m = H.Mesh(os.path.join(golden, "small_wedge.hmsh"))
    ref = np.load(os.path.join(golden, "ref_small_wedge.npz"))
    case = H.wedge_case(2.5)
    s = solver_for(m, *case)
    assert np.all(O.rel_linf(s.U(), ref["U0"]) <= 1e-15)
    s.step(1, H.FIXED_DT, float(ref["dt_fixed"]))
    assert np.all(O.rel_linf(s.U(), ref["U1"]) <= ONE_STEP)
    s.step(49, H.FIXED_DT, float(ref["dt_fixed"]))
    assert np.all(O.rel_linf(s.U(), ref["U50"]) <= 1e-11)
    # Global CFL 0.5: the reference stepped with the dt the oracle's CFL rule gives.
    s2 = solver_for(m, *case)
    dts = []
    for _ in range(20):
        dts.append(s2.step(1, H.GLOBAL_CFL, 0.5)["dt"])
    np.testing.assert_allclose(dts, ref["dts_cfl"], rtol=1e-12)
    assert np.all(O.rel_linf(s2.U(), ref["U_cfl20"]) <= 1e-11)


@pytest.mark.parametrize("kernel", [H.KERNEL_TILED, H.KERNEL_CELL])
@pytest.mark.parametrize("numbering", [H.NUMBER_RANDOM, H.NUMBER_RCM])
@pytest.mark.parametrize("limiter,K", [(H.LIMITER_BJ, 0.0), (H.LIMITER_VENKAT, 5.0)])
@pytest.mark.parametrize("mode", [H.GLOBAL_CFL, H.LOCAL_CFL])
def test_cfl_modes_and_limiters_match_oracle(numbering, limiter, K, mode, kernel):
    """The configuration of the 161 x 81 wedge (M = 2.5, 15 deg), 20 steps at CFL 0.5."""
    m = H.Mesh.wedge(161, 81, theta_deg=15.0, seed=1234, numbering=numbering)
    case = H.wedge_case(2.5)
    s = solver_for(m, *case, limiter=limiter, venkat_K=K, kernel=kernel)
    o = oracle_for(m, *case, limiter=limiter, K=K)
    for i in range(20):
        st = s.step(1, mode, 0.5)
        dt_o, res_o = o.step(mode, 0.5)
        assert abs(st["dt"] - dt_o) <= 1e-13 * dt_o
        assert abs(st["res_l2"] - res_o) <= 1e-10 * res_o
    assert np.all(O.rel_linf(s.U(), o.U()) <= 1e-11)


def test_many_steps_generated_wedge_match_oracle():
    m = H.Mesh.wedge(81, 41, theta_deg=15.0, seed=99, numbering=H.NUMBER_RANDOM)
    case = H.wedge_case(2.5)
    s = solver_for(m, *case)
    o = oracle_for(m, *case)
    s.step(1000, H.GLOBAL_CFL, 0.5, wait=False)
    for _ in range(1000):
        o.step(O.GLOBAL_CFL, 0.5)
    assert np.all(O.rel_linf(s.U(), o.U()) <= MANY_STEPS)


@pytest.mark.parametrize("types", [(H.WALL, H.WALL, H.SUBINLET, H.SUBOUTLET),
                                   (H.SYMMETRY, H.WALL, H.SUPINLET, H.SUPOUTLET)])
def test_boundary_types_match_oracle(types):
    m = H.Mesh.wedge(41, 21, theta_deg=10.0, seed=5, numbering=H.NUMBER_RANDOM)
    bcmap = np.array([H.SYMMETRY] + list(types))
    _, _, q = H.wedge_case(0.8)  # subsonic freestream so the subsonic BCs are meaningful
    qbc = np.tile(q, (4, 1))
    s = solver_for(m, bcmap, qbc, q)
    o = oracle_for(m, bcmap, qbc, q)
    assert np.all(O.rel_linf(s.U(), o.U()) <= 1e-15)
    for _ in range(10):
        s.step(1, H.GLOBAL_CFL, 0.4)
        o.step(O.GLOBAL_CFL, 0.4)
    assert np.all(O.rel_linf(s.U(), o.U()) <= 1e-11)


def test_runs_are_bit_identical():
    m = H.Mesh.wedge(161, 81, seed=3, numbering=H.NUMBER_RANDOM)
    case = H.wedge_case(2.5)
    out = []
    for _ in range(2):
        s = solver_for(m, *case, limiter=H.LIMITER_VENKAT, venkat_K=5.0)
        st = s.step(50, H.GLOBAL_CFL, 0.5)
        out.append((s.U(), st["res_l2"], st["dt"]))
    assert np.array_equal(out[0][0], out[1][0])
    assert out[0][1] == out[1][1] and out[0][2] == out[1][2]


def test_wall_cp_matches_oracle():
    m = H.Mesh.wedge(81, 41, seed=11, numbering=H.NUMBER_RCM)
    case = H.wedge_case(2.5)
    s = solver_for(m, *case)
    o = oracle_for(m, *case)
    s.step(30, H.GLOBAL_CFL, 0.5)
    for _ in range(30):
        o.step(O.GLOBAL_CFL, 0.5)
    cp_s = s.wall_cp(2, 1.4, 1.0, 2.5)
    cp_o = o.wall_cp(2, 1.4, 1.0, 2.5)
    assert cp_s.shape == cp_o.shape and cp_s.size == 80
    np.testing.assert_allclose(cp_s, cp_o, rtol=0, atol=1e-11 * np.abs(cp_o).max())


def test_nonfinite_state_is_reported():
    """A NaN planted in the host state before upload is caught by the step's finite check."""
    m = H.Mesh.wedge(41, 21, seed=1)
    s = solver_for(m, *H.wedge_case(2.5))
    U = s.U()
    U[0, 100] = np.nan
    s.upload(U)
    s.step(1, H.FIXED_DT, 1e-4, wait=False)
    with pytest.raises(H.HcfdError) as e:
        s.sync()
    assert e.value.code == -4


def test_upload_download_roundtrip():
    m = H.Mesh.wedge(41, 21, seed=2)
    s = solver_for(m, *H.wedge_case(2.5))
    U = s.U() * 1.01
    s.upload(U)
    assert np.array_equal(s.U(), U)


@pytest.mark.parametrize("precision", [H.FP64, H.FP32])
@pytest.mark.parametrize("tile", [0, 64])
def test_kernel_families_and_orders_agree(precision, tile):
    """Tiled vs per-cell kernels, Morton vs input order: every per-cell sum is formed in the
    same order, so the states agree to rounding of the fused multiply-adds the compiler picks
    in each kernel (bit-identical when it picks the same)."""
    m = H.Mesh.wedge(161, 81, seed=21, numbering=H.NUMBER_RANDOM)
    case = H.wedge_case(2.5)
    runs = []
    for kw in (dict(kernel=H.KERNEL_TILED, tile=tile), dict(kernel=H.KERNEL_CELL),
               dict(kernel=H.KERNEL_TILED, tile=tile, keep_numbering=True),
               dict(kernel=H.KERNEL_CELL, keep_numbering=True)):
        s = solver_for(m, *case, limiter=H.LIMITER_VENKAT, venkat_K=5.0, precision=precision, **kw)
        s.step(40, H.GLOBAL_CFL, 0.5)
        runs.append(s.U())
    tol = 1e-13 if precision == H.FP64 else 1e-6
    for r in runs[1:]:
        assert np.all(O.rel_linf(r, runs[0]) <= tol)


@pytest.mark.parametrize("kernel", [H.KERNEL_TILED, H.KERNEL_CELL])
@pytest.mark.parametrize("limiter,K", [(H.LIMITER_BJ, 0.0), (H.LIMITER_VENKAT, 5.0)])
def test_limiter_freezing_matches_oracle(kernel, limiter, K):
    """Limiter freezing (not in the reference): steps 1..N compute the limiter, later steps
    reuse step N's values; the GPU's device-side step count must switch at the same step.
    The oracle restarts each step from the GPU's state, so the comparison is per step and
    rounding differences cannot build up through the limiter's switches."""
    m = H.Mesh.wedge(81, 41, theta_deg=20.0, seed=1234, numbering=H.NUMBER_RANDOM)
    case = H.wedge_case(3.0)
    s = solver_for(m, *case, limiter=limiter, venkat_K=K, kernel=kernel, freeze_limiter_after=25)
    free = solver_for(m, *case, limiter=limiter, venkat_K=K, kernel=kernel)
    o = oracle_for(m, *case, limiter=limiter, K=K)
    o.set_freeze(25)
    for i in range(1, 41):
        o.set_U(s.U())
        st = s.step(1, H.LOCAL_CFL, 0.8)
        dt_o, res_o = o.step(O.LOCAL_CFL, 0.8)
        free.step(1, H.LOCAL_CFL, 0.8)
        assert abs(st["res_l2"] - res_o) <= 1e-11 * res_o, i
        assert np.all(O.rel_linf(s.U(), o.U()) <= 1e-11), i
        if i <= 25:
            assert np.array_equal(s.U(), free.U()), i     # the same kernels before the switch
        elif i == 26:
            assert not np.array_equal(s.U(), free.U())   # the frozen limiter is in use


@pytest.mark.parametrize("kernel", [H.KERNEL_TILED, H.KERNEL_CELL])
def test_imported_mixed_mesh_matches_oracle(tmp_path, kernel):
    """A gmsh-imported mesh of quadrangles and triangles (four faces per cell at most)."""
    from test_meshio import write_msh
    from cfd_optimisations_b200 import meshio
    write_msh(tmp_path / "r.msh", nx=41, ny=21)
    meshio.import_msh(str(tmp_path / "r.msh"), str(tmp_path / "r.hmsh"))
    m = H.Mesh(str(tmp_path / "r.hmsh"))
    bcmap = [H.SYMMETRY, H.SYMMETRY, H.SUPOUTLET, H.SYMMETRY, H.SUPINLET]
    q = (1.4, 2.2, 0.35, 1.0)          # oblique inflow: the walls turn it, so no variable stays at zero
    qbc = [q] * 4
    s = solver_for(m, bcmap, qbc, q, limiter=H.LIMITER_BJ, kernel=kernel)
    o = oracle_for(m, bcmap, qbc, q)
    for _ in range(20):
        st = s.step(1, H.GLOBAL_CFL, 0.5)
        dt_o, res_o = o.step(O.GLOBAL_CFL, 0.5)
        assert abs(st["dt"] - dt_o) <= 1e-13 * dt_o
    assert np.all(O.rel_linf(s.U(), o.U()) <= 1e-11)


def test_config1_2000_steps_match_the_reference(tmp_path):
    """The reference's CPU case, end to end: the 161 x 81 wedge (25,600 triangles, random
    numbering), M 2.5, 15 deg, Barth-Jespersen, global CFL 0.5, 2000 steps on the GPU; the
    reference (compiled unchanged) steps the same mesh with the GPU's dt sequence (it has no CFL
    control of its own)."""
    if not O.RefSolver.available():
        pytest.skip("the reference library was not built here")
    m = H.Mesh.wedge(161, 81, theta_deg=15.0, seed=1234, numbering=H.NUMBER_RANDOM)
    path = str(tmp_path / "c1.hmsh")
    m.write(path)
    bcmap, qbc, q = H.wedge_case(2.5)
    s = solver_for(m, bcmap, qbc, q)
    dts = np.array([s.step(1, H.GLOBAL_CFL, 0.5)["dt"] for _ in range(2000)])
    ref = O.RefSolver(path, bcmap, qbc, q)
    ref.steps(2000, dts)
    assert np.all(O.rel_linf(s.U(), ref.U()) <= MANY_STEPS)
