"""The allocation-free step, hcfd_step_noalloc, against the solver's own step.

Some callers cannot call cudaMalloc: a framework that owns every byte of device memory
through its own pool, or a caller that must not let a library allocate (cudaMalloc and
cudaFree can synchronise the device).  They keep the inputs and outputs in their own device
buffers and the step takes its scratch from a static device array of the library.  Here the
caller's buffers are allocated by torch, on the caller's side; the entry point is called
through the C ABI twice in a row and each result is checked against the existing entry
point (hcfd_gpu_step) on the same mesh and state, and against the oracle, at the one-step
tolerance of the parity tests.  The argument checks run on the host and need no GPU.  The
file is named so that pytest collects it last.
"""
import ctypes as ct

import numpy as np
import pytest

import cfd_optimisations_b200 as H
from cfd_optimisations_b200 import native as N
import oracle as O

ONE_STEP = 1e-12


def _tables(mesh):
    """Slot table, face records and 1/area of `mesh` in the layouts hcfd_noalloc_mesh
    documents (face records from the oracle's restatement of the reference's Domain)."""
    a = mesh.arrays()
    Nc, Nf = a["Nc"], a["Nf"]
    F_BC = int(a["coloff"][a["Ncol"] - a["NBCcol"]])
    fc = a["fc_con"].reshape(-1, 2)
    cf_off, cf_con = a["cf_off"], a["cf_con"]
    ghost = np.zeros(Nc, dtype=bool)
    ghost[fc[F_BC:, 1]] = True
    deg = np.diff(cf_off)
    W = 3 if deg[~ghost].max() <= 3 else (4 if deg[~ghost].max() <= 4 else 8)
    slot = np.full((W, Nc, 2), -1, dtype=np.int32)
    for c in np.nonzero(~ghost)[0]:
        for k, j in enumerate(range(cf_off[c], cf_off[c + 1])):
            f = int(cf_con[j])
            L, R = fc[f]
            slot[k, c] = (f, R) if L == c else (~f, L)
    d = O.Oracle(a).domain()
    geo = np.column_stack([d["nf"][:, 0], d["nf"][:, 1], d["Af"], d["If"],
                           d["rf"][:, 0, 0], d["rf"][:, 0, 1], d["rf"][:, 1, 0], d["rf"][:, 1, 1]])
    return a, F_BC, W, slot, np.ascontiguousarray(geo), d["iv"].copy()


def _planes(U):
    """Variable-major (4, Nc) state -> the two planes of pairs hcfd_step_noalloc takes."""
    return np.concatenate([np.column_stack([U[0], U[1]]).ravel(), np.column_stack([U[2], U[3]]).ravel()])


def _unplanes(p, Nc):
    p0 = p[:2 * Nc].reshape(Nc, 2)
    p1 = p[2 * Nc:].reshape(Nc, 2)
    return np.stack([p0[:, 0], p0[:, 1], p1[:, 0], p1[:, 1]])


def _noalloc_case(mesh, bcmap, qbc, q, limiter, K, time_mode, value):
    """Two steps through hcfd_step_noalloc from the initial state, each checked against the
    existing entry point (hcfd_gpu_step, per-cell kernels in the caller's numbering) and
    against the oracle, at the one-step tolerance."""
    torch = pytest.importorskip("torch")
    s = H.Solver(mesh, kernel=H.KERNEL_CELL, keep_numbering=True, limiter=limiter, venkat_K=K)
    s.gather_bcs(bcmap, qbc)
    s.initialise(q)
    U0 = s.U()
    o = O.Oracle(mesh.arrays())
    o.gather_bcs(bcmap, qbc)
    o.initialise(q)
    o.set_limiter(O.VENKAT if limiter == H.LIMITER_VENKAT else O.BJ, K)
    ref = []
    for _ in range(2):
        st = s.step(1, time_mode, value)
        dt_o, res_o = o.step(time_mode, value)
        ref.append((s.U(), st["dt"], st["res_l2"], o.U(), dt_o, res_o))

    # the caller's own device buffers
    a, F_BC, W, slot, geo, iv = _tables(mesh)
    Nc, Nf = a["Nc"], a["Nf"]
    assert Nc <= N.NOALLOC_MAX_CELLS
    dev = torch.device("cuda:0")
    d_slot = torch.from_numpy(slot.reshape(-1)).to(dev)
    d_geo = torch.from_numpy(geo.reshape(-1)).to(dev)
    d_iv = torch.from_numpy(iv).to(dev)
    d_U = [torch.from_numpy(_planes(U0)).to(dev), torch.zeros(4 * Nc, dtype=torch.float64, device=dev)]
    torch.cuda.synchronize()

    ncol, nbc = a["Ncol"], a["NBCcol"]
    bc_first = np.ascontiguousarray(a["coloff"][ncol - nbc:ncol + 1], dtype=np.int32)
    bc_type = np.ascontiguousarray(np.asarray(bcmap)[a["coltag"][ncol - nbc:ncol]], dtype=np.int32)
    bc_state = np.ascontiguousarray(qbc, dtype=np.float64).reshape(-1)
    m = N.NoallocMesh(Nc, Nf, F_BC, W, d_slot.data_ptr(), d_geo.data_ptr(), d_iv.data_ptr(),
                      nbc, bc_first.ctypes.data_as(N._ip), bc_type.ctypes.data_as(N._ip),
                      bc_state.ctypes.data_as(N._dp), 1.4, limiter, K)
    lib = N.lib()
    for i in range(2):
        dt, res = ct.c_double(), ct.c_double()
        rc = lib.hcfd_step_noalloc(ct.byref(m), d_U[i % 2].data_ptr(), d_U[(i + 1) % 2].data_ptr(),
                                   time_mode, value, None, ct.byref(dt), ct.byref(res))
        N.check(rc)
        torch.cuda.synchronize()
        U = _unplanes(d_U[(i + 1) % 2].cpu().numpy(), Nc)
        U_ref, dt_ref, res_ref, U_o, dt_o, res_o = ref[i]
        assert np.all(O.rel_linf(U, U_ref) <= ONE_STEP), O.rel_linf(U, U_ref)
        assert np.all(O.rel_linf(U, U_o) <= ONE_STEP), O.rel_linf(U, U_o)
        for d in (dt_ref, dt_o):
            assert abs(dt.value - d) <= 1e-13 * d
        for r in (res_ref, res_o):
            assert abs(res.value - r) <= 1e-10 * r
    return W


@pytest.mark.gpu
@pytest.mark.parametrize("limiter,K", [(H.LIMITER_BJ, 0.0), (H.LIMITER_VENKAT, 5.0)])
@pytest.mark.parametrize("time_mode,value", [(H.FIXED_DT, 2e-4), (H.GLOBAL_CFL, 0.5)])
def test_noalloc_step_matches_solver_step_twice(limiter, K, time_mode, value):
    mesh = H.Mesh.wedge(81, 41, theta_deg=15.0, seed=17, numbering=H.NUMBER_RANDOM)
    bcmap, qbc, q = H.wedge_case(2.5)
    assert _noalloc_case(mesh, bcmap, qbc, q, limiter, K, time_mode, value) == 3


@pytest.mark.gpu
def test_noalloc_step_on_a_mixed_quad_triangle_mesh(tmp_path):
    """A gmsh-imported mesh of quadrangles and triangles: four face slots per cell."""
    from test_meshio import write_msh
    from cfd_optimisations_b200 import meshio
    write_msh(tmp_path / "r.msh", nx=41, ny=21)
    meshio.import_msh(str(tmp_path / "r.msh"), str(tmp_path / "r.hmsh"))
    mesh = H.Mesh(str(tmp_path / "r.hmsh"))
    bcmap = [H.SYMMETRY, H.SYMMETRY, H.SUPOUTLET, H.SYMMETRY, H.SUPINLET]
    q = (1.4, 2.2, 0.35, 1.0)
    assert _noalloc_case(mesh, bcmap, [q] * 4, q, H.LIMITER_BJ, 0.0, H.GLOBAL_CFL, 0.5) == 4


def _bad_mesh(**kw):
    f = dict(Nc=100, Nf=160, F_BC=150, slots=3, nbc=2, bc_first=[150, 155, 160])
    f.update(kw)
    first = np.ascontiguousarray(f["bc_first"], dtype=np.int32)
    types = np.zeros(max(f["nbc"], 1), dtype=np.int32)
    state = np.ones(4 * max(f["nbc"], 1))
    m = N.NoallocMesh(f["Nc"], f["Nf"], f["F_BC"], f["slots"], 16, 16, 16, f["nbc"], first.ctypes.data_as(N._ip),
                      types.ctypes.data_as(N._ip), state.ctypes.data_as(N._dp), 1.4, 0, 5.0)
    return m, (first, types, state)


def _call(m, U_in=4096, U_out=65536):
    return N.lib().hcfd_step_noalloc(ct.byref(m), ct.c_void_p(U_in), ct.c_void_p(U_out), H.FIXED_DT, 1e-3,
                                     None, None, None)


def test_noalloc_rejects_meshes_above_the_scratch_size():
    m = N.NoallocMesh(N.NOALLOC_MAX_CELLS + 1, 10, 0, 3, 1, 1, 1, 0, None, None, None, 1.4, 0, 5.0)
    rc = N.lib().hcfd_step_noalloc(ct.byref(m), ct.c_void_p(16), ct.c_void_p(32), H.FIXED_DT, 1e-3,
                                   None, None, None)
    assert rc == N.EINVAL
    assert b"65536" in N.lib().hcfd_last_error()


@pytest.mark.parametrize("kw", [dict(bc_first=[140, 155, 160]), dict(bc_first=[150, 155, 159]),
                                dict(bc_first=[150, 161, 160]), dict(nbc=0, bc_first=[0]),
                                dict(F_BC=160, nbc=1, bc_first=[150, 160])])
def test_noalloc_rejects_a_boundary_table_that_does_not_cover_the_boundary_faces(kw):
    """Checked on the host before any CUDA call: runs without a GPU."""
    m, keep = _bad_mesh(**kw)
    assert _call(m) == N.EINVAL
    assert b"bc_first" in N.lib().hcfd_last_error() or b"boundary colours" in N.lib().hcfd_last_error()


@pytest.mark.parametrize("U_in,U_out", [(4096, 4096), (4096, 4096 + 8), (4096 + 3200 - 8, 4096)])
def test_noalloc_rejects_overlapping_state_buffers(U_in, U_out):
    """4 Nc doubles (3,200 bytes at Nc = 100) from each pointer: any shared byte is refused."""
    m, keep = _bad_mesh()
    assert _call(m, U_in, U_out) == N.EINVAL
    assert b"overlap" in N.lib().hcfd_last_error()
