"""The allocation-free step, hcfd_step_noalloc, against the solver's own step.

Some callers cannot call cudaMalloc: a framework that owns every byte of device memory
through its own pool, or a caller that must not let a library allocate (cudaMalloc and
cudaFree can synchronise the device).  They keep the inputs and outputs in their own device
buffers and the step takes its scratch from a static device array of the library.  Here the
caller's buffers are allocated by torch, on the caller's side; the entry point is called
through the C ABI twice in a row and each result is checked against the existing entry
point (hcfd_gpu_step) on the same mesh and state, at the one-step tolerance of the parity
tests.  The file is named so that pytest collects it last.
"""
import ctypes as ct

import numpy as np
import pytest

import cfd_optimisations_b200 as H
from cfd_optimisations_b200 import native as N
import oracle as O

pytestmark = pytest.mark.gpu

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


def test_noalloc_step_matches_solver_step_twice():
    torch = pytest.importorskip("torch")
    mesh = H.Mesh.wedge(81, 41, theta_deg=15.0, seed=17, numbering=H.NUMBER_RANDOM)
    bcmap, qbc, q = H.wedge_case(2.5)

    # the existing entry point
    s = H.Solver(mesh, kernel=H.KERNEL_CELL, keep_numbering=True)
    s.gather_bcs(bcmap, qbc)
    s.initialise(q)
    U0 = s.U()
    ref = []
    for _ in range(2):
        st = s.step(1, H.GLOBAL_CFL, 0.5)
        ref.append((s.U(), st["dt"], st["res_l2"]))

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
    bc_type = np.ascontiguousarray(bcmap[a["coltag"][ncol - nbc:ncol]], dtype=np.int32)
    bc_state = np.ascontiguousarray(qbc, dtype=np.float64).reshape(-1)
    m = N.NoallocMesh(Nc, Nf, F_BC, W, d_slot.data_ptr(), d_geo.data_ptr(), d_iv.data_ptr(),
                      nbc, bc_first.ctypes.data_as(N._ip), bc_type.ctypes.data_as(N._ip),
                      bc_state.ctypes.data_as(N._dp), 1.4, H.LIMITER_BJ, 5.0)
    lib = N.lib()
    for i in range(2):
        dt, res = ct.c_double(), ct.c_double()
        rc = lib.hcfd_step_noalloc(ct.byref(m), d_U[i % 2].data_ptr(), d_U[(i + 1) % 2].data_ptr(),
                                   H.GLOBAL_CFL, 0.5, None, ct.byref(dt), ct.byref(res))
        N.check(rc)
        torch.cuda.synchronize()
        U = _unplanes(d_U[(i + 1) % 2].cpu().numpy(), Nc)
        U_ref, dt_ref, res_ref = ref[i]
        assert np.all(O.rel_linf(U, U_ref) <= ONE_STEP), O.rel_linf(U, U_ref)
        assert abs(dt.value - dt_ref) <= 1e-13 * dt_ref
        assert abs(res.value - res_ref) <= 1e-10 * res_ref


def test_noalloc_rejects_meshes_above_the_scratch_size():
    m = N.NoallocMesh(N.NOALLOC_MAX_CELLS + 1, 10, 0, 3, 1, 1, 1, 0, None, None, None, 1.4, 0, 5.0)
    rc = N.lib().hcfd_step_noalloc(ct.byref(m), ct.c_void_p(16), ct.c_void_p(32), H.FIXED_DT, 1e-3,
                                   None, None, None)
    assert rc == N.EINVAL
    assert b"65536" in N.lib().hcfd_last_error()
