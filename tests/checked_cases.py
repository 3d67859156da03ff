"""Workloads run by test_gpu_checked.py in a child process, once with the default library and
once with the checked one (HCFD_LIB=checked, chosen when the package is imported, hence a
process of its own for each).

    python tests/checked_cases.py OUT.npz            every workload; results into OUT.npz
    python tests/checked_cases.py OUT.npz --corrupt  (checked library only) one noalloc step
                                                     with an out-of-range neighbour id and one
                                                     with an out-of-range face id

Each workload steps a solver, an arena or the allocation-free entry point on small wedges and
saves the states and step statistics.  The corrupt case writes its status codes and the
state of a clean step taken afterwards in the same context.
"""
import ctypes as ct
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))

import cfd_optimisations_b200 as H  # noqa: E402
from cfd_optimisations_b200 import native as N  # noqa: E402
from cfd_optimisations_b200.arena import Arena  # noqa: E402


def _solver_runs(out):
    m = H.Mesh.wedge(161, 81, theta_deg=10.0, seed=3, numbering=H.NUMBER_RCM)
    bcmap, qbc, q = H.wedge_case(2.5)
    cases = {
        "tiled_fp64": dict(precision=H.FP64),
        "tiled_fp32": dict(precision=H.FP32),
        "tiled_fp64_one_plan": dict(precision=H.FP64, tile=128),
        "cell_fp64": dict(precision=H.FP64, kernel=H.KERNEL_CELL),
        "cell_fp32": dict(precision=H.FP32, kernel=H.KERNEL_CELL),
    }
    for name, kw in cases.items():
        for lim in (H.LIMITER_BJ, H.LIMITER_VENKAT):
            s = H.Solver(m, limiter=lim, venkat_K=5.0, **kw)
            s.gather_bcs(bcmap, qbc)
            s.initialise(q)
            a = s.step(8, H.GLOBAL_CFL, 0.5)
            b = s.step(4, H.LOCAL_CFL, 0.5)
            key = f"{name}_{lim}"
            out[key + "_U"] = s.U()
            out[key + "_stats"] = np.array([a["dt"], a["res_l2"], b["dt"], b["res_l2"]])


def _arena_runs(out):
    cases = [(H.Mesh.wedge(41, 21, theta_deg=8.0, seed=1), 2.0), (H.Mesh.wedge(121, 61, theta_deg=12.0, seed=2), 3.1),
             (H.Mesh.wedge(81, 41, theta_deg=5.0, seed=3), 2.4)]
    for prec in (H.FP32, H.FP64):
        a = Arena(1 << 28, precision=prec, limiter=H.LIMITER_VENKAT)
        slots = []
        for m, M in cases:
            bcmap, qbc, q = H.wedge_case(M)
            slots.append(a.admit(m, bcmap, qbc, q, 0.5))
        a.step(12)
        st = a.poll()
        for i, k in enumerate(slots):
            out[f"arena_{prec}_{i}_U"] = a.fetch(k)
            out[f"arena_{prec}_{i}_stats"] = np.array([st[k]["dt"], st[k]["res_l2"]])


def _noalloc_setup():
    """A small wedge's tables in the caller's device buffers, as hcfd_noalloc_mesh takes them."""
    import torch
    sys.path.insert(0, HERE)
    from test_zz_no_alloc import _planes, _tables
    mesh = H.Mesh.wedge(81, 41, theta_deg=15.0, seed=17, numbering=H.NUMBER_RANDOM)
    bcmap, qbc, q = H.wedge_case(2.5)
    s = H.Solver(mesh, kernel=H.KERNEL_CELL, keep_numbering=True, limiter=H.LIMITER_VENKAT, venkat_K=5.0)
    s.gather_bcs(bcmap, qbc)
    s.initialise(q)
    U0 = s.U()
    a, F_BC, W, slot, geo, iv = _tables(mesh)
    Nc, Nf = a["Nc"], a["Nf"]
    dev = torch.device("cuda:0")
    bufs = {"slot": slot, "d_slot": torch.from_numpy(slot.reshape(-1).copy()).to(dev),
            "d_geo": torch.from_numpy(geo.reshape(-1)).to(dev), "d_iv": torch.from_numpy(iv).to(dev),
            "d_U": [torch.from_numpy(_planes(U0)).to(dev), torch.zeros(4 * Nc, dtype=torch.float64, device=dev)]}
    ncol, nbc = a["Ncol"], a["NBCcol"]
    bufs["bc_first"] = np.ascontiguousarray(a["coloff"][ncol - nbc:ncol + 1], dtype=np.int32)
    bufs["bc_type"] = np.ascontiguousarray(np.asarray(bcmap)[a["coltag"][ncol - nbc:ncol]], dtype=np.int32)
    bufs["bc_state"] = np.ascontiguousarray(qbc, dtype=np.float64).reshape(-1)
    torch.cuda.synchronize()
    m = N.NoallocMesh(Nc, Nf, F_BC, W, bufs["d_slot"].data_ptr(), bufs["d_geo"].data_ptr(), bufs["d_iv"].data_ptr(),
                      nbc, bufs["bc_first"].ctypes.data_as(N._ip), bufs["bc_type"].ctypes.data_as(N._ip),
                      bufs["bc_state"].ctypes.data_as(N._dp), 1.4, H.LIMITER_VENKAT, 5.0)
    return m, bufs, Nc, Nf, F_BC


def _noalloc_step(m, bufs, i):
    import torch
    dt, res = ct.c_double(), ct.c_double()
    rc = N.lib().hcfd_step_noalloc(ct.byref(m), bufs["d_U"][i % 2].data_ptr(), bufs["d_U"][(i + 1) % 2].data_ptr(),
                                   H.GLOBAL_CFL, 0.5, None, ct.byref(dt), ct.byref(res))
    torch.cuda.synchronize()
    return rc, dt.value, res.value


def _noalloc_runs(out):
    m, bufs, Nc, _, _ = _noalloc_setup()
    for i in range(2):
        rc, dt, res = _noalloc_step(m, bufs, i)
        N.check(rc)
        out[f"noalloc_{i}_U"] = bufs["d_U"][(i + 1) % 2].cpu().numpy()
        out[f"noalloc_{i}_stats"] = np.array([dt, res])


def _corrupt_runs(out):
    """An interior cell's first slot gets a neighbour id past the last cell, then (restored) a
    face id past the last face.  The checked library checks the slot table on the device
    before launching the step, so both calls return HCFD_EINVAL without stepping; a clean step
    in the same context follows."""
    import torch
    assert N.LIB_PATH == N.LIB_CHECKED, "the corrupt case runs on the checked library only"
    m, bufs, Nc, Nf, F_BC = _noalloc_setup()
    slot = bufs["slot"]                                   # (W, Nc, 2): {face or ~face, neighbour}
    c = int(np.nonzero(slot[0, :, 1] >= 0)[0][0])
    codes, msgs = [], []
    for field, value in ((1, Nc + 1000), (0, Nf + 7)):
        bad = slot.copy()
        bad[0, c, field] = value
        bufs["d_slot"].copy_(torch.from_numpy(bad.reshape(-1)))
        torch.cuda.synchronize()
        codes.append(_noalloc_step(m, bufs, 0)[0])
        msgs.append((N.lib().hcfd_last_error() or b"").decode())
    bufs["d_slot"].copy_(torch.from_numpy(slot.reshape(-1).copy()))
    torch.cuda.synchronize()
    rc, dt, res = _noalloc_step(m, bufs, 0)
    codes.append(rc)
    out["codes"] = np.array(codes)
    out["msgs"] = np.array(msgs)
    out["clean_U"] = bufs["d_U"][1].cpu().numpy()
    out["clean_stats"] = np.array([dt, res])


def main(argv):
    out = {"lib": np.array(os.path.basename(N.LIB_PATH))}
    if "--corrupt" in argv:
        _corrupt_runs(out)
    else:
        _solver_runs(out)
        _arena_runs(out)
        _noalloc_runs(out)
    np.savez(argv[1], **out)


if __name__ == "__main__":
    main(sys.argv)
