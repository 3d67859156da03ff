"""Parity at the full sizes the benchmark and the precision study run (FP64, through the C ABI).

* The benchmark case: the 2001 x 1001-node wedge (4,000,000 triangles, 6,000 ghosts,
  6,003,000 faces), M 2.5, 15 deg, Venkatakrishnan K = 5, global CFL 0.5, RCM numbering.
* The precision-study case: the 1025 x 513-node wedge (1,048,576 triangles), M 3.0, 20 deg,
  local time stepping at CFL 0.8, Barth-Jespersen.

These meshes have far more tiles, halo lists and tile-cut faces than the small parity meshes,
so they pin the tile plans the benchmark numbers come from.  Tolerance: relative L-infinity
(max |a-b| / max |b| per conserved variable, ghost cells included) <= 1e-12 after each of the
first two steps against the oracle (the C restatement of src/Base/*.cpp, with the
Venkatakrishnan limiter and CFL control it defines), the CFL dt to 1e-13 and the L2 density
residual to 1e-10; two GPU runs are bit-identical (no atomics in any sum).
"""
import numpy as np
import pytest

import cfd_optimisations_b200 as H
import oracle as O

pytestmark = pytest.mark.gpu

ONE_STEP = 1e-12

CASES = {
    "bench_2001x1001_venkat_global": dict(nx=2001, ny=1001, theta=15.0, mach=2.5, limiter=H.LIMITER_VENKAT,
                                          K=5.0, mode=H.GLOBAL_CFL, cfl=0.5),
    "precision_1025x513_bj_local": dict(nx=1025, ny=513, theta=20.0, mach=3.0, limiter=H.LIMITER_BJ,
                                        K=0.0, mode=H.LOCAL_CFL, cfl=0.8),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_full_size_first_steps_match_oracle(name):
    c = CASES[name]
    m = H.Mesh.wedge(c["nx"], c["ny"], theta_deg=c["theta"], jitter=0.15, seed=1234, numbering=H.NUMBER_RCM)
    bcmap, qbc, q = H.wedge_case(c["mach"])
    o = O.Oracle(m.arrays())
    o.gather_bcs(bcmap, qbc)
    o.initialise(q)
    o.set_limiter(O.VENKAT if c["limiter"] == H.LIMITER_VENKAT else O.BJ, c["K"])
    ref = []
    for _ in range(2):
        dt_o, res_o = o.step(c["mode"], c["cfl"])
        ref.append((o.U(), dt_o, res_o))
    del o
    for kernel in (H.KERNEL_TILED, H.KERNEL_CELL):
        runs = []
        for _ in range(2 if kernel == H.KERNEL_TILED else 1):
            s = H.Solver(m, limiter=c["limiter"], venkat_K=c["K"], precision=H.FP64, kernel=kernel)
            s.gather_bcs(bcmap, qbc)
            s.initialise(q)
            got = []
            for U_o, dt_o, res_o in ref:
                st = s.step(1, c["mode"], c["cfl"])
                U = s.U()
                assert np.all(O.rel_linf(U, U_o) <= ONE_STEP), (kernel, O.rel_linf(U, U_o))
                assert abs(st["dt"] - dt_o) <= 1e-13 * dt_o
                assert abs(st["res_l2"] - res_o) <= 1e-10 * res_o
                got.append((U, st["dt"], st["res_l2"]))
            runs.append(got)
            del s
        if len(runs) == 2:
            for a, b in zip(*runs):
                assert np.array_equal(a[0], b[0]) and a[1] == b[1] and a[2] == b[2]
