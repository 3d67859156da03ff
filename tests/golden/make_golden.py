"""Regenerates the committed fixtures of this directory (run where the reference's sources and
oracle/_ref, the reference built from them, are present):

    python tests/golden/make_golden.py <reference source tree>

* wedge.hmsh, Base_0.hsln, Base_1.hsln — the reference's own mesh and its shipped golden
  solutions (sols/Base_{0,1}.hsln: the initial state and the state after exactly 1000
  steps of dt = 1e-3 on wedge.hmsh, M = 2, BC map of src/Test.cpp:64), copied unchanged.
* ref_small_wedge.npz — the reference solver (compiled unchanged, oracle/_ref) on a
  41 x 21-node generated wedge (seed 7, random numbering, M = 2.5, 15 deg): the
  conservative state after 1 and after 50 fixed-dt steps, and after 20 steps whose dt is
  the global CFL-0.5 dt of the reference's own state (the CFL rule is the oracle's; the
  reference has none).  The mesh itself is stored too, so the fixture stands alone.
"""
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def main(REF: str):
    import oracle as O
    import cfd_optimisations_b200 as H

    shutil.copyfile(os.path.join(REF, "wedge.hmsh"), os.path.join(HERE, "wedge.hmsh"))
    for k in (0, 1):
        shutil.copyfile(os.path.join(REF, "sols", f"Base_{k}.hsln"), os.path.join(HERE, f"Base_{k}.hsln"))

    path = os.path.join(HERE, "small_wedge.hmsh")
    m = H.Mesh.wedge(41, 21, theta_deg=15.0, jitter=0.15, seed=7, numbering=H.NUMBER_RANDOM)
    m.write(path)
    bcmap, qbc, q = H.wedge_case(2.5)
    r = O.RefSolver(path, bcmap, qbc, q)
    U0 = r.U()
    r.steps(1, 2e-3)
    U1 = r.U()
    r.steps(49, 2e-3)
    U50 = r.U()
    r2 = O.RefSolver(path, bcmap, qbc, q)
    orc = O.Oracle(O.read_hmsh(path))
    dts = []
    for _ in range(20):
        orc.set_U(r2.U())
        dt = 0.5 * orc.get(O.F_DTLOC)[orc.get(O.F_IV) != 0].min()
        dts.append(dt)
        r2.steps(1, dt)
    np.savez_compressed(os.path.join(HERE, "ref_small_wedge.npz"), U0=U0, U1=U1, U50=U50, dt_fixed=2e-3,
                        U_cfl20=r2.U(), dts_cfl=np.array(dts))
    os.remove(path)
    m.write(os.path.join(HERE, "small_wedge.hmsh"))
    print("fixtures written to", HERE)


if __name__ == "__main__":
    if len(sys.argv) != 2 or not os.path.exists(os.path.join(sys.argv[1], "sols")):
        sys.exit("usage: make_golden.py <reference source tree>")
    main(sys.argv[1])
