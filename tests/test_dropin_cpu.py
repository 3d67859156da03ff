"""The C++ drop-in on the CPU: GPU::Domain built from the reference's own Mesh object (its
reader, compiled unchanged into the reference build) sees exactly what GPU::Mesh reads, and
without a GPU, GPU::Euler throws instead of running anything on the CPU."""
import os
import subprocess

import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "cfd_optimisations_b200", "lib")


@pytest.mark.skipif(not (O.RefSolver.available() and os.path.exists(os.path.join(O.REF_DIR, "includes", "Mesh.hpp"))),
                    reason="reference sources or build not present")
def test_domain_from_the_reference_mesh(tmp_path, golden):
    exe = str(tmp_path / "ref_mesh_domain")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(O.REF_DIR, "includes"), "-I",
                    os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "ref_mesh_domain.cpp"), "-o", exe,
                    O.REF_SO, "-L", LIB, "-lhcfd_gpu", "-Wl,-rpath," + LIB + ":" + os.path.dirname(O.REF_SO),
                    "-pthread"], check=True, capture_output=True, text=True, timeout=300)
    out = subprocess.run([exe, os.path.join(golden, "wedge.hmsh")], capture_output=True, text=True, timeout=120)
    assert "SAME Nc=3740 Nf=7120" in out.stdout, out.stdout + out.stderr
    if out.returncode == 0:                       # no GPU: the solver refused loudly
        assert "THREW hcfd:" in out.stdout and "CUDA" in out.stdout.upper()
    else:                                         # a GPU: the solver was created
        assert out.returncode == 3 and "NO-THROW" in out.stdout, out.stdout + out.stderr
