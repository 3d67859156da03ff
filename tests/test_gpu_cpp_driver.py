"""The C++ drop-in (include/hcfd_gpu.hpp): the reference's Test.cpp driver with Base:: swapped
for GPU:: (cfd_optimisations_b200/csrc/drivers/wedge_driver.cpp) reproduces the reference's
golden snapshots sols/Base_0.hsln and sols/Base_1.hsln."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "cfd_optimisations_b200", "lib", "hcfd_wedge_driver")


@pytest.mark.gpu
def test_cpp_driver_reproduces_base_snapshots(tmp_path, golden):
    prefix = str(tmp_path / "GPU")
    out = subprocess.run([DRIVER, os.path.join(golden, "wedge.hmsh"), prefix], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr
    for k, tol in ((0, 1e-15), (1, 1e-9)):
        names, mine = O.read_hsln(f"{prefix}_{k}.hsln")
        ref_names, ref = O.read_hsln(os.path.join(golden, f"Base_{k}.hsln"))
        assert names == ref_names
        assert np.all(O.rel_linf(mine, ref) <= tol), (k, O.rel_linf(mine, ref))
    assert not os.path.exists(f"{prefix}_2.hsln")


def test_cpp_driver_fails_loudly_without_a_gpu(tmp_path, golden):
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("a GPU is present")
    out = subprocess.run([DRIVER, os.path.join(golden, "wedge.hmsh"), str(tmp_path / "x")], capture_output=True,
                         text=True, timeout=60)
    assert out.returncode == 1 and "no CUDA device" in out.stderr
