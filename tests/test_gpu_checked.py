"""The checked build (lib/libhcfd_gpu_checked.so, HCFD_LIB=checked) against the default one.

The checked build range-checks on the device every index the step kernels take from their
tables (the tiled kernels' tile descriptors, halo ids, cell slots and face-entry metadata where
they read them; the per-cell kernels' face and neighbour ids in a check of the slot table
before any step) and reports a bad one as HCFD_EINVAL.  On valid meshes it must change
nothing: every workload of tests/checked_cases.py (tiled and per-cell solvers in FP64 and
FP32, both limiters, global and local CFL; FP32 and FP64 arenas of three wedges; two
allocation-free steps) gives bit-identical states and statistics with either library, and no
error.  The library is chosen when the package is imported, so each run is a child process.

On a corrupt slot table (handed to the allocation-free step, which takes the caller's device
tables as they are) the checked build finds the bad id before launching the step and returns
HCFD_EINVAL, and a clean step in the same context afterwards matches the default build's.
Only the checked library is given the corrupt table.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from cfd_optimisations_b200 import native as N

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = os.path.join(HERE, "checked_cases.py")


def _run(tmp_path, which, *extra):
    out = str(tmp_path / f"{which}{'_corrupt' if extra else ''}.npz")
    env = dict(os.environ, HCFD_LIB=which)
    r = subprocess.run([sys.executable, CASES, out, *extra], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    return np.load(out)


@pytest.fixture(scope="module")
def runs(tmp_path_factory):
    assert os.path.exists(N.LIB_CHECKED), "checked library not built"
    t = tmp_path_factory.mktemp("checked")
    return _run(t, "default"), _run(t, "checked"), _run(t, "checked", "--corrupt")


def test_checked_build_is_bit_identical_on_valid_meshes(runs):
    d, c, _ = runs
    assert str(d["lib"]) == "libhcfd_gpu.so" and str(c["lib"]) == "libhcfd_gpu_checked.so"
    keys = sorted(k for k in d.files if k != "lib")
    assert keys == sorted(k for k in c.files if k != "lib")
    assert len(keys) == 36                      # 20 solver, 12 arena, 4 allocation-free
    differ = {}
    for k in keys:
        assert np.all(np.isfinite(d[k])), k
        if not np.array_equal(d[k], c[k]):
            den = np.maximum(np.abs(d[k]), 1e-300)
            differ[k] = float(np.max(np.abs(c[k] - d[k]) / den))
    assert not differ, differ


def test_checked_build_reports_a_corrupt_slot_table(runs):
    d, _, x = runs
    assert list(x["codes"]) == [N.EINVAL, N.EINVAL, N.OK]
    for m in x["msgs"]:
        assert "out of range" in str(m)
    # the context stays usable: the clean step after the corrupt ones is the default build's step
    assert np.array_equal(x["clean_U"], d["noalloc_0_U"])
    assert np.array_equal(x["clean_stats"], d["noalloc_0_stats"])
