"""The C ABI library (CPU only): it loads without a GPU, exports every function declared in
include/*.h, and its host-only entry points work.  No compute call is made here."""
import ctypes as ct
import os
import re
import subprocess
import sys

import pytest

import cfd_optimisations_b200 as H
from cfd_optimisations_b200 import native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if not fn.endswith(".h"):
            continue
        with open(os.path.join(ROOT, "include", fn)) as fh:
            src = re.sub(r"/\*.*?\*/", "", fh.read(), flags=re.S)
        names |= set(re.findall(r"\b(hcfd_[a-z0-9_]+)\s*\(", src))
    return names


@pytest.mark.parametrize("path", [N.LIB_DEFAULT, N.LIB_CHECKED], ids=["default", "checked"])
def test_every_declared_symbol_is_exported(path):
    names = declared()
    assert len(names) >= 30
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (hcfd_[a-z0-9_]+)\b", out))
    assert names <= exported, sorted(names - exported)


def test_python_binding_covers_the_abi():
    assert declared() <= set(N._SIGS), sorted(declared() - set(N._SIGS))


def test_library_loads_and_reports_errors():
    L = N.lib()
    # host-only paths: a bad mesh argument fails cleanly with a message
    rc = L.hcfd_mesh_load(b"/nonexistent/file.hmsh", ct.byref(ct.c_void_p()))
    assert rc == N.EIO
    assert b"cannot open" in L.hcfd_last_error()
    assert L.hcfd_gpu_create(None, None, ct.byref(ct.c_void_p())) == N.EINVAL


def test_no_gpu_here_means_a_cuda_error_not_a_fallback():
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("a GPU is present")
    m = H.Mesh.wedge(11, 6, seed=1)
    with pytest.raises(H.HcfdError) as e:
        H.Solver(m)
    assert e.value.code == N.ECUDA


def _lib_choice(value):
    env = dict(os.environ, HCFD_LIB=value)
    code = ("from cfd_optimisations_b200 import native as N; L = N.lib(); "
            "print(N.LIB_PATH); print(L.hcfd_last_error())")
    return subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, cwd=ROOT)


def test_hcfd_lib_selects_the_checked_twin_and_rejects_other_values():
    r = _lib_choice("checked")
    assert r.returncode == 0, r.stderr
    assert r.stdout.splitlines()[0].endswith("libhcfd_gpu_checked.so")
    r = _lib_choice("default")
    assert r.returncode == 0, r.stderr
    assert r.stdout.splitlines()[0].endswith("libhcfd_gpu.so")
    r = _lib_choice("fast")
    assert r.returncode != 0 and "HCFD_LIB" in r.stderr
