"""Build of the native library libhcfd_gpu.so (in-tree, sm_100a only).

    python -m cfd_optimisations_b200._build

compiles csrc/*.cu and csrc/*.cpp with nvcc for sm_100a into
cfd_optimisations_b200/lib/libhcfd_gpu.so, and the C++ drop-in driver
(csrc/drivers/wedge_driver.cpp, the GPU:: counterpart of the reference's src/Test.cpp)
into cfd_optimisations_b200/lib/hcfd_wedge_driver.  Objects are rebuilt when a source or
header is newer than the library.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libhcfd_gpu.so")
LIB_CHECKED = os.path.join(LIBDIR, "libhcfd_gpu_checked.so")
DRIVER = os.path.join(LIBDIR, "hcfd_wedge_driver")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
           "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _deps():
    return _sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) + \
        glob.glob(os.path.join(INCLUDE, "*.h")) + glob.glob(os.path.join(INCLUDE, "*.hpp")) + [__file__]


def _stale(target, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _build_lib(lib, objdir, defines, verbose, force, ptxas_info) -> None:
    os.makedirs(objdir, exist_ok=True)
    nv = nvcc()
    objs = []
    for src in _sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + _deps()):
            cmd = [nv] + ARCH + NVFLAGS + defines + ["-c", src, "-o", obj]
            if ptxas_info and src.endswith(".cu"):
                cmd += ["-Xptxas", "-v"]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _stale(lib, objs):
        cmd = [nv] + ARCH + ["-shared", "-o", lib] + objs + ["-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False, checked: bool = True) -> str:
    """Builds the library, its checked twin (every tile index verified on the device before
    use; selected at run time with HCFD_LIB=checked) and the C++ driver."""
    os.makedirs(LIBDIR, exist_ok=True)
    _build_lib(LIB, os.path.join(PKG, "_build"), [], verbose, force, ptxas_info)
    if checked:
        _build_lib(LIB_CHECKED, os.path.join(PKG, "_build", "checked"), ["-DHCFD_CHECKED"], verbose, force, False)
    drv_src = os.path.join(CSRC, "drivers", "wedge_driver.cpp")
    if os.path.exists(drv_src) and (force or _stale(DRIVER, [drv_src, LIB] + _deps())):
        cmd = ["g++", "-O2", "-std=c++17", "-pthread", "-I", INCLUDE, drv_src, "-o", DRIVER,
               "-L", LIBDIR, "-lhcfd_gpu", "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, ptxas_info="--ptxas" in sys.argv)
